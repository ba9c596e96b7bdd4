"""ADCIG stitching (layercom_cig): the oracle against the reference tool's own
outputs, and the drop-in's checks that run before any device work."""
import ctypes
import json
import os
import subprocess

import numpy as np
import pytest

import stitch as so  # oracle/stitch.py

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLD = np.load(os.path.join(HERE, "golden", "golden_stitch.npz"))
META = json.load(open(os.path.join(HERE, "golden", "cases.json")))["stitch"]
CLI = os.path.join(ROOT, "kirch_datuming_b200", "bin", "layercom_cig")


def case_args(args):
    kv = {}
    for a in args:
        k, v = a.split("=", 1)
        kv[k] = v
    scales = None
    if "scale" in kv:
        vals = [float(np.float32(x)) for x in kv["scale"].replace(";", ",").split(",") if x]
        scales = vals * len(META["windows"]) if len(vals) == 1 else vals
    return dict(scales=scales, stitch_blend=int(kv.get("stitch_blend", 15)),
                scalex_aper=int(kv.get("scalex_aper", 0)), scalex_scale=float(kv.get("scalex_scale", 1.0)))


def windows():
    return [GOLD["window_%d" % (k + 1)] for k in range(len(META["windows"]))]


@pytest.mark.parametrize("name", sorted(META["cases"]))
def test_oracle_matches_reference_bit_for_bit(name):
    got = so.stitch(META["model"]["n"][0], [tuple(w) for w in META["windows"]], windows(),
                    **case_args(META["cases"][name]["args"]))
    ref = GOLD["out_" + name]
    assert got.shape == ref.shape
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_oracle_nonfinite_window():
    vols = windows()
    vols[1] = vols[1].copy()
    vols[1][3, 5, 2] = np.inf
    with pytest.raises(ValueError, match="window 2"):
        so.stitch(60, [tuple(w) for w in META["windows"]], vols)


def test_blend_and_lateral_tables():
    w = so.blend_weights(5)
    assert w[0] == 0.0 and w[-1] == 1.0 and np.all(np.diff(w) > 0)
    assert np.allclose(w + w[::-1], 1.0, atol=1e-7)          # complementary
    assert so.blend_weights(1)[0] == 1.0
    lat = so.lateral_scale(10, 3, 2.0)
    assert list(lat[:3]) == [2.0, 1.5, 1.0] and lat[3] == 1.0 and list(lat[-3:]) == [1.0, 1.5, 2.0]


def test_library_exports_stitching():
    lib = ctypes.CDLL(os.path.join(ROOT, "kirch_datuming_b200", "libkcig.so"))
    for sym in ("kcig_stitch_window", "kcig_run_layercom_cig_cli"):
        assert hasattr(lib, sym)


def _inputs(wd):
    from kirch_datuming_b200 import rsf
    m, a = META["model"], META["angles"]
    rsf.write(f"{wd}/model.rsf", np.zeros(m["n"][::-1], np.float32), m["n"], m["o"], m["d"])
    with open(f"{wd}/layers.txt", "w", encoding="utf-8") as f:
        f.write(META["layers"])
    for k, (s0, s1) in enumerate(META["windows"]):
        rsf.write(f"{wd}/adcig_{k + 1}.rsf", GOLD["window_%d" % (k + 1)], [s1 - s0 + 1, m["n"][1], a["n"]],
                  [m["o"][0] + s0 * m["d"][0], m["o"][1], a["o"]], [m["d"][0], m["d"][1], a["d"]],
                  extra=META["labels"])


COMMON = ["full_model=model.rsf", "layer_image_base=adcig.rsf", "layer_txt=layers.txt", "output_file=out.rsf"]


@pytest.mark.parametrize("name", ["nlayers", "scale_count", "blend", "bad_argument", "missing_key"])
def test_cli_errors_before_device_work(tmp_path, name):
    # these checks run before any device call, so they need no GPU
    e = META["errors"][name]
    _inputs(str(tmp_path))
    r = subprocess.run([CLI] + COMMON + e["args"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == e["returncode"]
    assert r.stderr == e["stderr"]
    assert not (tmp_path / "out.rsf").exists()
