"""layercom_cig against the reference tool (oracle/_ref/layercom_cig, built
from its source), on the CPU: the drop-in on malformed inputs (exit code, INFO
lines and ERROR text must be the same; every case fails before any device
work), and the oracle on random window layouts, blends, tapers and scales (the
volume must be the same bit for bit)."""
import os
import subprocess

import numpy as np
import pytest

from test_stitch_oracle import CLI, COMMON, META, _inputs

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "layercom_cig")

pytestmark = pytest.mark.skipif(not os.path.exists(REF), reason="reference tool not built (make -C oracle ref)")


def _layers(text):
    def setup(wd):
        with open(os.path.join(wd, "layers.txt"), "w", encoding="utf-8") as f:
            f.write(text)
    return setup


def _model_header(text):
    def setup(wd):
        with open(os.path.join(wd, "model.rsf"), "w") as f:
            f.write(text)
    return setup


def _first_window_n2(wd):
    from kirch_datuming_b200 import rsf
    m, a = META["model"], META["angles"]
    rsf.write(os.path.join(wd, "adcig_1.rsf"), np.zeros((a["n"], 20, 26), np.float32), [26, 20, a["n"]],
              [0.0, m["o"][1], a["o"]], [m["d"][0], m["d"][1], a["d"]])


CASES = {
    "first_not_zero": (_layers("5,25\n18,45\n40,END\n"), []),
    "no_overlap": (_layers("START,25\n30,45\n40,END\n"), []),
    "not_deeper": (_layers("START,25\n18,20\n40,END\n"), []),
    "last_not_end": (_layers("START,25\n18,45\n"), []),
    "needs_two": (_layers("START\n"), []),
    "bad_start": (_layers("abc,25\n"), []),
    "bad_end": (_layers("START,xyz\n"), []),
    "bad_datum": (_layers("START,25,q\n18,45\n40,END\n"), []),
    "empty_layers": (_layers("# nothing\n\n"), []),
    "range": (_layers("START,70\n"), []),
    "no_layer_file": (None, ["layer_txt=nope.txt"]),
    "no_model": (None, ["full_model=none.rsf"]),
    "model_no_n1": (_model_header('in="model.rsf@"\nn2=24\n'), []),
    "model_format": (_model_header('in="model.rsf@"\nn1=60\nn2=24\ndata_format="xdr_float"\n'), []),
    "model_bad_int": (_model_header('in="model.rsf@"\nn1=6o\nn2=24\n'), []),
    "model_no_in": (_model_header("n1=60\nn2=24\n"), []),
    "lateral_size": (_first_window_n2, []),
    "int_arg": (None, ["nlayers=3x"]),
    "real_arg": (None, ["scalex_scale=nan"]),
    "scale_value": (None, ["scale=1,abc,2"]),
    "nangle": (None, ["nangle=5"]),
    "aper": (None, ["scalex_aper=-1"]),
    "positional": (None, ["=3"]),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_same_failure_as_reference(tmp_path, name):
    setup, extra = CASES[name]
    results = []
    for tag, exe in (("ref", REF), ("kcig", CLI)):
        wd = tmp_path / tag
        wd.mkdir()
        _inputs(str(wd))
        if setup:
            setup(str(wd))
        r = subprocess.run([exe] + COMMON + extra, cwd=wd, capture_output=True, text=True)
        results.append((r.returncode, r.stdout, r.stderr, (wd / "out.rsf").exists()))
    ref, got = results
    assert ref[0] != 0 and ref[2].startswith("ERROR: ")
    assert got == ref


def _random_setup(rng):
    n1 = int(rng.integers(30, 90))
    nwin = int(rng.integers(2, 5))
    # window ends increase; each window starts inside the one above
    ends = sorted(rng.choice(np.arange(8, n1 - 1), size=nwin - 1, replace=False).tolist()) + [n1 - 1]
    wins, prev_end = [], None
    for k, e in enumerate(ends):
        s = 0 if k == 0 else int(rng.integers(max(1, prev_end - 25), prev_end + 1))
        wins.append((s, int(e)))
        prev_end = int(e)
    args = []
    blend = int(rng.choice([-1, 0, 1, 2, 5, 15, 40]))
    if blend != 15:
        args.append("stitch_blend=%d" % blend)
    aper = int(rng.integers(0, 7))
    sxs = float(np.round(rng.uniform(0.2, 3.0), 3))
    if aper:
        args += ["scalex_aper=%d" % aper, "scalex_scale=%g" % sxs]
    scales = None
    if rng.random() < 0.7:
        scales = [float(np.float32(np.round(rng.uniform(0.1, 3.0), 4))) for _ in wins]
        args.append("scale=" + ",".join("%g" % x for x in scales))
    return n1, wins, blend, aper, sxs if aper else 1.0, scales, args


@pytest.mark.parametrize("seed", range(12))
def test_oracle_vs_reference_random_layouts(tmp_path, seed):
    # random window layouts, blends, tapers and scales through the reference
    # tool: the oracle must give its volume bit for bit
    import stitch as so
    from kirch_datuming_b200 import rsf
    rng = np.random.default_rng(1000 + seed)
    n1, wins, blend, aper, sxs, scales, args = _random_setup(rng)
    n2, n3 = int(rng.integers(3, 20)), int(rng.integers(1, 6))
    rsf.write(str(tmp_path / "model.rsf"), np.zeros((n2, n1), np.float32), [n1, n2], [0.0, 0.0], [0.01, 0.02])
    with open(tmp_path / "layers.txt", "w") as f:
        f.write("".join("%d %d\n" % w for w in wins))
    vols = []
    for k, (s, e) in enumerate(wins):
        v = (rng.standard_normal((n3, n2, e - s + 1)) * 10 ** rng.uniform(-3, 3)).astype(np.float32)
        vols.append(v)
        rsf.write(str(tmp_path / ("adcig_%d.rsf" % (k + 1))), v, [e - s + 1, n2, n3], [s * 0.01, 0.0, 0.0],
                  [0.01, 0.02, 1.0])
    r = subprocess.run([REF] + COMMON + args, cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    ref = np.fromfile(tmp_path / "out.rsf@", dtype="<f4").reshape(n3, n2, n1)
    got = so.stitch(n1, wins, vols, scales, blend, aper, sxs)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
