"""ADCIG stitching on the device: the drop-in layercom_cig against the
reference tool's own outputs (bit for bit: samples, header, INFO lines,
errors), and kcig_stitch_window against the oracle on ragged windows and at
the full 601 x 1601 x 61 image size."""
import subprocess

import numpy as np
import pytest

import kirch_datuming_b200 as kd
import stitch as so  # oracle/stitch.py
from test_stitch_oracle import COMMON, GOLD, META, _inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(META["cases"]))
def test_cli_matches_reference(tmp_path, name):
    c = META["cases"][name]
    _inputs(str(tmp_path))
    r = subprocess.run([kd.layercom_cig_cli_path] + COMMON + c["args"], cwd=tmp_path, capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    assert r.stdout == c["stdout"]
    assert (tmp_path / "out.rsf").read_text() == c["header"]
    got = np.fromfile(tmp_path / "out.rsf@", dtype="<f4")
    assert np.array_equal(got.view(np.uint32), GOLD["out_" + name].reshape(-1).view(np.uint32))


def test_cli_nonfinite_window(tmp_path):
    from kirch_datuming_b200 import rsf
    e = META["errors"]["nonfinite"]
    _inputs(str(tmp_path))
    m, a = META["model"], META["angles"]
    for k, (s0, s1) in enumerate(META["windows"]):
        v = GOLD["window_%d" % (k + 1)].copy()
        if k == 1:
            v[3, 5, 2] = np.inf
        rsf.write(str(tmp_path / ("bad_%d.rsf" % (k + 1))), v, [s1 - s0 + 1, m["n"][1], a["n"]],
                  [m["o"][0] + s0 * m["d"][0], m["o"][1], a["o"]], [m["d"][0], m["d"][1], a["d"]],
                  extra=META["labels"])
    r = subprocess.run([kd.layercom_cig_cli_path] + COMMON + e["args"], cwd=tmp_path, capture_output=True,
                       text=True)
    assert r.returncode == e["returncode"] and r.stderr == e["stderr"]
    assert not (tmp_path / "out.rsf").exists()


def _stitch_device(n1, wins, vols, scales, blend, aper, sxs):
    import torch
    out = torch.zeros((vols[0].shape[0], vols[0].shape[1], n1), dtype=torch.float32, device="cuda")
    prev = -1
    for k, ((s, e), v) in enumerate(zip(wins, vols)):
        bad = kd.stitch_window(out, torch.from_numpy(v).cuda(), s, e, prev, blend, scales[k], k > 0, aper, sxs)
        assert bad == 0
        prev = e
    return out.cpu().numpy()


@pytest.mark.parametrize("blend,aper,sxs", [(15, 0, 1.0), (3, 4, 1.7), (0, 0, 1.0), (-1, 2, 0.6), (1, 1, 3.0),
                                            (40, 7, 0.25)])
def test_stitch_window_vs_oracle(blend, aper, sxs):
    rng = np.random.default_rng(blend + 100 * aper)
    n1, n2, n3 = 131, 33, 5
    wins = [(0, 50), (37, 90), (85, 130)]
    vols = [rng.standard_normal((n3, n2, e - s + 1)).astype(np.float32) for s, e in wins]
    scales = [1.0, 0.75, 1.25]
    ref = so.stitch(n1, wins, vols, scales, blend, aper, sxs)
    got = _stitch_device(n1, wins, vols, scales, blend, aper, sxs)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_stitch_window_full_image_size():
    # five depth windows of the 601 x 1601 image with 61 angle bins (235 MB)
    rng = np.random.default_rng(7)
    n1, n2, n3 = 601, 1601, 61
    wins = [(0, 130), (110, 250), (230, 370), (350, 490), (470, 600)]
    vols = [rng.standard_normal((n3, n2, e - s + 1), dtype=np.float32) for s, e in wins]
    scales = [1.0, 1.1, 0.9, 1.2, 0.8]
    ref = so.stitch(n1, wins, vols, scales, 15, 50, 1.5)
    got = _stitch_device(n1, wins, vols, scales, 15, 50, 1.5)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_stitch_window_counts_nonfinite():
    import torch
    out = torch.zeros((2, 3, 10), dtype=torch.float32, device="cuda")
    v = np.ones((2, 3, 10), np.float32)
    v[0, 1, 4] = np.inf
    v[1, 2, 9] = np.nan
    bad = kd.stitch_window(out, torch.from_numpy(v).cuda(), 0, 9)
    assert bad == 2
    o = out.cpu().numpy()
    assert o[0, 1, 4] == 0.0 and o[1, 2, 9] == 0.0 and np.count_nonzero(o) == 58
    # a finite value whose scaled product overflows counts as well
    out2 = torch.zeros_like(out)
    big = np.full((2, 3, 10), 3e38, np.float32)
    assert kd.stitch_window(out2, torch.from_numpy(big).cuda(), 0, 9, layer_scale=10.0) == 60


@pytest.mark.parametrize("blend,aper,sxs", [(15, 0, 1.0), (3, 4, 1.7), (0, 0, 1.0), (-1, 2, 0.6), (40, 7, 0.25)])
def test_stitch_windows_one_pass_equals_the_window_calls(blend, aper, sxs):
    # the one-pass kernel over all windows against the oracle (bit for bit),
    # with a window whose overlap reaches two windows back and a row range
    # no window covers (written as zeros)
    import torch
    rng = np.random.default_rng(blend + 7 * aper)
    n1, n2, n3 = 140, 29, 4
    wins = [(0, 50), (37, 90), (45, 120), (100, 131)]
    vols = [rng.standard_normal((n3, n2, e - s + 1)).astype(np.float32) for s, e in wins]
    scales = [1.0, 0.75, 1.25, 0.5]
    vols[1][1, 3, 5] = 0.0  # the oracle refuses non-finite windows: 0 there, NaN on the device
    ref = so.stitch(n1, wins, vols, scales, blend, aper, sxs)
    vols[1][1, 3, 5] = np.nan  # counted, and written as 0
    out = torch.full((n3, n2, n1), 7.0, dtype=torch.float32, device="cuda")  # overwritten everywhere
    bad = kd.stitch_windows(out, [torch.from_numpy(v).cuda() for v in vols], wins, blend, scales, True, aper, sxs)
    got = out.cpu().numpy()
    assert bad == [0, 1, 0, 0]
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    assert not got[:, :, 132:].any()


def test_stitch_windows_full_image_size():
    import torch
    rng = np.random.default_rng(8)
    n1, n2, n3 = 601, 1601, 61
    wins = [(0, 130), (110, 250), (230, 370), (350, 490), (470, 600)]
    vols = [rng.standard_normal((n3, n2, e - s + 1), dtype=np.float32) for s, e in wins]
    scales = [1.0, 1.1, 0.9, 1.2, 0.8]
    ref = so.stitch(n1, wins, vols, scales, 15, 50, 1.5)
    out = torch.empty((n3, n2, n1), dtype=torch.float32, device="cuda")
    kd.stitch_windows(out, [torch.from_numpy(v).cuda() for v in vols], wins, 15, scales, True, 50, 1.5)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), ref.view(np.uint32))
