"""The GPU table generator (kcig_eikods) against the CPU oracle's sweep
solver -- bit for bit: the same local update, the same sweep sequence, the
same rounding -- and, through the oracle, against the reference eikods2d's
committed outputs (identical for order 1 and for the v(z) migration tables;
the order-2 tolerance is the oracle's, tests/test_eikods_oracle.py).  The
drop-in eikods2d executable is checked file for file."""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

import kirch_datuming_b200 as kd
from kirch_datuming_b200 import rsf, synth

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu
GOLD = os.path.join(HERE, "golden")
FIELDS = ("time", "tdl1", "tds1", "gradz", "gradx")


def _gpu(vel, d, shots, **kw):
    import torch
    r = kd.eikods(torch.from_numpy(np.ascontiguousarray(vel)).cuda(), d, d, shots, grads=True, **kw)
    return {k: (v.cpu().numpy() if torch.is_tensor(v) else v) for k, v in r.items()}


def _salt():
    g = np.load(os.path.join(GOLD, "golden_eikods.npz"))
    with open(os.path.join(GOLD, "cases.json")) as f:
        return g, json.load(f)["eikods"]


@pytest.mark.parametrize("run", ["o2", "o1", "o2_l0"])
def test_gpu_equals_sweep_oracle_salt(run):
    g, meta = _salt()
    kw = dict(order=1 if run == "o1" else 2, l=0 if run.endswith("l0") else 1, b1=meta["b1"], b2=meta["b2"])
    got = _gpu(g["vel"], meta["d"], g["shots"], **kw)
    ref = O.eikods(g["vel"], meta["d"], meta["d"], g["shots"], method=1, grads=True, **kw)
    np.testing.assert_array_equal(got["sweeps"], ref["sweeps"])
    for k in FIELDS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
        key = "%s_%s" % (run, k)
        if run == "o1" and key in g.files:  # and the reference itself
            np.testing.assert_array_equal(got[k], g[key], err_msg=key)


def test_gpu_vz_equals_reference():
    gz = np.load(os.path.join(GOLD, "golden.npz"))
    with open(os.path.join(GOLD, "cases.json")) as f:
        meta = json.load(f)
    t = meta["table"]
    shots = np.zeros((t["n"][2], 3), np.float32)
    shots[:, 1] = np.float32(t["o"][2]) + np.arange(t["n"][2], dtype=np.float32) * np.float32(0.02)
    v = synth.velocity_linear_vz(meta["nz"], meta["nx"], meta["dz"])
    got = _gpu(v, meta["dz"], shots)
    for k, gk in (("time", "T"), ("tds1", "tds"), ("gradx", "gradx"), ("gradz", "gradz")):
        np.testing.assert_array_equal(got[k].ravel(), gz[gk], err_msg=k)


def test_gpu_tall_grid_several_rows_per_thread():
    # nz > 512: threads own two rows; shots buried, off-node and at the edges
    nz, nx, d = 700, 90, 0.01
    v, _ = synth.five_layer_salt(nz, nx, d, d, seed=3)
    shots = np.array([[0.0, 0.0, 0.0], [1.234, 0.4567, 0.0], [6.9, 0.89, 0.0]], np.float32)
    got = _gpu(v, d, shots)
    ref = O.eikods(v, d, d, shots, method=1, grads=True)
    np.testing.assert_array_equal(got["sweeps"], ref["sweeps"])
    for k in FIELDS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)


def test_gpu_slowness_input_and_origins():
    # vel=0 (slowness squared in), non-zero origins and another box
    g, meta = _salt()
    s2 = (1.0 / (g["vel"].astype(np.float32) ** 2)).astype(np.float32)
    kw = dict(o1=0.05, o2=-0.1, o3=0.02, b1=1, b2=3)
    shots = g["shots"] + np.array([0.05, -0.1, 0.0], np.float32)
    got = _gpu(s2, meta["d"], shots, vel_is_slowness2=True, **kw)
    ref = O.eikods(s2, meta["d"], meta["d"], shots, method=1, grads=True, vel_is_s2=True, **kw)
    for k in FIELDS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)


def test_gpu_reports_missing_fixed_point():
    g, meta = _salt()
    with pytest.raises(kd.KcigError):
        _gpu(g["vel"], meta["d"], g["shots"], max_iter=1)


def test_eikonal_tables_is_eikods():
    import torch
    nz, nx, d = 61, 121, 0.01
    v, _ = synth.five_layer_salt(nz, nx, d, d)
    vt = torch.from_numpy(v).cuda()
    T, D = kd.eikonal_tables(vt, d, d, 7, 0.1, 0.15, zsrc=0.02)
    shots = np.zeros((7, 3), np.float32)
    shots[:, 0] = 0.02
    shots[:, 1] = np.float32(0.1) + np.arange(7, dtype=np.float32) * np.float32(0.15)
    r = kd.eikods(vt, d, d, shots)
    assert torch.equal(T, r["time"]) and torch.equal(D, r["tds1"])


def test_drop_in_cli_order1_equals_reference_files():
    # the executable with the reference's own argv, file for file (order 1:
    # identical values; headers as eikods2d writes them)
    g, meta = _salt()
    with tempfile.TemporaryDirectory() as wd:
        rsf.write(f"{wd}/vel.rsf", g["vel"], [meta["nz"], meta["nx"]], [0, 0], [meta["d"], meta["d"]])
        rsf.write(f"{wd}/sht.rsf", g["shots"], [3, g["shots"].shape[0]], [0, 0], [1, 1])
        r = subprocess.run([kd.eikods_cli_path, "in=vel.rsf", "out=time.rsf", "shotfile=sht.rsf", "tdl1=tdl.rsf",
                            "tds1=tds.rsf", "gradz=gz.rsf", "gradx=gx.rsf", "b1=2", "b2=2", "order=1"], cwd=wd,
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        for f, k in (("time", "time"), ("tdl", "tdl1"), ("tds", "tds1"), ("gz", "gradz"), ("gx", "gradx")):
            h, a = rsf.read(f"{wd}/{f}.rsf")
            assert list(h.n[:3]) == meta["header"]["n"]
            np.testing.assert_allclose(h.o[:3], meta["header"]["o"], rtol=0, atol=1e-9)
            np.testing.assert_allclose(h.d[:3], meta["header"]["d"], rtol=0, atol=1e-9)
            np.testing.assert_array_equal(a.reshape(g["o1_" + k].shape), g["o1_" + k], err_msg=k)
        # a required output missing: the reference's message and a failing status
        r = subprocess.run([kd.eikods_cli_path, "in=vel.rsf", "out=t2.rsf", "shotfile=sht.rsf", "tds1=x.rsf"],
                           cwd=wd, capture_output=True, text=True)
        assert r.returncode != 0 and "Output derivative tdl1= missing." in r.stderr


def test_gpu_more_than_1024_rows():
    # nz > 1024: four rows per thread
    nz, nx, d = 1100, 40, 0.01
    v, _ = synth.five_layer_salt(nz, nx, d, d, seed=5)
    shots = np.array([[0.0, 0.2, 0.0], [5.55, 0.131, 0.0]], np.float32)
    got = _gpu(v, d, shots)
    ref = O.eikods(v, d, d, shots, method=1, grads=True)
    np.testing.assert_array_equal(got["sweeps"], ref["sweeps"])
    for k in FIELDS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
