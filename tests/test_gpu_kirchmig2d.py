"""The plain tool kirchmig2d on the GPU (kcig_params.tool = 1 through the same
plan and kernels): against the FP64 oracle (1e-5, as the angle tool), against
the reference's own images (no worse than the FP64 oracle is), and the drop-in
executable file for file."""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

import kirch_datuming_b200 as kd
from kirch_datuming_b200 import rsf

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
sys.path.insert(0, HERE)
import _cases  # noqa: E402
import oracle  # noqa: E402

pytestmark = pytest.mark.gpu
GD = _cases.Golden()


def _inputs(name):
    kp, geom, axis, op = _cases.k2d_setup(GD, name)
    T, D = GD.tables()
    data = GD.npz["data_" + GD.meta["k2d"][name]["data"]]
    return kp, geom, axis, op, T, D, data


@pytest.mark.parametrize("name", GD.k2d_cases)
def test_gpu_kirchmig2d(name):
    kp, geom, axis, op, T, D, data = _inputs(name)
    plan = kd.Plan(kp, kd.geometry(**geom))
    plan.set_tables(T, D, T, D)
    img = np.zeros((axis[0], geom["nx"], geom["nz"]), np.float32)
    plan.migrate(np.ascontiguousarray(data, dtype=np.float32), img)
    stats = plan.stats()
    plan.close()
    assert stats["sum_launches"] >= 1
    o64 = oracle.migrate_kirchmig2d(op, data, T, D, T, D, fp64=True)
    assert oracle.rel_l2(img, o64) <= 1e-5
    ref = GD.k2d_image(name)
    u = _cases.ub_columns(GD, name)
    ref_err = oracle.rel_l2(ref[:, u:], o64[:, u:])
    assert oracle.rel_l2(img[:, u:], ref[:, u:]) <= 1.5 * ref_err + 1e-6


def test_drop_in_kirchmig2d_cli():
    name = "k2d_cig_cmp0"
    c = GD.meta["k2d"][name]
    d = GD.meta["data"][c["data"]]
    t = GD.meta["table"]
    with tempfile.TemporaryDirectory() as wd:
        T, D = GD.tables()
        rsf.write(f"{wd}/time.rsf", T, t["n"], t["o"], t["d"])
        rsf.write(f"{wd}/tds.rsf", D, t["n"], t["o"], t["d"])
        rsf.write(f"{wd}/data.rsf", GD.npz["data_" + c["data"]], [GD.meta["nt"], d["nh"], d["ns"]],
                  [0, d["h0"], d["s0"]], [GD.meta["dt"], d["dh"], d["ds"]], extra={"unit1": "s"})
        r = subprocess.run([kd.kirchmig2d_cli_path, "seismic_data=data.rsf", "migration=img.rsf", "stable=time.rsf",
                            "sderiv=tds.rsf", "rtable=time.rsf", "rderiv=tds.rsf"] + c["tokens"], cwd=wd,
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        h, img = rsf.read(f"{wd}/img.rsf")
        assert list(h.n[:3]) == c["n"]
        np.testing.assert_allclose(h.o[:3], c["o"], rtol=0, atol=1e-9)
        np.testing.assert_allclose(h.d[:3], c["d"], rtol=0, atol=1e-9)
        for k, v in c["extra"].items():
            assert h.extra.get(k, "").strip('"') == v.strip('"'), k
        ref = GD.k2d_image(name)
        assert oracle.rel_l2(img.reshape(ref.shape), ref) < 1e-4
        r = subprocess.run([kd.kirchmig2d_cli_path, "seismic_data=data.rsf", "migration=x.rsf", "stable=time.rsf",
                            "sderiv=tds.rsf", "rtable=time.rsf", "rderiv=tds.rsf", "adj=0", "nt=10", "dt=0.002",
                            "dh=0.02", "ds=0.1"], cwd=wd, capture_output=True, text=True)
        assert r.returncode != 0 and "not built" in r.stderr
        r = subprocess.run([kd.kirchmig2d_cli_path, "migration=x.rsf"], cwd=wd, capture_output=True, text=True)
        assert r.returncode != 0 and "Need seismic_data=" in r.stderr
