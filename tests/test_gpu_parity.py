"""Parity of the CUDA path with the oracle and the reference, through the C ABI.

Tolerances (relative L2, ||a-b||/||b|| in double as src/rsf_l2cmp.cpp:9-10):
  * against the FP64 oracle: 1e-5 (the bound the table path is held to);
  * against the reference binary's FP32 image: 1.5x the distance between the
    reference and the FP64 oracle, plus 1e-6 (the reference's own rounding is
    the larger error; the GPU path must not add to it).
"""
import os
import subprocess

import numpy as np
import pytest

import _cases
import kirch_datuming_b200 as kd
import oracle
from kirch_datuming_b200 import rsf

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-5


def gpu_image(gd, case, device=False, scratch=0, data=None):
    import torch
    kp, geom, axis, _, use_grad = _cases.case_setup(gd, case)
    T, D = gd.tables()
    d = gd.data(case) if data is None else data
    plan = kd.Plan(kp, kd.geometry(**geom), scratch_bytes=scratch)
    img = np.zeros((axis[0], geom["nx"], geom["nz"]), np.float32)
    if device:
        tT, tD = torch.from_numpy(T).cuda(), torch.from_numpy(D).cuda()
        plan.set_tables(tT, tD, tT, tD)
        if use_grad:
            gx, gz = (torch.from_numpy(x).cuda() for x in gd.grads())
            plan.set_gradients(gx, gz, gx, gz)
        dimg = torch.zeros(img.shape, dtype=torch.float32, device="cuda")
        plan.migrate(torch.from_numpy(np.ascontiguousarray(d)).cuda(), dimg)
        img = dimg.cpu().numpy()
    else:
        plan.set_tables(T, D, T, D)
        if use_grad:
            gx, gz = gd.grads()
            plan.set_gradients(gx, gz, gx, gz)
        plan.migrate(np.ascontiguousarray(d, dtype=np.float32), img)
    stats = plan.stats()
    plan.close()
    return img, stats


@pytest.fixture(scope="module")
def o64(golden):
    return {c: _cases.oracle_image(golden, c, fp64=True) for c in golden.cases}


@pytest.mark.parametrize("case", _cases.Golden().cases)
def test_gpu_vs_fp64_oracle(golden, o64, case):
    img, stats = gpu_image(golden, case)
    assert stats["sum_launches"] >= 1
    err = oracle.rel_l2(img, o64[case])
    assert err <= TOL_FP64, err


@pytest.mark.parametrize("case", _cases.Golden().cases)
def test_gpu_vs_reference_golden(golden, o64, case):
    img, _ = gpu_image(golden, case)
    ref = golden.image(case)
    k = _cases.ub_columns(golden, case)
    ref_err = oracle.rel_l2(ref[:, k:], o64[case][:, k:])
    err = oracle.rel_l2(img[:, k:], ref[:, k:])
    assert err <= 1.5 * ref_err + 1e-6, (err, ref_err)


def test_device_pointers_match_host(golden):
    a, _ = gpu_image(golden, "base")
    b, _ = gpu_image(golden, "base", device=True)
    assert np.array_equal(a, b)


def test_small_scratch_batches_match(golden, o64):
    # a scratch cap of a few MB forces several shot batches and receiver chunks
    for case in ("base", "cmp1_half"):
        img, stats = gpu_image(golden, case, scratch=3 << 20)
        assert stats["sum_launches"] > 1
        assert oracle.rel_l2(img, o64[case]) <= TOL_FP64


def test_zero_data_and_linearity(golden):
    d = golden.data("base")
    z, _ = gpu_image(golden, "base", data=np.zeros_like(d))
    assert not np.any(z)
    rng = np.random.default_rng(1)
    e = rng.standard_normal(d.shape).astype(np.float32)
    a, _ = gpu_image(golden, "base", data=d)
    b, _ = gpu_image(golden, "base", data=e)
    c, _ = gpu_image(golden, "base", data=(2.0 * d + 0.5 * e).astype(np.float32))
    assert oracle.rel_l2(c, 2.0 * a.astype(np.float64) + 0.5 * b) < 1e-5


def test_many_bins_chunked(golden):
    # more bins than one launch keeps in shared memory: several bin chunks
    import oracle as O
    kp = kd.params("cig=1", "mode=angle", "cmp=0", "angle_min=0", "angle_max=90", "angle_step=0.2",
                   "oazmin=180", "oazmax=180")
    geom = golden.geometry_dict("base")
    axis = kd.output_axis(kp, kd.geometry(**geom))
    assert axis[0] == 451
    T, D = golden.tables()
    plan = kd.Plan(kp, kd.geometry(**geom))
    plan.set_tables(T, D, T, D)
    img = np.zeros((axis[0], geom["nx"], geom["nz"]), np.float32)
    plan.migrate(np.ascontiguousarray(golden.data("base")), img)
    assert plan.stats()["sum_launches"] == 2
    op = _cases.oracle_params(kp, geom, axis)
    ref = O.migrate_adj(op, golden.data("base"), T, D, T, D)
    assert oracle.rel_l2(img, ref) <= TOL_FP64


@pytest.mark.parametrize("aal", ["0", "-0.001", "3"])
def test_antialias_values(golden, aal):
    # the summation tests the pick window in two ways: a short form for
    # antialias >= 0 (half window >= 1 sample) and the reference's six tests
    # otherwise; both against the FP64 oracle
    import oracle as O
    kp = kd.params(*golden.tokens("base"), "antialias=" + aal)
    assert kp.antialias == np.float32(float(aal))
    geom = golden.geometry_dict("base")
    axis = kd.output_axis(kp, kd.geometry(**geom))
    T, D = golden.tables()
    plan = kd.Plan(kp, kd.geometry(**geom))
    plan.set_tables(T, D, T, D)
    img = np.zeros((axis[0], geom["nx"], geom["nz"]), np.float32)
    plan.migrate(np.ascontiguousarray(golden.data("base")), img)
    plan.close()
    ref = O.migrate_adj(_cases.oracle_params(kp, geom, axis), golden.data("base"), T, D, T, D)
    assert np.abs(ref).max() > 0
    assert oracle.rel_l2(img, ref) <= TOL_FP64


@pytest.mark.parametrize("ns,nh", [(1, 21), (5, 1), (1, 1)])
def test_single_shot_or_receiver(golden, ns, nh):
    import oracle as O
    kp = kd.params(*golden.tokens("base"))
    geom = golden.geometry_dict("base")
    geom.update(ns=ns, nh=nh)
    axis = kd.output_axis(kp, kd.geometry(**geom))
    d = np.ascontiguousarray(golden.data("base")[:ns, :nh])
    T, D = golden.tables()
    plan = kd.Plan(kp, kd.geometry(**geom))
    plan.set_tables(T, D, T, D)
    img = np.zeros((axis[0], geom["nx"], geom["nz"]), np.float32)
    plan.migrate(d, img)
    ref = O.migrate_adj(_cases.oracle_params(kp, geom, axis), d, T, D, T, D)
    assert oracle.rel_l2(img, ref) <= TOL_FP64


def test_doubint_device_vs_oracle(golden):
    import torch
    d = golden.data("base").reshape(-1, golden.meta["nt"])[:37]
    for isdiff in (0, 1):
        out = kd.doubint_device(torch.from_numpy(np.ascontiguousarray(d)).cuda(), isdiff=isdiff, dt=0.002)
        out = out.cpu().numpy()
        for k in range(d.shape[0]):
            ref = oracle.doubint(d[k], isdiff=isdiff, dt=0.002)
            assert np.allclose(out[k], ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("is_source,pos", [(1, 0.05), (1, 0.3133), (0, 0.2), (0, 0.7999), (1, -0.1), (0, 1.5)])
def test_leg_fields_vs_oracle(golden, is_source, pos):
    kp, geom, axis, op, _ = _cases.case_setup(golden, "base")
    T, D = golden.tables()
    plan = kd.Plan(kp, kd.geometry(**geom))
    plan.set_tables(T, D, T, D)
    pos = float(np.float32(pos))  # the oracle entry point takes a float position
    gT, gTx, gphi, gw = (x.cpu().numpy() for x in kd.leg_fields_device(plan, is_source, pos))
    oT, oTx, ogx, ogz = oracle.leg_fields(op, is_source, T, D, pos)
    assert np.allclose(gT, oT, rtol=1e-12, atol=1e-12)
    assert np.allclose(gTx, oTx, rtol=1e-6, atol=1e-6)
    ophi = np.arctan2(ogz, ogx)
    ok = np.hypot(ogx, ogz) > 1e-9
    dphi = np.abs(np.angle(np.exp(1j * (gphi[ok] - ophi[ok]))))
    assert dphi.max() < 1e-9
    assert np.all((gw >= 0) & (gw <= 1))


@pytest.mark.parametrize("radius,smooth", [(1, 0), (1, 1), (2, 2), (4, 6), (3, 9), (7, 11), (12, 20)])
def test_leg_direction_radii_vs_oracle(golden, radius, smooth):
    # the tiled gradient kernel (halo radius + 2 smooth) and, past its shared
    # memory limit, the plane-by-plane passes; halos wider than the 41 x 81 grid
    # check that the windows clamp to the grid and not to the tile
    kp, geom, axis, op, _ = _cases.case_setup(golden, "base")
    kp.angle_grad_radius = op.angle_grad_radius = radius
    kp.angle_smooth = op.angle_smooth = smooth
    T, D = golden.tables()
    plan = kd.Plan(kp, kd.geometry(**geom))
    plan.set_tables(T, D, T, D)
    for is_source, pos in ((1, 0.05), (0, 0.6133)):
        pos = float(np.float32(pos))
        _, _, gphi, _ = (x.cpu().numpy() for x in kd.leg_fields_device(plan, is_source, pos))
        _, _, ogx, ogz = oracle.leg_fields(op, is_source, T, D, pos)
        ok = np.hypot(ogx, ogz) > 1e-12
        assert np.array_equal(np.isnan(gphi), ~ok)
        dphi = np.abs(np.angle(np.exp(1j * (gphi[ok] - np.arctan2(ogz, ogx)[ok]))))
        assert dphi.max() < 1e-9
    plan.close()


def test_cli_end_to_end(golden, o64, tmp_path):
    meta = golden.meta
    t = meta["table"]
    T, D = golden.tables()
    rsf.write(str(tmp_path / "time.rsf"), T, t["n"], t["o"], t["d"])
    rsf.write(str(tmp_path / "tds.rsf"), D, t["n"], t["o"], t["d"])
    dd = meta["data"]["cmp0"]
    rsf.write(str(tmp_path / "data.rsf"), golden.data("base"), [meta["nt"], dd["nh"], dd["ns"]],
              [0, dd["h0"], dd["s0"]], [meta["dt"], dd["dh"], dd["ds"]], extra={"unit1": "s"})
    args = ["seismic_data=data.rsf", "migration=mig.rsf", "stable=time.rsf", "sderiv=tds.rsf", "rtable=time.rsf",
            "rderiv=tds.rsf"] + golden.tokens("base") + ["direct_mute_qc_shot=2", "direct_mute_qc_before=qb.rsf",
                                                          "direct_mute_qc_after=qa.rsf"]
    r = subprocess.run([kd.cli_path] + args, cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "Done. Elapsed time" in r.stderr
    h, img = rsf.read(str(tmp_path / "mig.rsf"))
    c = meta["cases"]["base"]
    assert h.n[:3] == c["n"] and h.native
    assert [round(v, 9) for v in h.o[:3]] == [round(v, 9) for v in c["o"]]
    assert [round(v, 9) for v in h.d[:3]] == [round(v, 9) for v in c["d"]]
    for k in ("label1", "label2", "label3", "unit1", "unit3"):
        assert h.extra[k] == c["extra"][k]
    assert oracle.rel_l2(img.reshape(o64["base"].shape), o64["base"]) <= TOL_FP64
    # QC gathers: the reference's FP32 mute of shot 2, before and after
    hb, qb = rsf.read(str(tmp_path / "qb.rsf"))
    ha, qa = rsf.read(str(tmp_path / "qa.rsf"))
    assert hb.n[:2] == [meta["nt"], dd["nh"]] and hb.extra["label2"] == "Receiver"
    shot = golden.data("base")[2]
    assert np.array_equal(qb.reshape(shot.shape), shot)
    s = np.float32(dd["s0"]) + np.float32(2) * np.float32(dd["ds"])
    for ih in range(dd["nh"]):
        rx = np.float32(dd["h0"]) + np.float32(ih) * np.float32(dd["dh"])
        ref = oracle.mute(shot[ih], 0.0, meta["dt"], s, rx, 0.5, 0.0, 0.05, fp64=False)
        assert np.array_equal(qa.reshape(shot.shape)[ih], ref)
    # the in-process entry point writes the same image
    cwd = os.getcwd()
    try:
        os.chdir(tmp_path)
        assert kd.run_cli([a if not a.startswith("migration=") else "migration=mig2.rsf" for a in args]) == 0
    finally:
        os.chdir(cwd)
    _, img2 = rsf.read(str(tmp_path / "mig2.rsf"))
    assert np.array_equal(img, img2)


# ------------------------------------------------------ forward (adj=0) path --
@pytest.mark.parametrize("name", _cases.Golden().fwd_cases)
def test_model_vs_oracle_and_reference(golden, name):
    kp, geom, axis, op, model = _cases.fwd_setup(golden, name)
    T, D = golden.tables()
    plan = kd.Plan(kp, kd.geometry(**geom))
    plan.set_tables(T, D, T, D)
    out = np.zeros((geom["ns"], geom["nh"], geom["nt"]), np.float32)
    plan.model(model, out)
    plan.close()
    o64 = oracle.model_fwd(op, model, T, D, T, D, fp64=True)
    ref = golden.fwd_data(name)
    assert oracle.rel_l2(out, o64) <= TOL_FP64
    ref_err = oracle.rel_l2(ref, o64)
    assert oracle.rel_l2(out, ref) <= 1.5 * ref_err + 1e-6


@pytest.mark.parametrize("name", _cases.Golden().fwd_cases)
def test_model_migrate_dot_product(golden, name):
    # <F m, d> = <m, F^T d> with the library's forward and adjoint operators
    import torch
    kp, geom, axis, op, model = _cases.fwd_setup(golden, name)
    kp.direct_mute = 0
    kp.isdiff = 0
    T, D = golden.tables()
    tT, tD = torch.from_numpy(T).cuda(), torch.from_numpy(D).cuda()
    plan = kd.Plan(kp, kd.geometry(**geom))
    plan.set_tables(tT, tD, tT, tD)
    g = torch.Generator(device="cuda").manual_seed(5)
    m = torch.randn(model.shape, generator=g, device="cuda")
    d = torch.randn((geom["ns"], geom["nh"], geom["nt"]), generator=g, device="cuda")
    Fm = torch.zeros_like(d)
    Ftd = torch.zeros_like(m)
    plan.model(m, Fm)
    plan.migrate(d, Ftd)
    plan.close()
    lhs = float((Fm.double() * d.double()).sum())
    rhs = float((m.double() * Ftd.double()).sum())
    assert abs(lhs - rhs) <= 1e-5 * float(Fm.double().norm() * d.double().norm())


def test_cli_forward_modelling(golden, tmp_path):
    # the drop-in executable with adj=0 (the reference's own adj=0 cannot read
    # its model; see oracle/ref_fixes.cpp) writes a three-axis data file
    name = "fwd_base"
    f = golden.meta["fwd"][name]
    ic = golden.meta["cases"][f["image"]]
    dd = golden.meta["data"][ic["data"]]
    t = golden.meta["table"]
    T, D = golden.tables()
    rsf.write(str(tmp_path / "time.rsf"), T, t["n"], t["o"], t["d"])
    rsf.write(str(tmp_path / "tds.rsf"), D, t["n"], t["o"], t["d"])
    rsf.write(str(tmp_path / "img.rsf"), golden.image(f["image"]), ic["n"], ic["o"], ic["d"])
    args = [os.path.join(os.path.dirname(kd.library_path), "bin", "kirchmig2d_cig"), "migration=img.rsf",
            "seismic_data=out.rsf", "stable=time.rsf", "sderiv=tds.rsf", "rtable=time.rsf", "rderiv=tds.rsf",
            "nt=%d" % golden.meta["nt"], "nh=%d" % dd["nh"], "ns=%d" % dd["ns"], "t0=0", "dt=%g" % golden.meta["dt"],
            "h0=%g" % dd["h0"], "dh=%g" % dd["dh"], "s0=%g" % dd["s0"], "ds=%g" % dd["ds"]] + f["tokens"]
    r = subprocess.run(args, cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    h, out = rsf.read(str(tmp_path / "out.rsf"))
    assert h.n[:3] == [golden.meta["nt"], dd["nh"], dd["ns"]] and h.extra["label3"] == "Shot"
    kp, geom, axis, op, model = _cases.fwd_setup(golden, name)
    o64 = oracle.model_fwd(op, model, T, D, T, D, fp64=True)
    assert oracle.rel_l2(out.reshape(o64.shape), o64) <= TOL_FP64
    # direct_mute is an adj=1 option, with the reference's message
    r = subprocess.run(args + ["direct_mute=1"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1 and "requires adj=1" in (r.stdout + r.stderr)
