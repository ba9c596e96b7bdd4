"""The oracle is pinned to the reference: its FP32 build must reproduce the
reference binary's images bit for bit on every golden case; its FP64 build is
the precision reference of the GPU path."""
import os

import numpy as np
import pytest

import _cases
import oracle


@pytest.mark.parametrize("case", _cases.Golden().cases)
def test_oracle_fp32_bitexact_vs_reference(golden, case):
    img = _cases.oracle_image(golden, case, fp64=False).astype(np.float32)
    ref = golden.image(case)
    assert img.shape == ref.shape
    k = _cases.ub_columns(golden, case)
    img, ref = img[:, k:, :], ref[:, k:, :]
    assert np.array_equal(img, ref), "max abs diff %g" % np.max(np.abs(img - ref))


@pytest.mark.parametrize("case", _cases.Golden().cases)
def test_oracle_fp64_close_to_reference(golden, case):
    # the reference's FP32 rounding keeps it within a few 1e-5 of exact math
    # on these short traces (2.8e-4 at nt=1001, 64x201 traces)
    img = _cases.oracle_image(golden, case, fp64=True)
    k = _cases.ub_columns(golden, case)
    assert oracle.rel_l2(golden.image(case)[:, k:, :], img[:, k:, :]) < 2e-4


def test_oracle_doubint_matches_definition():
    rng = np.random.default_rng(3)
    x = rng.standard_normal(257).astype(np.float32)
    d = oracle.doubint(x)
    c = np.cumsum(x.astype(np.float64))
    ref = np.cumsum(c[::-1])[::-1]
    assert np.allclose(d, ref, rtol=0, atol=1e-9 * np.abs(ref).max())


def test_oracle_pick_known_answer():
    # on a linear D the second difference vanishes; on a quadratic sampled at
    # the three pick times it is imp*(2*D(t) - D(t-a) - D(t+a)) = -imp*2*c*a^2
    # with a = deltat + dt and imp = (dt / (dt + 2a))^2
    nt, dt = 200, 0.004
    t = np.arange(nt) * dt
    assert abs(oracle.pick(0.3, 0.01, 3.0 + 2.0 * t, dt, 0.0)) < 1e-12
    c = 1.7
    a = 0.008 + dt
    imp = (dt / (dt + 2 * a)) ** 2
    v = oracle.pick(0.3 + 1e-12, 0.008, c * t * t, dt, 0.0)
    assert v == pytest.approx(-imp * 2 * c * a * a, rel=1e-6)
    # between samples the linear interpolation adds c*dt^2*f*(1-f) per term
    v = oracle.pick(0.3 + 1e-12, 0.01, c * t * t, dt, 0.0)
    a = 0.014
    assert v == pytest.approx(-(dt / (dt + 2 * a)) ** 2 * (2 * c * a * a + 0.5 * c * dt * dt), rel=1e-6)
    # reference early returns (kirmig.cpp:41-49)
    assert oracle.pick(-0.001, 0.0, c * t * t, dt, 0.0) == 0.0
    assert oracle.pick(0.003, 0.0, c * t * t, dt, 0.0) == 0.0  # t - dt < 0
    assert oracle.pick((nt - 1.5) * dt, 0.0, c * t * t, dt, 0.0) == 0.0


def test_oracle_mute_profile():
    nt, dt = 100, 0.01
    tr = np.ones(nt, np.float32)
    out = oracle.mute(tr, 0.0, dt, 1.0, 1.4, 0.5, 0.1, 0.2)
    boundary = 0.1 + 0.5 * 0.4
    t = np.arange(nt) * dt
    assert np.all(out[t <= boundary - 1e-6] == 0)
    assert np.all(out[t >= boundary + 0.2 + 1e-6] == 1)
    mid = (t > boundary) & (t < boundary + 0.2)
    u = (t[mid] - boundary) / 0.2
    assert np.allclose(out[mid], 0.5 * (1 - np.cos(np.pi * u)), atol=1e-6)


# ------------------------------------------------------ forward (adj=0) path --
@pytest.mark.parametrize("name", _cases.Golden().fwd_cases)
def test_oracle_fp32_forward_bitexact_vs_reference(golden, name):
    # oracle/_ref/kirchmig2d_cig_fwd: the reference tool, one OpenMP thread
    kp, geom, axis, op, model = _cases.fwd_setup(golden, name)
    T, D = golden.tables()
    got = oracle.model_fwd(op, model, T, D, T, D, fp64=False).astype(np.float32)
    assert np.array_equal(got, golden.fwd_data(name))


@pytest.mark.parametrize("name", _cases.Golden().fwd_cases)
def test_oracle_forward_is_adjoint_of_migration(golden, name):
    # <F m, d> = <m, F^T d>: the FP64 forward oracle against the FP64 adjoint
    # oracle (itself pinned bit-exact to the reference) with the forward's
    # own settings (the forward applies neither the direct mute nor diff2)
    kp, geom, axis, op, model = _cases.fwd_setup(golden, name)
    op.direct_mute = 0
    op.isdiff = 0
    T, D = golden.tables()
    rng = np.random.default_rng(3)
    m = rng.standard_normal(model.shape).astype(np.float32)
    d = rng.standard_normal((geom["ns"], geom["nh"], geom["nt"])).astype(np.float32)
    Fm = oracle.model_fwd(op, m, T, D, T, D, fp64=True)
    Ftd = oracle.migrate_adj(op, d, T, D, T, D, fp64=True)
    lhs = float(np.dot(Fm.ravel(), d.astype(np.float64).ravel()))
    rhs = float(np.dot(m.astype(np.float64).ravel(), Ftd.ravel()))
    assert abs(lhs - rhs) <= 1e-10 * (np.linalg.norm(Fm) * np.linalg.norm(d))


REF_MIG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "kirchmig2d_cig")


def _random_tokens(rng):
    t = ["cig=%d" % rng.integers(0, 2), "mode=%s" % rng.choice(["angle", "offset"]),
         "cmp=%d" % rng.integers(0, 2), "half_angle=%d" % rng.integers(0, 2),
         "type=%s" % rng.choice(["h", "l", "p"]), "antialias=%g" % rng.choice([0.5, 1.0, 2.0]),
         "tau=%g" % rng.choice([0.0, 0.004]), "diff=%d" % rng.integers(0, 2),
         "aperture=%g" % rng.choice([30.0, 60.0, 90.0]), "aperture_taper=%g" % rng.choice([5.0, 10.0]),
         "angle_interp=%d" % rng.integers(0, 2)]
    if rng.random() < 0.5:
        t += ["angle_min=0", "angle_max=%g" % rng.choice([40.0, 60.0, 90.0]), "angle_step=%g" % rng.choice([1.0, 2.5])]
    if rng.random() < 0.5:
        t += ["oazmin=%g" % rng.choice([70.0, 80.0]), "oazmax=%g" % rng.choice([40.0, 50.0]),
              "oaztaper=%g" % rng.choice([0.0, 10.0])]
    if rng.random() < 0.4:
        t += ["angle_taper_start=%g" % rng.choice([20.0, 30.0]), "angle_taper_end=%g" % rng.choice([45.0, 55.0])]
    if rng.random() < 0.4:
        t += ["direct_mute=1", "direct_mute_slope=%g" % rng.choice([0.3, 0.6]),
              "direct_mute_intercept=%g" % rng.choice([0.0, 0.02]), "direct_mute_taper=%g" % rng.choice([0.02, 0.05])]
    if rng.random() < 0.3:
        t += ["aperture_trace=%d" % rng.integers(4, 12), "aperture_trace_taper=%d" % rng.integers(0, 4)]
    return t


@pytest.mark.skipif(not os.path.exists(REF_MIG), reason="reference kirchmig2d_cig not built (make -C oracle ref)")
@pytest.mark.parametrize("seed", range(16))
def test_oracle_fp32_bitexact_random_configurations(golden, tmp_path, seed):
    # random parameter sets and geometries on the fixture tables, through the
    # reference binary (one thread): the FP32 mirror gives its image bit for bit
    import subprocess
    import kirch_datuming_b200 as kd
    from kirch_datuming_b200 import rsf
    rng = np.random.default_rng(700 + seed)
    t = golden.meta["table"]
    T, D = golden.tables()
    rsf.write(str(tmp_path / "time.rsf"), T, t["n"], t["o"], t["d"])
    rsf.write(str(tmp_path / "tds.rsf"), D, t["n"], t["o"], t["d"])
    toks = _random_tokens(rng)
    cmp1 = "cmp=1" in toks
    p0, dp, npos = t["o"][2], t["d"][2], t["n"][2]
    span = (npos - 1) * dp
    ns, nh = int(rng.integers(1, 4)), int(rng.integers(2, 7))
    f = lambda v: float(np.float32(v))  # noqa: E731
    ds = f(rng.choice([0.04, 0.06, 0.1]))
    dh = f(rng.choice([0.02, 0.04, 0.05]))
    if cmp1:   # receivers at s + h inside the tables
        h0 = f(-(nh // 2) * dh)
        s0 = f(p0 + (nh // 2) * dh + 0.02)
        ns = max(1, min(ns, int((span - (nh - 1) * dh - 0.04) / ds)))
    else:
        h0 = f(p0 + rng.uniform(0.0, span - (nh - 1) * dh))
        s0 = f(p0 + rng.uniform(0.0, span - (ns - 1) * ds))
    nt, dt = golden.meta["nt"], golden.meta["dt"]
    data = (rng.standard_normal((ns, nh, nt)) * 1e-2).astype(np.float32)
    rsf.write(str(tmp_path / "d.rsf"), data, [nt, nh, ns], [0.0, h0, s0], [dt, dh, ds], extra={"unit1": "s"})
    r = subprocess.run([REF_MIG, "seismic_data=d.rsf", "migration=m.rsf", "stable=time.rsf", "sderiv=tds.rsf",
                        "rtable=time.rsf", "rderiv=tds.rsf"] + toks, cwd=tmp_path, capture_output=True, text=True,
                       env=dict(os.environ, OMP_NUM_THREADS="1"))
    assert r.returncode == 0, r.stderr[-500:]
    h, ref = rsf.read(str(tmp_path / "m.rsf"))
    ref = ref.reshape(h.n[2], h.n[1], h.n[0])
    geom = dict(nt=nt, nh=nh, ns=ns, t0=0.0, dt=f(dt), h0=h0, dh=dh, s0=s0, ds=ds, nz=golden.meta["nz"],
                nx=golden.meta["nx"], z0=0.0, dz=f(golden.meta["dz"]), x0=0.0, dx=f(golden.meta["dz"]),
                sny=npos, sy0=f(p0), sdy=f(dp), rny=npos, ry0=f(p0), rdy=f(dp))
    kp = kd.params(*toks)
    axis = kd.output_axis(kp, kd.geometry(**geom))
    assert ref.shape == (axis[0], geom["nx"], geom["nz"])
    img = oracle.migrate_adj(_cases.oracle_params(kp, geom, axis), data, T, D, T, D, fp64=False).astype(np.float32)
    k = 3 if "type=p" in toks else 0
    assert np.abs(ref).max() > 0
    assert np.array_equal(img[:, k:, :], ref[:, k:, :]), "max abs diff %g" % np.max(np.abs(img - ref))
