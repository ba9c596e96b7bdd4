"""The oracle is pinned to the reference: its FP32 build must reproduce the
reference binary's images bit for bit on every golden case; its FP64 build is
the precision reference of the GPU path."""
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
