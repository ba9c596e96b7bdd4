"""The surrogate's CPU oracle against finite differences and the eikonal
equation (no GPU)."""
import numpy as np
import pytest

import surrogate as sg  # oracle/surrogate.py

# the straight-ray factored form and the linear-gradient background with an
# additive residual
BACKGROUNDS = [dict(vgrad=0.0, residual_ms=0.0), dict(vgrad=0.6, residual_ms=1.0), dict(vgrad=0.6, residual_ms=0.0)]


def _setup(n=7, seed=3, bg=None):
    rng = np.random.default_rng(seed)
    cfg = sg.Config(lo=[0.0, 0.0, 0.0], hi=[4.0, 2.0, 4.0], fmax=6.0, vref=1.5, zsrc=0.0, **(bg or BACKGROUNDS[0]))
    p = sg.init_params(seed, out_scale=0.3).astype(np.float64)
    xs = rng.uniform(0.2, 3.8, n)
    z = rng.uniform(0.1, 1.9, n)
    x = rng.uniform(0.1, 3.9, n)
    return cfg, p, xs, z, x


@pytest.mark.parametrize("bg", BACKGROUNDS)
def test_input_gradient_matches_finite_differences(bg):
    cfg, p, xs, z, x = _setup(bg=bg)
    T, dxs, dz, dx = sg.forward(p, cfg, xs, z, x)
    h = 1e-6
    for d, args in ((dxs, lambda e: (xs + e, z, x)), (dz, lambda e: (xs, z + e, x)), (dx, lambda e: (xs, z, x + e))):
        num = (sg.forward(p, cfg, *args(h))[0] - sg.forward(p, cfg, *args(-h))[0]) / (2 * h)
        assert np.allclose(d, num, rtol=1e-6, atol=1e-8)


@pytest.mark.parametrize("bg", BACKGROUNDS)
def test_parameter_gradient_matches_finite_differences(bg):
    cfg, p, xs, z, x = _setup(bg=bg)
    Ttrue = sg.forward(p, cfg, xs, z, x)[0] * 1.01 + 0.002
    loss, g = sg.loss_grad(p, cfg, xs, z, x, Ttrue)
    rng = np.random.default_rng(0)
    idx = np.concatenate([rng.integers(o, o + 200, 4) for o in (sg.OFF_W1, sg.OFF_W2, sg.OFF_W3, sg.OFF_W4)] +
                         [np.array([sg.OFF_B1 + 5, sg.OFF_B2 + 9, sg.OFF_B3 + 1, sg.OFF_B4 + 77, sg.OFF_WO + 3,
                                    sg.OFF_BO])])
    for k in idx:
        e = np.zeros_like(p)
        e[k] = 1e-6
        num = (sg.loss_grad(p + e, cfg, xs, z, x, Ttrue)[0] - sg.loss_grad(p - e, cfg, xs, z, x, Ttrue)[0]) / 2e-6
        assert abs(num - g[k]) <= 1e-5 * max(1.0, abs(g[k])), (k, num, g[k])


def test_bf16_rounding():
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1e-40])
    r = sg.bf16(a)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5


def test_linear_gradient_background_solves_the_eikonal_equation():
    # |grad Tb| = 1 / v(z) for v = vref + vgrad (z - zsrc), its derivatives
    # agree with finite differences, it is symmetric in x - xs, and it tends
    # to the straight-ray time as vgrad -> 0
    rng = np.random.default_rng(5)
    n = 500
    xs, z, x = rng.uniform(0, 4, n), rng.uniform(0.01, 2, n), rng.uniform(0, 4, n)
    cfg = sg.Config([0, 0, 0], [4, 2, 4], vref=1.5, zsrc=0.0, vgrad=0.6)
    Tb, dxs, dz, dx = sg._background(cfg, xs, z, x)
    v = 1.5 + 0.6 * z
    assert np.allclose(dx * dx + dz * dz, 1.0 / v ** 2, rtol=1e-10)
    assert np.allclose(dxs, -dx)
    h = 1e-6
    assert np.allclose((sg._background(cfg, xs, z + h, x)[0] - sg._background(cfg, xs, z - h, x)[0]) / (2 * h), dz,
                       rtol=1e-6, atol=1e-9)
    assert np.allclose(sg._background(cfg, xs, z, 2 * xs - x)[0], Tb)
    # the classical closed form acosh(1 + g^2 r^2 / (2 v0 v)) / g
    r2 = (x - xs) ** 2 + z ** 2
    assert np.allclose(Tb, np.arccosh(1 + 0.36 * r2 / (2 * 1.5 * v)) / 0.6, rtol=1e-12)
    for g in (1e-3, 1e-6, 0.0):
        c = sg.Config([0, 0, 0], [4, 2, 4], vref=1.5, zsrc=0.0, vgrad=g)
        assert np.allclose(sg._background(c, xs, z, x)[0], np.sqrt(r2) / 1.5, rtol=2 * g + 1e-12)
