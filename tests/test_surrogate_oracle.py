"""The surrogate's CPU oracle against finite differences (no GPU)."""
import numpy as np

import surrogate as sg  # oracle/surrogate.py


def _setup(n=7, seed=3):
    rng = np.random.default_rng(seed)
    cfg = sg.Config(lo=[0.0, 0.0, 0.0], hi=[4.0, 2.0, 4.0], fmax=6.0, vref=1.5, zsrc=0.0)
    p = sg.init_params(seed, out_scale=0.3).astype(np.float64)
    xs = rng.uniform(0.2, 3.8, n)
    z = rng.uniform(0.1, 1.9, n)
    x = rng.uniform(0.1, 3.9, n)
    return cfg, p, xs, z, x


def test_input_gradient_matches_finite_differences():
    cfg, p, xs, z, x = _setup()
    T, dxs, dz, dx = sg.forward(p, cfg, xs, z, x)
    h = 1e-6
    for d, args in ((dxs, lambda e: (xs + e, z, x)), (dz, lambda e: (xs, z + e, x)), (dx, lambda e: (xs, z, x + e))):
        num = (sg.forward(p, cfg, *args(h))[0] - sg.forward(p, cfg, *args(-h))[0]) / (2 * h)
        assert np.allclose(d, num, rtol=1e-6, atol=1e-8)


def test_parameter_gradient_matches_finite_differences():
    cfg, p, xs, z, x = _setup()
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
