"""CPU oracle of the learned traveltime surrogate (test infrastructure only).

The reference has no surrogate: this restates, in float64 numpy, the network
the CUDA kernels evaluate and train, so that their forward values, input
gradients and parameter gradients can be checked.  With ``mirror=True`` the
quantities the GPU feeds to its BF16 tensor cores (weights, Fourier features,
hidden activations, backpropagated gradients) are rounded to BF16 at the same
points; everything else stays float64.

Network (per leg position xs and image point (z, x), all in km):
    u_i   = (v_i - lo_i) * 2 / (hi_i - lo_i) - 1                    i = xs, z, x
    f     = [sin(th_ik), cos(th_ik)] interleaved, th_ik = (k+1) * fstep * u_i,
            k < 64, fstep = pi * fmax / 64            -> 384 features
    h_1   = SiLU(W_1 f + b_1),  h_l = SiLU(W_l h_{l-1} + b_l)  (l = 2..4, width 128)
    out   = w_o . h_4 + b_o
    T     = Tb + rscale * out   (additive residual, residual_ms > 0), or
    T     = Tb * (1 + out)      (factored form, residual_ms = 0)
with Tb the first arrival of the background medium v(z) = vref + vgrad (z -
zsrc): acosh(1 + g^2 r^2 / (2 vs vp)) / g for a constant velocity gradient g
(the straight-ray time r / vref at g = 0).  The factored form keeps the
source singularity out of the network, as in factored-eikonal learning
(e.g. EikoNet); the additive form lets it learn only what the background
misses.

Parameter vector layout (float32 on the device): W_1 [128][384], W_2, W_3,
W_4 [128][128] (row = output), b_1..b_4 [128], w_o [128], b_o.

Loss of a batch: mean((1000 * (T - T_true))^2) (milliseconds squared).
"""
from __future__ import annotations

import numpy as np

NF = 64
NIN = 3
H = 128
FEAT = NIN * 2 * NF
OFF_W1 = 0
OFF_W2 = OFF_W1 + H * FEAT
OFF_W3 = OFF_W2 + H * H
OFF_W4 = OFF_W3 + H * H
OFF_B1 = OFF_W4 + H * H
OFF_B2 = OFF_B1 + H
OFF_B3 = OFF_B2 + H
OFF_B4 = OFF_B3 + H
OFF_WO = OFF_B4 + H
OFF_BO = OFF_WO + H
NPARAM = OFF_BO + 1


def bf16(a):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    out = r.view(np.float32).astype(np.float64)
    return np.where(np.isfinite(f), out, f.astype(np.float64))


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    W = [p[OFF_W1:OFF_W2].reshape(H, FEAT), p[OFF_W2:OFF_W3].reshape(H, H), p[OFF_W3:OFF_W4].reshape(H, H),
         p[OFF_W4:OFF_B1].reshape(H, H)]
    b = [p[OFF_B1:OFF_B2], p[OFF_B2:OFF_B3], p[OFF_B3:OFF_B4], p[OFF_B4:OFF_WO]]
    return W, b, p[OFF_WO:OFF_BO], p[OFF_BO]


def init_params(seed: int = 0, out_scale: float = 0.01):
    """Seeded initial parameters (uniform, fan-in scaled; small output layer)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, np.float64)
    fans = [(OFF_W1, FEAT), (OFF_W2, H), (OFF_W3, H), (OFF_W4, H)]
    for off, fan in fans:
        lim = np.sqrt(6.0 / fan)
        p[off:off + H * fan] = rng.uniform(-lim, lim, H * fan)
    p[OFF_WO:OFF_BO] = rng.uniform(-out_scale, out_scale, H)
    return p.astype(np.float32)


class Config:
    def __init__(self, lo, hi, fmax=8.0, vref=1.5, zsrc=0.0, vgrad=0.0, residual_ms=0.0):
        self.lo = np.asarray(lo, np.float64)
        self.hi = np.asarray(hi, np.float64)
        self.fmax, self.vref, self.zsrc = float(fmax), float(vref), float(zsrc)
        self.vgrad, self.residual_ms = float(vgrad), float(residual_ms)

    @property
    def scale(self):
        return 2.0 / (self.hi - self.lo)

    @property
    def fstep(self):
        return np.pi * self.fmax / NF


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def _silu(z):
    return z * _sig(z)


def _dsilu(z):
    s = _sig(z)
    return s * (1.0 + z * (1.0 - s))


def _features(cfg, u):
    """u [n][3] -> features [n][384] and their u-derivatives (same shape, each
    feature depends on one input)."""
    n = u.shape[0]
    k = np.arange(1, NF + 1) * cfg.fstep
    f = np.empty((n, FEAT))
    df = np.empty((n, FEAT))
    for i in range(NIN):
        th = u[:, i:i + 1] * k[None, :]
        f[:, i * 2 * NF:(i + 1) * 2 * NF:2] = np.sin(th)
        f[:, i * 2 * NF + 1:(i + 1) * 2 * NF:2] = np.cos(th)
        df[:, i * 2 * NF:(i + 1) * 2 * NF:2] = k * np.cos(th)
        df[:, i * 2 * NF + 1:(i + 1) * 2 * NF:2] = -k * np.sin(th)
    return f, df


def _background(cfg, xs, z, x):
    """Tb and dTb/dxs, dTb/dz, dTb/dx of the linear-gradient medium
    (constant velocity at vgrad = 0)."""
    dxv = x - xs
    dzv = z - cfg.zsrc
    g, vs = cfg.vgrad, cfg.vref
    r2 = dxv * dxv + dzv * dzv
    r = np.sqrt(r2)
    vp = np.maximum(vs + g * dzv, 1e-3 * vs)
    q = vs * vp
    eps = g * g * r2 / (2.0 * q)
    with np.errstate(invalid="ignore", divide="ignore"):
        fac = np.where(eps < 1e-12, 1.0 - eps / 12.0,
                       np.log1p(eps + np.sqrt(eps * (2.0 + eps))) / np.sqrt(2.0 * np.maximum(eps, 1e-300)))
        Tb = r * fac / np.sqrt(q)
        k = np.where(r > 0, np.sqrt(2.0 / (q * (2.0 + eps))) / np.where(r > 0, r, 1.0), 0.0)
    dx = dxv * k
    return Tb, -dx, (dzv - r2 * g / (2.0 * vp)) * k, dx


def _out_scale(cfg, Tb):
    """(osc, m): T = Tb + osc * out and dT/dv = dTb/dv (1 + m out) + osc dout/dv."""
    if cfg.residual_ms > 0:
        return np.full_like(Tb, cfg.residual_ms * 1e-3), 0.0
    return Tb, 1.0


def forward(params, cfg: Config, xs, z, x, mirror: bool = False, keep: bool = False):
    """T and its derivatives (dT/dxs, dT/dz, dT/dx) at the given points."""
    rb = bf16 if mirror else (lambda a: np.asarray(a, np.float64))
    W, b, wo, bo = unpack(params)
    Wq = [rb(w) for w in W]
    xs, z, x = (np.asarray(a, np.float64) for a in (xs, z, x))
    v = np.stack([xs, z, x], axis=1)
    u = (v - cfg.lo) * cfg.scale - 1.0
    f, df = _features(cfg, u)
    a = rb(f)
    zs, hs = [], [a]
    for l in range(4):
        zl = hs[-1] @ Wq[l].T + b[l]
        zs.append(zl)
        hl = _silu(zl)
        hs.append(rb(hl) if l < 3 else hl)
    out = hs[4] @ wo + bo
    # input gradient of out: backpropagate d out / d out = 1
    g = rb(wo[None, :] * _dsilu(zs[3]))
    for l in (3, 2, 1):
        g = rb((g @ Wq[l]) * _dsilu(zs[l - 1]))
    G0 = g @ Wq[0]                                # d out / d feature
    dout_du = np.stack([(G0 * df)[:, i * 2 * NF:(i + 1) * 2 * NF].sum(1) for i in range(NIN)], axis=1)
    dout_dv = dout_du * cfg.scale
    Tb, dxs0, dz0, dx0 = _background(cfg, xs, z, x)
    osc, m = _out_scale(cfg, Tb)
    T = Tb + osc * out
    f1 = 1.0 + m * out
    res = (T, dxs0 * f1 + osc * dout_dv[:, 0], dz0 * f1 + osc * dout_dv[:, 1], dx0 * f1 + osc * dout_dv[:, 2])
    if keep:
        return res, dict(a=a, zs=zs, hs=hs, osc=osc, out=out, Wq=Wq, wo=wo)
    return res


def loss_grad(params, cfg: Config, xs, z, x, Ttrue, mirror: bool = False, ntotal=None):
    """Loss of the batch and its gradient with respect to the parameter
    vector (float64).  ntotal: the batch size the mean is taken over."""
    rb = bf16 if mirror else (lambda a: np.asarray(a, np.float64))
    (T, *_), k = forward(params, cfg, xs, z, x, mirror=mirror, keep=True)
    n = len(T) if ntotal is None else ntotal
    r = 1000.0 * (T - np.asarray(Ttrue, np.float64))
    loss = float((r * r).sum() / n)
    gout = 2.0 * r * 1000.0 * k["osc"] / n         # d loss / d out
    W, b, wo, bo = unpack(params)
    grad = np.zeros(NPARAM)
    zs, hs, Wq = k["zs"], k["hs"], k["Wq"]
    grad[OFF_WO:OFF_BO] = gout @ hs[4]
    grad[OFF_BO] = gout.sum()
    g = rb(gout[:, None] * wo[None, :] * _dsilu(zs[3]))
    offs = [(OFF_W1, OFF_B1, FEAT), (OFF_W2, OFF_B2, H), (OFF_W3, OFF_B3, H), (OFF_W4, OFF_B4, H)]
    for l in (3, 2, 1, 0):
        ow, ob, fan = offs[l]
        grad[ow:ow + H * fan] = (g.T @ hs[l]).ravel()
        grad[ob:ob + H] = g.sum(0)
        if l > 0:
            g = rb((g @ Wq[l]) * _dsilu(zs[l - 1]))
    return loss, grad
