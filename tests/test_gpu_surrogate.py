"""The traveltime surrogate's tensor-core kernels (tcgen05 + TMEM) against
float64 references computed on the host."""
import numpy as np
import pytest

import kirch_datuming_b200 as kd

pytestmark = pytest.mark.gpu


def test_tensor_core_operand_views():
    # X W^T (forward layer), X W (backward through a layer), X^T W (weight
    # gradient): BF16 inputs, FP32 accumulation -> products are exact, only
    # the FP32 sums round
    import torch
    g = torch.Generator().manual_seed(7)
    X = torch.randn(128, 128, generator=g).to(torch.bfloat16)
    W = torch.randn(128, 128, generator=g).to(torch.bfloat16)
    D = kd.tc_selftest(X.cuda(), W.cuda()).cpu().double().numpy()
    x, w = X.double().numpy(), W.double().numpy()
    for got, ref in ((D[0], x @ w.T), (D[1], x @ w), (D[2], x.T @ w)):
        assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max() + 1e-6


import surrogate as sgo  # oracle/surrogate.py: the float64 restatement of the network

LO, HI = (0.0, 0.0, 0.0), (4.0, 2.0, 4.0)


def _net(seed=5, out_scale=30.0, fmax=6.0):
    s = kd.Surrogate(LO, HI, fmax=fmax, vref=1.5, zsrc=0.0, seed=seed)
    p = s.get_params()
    p[sgo.OFF_WO:sgo.OFF_BO] *= out_scale  # tau visibly different from 1
    p[sgo.OFF_B1:sgo.OFF_WO] = np.random.default_rng(seed).uniform(-0.2, 0.2, 4 * sgo.H)
    s.set_params(p)
    cfg = sgo.Config(LO, HI, fmax=fmax, vref=1.5, zsrc=0.0)
    return s, cfg, p


def _points(n, seed=11):
    rng = np.random.default_rng(seed)
    return (rng.uniform(0.1, 3.9, n).astype(np.float32), rng.uniform(0.05, 1.95, n).astype(np.float32),
            rng.uniform(0.1, 3.9, n).astype(np.float32))


def _stats(e):
    return np.median(e), np.percentile(e, 95), e.max()


def test_surrogate_eval_vs_oracle():
    # forward value and input gradient through the tcgen05 kernels against the
    # float64 oracle with the same BF16 rounding points.  The GPU builds the
    # Fourier features by rotation (a few FP32 ulp off the exact sines), so a
    # value close to a BF16 rounding boundary occasionally rounds the other
    # way (one BF16 ulp, 2^-8 relative) and moves that point by up to ~1e-3:
    # most points agree to FP32 accumulation order, a few percent carry a flip.
    # A wrong operand layout or TMEM mapping is off by O(1) everywhere.
    s, cfg, p = _net()
    xs, z, x = _points(1000)
    got = [t.cpu().double().numpy() for t in s.eval(xs, z, x)]
    ref = sgo.forward(p, cfg, xs.astype(np.float64), z.astype(np.float64), x.astype(np.float64), mirror=True)
    T0 = np.hypot(x - xs, z) / 1.5
    assert np.abs(ref[0] / T0 - 1).max() > 0.05  # the network does something
    e = np.abs(got[0] - ref[0]) / T0
    print("tau err median %.2e p95 %.2e max %.2e" % _stats(e))
    med, p95, mx = _stats(e)
    assert med < 1e-5 and p95 < 2e-3 and mx < 2e-2
    for k in (1, 2, 3):
        e = np.abs(got[k] - ref[k]) / np.sqrt(np.mean(ref[k] ** 2))
        print("dT/d%s err median %.2e p95 %.2e max %.2e" % (("xs", "z", "x")[k - 1], *_stats(e)))
        med, p95, mx = _stats(e)
        assert med < 1e-4 and p95 < 5e-3 and mx < 5e-2
    s.close()


def test_surrogate_loss_grad_vs_oracle():
    s, cfg, p = _net(seed=6)
    xs, z, x = _points(300, seed=12)  # two full tiles and a partial one
    Tt = (sgo.forward(p, cfg, xs, z, x)[0] * 1.02 + 0.003).astype(np.float32)
    loss, grad = s.loss_grad(xs, z, x, Tt)
    grad = grad.cpu().double().numpy()
    rl, rg = sgo.loss_grad(p, cfg, xs.astype(np.float64), z.astype(np.float64), x.astype(np.float64),
                           Tt.astype(np.float64), mirror=True)
    print("loss %.6e ref %.6e" % (loss, rl))
    assert abs(loss - rl) <= 2e-3 * rl
    blocks = [("W1", sgo.OFF_W1, sgo.OFF_W2), ("W2", sgo.OFF_W2, sgo.OFF_W3), ("W3", sgo.OFF_W3, sgo.OFF_W4),
              ("W4", sgo.OFF_W4, sgo.OFF_B1), ("b", sgo.OFF_B1, sgo.OFF_WO), ("wo", sgo.OFF_WO, sgo.OFF_BO),
              ("bo", sgo.OFF_BO, sgo.NPARAM)]
    for name, a, b in blocks:
        d = np.linalg.norm(grad[a:b] - rg[a:b]) / max(np.linalg.norm(rg[a:b]), 1e-30)
        print("grad %s rel %.3e" % (name, d))
        assert d < 1e-2, name
    s.close()


def test_surrogate_eval_stages_vs_oracle():
    # the accumulators of each tensor-core step of the first tile (forward
    # layer 4, the three backward-data GEMMs, d tau/d f of the xs features)
    s, cfg, p = _net(seed=8)
    xs, z, x = _points(128, seed=13)
    st = s.eval_stages(xs, z, x).cpu().double().numpy()
    _, k = sgo.forward(p, cfg, xs.astype(np.float64), z.astype(np.float64), x.astype(np.float64), mirror=True,
                       keep=True)
    W, b, wo, bo = sgo.unpack(p)
    Wq, zs, hs = k["Wq"], k["zs"], k["hs"]
    refs = [hs[3] @ Wq[3].T]
    g = sgo.bf16(wo[None, :] * sgo._dsilu(zs[3]))
    for l in (3, 2, 1):
        G = g @ Wq[l]
        refs.append(G)
        g = sgo.bf16(G * sgo._dsilu(zs[l - 1]))
    refs.append(g @ Wq[0][:, :128])
    names = ["z4", "G3", "G2", "G1", "G0xs"]
    bad = []
    for i, (nm, ref) in enumerate(zip(names, refs)):
        e = np.abs(st[i] - ref) / np.sqrt(np.mean(ref ** 2))
        print("%s median %.2e p95 %.2e max %.2e" % (nm, *_stats(e)))
        if np.median(e) > 1e-3:
            bad.append(nm)
    s.close()
    assert not bad, bad
