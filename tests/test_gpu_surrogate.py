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


# the straight-ray factored form T = T0 (1 + out) and the linear-gradient
# background with an additive residual T = Tb + 1 ms * out
BACKGROUNDS = {"straight_factored": dict(vgrad=0.0, residual_ms=0.0), "lingrad_additive": dict(vgrad=0.6, residual_ms=1.0)}


def _net(seed=5, out_scale=30.0, fmax=6.0, bg="straight_factored"):
    s = kd.Surrogate(LO, HI, fmax=fmax, vref=1.5, zsrc=0.0, seed=seed, **BACKGROUNDS[bg])
    p = s.get_params()
    p[sgo.OFF_WO:sgo.OFF_BO] *= out_scale  # the network's term visibly non-zero
    p[sgo.OFF_B1:sgo.OFF_WO] = np.random.default_rng(seed).uniform(-0.2, 0.2, 4 * sgo.H)
    s.set_params(p)
    cfg = sgo.Config(LO, HI, fmax=fmax, vref=1.5, zsrc=0.0, **BACKGROUNDS[bg])
    return s, cfg, p


def _points(n, seed=11):
    rng = np.random.default_rng(seed)
    return (rng.uniform(0.1, 3.9, n).astype(np.float32), rng.uniform(0.05, 1.95, n).astype(np.float32),
            rng.uniform(0.1, 3.9, n).astype(np.float32))


def _stats(e):
    return np.median(e), np.percentile(e, 95), e.max()


@pytest.mark.parametrize("bg", sorted(BACKGROUNDS))
def test_surrogate_eval_vs_oracle(bg):
    # forward value and input gradient through the tcgen05 kernels against the
    # float64 oracle with the same BF16 rounding points.  The GPU builds the
    # Fourier features by rotation (a few FP32 ulp off the exact sines), so a
    # value close to a BF16 rounding boundary occasionally rounds the other
    # way (one BF16 ulp, 2^-8 relative) and moves that point by up to ~1e-3:
    # most points agree to FP32 accumulation order, a few percent carry a flip.
    # A wrong operand layout or TMEM mapping is off by O(1) everywhere.
    # Errors are in units of the network's output (T - Tb) / osc.
    s, cfg, p = _net(bg=bg)
    xs, z, x = _points(1000)
    got = [t.cpu().double().numpy() for t in s.eval(xs, z, x)]
    v64 = [a.astype(np.float64) for a in (xs, z, x)]
    ref = sgo.forward(p, cfg, *v64, mirror=True)
    Tb = sgo._background(cfg, *v64)[0]
    osc = np.maximum(sgo._out_scale(cfg, Tb)[0], 1e-4)
    assert np.abs((ref[0] - Tb) / osc).max() > 0.05  # the network does something
    e = np.abs(got[0] - ref[0]) / osc
    print("out err median %.2e p95 %.2e max %.2e" % _stats(e))
    med, p95, mx = _stats(e)
    if BACKGROUNDS[bg]["residual_ms"] > 0:
        # T = Tb + 1 ms * out comes back in FP32: at 1-2 s its rounding
        # (~1e-7 s) is ~1e-4 of the residual scale, which bounds the median
        ea = np.abs(got[0] - ref[0])
        assert np.median(ea) < 2e-7 and np.percentile(ea, 95) < 2e-6 and ea.max() < 2e-5
    else:
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


import _cases  # noqa: E402


def _fd_direction(T, r, sm, dz, dx):
    """Direction of the stabilised traveltime gradient of one field T[nx][nz]
    as the table path forms it (float64): centred differences of radius r
    clamped to the grid and divided by the actual span
    (src/kirchmig2d_cig.cpp:130-152, :424-435), then two passes of a box
    average of radius sm along depth and then lateral position, windows
    clamped to the grid (:438-492); NaN where the gradient vanishes."""
    nx, nz = T.shape
    gx, gz = np.zeros_like(T), np.zeros_like(T)
    for ix in range(nx):
        il, ir = max(0, ix - r), min(nx - 1, ix + r)
        if ir != il:
            gx[ix] = (T[ir] - T[il]) / ((ir - il) * dx)
    for iz in range(nz):
        it, ib = max(0, iz - r), min(nz - 1, iz + r)
        if ib != it:
            gz[:, iz] = (T[:, ib] - T[:, it]) / ((ib - it) * dz)

    def box(a, axis):
        n = a.shape[axis]
        out = np.empty_like(a)
        for k in range(n):
            lo, hi = max(0, k - sm), min(n - 1, k + sm)
            sl = [slice(None)] * 2
            sl[axis] = slice(lo, hi + 1)
            o = [slice(None)] * 2
            o[axis] = k
            out[tuple(o)] = a[tuple(sl)].mean(axis=axis)
        return out
    for _ in range(2 if sm > 0 else 0):
        gx, gz = box(box(gx, 1), 0), box(box(gz, 1), 0)
    phi = np.arctan2(gz, gx)
    phi[np.hypot(gx, gz) <= 1e-12] = np.nan
    return phi


def test_surrogate_fd_angle_and_table_derivative(golden):
    # angle="fd": the direction is the table path's finite-difference
    # gradient of the surrogate's own traveltime field; tx="table": the
    # antialias derivative and the aperture weight are the table path's
    kp, geom, axis, op, _ = _cases.case_setup(golden, "base")
    T, Dt = golden.tables()
    nz, nx, dz = geom["nz"], geom["nx"], geom["dz"]
    s = kd.Surrogate((0.0, 0.0, 0.0), (0.8, 0.4, 0.8), fmax=4.0, vref=1.5, zsrc=0.0, seed=9, vgrad=0.6,
                     residual_ms=1.0)
    p = s.get_params()
    p[sgo.OFF_WO:sgo.OFF_BO] *= 30.0
    s.set_params(p)
    ref_plan = kd.Plan(kp, kd.geometry(**geom))
    ref_plan.set_tables(T, Dt, T, Dt)
    for tx in ("network", "table"):
        plan = kd.Plan(kp, kd.geometry(**geom))
        plan.set_tables(T, Dt, T, Dt)
        plan.set_surrogate(s, s, angle="fd", tx=tx)
        net_plan = kd.Plan(kp, kd.geometry(**geom))
        net_plan.set_tables(T, Dt, T, Dt)
        net_plan.set_surrogate(s, s, angle="network", tx="network")
        for is_source, pos in ((1, 0.05), (0, 0.4133)):
            pos = float(np.float32(pos))
            gT, gTx, gphi, gw = (t.cpu().numpy().reshape(nx, nz) for t in kd.leg_fields_device(plan, is_source, pos))
            nT, nTx, _, nw = (t.cpu().numpy().reshape(nx, nz) for t in kd.leg_fields_device(net_plan, is_source, pos))
            rT, rTx, _, rw = (t.cpu().numpy().reshape(nx, nz) for t in kd.leg_fields_device(ref_plan, is_source, pos))
            assert np.array_equal(gT, nT)  # the same traveltime whichever quantities the network supplies
            assert np.abs(gT - rT).max() > 1e-4  # ... and not the table's
            ref_phi = _fd_direction(gT.astype(np.float64), kp.angle_grad_radius, kp.angle_smooth, dz, dz)
            nan = np.isnan(ref_phi)
            assert np.array_equal(np.isnan(gphi), nan)
            assert np.abs(np.angle(np.exp(1j * (gphi[~nan] - ref_phi[~nan])))).max() < 1e-9
            if tx == "table":
                assert np.array_equal(gTx, rTx) and np.array_equal(gw, rw)
            else:
                assert np.array_equal(gTx, nTx) and np.array_equal(gw, nw)
        plan.close()
        net_plan.close()
    ref_plan.close()
    s.close()


def test_surrogate_training_is_reproducible():
    # fixed-order gradient sums: two runs from the same seed give the same
    # parameters bit for bit
    import torch
    vol = torch.rand((6, 40, 30), device="cuda") + 0.5  # [npos][nx][nz]
    out = []
    for _ in range(2):
        s = kd.Surrogate((0.0, 0.0, 0.0), (1.0, 0.3, 0.4), fmax=3.0, vref=1.5, zsrc=0.0, seed=2, vgrad=0.6,
                         residual_ms=1.0)
        s.train(vol, 0.0, 0.2, 0.0, 0.01, 0.0, 0.01, 50, batch=1024, lr=1e-3, lr_final=1e-4, seed=4)
        out.append(s.get_params())
        s.close()
    assert np.array_equal(out[0], out[1])


def test_surrogate_leg_fields_match_eval(golden):
    # the persistent leg-field kernel (resident weights, per-leg xs features)
    # against the general evaluation kernel at the same points, and the
    # aperture weight against the table path's
    kp, geom, axis, op, _ = _cases.case_setup(golden, "base")
    T, Dt = golden.tables()
    nz, nx, dz = geom["nz"], geom["nx"], geom["dz"]
    lo, hi = (0.0, 0.0, 0.0), (0.8, 0.4, 0.8)
    s = kd.Surrogate(lo, hi, fmax=4.0, vref=1.5, zsrc=0.0, seed=9)
    p = s.get_params()
    p[sgo.OFF_WO:sgo.OFF_BO] *= 30.0
    s.set_params(p)
    plan = kd.Plan(kp, kd.geometry(**geom))
    plan.set_tables(T, Dt, T, Dt)
    ref_plan = kd.Plan(kp, kd.geometry(**geom))
    ref_plan.set_tables(T, Dt, T, Dt)
    plan.set_surrogate(s, s, angle="network")
    zz, xx = np.meshgrid(np.arange(nz) * dz, np.arange(nx) * dz)  # [nx][nz]
    for is_source, pos in ((1, 0.05), (0, 0.4133), (1, 0.7)):
        pos = float(np.float32(pos))
        gT, gTx, gphi, gw = (t.cpu().numpy() for t in kd.leg_fields_device(plan, is_source, pos))
        eT, exs, ez, ex = (t.cpu().double().numpy().reshape(nx, nz) for t in
                           s.eval(np.full(nx * nz, pos, np.float32), zz.ravel().astype(np.float32),
                                  xx.ravel().astype(np.float32)))
        gT, gTx, gphi, gw = (a.reshape(nx, nz) for a in (gT, gTx, gphi, gw))
        # the leg kernel folds the xs features into a per-leg bias (an FP32
        # GEMV) where the evaluation kernel runs them through the MMA: the two
        # agree except for BF16 rounding flips (tau off by <~1e-2, see above)
        scale = np.sqrt(np.mean(exs ** 2))
        T0 = np.maximum(np.hypot(xx - pos, zz) / 1.5, 1e-3)
        eT0 = np.abs(gT - eT) / T0
        assert np.median(eT0) < 1e-6 and np.percentile(eT0, 99) < 2e-3 and eT0.max() < 2e-2
        assert np.median(np.abs(gTx - exs)) < 1e-4 * scale and np.percentile(np.abs(gTx - exs), 99) < 1e-2 * scale
        # phi is NaN where the gradient vanishes (the source point itself)
        nan = np.isnan(gphi)
        assert np.all(np.hypot(ez, ex)[nan] < 1e-6)
        dphi = np.abs(np.angle(np.exp(1j * (gphi[~nan] - np.arctan2(ez, ex)[~nan]))))
        assert np.median(dphi) < 1e-5 and np.percentile(dphi, 99) < 1e-2
        _, _, _, rw = (t.cpu().numpy().reshape(nx, nz) for t in kd.leg_fields_device(ref_plan, is_source, pos))
        assert np.array_equal(gw, rw)
    plan.close()
    ref_plan.close()
    s.close()


def test_surrogate_training_gain_and_migration():
    # train on the v(z) 201x401 tables (GPU eikonal, 401 positions) and
    # migrate its gathers with the surrogate's traveltimes, every image judged
    # against the FP64 oracle of the table path.  What the network gains over
    # the method without it (the linear-gradient background alone), and what
    # the angle source costs: the network's own input gradient against the
    # finite-difference gradient of its traveltime (the tables' way).
    # Bounds from the measured sweep (40k steps: 0.98 us rms traveltime,
    # image 2.8e-3; the background alone 0.87 ms and 0.21).
    import torch
    import _cases
    import oracle
    from kirch_datuming_b200 import synth
    vel, T1, D1, data1, g = synth.vz_small_workload(seed=4)
    net = kd.Surrogate((0.0, 0.0, 0.0), (4.0, 2.0, 4.0), fmax=3.0, vref=1.5, zsrc=0.0, seed=1, vgrad=0.6,
                       residual_ms=1.0)
    losses = net.train(T1, 0.0, g.dp, 0.0, g.dz, 0.0, g.dx, 40000, batch=16384, lr=1e-3, lr_final=1e-5, seed=3)
    assert np.all(np.isfinite(losses)) and losses[-50:].mean() < 1e-3 * losses[:50].mean()
    bg = kd.Surrogate((0.0, 0.0, 0.0), (4.0, 2.0, 4.0), fmax=3.0, vref=1.5, zsrc=0.0, seed=1, vgrad=0.6,
                      residual_ms=1.0)
    p = bg.get_params()
    p[sgo.OFF_WO:] = 0.0  # T = the background alone
    bg.set_params(p)
    rng = np.random.default_rng(1)
    n = 50000
    ip, iz, ix = rng.integers(0, g.npos, n), rng.integers(0, g.nz, n), rng.integers(0, g.nx, n)
    Tt = T1[torch.from_numpy(ip).cuda(), torch.from_numpy(ix).cuda(), torch.from_numpy(iz).cuda()].cpu().numpy()
    pts = ((ip * g.dp).astype(np.float32), (iz * g.dz).astype(np.float32), (ix * g.dx).astype(np.float32))
    rms = lambda s: 1e6 * np.sqrt(np.mean((s.eval(*pts)[0].cpu().numpy() - Tt) ** 2))  # noqa: E731
    rms_net, rms_bg = rms(net), rms(bg)
    print("traveltime rms: network %.3f us, background %.1f us" % (rms_net, rms_bg))
    assert rms_net < 2.0 and rms_net < 0.01 * rms_bg

    f = lambda v: float(np.float32(v))  # noqa: E731
    gd = dict(nt=g.nt, nh=g.nh, ns=g.ns, t0=0.0, dt=f(g.dt), h0=f(g.h0), dh=f(g.dh), s0=0.0, ds=f(g.ds), nz=g.nz,
              nx=g.nx, z0=0.0, dz=f(g.dz), x0=0.0, dx=f(g.dx), sny=g.npos, sy0=0.0, sdy=f(g.dp), rny=g.npos,
              ry0=0.0, rdy=f(g.dp))
    geom = kd.geometry(**gd)
    kp = kd.params("cig=1", "mode=angle", "cmp=0", "angle_min=0", "angle_max=60", "angle_step=1", "angle_n=61",
                   "direct_mute=1", "direct_mute_slope=0.5", "direct_mute_intercept=0", "direct_mute_taper=0.05")
    Th, Dh = T1.cpu().numpy(), D1.cpu().numpy()
    o64 = oracle.migrate_adj(_cases.oracle_params(kp, gd, kd.output_axis(kp, geom)), data1.cpu().numpy(), Th, Dh,
                             Th, Dh, fp64=True)

    def image(sur, angle="fd", tx="network"):
        plan = kd.Plan(kp, geom)
        plan.set_tables(T1, D1, T1, D1)
        plan.set_surrogate(sur, sur, angle=angle, tx=tx)
        img = torch.zeros((plan.ng, g.nx, g.nz), device="cuda")
        plan.migrate(data1, img)
        plan.close()
        return oracle.rel_l2(img.cpu().numpy(), o64)

    r_net, r_tab, r_ang, r_bg = image(net), image(net, tx="table"), image(net, angle="network"), image(bg)
    print("image relL2 vs FP64 oracle: network %.2e, with table derivative %.2e, network angle %.2e, "
          "background %.2e" % (r_net, r_tab, r_ang, r_bg))
    assert r_net < 5e-3 and r_tab < 5e-3 and r_net < 0.05 * r_bg and r_ang > 5 * r_net
    net.close()
    bg.close()
