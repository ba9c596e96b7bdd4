"""The GPU table generator against the closed-form first-arrival time of a
linear-gradient medium v(z) = v0 + g z (source at the surface):
    T = arccosh(1 + g^2 r^2 / (2 v0 v(z))) / g,  r^2 = (x - xs)^2 + z^2."""
import numpy as np
import pytest

import kirch_datuming_b200 as kd
from kirch_datuming_b200 import synth

pytestmark = pytest.mark.gpu


def analytic(nz, nx, dz, xs, v0=1.5, g=0.6):
    z = np.arange(nz) * dz
    x = np.arange(nx) * dz
    zz, xx = np.meshgrid(z, x)  # [nx][nz]
    r2 = (xx - xs) ** 2 + zz ** 2
    v = v0 + g * zz
    return np.arccosh(1.0 + g * g * r2 / (2.0 * v0 * v)) / g


def test_eikonal_linear_vz_accuracy():
    import torch
    nz, nx, dz = 121, 241, 0.01
    vel = torch.from_numpy(synth.velocity_linear_vz(nz, nx, dz)).cuda()
    npos, p0, dp = 5, 0.4, 0.35
    T, D = kd.eikonal_tables(vel, dz, dz, npos, p0, dp)
    T = T.cpu().numpy()
    # the relative error of the upwind update is largest beside the (b1=b2=2)
    # source box and decays with distance
    z, x = np.arange(nz) * dz, np.arange(nx) * dz
    zz, xx = np.meshgrid(z, x)
    for j in range(npos):
        xs = p0 + j * dp
        ref = analytic(nz, nx, dz, xs)
        far = ref > 0.05
        rel = np.abs(T[j] - ref) / np.maximum(ref, 1e-9)
        assert rel[far].max() < 0.05, rel[far].max()
        assert rel[far].mean() < 0.012, rel[far].mean()
        assert rel[np.hypot(xx - xs, zz) > 0.3].max() < 0.03
    # the position derivative follows dT/dxs = -(x - xs) p(xs) (horizontal slowness at the source)
    D = D.cpu().numpy()
    assert np.all(np.isfinite(D))
    mid = D[2]
    assert mid[0, 5] > 0 and mid[-1, 5] < 0  # left of the source times grow as the source moves right


def test_eikonal_tables_feed_the_migration():
    # tables from the generator migrate a flat-reflector gather into an image
    # whose strongest depth row is the reflector's
    import torch
    nz, nx, dz = 81, 161, 0.01
    vel = torch.from_numpy(synth.velocity_linear_vz(nz, nx, dz)).cuda()
    npos, dp = 41, 0.04
    T, D = kd.eikonal_tables(vel, dz, dz, npos, 0.0, dp)
    g = synth.Geometry(nz=nz, nx=nx, dz=dz, dx=dz, z0=0, x0=0, ns=9, s0=0.2, ds=0.16, nh=41, h0=0.0, dh=dp, cmp=0,
                       nt=501, dt=0.002, t0=0.0, npos=npos, p0=0.0, dp=dp)
    data = synth.shot_gathers(T, g, [(np.full(nx, 50), 0.2)], 20.0, seed=3, snr_amp=1e6)
    kp = kd.params("cig=1", "mode=angle", "cmp=0", "angle_min=0", "angle_max=60", "angle_step=2", "angle_n=31")
    geom = dict(nt=501, nh=41, ns=9, t0=0.0, dt=0.002, h0=0.0, dh=dp, s0=0.2, ds=0.16, nz=nz, nx=nx, z0=0.0,
                dz=dz, x0=0.0, dx=dz, sny=npos, sy0=0.0, sdy=dp, rny=npos, ry0=0.0, rdy=dp)
    plan = kd.Plan(kp, kd.geometry(**{k: float(np.float32(v)) if isinstance(v, float) else v
                                      for k, v in geom.items()}))
    plan.set_tables(T, D, T, D)
    img = torch.zeros((plan.ng, nx, nz), device="cuda")
    plan.migrate(data.contiguous(), img)
    stack = img.sum(0).abs().cpu().numpy()  # [nx][nz]
    prof = stack[40:120].sum(0)
    assert abs(int(np.argmax(prof)) - 50) <= 2
