"""The allocation-free leg-field entry point (kcig_leg_fields_noalloc) gives
the same fields as the allocating one (kcig_leg_fields_device).

It serves callers that cannot allocate device memory (an application that
owns the device's memory through its own allocator or budgets it exactly);
its scratch is a fixed array inside the library, limited to nz*nx <= 262144.
Both entry points run the same kernels on the same inputs, so their outputs
are compared bit for bit.  The cases cover every use of the scratch array:
the fused gradient kernel (no work planes), gradient volumes and a smoothing
radius too wide for the fused kernel (both go through the four FP64 work
planes at the end of the array), and a grid at the 262144-point limit.
This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

import _cases
import kirch_datuming_b200 as kd

pytestmark = pytest.mark.gpu


def _noalloc(kp, geom, T, D, is_source, pos, outs, stream, grads=None):
    L = kd.lib()
    f = L.kcig_leg_fields_noalloc
    f.argtypes = [ctypes.POINTER(kd.Params), ctypes.POINTER(kd.Geometry)] + [ctypes.c_void_p] * 4 + [
        ctypes.c_int, ctypes.c_double] + [ctypes.c_void_p] * 5
    g = kd.geometry(**geom)
    gx, gz = (None, None) if grads is None else (grads[0].data_ptr(), grads[1].data_ptr())
    rc = f(ctypes.byref(kp), ctypes.byref(g), T.data_ptr(), D.data_ptr(), gx, gz, int(is_source), float(pos),
           *[o.data_ptr() for o in outs], ctypes.c_void_p(stream))
    if rc != 0:
        raise kd.KcigError(rc, L.kcig_last_error().decode())


def _compare_two_calls(kp, geom, T, D, legs, grads=None):
    """Two calls in a row into the same outputs, each compared bit for bit
    with kcig_leg_fields_device on a plan holding the same tables."""
    import torch
    plan = kd.Plan(kp, kd.geometry(**geom))
    plan.set_tables(T, D, T, D)
    if grads is not None:
        plan.set_gradients(grads[0], grads[1], grads[0], grads[1])
    n = geom["nz"] * geom["nx"]
    stream = torch.cuda.current_stream().cuda_stream
    outs = [torch.full((n,), np.nan, dtype=dt, device="cuda")
            for dt in (torch.float64, torch.float32, torch.float64, torch.float32)]
    for is_source, pos in legs:
        _noalloc(kp, geom, T, D, is_source, pos, outs, stream, grads)
        ref = [x.cpu().numpy() for x in kd.leg_fields_device(plan, is_source, pos)]
        got = [x.cpu().numpy() for x in outs]
        for name, a, b in zip(("T", "Tx", "phi", "w"), got, ref):
            assert np.array_equal(a, b, equal_nan=True), name
        assert np.isfinite(got[0]).all() and np.isfinite(got[1]).all()
    plan.close()


@pytest.mark.parametrize("case,extra", [("base", ()), ("grads", ()), ("base", ("angle_smooth=12",))])
def test_noalloc_matches_allocating_entry_point_twice(case, extra):
    import torch
    gd = _cases.Golden()
    _, geom, _, _, use_grad = _cases.case_setup(gd, case)
    kp = kd.params(*gd.tokens(case), *extra)
    Th, Dh = gd.tables()
    T, D = torch.from_numpy(Th).cuda(), torch.from_numpy(Dh).cuda()
    grads = tuple(torch.from_numpy(x).cuda() for x in gd.grads()) if use_grad else None
    legs = ((1, float(np.float32(0.3133))), (0, float(np.float32(0.62))))
    _compare_two_calls(kp, geom, T, D, legs, grads)


def test_noalloc_at_its_point_limit_with_gradient_volumes():
    """512 x 512 = 262144 points, the largest grid the fixed scratch holds,
    with gradient volumes: the work planes reach the end of the layout."""
    import torch
    nz = nx = 512
    npos, d = 4, 0.01
    z = torch.arange(nz, dtype=torch.float64, device="cuda") * d
    x = torch.arange(nx, dtype=torch.float64, device="cuda") * d
    xs = torch.arange(npos, dtype=torch.float64, device="cuda") * 1.5
    # v(z) = 1.5 + 0.6 z traveltimes from surface sources, their source
    # derivative and spatial gradients (layout [npos][nx][nz])
    X = x[None, :, None] - xs[:, None, None]
    Z = z[None, None, :].expand(npos, nx, nz)
    v = 1.5 + 0.6 * Z
    arg = 1.0 + 0.36 * (X * X + Z * Z) / (2.0 * 1.5 * v)
    T = torch.acosh(arg) / 0.6
    dTdx = 0.6 * X / (1.5 * v * torch.sqrt(arg * arg - 1.0).clamp_min(1e-9))
    dT = -dTdx  # derivative with respect to the source position
    gx, gz = dTdx, torch.gradient(T, spacing=d, dim=2)[0]
    f32 = lambda a: a.float().contiguous()  # noqa: E731
    geom = dict(nt=10, nh=1, ns=1, t0=0.0, dt=0.004, h0=0.0, dh=0.0, s0=0.0, ds=0.0, nz=nz, nx=nx, z0=0.0,
                dz=float(np.float32(d)), x0=0.0, dx=float(np.float32(d)), sny=npos, sy0=0.0,
                sdy=float(np.float32(1.5)), rny=npos, ry0=0.0, rdy=float(np.float32(1.5)))
    kp = kd.params("cig=1", "mode=angle", "angle_min=0", "angle_max=60", "angle_step=1", "angle_n=61")
    legs = ((1, float(np.float32(2.2))), (0, float(np.float32(3.71))))
    _compare_two_calls(kp, geom, f32(T), f32(dT), legs, (f32(gx), f32(gz)))


def test_noalloc_rejects_grids_beyond_its_limit():
    import torch
    kp = kd.params("cig=1", "mode=angle")
    geom = dict(nt=10, nh=1, ns=1, dt=0.01, nz=600, nx=600, dz=0.01, dx=0.01, sny=2, sdy=0.01, rny=2, rdy=0.01)
    t = torch.zeros(1, device="cuda")
    with pytest.raises(kd.KcigError) as e:
        _noalloc(kp, geom, t, t, 1, 0.0, [t, t, t, t], 0)
    assert "allocation-free limit" in e.value.msg
