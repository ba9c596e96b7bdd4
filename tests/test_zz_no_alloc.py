"""The allocation-free leg-field entry point (kcig_leg_fields_noalloc) gives
the same fields as the allocating one (kcig_leg_fields_device).

It serves callers that cannot allocate device memory (an application that
owns the device's memory through its own allocator or budgets it exactly);
its scratch is a fixed array inside the library, limited to nz*nx <= 262144.
This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

import _cases
import kirch_datuming_b200 as kd

pytestmark = pytest.mark.gpu


def _noalloc(kp, geom, T, D, is_source, pos, outs, stream):
    L = kd.lib()
    f = L.kcig_leg_fields_noalloc
    f.argtypes = [ctypes.POINTER(kd.Params), ctypes.POINTER(kd.Geometry)] + [ctypes.c_void_p] * 4 + [
        ctypes.c_int, ctypes.c_double] + [ctypes.c_void_p] * 5
    g = kd.geometry(**geom)
    rc = f(ctypes.byref(kp), ctypes.byref(g), T.data_ptr(), D.data_ptr(), None, None, int(is_source), float(pos),
           *[o.data_ptr() for o in outs], ctypes.c_void_p(stream))
    if rc != 0:
        raise kd.KcigError(rc, L.kcig_last_error().decode())


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    gd = _cases.Golden()
    kp, geom, _, _, _ = _cases.case_setup(gd, "base")
    Th, Dh = gd.tables()
    T, D = torch.from_numpy(Th).cuda(), torch.from_numpy(Dh).cuda()
    plan = kd.Plan(kp, kd.geometry(**geom))
    plan.set_tables(T, D, T, D)
    n = geom["nz"] * geom["nx"]
    stream = torch.cuda.current_stream().cuda_stream
    # two calls in a row, a source and then a receiver leg, into the same outputs
    outs = [torch.full((n,), np.nan, dtype=dt, device="cuda")
            for dt in (torch.float64, torch.float32, torch.float64, torch.float32)]
    for is_source, pos in ((1, float(np.float32(0.3133))), (0, float(np.float32(0.62)))):
        _noalloc(kp, geom, T, D, is_source, pos, outs, stream)
        ref = [x.cpu().numpy() for x in kd.leg_fields_device(plan, is_source, pos)]
        got = [x.cpu().numpy() for x in outs]
        assert np.allclose(got[0], ref[0], rtol=1e-12, atol=1e-12)       # T
        assert np.allclose(got[1], ref[1], rtol=1e-6, atol=1e-6)         # Tx
        ok = ~np.isnan(ref[2])
        assert np.array_equal(np.isnan(got[2]), ~ok)                     # phi
        assert np.abs(np.angle(np.exp(1j * (got[2][ok] - ref[2][ok])))).max() < 1e-9
        assert np.allclose(got[3], ref[3], rtol=1e-6, atol=1e-6)         # w
    plan.close()


def test_noalloc_rejects_grids_beyond_its_limit():
    import torch
    kp = kd.params("cig=1", "mode=angle")
    geom = dict(nt=10, nh=1, ns=1, dt=0.01, nz=600, nx=600, dz=0.01, dx=0.01, sny=2, sdy=0.01, rny=2, rdy=0.01)
    t = torch.zeros(1, device="cuda")
    with pytest.raises(kd.KcigError) as e:
        _noalloc(kp, geom, t, t, 1, 0.0, [t, t, t, t], 0)
    assert "allocation-free limit" in e.value.msg
