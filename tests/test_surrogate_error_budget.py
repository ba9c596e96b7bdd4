"""What a traveltime surrogate must reproduce to stay within 1e-3 relative L2
of the table path's FP64 image (FP64 oracle on the 41x81 v(z) fixtures, no
GPU).  These are properties of the summation, independent of any network:

* a coherent traveltime error of 1 us already costs ~2.4e-4 of image relative
  L2 (10 us: ~2.4e-3) -- the surrogate's traveltime must be good to a few us;
* the antialias width uses eikods2d's tds1 (the source-position derivative
  its marching recursion computes).  The central difference of the same
  tables across neighbouring positions differs from tds1 by a few percent
  (it carries the tables' grid-scale noise from position to position) and
  moves the image by more than 1e-3 -- a surrogate's own derivative must
  follow tds1, not that difference (a smooth network's derivative does: on
  the GPU it gives the same image error as tds1 itself);
* the scattering angle comes from the finite-difference gradient of the
  traveltime with triangle smoothing.  Taking it from the exact eikonal
  gradient (eikods2d's gradient volumes) instead moves the image by more than
  1e-2 -- so a surrogate must form its angle from its traveltime field the
  way the tables do, not from its analytic input gradient.
"""
import numpy as np

import _cases
import oracle


def _setup(gd, case="base"):
    kp, geom, axis, op, _ = _cases.case_setup(gd, case)
    T, D = gd.tables()
    return kp, geom, axis, op, T, D, gd.data(case)


def test_coherent_traveltime_error_sensitivity(golden):
    _, _, _, op, T, D, data = _setup(golden)
    ref = oracle.migrate_adj(op, data, T, D, T, D)
    for dt_s, lo, hi in ((1e-6, 1e-4, 5e-4), (1e-5, 1e-3, 5e-3)):
        Ts = (T.astype(np.float64) + dt_s).astype(np.float32)
        err = oracle.rel_l2(oracle.migrate_adj(op, data, Ts, D, Ts, D), ref)
        assert lo < err < hi, (dt_s, err)


def test_source_derivative_of_the_traveltime_is_not_tds1(golden):
    _, _, _, op, T, D, data = _setup(golden)
    t = golden.meta["table"]
    npos, dp = t["n"][2], t["d"][2]
    T3 = T.reshape(npos, golden.nx, golden.nz).astype(np.float64)
    Dfd = np.empty_like(T3)
    Dfd[1:-1] = (T3[2:] - T3[:-2]) / (2 * dp)
    Dfd[0], Dfd[-1] = (T3[1] - T3[0]) / dp, (T3[-1] - T3[-2]) / dp
    Dfd = Dfd.astype(np.float32).ravel()
    assert np.linalg.norm(Dfd - D) / np.linalg.norm(D) > 1e-2
    ref = oracle.migrate_adj(op, data, T, D, T, D)
    assert oracle.rel_l2(oracle.migrate_adj(op, data, T, Dfd, T, Dfd), ref) > 1e-3


def test_angle_from_the_exact_gradient_is_not_the_tables_angle(golden):
    kp, geom, axis, op, T, D, data = _setup(golden)
    ref = oracle.migrate_adj(op, data, T, D, T, D)
    gx, gz = golden.grads()
    opg = _cases.oracle_params(kp, geom, axis, use_grad=True)
    img = oracle.migrate_adj(opg, data, T, D, T, D, grads=(gx, gz, gx, gz))
    assert oracle.rel_l2(img, ref) > 1e-2
