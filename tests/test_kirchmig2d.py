"""The plain tool kirchmig2d: the oracle's restatement (oracle_kirchmig2d_adj)
against the reference kirchmig2d's own images (tests/golden/golden_k2d.npz,
made by tests/golden/make_golden.py --kirchmig2d), and its parameter block.

The FP32 mirror build follows the reference's arithmetic and must agree to
rounding; the FP64 oracle differs where the reference's FP32 pick position
lands on a gate (a pick position of exactly the last sample in FP32 that is
just below it in FP64 drops a pick in the reference only), which bounds it at
1e-4 here."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
sys.path.insert(0, HERE)
import _cases  # noqa: E402
import oracle  # noqa: E402

GD = _cases.Golden()


@pytest.mark.parametrize("name", GD.k2d_cases)
def test_oracle_matches_reference_kirchmig2d(name):
    kp, geom, axis, op = _cases.k2d_setup(GD, name)
    T, D = GD.tables()
    data = GD.npz["data_" + GD.meta["k2d"][name]["data"]]
    ref = GD.k2d_image(name)
    u = _cases.ub_columns(GD, name)
    assert ref.shape[0] == axis[0]
    mirror = oracle.migrate_kirchmig2d(op, data, T, D, T, D, fp64=False)
    o64 = oracle.migrate_kirchmig2d(op, data, T, D, T, D, fp64=True)
    assert oracle.rel_l2(mirror[:, u:], ref[:, u:]) < 1e-6
    assert oracle.rel_l2(o64[:, u:], ref[:, u:]) < 1e-4


def test_kirchmig2d_params():
    import kirch_datuming_b200 as kd
    p = kd.params_kirchmig2d()
    assert (p.tool, p.adj, p.cig, p.cmp, p.isdiff, p.aperture_trace) == (1, 1, 0, 1, 0, -1)
    assert (p.aperture, p.antialias, p.tau, chr(p.interp_type)) == (90.0, 1.0, 0.0, "h")
    assert (p.direct_mute, p.cig_is_angle, p.aperture_taper, p.aperture_trace_taper) == (0, 0, 0.0, 0)
    p = kd.params_kirchmig2d("cig=1", "cmp=0", "type=partial", "aperture=30", "aperture_trace=5", "diff=1")
    assert (p.cig, p.cmp, chr(p.interp_type), p.aperture, p.aperture_trace, p.isdiff) == (1, 0, "p", 30.0, 5, 1)
    g = kd.geometry(nt=10, nh=7, ns=2, dt=0.001, h0=-0.3, dh=0.1, ds=0.1, nz=5, nx=5, dz=0.01, dx=0.01, sny=2,
                    sdy=0.1, rny=2, rdy=0.1)
    ng, g0, dg = kd.output_axis(p, g)
    assert ng == 7 and abs(g0 + 0.3) < 1e-7 and abs(dg - 0.1) < 1e-7
    with pytest.raises(kd.KcigError, match="Unknown interpolation type"):
        kd.params_kirchmig2d("type=cubic")
