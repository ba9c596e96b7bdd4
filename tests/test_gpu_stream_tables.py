"""Tables kept in host memory (KCIG_MEM_HOST_STREAM): every leg batch copies
only the slices it interpolates, so tables larger than the device memory can
be migrated.  The image must be the same, bit for bit, as with the tables on
the device at the same scratch budget (the budget sets the shot batching and
with it the FP32 accumulation order of the image) -- with a staging buffer
that holds the whole batch and with one so small (a tiny scratch budget)
that every leg or two is a group of its own."""
import os
import sys

import numpy as np
import pytest

import kirch_datuming_b200 as kd

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _cases  # noqa: E402

pytestmark = pytest.mark.gpu
GD = _cases.Golden()


def _image(case, stream, scratch=0, k2d=False):
    if k2d:
        kp, geom, axis, _ = _cases.k2d_setup(GD, case)
        data = GD.npz["data_" + GD.meta["k2d"][case]["data"]]
        use_grad = False
    else:
        kp, geom, axis, _, use_grad = _cases.case_setup(GD, case)
        data = GD.data(case)
    T, D = GD.tables()
    plan = kd.Plan(kp, kd.geometry(**geom), scratch_bytes=scratch)
    plan.set_tables(T, D, T, D, stream=stream)
    if use_grad:
        gx, gz = GD.grads()
        plan.set_gradients(gx, gz, gx, gz)
    img = np.zeros((axis[0], geom["nx"], geom["nz"]), np.float32)
    plan.migrate(np.ascontiguousarray(data, dtype=np.float32), img)
    plan.close()
    return img


@pytest.mark.parametrize("case", ["base", "cmp1_half", "options", "trace_aperture", "offset", "grads"])
def test_streamed_tables_equal_device_tables(case):
    np.testing.assert_array_equal(_image(case, stream=True), _image(case, stream=False))
    # a 300 KB budget stages two slices at a time
    np.testing.assert_array_equal(_image(case, stream=True, scratch=300 << 10),
                                  _image(case, stream=False, scratch=300 << 10))


def test_streamed_tables_kirchmig2d():
    ref = _image("k2d_trace_ap", stream=False, scratch=300 << 10, k2d=True)
    np.testing.assert_array_equal(_image("k2d_trace_ap", stream=True, scratch=300 << 10, k2d=True), ref)


def test_streamed_tables_leg_fields_and_prepared_path():
    kp, geom, axis, _, _ = _cases.case_setup(GD, "base")
    T, D = GD.tables()
    a = kd.Plan(kp, kd.geometry(**geom))
    a.set_tables(T, D, T, D)
    b = kd.Plan(kp, kd.geometry(**geom))
    b.set_tables(T, D, T, D, stream=True)
    for is_source, pos in ((1, 0.05), (0, 0.4133)):
        fa = [t.cpu().numpy() for t in kd.leg_fields_device(a, is_source, float(np.float32(pos)))]
        fb = [t.cpu().numpy() for t in kd.leg_fields_device(b, is_source, float(np.float32(pos)))]
        for x, y in zip(fa, fb):
            np.testing.assert_array_equal(x, y)
    a.close()
    b.close()
