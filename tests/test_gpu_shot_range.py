"""Shot ranges of one survey (kcig_plan_set_shot_range), the per-rank work of
the shot-sharded multi-GPU migration, run one after another on one GPU: the
ranges' images add up to the whole survey's image, and each range matches the
FP64 oracle run on the whole survey with the other shots' traces zeroed."""
import numpy as np
import pytest

import _cases
import kirch_datuming_b200 as kd
import oracle
from kirch_datuming_b200 import shard

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case,world", [("base", 2), ("base", 3), ("cmp1_half", 2)])
def test_shot_ranges_add_up_to_the_survey(golden, case, world):
    import torch
    kp, geom, axis, op, _ = _cases.case_setup(golden, case)
    T, D = golden.tables()
    data = np.ascontiguousarray(golden.data(case))
    dT, dD = torch.from_numpy(T).cuda(), torch.from_numpy(D).cuda()
    shape = (axis[0], geom["nx"], geom["nz"])

    def run(first=0, count=-1):
        plan = kd.Plan(kp, kd.geometry(**geom))
        plan.set_tables(dT, dD, dT, dD)
        plan.set_shot_range(first, count)
        img = torch.zeros(shape, dtype=torch.float32, device="cuda")
        sub = data if count < 0 else data[first:first + count]
        plan.migrate(torch.from_numpy(np.ascontiguousarray(sub)).cuda(), img)
        plan.close()
        return img.cpu().numpy().astype(np.float64)

    full = run()
    parts = []
    for r in range(world):
        first, count = shard.shot_range(geom["ns"], r, world)
        img = run(first, count)
        masked = np.zeros_like(data)
        masked[first:first + count] = data[first:first + count]
        ref = oracle.migrate_adj(op, masked, T, D, T, D, fp64=True)
        assert oracle.rel_l2(img, ref) <= 1e-5
        parts.append(img)
    # the same pairs, accumulated per range in FP32 and then summed
    assert oracle.rel_l2(sum(parts), full) <= 1e-6


def test_shot_range_rejects_shots_outside_the_survey(golden):
    kp, geom, _, _, _ = _cases.case_setup(golden, "base")
    plan = kd.Plan(kp, kd.geometry(**geom))
    with pytest.raises(kd.KcigError):
        plan.set_shot_range(geom["ns"] - 1, 2)
    with pytest.raises(kd.KcigError):
        plan.set_shot_range(-1, 1)
    plan.set_shot_range(0, -1)
    plan.close()
