"""Shot sharding of one survey over ranks (gloo, CPU): each rank migrates its
block of shots at their positions in the whole survey (the oracle standing in
for the GPU engine) and one all-reduce sums the images; the result equals the
single-process migration of all shots.  The shot positions a rank's plan uses
(kcig_shot_positions, host code of the library) are the whole survey's, bit
for bit."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from kirch_datuming_b200 import shard


def test_shot_slices_cover_and_balance():
    for ns in (1, 5, 64, 401):
        for world in (1, 2, 3, 8):
            sl = [shard.shot_slice(ns, r, world) for r in range(world)]
            assert sl[0].start == 0 and sl[-1].stop == ns
            assert all(a.stop == b.start for a, b in zip(sl, sl[1:]))
            sizes = [s.stop - s.start for s in sl]
            assert max(sizes) - min(sizes) <= 1


def test_shot_ranges_keep_the_survey_positions_bit_for_bit():
    import kirch_datuming_b200 as kd
    g = kd.geometry(nt=10, nh=3, ns=400, dt=0.001, s0=0.0, ds=float(np.float32(0.04)), nz=5, nx=5, dz=0.01,
                    dx=0.01, sny=2, sdy=0.01, rny=2, rdy=0.01)
    full64, full32 = kd.shot_positions(g)
    moved = 0
    for world in (2, 3, 8):
        parts = [kd.shot_positions(g, *shard.shot_range(400, r, world)) for r in range(world)]
        assert np.array_equal(np.concatenate([p[0] for p in parts]), full64)
        assert np.array_equal(np.concatenate([p[1] for p in parts]), full32)
        for r in range(world):
            # a rank re-based as a survey of its own rounds its positions differently
            sg = shard.shard_geometry(dict(ns=400, s0=0.0, ds=g.ds), r, world)
            first, count = shard.shot_range(400, r, world)
            pf = np.float32(sg["s0"]) + np.arange(count, dtype=np.float32) * np.float32(sg["ds"])
            moved += int((pf != full32[first:first + count]).sum())
    assert moved > 0
    with pytest.raises(kd.KcigError):
        kd.shot_positions(g, 390, 20)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle"), os.path.join(root, "tests")):
        sys.path.insert(0, p)
    import _cases
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        gd = _cases.Golden()
        kp, geom, axis, op, _ = _cases.case_setup(gd, "base")
        first, count = shard.shot_range(geom["ns"], rank, world)
        # this rank's shots at their survey positions: the whole survey's
        # geometry with the other ranks' traces left out (zero traces add
        # exactly nothing)
        data = np.zeros_like(gd.data("base"))
        data[first:first + count] = gd.data("base")[first:first + count]
        T, D = gd.tables()
        part = oracle.migrate_adj(op, data, T, D, T, D)
        img = torch.from_numpy(part)
        shard.reduce_image(img)
        if rank == 0:
            np.save(out, img.numpy())
    finally:
        dist.destroy_process_group()


def test_two_rank_shot_sharding_equals_single_process(tmp_path, golden):
    import _cases
    import oracle
    out = str(tmp_path / "img.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn")
    img = np.load(out)
    full = _cases.oracle_image(golden, "base")
    # the same pairs summed in another order (FP64): equal to rounding
    assert oracle.rel_l2(img, full) < 1e-12
