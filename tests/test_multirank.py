"""Shot sharding over 2 ranks (gloo, CPU): each rank migrates its block of
shots (with the oracle standing in for the GPU engine) and one all-reduce sums
the images; the result equals the single-process migration of all shots."""
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
        kp, geom, axis, _, _ = _cases.case_setup(gd, "base")
        g = shard.shard_geometry(geom, rank, world)
        sl = shard.shot_slice(geom["ns"], rank, world)
        op = _cases.oracle_params(kp, g, axis)
        T, D = gd.tables()
        part = oracle.migrate_adj(op, np.ascontiguousarray(gd.data("base")[sl]), T, D, T, D)
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
    # a rank's shot axis starts at s0 + start*ds, so its positions round
    # differently in FP32 than s0 + is*ds: equal to the parity tolerance
    assert oracle.rel_l2(img, full) < 1e-5
