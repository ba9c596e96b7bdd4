"""Shot sharding of one survey over ranks (one process per GPU).

The migrated image is a sum over traces, so a survey split by shots over
ranks gives the full image after one sum-reduction of the per-rank images --
the only exchange step of the path.  Works with any torch.distributed backend
(NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations


def shot_slice(ns: int, rank: int, world: int) -> slice:
    """Contiguous, balanced block of shots for `rank` (sizes differ by <= 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(ns, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def shot_range(ns: int, rank: int, world: int) -> tuple:
    """(first, count) of this rank's shots, for Plan.set_shot_range: the rank
    keeps the whole survey's geometry, so its shots sit at exactly the
    positions (and antialias spacing) a single-process run gives them."""
    sl = shot_slice(ns, rank, world)
    return sl.start, sl.stop - sl.start


def shard_geometry(geom: dict, rank: int, world: int) -> dict:
    """Geometry of this rank's shots as a survey of its own: the shot axis
    origin moves to the first shot and the spacing stays.  Positions are then
    re-derived from the new origin and can round differently in FP32 from the
    whole survey's; Plan.set_shot_range with shot_range() avoids that."""
    sl = shot_slice(geom["ns"], rank, world)
    g = dict(geom)
    g["ns"] = sl.stop - sl.start
    g["s0"] = float(geom["s0"] + sl.start * (geom["ds"] if geom["ns"] > 1 else 0.0))
    return g


def reduce_image(image, group=None):
    """Sum the ranks' partial images in place (torch tensor)."""
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(image, op=dist.ReduceOp.SUM, group=group)
    return image
