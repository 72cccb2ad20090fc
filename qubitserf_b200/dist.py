"""Multi-process plumbing for running the engine on several GPUs of one node.

One process per GPU (torchrun), the library bound to LOCAL_RANK through QSFB_DEVICE.
Codes are independent, so the data path has no collective: every rank certifies its own
share (or its own copy, for weak scaling) and only the timing is combined -- the max over
ranks, with a one-float all-reduce on a gloo group.
"""
from __future__ import annotations

import datetime
import os


def init_from_env(timeout_s: float = 600.0):
    """(rank, world, local_rank, group-or-None) from the torchrun environment."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        os.environ["QSFB_DEVICE"] = str(local)
        if not dist.is_initialized():
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=timeout_s))
        pg = dist
    else:
        os.environ.setdefault("QSFB_DEVICE", "0")
    return rank, world, local, pg


def max_over_ranks(pg, x: float) -> float:
    if pg is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, x: float) -> float:
    if pg is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def shard(items, rank: int, world: int):
    """Round-robin share of `items` for strong scaling (heavy codes spread over ranks)."""
    return items[rank::world]


def unshard(parts):
    """Inverse of shard(): parts[r] is rank r's share; returns the items in their order."""
    world = len(parts)
    out = [None] * sum(len(p) for p in parts)
    for r, part in enumerate(parts):
        out[r::world] = part
    return out


def gather_to_root(pg, obj, world: int):
    """Every rank's `obj`, in rank order, on rank 0 (None elsewhere); one gloo gather."""
    if pg is None:
        return [obj]
    out = [None] * world if pg.get_rank() == 0 else None
    pg.gather_object(obj, out, dst=0)
    return out
