"""Multi-GPU by replicas: one process per GPU, each running its own streams.

The path has no cross-stream exchange (all state is per stream; the only
global coupling is the per-frame threshold inside one stream), so N GPUs
serve N disjoint sets of streams and nothing crosses NVLink on the data
path.  The process group carries only the measurement: each rank's pixel
count and device time, reduced once at the end (sum of pixels, max of time).
"""
from __future__ import annotations

import datetime
import os


def shard(items, rank: int, world: int):
    """The streams rank `rank` of `world` serves (round-robin, disjoint)."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    return list(items)[rank::world]


def init(backend: str, timeout_s: float = 120.0):
    """Joins the job's process group (torchrun's env:// variables); None when
    the job has one rank.  A short timeout turns a rank that died into an
    error on the others' next collective instead of a hang."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world <= 1:
        return None
    import torch.distributed as dist
    dist.init_process_group(backend, init_method="env://",
                            timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def aggregate(pixels: float, ms: float, dist=None, device=None):
    """(total pixels over ranks, max time over ranks in ms, Mpix-frames/s)."""
    if dist is None:
        return pixels, ms, pixels / (ms * 1e-3) / 1e6
    import torch
    p = torch.tensor([float(pixels)], dtype=torch.float64, device=device)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(p, op=dist.ReduceOp.SUM)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    tp, tm = float(p[0]), float(t[0])
    return tp, tm, tp / (tm * 1e-3) / 1e6
