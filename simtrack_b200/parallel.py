"""Multi-GPU plumbing: one process per GPU over torch.distributed.

Tracking shards with no data-path exchange: particles (and the (seed,
particle) units of a DA scan) are independent, so each rank tracks its own
contiguous share and the only collectives are the max of the per-rank device
times, sums of counts and the final gather of per-particle results.  Every
rank takes the same collective steps in the same order.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np


def shard_bounds(n: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous, balanced share [lo, hi) of n units for `rank` (sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def seeds_for_rank(seeds: Sequence[int], rank: int, world: int) -> List[int]:
    lo, hi = shard_bounds(len(seeds), rank, world)
    return list(seeds[lo:hi])


def _device_for(dist):
    import torch
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def reduce_scalar(value: float, op: str = "max") -> float:
    """All-reduce of one number ("max" or "sum") over the default group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device_for(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t[0])


def gather_concat(local: np.ndarray) -> np.ndarray:
    """Concatenation, in rank order, of every rank's 1-D or 2-D array (rows),
    returned on every rank.  Arrays may differ in length; dtype and trailing
    shape must agree."""
    import torch
    import torch.distributed as dist
    local = np.ascontiguousarray(local)
    if not (dist.is_available() and dist.is_initialized()):
        return local
    dev = _device_for(dist)
    world = dist.get_world_size()
    n = torch.tensor([local.shape[0]], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n)
    sizes = [int(s[0]) for s in sizes]
    mx = max(sizes)
    tail = local.shape[1:]
    buf = np.zeros((mx,) + tail, dtype=local.dtype)
    buf[:local.shape[0]] = local
    t = torch.from_numpy(buf).to(dev)
    outs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(outs, t)
    return np.concatenate([o.cpu().numpy()[:s] for o, s in zip(outs, sizes)], axis=0)
