"""Multi-GPU plumbing: one process per GPU, no data-path collective.

The join hot path partitions naturally into independent units (windows, or
R/S pairs), so N GPUs run N independent shards of the units (weak scaling);
the only cross-rank steps are bookkeeping after the timed work:
  * the step time of the job is the maximum over ranks;
  * match counts and checksums add up over ranks (exact: both are sums mod 2^64).
torch.distributed carries these (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import numpy as np


def shard(n_units: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous unit range [lo, hi) of `rank` out of `world` (sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world")
    base, extra = divmod(n_units, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def max_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_results(count: int, checksum: int, device=None) -> tuple[int, int]:
    """Adds (count, checksum) over ranks modulo 2^64."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return int(count), int(checksum)
    as_i64 = np.array([count, checksum], dtype=np.uint64).view(np.int64)
    t = torch.tensor(as_i64, dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)   # two's-complement wrap == mod 2^64
    out = t.cpu().numpy().view(np.uint64)
    return int(out[0]), int(out[1])
