"""Multi-GPU plumbing: one process per GPU.

Two forms:
  * independent units (windows, requests, R/S pairs): N GPUs run N shards of
    the units with no data-path collective (weak scaling); afterwards the step
    time of the job is the maximum over ranks and match counts and checksums
    add up over ranks (exact: both are sums mod 2^64);
  * one join over N GPUs (sharded_join): every rank splits its share of R and
    S by the destination rank of each key (adb_shard_split on the device), one
    all-to-all of each relation moves the parts, every rank joins what it
    received (all tuples of its keys), and one all-reduce adds the (count,
    checksum) pairs.  The exchange and the reduction are the only collectives.
torch.distributed carries them (NCCL on GPUs, gloo in the CPU tests).
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


def shard_of(keys, parts: int):
    """Destination rank of each key: (key * 0x9E3779B1 mod 2^32) * parts / 2^32
    (the rule of adb_shard_split)."""
    k = np.asarray(keys, dtype=np.uint64)
    h = (k * np.uint64(0x9E3779B1)) & np.uint64(0xFFFFFFFF)
    return ((h * np.uint64(parts)) >> np.uint64(32)).astype(np.int64)


def exchange(send, counts, device=None):
    """All-to-all of a tensor grouped by destination rank (counts[p] elements
    for rank p, in rank order): returns the elements every rank sent here, in
    source-rank order."""
    import torch
    import torch.distributed as dist
    c = torch.tensor([int(x) for x in counts], dtype=torch.int64, device=device)
    rc = torch.empty_like(c)
    dist.all_to_all_single(rc, c)
    recv_counts = [int(x) for x in rc.tolist()]
    recv = torch.empty(sum(recv_counts), dtype=send.dtype, device=send.device)
    dist.all_to_all_single(recv, send, recv_counts, [int(x) for x in counts])
    return recv


def sharded_join_with(R_local, S_local, split, join, device=None):
    """One join over the ranks of the default process group.

    R_local / S_local: this rank's share of each relation (tensors of 64-bit
    tuple words); split(T, parts) -> (T grouped by destination rank, counts);
    join(R, S) -> (count, checksum) of the tuples this rank received.  Returns
    the (count, checksum) of the whole join, equal on every rank."""
    import torch.distributed as dist
    world = dist.get_world_size() if dist.is_initialized() else 1
    Rg, rc = split(R_local, world)
    Sg, sc = split(S_local, world)
    if dist.is_initialized():   # (one rank: the collectives run and copy the parts to themselves)
        Rg = exchange(Rg, rc, device)
        Sg = exchange(Sg, sc, device)
    cnt, ck = join(Rg, Sg)
    return sum_results(cnt, ck, device)


def sharded_join(algo: str, dR, dS, params=None):
    """sharded_join_with on the GPU: dR / dS are this rank's shares as int64
    CUDA tensors; the split is adb_shard_split, the local join adb_join_device
    (algo = any lazy join name) on this rank's device."""
    import ctypes as C
    import torch
    import alliancedb_b200 as adb
    dev = dR.device
    stream = adb.stream_handle(torch.cuda.current_stream(dev))   # where NCCL's results are ordered

    def split(T, parts):
        out = torch.empty_like(T)
        counts = (C.c_uint64 * parts)()
        adb._check(adb.lib().adb_shard_split(T.data_ptr() if T.numel() else None, T.numel(), parts,
                                             out.data_ptr() if T.numel() else None, counts, stream))
        return out, [int(x) for x in counts]

    def join(R, S):
        r = adb.join_device(algo, R.data_ptr() if R.numel() else 0, R.numel(), S.data_ptr() if S.numel() else 0,
                            S.numel(), params, stream)
        return r.count, r.checksum

    return sharded_join_with(dR, dS, split, join, dev)
