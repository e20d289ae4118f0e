"""The N > 1 host path with world size 2 over gloo, on CPU: each rank joins its
shard of the windows (with the CPU oracle standing in for the device, since no
GPU is used here), then the ranks combine results and take the max time; the
combined result must equal the single-process result."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from alliancedb_b200.dist import shard


def test_shard_covers_units_once():
    for n in (0, 1, 7, 4096):
        for world in (1, 2, 3, 8):
            ranges = [shard(n, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
            sizes = [hi - lo for lo, hi in ranges]
            assert max(sizes) - min(sizes) <= 1


def _windows(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for w in range(n):
        nr, ns = int(rng.integers(1, 400)), int(rng.integers(1, 400))
        kr = int(rng.integers(1, 200))
        R = np.empty(nr, dtype=[("payload", "<u4"), ("key", "<u4")])
        S = np.empty(ns, dtype=R.dtype)
        R["key"], R["payload"] = rng.integers(0, kr, nr), np.arange(nr)
        S["key"], S["payload"] = rng.integers(0, kr, ns), np.arange(ns)
        out.append((R, S))
    return out


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import torch.distributed as dist
    from alliancedb_b200.dist import max_over_ranks, shard, sum_results
    from tests.oracle_bind import Oracle
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        wins = _windows(24, 5)
        lo, hi = shard(len(wins), rank, world)
        o = Oracle()
        cnt, ck = 0, 0
        for R, S in wins[lo:hi]:
            c, k = o.truth(R, S)
            cnt += c
            ck = (ck + k) % (1 << 64)
        tot = sum_results(cnt, ck)
        tmax = max_over_ranks(1.0 + rank)
        q.put((rank, tot, tmax))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_gloo_combine_equals_single():
    from tests.oracle_bind import Oracle
    o = Oracle()
    want_c, want_k = 0, 0
    for R, S in _windows(24, 5):
        c, k = o.truth(R, S)
        want_c += c
        want_k = (want_k + k) % (1 << 64)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, tot, tmax in got:
        assert tot == (want_c, want_k)
        assert tmax == 2.0


def _split_np(T, parts):
    """The split of adb_shard_split, restated with numpy on the CPU."""
    import torch
    from alliancedb_b200.dist import shard_of
    w = T.numpy().view(np.uint64)
    dst = shard_of(w >> np.uint64(32), parts)
    order = np.argsort(dst, kind="stable")
    counts = np.bincount(dst, minlength=parts)
    return torch.from_numpy(w[order].view(np.int64).copy()), [int(c) for c in counts]


def _sharded_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import torch
    import torch.distributed as dist
    import alliancedb_b200 as adb
    from alliancedb_b200.dist import shard, shard_of, sharded_join_with
    from tests.oracle_bind import Oracle
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        o = Oracle()
        R = adb.gen_uniform(30011, 9000, 71).view(np.int64)
        S = adb.gen_uniform(25013, 9000, 72).view(np.int64)
        rl, rh = shard(len(R), rank, world)
        sl, sh = shard(len(S), rank, world)
        seen = []

        def join(Rr, Sr):
            Rw, Sw = Rr.numpy().view(np.uint64), Sr.numpy().view(np.uint64)
            seen.append((len(Rw), len(Sw), bool((shard_of(Rw >> np.uint64(32), world) == rank).all() and
                                                (shard_of(Sw >> np.uint64(32), world) == rank).all())))
            return o.truth(Rw, Sw)

        tot = sharded_join_with(torch.from_numpy(R[rl:rh].copy()), torch.from_numpy(S[sl:sh].copy()), _split_np,
                                join)
        q.put((rank, tot, *seen[0]))
    finally:
        dist.destroy_process_group()


def test_sharded_join_two_ranks_equals_single_join(oracle):
    """One join over two gloo ranks: split by destination, all-to-all, local
    joins (the oracle stands in for the device), all-reduce -- equals the join
    of the whole relations on both ranks, and every tuple reaches exactly the
    rank its key is bound for."""
    import alliancedb_b200 as adb
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    R = adb.gen_uniform(30011, 9000, 71)
    S = adb.gen_uniform(25013, 9000, 72)
    want = oracle.truth(R, S)
    assert all(r[1] == want for r in res)
    assert sum(r[2] for r in res) == len(R) and sum(r[3] for r in res) == len(S)
    assert all(r[4] for r in res)
