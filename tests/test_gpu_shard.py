"""The split step of one join sharded over several GPUs (adb_shard_split),
and the sharded path itself on the one GPU of this run.

* every part of the split holds exactly the tuples whose key is bound for it,
  by the rule (key * 0x9E3779B1 mod 2^32) * parts / 2^32 restated in numpy;
* the sharded join through a one-rank NCCL process group (split, the
  all-to-all of both relations, local join, all-reduce: the real collective
  calls, each rank being its own peer) equals the plain join and the oracle.
The two-rank exchange logic itself runs on CPU over gloo (tests/test_dist.py).
"""
import ctypes as C
import datetime
import socket

import numpy as np
import pytest

import alliancedb_b200 as adb
from alliancedb_b200.dist import shard_of

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("parts", [1, 2, 3, 8, 32])
@pytest.mark.parametrize("n", [0, 1, 1000, (1 << 20) + 7])
def test_split_parts_hold_their_keys(parts, n):
    import torch
    R = adb.gen_uniform(n, max(1, 3 * n), 11) if n else np.zeros(0, dtype=adb.TUPLE)
    w = R.view(np.uint64)
    dev = torch.device("cuda", 0)
    d_in = torch.from_numpy(w.view(np.int64).copy()).to(dev)
    d_out = torch.empty_like(d_in)
    counts = (C.c_uint64 * parts)()
    stream = adb.stream_handle(torch.cuda.current_stream(dev))   # the stream that wrote d_in
    st = adb.lib().adb_shard_split(d_in.data_ptr() if n else None, n, parts, d_out.data_ptr() if n else None, counts,
                                   stream)
    assert st == 0, adb.lib().adb_last_error().decode()
    out = d_out.cpu().numpy().view(np.uint64)
    dst = shard_of(w >> np.uint64(32), parts)
    off = 0
    for p in range(parts):
        seg = out[off:off + counts[p]]
        assert counts[p] == int((dst == p).sum())
        assert np.array_equal(np.sort(seg), np.sort(w[dst == p]))
        off += counts[p]
    assert off == n


def test_split_rejects_bad_parts():
    counts = (C.c_uint64 * 64)()
    assert adb.lib().adb_shard_split(None, 0, 33, None, counts, None) == adb.ADB_ERR_ARG
    assert adb.lib().adb_shard_split(None, 0, 0, None, counts, None) == adb.ADB_ERR_ARG


@pytest.mark.parametrize("algo", ["PRO", "NPO", "m-way"])
def test_sharded_join_one_rank_nccl(oracle, algo):
    import torch
    import torch.distributed as dist
    from alliancedb_b200.dist import sharded_join
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        R = adb.gen_pk(1 << 18, 21)
        S = adb.gen_fk((1 << 18) + 5, R, 0.8, 22)
        dR = torch.from_numpy(R.view(np.int64).copy()).to(dev)
        dS = torch.from_numpy(S.view(np.int64).copy()).to(dev)
        got = sharded_join(algo, dR, dS)
        want = oracle.truth(R, S)
        assert got == want
        plain = adb.join(algo, R, S)
        assert (plain.count, plain.checksum) == want
    finally:
        dist.destroy_process_group()
