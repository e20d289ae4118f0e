"""Eager stream joins (SHJ_*, PMJ_*) on the B200 against the CPU oracle.

The reference's own check for these joins is that every distribution model
returns the same count on the same input (all twelve SHJ/PMJ variants agree);
here count and checksum must also equal the oracle's restatement of SHJ and
PMJ, bit for bit, for every model, batch size and window.
"""
import numpy as np
import pytest

import alliancedb_b200 as adb

pytestmark = pytest.mark.gpu

EAGER = ["SHJ_st", "SHJ_JM_P", "SHJ_JM_NP", "SHJ_JB_NP", "SHJ_JBCR_NP", "SHJ_JBCR_P", "SHJ_HS_NP",
         "PMJ_st", "PMJ_JM_NP", "PMJ_JM_P", "PMJ_JB_NP", "PMJ_JB_P", "PMJ_JBCR_NP", "PMJ_JBCR_P", "PMJ_HS_NP"]


def dup_streams(n, key_range, dup, seed):
    """Relations whose keys are drawn, then materialised `dup` times and shuffled
    (the reference's duplicate(), hashing/utils/generator.cpp:518-542)."""
    rng = np.random.default_rng(seed)
    base = rng.integers(1, key_range + 1, size=n // dup, dtype=np.uint32)
    keys = rng.permutation(np.tile(base, dup))
    return adb.tuples(keys)


@pytest.mark.parametrize("algo", EAGER)
def test_eager_relations_fk(oracle, algo):
    R = adb.gen_pk(20000, 3)
    S = adb.gen_fk(30001, R, 0.9, 4)
    p = adb.default_params(nthreads=8, group_size=2, progressive_step=10)
    got = adb.join(algo, R, S, p)
    assert (got.count, got.checksum) == oracle.truth(R, S)
    assert got.count == len(S)


@pytest.mark.parametrize("algo", EAGER)
def test_eager_relations_duplicates(oracle, algo):
    R = dup_streams(24000, 5000, 4, 1)
    S = dup_streams(20000, 5000, 4, 2)
    p = adb.default_params(nthreads=4, group_size=2, progressive_step=20)
    got = adb.join(algo, R, S, p)
    assert (got.count, got.checksum) == oracle.by_name(algo, R, S, progressive_step=20)


def test_oracle_eager_restatements_agree(oracle):
    R = dup_streams(4000, 700, 4, 5)
    S = dup_streams(3000, 700, 4, 6)
    want = oracle.truth(R, S)
    assert oracle.shj(R, S) == want
    assert oracle.pmj(R, S, 400, 300) == want
    assert oracle.pmj(R, S, 1, 1) == want


@pytest.mark.parametrize("batch", [1, 7, 1600, 1 << 20])
@pytest.mark.parametrize("algo", ["SHJ_JM_NP", "SHJ_JB_NP"])
def test_shj_batch_size_invariance(oracle, algo, batch):
    R = dup_streams(10000, 3000, 4, 7)
    S = dup_streams(9996, 3000, 4, 8)
    got = adb.join(algo, R, S, adb.default_params(batch_tuples=batch, nthreads=16))
    assert (got.count, got.checksum) == oracle.truth(R, S)


@pytest.mark.parametrize("step", [1, 5, 33, 100])
def test_pmj_progressive_step_invariance(oracle, step):
    R = dup_streams(12000, 3000, 4, 9)
    S = dup_streams(12000, 3000, 4, 10)
    got = adb.join("PMJ_JM_NP", R, S, adb.default_params(progressive_step=step))
    assert (got.count, got.checksum) == oracle.truth(R, S)


def test_eager_edge_cases(oracle):
    keys = np.array([0xFFFFFFFF, 0, 0xFFFFFFFF, 5], np.uint32)
    R = adb.tuples(keys, np.array([0xFFFFFFFF, 1, 2, 0xFFFFFFFF], np.uint32))
    S = adb.tuples(np.array([0xFFFFFFFF, 5, 0], np.uint32), np.array([0xFFFFFFFF, 3, 4], np.uint32))
    for algo in ("SHJ_JM_NP", "SHJ_JB_NP", "PMJ_JM_NP"):
        got = adb.join(algo, R, S, adb.default_params(batch_tuples=1, nthreads=4))
        assert (got.count, got.checksum) == oracle.truth(R, S)
        e = R[:0]
        assert adb.join(algo, e, S).count == 0
        assert adb.join(algo, R, e).count == 0


def make_streams(n_per_side, rate_per_ms, key_range, dup, seed):
    """Two ts-ordered streams: Poisson arrivals, keys drawn then materialised dup times."""
    out = []
    rng = np.random.default_rng(seed)
    for side in range(2):
        gaps = rng.exponential(1.0 / rate_per_ms, size=n_per_side)
        ts = np.floor(np.cumsum(gaps)).astype(np.uint64)
        rel = dup_streams(n_per_side, key_range, dup, seed * 10 + side)
        st = np.empty(n_per_side, dtype=adb.STREAM_TUPLE)
        st["ts_ms"] = ts
        st["key"] = rel["key"]
        st["payload"] = rel["payload"]
        out.append(st)
    return out


@pytest.mark.parametrize("algo", ["SHJ_JM_NP", "SHJ_JBCR_NP", "PMJ_JB_NP", "PMJ_JBCR_P"])
def test_stream_windows(oracle, algo):
    """Tumbling windows over two streams: each window's result equals the join of its tuples."""
    R, S = make_streams(60000, 16.0, 4000, 4, 11)     # ~3.7 s of stream, 1000 ms windows
    p = adb.default_params(window_size=1000, batch_tuples=500, nthreads=8, group_size=2, progressive_step=10)
    wins = adb.stream_join(algo, R, S, p)
    assert len(wins) >= 3
    total_r = total_s = 0
    for w in wins:
        lo, hi = w.window_start_ms, w.window_start_ms + 1000
        r = R[(R["ts_ms"] >= lo) & (R["ts_ms"] < hi)]
        s = S[(S["ts_ms"] >= lo) & (S["ts_ms"] < hi)]
        assert (w.n_r, w.n_s) == (len(r), len(s))
        rt = adb.tuples(r["key"], r["payload"])
        stt = adb.tuples(s["key"], s["payload"])
        assert (w.count, w.checksum) == oracle.truth(rt, stt)
        total_r += w.n_r
        total_s += w.n_s
    assert (total_r, total_s) == (len(R), len(S))


def test_stream_models_agree():
    R, S = make_streams(30000, 20.0, 2000, 4, 12)
    p = adb.default_params(window_size=500, batch_tuples=256, nthreads=8, group_size=4)
    ref = [(w.count, w.checksum) for w in adb.stream_join("SHJ_st", R, S, p)]
    for algo in EAGER[1:]:
        got = [(w.count, w.checksum) for w in adb.stream_join(algo, R, S, p)]
        assert got == ref, algo


@pytest.mark.parametrize("algo", ["SHJ_JM_NP", "PMJ_JM_NP"])
@pytest.mark.parametrize("realtime", [0, 1])
def test_stream_progress(oracle, algo, realtime):
    """Progressiveness per window (adb_stream_join_progress): results equal the
    plain call's, the time to k % of the matches grows with k and ends at the
    last batch, latency percentiles are ordered, and with the arrival schedule
    (realtime) a 1 ms micro-batch has its results within the window."""
    R, S = make_streams(6000, 6.0, 1000, 4, 13)      # ~1 s of stream at 6 tuples/ms per side
    p = adb.default_params(window_size=250, batch_tuples=6, progressive_step=10, realtime=realtime)
    plain = adb.stream_join(algo, R, S, p)
    wins, prog = adb.stream_join(algo, R, S, p, progress=True)
    assert [(w.count, w.checksum) for w in wins] == [(w.count, w.checksum) for w in plain]
    for w, g in zip(wins, prog):
        t = list(g.t_pct)
        assert g.batches >= 1
        if w.count == 0:
            assert t == [0.0] * 9
            continue
        assert all(a <= b for a, b in zip(t, t[1:])), t
        assert t[0] >= 0 and g.lat_p50 <= g.lat_p95 <= g.lat_p99
        if realtime:
            assert t[-1] < 250 + 50      # the last batch is released near the window's end
            assert g.lat_p99 < 50        # a batch's results follow its release closely


def test_long_streams_staged_copy_and_order_check(oracle):
    """Streams above the direct-copy threshold (16 MiB per side) reach the
    device through the staged host copy from pageable memory: the windows
    equal those of the same streams in pinned memory (one direct copy) and the
    oracle's join of each window.  A long stream out of timestamp order is
    refused after its copy, with the first offending index."""
    import torch
    R, S = make_streams(1_300_000, 650.0, 1 << 18, 4, 14)   # ~2 s, 20.8 MB per side
    assert R.nbytes > (16 << 20) and S.nbytes > (16 << 20)
    p = adb.default_params(window_size=1000, batch_tuples=1600, nthreads=8)
    got = adb.stream_join("SHJ_JM_NP", R, S, p)
    Rp = torch.empty(R.nbytes, dtype=torch.uint8, pin_memory=True).numpy().view(adb.STREAM_TUPLE)
    Sp = torch.empty(S.nbytes, dtype=torch.uint8, pin_memory=True).numpy().view(adb.STREAM_TUPLE)
    Rp[:] = R
    Sp[:] = S
    pinned = adb.stream_join("SHJ_JM_NP", Rp, Sp, p)
    assert [(w.n_r, w.n_s, w.count, w.checksum) for w in got] == \
           [(w.n_r, w.n_s, w.count, w.checksum) for w in pinned]
    w = got[0]
    r = R[R["ts_ms"] < w.window_start_ms + 1000]
    s = S[S["ts_ms"] < w.window_start_ms + 1000]
    assert (w.count, w.checksum) == oracle.truth(adb.tuples(r["key"], r["payload"]),
                                                 adb.tuples(s["key"], s["payload"]))
    for side in ("R", "S"):
        bad_r, bad_s = R.copy(), S.copy()
        bad = bad_r if side == "R" else bad_s
        bad["ts_ms"][700_001] = 0
        with pytest.raises(adb.AdbError) as e:
            adb.stream_join("SHJ_JM_NP", bad_r, bad_s, p)
        assert e.value.status == adb.ADB_ERR_ARG
        assert f"{side} is not ordered by timestamp (index 700001)" in str(e.value)
    # the context is still usable
    again = adb.stream_join("SHJ_JM_NP", R, S, p)
    assert [(w.count, w.checksum) for w in again] == [(w.count, w.checksum) for w in got]


@pytest.mark.parametrize("nthreads,group_size", [(8, 1), (8, 2), (8, 4), (8, 8), (6, 3), (4, 16)])
@pytest.mark.parametrize("seed", [0, 12345])
def test_jbcr_groups_members_and_seeds(oracle, nthreads, group_size, seed):
    """JBCR: R replicated to every member of its key group, each S tuple sent
    to one seeded random member.  Any group layout and seed gives the oracle's
    join, and the per-batch form (progress) the same windows as the
    throughput form."""
    R = dup_streams(20000, 3000, 4, 5)
    S = dup_streams(30000, 3000, 4, 6)
    p = adb.default_params(nthreads=nthreads, group_size=group_size, seed=seed)
    for algo in ("SHJ_JBCR_NP", "SHJ_JBCR_P"):
        got = adb.join(algo, R, S, p)
        assert (got.count, got.checksum) == oracle.truth(R, S), algo
    Rs, Ss = make_streams(8000, 8.0, 800, 4, 15)
    q = adb.default_params(window_size=500, batch_tuples=64, nthreads=nthreads, group_size=group_size, seed=seed)
    plain = adb.stream_join("SHJ_JBCR_NP", Rs, Ss, q)
    wins, _ = adb.stream_join("SHJ_JBCR_NP", Rs, Ss, q, progress=True)
    assert [(w.count, w.checksum) for w in wins] == [(w.count, w.checksum) for w in plain]
    assert sum(w.n_r for w in wins) == len(Rs)
