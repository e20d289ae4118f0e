"""The serving loop: every request's result served in a mix equals the same
request joined alone; admission respects the memory budget; latency and
throughput statistics are filled."""
import numpy as np
import pytest

import alliancedb_b200 as adb

pytestmark = pytest.mark.gpu


def requests(n, rate_per_s, lo, hi, seed):
    """Open-loop Poisson arrivals, sizes log-uniform in [2^lo, 2^hi] per side."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1e6 / rate_per_s, size=n))
    out = []
    for i in range(n):
        nr = int(2 ** rng.uniform(lo, hi))
        ns = int(2 ** rng.uniform(lo, hi))
        out.append((int(t[i]), nr, ns, 1000 + i))
    return out


def alone(nr, ns, seed):
    R = adb.gen_pk(nr, seed)
    S = adb.gen_fk(ns, R, 0.0, seed + 1)
    r = adb.join("PRO", R, S)
    return r.count, r.checksum


@pytest.mark.parametrize("slots", [1, 2])
def test_served_results_equal_alone(slots):
    reqs = requests(60, 2000.0, 8, 15, 7)
    res, st = adb.serve_run(reqs, budget_bytes=256 << 20, max_batch=16, realtime=True, slots=slots)
    assert st.requests == 60 and st.batches >= 4
    for (t, nr, ns, seed), r in zip(reqs, res):
        assert r.status == 0
        assert r.count == ns   # FK: every S tuple matches once
        assert (r.count, r.checksum) == alone(nr, ns, seed)
        assert r.latency_ms >= 0 and r.queue_ms <= r.latency_ms
    assert 0 < st.p50_ms <= st.p99_ms <= st.p999_ms
    assert st.tuples_per_s > 0


def test_tight_budget_forces_small_batches():
    reqs = requests(40, 1e9, 14, 15, 8)       # everything arrives at once
    big = max(nr + ns for _, nr, ns, _ in reqs) * 8
    res, st = adb.serve_run(reqs, budget_bytes=4 * 3 * big, max_batch=64, realtime=False, slots=2)
    assert st.peak_arena_bytes <= st.arena_bytes
    assert st.mean_batch < 40
    for (t, nr, ns, seed), r in zip(reqs[:5], res[:5]):
        assert (r.count, r.checksum) == alone(nr, ns, seed)


def test_request_larger_than_budget_is_refused():
    with pytest.raises(adb.AdbError) as e:
        adb.serve_run([(0, 1 << 20, 1 << 20, 1)], budget_bytes=1 << 20)
    assert e.value.status == adb.ADB_ERR_BUSY
