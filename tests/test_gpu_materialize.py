"""Result materialisation (adb_join_materialize_device) on the B200.

The reference stores, per match, the probe side's <S-key, S-payload> in
chained tuple buffers when JOIN_RESULT_MATERIALIZE is defined
(hashing/joins/common_functions.cpp:255-258, sorting/joins/common_functions.cpp
:331-336).  The device writes the same tuples into a caller's array; their
order is arbitrary, so the test compares the sorted multiset with the oracle's
(every S tuple once per R tuple of equal key), next to count and checksum.
"""
import numpy as np
import pytest

import alliancedb_b200 as adb

pytestmark = pytest.mark.gpu

ALGOS = ["PRO", "RJ_st", "PRH", "NPO", "m-way", "m-pass"]


def words(t):
    return np.ascontiguousarray(t).view(np.uint64)


def materialize(algo, R, S, cap):
    dR, dS = adb.DeviceBuffer.from_host(R), adb.DeviceBuffer.from_host(S)
    dO = adb.DeviceBuffer(max(cap, 1) * 8)
    try:
        res = adb.join_materialize_device(algo, dR.ptr, len(R), dS.ptr, len(S), dO.ptr, cap)
        out = dO.to_host(np.uint64, min(res.materialized, cap))
    finally:
        for b in (dR, dS, dO):
            b.close()
    return res, out


@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("case", ["fk", "dups", "zipf"])
def test_materialized_tuples_match_oracle(oracle, algo, case):
    if case == "fk":
        R = adb.gen_pk(50000, 3)
        S = adb.gen_fk(70001, R, 0.0, 4)
    elif case == "zipf":
        R = adb.gen_pk(40000, 5)
        S = adb.gen_fk(60000, R, 1.2, 6)
    else:
        R = adb.gen_uniform(6000, 1500, 7)
        S = adb.gen_uniform(5000, 1500, 8)
    n_want, want = oracle.materialize_sorted(R, S, 1 << 22)
    res, got = materialize(algo, R, S, 1 << 22)
    assert (res.count, res.checksum) == oracle.by_name(algo, R, S)
    assert res.count == n_want == res.materialized
    assert np.array_equal(np.sort(got), words(want))


@pytest.mark.parametrize("algo", ["PRO", "NPO", "m-way"])
def test_capacity_smaller_than_matches(oracle, algo):
    """Past `cap` the matches are still counted; the stored ones are `cap` of them."""
    R = adb.gen_uniform(3000, 200, 9)
    S = adb.gen_uniform(3000, 200, 10)
    n_want, want = oracle.materialize_sorted(R, S, 1 << 22)
    cap = n_want // 3
    res, got = materialize(algo, R, S, cap)
    assert res.count == n_want and res.materialized == cap
    # every stored tuple is one of the true results, no more often than it occurs there
    keys, counts = np.unique(words(want), return_counts=True)
    gk, gc = np.unique(got, return_counts=True)
    idx = np.searchsorted(keys, gk)
    assert np.all(idx < len(keys)) and np.array_equal(keys[idx], gk)
    assert np.all(gc <= counts[idx])
