"""The library's seeded generator (host side) against its numpy restatement."""
import numpy as np
import pytest

import alliancedb_b200 as adb
from tests.golden.make_golden import gen_numpy_fk_uniform, gen_numpy_pk, gen_numpy_uniform


@pytest.mark.parametrize("n,seed", [(1, 1), (2, 5), (1000, 1), (4096, 3), (99991, 12)])
def test_pk_matches_numpy_and_is_a_permutation(n, seed):
    R = adb.gen_pk(n, seed)
    assert np.array_equal(R.view(np.uint64), gen_numpy_pk(n, seed))
    assert np.array_equal(np.sort(R["key"]), np.arange(1, n + 1, dtype=np.uint32))
    assert np.array_equal(R["payload"], np.arange(n, dtype=np.uint32))


def test_fk_uniform_matches_numpy():
    R = adb.gen_pk(5000, 3)
    S, idx = adb.gen_fk(7000, R, 0.0, 4, want_idx=True)
    assert np.array_equal(S.view(np.uint64), gen_numpy_fk_uniform(7000, R.view(np.uint64), 4))
    assert np.array_equal(S["key"], R["key"][idx])


def test_uniform_matches_numpy():
    T = adb.gen_uniform(10000, 777, 9)
    assert np.array_equal(T.view(np.uint64), gen_numpy_uniform(10000, 777, 9))
    assert T["key"].min() >= 1 and T["key"].max() <= 777


@pytest.mark.parametrize("theta", [0.5, 1.0, 1.5])
def test_zipf_rank_frequencies(theta):
    """Zipf(theta) over R's keys: the k-th most frequent key has frequency ~ k^-theta / H."""
    n = 1000
    R = adb.gen_pk(n, 21)
    S, idx = adb.gen_fk(200000, R, theta, 22, want_idx=True)
    counts = np.sort(np.bincount(idx, minlength=n))[::-1].astype(np.float64)
    w = np.arange(1, n + 1, dtype=np.float64) ** -theta
    p = w / w.sum()
    # top ranks within 3 standard deviations of the expected counts
    for k in range(5):
        mu = 200000 * p[k]
        assert abs(counts[k] - mu) < 3 * np.sqrt(mu) + 5, (k, counts[k], mu)


def test_generator_is_counter_based():
    """Element i depends only on (seed, i): a prefix equals the smaller call."""
    a = adb.gen_uniform(5000, 1 << 20, 4)
    b = adb.gen_uniform(3000, 1 << 20, 4)
    assert np.array_equal(a[:3000], b)
