"""GPU parity on the benchmark's own configurations, at their full sizes.

* 2^22 x 2^22 foreign-key join (R keys a seeded permutation of 1..2^22, S keys
  uniform over R's keys): PRO and NPO against the oracle's restatement of the
  reference join of the same name, and against the direct-address truth.
* 2^27 x 2^27, S keys Zipf(theta) over R's keys, theta in {0, 0.5, 1.0, 1.5}:
  PRO, NPO and m-way against the direct-address truth (a key -> payload table
  filled from R, one lookup per S tuple; it shares no code with any join), and
  the count against the foreign-key known answer |S| (hashing/test/test.cpp:72).
  The seeds are those of bench.py's default workload, so the theta = 0 case
  also checks the checksum that the benchmark reports.

Integer work: count and checksum must be bit-identical.
"""
import numpy as np
import pytest

import alliancedb_b200 as adb

pytestmark = pytest.mark.gpu

# bench.py's workload at 2^27, theta 0: count and checksum from the direct-address truth
BENCH_2E27_THETA0 = (1 << 27, 0xF5177842024F3CC8)


def fk(n, theta, seed=1):
    R = adb.gen_pk(n, seed)
    S = adb.gen_fk(n, R, theta, seed + 1)
    return R, S


@pytest.fixture(scope="module")
def c1():
    return fk(1 << 22, 0.0)


@pytest.mark.parametrize("algo", ["PRO", "NPO"])
def test_c1_2e22(oracle, c1, algo):
    R, S = c1
    got = adb.join(algo, R, S)
    truth = oracle.pk_truth(R, S)
    assert truth[0] == 1 << 22
    assert (got.count, got.checksum) == truth
    assert oracle.by_name(algo, R, S) == truth


_c2_cache = {}


def c2(theta):
    if theta not in _c2_cache:
        _c2_cache.clear()   # one 2 GiB pair in host memory at a time
        _c2_cache[theta] = fk(1 << 27, theta)
    return _c2_cache[theta]


_truth_cache = {}


@pytest.mark.parametrize("algo", ["PRO", "NPO", "m-way"])
@pytest.mark.parametrize("theta", [0.0, 0.5, 1.0, 1.5])
def test_c2_2e27(oracle, theta, algo):
    R, S = c2(theta)
    if theta not in _truth_cache:
        _truth_cache[theta] = oracle.pk_truth(R, S)
    truth = _truth_cache[theta]
    assert truth[0] == 1 << 27
    if theta == 0.0:
        assert truth == BENCH_2E27_THETA0
    got = adb.join(algo, R, S)
    assert (got.count, got.checksum) == truth, f"{algo} theta={theta}: {(got.count, hex(got.checksum))}"
