"""NPO with its inputs grouped by table region, on the B200.

Above a 256 MB table (|R| > 2^24) NPO groups R and S by the top bits of the
hash (the table region of each key) with one partition pass, then builds and
probes in region order so that the region being worked on stays in L2.  The
table is the same single open-addressing array; only the order of inserts and
probes changes, so count and checksum must equal the oracle's NPO
(no_partitioning_join.cpp:383-476) and the ungrouped join exactly.

radix_bits selects the grouping for NPO: > 0 forces that many region bits
(up to 9), < 0 turns grouping off, 0 chooses from |R|.
"""
import numpy as np
import pytest

import alliancedb_b200 as adb

pytestmark = pytest.mark.gpu


def check(oracle, R, S, bits, algo="NPO"):
    got = adb.join(algo, R, S, adb.default_params(radix_bits=bits))
    want = oracle.by_name(algo, R, S)
    assert (got.count, got.checksum) == want, f"bits={bits}: got {(got.count, hex(got.checksum))} want {want}"
    return got


@pytest.mark.parametrize("algo", ["NPO", "NPO_st"])
@pytest.mark.parametrize("bits", [1, 3, 7, 9])
@pytest.mark.parametrize("n", [1, 63, 65, 4097, (1 << 18) + 11])
def test_region_bits_fk(oracle, algo, bits, n):
    R = adb.gen_pk(n, 21)
    S = adb.gen_fk(n + 5, R, 0.0, 22)
    got = check(oracle, R, S, bits, algo)
    assert got.count == n + 5


@pytest.mark.parametrize("theta", [0.5, 1.0, 1.5])
def test_region_bits_zipf(oracle, theta):
    R = adb.gen_pk(1 << 17, 23)
    S = adb.gen_fk(3 << 16, R, theta, 24)
    check(oracle, R, S, 6)


def test_region_bits_duplicates_and_long_runs(oracle):
    """Repeated build keys make long linear-probing runs that cross sectors and region borders."""
    R = adb.gen_uniform(1 << 15, 1 << 9, 25)
    S = adb.gen_uniform(3 << 14, 1 << 9, 26)
    for bits in (2, 5, 9):
        check(oracle, R, S, bits)


def test_region_bits_all_equal_keys(oracle):
    R = adb.tuples(np.full(3000, 42, np.uint32))
    S = adb.tuples(np.full(2500, 42, np.uint32))
    got = check(oracle, R, S, 4)
    assert got.count == 3000 * 2500


def test_region_bits_extreme_keys(oracle):
    """Keys 0 and 0xFFFFFFFF, and R tuples equal to the table's empty marker (counted on the side)."""
    keys = np.array([0, 0xFFFFFFFF, 1, 0x80000000, 0xFFFFFFFF, 0, 7, 0xFFFFFFFF], np.uint32)
    R = adb.tuples(keys, np.array([0xFFFFFFFF, 0xFFFFFFFF, 5, 6, 0, 9, 0xFFFFFFFF, 0xFFFFFFFF], np.uint32))
    S = adb.tuples(np.array([0xFFFFFFFF, 0, 0x80000000, 3, 0xFFFFFFFF, 7], np.uint32),
                   np.array([1, 2, 3, 4, 0xFFFFFFFF, 6], np.uint32))
    for bits in (1, 2):
        check(oracle, R, S, bits)


def test_region_bits_empty_sides():
    R = adb.gen_pk(1000, 27)
    S = adb.gen_fk(1000, R, 0.0, 28)
    e = R[:0]
    for a, b in ((e, S), (R, e), (e, e)):
        got = adb.join("NPO", a, b, adb.default_params(radix_bits=5))
        assert (got.count, got.checksum) == (0, 0)


def test_grouped_equals_ungrouped(oracle):
    R = adb.gen_uniform(200_000, 60_000, 29)
    S = adb.gen_uniform(300_001, 60_000, 30)
    want = oracle.by_name("NPO", R, S)
    for bits in (-1, 0, 1, 4, 8):
        got = adb.join("NPO", R, S, adb.default_params(radix_bits=bits))
        assert (got.count, got.checksum) == want, f"bits={bits}"


def test_grouped_materialization(oracle):
    R = adb.gen_uniform(6000, 1500, 31)
    S = adb.gen_uniform(5000, 1500, 32)
    n_want, want = oracle.materialize_sorted(R, S, 1 << 22)
    dR, dS = adb.DeviceBuffer.from_host(R), adb.DeviceBuffer.from_host(S)
    dO = adb.DeviceBuffer((1 << 22) * 8)
    try:
        res = adb.join_materialize_device("NPO", dR.ptr, len(R), dS.ptr, len(S), dO.ptr, 1 << 22,
                                          adb.default_params(radix_bits=3))
        got = dO.to_host(np.uint64, res.materialized)
    finally:
        for b in (dR, dS, dO):
            b.close()
    assert (res.count, res.checksum) == oracle.by_name("NPO", R, S)
    assert res.count == n_want == res.materialized
    assert np.array_equal(np.sort(got), np.ascontiguousarray(want).view(np.uint64))


def test_automatic_grouping_above_l2(oracle):
    """|R| = 2^25: a 512 MB table, grouped into 32 regions by default; phase 0 is the grouping pass."""
    R = adb.gen_pk(1 << 25, 33)
    S = adb.gen_fk(1 << 23, R, 0.7, 34)
    truth = oracle.pk_truth(R, S)
    got = adb.join("NPO", R, S)
    assert (got.count, got.checksum) == truth
    assert got.ms_phase[0] > 0
    flat = adb.join("NPO", R, S, adb.default_params(radix_bits=-1))
    assert (flat.count, flat.checksum) == truth
    assert flat.ms_phase[0] < 0.05
