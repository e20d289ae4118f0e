"""GPU parity: every provided lazy join on the B200 against the CPU oracle.

Bit-exact on count and checksum (integer work: no tolerance).  Inputs are the
seeded generator's relations plus the edge cases the reference's own checks
and code paths imply (empty relations, one tuple, all-equal keys, keys 0 and
0xFFFFFFFF, non-power-of-two sizes, unaligned relation pointers).
"""
import numpy as np
import pytest

import alliancedb_b200 as adb

pytestmark = pytest.mark.gpu

LAZY = ["PRO", "RJ_st", "PRH", "PRHO", "NPO", "NPO_st", "m-way", "m-pass", "m-way+skew"]


def fk_pair(n_r, n_s, theta=0.0, seed=7):
    R = adb.gen_pk(n_r, seed)
    S = adb.gen_fk(n_s, R, theta, seed + 1)
    return R, S


def check(oracle, algo, R, S, **kw):
    params = adb.default_params(**kw) if kw else None
    got = adb.join(algo, R, S, params)
    want = oracle.by_name(algo, R, S)
    assert (got.count, got.checksum) == want, f"{algo}: got {(got.count, got.checksum)} want {want}"
    return got


@pytest.mark.parametrize("algo", LAZY)
@pytest.mark.parametrize("n", [1, 2, 3, 1000, 4097, 1 << 16, (1 << 20) + 3])
def test_fk_sizes(oracle, algo, n):
    R, S = fk_pair(n, n)
    got = check(oracle, algo, R, S)
    assert got.count == n   # PK-FK: every S tuple matches once (hashing/test/test.cpp:72)


@pytest.mark.parametrize("algo", LAZY)
@pytest.mark.parametrize("theta", [0.5, 1.0, 1.5])
def test_zipf(oracle, algo, theta):
    R, S = fk_pair(1 << 16, 1 << 17, theta)
    got = check(oracle, algo, R, S)
    assert got.count == 1 << 17


@pytest.mark.parametrize("algo", LAZY)
def test_duplicates_both_sides(oracle, algo):
    R = adb.gen_uniform(1 << 14, 1 << 10, 3)
    S = adb.gen_uniform(3 << 13, 1 << 10, 4)
    check(oracle, algo, R, S)


@pytest.mark.parametrize("algo", LAZY)
def test_all_equal_keys(oracle, algo):
    R = adb.tuples(np.full(3000, 42, np.uint32))
    S = adb.tuples(np.full(2500, 42, np.uint32))
    got = check(oracle, algo, R, S)
    assert got.count == 3000 * 2500


@pytest.mark.parametrize("algo", LAZY)
def test_extreme_keys(oracle, algo):
    keys = np.array([0, 0xFFFFFFFF, 1, 0x80000000, 0xFFFFFFFF, 0, 7], np.uint32)
    R = adb.tuples(keys, np.array([0xFFFFFFFF, 0xFFFFFFFF, 5, 6, 0, 9, 0xFFFFFFFF], np.uint32))
    S = adb.tuples(np.array([0xFFFFFFFF, 0, 0x80000000, 3, 0xFFFFFFFF, 7], np.uint32),
                   np.array([1, 2, 3, 4, 0xFFFFFFFF, 6], np.uint32))
    check(oracle, algo, R, S)


@pytest.mark.parametrize("algo", LAZY)
def test_empty(oracle, algo):
    R, S = fk_pair(100, 100)
    e = R[:0]
    for a, b in ((e, S), (R, e), (e, e)):
        got = adb.join(algo, a, b)
        assert (got.count, got.checksum) == (0, 0)


@pytest.mark.parametrize("algo", ["PRO", "PRH", "NPO"])
@pytest.mark.parametrize("bits", [1, 4, 8, 9, 10, 11, 12, 13, 14])
def test_radix_bits(oracle, algo, bits):
    R, S = fk_pair(50000, 70001, 0.8)
    check(oracle, algo, R, S, radix_bits=bits)


@pytest.mark.parametrize("algo", ["PRO", "PRH"])
@pytest.mark.parametrize("bits", [10, 13])
def test_two_pass_fanouts_many_tiles(oracle, algo, bits):
    """Two-pass fan-outs (2^5 x 2^5, 2^6 x 2^7) over several tiles per CTA and pass-2 unit, skewed S."""
    R, S = fk_pair((1 << 21) + 5, (1 << 21) + 77, 1.0)
    check(oracle, algo, R, S, radix_bits=bits)


@pytest.mark.parametrize("fanout", [2, 64, 1 << 12, 1 << 16])
def test_smj_part_fanout(oracle, fanout):
    """joinconfig_t.PARTFANOUT (sorting/utils/types.h:117-124) changes the plan, not the result."""
    R, S = fk_pair(40000, 50001, 1.2)
    check(oracle, "m-way", R, S, part_fanout=fanout)


@pytest.mark.parametrize("algo", ["m-way", "PRO"])
def test_clustered_keys_with_outlier(oracle, algo):
    """Dense small keys plus one far key: one sort bucket would hold nearly all tuples."""
    keys = np.concatenate([np.arange(1, 60001, dtype=np.uint32) * 8, np.array([0x80000000], np.uint32)])
    R = adb.tuples(np.random.default_rng(5).permutation(keys))
    S = adb.tuples(np.random.default_rng(6).choice(keys, 70000))
    check(oracle, algo, R, S)


@pytest.mark.parametrize("algo", LAZY)
def test_device_pointers_unaligned(oracle, algo):
    """Relations that start 8 bytes past a 16-byte boundary (sub-relations)."""
    R, S = fk_pair(30001, 40003, 1.0)
    L = adb.lib()
    import ctypes as C
    ptrs = []
    try:
        for rel in (R, S):
            p = C.c_void_p()
            assert L.adb_device_alloc(C.byref(p), rel.nbytes + 16) == 0
            ptrs.append(p.value)
            assert L.adb_memcpy_h2d(p.value + 8, rel.ctypes.data, rel.nbytes) == 0
        got = adb.join_device(algo, ptrs[0] + 8, len(R), ptrs[1] + 8, len(S))
        assert (got.count, got.checksum) == oracle.by_name(algo, R, S)
    finally:
        for p in ptrs:
            L.adb_device_free(p)


def test_repeat_calls_same_result(oracle):
    R, S = fk_pair(1 << 18, 1 << 18, 0.5)
    want = oracle.pro(R, S)
    for _ in range(3):
        got = adb.join("PRO", R, S)
        assert (got.count, got.checksum) == want


def test_inputs_not_modified():
    R, S = fk_pair(1 << 16, 1 << 16)
    R0, S0 = R.copy(), S.copy()
    adb.join("PRO", R, S)
    assert np.array_equal(R, R0) and np.array_equal(S, S0)


@pytest.mark.parametrize("algo", LAZY + ["SHJ_JM_NP", "SHJ_JB_NP", "PMJ_JM_NP", "PMJ_JBCR_NP"])
def test_golden_fixtures(algo):
    """Results equal the committed fixtures, whose counts the reference itself produced."""
    import json
    from pathlib import Path
    golden = Path(__file__).resolve().parent / "golden"
    meta = json.loads((golden / "cases.json").read_text())
    for name, m in meta.items():
        R = np.load(golden / f"{name}_R.npy")
        S = np.load(golden / f"{name}_S.npy")
        got = adb.join(algo, R, S, adb.default_params(batch_tuples=64, nthreads=4, progressive_step=10))
        assert (got.count, got.checksum) == (m["count"], int(m["checksum"])), name


def test_threads_share_device_context(oracle):
    # calls from several host threads serialise on the device's context
    import threading
    cases = [(adb.gen_pk(1 << 16, 40 + t), None) for t in range(4)]
    cases = [(R, adb.gen_fk(1 << 17, R, 0.5, 50 + t)) for t, (R, _) in enumerate(cases)]
    want = [oracle.truth(R, S) for R, S in cases]
    got = [None] * len(cases)

    def work(i):
        algo = ("PRO", "NPO", "m-way", "PRH")[i]
        for _ in range(3):
            r = adb.join(algo, *cases[i])
            got[i] = (r.count, r.checksum)

    th = [threading.Thread(target=work, args=(i,)) for i in range(len(cases))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert got == want


@pytest.mark.parametrize("algo", ["m-way", "m-pass", "m-way+skew", "PRO", "NPO"])
def test_single_key_probe_blocks(oracle, algo):
    """S blocks of one key (a hot key under skew: the sort-merge join leaves such
    a block unsorted and pairs it with R's run of that key), next to blocks with
    a few other keys; R holds the hot key once and another key many times."""
    rng = np.random.default_rng(17)
    rk = rng.permutation(np.arange(1, 20001, dtype=np.uint32))
    rk[:600] = 777                                           # a key repeated 600 times in R
    R = adb.tuples(rk)
    sk = np.full(40000, 4242, np.uint32)                     # the hot key (once in R)
    sk[::997] = rng.integers(1, 20001, size=len(sk[::997]), dtype=np.uint32)
    sk[20000:26000] = 777                                    # a block of the repeated key
    S = adb.tuples(sk)
    check(oracle, algo, R, S)


@pytest.mark.parametrize("algo", ["m-way", "m-way+skew"])
def test_single_key_block_with_all_ones_tuples(oracle, algo):
    """An S block of one key plus real all-ones tuples (key and payload
    0xFFFFFFFF, the pad word's value): they must join R's key-0xFFFFFFFF tuples."""
    R = adb.tuples(np.array([5, 0xFFFFFFFF, 9, 0xFFFFFFFF], np.uint32),
                   np.array([1, 0xFFFFFFFF, 3, 7], np.uint32))
    sk = np.full(3000, 5, np.uint32)
    sp = np.arange(3000, dtype=np.uint32)
    sk[[10, 2000]] = 0xFFFFFFFF
    sp[[10, 2000]] = 0xFFFFFFFF
    S = adb.tuples(sk, sp)
    check(oracle, algo, R, S)


@pytest.mark.parametrize("algo", ["PRO", "NPO", "m-way"])
def test_host_inputs_through_the_staged_copy(oracle, algo):
    """Host relations above the direct-copy threshold (16 MiB) in pageable
    memory reach the device through the staged copy: a ragged last 4 MiB
    chunk, and a source that starts one tuple into its array (8-byte aligned
    only), both equal the direct-address truth."""
    n = (1 << 22) + 12345
    R = adb.gen_pk(n, 31)
    S = adb.gen_fk(n + 7, R, 0.0, 32)
    assert S.nbytes > (16 << 20)
    got = adb.join(algo, R, S)
    assert (got.count, got.checksum) == oracle.pk_truth(R, S)
    Sv = S[1:]
    got = adb.join(algo, R, Sv)
    assert (got.count, got.checksum) == oracle.pk_truth(R, Sv)


@pytest.mark.parametrize("algo", ["m-way", "m-way+skew"])
@pytest.mark.parametrize("case", ["one_key", "many_keys", "max_key"])
def test_sort_merge_small_r_large_s(oracle, algo, case):
    """A small R against a large S: each partition has hundreds of S blocks against one R chunk (S
    blocks of one key, S blocks of many keys joined by bucket, and blocks holding key 0xFFFFFFFF, which
    take the merge path with S sorted)."""
    R = adb.gen_pk(4096, 41)
    n_s = 1 << 22
    if case == "one_key":
        S = adb.tuples(np.full(n_s, R["key"][7], np.uint32))
    elif case == "many_keys":
        S = adb.gen_fk(n_s, R, 0.9, 42)
    else:
        R["key"][:3] = 0xFFFFFFFF
        keys = np.random.default_rng(43).choice(R["key"], n_s)
        S = adb.tuples(keys.astype(np.uint32))
    check(oracle, algo, R, S)
