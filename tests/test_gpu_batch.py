"""Batched windows: one launch sequence for many windows (mode 0) against one
sequence per window (mode 1) and against the CPU oracle, window by window."""
import numpy as np
import pytest

import alliancedb_b200 as adb

pytestmark = pytest.mark.gpu


def make_batch(n_windows, lo, hi, seed, zipf_share=0.25):
    """Window sizes log-uniform in [2^lo, 2^hi] per side, keys uniform over 4x the
    window size (match rate about 0.25), a quarter of the windows Zipf(0.8)."""
    rng = np.random.default_rng(seed)
    Rs, Ss = [], []
    for w in range(n_windows):
        nr = int(2 ** rng.uniform(lo, hi))
        ns = int(2 ** rng.uniform(lo, hi))
        kr = 4 * max(nr, ns)
        if rng.random() < zipf_share:
            ranks = np.arange(1, kr + 1, dtype=np.float64)
            p = ranks ** -0.8
            p /= p.sum()
            perm = rng.permutation(kr).astype(np.uint32) + 1
            rk = perm[rng.choice(kr, size=nr, p=p)]
            sk = perm[rng.choice(kr, size=ns, p=p)]
        else:
            rk = rng.integers(1, kr + 1, size=nr, dtype=np.uint64).astype(np.uint32)
            sk = rng.integers(1, kr + 1, size=ns, dtype=np.uint64).astype(np.uint32)
        Rs.append(adb.tuples(rk))
        Ss.append(adb.tuples(sk))
    return Rs, Ss


def run_batch(Rs, Ss, mode):
    r_off = np.concatenate([[0], np.cumsum([len(r) for r in Rs])]).astype(np.uint64)
    s_off = np.concatenate([[0], np.cumsum([len(s) for s in Ss])]).astype(np.uint64)
    R = np.concatenate(Rs) if Rs else np.zeros(0, adb.TUPLE)
    S = np.concatenate(Ss) if Ss else np.zeros(0, adb.TUPLE)
    dR, dS = adb.DeviceBuffer.from_host(R), adb.DeviceBuffer.from_host(S)
    try:
        return adb.batch_join_device(dR.ptr, r_off, dS.ptr, s_off, mode)
    finally:
        dR.close()
        dS.close()


@pytest.mark.parametrize("seed", [1, 2])
def test_batch_modes_agree_with_oracle(oracle, seed):
    Rs, Ss = make_batch(48, 4, 16, seed)
    c0, k0, _ = run_batch(Rs, Ss, 0)
    c1, k1, _ = run_batch(Rs, Ss, 1)
    for w, (R, S) in enumerate(zip(Rs, Ss)):
        want = oracle.truth(R, S)
        assert (int(c0[w]), int(k0[w])) == want, w
        assert (int(c1[w]), int(k1[w])) == want, w


def test_batch_edge_windows(oracle):
    rng = np.random.default_rng(3)
    Rs = [adb.tuples(np.array([], np.uint32)), adb.tuples(np.array([7], np.uint32)),
          adb.tuples(np.full(5000, 9, np.uint32)), adb.tuples(rng.integers(1, 50, 3000).astype(np.uint32)),
          adb.tuples(np.array([0xFFFFFFFF, 0], np.uint32), np.array([0xFFFFFFFF, 1], np.uint32))]
    Ss = [adb.tuples(rng.integers(1, 9, 100).astype(np.uint32)), adb.tuples(np.array([7, 7], np.uint32)),
          adb.tuples(np.full(700, 9, np.uint32)), adb.tuples(np.array([], np.uint32)),
          adb.tuples(np.array([0xFFFFFFFF, 0, 0], np.uint32))]
    c, k, _ = run_batch(Rs, Ss, 0)
    for w, (R, S) in enumerate(zip(Rs, Ss)):
        assert (int(c[w]), int(k[w])) == oracle.truth(R, S), w


def test_batch_large_windows_split_across_units(oracle):
    """Windows bigger than one work unit (2^17 tuples) and skewed keys."""
    R = adb.gen_pk(300000, 5)
    S = adb.gen_fk(400000, R, 1.2, 6)
    Rs, Ss = [R[:1000], R, R[:70000]], [S[:5000], S, S[:1]]
    c, k, _ = run_batch(Rs, Ss, 0)
    for w, (r, s) in enumerate(zip(Rs, Ss)):
        assert (int(c[w]), int(k[w])) == oracle.truth(r, s), w


def test_autotune_table_changes_plan_not_results(oracle):
    table = adb.batch_autotune(10, 12)
    assert len(table) == 33 and all(0 <= b <= 9 for b in table)
    Rs, Ss = make_batch(16, 9, 13, 4)
    want = [oracle.truth(r, s) for r, s in zip(Rs, Ss)]
    for forced in ([0] * 33, [5] * 33, None):
        adb.batch_set_tuning(forced)
        c, k, _ = run_batch(Rs, Ss, 0)
        assert [(int(a), int(b)) for a, b in zip(c, k)] == want
    adb.batch_set_tuning(None)
