"""The allocation-free NPO entry point (adb_npo_join_noalloc).

adb_npo_join_noalloc serves callers that may not allocate device memory
while they run (an engine that budgets all of HBM up front, a memory-capped
sandbox, a pipeline that must never wait on an allocator): its hash table is a
fixed 32 MiB array inside the library.  This test calls it through the C ABI
three times in a row on the same inputs, because every call reuses the same
array and must start from a clean table, and checks each result bit-exactly
(integer work, no tolerance) against the CPU oracle's NPO and against the
ordinary allocating entry point adb_join("NPO").

The first call does the per-device set-up (the array's address; the module
that holds the array may be loaded then).  Free device memory is read after
it and again after the later calls: it must not change, since the entry point
allocates nothing.  The allocating entry point runs only after those calls.

The file name sorts last so that a run stopping at its first failure has
already run every other test.  It also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import alliancedb_b200 as adb

pytestmark = pytest.mark.gpu


def _dev_copy(L, arr):
    p = C.c_void_p()
    assert L.adb_device_alloc(C.byref(p), max(arr.nbytes, 16)) == 0
    if arr.nbytes:
        assert L.adb_memcpy_h2d(p.value, arr.ctypes.data, arr.nbytes) == 0
    return p.value


def _fn(L):
    f = L.adb_npo_join_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
    return f


@pytest.mark.parametrize("case", ["fk", "dups", "limit"])
def test_noalloc_matches_oracle_and_npo(oracle, case):
    import torch
    L = adb.lib()
    f = _fn(L)
    if case == "fk":
        R = adb.gen_pk(1 << 20, 5)
        S = adb.gen_fk(3 << 19, R, 0.7, 6)
    elif case == "dups":
        R = adb.gen_uniform(100_000, 20_000, 7)
        S = adb.gen_uniform(150_001, 20_000, 8)
    else:   # the largest build side the fixed table accepts
        R = adb.gen_pk(1 << 21, 9)
        S = adb.gen_fk(1 << 21, R, 0.0, 10)
    want = oracle.npo(R, S)
    dR, dS = _dev_copy(L, R), _dev_copy(L, S)
    out = C.c_void_p()
    assert L.adb_device_alloc(C.byref(out), 16) == 0
    free_after_setup = None
    try:
        for call in range(3):
            st = f(dR, len(R), dS, len(S), out.value, None)
            assert st == 0, L.adb_last_error().decode()
            assert L.adb_device_sync() == 0
            got = np.zeros(2, np.uint64)
            assert L.adb_memcpy_d2h(got.ctypes.data, out.value, 16) == 0
            assert (int(got[0]), int(got[1])) == want, f"call {call}"
            free_now = torch.cuda.mem_get_info()[0]
            if call == 0:
                free_after_setup = free_now
            else:
                assert free_now == free_after_setup, "the allocation-free entry point changed free device memory"
        npo = adb.join("NPO", R, S)
        assert (npo.count, npo.checksum) == want
    finally:
        for p in (dR, dS, out.value):
            L.adb_device_free(p)


def test_noalloc_rejects_oversized_build():
    L = adb.lib()
    f = _fn(L)
    # pointers are never dereferenced: the size check comes first
    st = f(C.c_void_p(16), (1 << 21) + 1, C.c_void_p(16), 4, C.c_void_p(16), None)
    assert st == adb.ADB_ERR_ARG
    assert "exceeds" in L.adb_last_error().decode()
