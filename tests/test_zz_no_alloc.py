"""The allocation-free NPO entry point (adb_npo_join_noalloc) against adb_join("NPO").

adb_npo_join_noalloc serves callers that may not allocate device memory
while they run (an engine that budgets all of HBM up front, a memory-capped
sandbox, a pipeline that must never wait on an allocator): its hash table is a
fixed 32 MiB array inside the library.  This test calls it through the C ABI
twice in a row on the same inputs, because every call reuses the same array
and must start from a clean table, and checks both results bit-exactly
(integer work, no tolerance) against the ordinary allocating entry point.

The file name sorts last so that a run stopping at its first failure has
already run every other test.  It also passes alone in a fresh process: the
first call performs the per-device set-up.
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


@pytest.mark.parametrize("case", ["fk", "dups", "limit"])
def test_noalloc_matches_npo_twice(case):
    L = adb.lib()
    f = L.adb_npo_join_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
    if case == "fk":
        R = adb.gen_pk(1 << 20, 5)
        S = adb.gen_fk(3 << 19, R, 0.7, 6)
    elif case == "dups":
        R = adb.gen_uniform(100_000, 20_000, 7)
        S = adb.gen_uniform(150_001, 20_000, 8)
    else:   # the largest build side the fixed table accepts
        R = adb.gen_pk(1 << 21, 9)
        S = adb.gen_fk(1 << 21, R, 0.0, 10)
    want = adb.join("NPO", R, S)
    dR, dS = _dev_copy(L, R), _dev_copy(L, S)
    out = C.c_void_p()
    assert L.adb_device_alloc(C.byref(out), 16) == 0
    try:
        for _ in range(2):
            st = f(dR, len(R), dS, len(S), out.value, None)
            assert st == 0, L.adb_last_error().decode()
            assert L.adb_device_sync() == 0
            got = np.zeros(2, np.uint64)
            assert L.adb_memcpy_d2h(got.ctypes.data, out.value, 16) == 0
            assert (int(got[0]), int(got[1])) == (want.count, want.checksum)
    finally:
        for p in (dR, dS, out.value):
            L.adb_device_free(p)


def test_noalloc_rejects_oversized_build():
    L = adb.lib()
    f = L.adb_npo_join_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
    # pointers are never dereferenced: the size check comes first
    st = f(C.c_void_p(16), (1 << 21) + 1, C.c_void_p(16), 4, C.c_void_p(16), None)
    assert st == adb.ADB_ERR_ARG
    assert "exceeds" in L.adb_last_error().decode()
