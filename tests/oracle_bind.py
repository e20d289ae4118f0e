"""ctypes binding of the CPU oracle (oracle/liboracle.so) -- test infrastructure only.

The oracle is the checker: tests compare the CUDA library's results with it.
It is built from oracle/adb_oracle.c by ``alliancedb_b200.build.build_oracle``.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
ORACLE_LIB = ROOT / "oracle" / "liboracle.so"

TUPLE = np.dtype([("payload", "<u4"), ("key", "<u4")])


class _Res(C.Structure):
    _fields_ = [("count", C.c_uint64), ("checksum", C.c_uint64)]


def _words(rel):
    rel = np.ascontiguousarray(rel)
    if rel.dtype == TUPLE:
        return rel.view(np.uint64)
    assert rel.dtype == np.uint64
    return rel


class Oracle:
    def __init__(self):
        if not ORACLE_LIB.exists():
            from alliancedb_b200.build import build_oracle
            build_oracle()
        L = C.CDLL(str(ORACLE_LIB))
        P, U = C.c_void_p, C.c_uint64
        R = C.POINTER(_Res)
        L.ora_pro.argtypes = [P, U, P, U, C.c_int, R]
        L.ora_prh.argtypes = [P, U, P, U, C.c_int, R]
        L.ora_npo.argtypes = [P, U, P, U, R]
        L.ora_smj.argtypes = [P, U, P, U, R]
        L.ora_shj.argtypes = [P, U, P, U, R]
        L.ora_pmj.argtypes = [P, U, P, U, U, U, R]
        L.ora_truth.argtypes = [P, U, P, U, R]
        L.ora_pk_truth.argtypes = [P, U, P, U, R]
        L.ora_materialize_sorted.argtypes = [P, U, P, U, P, U]
        L.ora_materialize_sorted.restype = U
        L.ora_pair_hash.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32]
        L.ora_pair_hash.restype = U
        for f in ("ora_pro", "ora_prh", "ora_npo", "ora_smj", "ora_shj", "ora_pmj", "ora_truth", "ora_pk_truth"):
            getattr(L, f).restype = C.c_int
        self.L = L

    def _call(self, fn, R, S, *extra):
        Rw, Sw = _words(R), _words(S)
        r = _Res()
        st = fn(Rw.ctypes.data if Rw.size else None, Rw.size, Sw.ctypes.data if Sw.size else None, Sw.size,
                *extra, C.byref(r))
        assert st == 0
        return int(r.count), int(r.checksum)

    def pro(self, R, S, bits=8):
        return self._call(self.L.ora_pro, R, S, bits)

    def prh(self, R, S, bits=8):
        return self._call(self.L.ora_prh, R, S, bits)

    def npo(self, R, S):
        return self._call(self.L.ora_npo, R, S)

    def smj(self, R, S):
        return self._call(self.L.ora_smj, R, S)

    def shj(self, R, S):
        return self._call(self.L.ora_shj, R, S)

    def pmj(self, R, S, step_r, step_s):
        return self._call(self.L.ora_pmj, R, S, step_r, step_s)

    def truth(self, R, S):
        return self._call(self.L.ora_truth, R, S)

    def pk_truth(self, R, S):
        """Truth for an R with unique keys, by direct addressing on the key
        (linear time; used at the benchmark's full sizes)."""
        Rw, Sw = _words(R), _words(S)
        r = _Res()
        st = self.L.ora_pk_truth(Rw.ctypes.data if Rw.size else None, Rw.size,
                                 Sw.ctypes.data if Sw.size else None, Sw.size, C.byref(r))
        if st != 0:
            raise ValueError(f"ora_pk_truth: R's keys repeat or are not dense (status {st})")
        return int(r.count), int(r.checksum)

    def pair_hash(self, key, rp, sp):
        return int(self.L.ora_pair_hash(key, rp, sp))

    def materialize_sorted(self, R, S, cap):
        Rw, Sw = _words(R), _words(S)
        out = np.zeros(max(cap, 1), dtype=np.uint64)
        n = self.L.ora_materialize_sorted(Rw.ctypes.data if Rw.size else None, Rw.size,
                                          Sw.ctypes.data if Sw.size else None, Sw.size, out.ctypes.data, cap)
        return int(n), out[:min(n, cap)]

    def by_name(self, algo, R, S, progressive_step=1):
        """The oracle function that restates reference algorithm `algo`."""
        if algo in ("PRO", "RJ_st"):
            return self.pro(R, S)
        if algo in ("PRH", "PRHO"):
            return self.prh(R, S)
        if algo in ("NPO", "NPO_st"):
            return self.npo(R, S)
        if algo in ("m-way", "m-pass", "m-way+skew"):
            return self.smj(R, S)
        if algo.startswith("SHJ"):
            return self.shj(R, S)
        if algo.startswith("PMJ"):
            nR, nS = len(R), len(S)
            return self.pmj(R, S, max(1, nR * progressive_step // 100), max(1, nS * progressive_step // 100))
        raise KeyError(algo)
