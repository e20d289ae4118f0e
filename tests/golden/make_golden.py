"""Regenerate the golden fixtures under tests/golden/.

Run on the machine that has the AllianceDB sources (the reference binaries
oracle/_ref/adb_ref_ck_{hash,sort} are built from them by
`make -C oracle ck REF_ROOT=<AllianceDB tree>`):

    python tests/golden/make_golden.py

Each case stores its relations (uint64 words key << 32 | payload, .npy) and, in
cases.json, the expected match count and checksum:
  * ref[label]       count and checksum of the reference's own join code run on
                     the case (every hashing join but the HS model, which does
                     not finish in this reference, and m-way / m-pass /
                     m-way+skew), the checksum taken at the reference's match
                     sites; or the error the reference run ended with;
  * count, checksum  the oracle's independent sort-based truth.
The relations come from `gen_numpy`, a numpy restatement of the seeded
generator of the library (alliancedb_b200/csrc/datagen.cuh); tests check that
the library's generator reproduces them exactly.
"""
from __future__ import annotations

import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

M64 = (1 << 64) - 1


def fmix64(z):
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def mix3(seed, stream, i):
    with np.errstate(over="ignore"):
        a = fmix64(np.uint64((seed + stream * 0x632BE59BD9B4E019) & M64))
        b = np.asarray(i, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15) + np.uint64(1)
    return fmix64(a ^ b)


def uniform_below(seed, stream, i, n):
    x = mix3(seed, stream, i)
    hi, lo = x >> np.uint64(32), x & np.uint64(0xFFFFFFFF)
    # floor(x * n / 2^64) for n < 2^32, in 64-bit pieces
    n = np.uint64(n)
    return ((hi * n) + ((lo * n) >> np.uint64(32))) >> np.uint64(32)


class Feistel:
    def __init__(self, n, seed):
        bits = 2
        while bits < 64 and (1 << bits) < n:
            bits += 1
        bits = (bits + 1) & ~1
        self.n, self.half = n, bits // 2
        self.hmask = np.uint64((1 << self.half) - 1)
        self.k = [mix3(seed, 1000 + r, 0) for r in range(4)]

    def once(self, x):
        L, R = x >> np.uint64(self.half), x & self.hmask
        for r in range(4):
            L, R = R, L ^ (fmix64(self.k[r] ^ R) & self.hmask)
        return (L << np.uint64(self.half)) | R

    def __call__(self, i):
        x = self.once(np.asarray(i, dtype=np.uint64))
        bad = x >= np.uint64(self.n)
        while bad.any():
            x[bad] = self.once(x[bad])
            bad = x >= np.uint64(self.n)
        return x


def words(keys, pays):
    return (np.asarray(keys, np.uint64) << np.uint64(32)) | np.asarray(pays, np.uint64)


def gen_numpy_pk(n, seed):
    i = np.arange(n, dtype=np.uint64)
    return words(np.uint64(1) + Feistel(max(n, 1), seed)(i), i)


def gen_numpy_fk_uniform(nS, R, seed):
    j = np.arange(nS, dtype=np.uint64)
    idx = uniform_below(seed, 3, j, len(R)).astype(np.int64)
    return words(R[idx] >> np.uint64(32), j)


def gen_numpy_uniform(n, key_range, seed):
    i = np.arange(n, dtype=np.uint64)
    return words(np.uint64(1) + uniform_below(seed, 5, i, key_range), i)


def cases():
    out = {}
    R = gen_numpy_pk(1000, 1)
    out["fk_1000"] = (R, gen_numpy_fk_uniform(1000, R, 2))
    R = gen_numpy_pk(4096, 3)
    out["fk_4096_x_6000"] = (R, gen_numpy_fk_uniform(6000, R, 4))
    out["dups_3000_2500"] = (gen_numpy_uniform(3000, 500, 5), gen_numpy_uniform(2500, 500, 6))
    out["all_equal_200_300"] = (words(np.full(200, 77), np.arange(200)), words(np.full(300, 77), np.arange(300)))
    keys_r = np.array([0, 0xFFFFFFFF, 1, 0x80000000, 0xFFFFFFFF, 0, 7, 9], np.uint64)
    pays_r = np.array([0xFFFFFFFF, 0xFFFFFFFF, 5, 6, 0, 9, 0xFFFFFFFF, 1], np.uint64)
    keys_s = np.array([0xFFFFFFFF, 0, 0x80000000, 3, 0xFFFFFFFF, 7, 9, 9], np.uint64)
    pays_s = np.array([1, 2, 3, 4, 0xFFFFFFFF, 6, 7, 8], np.uint64)
    out["extreme_keys"] = (words(keys_r, pays_r), words(keys_s, pays_s))
    out["non_pow2_1023_x_777"] = (gen_numpy_uniform(1023, 900, 7), gen_numpy_uniform(777, 900, 8))
    return out


# The reference's joins recorded per case: (label, binary, algorithm, threads).
# Threads: 4 for the eager distribution models (JB / JBCR split work by
# thread) and the partitioned joins; NPO at 1 thread (its multi-threaded build
# loses tuples at random on repeated keys, so no fixture can hold it); the
# sort-merge joins at 1 and at 4 threads.
REF_RUNS = [(a, "hash", a, 4) for a in ("PRO", "PRH", "RJ_st", "NPO_st", "SHJ_st", "SHJ_JM_NP", "SHJ_JB_NP",
                                        "SHJ_JBCR_NP", "PMJ_st", "PMJ_JM_NP", "PMJ_JB_NP", "PMJ_JBCR_NP")] + \
           [("NPO@1", "hash", "NPO", 1)] + \
           [(f"{a}@{t}", "sort", a, t) for a in ("m-way", "m-pass", "m-way+skew") for t in (1, 4)]
REF_BIN = {"hash": ROOT / "oracle" / "_ref" / "adb_ref_ck_hash", "sort": ROOT / "oracle" / "_ref" / "adb_ref_ck_sort"}


def run_ref(kind, algo, threads, rf, sf):
    """One reference join on the relation files: {"count", "checksum"} or {"error"}."""
    res = subprocess.run([str(REF_BIN[kind]), algo, "files", str(rf), str(sf), str(threads)], capture_output=True,
                         text=True, timeout=120)
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    if res.returncode != 0 or not lines:
        return {"error": f"exit status {res.returncode}"}
    d = json.loads(lines[-1])
    return {"count": d["count"], "checksum": str(d["checksum"])}


def main():
    from tests.oracle_bind import Oracle
    for b in REF_BIN.values():
        if not b.exists():
            sys.exit(f"{b} is missing: run `make -C oracle ck REF_ROOT=<AllianceDB tree>` first")
    o = Oracle()
    meta = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, (R, S) in cases().items():
            np.save(HERE / f"{name}_R.npy", R)
            np.save(HERE / f"{name}_S.npy", S)
            count, checksum = o.truth(R, S)
            rf, sf = Path(tmp) / "R.bin", Path(tmp) / "S.bin"
            R.tofile(rf)
            S.tofile(sf)
            ref = {label: run_ref(kind, algo, t, rf, sf) for label, kind, algo, t in REF_RUNS}
            meta[name] = {"n_r": int(len(R)), "n_s": int(len(S)), "count": count, "checksum": str(checksum),
                          "ref": ref}
    (HERE / "cases.json").write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
    print(json.dumps(meta, indent=1))


if __name__ == "__main__":
    main()
