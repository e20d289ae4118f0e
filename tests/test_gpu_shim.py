"""The reference's call sites on the GPU library.

* oracle/_ref/adb_ref_bench_gpu: the hashing harness linked against
  alliancedb_b200/shim/reference_shim.cpp (the reference's
  `result_t *NAME(relation_t *, relation_t *, param_t)` functions implemented on
  libadb_b200.so) instead of the reference's join objects;
* oracle/_ref/adb_ref_sort_gpu: the sorting harness linked against
  alliancedb_b200/shim/reference_shim_sort.cpp (`sortmergejoin_multiway`,
  `_multipass`, `_multiway_skewhandling`, `_mpsm` with the reference's
  `(relation_t *, relation_t *, joinconfig_t *, int, int, int)` signature).
Counts and checksums must equal the reference's own joins on the same generated
input (oracle/_ref/adb_ref_ck_*, the checksum taken at the reference's match
sites) and the oracle's truth."""
import json
import subprocess
from pathlib import Path

import pytest

import alliancedb_b200 as adb

ROOT = Path(__file__).resolve().parent.parent
SHIM_BIN = ROOT / "oracle" / "_ref" / "adb_ref_bench_gpu"
REF_BIN = ROOT / "oracle" / "_ref" / "adb_ref_bench"
SHIM_SORT_BIN = ROOT / "oracle" / "_ref" / "adb_ref_sort_gpu"
REF_CK_SORT = ROOT / "oracle" / "_ref" / "adb_ref_ck_sort"
REF_CK_HASH = ROOT / "oracle" / "_ref" / "adb_ref_ck_hash"

pytestmark = pytest.mark.gpu

N = 1 << 18


def _run(binary, algo, n, threads=4):
    r = subprocess.run([str(binary), algo, "gen", str(n), str(threads), "1"], capture_output=True, text=True,
                       timeout=300)
    return r.returncode, r.stdout.strip().splitlines()[-1] if r.stdout.strip() else "", r.stderr


@pytest.fixture(scope="module")
def truth(oracle):
    if not SHIM_BIN.exists():
        pytest.skip("reference shim harness not built (needs the reference's headers at build time)")
    R = adb.gen_pk(N, 1)
    S = adb.gen_fk(N, R, 0.0, 2)
    return oracle.truth(R, S)


@pytest.mark.parametrize("algo", ["PRO", "RJ_st", "PRH", "PRHO", "NPO", "NPO_st", "SHJ_JM_NP", "SHJ_JB_NP",
                                  "SHJ_JBCR_NP", "PMJ_JM_NP", "PMJ_JB_NP"])
def test_shim_matches_reference_and_oracle(algo, truth):
    rc, line, err = _run(SHIM_BIN, algo, N)
    assert rc == 0, err
    got = json.loads(line)
    assert (got["count"], got["checksum"]) == truth, got
    if REF_BIN.exists() and algo in ("PRO", "RJ_st", "PRH", "NPO", "NPO_st"):
        rc, line, err = _run(REF_BIN, algo, N)
        assert rc == 0, err
        assert json.loads(line)["count"] == got["count"]


def test_shim_unsupported_returns_null(truth):
    # ripple joins are unfinished in the reference; the shim returns NULL and
    # the harness reports it
    rc, _, err = _run(SHIM_BIN, "RPJ_st", 1024)
    assert rc == 1 and "RPJ_st" in err


def _ref_ck(binary, algo, n, threads=4):
    rc, line, err = _run(binary, algo, n, threads)
    assert rc == 0, err
    d = json.loads(line)
    return d["count"], d["checksum"]


@pytest.mark.parametrize("algo", ["m-way", "m-pass", "m-way+skew"])
def test_sort_shim_matches_reference_and_oracle(algo, truth):
    if not SHIM_SORT_BIN.exists():
        pytest.skip("sorting shim harness not built (needs the reference's headers at build time)")
    rc, line, err = _run(SHIM_SORT_BIN, algo, N, 3)   # any thread count: no power-of-two rule on the GPU
    assert rc == 0, err
    got = json.loads(line)
    assert (got["count"], got["checksum"]) == truth, got
    if REF_CK_SORT.exists():
        assert _ref_ck(REF_CK_SORT, algo, N) == truth


def test_sort_shim_mpsm_returns_null(truth):
    if not SHIM_SORT_BIN.exists():
        pytest.skip("sorting shim harness not built")
    rc, _, err = _run(SHIM_SORT_BIN, "mpsm", 1024)
    assert rc == 1 and "mpsm" in err


@pytest.mark.parametrize("algo", ["PRO", "PRH", "NPO_st", "SHJ_JM_NP", "SHJ_JBCR_NP", "PMJ_JM_NP", "PMJ_JBCR_NP"])
def test_hash_shim_checksum_equals_reference_match_sites(algo, truth):
    """The reference's own joins with the checksum at their match sites, on the
    same generated input the shim ran: both equal the truth."""
    if not REF_CK_HASH.exists():
        pytest.skip("the reference's checksum build exists only where its sources were")
    assert _ref_ck(REF_CK_HASH, algo, N) == truth
