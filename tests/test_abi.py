"""The C ABI of libadb_b200.so, checked without a GPU.

The library must load, export every entry point include/adb/*.h declares, keep
the reference's algorithm names (hashing/main.cpp:306-338, sorting/main.cpp:481-486)
and reject bad calls with status codes before touching a device.  Compute calls
themselves are the GPU tests' job.
"""
import ctypes as C
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import alliancedb_b200 as adb

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").rglob("*.h"))

# hashing/main.cpp:306-338 and sorting/main.cpp:481-486
HASHING = ["PRO", "RJ_st", "PRH", "PRHO", "NPO", "NPO_st", "SHJ_st", "SHJ_JM_P", "SHJ_JM_NP", "SHJ_JB_NP",
           "SHJ_JBCR_NP", "SHJ_JBCR_P", "SHJ_HS_NP", "PMJ_st", "PMJ_JM_NP", "PMJ_JM_P", "PMJ_JB_NP", "PMJ_JBCR_NP",
           "PMJ_JBCR_P", "PMJ_HS_NP", "RPJ_st", "RPJ_JM_NP", "RPJ_JB_NP", "RPJ_JBCR_NP", "RPJ_HS_NP"]
SORTING = ["m-way", "m-pass", "mpsm", "m-way+skew"]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(adb_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_headers_declare_the_entry_points():
    names = declared_functions()
    for must in ("adb_join", "adb_join_device", "adb_stream_join", "adb_batch_join_device", "adb_npo_join_noalloc",
                 "adb_serve_run", "adb_batch_autotune"):
        assert must in names, must


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", str(adb.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = declared_functions() - exported
    assert not missing, missing


def test_library_loads_and_binds_without_a_gpu():
    L = adb.lib()
    assert L.adb_version().decode().startswith("adb_b200")
    for name in declared_functions():
        assert hasattr(L, name)


def test_algorithm_registry_keeps_the_reference_names():
    algos = adb.algorithms()
    assert set(HASHING + SORTING) <= set(algos)
    not_provided = {k for k, v in algos.items() if not v}
    # the reference's ripple joins are unfinished (hashing/main.cpp:331) and mpsm is a stub
    # (sorting/joins/sortmergejoin_mpsm.cpp:38-42)
    assert not_provided == {"RPJ_st", "RPJ_JM_NP", "RPJ_JB_NP", "RPJ_JBCR_NP", "RPJ_HS_NP", "mpsm"}


def test_param_defaults_follow_the_reference():
    p = adb.default_params()
    # hashing/main.cpp:340-390 defaultParam
    assert (p.window_size, p.step_size_r, p.step_size_s, p.interval) == (1000, 1600, 1600, 1)
    assert (p.progressive_step, p.merge_step, p.group_size) == (1, 2, 2)


def test_errors_before_the_device():
    R = adb.gen_pk(10, 1)
    with pytest.raises(adb.AdbError) as e:
        adb.join("NOPE", R, R)
    assert e.value.status == adb.ADB_ERR_ARG
    with pytest.raises(adb.AdbError) as e:
        adb.join("RPJ_st", R, R)
    assert e.value.status == adb.ADB_ERR_UNSUPPORTED
    with pytest.raises(adb.AdbError) as e:
        adb.join("mpsm", R, R)
    assert e.value.status == adb.ADB_ERR_UNSUPPORTED
    L = adb.lib()
    r = adb.JoinResult()
    # relations of 2^32 tuples or more are refused by size alone (pointers never read)
    st = L.adb_join_device(b"PRO", C.c_void_p(16), 1 << 32, C.c_void_p(16), 4, None, C.byref(r), None)
    assert st == adb.ADB_ERR_ARG
    st = L.adb_join(b"PRO", None, 5, None, 0, None, C.byref(r))
    assert st == adb.ADB_ERR_ARG


@pytest.mark.skipif(shutil.which("nvidia-smi") is not None, reason="this machine has a GPU")
def test_no_device_is_reported_not_hidden():
    R = adb.gen_pk(100, 1)
    with pytest.raises(adb.AdbError) as e:
        adb.join("PRO", R, R)
    assert e.value.status == adb.ADB_ERR_NO_DEVICE


def test_stream_join_argument_checks():
    R = np.zeros(3, dtype=adb.STREAM_TUPLE)
    R["ts_ms"] = [5, 3, 9]   # not ordered
    with pytest.raises(adb.AdbError) as e:
        adb.stream_join("SHJ_JM_NP", R, R[:0])
    assert e.value.status == adb.ADB_ERR_ARG
    with pytest.raises(adb.AdbError) as e:
        adb.stream_join("PRO", R[:0], R[:0])
    assert e.value.status == adb.ADB_ERR_ARG
