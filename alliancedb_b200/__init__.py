"""alliancedb_b200 -- B200-native join hot path of AllianceDB, driven through its C ABI.

The native library ``libadb_b200.so`` (CUDA, sm_100a) holds every kernel and
the host orchestration (C++).  This module is a thin ctypes binding used by the
tests and the benchmark; it adds no compute of its own and has no CPU
fallback: if the library is missing or no B200 is visible, calls raise.

Relations are numpy arrays of dtype ``TUPLE`` (``{payload: u4, key: u4}``,
the reference's tuple_t layout, hashing/utils/types.h:67-70) or uint64 words
``key << 32 | payload``; device relations are raw pointers (ints), for example
``torch.Tensor.data_ptr()``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libadb_b200.so"

TUPLE = np.dtype([("payload", "<u4"), ("key", "<u4")])

ADB_OK, ADB_ERR_ARG, ADB_ERR_OOM, ADB_ERR_DEVICE, ADB_ERR_TIMEOUT, ADB_ERR_UNSUPPORTED, ADB_ERR_BUSY, \
    ADB_ERR_NO_DEVICE = range(8)
STATUS_NAMES = ["OK", "ERR_ARG", "ERR_OOM", "ERR_DEVICE", "ERR_TIMEOUT", "ERR_UNSUPPORTED", "ERR_BUSY",
                "ERR_NO_DEVICE"]


class JoinParams(C.Structure):
    _fields_ = [
        ("nthreads", C.c_uint32),
        ("window_size", C.c_int32),
        ("step_size_r", C.c_int32),
        ("step_size_s", C.c_int32),
        ("interval", C.c_int32),
        ("group_size", C.c_int32),
        ("progressive_step", C.c_int32),
        ("merge_step", C.c_int32),
        ("radix_bits", C.c_int32),
        ("part_fanout", C.c_int32),
        ("materialize", C.c_int32),
        ("batch_tuples", C.c_int32),
        ("seed", C.c_uint64),
        ("realtime", C.c_int32),
        ("test_flags", C.c_int32),
    ]


class JoinResult(C.Structure):
    _fields_ = [
        ("count", C.c_uint64),
        ("checksum", C.c_uint64),
        ("status", C.c_int32),
        ("kernels", C.c_int32),
        ("ms_device", C.c_float),
        ("ms_phase", C.c_float * 4),
        ("ms_h2d", C.c_float),
        ("materialized", C.c_uint64),
    ]


class StreamTuple(C.Structure):
    _fields_ = [("ts_ms", C.c_uint64), ("payload", C.c_uint32), ("key", C.c_uint32)]


class WindowResult(C.Structure):
    _fields_ = [
        ("window_start_ms", C.c_uint64),
        ("n_r", C.c_uint64),
        ("n_s", C.c_uint64),
        ("count", C.c_uint64),
        ("checksum", C.c_uint64),
        ("latency_ms", C.c_float),
        ("reserved", C.c_float),
    ]


class WindowProgress(C.Structure):
    """adb_window_progress: ms to pct = 1, 5, 10, 25, 50, 75, 95, 99, 100 % of a
    window's matches, and match-weighted batch latency percentiles (ms)."""
    PCT = (1, 5, 10, 25, 50, 75, 95, 99, 100)
    _fields_ = [
        ("t_pct", C.c_float * 9),
        ("lat_p50", C.c_float),
        ("lat_p95", C.c_float),
        ("lat_p99", C.c_float),
        ("batches", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


class ServeRequest(C.Structure):
    _fields_ = [("arrival_us", C.c_uint64), ("n_r", C.c_uint32), ("n_s", C.c_uint32), ("seed", C.c_uint64)]


class ServeResult(C.Structure):
    _fields_ = [("count", C.c_uint64), ("checksum", C.c_uint64), ("latency_ms", C.c_float),
                ("queue_ms", C.c_float), ("batch", C.c_uint32), ("status", C.c_int32)]


class ServeConfig(C.Structure):
    _fields_ = [("budget_bytes", C.c_uint64), ("max_batch", C.c_uint32), ("realtime", C.c_int32),
                ("slots", C.c_uint32), ("reserved", C.c_uint32)]


class ServeStats(C.Structure):
    _fields_ = [("requests", C.c_uint64), ("tuples", C.c_uint64), ("batches", C.c_uint64),
                ("makespan_ms", C.c_double), ("tuples_per_s", C.c_double), ("p50_ms", C.c_double),
                ("p99_ms", C.c_double), ("p999_ms", C.c_double), ("mean_batch", C.c_double),
                ("peak_arena_bytes", C.c_uint64), ("arena_bytes", C.c_uint64)]


STREAM_TUPLE = np.dtype([("ts_ms", "<u8"), ("payload", "<u4"), ("key", "<u4")])
assert STREAM_TUPLE.itemsize == C.sizeof(StreamTuple) == 16


class AdbError(RuntimeError):
    def __init__(self, status: int, msg: str):
        self.status = status
        name = STATUS_NAMES[status] if 0 <= status < len(STATUS_NAMES) else str(status)
        super().__init__(f"{name}: {msg}")


_lib = None

# every entry point of include/adb/adb_join.h: name -> (restype, argtypes)
_P = C.c_void_p
_U64 = C.c_uint64
_SIGS = {
    "adb_params_default": (None, [C.POINTER(JoinParams)]),
    "adb_last_error": (C.c_char_p, []),
    "adb_version": (C.c_char_p, []),
    "adb_algo_count": (C.c_int, []),
    "adb_algo_name": (C.c_char_p, [C.c_int, C.POINTER(C.c_int)]),
    "adb_join": (C.c_int, [C.c_char_p, _P, _U64, _P, _U64, C.POINTER(JoinParams), C.POINTER(JoinResult)]),
    "adb_join_device": (C.c_int, [C.c_char_p, _P, _U64, _P, _U64, C.POINTER(JoinParams),
                                  C.POINTER(JoinResult), _P]),
    "adb_join_materialize_device": (C.c_int, [C.c_char_p, _P, _U64, _P, _U64, C.POINTER(JoinParams), _P, _U64,
                                              C.POINTER(JoinResult), _P]),
    "adb_stream_join_progress": (C.c_int, [C.c_char_p, _P, _U64, _P, _U64, C.POINTER(JoinParams),
                                           C.POINTER(WindowResult), C.POINTER(WindowProgress), _U64,
                                           C.POINTER(C.c_uint64)]),
    "adb_stream_join": (C.c_int, [C.c_char_p, _P, _U64, _P, _U64, C.POINTER(JoinParams),
                                  C.POINTER(WindowResult), _U64, C.POINTER(C.c_uint64)]),
    "adb_batch_join_device": (C.c_int, [_P, C.POINTER(C.c_uint64), _P, C.POINTER(C.c_uint64), C.c_uint32,
                                        C.c_int, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                        C.POINTER(C.c_float), _P]),
    "adb_batch_autotune": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "adb_serve_run": (C.c_int, [C.POINTER(ServeConfig), C.POINTER(ServeRequest), C.c_uint32,
                                C.POINTER(ServeResult), C.POINTER(ServeStats)]),
    "adb_batch_set_tuning": (C.c_int, [C.POINTER(C.c_int)]),
    "adb_npo_join_noalloc": (C.c_int, [_P, _U64, _P, _U64, _P, _P]),
    "adb_shard_split": (C.c_int, [_P, _U64, C.c_uint32, _P, C.POINTER(C.c_uint64), _P]),
    "adb_device_alloc": (C.c_int, [C.POINTER(C.c_void_p), C.c_size_t]),
    "adb_device_free": (C.c_int, [_P]),
    "adb_host_alloc_pinned": (C.c_int, [C.POINTER(C.c_void_p), C.c_size_t]),
    "adb_host_free_pinned": (C.c_int, [_P]),
    "adb_memcpy_h2d": (C.c_int, [_P, _P, C.c_size_t]),
    "adb_memcpy_d2h": (C.c_int, [_P, _P, C.c_size_t]),
    "adb_device_sync": (C.c_int, []),
    "adb_release_workspace": (C.c_int, []),
    "adb_gen_pk": (C.c_int, [_P, _U64, _U64, C.c_int]),
    "adb_gen_fk": (C.c_int, [_P, _U64, _P, _U64, C.c_double, _U64, _P, C.c_int]),
    "adb_gen_uniform": (C.c_int, [_P, _U64, _U64, _U64, C.c_int]),
    "adb_load_relation": (C.c_int, [C.c_char_p, C.c_int32, C.c_int32, C.c_uint32, _U64, _P, _P]),
}


def lib() -> C.CDLL:
    """Load libadb_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m alliancedb_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(status: int) -> None:
    if status != ADB_OK:
        raise AdbError(status, lib().adb_last_error().decode())


def default_params(**kw) -> JoinParams:
    p = JoinParams()
    lib().adb_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def algorithms() -> dict[str, bool]:
    L = lib()
    out = {}
    for i in range(L.adb_algo_count()):
        prov = C.c_int(0)
        name = L.adb_algo_name(i, C.byref(prov)).decode()
        out[name] = bool(prov.value)
    return out


def as_words(rel: np.ndarray) -> np.ndarray:
    """View a TUPLE array (or uint64 words) as contiguous uint64 words."""
    rel = np.ascontiguousarray(rel)
    if rel.dtype == np.uint64:
        return rel
    if rel.dtype == TUPLE:
        return rel.view(np.uint64)
    raise TypeError(f"relation dtype {rel.dtype} is neither TUPLE nor uint64")


def tuples(keys, payloads=None) -> np.ndarray:
    keys = np.asarray(keys, dtype=np.uint32)
    out = np.empty(keys.shape[0], dtype=TUPLE)
    out["key"] = keys
    out["payload"] = np.arange(keys.shape[0], dtype=np.uint32) if payloads is None else payloads
    return out


@dataclass
class Result:
    count: int
    checksum: int
    ms_device: float
    ms_phase: tuple
    ms_h2d: float
    kernels: int
    materialized: int = 0


def _result(r: JoinResult) -> Result:
    return Result(r.count, r.checksum, r.ms_device, tuple(r.ms_phase), r.ms_h2d, r.kernels, r.materialized)


def join(algo: str, R: np.ndarray, S: np.ndarray, params: JoinParams | None = None) -> Result:
    """Join host relations through adb_join (copies in, joins, reads back)."""
    Rw, Sw = as_words(R), as_words(S)
    r = JoinResult()
    st = lib().adb_join(algo.encode(), Rw.ctypes.data if Rw.size else None, Rw.size,
                        Sw.ctypes.data if Sw.size else None, Sw.size,
                        C.byref(params) if params is not None else None, C.byref(r))
    _check(st)
    return _result(r)


CUDA_STREAM_LEGACY = 1   # cudaStreamLegacy, the legacy default stream


def stream_handle(stream) -> int | None:
    """The cudaStream_t to hand the C API for `stream`: None keeps the
    library's own stream (NULL there, a non-blocking stream that is not ordered
    with the legacy default stream); a torch.cuda.Stream or a raw handle is
    passed on, and handle 0, torch's default stream (the legacy NULL stream),
    becomes cudaStreamLegacy so that the work is ordered with what torch and
    torch.distributed queue on that stream."""
    if stream is None:
        return None
    h = stream if isinstance(stream, int) else stream.cuda_stream
    return h or CUDA_STREAM_LEGACY


def join_device(algo: str, dR: int, nR: int, dS: int, nS: int, params: JoinParams | None = None,
                stream=None) -> Result:
    """Join device-resident relations (raw device pointers) through
    adb_join_device, on `stream` (see stream_handle)."""
    r = JoinResult()
    st = lib().adb_join_device(algo.encode(), dR or None, nR, dS or None, nS,
                               C.byref(params) if params is not None else None, C.byref(r), stream_handle(stream))
    _check(st)
    return _result(r)


def join_materialize_device(algo: str, dR: int, nR: int, dS: int, nS: int, dOut: int, cap: int,
                            params: JoinParams | None = None) -> Result:
    r = JoinResult()
    st = lib().adb_join_materialize_device(algo.encode(), dR or None, nR, dS or None, nS,
                                           C.byref(params) if params is not None else None, dOut or None, cap,
                                           C.byref(r), None)
    _check(st)
    return _result(r)


def stream_join(algo: str, R: np.ndarray, S: np.ndarray, params: JoinParams | None = None,
                max_windows: int = 1 << 16, progress: bool = False):
    """Windowed eager join of two timestamp-ordered STREAM_TUPLE arrays: the
    per-window results, and with progress=True also their WindowProgress
    (adb_stream_join_progress) as a second list."""
    R = np.ascontiguousarray(R, dtype=STREAM_TUPLE)
    S = np.ascontiguousarray(S, dtype=STREAM_TUPLE)
    out = (WindowResult * max_windows)()
    prog = (WindowProgress * max_windows)() if progress else None
    nw = C.c_uint64(0)
    st = lib().adb_stream_join_progress(algo.encode(), R.ctypes.data if R.size else None, R.size,
                                        S.ctypes.data if S.size else None, S.size,
                                        C.byref(params) if params is not None else None, out, prog, max_windows,
                                        C.byref(nw))
    _check(st)
    n = min(nw.value, max_windows)
    wins = [out[i] for i in range(n)]
    return (wins, [prog[i] for i in range(n)]) if progress else wins


def batch_join_device(dR: int, r_off: np.ndarray, dS: int, s_off: np.ndarray, mode: int = 0):
    """Join many device-resident windows; returns (counts, checksums, ms_device)."""
    r_off = np.ascontiguousarray(r_off, dtype=np.uint64)
    s_off = np.ascontiguousarray(s_off, dtype=np.uint64)
    nw = r_off.size - 1
    counts = np.zeros(nw, dtype=np.uint64)
    sums = np.zeros(nw, dtype=np.uint64)
    ms = C.c_float(0)
    u64p = C.POINTER(C.c_uint64)
    st = lib().adb_batch_join_device(dR or None, r_off.ctypes.data_as(u64p), dS or None,
                                     s_off.ctypes.data_as(u64p), nw, mode, counts.ctypes.data_as(u64p),
                                     sums.ctypes.data_as(u64p), C.byref(ms), None)
    _check(st)
    return counts, sums, ms.value


def batch_autotune(lo: int, hi: int) -> list[int]:
    """Measure the per-window fan-out table for window sizes 2^lo .. 2^hi."""
    out = (C.c_int * 33)()
    _check(lib().adb_batch_autotune(lo, hi, out))
    return list(out)


def serve_run(requests, budget_bytes: int = 0, max_batch: int = 0, realtime: bool = True, slots: int = 0):
    """Run the serving loop; requests = iterable of (arrival_us, n_r, n_s, seed).
    Returns (list of ServeResult, ServeStats)."""
    reqs = list(requests)
    arr = (ServeRequest * max(len(reqs), 1))()
    for i, (t, nr, ns, seed) in enumerate(reqs):
        arr[i] = ServeRequest(int(t), int(nr), int(ns), int(seed))
    res = (ServeResult * max(len(reqs), 1))()
    st = ServeStats()
    cfg = ServeConfig(int(budget_bytes), int(max_batch), 1 if realtime else 0, int(slots), 0)
    _check(lib().adb_serve_run(C.byref(cfg), arr, len(reqs), res, C.byref(st)))
    return [res[i] for i in range(len(reqs))], st


def batch_set_tuning(bits: list[int] | None) -> None:
    if bits is None:
        _check(lib().adb_batch_set_tuning(None))
    else:
        arr = (C.c_int * 33)(*bits)
        _check(lib().adb_batch_set_tuning(arr))


class DeviceBuffer:
    """Device memory from the library's allocator (freed on close / garbage collection)."""

    def __init__(self, nbytes: int):
        p = C.c_void_p()
        _check(lib().adb_device_alloc(C.byref(p), max(int(nbytes), 16)))
        self.ptr, self.nbytes = p.value, int(nbytes)

    @classmethod
    def from_host(cls, arr: np.ndarray) -> "DeviceBuffer":
        arr = np.ascontiguousarray(arr)
        d = cls(arr.nbytes)
        if arr.nbytes:
            _check(lib().adb_memcpy_h2d(d.ptr, arr.ctypes.data, arr.nbytes))
        return d

    def to_host(self, dtype, count: int) -> np.ndarray:
        out = np.empty(count, dtype=dtype)
        if out.nbytes:
            _check(lib().adb_memcpy_d2h(out.ctypes.data, self.ptr, out.nbytes))
        return out

    def close(self):
        if self.ptr:
            lib().adb_device_free(self.ptr)
            self.ptr = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- generators (host) ----
def load_relation(path: str, num_tuples: int, key_col: int = 0, ts_col: int = 0, partitions: int = 1):
    """Relation of num_tuples records from a ',' or '|' separated text file, as
    the reference's file loader reads it (adb_load_relation): returns
    (tuples, timestamps); the timestamps are 0 when ts_col is 0."""
    t = np.empty(num_tuples, dtype=TUPLE)
    ts = np.empty(num_tuples, dtype=np.uint64)
    _check(lib().adb_load_relation(str(path).encode(), key_col, ts_col, partitions, num_tuples,
                                   t.ctypes.data if num_tuples else None, ts.ctypes.data if num_tuples else None))
    return t, ts


def gen_pk(n: int, seed: int) -> np.ndarray:
    out = np.empty(n, dtype=TUPLE)
    _check(lib().adb_gen_pk(out.ctypes.data if n else None, n, seed, 0))
    return out


def gen_fk(nS: int, R: np.ndarray, theta: float, seed: int, want_idx: bool = False):
    out = np.empty(nS, dtype=TUPLE)
    idx = np.empty(nS, dtype=np.uint32) if want_idx else None
    Rw = as_words(R)
    _check(lib().adb_gen_fk(out.ctypes.data if nS else None, nS, Rw.ctypes.data, Rw.size, float(theta), seed,
                            idx.ctypes.data if want_idx and nS else None, 0))
    return (out, idx) if want_idx else out


def gen_uniform(n: int, key_range: int, seed: int) -> np.ndarray:
    out = np.empty(n, dtype=TUPLE)
    _check(lib().adb_gen_uniform(out.ctypes.data if n else None, n, key_range, seed, 0))
    return out
