"""Synthetic workloads of the benchmark configurations beyond the single join.

* batch   4096 independent R/S window pairs, sizes log-uniform in [2^10, 2^22]
          per side, keys uniform over 4x the window size (match rate about
          0.25), a quarter of the windows Zipf(0.8) over that key range; joined
          by one launch sequence (mode 0) and by one sequence per window (mode 1)
* serve   open-loop Poisson arrivals at 2000 requests/s, sizes log-uniform in
          [2^12, 2^24] per side, FK relation with uniform keys, admission
          budget 120 GB; throughput and p50 / p99 / p999 latency
* stream  two streams of (ts, key, payload) at 1.6 M tuples/s each (Poisson
          arrivals), keys uniform over 2^20 values materialised 4 times,
          1000 ms tumbling windows, eager SHJ / PMJ

All data is seeded and synthetic (no public dataset is involved); every
workload generates its relations on the device from seeds unless stated.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import tempfile
import time
from pathlib import Path

import numpy as np

import alliancedb_b200 as adb

ROOT = Path(__file__).resolve().parent.parent
# algorithmic bytes per input tuple: partitioned (batched / served) 24, eager 16
ALG_BYTES_PARTITIONED = 24
ALG_BYTES_EAGER = 16


def hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())["hbm_gbs"], "measured"
    return 6650.0, "fallback"


def roofline(tuples_per_s: float, bytes_per_tuple: int):
    peak, kind = hbm_peak()
    gbs = tuples_per_s * bytes_per_tuple / 1e9
    return {"bound": "hbm", "alg_bytes_per_tuple": bytes_per_tuple, "achieved": gbs, "peak": peak,
            "unit": "GB/s", "frac": gbs / peak, "peak_source": kind}


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def ref_windows(algo: str, windows, threads: int, binary: str = "adb_ref_bench"):
    """The reference's own `algo` (oracle/_ref, compiled from its sources) on
    each (R, S) window of `windows` in turn, one call per window, on this host:
    returns the harness's JSON (tuples, count, summed call ms, tuples_per_s),
    or None when the reference build is absent."""
    ref = ROOT / "oracle" / "_ref" / binary
    if not ref.exists() or not windows:
        return None
    with tempfile.TemporaryDirectory(dir=os.environ.get("ADB_TMP")) as tmp:
        t = Path(tmp)
        r_off = np.concatenate([[0], np.cumsum([len(r) for r, _ in windows])]).astype(np.uint64)
        s_off = np.concatenate([[0], np.cumsum([len(s) for _, s in windows])]).astype(np.uint64)
        np.concatenate([adb.as_words(r) for r, _ in windows]).tofile(t / "R.bin")
        np.concatenate([adb.as_words(s) for _, s in windows]).tofile(t / "S.bin")
        np.concatenate([r_off, s_off]).tofile(t / "off.bin")
        out = subprocess.run([str(ref), algo, "windows", str(t / "R.bin"), str(t / "S.bin"), str(t / "off.bin"),
                              str(threads)], capture_output=True, text=True, timeout=1800, check=True).stdout
    return json.loads([ln for ln in out.splitlines() if ln.startswith("{")][-1])


def ref_arrivals(algo: str, R, S, threads: int):
    """The reference's own eager `algo` built with WAIT kept
    (oracle/_ref/adb_ref_hash_wait) on one window of two STREAM_TUPLE arrays
    whose payloads are their row numbers: every tuple is released at its
    timestamp (ms from the window's first), so the call lasts the window;
    returns the harness's JSON (count, call ms, last arrival, latency after
    it), or None when that build is absent."""
    ref = ROOT / "oracle" / "_ref" / "adb_ref_hash_wait"
    if not ref.exists() or not len(R) or not len(S):
        return None
    t0 = int(min(R["ts_ms"][0], S["ts_ms"][0]))
    with tempfile.TemporaryDirectory(dir=os.environ.get("ADB_TMP")) as tmp:
        t = Path(tmp)
        adb.tuples(R["key"], np.arange(len(R), dtype=np.uint32)).view(np.uint64).tofile(t / "R.bin")
        adb.tuples(S["key"], np.arange(len(S), dtype=np.uint32)).view(np.uint64).tofile(t / "S.bin")
        (R["ts_ms"].astype(np.uint64) - np.uint64(t0)).tofile(t / "tR.bin")
        (S["ts_ms"].astype(np.uint64) - np.uint64(t0)).tofile(t / "tS.bin")
        out = subprocess.run([str(ref), algo, "arrivals", *(str(t / f) for f in ("R.bin", "S.bin", "tR.bin", "tS.bin")),
                              str(threads)], capture_output=True, text=True, timeout=600, check=True).stdout
    return json.loads([ln for ln in out.splitlines() if ln.startswith("{")][-1])


def _logu(rng, lo, hi, n):
    return np.floor(2.0 ** rng.uniform(lo, hi, size=n)).astype(np.uint64)


def batch_windows(n_windows: int, lo: int, hi: int, seed: int):
    """Device-resident batch: returns (dR, r_off, dS, s_off, keepalive)."""
    rng = np.random.default_rng(seed)
    nr = _logu(rng, lo, hi, n_windows)
    ns = _logu(rng, lo, hi, n_windows)
    zipf = rng.random(n_windows) < 0.25
    r_off = np.concatenate([[0], np.cumsum(nr)]).astype(np.uint64)
    s_off = np.concatenate([[0], np.cumsum(ns)]).astype(np.uint64)
    L = adb.lib()
    dR = adb.DeviceBuffer(int(r_off[-1]) * 8 + 16)
    dS = adb.DeviceBuffer(int(s_off[-1]) * 8 + 16)
    keep = [dR, dS]
    dom_cap = int(4 * max(nr.max(), ns.max()))
    dom = adb.DeviceBuffer(dom_cap * 8)
    keep.append(dom)
    for w in range(n_windows):
        krange = int(4 * max(nr[w], ns[w]))
        pr, ps = dR.ptr + int(r_off[w]) * 8, dS.ptr + int(s_off[w]) * 8
        if zipf[w]:
            # key domain 1..krange through a seeded permutation, both sides Zipf(0.8) over it
            adb._check(L.adb_gen_pk(dom.ptr, krange, 7000 + w, 1))
            adb._check(L.adb_gen_fk(pr, int(nr[w]), dom.ptr, krange, C.c_double(0.8), 8000 + w, None, 1))
            adb._check(L.adb_gen_fk(ps, int(ns[w]), dom.ptr, krange, C.c_double(0.8), 9000 + w, None, 1))
        else:
            adb._check(L.adb_gen_uniform(pr, int(nr[w]), krange, 7000 + w, 1))
            adb._check(L.adb_gen_uniform(ps, int(ns[w]), krange, 8000 + w, 1))
    return dR.ptr, r_off, dS.ptr, s_off, keep


def _batch_cpu_sample(dR, r_off, dS, s_off, max_tuples=1 << 25, max_windows=256, seed=5):
    """A seeded random sample of the batch's windows, copied to the host, of at
    most max_windows windows and about max_tuples tuples."""
    L = adb.lib()
    rng = np.random.default_rng(seed)
    out, total = [], 0
    for w in rng.permutation(len(r_off) - 1):
        nr, ns = int(r_off[w + 1] - r_off[w]), int(s_off[w + 1] - s_off[w])
        if out and total + nr + ns > max_tuples:
            continue
        R = np.empty(nr, np.uint64)
        S = np.empty(ns, np.uint64)
        adb._check(L.adb_memcpy_d2h(R.ctypes.data, dR + int(r_off[w]) * 8, nr * 8))
        adb._check(L.adb_memcpy_d2h(S.ctypes.data, dS + int(s_off[w]) * 8, ns * 8))
        out.append((R, S))
        total += nr + ns
        if len(out) >= max_windows or total >= max_tuples:
            break
    return out


def bench_batch(args, cpu: bool = True):
    lo, hi = 10, 22
    dR, r_off, dS, s_off, keep = batch_windows(args.windows, lo, hi, 11)
    tuples = int(r_off[-1] + s_off[-1])
    table = adb.batch_autotune(lo, hi)
    c0, k0, _ = adb.batch_join_device(dR, r_off, dS, s_off, 0)   # warm-up
    ms0 = []
    for _ in range(max(1, args.steps // 2)):
        c, k, ms = adb.batch_join_device(dR, r_off, dS, s_off, 0)
        assert np.array_equal(c, c0) and np.array_equal(k, k0)
        ms0.append(ms)
    c1, k1, ms1 = adb.batch_join_device(dR, r_off, dS, s_off, 1)
    assert np.array_equal(c1, c0) and np.array_equal(k1, k0), "per-window and batched results differ"
    best0 = float(np.median(ms0))
    v0, v1 = tuples / (best0 / 1e3), tuples / (ms1 / 1e3)
    out = {"metric": "batched windows join input tuples/s", "value": v0, "unit": "tuples/s",
           "higher_is_better": True, "n_gpus": 1, "data": "synthetic",
           "config": {"workload": f"{args.windows} window pairs, sizes log-uniform [2^{lo}, 2^{hi}] per side, "
                                  "keys uniform over 4x window size, 25% windows Zipf 0.8",
                      "windows": args.windows, "tuples": tuples},
           "ms_batched": best0, "ms_per_window_launches": ms1, "per_window_value": v1,
           "speedup_batched_vs_per_window": v0 / v1, "matches": int(c0.sum()),
           "roofline": roofline(v0, ALG_BYTES_PARTITIONED),
           "fanout_bits_by_size_bucket": table[lo:hi + 1]}
    if cpu:
        sample = _batch_cpu_sample(dR, r_off, dS, s_off)
        th = host_threads()
        d = ref_windows("PRO", sample, th)
        if d is not None:
            out["cpu_baseline"] = {"value": d["tuples_per_s"], "unit": "tuples/s", "cores": th, "kind": "reference",
                                   "sample": f"reference PRO run per window, one window after the other, on "
                                             f"{d['windows']} windows ({d['tuples']} tuples) drawn at random from "
                                             f"the batch, {th} threads; {d['count']} matches"}
    del keep
    return out


def serve_requests(n: int, seed: int = 21):
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1e6 / 2000.0, size=n))
    nr = _logu(rng, 12, 24, n)
    ns = _logu(rng, 12, 24, n)
    return [(int(t[i]), int(nr[i]), int(ns[i]), 5000 + i) for i in range(n)], t, nr, ns


def bench_serve(args, cpu: bool = True):
    n = args.requests
    reqs, t, nr, ns = serve_requests(n)
    adb.serve_run(reqs[:50], budget_bytes=120 << 30, max_batch=256, realtime=False)   # warm-up
    res, st = adb.serve_run(reqs, budget_bytes=120 << 30, max_batch=256, realtime=True)
    assert all(r.status == 0 and r.count == reqs[i][2] for i, r in enumerate(res))
    out = {"metric": "served join input tuples/s", "value": st.tuples_per_s, "unit": "tuples/s",
           "higher_is_better": True, "n_gpus": 1, "data": "synthetic",
           "config": {"workload": f"{n} requests, Poisson 2000 req/s, sizes log-uniform [2^12, 2^24] per side, "
                                  "FK uniform keys, budget 120 GB", "requests": n},
           "latency_ms": {"p50": st.p50_ms, "p99": st.p99_ms, "p999": st.p999_ms},
           "batches": int(st.batches), "mean_batch": st.mean_batch, "makespan_ms": st.makespan_ms,
           "offered_tuples_per_s": float((nr + ns).sum() / (t[-1] / 1e6)),
           "roofline": roofline(st.tuples_per_s, ALG_BYTES_PARTITIONED),
           "peak_arena_gb": st.peak_arena_bytes / 2**30}
    if cpu:
        # the first requests, generated on the host exactly as the device generates them
        sample, total = [], 0
        for (_, a, b, seed) in reqs:
            if sample and total + a + b > (1 << 26):
                break
            R = adb.gen_pk(a, seed)
            sample.append((R, adb.gen_fk(b, R, 0.0, seed + 1)))
            total += a + b
        th = host_threads()
        d = ref_windows("PRO", sample, th)
        if d is not None:
            out["cpu_baseline"] = {"value": d["tuples_per_s"], "unit": "tuples/s", "cores": th, "kind": "reference",
                                   "sample": f"reference PRO run per request, one after the other (no arrival "
                                             f"gaps), on the first {d['windows']} requests ({d['tuples']} tuples), "
                                             f"{th} threads; {d['count']} matches"}
    return out


def make_streams(seconds: float, rate_per_s: float, key_space: int, dup: int, seed: int):
    rng = np.random.default_rng(seed)
    out = []
    for side in range(2):
        n = int(seconds * rate_per_s)
        n -= n % dup
        ts = np.floor(np.cumsum(rng.exponential(1000.0 / rate_per_s, size=n))).astype(np.uint64)
        base = rng.integers(1, key_space + 1, size=n // dup, dtype=np.uint64).astype(np.uint32)
        keys = rng.permutation(np.tile(base, dup))
        st = np.empty(n, dtype=adb.STREAM_TUPLE)
        st["ts_ms"], st["key"], st["payload"] = ts, keys, np.arange(n, dtype=np.uint32)
        out.append(st)
    return out


def pinned_copy(a: np.ndarray):
    """A copy of array `a` in page-locked host memory (torch's pinned
    allocator): returns the numpy view and the buffer that owns it."""
    import torch
    buf = torch.empty(max(a.nbytes, 1), dtype=torch.uint8, pin_memory=True)
    v = buf.numpy()[:a.nbytes].view(a.dtype)
    v[:] = a
    return v, buf


def bench_stream(args, cpu: bool = True):
    R, S = make_streams(8.0, 1.6e6, 1 << 20, 4, 31)
    Rp, keep_r = pinned_copy(R)
    Sp, keep_s = pinned_copy(S)
    out = {"metric": "stream join input tuples/s", "unit": "tuples/s", "higher_is_better": True, "n_gpus": 1,
           "data": "synthetic",
           "config": {"workload": "2 streams x 1.6M tuples/s (Poisson), keys uniform over 2^20 materialised 4x, "
                                  "1000 ms tumbling windows, micro-batches of 1 ms (1600 tuples per side)",
                      "host_memory": "streams in pinned host memory, as the join line's e2e inputs "
                                     "(tuples_per_s_pageable: the same call on pageable numpy arrays)"}}
    for algo in ("SHJ_JM_NP", "SHJ_JB_NP", "PMJ_JM_NP"):
        p = adb.default_params(window_size=1000, batch_tuples=1600, nthreads=8, progressive_step=1)
        adb.stream_join(algo, Rp, Sp, p)   # warm-up on the whole stream (device workspace sized)
        t0 = time.perf_counter()
        wins = adb.stream_join(algo, Rp, Sp, p)
        dt = time.perf_counter() - t0
        adb.stream_join(algo, R, S, p)
        t1 = time.perf_counter()
        adb.stream_join(algo, R, S, p)
        dt_pageable = time.perf_counter() - t1
        lat = np.array([w.latency_ms for w in wins])   # device time of each window's join
        out[algo] = {"tuples_per_s": (len(R) + len(S)) / dt,
                     "tuples_per_s_pageable": (len(R) + len(S)) / dt_pageable,
                     "device_tuples_per_s": (len(R) + len(S)) / (lat.sum() / 1e3),
                     "windows": len(wins), "matches": int(sum(w.count for w in wins)),
                     "window_device_ms": {"p50": float(np.percentile(lat, 50)),
                                          "p99": float(np.percentile(lat, 99))}}
    # offered load in real time: every micro-batch released at its timestamp
    p = adb.default_params(window_size=1000, batch_tuples=1600, nthreads=8, realtime=1)
    Rt, St = R[R["ts_ms"] < 3000], S[S["ts_ms"] < 3000]
    wins, prog = adb.stream_join("SHJ_JM_NP", Rt, St, p, progress=True)
    lat = np.array([w.latency_ms for w in wins])
    tp = np.array([list(g.t_pct) for g in prog])           # windows x pct
    out["SHJ_JM_NP_realtime"] = {
        "windows": len(wins), "window_latency_ms": {
            "p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)), "max": float(lat.max())},
        # progressiveness (the reference's dump_timing): ms from a window's first
        # batch to k % of its matches, median over windows; match-weighted batch latency
        "ms_to_pct_of_results": {f"{k}%": float(np.median(tp[:, i])) for i, k in enumerate(adb.WindowProgress.PCT)},
        "match_latency_ms": {"p50": float(np.median([g.lat_p50 for g in prog])),
                             "p95": float(np.median([g.lat_p95 for g in prog])),
                             "p99": float(np.median([g.lat_p99 for g in prog]))}}
    # value: through the public API with the streams in host memory (their
    # host -> device copy inside); the roofline from the windows' device time
    out["value"] = out["SHJ_JM_NP"]["tuples_per_s"]
    out["device_value"] = out["SHJ_JM_NP"]["device_tuples_per_s"]
    out["roofline"] = roofline(out["device_value"], ALG_BYTES_EAGER)
    if cpu:
        # the reference's eager joins on the first window (WAIT off: every tuple
        # has arrived, the throughput configuration), one call per algorithm
        r0, s0 = R[R["ts_ms"] < 1000], S[S["ts_ms"] < 1000]
        w0 = [(adb.tuples(r0["key"], r0["payload"]), adb.tuples(s0["key"], s0["payload"]))]
        th = host_threads()
        base = {}
        for algo in ("SHJ_JM_NP", "SHJ_JBCR_NP", "PMJ_JM_NP", "PMJ_JBCR_NP"):
            d = ref_windows(algo, w0, th, "adb_ref_hash")
            if d is not None:
                base[algo] = {"value": d["tuples_per_s"], "count": d["count"]}
        if base:
            out["cpu_baseline"] = {"value": base.get("SHJ_JM_NP", {}).get("value"), "unit": "tuples/s",
                                   "cores": th, "kind": "reference", "per_algorithm": base,
                                   "sample": f"the reference's eager joins (WAIT off: throughput) on the first "
                                             f"1000 ms window ({len(w0[0][0])} + {len(w0[0][1])} tuples), one call "
                                             f"each, {th} threads"}
            # latency: the same window with WAIT kept, each tuple released at its
            # timestamp; the latency is the call's end after the last arrival
            lat = {}
            for algo in ("SHJ_JM_NP", "PMJ_JM_NP"):
                d = ref_arrivals(algo, r0, s0, th)
                if d is not None:
                    lat[algo] = {"window_ms": d["ms"], "last_arrival_ms": d["last_arrival_ms"],
                                 "latency_ms": d["latency_ms"], "count": d["count"]}
            if lat:
                out["cpu_baseline"]["latency_wait_on"] = lat
    return out


def forms_summary(args):
    """Compact C3 / C4 / C5 results for the default benchmark line."""
    b = bench_batch(args)
    sv = bench_serve(args)
    st = bench_stream(args)
    keep = ("value", "unit", "roofline", "cpu_baseline", "config")
    return {
        "batch": {**{k: b[k] for k in keep if k in b}, "per_window_value": b["per_window_value"],
                  "speedup_batched_vs_per_window": b["speedup_batched_vs_per_window"],
                  "ms_batched": b["ms_batched"], "ms_per_window_launches": b["ms_per_window_launches"]},
        "serve": {**{k: sv[k] for k in keep if k in sv}, "latency_ms": sv["latency_ms"],
                  "offered_tuples_per_s": sv["offered_tuples_per_s"], "mean_batch": sv["mean_batch"]},
        "stream": {**{k: st[k] for k in keep if k in st}, "algorithm": "SHJ_JM_NP",
                   "device_value": st["device_value"],
                   "per_algorithm_tuples_per_s": {a: st[a]["tuples_per_s"] for a in ("SHJ_JM_NP", "SHJ_JB_NP",
                                                                                       "PMJ_JM_NP")},
                   "SHJ_JM_NP_tuples_per_s_pageable": st["SHJ_JM_NP"]["tuples_per_s_pageable"],
                   "per_algorithm_device_tuples_per_s": {a: st[a]["device_tuples_per_s"]
                                                         for a in ("SHJ_JM_NP", "SHJ_JB_NP", "PMJ_JM_NP")},
                   "realtime_window_latency_ms": st["SHJ_JM_NP_realtime"]["window_latency_ms"],
                   "realtime_match_latency_ms": st["SHJ_JM_NP_realtime"]["match_latency_ms"]},
    }
