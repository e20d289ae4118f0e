"""Benchmark of the B200 join hot path (one JSON line on rank 0).

Workload (N=1): PRO radix hash join, |R| = |S| = 2^27 tuples of (u32 key, u32
payload); R keys a seeded permutation of 1..|R|, S keys drawn uniformly from
R's keys (the foreign-key case of the NPO / m-way config at 2^27, Zipf theta 0),
payload = row index; output the match count plus the order-independent 64-bit
checksum.  A step = one join of the full relations.

  value   join input tuples/s, inputs resident in HBM (2 GiB, larger than the
          126 MB L2, so no flush is needed between steps), CUDA events on the
          stream the library launches on, max over ranks
  e2e     the same metric through adb_join with pinned host buffers: the
          host->device copy of R and S and the read-back of the result are
          inside every timed step
  roofline  the dominant kernel's algorithmic bytes / its device time vs the
          measured HBM copy bandwidth (MEASURED_PEAKS.json)
  cpu_baseline  the reference's CPU join timed on this host (rank 0, N=1) on
          the same workload
  batch / serve / stream  (rank 0, N=1) the batched-windows, serving-loop and
          eager stream-join forms: tuples/s, HBM roofline fraction, latency
          percentiles, and the reference's CPU code on a stated sample

`--impl reference` times the reference CPU join of the same workload instead:
the reference's own code compiled from its sources (oracle/_ref) when present,
otherwise the oracle's CPU restatement, using the host's threads.

Multi-GPU (`--gpus N` under torchrun): every rank joins its own R/S pair of the
same size (independent windows, no exchange): weak scaling.  With `--shard`
the ranks run ONE join together (split by key hash, one all-to-all per
relation, local joins, one all-reduce): strong scaling.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# algorithmic bytes per input tuple of each family (whole pipeline)
ALG_BYTES = {"PRO": 24, "RJ_st": 24, "PRH": 24, "PRHO": 24, "NPO": 16, "NPO_st": 16,
             "m-way": 24, "m-pass": 24, "m-way+skew": 24}
# Per family: phase index (adb_join_result.ms_phase) -> (kernel, algorithmic
# bytes per input tuple of one launch, DRAM bytes per input tuple of one launch
# from an ncu capture of dram__bytes_read.sum + dram__bytes_write.sum at
# |R| = |S| = 2^24, for NPO at 2^25, the smallest size it groups by table
# region; None where not captured).  The traffic of a full-size
# launch is that figure times the launch's tuples: the kernels stream every
# tuple once, so traffic grows in proportion.
KERNELS = {
    "radix": {0: ("partition_pass<0,512> (pass 1)", 16, (270247168 + 213934080) / 2**25),
              1: ("partition_pass<1,512> (pass 2)", 16, (276288768 + 214363648) / 2**25),
              3: ("radix_join_items<Chain>", 8, (273622272 + 3668736) / 2**25)},
    "npo": {0: ("partition_pass<0,512,hashed> (grouping by table region)", 16, (540667392 + 486182144) / 2**26),
            1: ("npo_build_pages", 8, (812415744 + 381705728) / 2**26),
            3: ("npo_probe_pages", 8, (809180672 + 3512320) / 2**26)},
    "smj": {0: ("partition_pass (both passes)", 32,
                (271074048 + 215111680 + 279591680 + 219554048) / 2**25),
            3: ("smj_items", 8, (282003456 + 3525376) / 2**25)},
}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and throttle reasons sampled through NVML every 5 ms while the
    timed region runs (read-only queries; no setting is changed).  The GPU is
    found by the PCI bus id of the CUDA device, so CUDA_VISIBLE_DEVICES is
    honoured."""

    @staticmethod
    def _reasons(nv):
        return {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "hw_power_brake_slowdown": nv.nvmlClocksEventReasonHwPowerBrakeSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}

    def __init__(self, cuda_index: int, period_s: float = 0.005):
        self.cuda_index = cuda_index
        self.period = period_s
        self.samples = []   # (sm_mhz, reasons bitmask)
        self.bits = {}
        self.max_mhz = None
        self.error = None
        self._stop = threading.Event()

    def _handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.cuda_index)
        bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)

    def _run(self, nv, h):
        try:
            while not self._stop.is_set():
                self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM),
                                     nv.nvmlDeviceGetCurrentClocksEventReasons(h)))
                self._first.set()
                self._stop.wait(self.period)
        except Exception as e:
            self.error = f"{type(e).__name__}: {e}"
        self._first.set()

    def __enter__(self):
        # NVML is set up here, and the first sample taken, before the timed
        # region starts, so that short regions are sampled too
        self._first = threading.Event()
        self.t = None
        try:
            nv, h = self._handle()
            self.bits = self._reasons(nv)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        except Exception as e:   # no NVML: the line says so instead of guessing clocks
            self.error = f"{type(e).__name__}: {e}"
            return self
        self.t = threading.Thread(target=self._run, args=(nv, h), daemon=True)
        self.t.start()
        self._first.wait(timeout=2)
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self.t is not None:
            self.t.join(timeout=5)

    def summary(self):
        run = self.samples[1:] or self.samples   # the first sample precedes the timed region
        sm = [c for c, _ in run]
        reasons = sorted({name for _, r in run for name, bit in self.bits.items() if r & bit})
        out = {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz, "reasons": reasons,
               "samples": len(sm), "source": "NVML every 5 ms during the timed region"}
        if self.error:
            out["error"] = self.error
        return out


def make_inputs(adb, n: int, theta: float, seed: int):
    R = adb.gen_pk(n, seed)
    S, idx = adb.gen_fk(n, R, theta, seed + 1, want_idx=True)
    return R, S, idx


def _fmix64(z):
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def fk_closed_form(R, S, idx):
    """(count, checksum) of a foreign-key join from the generator's drawn
    indices: S tuple j matches R tuple idx[j] and nothing else (R's keys are
    unique), so count = |S| and checksum = sum_j H(R.key[idx_j], R.payload[idx_j],
    S.payload[j]) mod 2^64, H the pair hash of the result contract.  numpy,
    chunked over host threads; runs outside every timed region."""
    import concurrent.futures as cf
    Rw, Sw = R.view(np.uint64), S.view(np.uint64)
    lo = np.uint64(0xFFFFFFFF)
    s32 = np.uint64(32)

    def part(b):
        e = min(len(Sw), b + (1 << 22))
        rw = Rw[idx[b:e]]
        key, rp = rw >> s32, rw & lo
        sp = Sw[b:e] & lo
        h = _fmix64(((key << s32) | rp) ^ _fmix64((sp << s32) | key))
        return int(h.sum(dtype=np.uint64))

    with cf.ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1)) as ex:
        total = sum(ex.map(part, range(0, len(Sw), 1 << 22)))
    return len(Sw), total % (1 << 64)


def cpu_baseline_port(algo: str, R, S, budget_s: float):
    """Time the oracle's CPU restatement (single thread) on the workload: calls
    until budget_s seconds have run (at least one); returns (tuples/s, calls)."""
    from tests.oracle_bind import Oracle
    o = Oracle()
    fn = {"PRO": o.pro, "RJ_st": o.pro, "PRH": o.prh, "PRHO": o.prh, "NPO": o.npo, "NPO_st": o.npo,
          "m-way": o.smj, "m-pass": o.smj, "m-way+skew": o.smj}[algo]
    t_tot, reps = 0.0, 0
    while t_tot < budget_s or reps < 1:
        t0 = time.perf_counter()
        cnt, _ = fn(R, S)
        t_tot += time.perf_counter() - t0
        assert cnt == len(S)
        reps += 1
    return (len(R) + len(S)) * reps / t_tot, reps


REF_HASH_ALGOS = ("PRO", "PRH", "RJ_st", "NPO", "NPO_st")
REF_SORT_ALGOS = ("m-way", "m-pass", "m-way+skew")


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def ref_cpu(algo: str, n: int, theta: float, threads: int, reps: int, warmup: int, budget_s: float):
    """The reference's own join (oracle/_ref, compiled from its sources) on this
    host, on the benchmark's relations (n tuples per side, S Zipf(theta) over R's
    keys): `warmup` untimed calls, then up to `reps` timed calls, stopping once
    budget_s seconds of timed calls have run.  The sort-merge joins run on the
    largest power of two <= threads (sortmergejoin_multiway.cpp:59).  Returns
    the harness's JSON (median ms, tuples_per_s, reps made, threads, count),
    or None when the reference build is absent or lacks `algo`."""
    if algo in REF_HASH_ALGOS:
        ref = ROOT / "oracle" / "_ref" / "adb_ref_bench"
    elif algo in REF_SORT_ALGOS:
        ref = ROOT / "oracle" / "_ref" / "adb_ref_sort"
        threads = 1 << (max(1, threads).bit_length() - 1)
    else:
        return None
    if not ref.exists():
        return None
    out = subprocess.run([str(ref), algo, "gen", str(n), str(threads), str(max(1, reps)), str(theta),
                          str(warmup), str(budget_s)], check=True, capture_output=True, text=True,
                         timeout=1800).stdout
    return json.loads([ln for ln in out.splitlines() if ln.startswith("{")][-1])


def reference_arm(args):
    """--impl reference: the reference's CPU join on this host (rank 0 only),
    on the full workload of `config` (same n and theta as our arm)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n = 1 << args.log2n
    threads = host_threads()
    warm = min(args.warmup, 2)
    d = ref_cpu(args.algo, n, args.theta, threads, args.steps, warm, args.ref_budget)
    if d is not None:
        value, kind, cores = d["tuples_per_s"], "reference", d["threads"]
        sample = (f"{args.algo} |R|=|S|=2^{args.log2n}, S Zipf theta={args.theta} over R's keys (the full "
                  f"workload), reference code compiled from its sources, {d['threads']} threads, median of "
                  f"{d['reps']} timed join calls after {warm} warm-up calls, fresh input copies per call; "
                  f"the reference returned {d['count']} matches (|S| = {n})")
    else:
        import alliancedb_b200 as adb
        R, S, _ = make_inputs(adb, n, args.theta, 1)
        value, reps = cpu_baseline_port(args.algo, R, S, args.ref_budget)
        kind, cores = "port", 1
        sample = (f"{args.algo} |R|=|S|=2^{args.log2n}, S Zipf theta={args.theta} (the full workload), "
                  f"oracle restatement, 1 thread, {reps} calls")
    line = {"impl": "reference", "metric": "join input tuples/s", "value": value, "unit": "tuples/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32 key/payload (integer)", "data": "synthetic",
            "config": workload_config(args),
            "cpu_baseline": {"value": value, "unit": "tuples/s", "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "tuples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def workload_config(args):
    return {"workload": f"{args.algo} join |R|=|S|=2^{args.log2n}, R unique dense keys, S FK Zipf theta={args.theta}",
            "algo": args.algo, "r_tuples": 1 << args.log2n, "s_tuples": 1 << args.log2n, "theta": args.theta,
            "tuple": "u32 key + u32 payload",
            "l2": (f"inputs {16 << args.log2n >> 20} MiB, larger than the 126 MB L2 (no flush needed)"
                   if (16 << args.log2n) > 126e6 else "inputs smaller than L2")}


def shard_main(args):
    """--shard: ONE join of |R| = |S| = 2^log2n sharded over the ranks (strong
    scaling): rank r holds slice r of each relation, splits it by key hash
    (adb_shard_split), one NCCL all-to-all per relation moves the parts, every
    rank joins what it received, one all-reduce adds (count, checksum).  The
    timed step is all of that; value = 2^(log2n+1) / max-over-ranks step time."""
    import datetime
    import socket
    import torch
    import torch.distributed as dist
    import alliancedb_b200 as adb
    from alliancedb_b200.dist import max_over_ranks, shard, sharded_join

    if "WORLD_SIZE" not in os.environ:   # plain `python bench.py --shard`: a one-rank group
        s = socket.socket()
        s.bind(("127.0.0.1", 0))
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(s.getsockname()[1]), RANK="0", WORLD_SIZE="1",
                          LOCAL_RANK="0")
        s.close()
    world, rank = int(os.environ["WORLD_SIZE"]), int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    try:
        n = 1 << args.log2n
        R, S, idx = make_inputs(adb, n, args.theta, 1)   # the same relations on every rank
        lo, hi = shard(n, rank, world)
        hR = torch.from_numpy(R.view(np.int64)[lo:hi].copy()).pin_memory()
        hS = torch.from_numpy(S.view(np.int64)[lo:hi].copy()).pin_memory()
        dR, dS = hR.to(dev), hS.to(dev)
        stream = torch.cuda.current_stream(dev)

        def barrier():
            dist.barrier()
            torch.cuda.synchronize(dev)

        for _ in range(args.warmup):
            got = sharded_join(args.algo, dR, dS)
        if rank == 0:
            closed = fk_closed_form(R, S, idx)
            if got != closed:
                raise AssertionError(f"sharded join {got} != closed form {closed}")
        del idx
        barrier()
        with ClockSampler(local) as clk:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                step = sharded_join(args.algo, dR, dS)
                if step != got:
                    raise AssertionError(f"sharded join {step} != {got} of the warm-up")
            e1.record(stream)
            barrier()
        ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dev)
        # end to end: this rank's slice from pinned host memory each step
        e_ms = []
        for _ in range(max(1, args.steps // 2)):
            barrier()
            a = time.perf_counter()
            step = sharded_join(args.algo, hR.to(dev, non_blocking=True), hS.to(dev, non_blocking=True))
            if step != got:
                raise AssertionError(f"sharded join {step} != {got} of the warm-up")
            torch.cuda.synchronize(dev)
            e_ms.append((time.perf_counter() - a) * 1e3)
        e2e_ms = max_over_ranks(statistics.median(e_ms), dev)
        hbm, peak_kind = peaks()
        pipe_gbs = ALG_BYTES.get(args.algo, 24) * 2 * n / (ms / 1e3) / 1e9 / world
        line = {"metric": "join input tuples/s", "value": 2 * n / (ms / 1e3), "unit": "tuples/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "u32 key/payload (integer)", "data": "synthetic",
                "config": {**workload_config(args),
                           "sharding": f"one join over {world} GPU(s): split by key hash, one NCCL all-to-all per "
                                       "relation, local joins, one all-reduce of (count, checksum)"},
                "e2e": {"value": 2 * n / (e2e_ms / 1e3), "unit": "tuples/s", "h2d_bytes_per_step": 16 * n,
                        "d2h_bytes_per_step": 32 * world, "ms_per_step": e2e_ms},
                "roofline": {"bound": "hbm", "kernel": "whole sharded pipeline, per GPU", "achieved": pipe_gbs,
                             "peak": hbm, "unit": "GB/s", "frac": pipe_gbs / hbm, "peak_source": peak_kind,
                             "traffic": None},
                "clocks": clk.summary(),
                "result": {"count": got[0], "checksum": hex(got[1]),
                           "verified": "equal to the closed form of the foreign-key workload"}}
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--algo", default="PRO")
    ap.add_argument("--log2n", type=int, default=27)
    ap.add_argument("--theta", type=float, default=0.0)
    ap.add_argument("--cpu-budget", type=float, default=20.0,
                    help="seconds of timed reference calls for the cpu_baseline of our arm")
    ap.add_argument("--ref-budget", type=float, default=120.0,
                    help="--impl reference: stop timing once this many seconds of calls have run")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--shard", action="store_true",
                    help="one join sharded over the ranks (strong scaling) instead of one join per rank")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the batched / served / stream sub-objects of the default line")
    ap.add_argument("--workload", default="join", choices=["join", "batch", "serve", "stream"],
                    help="join: one R/S pair (default, the headline); batch: 4096 windows, one launch "
                         "sequence vs one per window; serve: open-loop requests, p50/p99/p999; "
                         "stream: two timestamped streams in 1000 ms tumbling windows")
    ap.add_argument("--windows", type=int, default=4096)
    ap.add_argument("--requests", type=int, default=4000)
    ap.add_argument("--radix-bits", type=int, default=0,
                    help="partitioned joins: fan-out bits (0 = the library's choice)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        return reference_arm(args)
    if args.workload != "join":
        from alliancedb_b200 import workloads
        line = {"batch": workloads.bench_batch, "serve": workloads.bench_serve,
                "stream": workloads.bench_stream}[args.workload](args, cpu=not args.no_cpu)
        print(json.dumps(line), flush=True)
        return

    if args.shard:
        return shard_main(args)

    import torch
    import alliancedb_b200 as adb
    from alliancedb_b200.dist import max_over_ranks, sum_results

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    n = 1 << args.log2n
    R, S, idx = make_inputs(adb, n, args.theta, 1 + 1000 * rank)
    dev = torch.device("cuda", local)
    dR = torch.from_numpy(R.view(np.int64)).to(dev)
    dS = torch.from_numpy(S.view(np.int64)).to(dev)
    hR = torch.from_numpy(R.view(np.int64)).pin_memory()
    hS = torch.from_numpy(S.view(np.int64)).pin_memory()
    stream = torch.cuda.current_stream(dev)
    sp = adb.stream_handle(stream)   # torch's stream, so the events below bracket the join's kernels

    params = adb.default_params(radix_bits=args.radix_bits) if args.radix_bits else None

    def step():
        return adb.join_device(args.algo, dR.data_ptr(), n, dS.data_ptr(), n, params, sp)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        r = step()
    want = (r.count, r.checksum)
    # the result against the closed form of the foreign-key workload (untimed)
    closed = fk_closed_form(R, S, idx)
    if want != closed:
        raise AssertionError(f"join result {want[0]}, {want[1]:#x} != closed form {closed[0]}, {closed[1]:#x}")
    del idx

    # ---- device-resident timed region
    phases = []
    barrier()
    with ClockSampler(local) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            r = step()
            phases.append(r.ms_phase)
            assert (r.count, r.checksum) == want
        e1.record(stream)
        barrier()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dev)
    kernels_per_step = r.kernels
    value = 2 * n * world / (ms / 1e3)

    # ---- end to end through adb_join with pinned host buffers
    L = adb.lib()
    res = adb.JoinResult()

    def step_e2e():
        st = L.adb_join(args.algo.encode(), hR.data_ptr(), n, hS.data_ptr(), n,
                        C.byref(params) if params is not None else None, C.byref(res))
        if st != 0:
            raise RuntimeError(L.adb_last_error().decode())
        return res

    for _ in range(2):
        step_e2e()
    barrier()
    t0 = time.perf_counter()
    e_ms = []
    for _ in range(max(1, args.steps // 2)):
        a = time.perf_counter()
        rr = step_e2e()
        e_ms.append((time.perf_counter() - a) * 1e3)
        assert (rr.count, rr.checksum) == want
    barrier()
    e2e_ms = max_over_ranks(statistics.median(e_ms), dev)
    total = sum_results(want[0], want[1], dev)
    e2e_value = 2 * n * world / (e2e_ms / 1e3)

    # ---- roofline of the dominant kernel
    fam = "npo" if args.algo.startswith("NPO") else ("smj" if args.algo.startswith("m-") else "radix")
    ph = np.array(phases).mean(axis=0)
    cands = KERNELS[fam]
    dom = max(cands, key=lambda k: ph[k])
    kname, alg_per_tuple, traffic_per_tuple = cands[dom]
    hbm, peak_kind = peaks()
    dom_bytes = alg_per_tuple * 2 * n
    achieved = dom_bytes / (ph[dom] / 1e3) / 1e9
    traffic = traffic_per_tuple * 2 * n if traffic_per_tuple else None
    pipe_bytes = ALG_BYTES.get(args.algo, 24) * 2 * n
    pipe_gbs = pipe_bytes / (ms / 1e3) / 1e9

    line = {
        "metric": "join input tuples/s", "value": value, "unit": "tuples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32 key/payload (integer)", "data": "synthetic",
        "config": workload_config(args),
        "e2e": {"value": e2e_value, "unit": "tuples/s", "h2d_bytes_per_step": 16 * n, "d2h_bytes_per_step": 32,
                "ms_per_step": e2e_ms},
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_source": peak_kind,
                     "alg_bytes_per_launch": dom_bytes, "kernel_ms": float(ph[dom]),
                     "traffic": traffic, "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum "
                                                           "per tuple at |R|=|S|=2^24 (NPO 2^25), scaled to this launch"
                                                           if traffic else None,
                     "pipeline": {"alg_bytes_per_tuple": ALG_BYTES.get(args.algo, 24), "achieved": pipe_gbs,
                                  "frac": pipe_gbs / hbm}},
        "phases_ms": [float(x) for x in ph],
        **({"random_access": {
            "note": "NPO's table (2 slots per R tuple) is far larger than L2; R and S are grouped by table region "
                    "first, so the inserts (one compare-and-swap each) and the probes (one 32-byte sector each) "
                    "hit the L2-resident region",
            "build_cas_per_s": n / (ph[1] / 1e3), "probes_per_s": n / (ph[3] / 1e3)}} if fam == "npo" else {}),
        "gpu_launches": kernels_per_step * args.steps,
        "clocks": clk.summary(),
        "result": {"count": total[0], "checksum": hex(total[1]), "over_ranks": world,
                   "verified": "equal to the closed form of the foreign-key workload on every rank (numpy, "
                               "from the generator's drawn indices)"},
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = host_threads()
        d = ref_cpu(args.algo, n, args.theta, threads, 3, 1, args.cpu_budget)
        if d is not None:
            line["cpu_baseline"] = {"value": d["tuples_per_s"], "unit": "tuples/s", "cores": d["threads"],
                                    "kind": "reference",
                                    "sample": f"reference {args.algo} on the full workload (|R|=|S|=2^{args.log2n}, "
                                              f"theta={args.theta}), {d['threads']} threads, median of {d['reps']} "
                                              f"timed join calls after 1 warm-up; {d['count']} matches"}
        else:
            v, reps = cpu_baseline_port(args.algo, R, S, args.cpu_budget)
            line["cpu_baseline"] = {"value": v, "unit": "tuples/s", "cores": 1, "kind": "port",
                                    "sample": f"oracle {args.algo} restatement on the full workload "
                                              f"(|R|=|S|=2^{args.log2n}, theta={args.theta}), {reps} calls"}
    if rank == 0 and world == 1 and not args.no_forms:
        # the batched, served and stream forms of the same join library
        # (batched windows, serving loop, eager stream joins), each with its own
        # roofline and CPU baseline, outside the timed region above
        from alliancedb_b200 import workloads
        del dR, dS
        torch.cuda.empty_cache()
        fargs = argparse.Namespace(**{**vars(args), "steps": 6})
        line.update(workloads.forms_summary(fargs))
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
