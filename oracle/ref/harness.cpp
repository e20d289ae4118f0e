// harness.cpp -- TEST INFRASTRUCTURE ONLY.  Drives the reference's own join
// functions (compiled unmodified from hashing/ by oracle/Makefile) for two
// purposes: the reference counts the tests pin against, and the CPU baseline
// (bench.py --impl reference) timed on the host's cores.
//
// Usage:
//   adb_ref_bench <PRO|PRH|RJ_st|NPO|NPO_st> gen <n> <threads> <reps> [theta] [warmup] [budget_s]
//       PK-FK relations of n tuples each (R keys a seeded permutation of 1..n,
//       S keys drawn from R's keys uniformly (theta 0) or Zipf(theta) through a
//       seeded rank permutation; the generator of the benchmark configs,
//       restated here), `warmup` untimed calls (default 1 when reps > 1), then
//       up to reps timed calls, stopping early once budget_s seconds of timed
//       calls have run (at least one timed call)
//   adb_ref_bench <algo> files <R.bin> <S.bin> <threads> [progressive_step] [merge_step] [group_size]
//       relations from files of 8-byte {payload, key} tuples, one call (the
//       last three are param_t fields of the eager joins; defaults 1, 2, 2)
//   adb_ref_bench <algo> windows <R.bin> <S.bin> <off.bin> <threads>
//       many independent R/S window pairs joined one after the other (below)
//   adb_ref_hash[_wait] <algo> arrivals <R.bin> <S.bin> <tsR.bin> <tsS.bin> <threads>
//       one call on two relations whose tuples arrive over time (tsX.bin: one
//       u64 ms offset per tuple, from the start of the call; payloadID = row).
//       Built with the reference's WAIT on (adb_ref_hash_wait) its fetchers
//       release each tuple once its time has passed (hashing/helper/
//       fetcher.cpp:127-131, 164-168) on the time-stamp counter of
//       hashing/timer/rdtsc.h; the offsets are converted to that counter at
//       the rate measured here.  Prints count, the call's ms, the last arrival
//       and the latency (call ms - last arrival ms).
//   adb_ref_bench dump <n> <theta> <R.bin> <S.bin>
//       writes the relations that `gen` would join (to check the restated
//       generator against the benchmark's)
// Prints one JSON line: algo, n_r, n_s, threads, count, ms (median), reps (timed
// calls made), tuples_per_s.
//
// Built by oracle/Makefile: adb_ref_bench links the reference's PRO / NPO join
// objects; adb_ref_hash (ADB_REF_FULL) and adb_ref_ck_hash (ADB_REF_CK, with the
// checksum) link the whole prepared hashing/ tree, eager joins included;
// adb_ref_bench_gpu (ADB_SHIM defined) links the same calls against
// alliancedb_b200/shim/reference_shim.cpp + libadb_b200.so instead, i.e. the
// reference's call sites running the GPU library through the reference's
// function signatures, and also prints the result's checksum.
//
// Platform utilities the reference links against (CPU pinning, NUMA queries,
// the global thread count of hashing/utils/generator.cpp:57) are provided
// below: identity CPU mapping over the online cores, one NUMA node.
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <thread>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "joins/no_partitioning_join.h"
#include "joins/parallel_radix_join.h"
#include "joins/prj_params.h"
#include "utils/generator.h"

#ifdef ADB_REF_CK
#define ADB_REF_FULL 1
#endif

#ifdef ADB_REF_FULL
// Whole-tree builds: the hashing/ tree prepared by oracle/ref/ref_tree.py is
// linked (its own cpu mapping, generator globals and eager joins).  With
// ADB_REF_CK its match sites add into these accumulators (oracle/ref/checksum.h).
#include "joins/onlinejoins.h"
#ifdef ADB_REF_CK
uint64_t adb_ref_checksum_total = 0;
thread_local AdbRefAcc adb_ref_acc;
thread_local bool adb_ref_probe_r = false;
AdbRefAcc::~AdbRefAcc() { __atomic_fetch_add(&adb_ref_checksum_total, sum, __ATOMIC_RELAXED); }
#endif
static void *alloc_aligned_rel(size_t size) {
    void *p = nullptr;
    if (posix_memalign(&p, 64, size)) return nullptr;
    return p;
}
#define alloc_aligned alloc_aligned_rel
#else
int nthreads = 1;
int numalocalize = 0;

int get_cpu_id(int thread_id) { return thread_id % (int)sysconf(_SC_NPROCESSORS_ONLN); }
int get_numa_id(int) { return 0; }
int get_num_numa_regions(void) { return 1; }
int get_numa_node_of_address(void *) { return 0; }
int numa_localize(tuple_t *, int64_t, uint32_t) { return 0; }
void *alloc_aligned(size_t size) {
    void *p = nullptr;
    if (posix_memalign(&p, 64, size)) return nullptr;
    return p;
}
#endif

#include "gen.h"

static tuple_t *alloc_rel(uint64_t n) {
    // the reference allocates RELATION_PADDING of slack behind every relation,
    // which PRO uses as partitioning space (hashing/benchmark.cpp:15-17, 60)
    return (tuple_t *)alloc_aligned(n * sizeof(tuple_t) + RELATION_PADDING);
}

typedef result_t *(*join_fn)(relation_t *, relation_t *, param_t);

#ifdef ADB_SHIM
#include "joins/onlinejoins.h"
extern "C" uint64_t adb_shim_checksum(const result_t *res);
#endif
#if defined(ADB_SHIM) || defined(ADB_REF_FULL)
#define ADB_ALL_HASHING_NAMES 1
#endif

static join_fn lookup(const std::string &algo) {
    static const struct {
        const char *name;
        join_fn fn;
    } table[] = {
        {"PRO", PRO}, {"PRH", PRH}, {"RJ_st", RJ_st}, {"NPO", NPO}, {"NPO_st", NPO_st},
#ifdef ADB_ALL_HASHING_NAMES
        {"PRHO", PRHO}, {"SHJ_st", SHJ_st}, {"SHJ_JM_NP", SHJ_JM_NP}, {"SHJ_JB_NP", SHJ_JB_NP},
        {"SHJ_JBCR_NP", SHJ_JBCR_NP}, {"SHJ_HS_NP", SHJ_HS_NP}, {"PMJ_st", PMJ_st}, {"PMJ_JM_NP", PMJ_JM_NP},
        {"PMJ_JB_NP", PMJ_JB_NP}, {"PMJ_JBCR_NP", PMJ_JBCR_NP}, {"PMJ_HS_NP", PMJ_HS_NP},
#endif
#ifdef ADB_SHIM
        {"RPJ_st", RPJ_st},
#endif
    };
    for (const auto &e : table)
        if (algo == e.name) return e.fn;
    return nullptr;
}

// `windows` mode: window w is R[r_off[w], r_off[w+1]) joined with
// S[s_off[w], s_off[w+1]) (off.bin: the W+1 entries of r_off, then the W+1 of
// s_off, as u64), joined one after the other by one call each, the way a
// per-window CPU deployment of the reference runs them.  Times every call
// (fresh copies of the window outside the timed part) and prints the sum of
// counts and of the call times.
static int run_windows(join_fn fn, const std::string &algo, char **argv) {
    std::vector<tuple_t> R0, S0;
    std::vector<uint64_t> off;
    if (!read_rel(argv[3], R0) || !read_rel(argv[4], S0)) return 2;
    {
        std::ifstream f(argv[5], std::ios::binary | std::ios::ate);
        if (!f) return 2;
        off.resize((size_t)f.tellg() / 8);
        f.seekg(0);
        f.read(reinterpret_cast<char *>(off.data()), (std::streamsize)(off.size() * 8));
    }
    nthreads = std::max(1, atoi(argv[6]));
    const size_t W = off.size() / 2 - 1;
    const uint64_t *r_off = off.data(), *s_off = off.data() + W + 1;
    param_t p;
    memset((void *)&p, 0, sizeof(p));
    p.nthreads = nthreads;
    p.duplicate_num = 1;
    p.progressive_step = 1;
    p.merge_step = 2;
    p.group_size = 2;
    uint64_t maxr = 0, maxs = 0;
    for (size_t w = 0; w < W; w++) {
        maxr = std::max(maxr, r_off[w + 1] - r_off[w]);
        maxs = std::max(maxs, s_off[w + 1] - s_off[w]);
    }
    tuple_t *rt = alloc_rel(maxr), *st = alloc_rel(maxs);
    double ms = 0;
    int64_t count = 0;
    for (size_t w = 0; w < W; w++) {
        const uint64_t nr = r_off[w + 1] - r_off[w], ns = s_off[w + 1] - s_off[w];
        memcpy(rt, R0.data() + r_off[w], nr * sizeof(tuple_t));
        memcpy(st, S0.data() + s_off[w], ns * sizeof(tuple_t));
        relation_t relR{rt, nr, nullptr}, relS{st, ns, nullptr};
        const auto t0 = std::chrono::steady_clock::now();
        result_t *res = fn(&relR, &relS, p);
        const auto t1 = std::chrono::steady_clock::now();
        if (!res) return 1;
        count += res->totalresults;
        free(res);
        ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
    }
    printf("{\"algo\": \"%s\", \"windows\": %zu, \"tuples\": %llu, \"threads\": %d, \"count\": %lld, "
           "\"ms\": %.3f, \"tuples_per_s\": %.1f}\n",
           algo.c_str(), W, (unsigned long long)(r_off[W] + s_off[W]), nthreads, (long long)count, ms,
           (r_off[W] + s_off[W]) / (ms / 1e3));
    return 0;
}

#ifdef ADB_REF_FULL
#include <x86intrin.h>

// `arrivals` mode (above): one timed call, arrival times on the TSC.
static int run_arrivals(join_fn fn, const std::string &algo, char **argv) {
    std::vector<tuple_t> R0, S0;
    std::vector<uint64_t> msR, msS;
    if (!read_rel(argv[3], R0) || !read_rel(argv[4], S0) || !read_rel(argv[5], msR) || !read_rel(argv[6], msS) ||
        msR.size() != R0.size() || msS.size() != S0.size())
        return 2;
    for (size_t i = 0; i < R0.size(); i++)
        if ((uint64_t)(uint32_t)R0[i].payloadID != i) return 2;
    for (size_t i = 0; i < S0.size(); i++)
        if ((uint64_t)(uint32_t)S0[i].payloadID != i) return 2;
    nthreads = std::max(1, atoi(argv[7]));
    // counter ticks per ms
    const auto c0 = std::chrono::steady_clock::now();
    const uint64_t k0 = __rdtsc();
    std::this_thread::sleep_for(std::chrono::milliseconds(200));
    const uint64_t k1 = __rdtsc();
    const double per_ms = (double)(k1 - k0) /
                          std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - c0).count();
    std::vector<uint64_t> tsR(R0.size() + 1, 0), tsS(S0.size() + 1, 0);
    uint64_t last = 0;
    for (size_t i = 0; i < R0.size(); i++) { tsR[i] = (uint64_t)(msR[i] * per_ms); last = std::max(last, msR[i]); }
    for (size_t i = 0; i < S0.size(); i++) { tsS[i] = (uint64_t)(msS[i] * per_ms); last = std::max(last, msS[i]); }
    param_t p;
    memset((void *)&p, 0, sizeof(p));
    p.nthreads = nthreads;
    p.duplicate_num = 1;
    p.progressive_step = 1;
    p.merge_step = 2;
    p.group_size = 2;
    tuple_t *rt = alloc_rel(R0.size()), *st = alloc_rel(S0.size());
    memcpy(rt, R0.data(), R0.size() * sizeof(tuple_t));
    memcpy(st, S0.data(), S0.size() * sizeof(tuple_t));
    relation_t relR{rt, R0.size(), nullptr}, relS{st, S0.size(), nullptr};
    relation_payload_t payR{tsR.data(), R0.size()}, payS{tsS.data(), S0.size()};
    relR.payload = &payR;
    relS.payload = &payS;
    const auto t0 = std::chrono::steady_clock::now();
    result_t *res = fn(&relR, &relS, p);
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (!res) return 1;
    printf("{\"algo\": \"%s\", \"n_r\": %zu, \"n_s\": %zu, \"threads\": %d, \"count\": %lld, "
           "\"ms\": %.3f, \"last_arrival_ms\": %llu, \"latency_ms\": %.3f, \"tsc_ticks_per_ms\": %.0f}\n",
           algo.c_str(), R0.size(), S0.size(), nthreads, (long long)res->totalresults, ms,
           (unsigned long long)last, ms - (double)last, per_ms);
    free(res);
    return 0;
}
#endif

int main(int argc, char **argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s <algo> gen <n> <threads> <reps> | <algo> files <R> <S> <threads>\n", argv[0]);
        return 2;
    }
    const std::string algo = argv[1];
    if (algo == "dump" && argc >= 6) {
        std::vector<tuple_t> R, S;
        gen_pkfk(strtoull(argv[2], nullptr, 10), atof(argv[3]), R, S);
        FILE *fr = fopen(argv[4], "wb"), *fs = fopen(argv[5], "wb");
        if (!fr || !fs) return 2;
        const bool ok = fwrite(R.data(), sizeof(tuple_t), R.size(), fr) == R.size() &&
                        fwrite(S.data(), sizeof(tuple_t), S.size(), fs) == S.size();
        fclose(fr);
        fclose(fs);
        return ok ? 0 : 1;
    }
    join_fn fn = lookup(algo);
    if (!fn) {
        fprintf(stderr, "unsupported algorithm %s\n", algo.c_str());
        return 2;
    }
    if (std::string(argv[2]) == "windows" && argc >= 7) return run_windows(fn, algo, argv);
#ifdef ADB_REF_FULL
    if (std::string(argv[2]) == "arrivals" && argc >= 8) return run_arrivals(fn, algo, argv);
#endif
    std::vector<tuple_t> R0, S0;
    int reps = 1, warmup = 0;
    int progressive_step = 1, merge_step = 2, group_size = 2;
    double budget_s = 1e30;
    if (std::string(argv[2]) == "gen" && argc >= 6) {
        const double theta = argc >= 7 ? atof(argv[6]) : 0.0;
        gen_pkfk(strtoull(argv[3], nullptr, 10), theta, R0, S0);
        nthreads = atoi(argv[4]);
        reps = std::max(1, atoi(argv[5]));
        warmup = argc >= 8 ? std::max(0, atoi(argv[7])) : (reps > 1 ? 1 : 0);
        if (argc >= 9) budget_s = atof(argv[8]);
    } else if (std::string(argv[2]) == "files" && argc >= 6) {
        if (!read_rel(argv[3], R0) || !read_rel(argv[4], S0)) {
            fprintf(stderr, "cannot read relations\n");
            return 2;
        }
        nthreads = atoi(argv[5]);
        if (argc >= 7) progressive_step = atoi(argv[6]);
        if (argc >= 8) merge_step = atoi(argv[7]);
        if (argc >= 9) group_size = atoi(argv[8]);
    } else {
        return 2;
    }
    if (nthreads < 1) nthreads = 1;
    param_t p;
    memset((void *)&p, 0, sizeof(p));
    p.nthreads = nthreads;
    p.duplicate_num = 1;
    p.progressive_step = progressive_step;
    p.merge_step = merge_step;
    p.group_size = group_size;
    tuple_t *rt = alloc_rel(R0.size()), *st = alloc_rel(S0.size());
    std::vector<double> ms;
#ifdef ADB_REF_FULL
    std::vector<uint64_t> tsR(R0.size() + 1, 0), tsS(S0.size() + 1, 0);
    bool ts_ok = true;
    for (const auto &t : R0) ts_ok = ts_ok && (uint64_t)(uint32_t)t.payloadID < R0.size();
    for (const auto &t : S0) ts_ok = ts_ok && (uint64_t)(uint32_t)t.payloadID < S0.size();
#endif
    int64_t count = -1;
    uint64_t checksum = 0;
    double timed_s = 0;
    for (int r = 0; r < warmup + reps; r++) {
        // fresh copies: PRO overwrites its inputs (parallel_radix_join.cpp:1176-1181)
        memcpy(rt, R0.data(), R0.size() * sizeof(tuple_t));
        memcpy(st, S0.data(), S0.size() * sizeof(tuple_t));
        relation_t relR{rt, R0.size(), nullptr}, relS{st, S0.size(), nullptr};
#ifdef ADB_REF_FULL
        // arrival timestamps (all 0: every tuple has arrived when the join
        // starts), read by the eager joins' fetchers only when WAIT is defined,
        // at ts[payloadID]; attached only when every payload indexes its row
        relation_payload_t payR{tsR.data(), R0.size()}, payS{tsS.data(), S0.size()};
        if (ts_ok) {
            relR.payload = &payR;
            relS.payload = &payS;
        }
#endif
#ifdef ADB_REF_CK
        adb_ref_checksum_total = 0;
        adb_ref_acc.sum = 0;
#endif
        const auto t0 = std::chrono::steady_clock::now();
        result_t *res = fn(&relR, &relS, p);
        const auto t1 = std::chrono::steady_clock::now();
        if (!res) {
            fprintf(stderr, "%s returned no result\n", algo.c_str());
            return 1;
        }
        count = res->totalresults;
#ifdef ADB_SHIM
        checksum = adb_shim_checksum(res);
#endif
#ifdef ADB_REF_CK
        checksum = adb_ref_checksum_total + adb_ref_acc.sum;
#endif
        free(res);
        if (r < warmup) continue;
        ms.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
        timed_s += ms.back() / 1e3;
        if (timed_s >= budget_s) break;
    }
    std::sort(ms.begin(), ms.end());
    const double med = ms[ms.size() / 2];
    printf("{\"algo\": \"%s\", \"n_r\": %zu, \"n_s\": %zu, \"threads\": %d, \"count\": %lld, "
           "\"checksum\": %llu, \"ms\": %.3f, \"reps\": %zu, \"tuples_per_s\": %.1f}\n",
           algo.c_str(), R0.size(), S0.size(), nthreads, (long long)count, (unsigned long long)checksum, med,
           ms.size(),
           (R0.size() + S0.size()) / (med / 1e3));
    return 0;
}
