// harness_sort.cpp -- TEST INFRASTRUCTURE ONLY.  Drives the reference's own
// sort-merge joins (sorting/joins/sortmergejoin_{multiway,multipass,
// multiway_skewhandling}.cpp, compiled from the tree that oracle/ref/ref_tree.py
// prepares) through a name -> function table with the signature of the
// reference's algos[] (sorting/main.cpp:420-425, :481-486), filling
// joinconfig_t as sorting/main.cpp:726-733 does with its defaults (fan-out 128,
// AVX sort and merge, the default multi-way merge buffer, NEXT NUMA strategy).
//
// Usage:
//   adb_ref_sort <m-way|m-pass|m-way+skew> gen <n> <threads> <reps> [theta] [warmup] [budget_s]
//   adb_ref_sort <algo> files <R.bin> <S.bin> <threads>
// (the relations and options of oracle/ref/harness.cpp; threads must be a power
// of two, sortmergejoin_multiway.cpp:59).  Prints one JSON line: algo, n_r,
// n_s, threads, count, checksum (the checksum build: the match site of
// merge_join adds into oracle/ref/checksum.h's accumulators; 0 otherwise),
// ms (median), reps, tuples_per_s.
//
// Built with ADB_SHIM defined (oracle/Makefile shim-sort), the same calls go to
// alliancedb_b200/shim/reference_shim_sort.cpp on libadb_b200.so: the
// reference's call site running the GPU library through the reference's
// sort-merge signatures; the checksum then comes from the library's result.
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "affinity/numa_shuffle.h"
#include "joins/sortmergejoin_mpsm.h"
#include "joins/sortmergejoin_multipass.h"
#include "joins/sortmergejoin_multiway.h"
#include "joins/sortmergejoin_multiway_skewhandling.h"
#include "utils/params.h"

#ifdef ADB_SHIM
extern "C" uint64_t adb_shim_sort_checksum(const result_t *res);
#endif

#ifdef ADB_REF_CK
uint64_t adb_ref_checksum_total = 0;
thread_local AdbRefAcc adb_ref_acc;
thread_local bool adb_ref_probe_r = false;
AdbRefAcc::~AdbRefAcc() { __atomic_fetch_add(&adb_ref_checksum_total, sum, __ATOMIC_RELAXED); }
#endif

#include "gen.h"

typedef result_t *(*sort_join_fn)(relation_t *, relation_t *, joinconfig_t *, int, int, int);

static sort_join_fn lookup(const std::string &algo) {
    static const struct {
        const char *name;
        sort_join_fn fn;
    } table[] = {
        {"m-way", sortmergejoin_multiway},
        {"m-pass", sortmergejoin_multipass},
        {"m-way+skew", sortmergejoin_multiway_skewhandling},
#ifdef ADB_SHIM
        {"mpsm", sortmergejoin_mpsm},
#endif
    };
    for (const auto &e : table)
        if (algo == e.name) return e.fn;
    return nullptr;
}

static tuple_t *alloc_rel(uint64_t n) {
    void *p = nullptr;
    if (posix_memalign(&p, 64, n * sizeof(tuple_t) + 64)) return nullptr;
    return (tuple_t *)p;
}

int main(int argc, char **argv) {
    if (argc < 6) {
        fprintf(stderr, "usage: %s <algo> gen <n> <threads> <reps> [theta] [warmup] [budget_s] | "
                        "<algo> files <R> <S> <threads>\n", argv[0]);
        return 2;
    }
    const std::string algo = argv[1];
    sort_join_fn fn = lookup(algo);
    if (!fn) {
        fprintf(stderr, "unsupported algorithm %s\n", algo.c_str());
        return 2;
    }
    std::vector<tuple_t> R0, S0;
    int reps = 1, warmup = 0, threads = 1;
    double budget_s = 1e30;
    if (std::string(argv[2]) == "gen") {
        gen_pkfk(strtoull(argv[3], nullptr, 10), argc >= 7 ? atof(argv[6]) : 0.0, R0, S0);
        threads = atoi(argv[4]);
        reps = std::max(1, atoi(argv[5]));
        warmup = argc >= 8 ? std::max(0, atoi(argv[7])) : (reps > 1 ? 1 : 0);
        if (argc >= 9) budget_s = atof(argv[8]);
    } else if (std::string(argv[2]) == "files") {
        if (!read_rel(argv[3], R0) || !read_rel(argv[4], S0)) {
            fprintf(stderr, "cannot read relations\n");
            return 2;
        }
        threads = atoi(argv[5]);
    } else {
        return 2;
    }
#ifndef ADB_SHIM   // the library takes any thread count; the reference a power of two
    if (threads < 1 || (threads & (threads - 1))) {
        fprintf(stderr, "threads must be a power of two\n");
        return 2;
    }
#endif
    joinconfig_t cfg;
    cfg.NTHREADS = threads;
    cfg.PARTFANOUT = PARTFANOUT_DEFAULT;
    cfg.SCALARSORT = 0;
    cfg.SCALARMERGE = 0;
    cfg.MWAYMERGEBUFFERSIZE = MWAY_MERGE_BUFFER_SIZE_DEFAULT;
    cfg.NUMASTRATEGY = NEXT;
#ifndef ADB_SHIM
    numa_shuffle_init(cfg.NUMASTRATEGY, cfg.NTHREADS);
#endif

    tuple_t *rt = alloc_rel(R0.size()), *st = alloc_rel(S0.size());
    std::vector<double> ms;
    int64_t count = -1;
    uint64_t checksum = 0;
    double timed_s = 0;
    for (int r = 0; r < warmup + reps; r++) {
        memcpy(rt, R0.data(), R0.size() * sizeof(tuple_t));
        memcpy(st, S0.data(), S0.size() * sizeof(tuple_t));
        relation_t relR, relS;
        memset(&relR, 0, sizeof relR);
        memset(&relS, 0, sizeof relS);
        relR.tuples = rt;
        relR.num_tuples = R0.size();
        relS.tuples = st;
        relS.num_tuples = S0.size();
#ifdef ADB_REF_CK
        adb_ref_checksum_total = 0;
        adb_ref_acc.sum = 0;
#endif
        const auto t0 = std::chrono::steady_clock::now();
        result_t *res = fn(&relR, &relS, &cfg, 0, 0, 0);
        const auto t1 = std::chrono::steady_clock::now();
        if (!res) {
            fprintf(stderr, "%s returned no result\n", algo.c_str());
            return 1;
        }
        count = res->totalresults;
#ifdef ADB_REF_CK
        checksum = adb_ref_checksum_total + adb_ref_acc.sum;
#endif
#ifdef ADB_SHIM
        checksum = adb_shim_sort_checksum(res);
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
           algo.c_str(), R0.size(), S0.size(), threads, (long long)count, (unsigned long long)checksum, med,
           ms.size(), (R0.size() + S0.size()) / (med / 1e3));
    return 0;
}
