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
//   adb_ref_bench <algo> files <R.bin> <S.bin> <threads>
//       relations from files of 8-byte {payload, key} tuples, one call
//   adb_ref_bench dump <n> <theta> <R.bin> <S.bin>
//       writes the relations that `gen` would join (to check the restated
//       generator against the benchmark's)
// Prints one JSON line: algo, n_r, n_s, threads, count, ms (median), reps (timed
// calls made), tuples_per_s.
//
// Built twice by oracle/Makefile: adb_ref_bench links the reference's join
// objects; adb_ref_bench_gpu (ADB_SHIM defined) links the same calls against
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

// ---- the benchmark generator (counter-based; see alliancedb_b200/csrc/datagen.cuh)
static uint64_t fmix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
static uint64_t mix3(uint64_t seed, uint64_t stream, uint64_t i) {
    return fmix64(fmix64(seed + stream * 0x632BE59BD9B4E019ULL) ^ (i * 0x9E3779B97F4A7C15ULL + 1));
}
struct Feistel {
    uint64_t n, hmask;
    uint32_t half;
    uint64_t k[4];
    Feistel(uint64_t n_, uint64_t seed) : n(n_) {
        uint32_t bits = 2;
        while (bits < 64 && (1ULL << bits) < n_) bits++;
        bits = (bits + 1) & ~1u;
        half = bits / 2;
        hmask = (1ULL << half) - 1;
        for (int r = 0; r < 4; r++) k[r] = mix3(seed, 1000 + r, 0);
    }
    uint64_t once(uint64_t x) const {
        uint64_t L = x >> half, R = x & hmask;
        for (int r = 0; r < 4; r++) {
            const uint64_t t = R;
            R = L ^ (fmix64(k[r] ^ R) & hmask);
            L = t;
        }
        return (L << half) | R;
    }
    uint64_t operator()(uint64_t i) const {
        uint64_t x = once(i);
        while (x >= n) x = once(x);
        return x;
    }
};

static tuple_t *alloc_rel(uint64_t n) {
    // the reference allocates RELATION_PADDING of slack behind every relation,
    // which PRO uses as partitioning space (hashing/benchmark.cpp:15-17, 60)
    return (tuple_t *)alloc_aligned(n * sizeof(tuple_t) + RELATION_PADDING);
}

// Zipf(theta) rank in [0, n) by rejection-inversion (Hormann and Derflinger,
// ACM TOMACS 6(3), 1996), as the benchmark generator draws it.
struct ZipfRank {
    double s, n, hx1, hn, sq;
    static double helper1(double x) { return fabs(x) > 1e-8 ? log1p(x) / x : 1.0 - x * (0.5 - x * (1.0 / 3.0 - 0.25 * x)); }
    static double helper2(double x) {
        return fabs(x) > 1e-8 ? expm1(x) / x : 1.0 + x * 0.5 * (1.0 + x * (1.0 / 3.0) * (1.0 + 0.25 * x));
    }
    double h(double x) const { return exp(-s * log(x)); }
    double hint(double x) const {
        const double lx = log(x);
        return helper2((1.0 - s) * lx) * lx;
    }
    double hinv(double x) const {
        double t = x * (1.0 - s);
        if (t < -1.0) t = -1.0;
        return exp(helper1(t) * x);
    }
    ZipfRank(uint64_t n_, double theta) : s(theta), n((double)n_) {
        hx1 = hint(1.5) - 1.0;
        hn = hint(n + 0.5);
        sq = 2.0 - hinv(hint(2.5) - h(2.0));
    }
    uint64_t sample(uint64_t seed, uint64_t j) const {
        for (uint32_t attempt = 0; attempt < 64; attempt++) {
            const double u01 = ((mix3(seed, 7, j * 64 + attempt) >> 11) + 1) * (1.0 / 9007199254740992.0);
            const double u = hn + u01 * (hx1 - hn);
            const double x = hinv(u);
            double kd = floor(x + 0.5);
            if (kd < 1.0) kd = 1.0;
            if (kd > n) kd = n;
            if (kd - x <= sq || u >= hint(kd + 0.5) - h(kd)) return (uint64_t)kd - 1;
        }
        return 0;
    }
};

template <class F>
static void par_for(uint64_t n, F f) {
    unsigned nt = std::thread::hardware_concurrency();
    if (nt == 0 || n < (1u << 16)) nt = 1;
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; t++) {
        const uint64_t b = n * t / nt, e = n * (t + 1) / nt;
        th.emplace_back([=] { for (uint64_t i = b; i < e; i++) f(i); });
    }
    for (auto &x : th) x.join();
}

// R: key = 1 + perm_1(i), payload = i.  S: payload = j, key = R.key[idx_j], idx_j
// uniform over 0..n-1 (theta 0) or rank_perm(Zipf(theta) rank) (seed 2).
static void gen_pkfk(uint64_t n, double theta, std::vector<tuple_t> &R, std::vector<tuple_t> &S) {
    R.resize(n);
    S.resize(n);
    Feistel perm(n ? n : 1, 1);
    par_for(n, [&](uint64_t i) {
        R[i].payloadID = (int32_t)i;
        R[i].key = (int32_t)(1 + perm(i));
    });
    Feistel rank_perm(n ? n : 1, 2 ^ 0x5A5A5A5A5A5A5A5AULL);
    ZipfRank z(n ? n : 1, theta > 0 ? theta : 1.0);
    par_for(n, [&](uint64_t j) {
        const uint64_t idx = theta > 0 ? rank_perm(z.sample(2, j))
                                       : (uint64_t)(((unsigned __int128)mix3(2, 3, j) * n) >> 64);
        S[j].payloadID = (int32_t)j;
        S[j].key = R[idx].key;
    });
}

static bool read_rel(const char *path, std::vector<tuple_t> &out) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) return false;
    const std::streamsize bytes = f.tellg();
    f.seekg(0);
    out.resize(bytes / sizeof(tuple_t));
    f.read(reinterpret_cast<char *>(out.data()), (std::streamsize)(out.size() * sizeof(tuple_t)));
    return (bool)f;
}

typedef result_t *(*join_fn)(relation_t *, relation_t *, param_t);

#ifdef ADB_SHIM
#include "joins/onlinejoins.h"
extern "C" uint64_t adb_shim_checksum(const result_t *res);
#endif

static join_fn lookup(const std::string &algo) {
    static const struct {
        const char *name;
        join_fn fn;
    } table[] = {
        {"PRO", PRO}, {"PRH", PRH}, {"RJ_st", RJ_st}, {"NPO", NPO}, {"NPO_st", NPO_st},
#ifdef ADB_SHIM
        {"PRHO", PRHO}, {"SHJ_st", SHJ_st}, {"SHJ_JM_NP", SHJ_JM_NP}, {"SHJ_JB_NP", SHJ_JB_NP},
        {"SHJ_JBCR_NP", SHJ_JBCR_NP}, {"PMJ_st", PMJ_st}, {"PMJ_JM_NP", PMJ_JM_NP}, {"PMJ_JB_NP", PMJ_JB_NP},
        {"RPJ_st", RPJ_st},
#endif
    };
    for (const auto &e : table)
        if (algo == e.name) return e.fn;
    return nullptr;
}

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
    std::vector<tuple_t> R0, S0;
    int reps = 1, warmup = 0;
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
    } else {
        return 2;
    }
    if (nthreads < 1) nthreads = 1;
    param_t p;
    memset((void *)&p, 0, sizeof(p));
    p.nthreads = nthreads;
    p.duplicate_num = 1;
    p.progressive_step = 1;
    p.merge_step = 2;
    tuple_t *rt = alloc_rel(R0.size()), *st = alloc_rel(S0.size());
    std::vector<double> ms;
    int64_t count = -1;
    uint64_t checksum = 0;
    double timed_s = 0;
    for (int r = 0; r < warmup + reps; r++) {
        // fresh copies: PRO overwrites its inputs (parallel_radix_join.cpp:1176-1181)
        memcpy(rt, R0.data(), R0.size() * sizeof(tuple_t));
        memcpy(st, S0.data(), S0.size() * sizeof(tuple_t));
        relation_t relR{rt, R0.size(), nullptr}, relS{st, S0.size(), nullptr};
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
