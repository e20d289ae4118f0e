// eager.cu -- eager (stream) joins: SHJ_* and PMJ_* with the JM / JB / JBCR / HS
// distribution models, over arrival-ordered relations (adb_join) and over
// timestamped streams in tumbling windows (adb_stream_join).
//
// Reference:
//   SHJ: shj() hashing/helper/localjoiner.cpp:33-59 feeds one R and one S tuple
//        at a time; SHJJoiner::join (:73-94) inserts the tuple into its own
//        side's table and probes the other side's table (build_hashtable_single
//        / probe_hashtable_single, hashing/joins/common_functions.cpp:172-280).
//   PMJ: PMJJoiner::join (localjoiner.cpp:512-600) buffers progressive_step % of
//        each side, sorting_phase (pmj_helper.cpp:198-240) sorts the chunk pair
//        and joins it (earlyJoinInitialRuns :11-32), and merging_phase
//        (:188-196, earlyJoinMergedRuns :41-173) joins R of one run with S of
//        every other run.
//   Distribution models: the fetchers/shufflers of hashing/helper/fetcher.h:146-288
//        and shuffler.cpp:20-168 decide which worker sees which tuple; every model
//        yields the same matches (all twelve variants return equal counts).
//
// Device design.  Tuples arrive in micro-batches (batch_tuples per side); in
// arrival order batch b of R comes before batch b of S (shj() alternates R and
// S), and a pair (r, s) belongs to whichever of the two arrived later.
//   SHJ: per window two open-addressing tables HR, HS in device memory of
//        16-byte records {tuple word, arrival batch}, a record claimed by one
//        32-bit CAS on its batch field (every tuple value can be stored).
//        With arrivals released in real time (realtime = 1), or with progress
//        stamps, each batch runs two launches: R_b inserts into HR and probes
//        HS, then S_b inserts into HS and probes HR, so every pair is found
//        once, by its later tuple.  Otherwise (the throughput configuration,
//        the reference's WAIT undefined) a window runs two launches in all:
//        every tuple of both sides is inserted, then every tuple probes the
//        other side's table and keeps only the tuples that arrived before it
//        (an S tuple: R batches <= its own; an R tuple: S batches < its own) --
//        the same pairs, each found once by its later tuple.  The models map
//        to the table layout: JM (R replicated, S split) and HS use one shared
//        table per side; JB (key-hash routing to nthreads joiners) splits each
//        table into nthreads key-hash sub-tables; JBCR (groups of group_size
//        joiners with R replicated inside a group) into nthreads / group_size
//        sub-tables.  _P and _NP differ in the reference only in copying tuples.
//   PMJ: each run (progressive_step % of each side) is sorted on the device
//        (shared-memory block sort + merge-path merge passes), then joined with
//        itself (the initial-run join) and, merge-path style, with the sorted
//        accumulation of all earlier runs of the other side (the merged-run
//        join, done eagerly as each run arrives), then merged into its side's
//        accumulation.  adb_stream_join without real-time release or progress
//        stamps (the throughput configuration) joins a window as one run: its
//        matches are the same, and progressiveness needs arrival gating.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <thread>
#include <vector>

#include "joins.cuh"
#include "npo_join.cuh"
#include "smj_sort.cuh"

namespace adb {

enum { M_JM_NP = 0, M_JM_P = 1, M_JB_NP = 2, M_JB_P = 3, M_JBCR_NP = 4, M_JBCR_P = 5, M_HS_NP = 6, M_ST = 7 };

// ---------------------------------------------------------------------------
// SHJ
// ---------------------------------------------------------------------------
constexpr uint32_t kNoBatch = 0xFFFFFFFFu;   // batch field of an empty record

// Sub-tables: 2^log2parts key groups (the JB / JBCR key split) x 2^log2members
// members per group (JBCR: the group's threads).  JBCR replicates R to every
// member of its key's group and sends each S tuple to one member chosen at
// random (ContRandShuffler::push, hashing/helper/shuffler.cpp:143-168), so an
// R tuple is inserted into, and probes, every member's sub-table, an S tuple
// only its own member's; each pair still meets exactly once.
struct ShjTables {
    ulonglong2 *tab[2];        // R, S: records {x = tuple word, y = arrival batch (low 32 bits)}
    uint32_t log2sub[2];       // slots per sub-table (log2)
    uint32_t log2parts;        // key groups (log2)
    uint32_t log2members;      // members per group (log2; 0 unless JBCR)
    uint64_t seed;             // JBCR: the random member of each S tuple
};

__device__ __forceinline__ uint32_t shj_part(uint32_t key, uint32_t log2parts) {
    return log2parts ? (uint32_t)((key * 0x85EBCA6Bu) >> (32 - log2parts)) : 0u;
}

// JBCR: the member of S tuple number sidx of the window (its arrival
// position), a counter-based draw (SplitMix64 of seed and sidx), so insert and
// probe agree without storing it.
__device__ __forceinline__ uint32_t shj_member(const ShjTables &t, uint64_t sidx) {
    if (!t.log2members) return 0u;
    return (uint32_t)(fmix64(t.seed + 0x9E3779B97F4A7C15ULL * (sidx + 1)) >> (64 - t.log2members));
}

__device__ __forceinline__ uint64_t shj_sub(const ShjTables &t, int side, uint32_t key, uint32_t member) {
    return ((((uint64_t)shj_part(key, t.log2parts) << t.log2members) | member) << t.log2sub[side]);
}

// Inserts tuple word w of arrival batch `batch` into member `member`'s
// sub-table of side `side`.
__device__ __forceinline__ void shj_insert(const ShjTables &t, int side, uint64_t w, uint32_t batch, uint32_t member,
                                           int *err) {
    const uint32_t lo = t.log2sub[side];
    const uint64_t m = (1ULL << lo) - 1;
    const uint32_t key = tkey(w);
    ulonglong2 *tab = t.tab[side] + shj_sub(t, side, key, member);
    uint64_t slot = npo_hash(key, lo);
    for (uint64_t tries = 0;; tries++) {
        unsigned int *bf = reinterpret_cast<unsigned int *>(&tab[slot].y);
        if (atomicCAS(bf, kNoBatch, batch) == kNoBatch) {
            tab[slot].x = w;
            return;
        }
        slot = (slot + 1) & m;
        if (tries > m) { atomicExch(err, 2); return; }   // table full: cannot happen at load <= 0.5
    }
}

// Probes member `member`'s sub-table of side `side` with tuple word w (of the
// other side) and adds the matches whose arrival batch is <= max_batch.
// r_probe: w is an R tuple.
__device__ __forceinline__ void shj_probe(const ShjTables &t, int side, uint64_t w, uint32_t max_batch, bool r_probe,
                                          uint32_t member, Acc &a) {
    const uint32_t lo = t.log2sub[side];
    const uint64_t m = (1ULL << lo) - 1;
    const uint32_t key = tkey(w);
    const ulonglong2 *tab = t.tab[side] + shj_sub(t, side, key, member);
    uint64_t slot = npo_hash(key, lo);
    for (uint64_t tries = 0; tries <= m; tries++) {
        const ulonglong2 rec = tab[slot];
        const uint32_t b = (uint32_t)rec.y;
        if (b == kNoBatch) break;
        if (tkey(rec.x) == key && b <= max_batch) {
            a.count++;
            a.sum += r_probe ? pair_hash(key, tpay(w), tpay(rec.x)) : pair_hash(key, tpay(rec.x), tpay(w));
        }
        slot = (slot + 1) & m;
    }
}

// One micro-batch of one side (per-batch form): insert into the own table,
// probe the other (which holds only earlier arrivals).  `in` holds elements of
// `stride` 64-bit words with the tuple in the last word (1: plain tuples, 2:
// adb_stream_tuple); in[0] is tuple number `base` of its side in the window.
__global__ void shj_batch(const uint64_t *__restrict__ in, uint32_t stride, uint64_t n, int side, uint32_t batch,
                          uint64_t base, ShjTables t, unsigned long long *acc, int *err) {
    __shared__ uint64_t red[64];
    Acc a;
    const uint32_t members = 1u << t.log2members;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t w = in[i * stride + (stride - 1)];
        if (side == 0) {   // R: every member of the group
            for (uint32_t m = 0; m < members; m++) shj_insert(t, 0, w, batch, m, err);       // (1)
            for (uint32_t m = 0; m < members; m++) shj_probe(t, 1, w, kNoBatch - 1, true, m, a);   // (2)
        } else {           // S: its own member
            const uint32_t m = shj_member(t, base + i);
            shj_insert(t, 1, w, batch, m, err);                     // (3)
            shj_probe(t, 0, w, kNoBatch - 1, false, m, a);          // (4)
        }
    }
    block_flush(a, acc, red);
}

// Throughput form, step 1: every tuple of the window (R tuples 0 .. nR - 1,
// then S tuples) into its side's table with its arrival batch (index / step).
__global__ void shj_insert_window(const uint64_t *__restrict__ R, uint64_t nR, const uint64_t *__restrict__ S,
                                  uint64_t nS, uint32_t stride, uint64_t sr, uint64_t ss, ShjTables t, int *err) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nR + nS;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const bool isr = i < nR;
        const uint64_t k = isr ? i : i - nR;
        const uint64_t w = (isr ? R : S)[k * stride + (stride - 1)];
        const uint32_t b = (uint32_t)(k / (isr ? sr : ss));
        if (isr)
            for (uint32_t m = 0; m < (1u << t.log2members); m++) shj_insert(t, 0, w, b, m, err);
        else
            shj_insert(t, 1, w, b, shj_member(t, k), err);
    }
}

// Throughput form, step 2: every tuple probes the other side's table for the
// tuples that arrived before it: an S tuple of batch b meets R batches <= b,
// an R tuple of batch b meets S batches < b (R batch b is released first).
__global__ void shj_probe_window(const uint64_t *__restrict__ R, uint64_t nR, const uint64_t *__restrict__ S,
                                 uint64_t nS, uint32_t stride, uint64_t sr, uint64_t ss, ShjTables t,
                                 unsigned long long *acc) {
    __shared__ uint64_t red[64];
    Acc a;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nR + nS;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const bool isr = i < nR;
        const uint64_t k = isr ? i : i - nR;
        const uint64_t w = (isr ? R : S)[k * stride + (stride - 1)];
        const uint32_t b = (uint32_t)(k / (isr ? sr : ss));
        if (isr) {
            if (b)
                for (uint32_t m = 0; m < (1u << t.log2members); m++) shj_probe(t, 1, w, b - 1, true, m, a);
        } else {
            shj_probe(t, 0, w, b, false, shj_member(t, k), a);
        }
    }
    block_flush(a, acc, red);
}

static uint32_t floor_log2(int v) {
    uint32_t l = 0;
    while ((1 << (l + 1)) <= v) l++;
    return l;
}

// Key groups: JB one per thread, JBCR nthreads / group_size (both rounded
// down to a power of two); JM, HS and the single-thread forms one table.
static uint32_t shj_log2parts(int model, int nthreads, int group_size) {
    int parts = 1;
    if (model == M_JB_NP || model == M_JB_P) parts = nthreads > 0 ? nthreads : 1;
    if (model == M_JBCR_NP || model == M_JBCR_P)
        parts = std::max(1, (nthreads > 0 ? nthreads : 1) / std::max(1, group_size > 0 ? group_size : 1));
    return floor_log2(parts);
}

// Members per group: JBCR's group_size (at most nthreads, rounded down to a
// power of two); 1 otherwise.
static uint32_t shj_log2members(int model, int nthreads, int group_size) {
    if (model != M_JBCR_NP && model != M_JBCR_P) return 0;
    const int n = nthreads > 0 ? nthreads : 1;
    return floor_log2(std::max(1, std::min(n, group_size > 0 ? group_size : 1)));
}

static uint32_t shj_log2sub(uint64_t n, uint32_t log2parts) {
    // two slots per tuple in each sub-table, with slack for an uneven key split
    // when the table is split
    const uint64_t per = (n >> log2parts) + (log2parts ? (n >> (log2parts + 1)) : 0) + 64;
    uint32_t l = ceil_log2_u64(2 * per);
    return l < 4 ? 4 : l;
}

// ---------------------------------------------------------------------------
// PMJ helpers: sort a run, accumulate sorted runs
// ---------------------------------------------------------------------------
// Sorts n tuples of `in` (stride words per element, tuple last) into out, using
// tmp (n words) as the ping-pong buffer.  Returns the buffer holding the result.
__global__ void gather_tuples(const uint64_t *in, uint32_t stride, uint64_t n, uint64_t *out) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = in[i * stride + (stride - 1)];
}

static uint64_t *device_sort(Context *ctx, uint64_t *a, uint64_t *b, uint64_t n) {
    cudaStream_t st = ctx->stream;
    if (n == 0) return a;
    block_sort_kernel<<<(unsigned)((n + kSortBlock - 1) / kSortBlock), 1024, kBlockSortSmem, st>>>(a, n, b);
    ctx->kernels++;
    uint64_t *src = b, *dst = a;
    for (uint64_t run = kSortBlock; run < n; run *= 2) {
        const uint64_t threads = (n + kMergeSeg - 1) / kMergeSeg;
        merge_pass_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(src, n, run, dst);
        ctx->kernels++;
        std::swap(src, dst);
    }
    return src;
}

static void launch_merge_join(Context *ctx, const uint64_t *A, uint64_t na, const uint64_t *B, uint64_t nb,
                              int a_is_r, unsigned long long *acc) {
    if (!na || !nb) return;
    const uint64_t threads = (na + nb + kMergeSeg - 1) / kMergeSeg;
    merge_join_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, ctx->stream>>>(A, na, B, nb, a_is_r, acc);
    ctx->kernels++;
}

static void launch_merge(Context *ctx, const uint64_t *A, uint64_t na, const uint64_t *B, uint64_t nb, uint64_t *out) {
    const uint64_t threads = (na + nb + kMergeSeg - 1) / kMergeSeg;
    if (!threads) return;
    merge_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, ctx->stream>>>(A, na, B, nb, out);
    ctx->kernels++;
}

// State of one window of an eager join.
struct EagerWindow {
    // SHJ
    ShjTables t;
    uint64_t tab_slots[2];
    // PMJ: sorted accumulations (double-buffered) and run scratch
    uint64_t *accum[2][2];
    uint64_t n_accum[2];
    int cur[2];
    uint64_t *run_a, *run_b;
};

struct EagerPlan {
    Family fam;
    uint32_t log2parts, log2members;
    uint32_t log2sub[2];
    uint64_t capR, capS;   // most tuples of one window
    uint64_t run_cap;      // PMJ: most tuples of one run
};

static EagerPlan plan_eager(Family fam, int model, int nthreads, int group_size, uint64_t capR, uint64_t capS,
                            uint64_t run_cap) {
    EagerPlan p{};
    p.fam = fam;
    p.capR = capR;
    p.capS = capS;
    p.run_cap = run_cap;
    if (fam == Family::Shj) {
        p.log2parts = shj_log2parts(model, nthreads, group_size);
        p.log2members = shj_log2members(model, nthreads, group_size);
        p.log2sub[0] = shj_log2sub(capR, p.log2parts);                   // a member holds its group's whole R
        p.log2sub[1] = shj_log2sub(capS, p.log2parts + p.log2members);   // and its random share of S
    }
    return p;
}

static size_t eager_plan_bytes(const EagerPlan &p) {
    if (p.fam == Family::Shj)
        return Workspace::need(1ULL << (p.log2sub[0] + p.log2parts + p.log2members), 16) +
               Workspace::need(1ULL << (p.log2sub[1] + p.log2parts + p.log2members), 16);
    return 2 * Workspace::need(p.capR + 1, 8) + 2 * Workspace::need(p.capS + 1, 8) +
           2 * Workspace::need(p.run_cap + 1, 8);
}

static void take_window(Context *ctx, const EagerPlan &p, EagerWindow &w, uint64_t seed) {
    if (p.fam == Family::Shj) {
        for (int s = 0; s < 2; s++) {
            w.tab_slots[s] = 1ULL << (p.log2sub[s] + p.log2parts + p.log2members);
            w.t.tab[s] = ctx->ws.take<ulonglong2>(w.tab_slots[s]);
            w.t.log2sub[s] = p.log2sub[s];
        }
        w.t.log2parts = p.log2parts;
        w.t.log2members = p.log2members;
        w.t.seed = seed;
    } else {
        for (int s = 0; s < 2; s++) {
            const uint64_t cap = s ? p.capS : p.capR;
            w.accum[s][0] = ctx->ws.take<uint64_t>(cap + 1);
            w.accum[s][1] = ctx->ws.take<uint64_t>(cap + 1);
        }
        w.run_a = ctx->ws.take<uint64_t>(p.run_cap + 1);
        w.run_b = ctx->ws.take<uint64_t>(p.run_cap + 1);
    }
}

static int reset_window(Context *ctx, const EagerPlan &p, EagerWindow &w) {
    if (p.fam == Family::Shj) {
        for (int s = 0; s < 2; s++) ADB_CK(cudaMemsetAsync(w.t.tab[s], 0xFF, w.tab_slots[s] * 16, ctx->stream));
    } else {
        w.n_accum[0] = w.n_accum[1] = 0;
        w.cur[0] = w.cur[1] = 0;
    }
    return ADB_OK;
}

static int grid_for(Context *ctx, uint64_t n) {
    uint64_t b = (n + 255) / 256;
    const uint64_t cap = (uint64_t)ctx->num_sms * 8;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

// SHJ: micro-batch k of each side, R first (shj() alternates R then S); S[0]
// is S tuple number s_base of the window.
static int shj_step(Context *ctx, EagerWindow &w, const uint64_t *R, uint64_t nr, const uint64_t *S, uint64_t ns,
                    uint64_t s_base, uint32_t stride, uint32_t k, unsigned long long *acc) {
    cudaStream_t st = ctx->stream;
    int *err = reinterpret_cast<int *>(acc + 2);
    if (nr) {
        shj_batch<<<grid_for(ctx, nr), 256, 0, st>>>(R, stride, nr, 0, k, 0, w.t, acc, err);
        ctx->kernels++;
    }
    if (ns) {
        shj_batch<<<grid_for(ctx, ns), 256, 0, st>>>(S, stride, ns, 1, k, s_base, w.t, acc, err);
        ctx->kernels++;
    }
    ADB_CK(cudaGetLastError());
    return ADB_OK;
}

// PMJ: one run of each side.
static int pmj_step(Context *ctx, EagerWindow &w, const uint64_t *R, uint64_t nr, const uint64_t *S, uint64_t ns,
                    uint32_t stride, unsigned long long *acc) {
    cudaStream_t st = ctx->stream;
    // sorted run of R -> run_a/run_b; keep the sorted copy in place, sort S into
    // the accumulation's spare buffer region afterwards
    const uint64_t *run_sorted[2] = {nullptr, nullptr};
    uint64_t nrun[2] = {nr, ns};
    // sort R's run
    uint64_t *rs = nullptr, *ss = nullptr;
    if (nr) {
        gather_tuples<<<grid_for(ctx, nr), 256, 0, st>>>(R, stride, nr, w.run_a);
        ctx->kernels++;
        rs = device_sort(ctx, w.run_a, w.run_b, nr);
    }
    // S's run goes through the spare accumulation buffer of S as scratch
    uint64_t *s_spare = w.accum[1][w.cur[1] ^ 1];
    uint64_t *r_spare = w.accum[0][w.cur[0] ^ 1];
    if (ns) {
        // two scratch halves: the other run buffer and the spare accumulation of R
        uint64_t *a = rs == w.run_a ? w.run_b : w.run_a;
        gather_tuples<<<grid_for(ctx, ns), 256, 0, st>>>(S, stride, ns, a);
        ctx->kernels++;
        ss = device_sort(ctx, a, s_spare, ns);
        if (ss == s_spare) {   // keep the sorted S run out of the spare buffer, which the merge below writes
            ADB_CK(cudaMemcpyAsync(a, s_spare, ns * 8, cudaMemcpyDeviceToDevice, st));
            ss = a;
        }
    }
    run_sorted[0] = rs;
    run_sorted[1] = ss;
    // initial-run join (earlyJoinInitialRuns) and merged-run joins against the
    // earlier runs of the other side (earlyJoinMergedRuns), eagerly
    launch_merge_join(ctx, rs, nr, ss, ns, 1, acc);
    launch_merge_join(ctx, w.accum[0][w.cur[0]], w.n_accum[0], ss, ns, 1, acc);
    launch_merge_join(ctx, w.accum[1][w.cur[1]], w.n_accum[1], rs, nr, 0, acc);
    // accumulate: merge each sorted run into its side's sorted accumulation
    for (int s = 0; s < 2; s++) {
        if (!nrun[s]) continue;
        uint64_t *spare = s ? s_spare : r_spare;
        launch_merge(ctx, w.accum[s][w.cur[s]], w.n_accum[s], run_sorted[s], nrun[s], spare);
        w.cur[s] ^= 1;
        w.n_accum[s] += nrun[s];
    }
    ADB_CK(cudaGetLastError());
    return ADB_OK;
}

static int eager_step(Context *ctx, const EagerPlan &p, EagerWindow &w, const uint64_t *R, uint64_t nr,
                      const uint64_t *S, uint64_t ns, uint64_t s_base, uint32_t stride, uint32_t k,
                      unsigned long long *acc) {
    return p.fam == Family::Shj ? shj_step(ctx, w, R, nr, S, ns, s_base, stride, k, acc)
                                : pmj_step(ctx, w, R, nr, S, ns, stride, acc);
}

// Throughput form of one whole window: SHJ in two launches (insert all, probe
// all with the arrival rule, micro-batches of sr / ss tuples), PMJ as one run.
static int eager_window_throughput(Context *ctx, const EagerPlan &p, EagerWindow &w, const uint64_t *R, uint64_t nr,
                                   const uint64_t *S, uint64_t ns, uint32_t stride, uint64_t sr, uint64_t ss,
                                   unsigned long long *acc) {
    if (p.fam != Family::Shj) return pmj_step(ctx, w, R, nr, S, ns, stride, acc);
    if (!nr && !ns) return ADB_OK;
    cudaStream_t st = ctx->stream;
    int *err = reinterpret_cast<int *>(acc + 2);
    const int grid = grid_for(ctx, nr + ns);
    sr = std::max<uint64_t>(1, sr);
    ss = std::max<uint64_t>(1, ss);
    shj_insert_window<<<grid, 256, 0, st>>>(R, nr, S, ns, stride, sr, ss, w.t, err);
    shj_probe_window<<<grid, 256, 0, st>>>(R, nr, S, ns, stride, sr, ss, w.t, acc);
    ctx->kernels += 2;
    ADB_CK(cudaGetLastError());
    return ADB_OK;
}

// ---------------------------------------------------------------------------
// Relations given as arrival sequences (adb_join with an eager algorithm name)
// ---------------------------------------------------------------------------
static void eager_steps(Family fam, uint64_t nR, uint64_t nS, uint64_t batch, int progressive_step, uint64_t *sr,
                        uint64_t *ss) {
    if (fam == Family::Shj) {
        // micro-batches of `batch` tuples per side, at most 256 of them
        uint64_t b = std::max<uint64_t>(batch, 1);
        b = std::max<uint64_t>(b, (std::max(nR, nS) + 255) / 256);
        *sr = *ss = b;
    } else {
        // launcher.cpp:38-43: progressive_step % of each side per run
        const uint64_t ps = progressive_step > 0 ? (uint64_t)progressive_step : 1;
        *sr = std::max<uint64_t>(1, nR * ps / 100);
        *ss = std::max<uint64_t>(1, nS * ps / 100);
    }
}

size_t eager_scratch(uint64_t nR, uint64_t nS, Family fam, int model, int nthreads, int group_size) {
    return eager_plan_bytes(plan_eager(fam, model, nthreads, group_size, nR, nS, std::max(nR, nS)));
}

int run_eager(Context *ctx, const DevJoin &j, Family fam, int model, uint64_t batch, int nthreads, int group_size,
              int progressive_step, uint64_t seed, unsigned long long *acc) {
    uint64_t sr, ss;
    eager_steps(fam, j.nR, j.nS, batch, progressive_step, &sr, &ss);
    const uint64_t runs = std::max((j.nR + sr - 1) / sr, (j.nS + ss - 1) / ss);
    const EagerPlan p = plan_eager(fam, model, nthreads, group_size, j.nR, j.nS, std::max(j.nR, j.nS));
    EagerWindow w;
    take_window(ctx, p, w, seed);
    ADB_TRY(reset_window(ctx, p, w));
    ADB_CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    ADB_CK(cudaEventRecord(ctx->ev[2], ctx->stream));
    ADB_CK(cudaEventRecord(ctx->ev[3], ctx->stream));
    if (fam == Family::Shj)   // arrival order = micro-batch order; no real-time release
        return eager_window_throughput(ctx, p, w, j.R, j.nR, j.S, j.nS, 1, sr, ss, acc);
    for (uint64_t k = 0; k < runs; k++) {
        // the last step takes the left-over of both sides (localjoiner.cpp:575-590)
        const uint64_t r0 = std::min(j.nR, k * sr), r1 = k + 1 == runs ? j.nR : std::min(j.nR, (k + 1) * sr);
        const uint64_t s0 = std::min(j.nS, k * ss), s1 = k + 1 == runs ? j.nS : std::min(j.nS, (k + 1) * ss);
        ADB_TRY(eager_step(ctx, p, w, j.R + r0, r1 - r0, j.S + s0, s1 - s0, s0, 1, (uint32_t)k, acc));
    }
    return ADB_OK;
}

int eager_set_attrs() {
    ADB_CK(cudaFuncSetAttribute(block_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kBlockSortSmem));
    return ADB_OK;
}

// ---------------------------------------------------------------------------
// Timestamped streams in tumbling windows
// ---------------------------------------------------------------------------

// One thread: out[0] = the device's global nanosecond clock, out[1] = the
// window's match count so far (when acc is given).  Stream-ordered after (or
// before) a micro-batch's kernels, it stamps when the batch's results exist.
static __global__ void stamp_kernel(const unsigned long long *acc, unsigned long long *out) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    out[0] = t;
    if (acc) out[1] = acc[0];
}

// Progress of one window from its per-batch stamps: rel[k] = release time,
// done[k] = results time (ns), cum[k] = matches after batch k.
static void window_progress(const std::vector<unsigned long long> &st, uint64_t steps, adb_window_progress *o) {
    static const double kPct[9] = {1, 5, 10, 25, 50, 75, 95, 99, 100};
    auto rel = [&](uint64_t k) { return st[3 * k]; };
    auto done = [&](uint64_t k) { return st[3 * k + 1]; };
    auto cum = [&](uint64_t k) { return st[3 * k + 2]; };
    *o = adb_window_progress{};
    o->batches = (uint32_t)steps;
    if (!steps) return;
    const uint64_t total = cum(steps - 1);
    uint64_t k = 0;
    for (int i = 0; i < 9; i++) {
        const uint64_t target = (uint64_t)std::ceil((double)total * kPct[i] / 100.0);
        while (k + 1 < steps && cum(k) < target) k++;
        o->t_pct[i] = total ? (float)((double)(done(k) - rel(0)) / 1e6) : 0.f;
    }
    // match-weighted latency percentiles of the batches
    std::vector<std::pair<double, uint64_t>> lat;
    for (uint64_t b = 0; b < steps; b++) {
        const uint64_t m = cum(b) - (b ? cum(b - 1) : 0);
        if (m) lat.emplace_back((double)(done(b) - rel(b)) / 1e6, m);
    }
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double q) {
        uint64_t seen = 0;
        for (const auto &x : lat) {
            seen += x.second;
            if ((double)seen >= q * (double)total) return (float)x.first;
        }
        return lat.empty() ? 0.f : (float)lat.back().first;
    };
    o->lat_p50 = pct(0.50);
    o->lat_p95 = pct(0.95);
    o->lat_p99 = pct(0.99);
}

// Smallest i in [max(lo, 1), hi) with T[i].ts_ms < T[i - 1].ts_ms, by
// atomicMin into *bad (left as it is when that range is ordered).  T: stream
// tuples as words {ts, tuple}.
static __global__ void ts_order_check(const uint64_t *__restrict__ T, uint64_t lo, uint64_t hi,
                                      unsigned long long *bad) {
    for (uint64_t i = max(lo, (uint64_t)1) + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < hi;
         i += (uint64_t)gridDim.x * blockDim.x)
        if (T[2 * i] < T[2 * (i - 1)]) atomicMin(bad, (unsigned long long)i);
}

int stream_join(Context *ctx, Family fam, int model, const adb_stream_tuple *R, uint64_t nR,
                const adb_stream_tuple *S, uint64_t nS, const adb_join_params *p, adb_window_result *out,
                adb_window_progress *progress, uint64_t max_windows, uint64_t *n_windows) {
    cudaStream_t st = ctx->stream;
    const uint64_t W = p && p->window_size > 0 ? (uint64_t)p->window_size : 1000;
    const uint64_t batch = p && p->batch_tuples > 0 ? (uint64_t)p->batch_tuples : 1600;
    const int nthreads = p && p->nthreads ? (int)p->nthreads : 1;
    const int group_size = p ? p->group_size : 0;
    const int pstep = p && p->progressive_step > 0 ? p->progressive_step : 1;
    const bool realtime = p && p->realtime;
    *n_windows = 0;
    if (!nR && !nS) return ADB_OK;
    // window boundaries from the timestamps (both streams are ts-ordered)
    const uint64_t t0 = std::min(nR ? R[0].ts_ms : ~0ULL, nS ? S[0].ts_ms : ~0ULL);
    const uint64_t tend = std::max(nR ? R[nR - 1].ts_ms : 0ULL, nS ? S[nS - 1].ts_ms : 0ULL);
    const uint64_t wbase = t0 / W * W;
    const uint64_t nwin = (tend - wbase) / W + 1;
    std::vector<uint64_t> rb(nwin + 1), sb(nwin + 1);
    {
        // first tuple of each window: one binary search per boundary (log n
        // timestamp reads instead of a pass over the streams)
        auto first_at = [](const adb_stream_tuple *T, uint64_t lo, uint64_t hi, uint64_t lim) {
            while (lo < hi) {
                const uint64_t mid = lo + (hi - lo) / 2;
                if (T[mid].ts_ms < lim) lo = mid + 1; else hi = mid;
            }
            return lo;
        };
        uint64_t i = 0, k = 0;
        for (uint64_t w = 0; w < nwin; w++) {
            const uint64_t lim = wbase + w * W;
            i = first_at(R, i, nR, lim);
            k = first_at(S, k, nS, lim);
            rb[w] = i;
            sb[w] = k;
        }
        rb[nwin] = nR;
        sb[nwin] = nS;
    }
    uint64_t capR = 0, capS = 0;
    for (uint64_t w = 0; w < nwin; w++) {
        capR = std::max(capR, rb[w + 1] - rb[w]);
        capS = std::max(capS, sb[w + 1] - sb[w]);
    }
    const EagerPlan plan = plan_eager(fam, model, nthreads, group_size, capR, capS, std::max(capR, capS));
    // micro-batches of window w: SHJ `batch` tuples per side, PMJ progressive_step % runs
    auto step_sizes = [&](uint64_t w, uint64_t *sr, uint64_t *ss) {
        *sr = *ss = batch;
        if (fam == Family::Pmj) {
            *sr = std::max<uint64_t>(1, (rb[w + 1] - rb[w]) * pstep / 100);
            *ss = std::max<uint64_t>(1, (sb[w + 1] - sb[w]) * pstep / 100);
        }
        return std::max<uint64_t>(1, std::max((rb[w + 1] - rb[w] + *sr - 1) / *sr, (sb[w + 1] - sb[w] + *ss - 1) / *ss));
    };
    uint64_t max_steps = 1;
    if (progress)
        for (uint64_t w = 0; w < nwin && w < max_windows; w++) {
            uint64_t a, b;
            max_steps = std::max(max_steps, step_sizes(w, &a, &b));
        }
    const size_t in_bytes = Workspace::need(nR + 1, 16) + Workspace::need(nS + 1, 16) + Workspace::need(2, 8) +
                            (progress ? Workspace::need(3 * max_steps, 8) : 0);
    ADB_TRY(ctx->ws.reserve(in_bytes + eager_plan_bytes(plan) + 4096));
    uint64_t *dR = reinterpret_cast<uint64_t *>(ctx->ws.take<adb_stream_tuple>(nR + 1));
    uint64_t *dS = reinterpret_cast<uint64_t *>(ctx->ws.take<adb_stream_tuple>(nS + 1));
    unsigned long long *acc = ctx->ws.take<unsigned long long>(4);
    unsigned long long *bad = ctx->ws.take<unsigned long long>(2);   // first out-of-order index of R, S
    unsigned long long *stamps = progress ? ctx->ws.take<unsigned long long>(3 * max_steps) : nullptr;
    std::vector<unsigned long long> h_stamps(progress ? 3 * max_steps : 0);
    EagerWindow win;
    take_window(ctx, plan, win, p ? p->seed : 0);
    // Throughput form without progress, streams in pinned memory: window w + 1's
    // tuples are copied (one DMA per side) while window w is joined.  Otherwise
    // both streams are copied first (pageable ones through the staged copy,
    // whose host threads work best on one large copy).  Streams too long for
    // the host's order check are checked on their device copies, rows [lo, hi)
    // at a time, into bad[] (read back as h_res[8], h_res[9]).
    auto is_pinned = [](const void *ptr) {
        cudaPointerAttributes at{};
        const bool pinned = cudaPointerGetAttributes(&at, ptr) == cudaSuccess && at.type == cudaMemoryTypeHost;
        cudaGetLastError();
        return pinned;
    };
    const bool pipelined = !realtime && !progress && (!nR || is_pinned(R)) && (!nS || is_pinned(S));
    const bool check_r = nR > kHostOrderCheck, check_s = nS > kHostOrderCheck;
    auto order_check = [&](uint64_t r_lo, uint64_t r_hi, uint64_t s_lo, uint64_t s_hi) {
        if (check_r && r_hi > r_lo) {
            ts_order_check<<<ctx->num_sms * 4, 256, 0, st>>>(dR, r_lo, r_hi, bad);
            ctx->kernels++;
        }
        if (check_s && s_hi > s_lo) {
            ts_order_check<<<ctx->num_sms * 4, 256, 0, st>>>(dS, s_lo, s_hi, bad + 1);
            ctx->kernels++;
        }
        return cudaGetLastError();
    };
    auto order_error = [&]() {
        if (check_r && ctx->h_res[8] < nR) {
            set_error("R is not ordered by timestamp (index %llu)", (unsigned long long)ctx->h_res[8]);
            return true;
        }
        if (check_s && ctx->h_res[9] < nS) {
            set_error("S is not ordered by timestamp (index %llu)", (unsigned long long)ctx->h_res[9]);
            return true;
        }
        return false;
    };
    // window w's rows and the pair across its first boundary, copied without
    // waiting for the windows before it (their rows are elsewhere)
    auto copy_window = [&](uint64_t w) -> int {
        ADB_TRY(h2d_copy(ctx, dR + 2 * rb[w], R + rb[w], (rb[w + 1] - rb[w]) * 16, st, false));
        ADB_TRY(h2d_copy(ctx, dS + 2 * sb[w], S + sb[w], (sb[w + 1] - sb[w]) * 16, st, false));
        ADB_CK(order_check(rb[w], rb[w + 1], sb[w], sb[w + 1]));
        return ADB_OK;
    };
    ctx->h_res[8] = nR;
    ctx->h_res[9] = nS;
    ADB_CK(cudaMemcpyAsync(bad, ctx->h_res + 8, 16, cudaMemcpyHostToDevice, st));
    if (pipelined) {
        if (nwin) ADB_TRY(copy_window(0));
    } else {
        ADB_TRY(h2d_copy(ctx, dR, R, nR * 16, st));
        ADB_TRY(h2d_copy(ctx, dS, S, nS * 16, st));
        ADB_CK(order_check(0, nR, 0, nS));
        ADB_CK(cudaMemcpyAsync(ctx->h_res + 8, bad, 16, cudaMemcpyDeviceToHost, st));
        ADB_CK(cudaStreamSynchronize(st));
        if (order_error()) return ADB_ERR_ARG;
    }

    const auto wall0 = std::chrono::steady_clock::now();
    for (uint64_t w = 0; w < nwin; w++) {
        const uint64_t r0 = rb[w], r1 = rb[w + 1], s0 = sb[w], s1 = sb[w + 1];
        ADB_CK(cudaEventRecord(ctx->ev[4], st));   // throughput form: the window's device time from here
        ADB_TRY(reset_window(ctx, plan, win));
        ADB_CK(cudaMemsetAsync(acc, 0, 32, st));
        uint64_t sr, ss;
        const uint64_t steps = step_sizes(w, &sr, &ss);
        const bool stamp = progress && w < max_windows;
        if (!realtime && !stamp) {
            // throughput configuration: the whole window at once (same matches)
            ADB_TRY(eager_window_throughput(ctx, plan, win, dR + 2 * r0, r1 - r0, dS + 2 * s0, s1 - s0, 2, sr, ss, acc));
        }
        for (uint64_t k = 0; (realtime || stamp) && k < steps; k++) {
            const uint64_t a0 = std::min(r1, r0 + k * sr), a1 = k + 1 == steps ? r1 : std::min(r1, r0 + (k + 1) * sr);
            const uint64_t c0 = std::min(s1, s0 + k * ss), c1 = k + 1 == steps ? s1 : std::min(s1, s0 + (k + 1) * ss);
            if (realtime) {
                // release the batch when its last tuple has arrived (WAIT, fetcher.cpp:120-190)
                uint64_t last = 0;
                if (a1 > a0) last = std::max(last, R[a1 - 1].ts_ms);
                if (c1 > c0) last = std::max(last, S[c1 - 1].ts_ms);
                const auto due = wall0 + std::chrono::milliseconds(last - t0);
                std::this_thread::sleep_until(due);
            }
            if (k + 1 == steps) ADB_CK(cudaEventRecord(ctx->ev[4], st));
            if (stamp) stamp_kernel<<<1, 1, 0, st>>>(nullptr, stamps + 3 * k);
            ADB_TRY(eager_step(ctx, plan, win, dR + 2 * a0, a1 - a0, dS + 2 * c0, c1 - c0, c0 - s0, 2, (uint32_t)k,
                               acc));
            if (stamp) {
                stamp_kernel<<<1, 1, 0, st>>>(acc, stamps + 3 * k + 1);
                ctx->kernels += 2;
            }
        }
        if (stamp) ADB_CK(cudaMemcpyAsync(h_stamps.data(), stamps, 3 * steps * 8, cudaMemcpyDeviceToHost, st));
        const auto close = std::chrono::steady_clock::now();
        ADB_CK(cudaMemcpyAsync(ctx->h_res, acc, 32, cudaMemcpyDeviceToHost, st));
        if (pipelined) ADB_CK(cudaMemcpyAsync(ctx->h_res + 8, bad, 16, cudaMemcpyDeviceToHost, st));
        ADB_CK(cudaEventRecord(ctx->ev[5], st));
        if (pipelined && w + 1 < nwin) ADB_TRY(copy_window(w + 1));   // while window w runs
        ADB_CK(cudaEventSynchronize(ctx->ev[5]));
        if (pipelined && order_error()) return ADB_ERR_ARG;
        if (ctx->h_res[2]) {
            set_error("device table overflow in window %llu", (unsigned long long)w);
            return ADB_ERR_DEVICE;
        }
        if (w < max_windows && out) {
            adb_window_result &o = out[w];
            o.window_start_ms = wbase + w * W;
            o.n_r = r1 - r0;
            o.n_s = s1 - s0;
            o.count = ctx->h_res[0];
            o.checksum = ctx->h_res[1];
            float ms = 0;
            if (realtime) {
                ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - close).count();
            } else {
                cudaEventElapsedTime(&ms, ctx->ev[4], ctx->ev[5]);
            }
            o.latency_ms = ms;
            o.reserved = 0;
            if (progress) window_progress(h_stamps, steps, &progress[w]);
        }
    }
    *n_windows = nwin;
    return ADB_OK;
}

}  // namespace adb
