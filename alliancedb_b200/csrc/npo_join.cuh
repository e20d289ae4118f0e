// npo_join.cuh -- no-partitioning hash join (NPO, NPO_st) on one global table.
//
// Replaces hashing/joins/no_partitioning_join.cpp:112-476 (NPO_st, npo_thread,
// np_distribute, NPO) and its table code in hashing/joins/common_functions.cpp
// (allocate_hashtable :75-102, build_hashtable_mt :350-400, probe_hashtable
// :221-280).  The reference chains 32-byte buckets of two tuples behind
// per-bucket latches; on the GPU the table is an open-addressing array of
// 8-byte tuple slots (the tuple word itself is the slot content), claimed with
// one 64-bit atomicCAS, probed linearly from a four-slot window.
// With 2 slots per build tuple (load <= 0.5) a probe touches one or two
// sectors; a table of up to ~60 MB stays resident in the 126 MB L2.
//
// The empty marker is the all-ones word.  A build tuple equal to it (key and
// payload both 0xFFFFFFFF) is counted on the side instead of stored, and
// probes with key 0xFFFFFFFF add those matches, so no key value is reserved.
#pragma once

#include "adb_common.cuh"

namespace adb {

constexpr uint64_t kEmpty = ~0ULL;

__host__ __device__ __forceinline__ uint32_t npo_hash(uint32_t key, uint32_t log2n) {
    // Fibonacci hashing: the top log2n bits of key * 2^32/phi
    return log2n ? (uint32_t)((key * kFibMul) >> (32 - log2n)) : 0u;
}

// Inserts tuple word w (not the empty marker) by linear probing from `slot`.
__device__ __forceinline__ void npo_insert_from(uint64_t *table, uint64_t mask, uint64_t slot, uint64_t w,
                                                int *err) {
    for (uint64_t tries = 0;;) {
        const unsigned long long prev = atomicCAS(reinterpret_cast<unsigned long long *>(table + slot),
                                                  (unsigned long long)kEmpty, (unsigned long long)w);
        if (prev == kEmpty) return;
        slot = (slot + 1) & mask;
        if (++tries > mask) { atomicExch(err, 2); return; }   // table full: cannot happen at load <= 0.5
    }
}

// static: each translation unit that includes this header gets its own copy
static __global__ void npo_build(const uint64_t *__restrict__ R, uint64_t nR, uint64_t *__restrict__ table,
                          uint32_t log2n, unsigned long long *sentinel_cnt, int *err) {
    const uint64_t mask = (1ULL << log2n) - 1;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nR; i += stride) {
        const uint64_t w = R[i];
        if (w == kEmpty) { atomicAdd(sentinel_cnt, 1ull); continue; }
        npo_insert_from(table, mask, npo_hash(tkey(w), log2n), w, err);
    }
}

// Count, checksum and optional materialisation of a probe's matches.
template <bool kMaterialize>
struct NpoSink {
    Acc a;
    uint64_t *mat;
    unsigned long long *mat_n;
    uint64_t mat_cap;
    __device__ __forceinline__ void match(uint64_t s, uint32_t key, uint32_t rpay, uint64_t sh) {
        a.count++;
        a.sum += pair_hash_pre(key, rpay, sh);
        if (kMaterialize) {
            const unsigned long long k = atomicAdd(mat_n, 1ull);
            if (k < mat_cap) mat[k] = s;
        }
    }
};

// A probe's first read: the four slots b .. b + 3 from b = slot & ~1, the
// 16-byte pair holding the start slot and the pair after it (wrapping at the
// table's end), two 16-byte loads.  Starting the window at the start slot's
// pair instead of its aligned 32-byte sector leaves one or two slots after
// the start slot in every window (the sector leaves none for a start slot in
// its last place): at load 0.5 a probe then has to read on past the window
// about 19 % of the time instead of about 47 %.
__device__ __forceinline__ void npo_window(const uint64_t *table, uint64_t mask, uint64_t slot, ulonglong2 &lo,
                                           ulonglong2 &hi) {
    const uint64_t b = slot & ~1ULL;
    lo = __ldg(reinterpret_cast<const ulonglong2 *>(table + b));
    hi = __ldg(reinterpret_cast<const ulonglong2 *>(table + ((b + 2) & mask)));
}

// The slots after a probe's window: linear probing from slot
// (slot & ~1) + 4 until the first empty slot, for a probe whose run of
// occupied slots reached the window's end.
template <bool kMaterialize>
__device__ __forceinline__ void npo_probe_rest(NpoSink<kMaterialize> &sink, const uint64_t *table, uint64_t mask,
                                               uint64_t s, uint64_t slot, uint64_t sh) {
    const uint32_t key = tkey(s);
    uint64_t sl = ((slot & ~1ULL) + 4) & mask;
    for (uint64_t tries = 0; tries <= mask; tries++) {
        const uint64_t v = table[sl];
        if (v == kEmpty) break;
        if (tkey(v) == key) sink.match(s, key, tpay(v), sh);
        sl = (sl + 1) & mask;
    }
}

// One probe's window: S tuple s with start slot `slot`, given its window
// (lo, hi, read by npo_window), scanned from the start slot; the matches of
// build tuples equal to the empty marker (nsent of them, key 0xFFFFFFFF) are
// added here too.  Returns true when the run of occupied slots reaches the
// window's end, so that npo_probe_rest must go on.
template <bool kMaterialize>
__device__ __forceinline__ bool npo_probe_window(NpoSink<kMaterialize> &sink, uint64_t s, uint64_t slot,
                                                 ulonglong2 lo, ulonglong2 hi, uint64_t nsent, uint64_t &sh) {
    const uint32_t key = tkey(s);
    sh = s_half(key, tpay(s));
    const uint64_t w4[4] = {lo.x, lo.y, hi.x, hi.y};
    bool open = true;   // no empty slot met yet
    uint32_t hits = 0;  // matching slots of the window
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if (open && (uint64_t)j >= (slot & 1)) {
            if (w4[j] == kEmpty) open = false;
            else if (tkey(w4[j]) == key) hits |= 1u << j;
        }
    }
    while (hits) {       // one call site for the checksum (usually one match)
        const int j = __ffs(hits) - 1;
        hits &= hits - 1;
        const ulonglong2 h2 = j & 2 ? hi : lo;
        sink.match(s, key, tpay(j & 1 ? h2.y : h2.x), sh);
    }
    if (key == 0xFFFFFFFFu && nsent) {
        sink.a.count += nsent;
        sink.a.sum += nsent * pair_hash_pre(key, 0xFFFFFFFFu, sh);
        if (kMaterialize)
            for (uint64_t t = 0; t < nsent; t++) {
                const unsigned long long k = atomicAdd(sink.mat_n, 1ull);
                if (k < sink.mat_cap) sink.mat[k] = s;
            }
    }
    return open;
}

// One whole probe: the window, then the slots after it where needed.
template <bool kMaterialize>
__device__ __forceinline__ void npo_probe_one(NpoSink<kMaterialize> &sink, const uint64_t *table, uint64_t mask,
                                              uint64_t s, uint64_t slot, ulonglong2 lo, ulonglong2 hi,
                                              uint64_t nsent) {
    uint64_t sh;
    if (npo_probe_window(sink, s, slot, lo, hi, nsent, sh)) npo_probe_rest(sink, table, mask, s, slot, sh);
}

// Probe: each thread takes kProbeU S tuples at a time (a grid-stride group),
// so that kProbeU random table reads are in flight per thread; a probe reads
// its four-slot window first (npo_window: two 16-byte loads).
constexpr int kProbeU = 4;

template <bool kMaterialize>
__global__ void npo_probe(const uint64_t *__restrict__ S, uint64_t nS, const uint64_t *__restrict__ table,
                          uint32_t log2n, const unsigned long long *sentinel_cnt, unsigned long long *acc,
                          uint64_t *mat, unsigned long long *mat_n, uint64_t mat_cap) {
    __shared__ uint64_t red[64];
    const uint64_t mask = (1ULL << log2n) - 1;
    const uint64_t T = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nsent = *sentinel_cnt;
    NpoSink<kMaterialize> sink{Acc(), mat, mat_n, mat_cap};
    for (uint64_t g0 = tid; g0 < nS; g0 += T * kProbeU) {
        uint64_t s[kProbeU], slot[kProbeU];
        ulonglong2 lo[kProbeU], hi[kProbeU];
        bool ok[kProbeU];
#pragma unroll
        for (int u = 0; u < kProbeU; u++) {   // S tuples g0, g0 + T, ...: coalesced across the warp
            const uint64_t i = g0 + (uint64_t)u * T;
            ok[u] = i < nS;
            s[u] = ok[u] ? __ldcs(reinterpret_cast<const unsigned long long *>(S) + i) : 0ULL;
        }
#pragma unroll
        for (int u = 0; u < kProbeU; u++) {   // the windows: all loads issued before any is used
            slot[u] = npo_hash(tkey(s[u]), log2n);
            if (ok[u]) npo_window(table, mask, slot[u], lo[u], hi[u]);
        }
#pragma unroll
        for (int u = 0; u < kProbeU; u++)
            if (ok[u]) npo_probe_one(sink, table, mask, s[u], slot[u], lo[u], hi[u], nsent);
    }
    block_flush(sink.a, acc, red);
}

}  // namespace adb
