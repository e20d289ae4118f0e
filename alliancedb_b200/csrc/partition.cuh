// partition.cuh -- one-pass radix / range partitioning of R and S on the device.
//
// Replaces the reference's two-pass radix clustering
//   parallel_radix_partition  hashing/joins/parallel_radix_join.cpp:739-806
//   serial_radix_partition    :688-729, radix_cluster :573-614
//   partition_relation_optimized  sorting/joins/partition.cpp:327-350
// with three kernels per call, both relations in the same launch (grid.y):
//   1. part_hist     per-CTA histograms of the digit, shared-memory counters
//                    with warp-aggregated increments (__match_any_sync);
//   2. part_scan     row scan (per digit over CTAs) + digit totals, then the
//                    scan of the totals -> partition starts;
//   3. part_scatter  each CTA re-reads its chunk tile by tile, counting-sorts
//                    the tile by digit in shared memory and writes each digit's
//                    run contiguously at its cursor, so a warp's stores land on
//                    consecutive addresses and successive tiles of one CTA
//                    extend the same runs (write-combined in L2).
// The digit is ((key - kmin) >> shift) & (F - 1): shift 0 / kmin 0 is the low-bit
// radix of PRO; a range partition for the sort-merge join uses the high bits.
#pragma once

#include "adb_common.cuh"

namespace adb {

__device__ __forceinline__ uint64_t ld_stream(const uint64_t *p) {
    return __ldcs(reinterpret_cast<const unsigned long long *>(p));
}

struct DigitFn {
    uint32_t kmin;
    uint32_t shift;
    uint32_t mask;      // F - 1
    __host__ __device__ __forceinline__ uint32_t operator()(uint32_t key) const {
        return ((key - kmin) >> shift) & mask;
    }
};

struct RelPair {
    const uint64_t *in[2];
    uint64_t n[2];
    uint64_t *out[2];
};

// Workspace layout of one partition call (all device pointers).
struct PartWs {
    uint32_t *hist;        // [2][F][G]  counts, then row-exclusive offsets
    uint32_t *totals;      // [2][F]
    uint64_t *starts;      // [2][F+1]  partition start offsets (exclusive scan), starts[F] = n
};

constexpr int kPartThreads = 1024;
constexpr int kScatterTile = 8192;              // tuples per tile (64 KB staging)

__host__ __device__ __forceinline__ uint64_t chunk_of(uint64_t n, int G) {
    uint64_t c = (n + G - 1) / G;
    return (c + 1) & ~1ULL;                     // even -> 16-byte aligned chunk starts
}

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kPartThreads)
part_hist(RelPair rp, DigitFn df, uint32_t *hist, int G) {
    extern __shared__ uint32_t sh_hist[];
    const int rel = blockIdx.y, g = blockIdx.x;
    const uint32_t F = df.mask + 1;
    for (uint32_t i = threadIdx.x; i < F; i += blockDim.x) sh_hist[i] = 0;
    __syncthreads();

    const uint64_t n = rel ? rp.n[1] : rp.n[0];
    const uint64_t chunk = chunk_of(n, G);
    const uint64_t b = (uint64_t)g * chunk;
    const uint64_t e = min(n, b + chunk);
    const int lane = threadIdx.x & 31;
    if (b < e) {
        const uint64_t *src = rel ? rp.in[1] : rp.in[0];
        uint64_t bb = b;
        // a chunk that starts off a 16-byte boundary (sub-relation pointers of
        // batched windows) takes its first tuple singly
        if ((reinterpret_cast<uintptr_t>(src + bb) & 15) != 0) {
            if (threadIdx.x == 0) atomicAdd(&sh_hist[df(tkey(src[bb]))], 1u);
            bb++;
        }
        const uint4 *in4 = reinterpret_cast<const uint4 *>(src + bb);
        const uint64_t n2 = (e - bb) >> 1;
        // warp-uniform trip count so every lane takes part in __match_any_sync
        for (uint64_t base = 0; base < n2; base += blockDim.x) {
            const uint64_t i = base + threadIdx.x;
            const bool ok = i < n2;
            uint4 v = ok ? __ldcs(in4 + i) : make_uint4(0, 0, 0, 0);
            uint32_t d0 = ok ? df(v.y) : 0xFFFFFFFFu;
            uint32_t d1 = ok ? df(v.w) : 0xFFFFFFFFu;
            unsigned m0 = __match_any_sync(0xffffffffu, d0);
            unsigned m1 = __match_any_sync(0xffffffffu, d1);
            if (ok && lane == __ffs(m0) - 1) atomicAdd(&sh_hist[d0], __popc(m0));
            if (ok && lane == __ffs(m1) - 1) atomicAdd(&sh_hist[d1], __popc(m1));
        }
        if (bb < e && ((e - bb) & 1) && threadIdx.x == 0) {
            uint64_t w = src[e - 1];
            atomicAdd(&sh_hist[df(tkey(w))], 1u);
        }
    }
    __syncthreads();
    uint32_t *h = hist + (size_t)rel * F * G;
    for (uint32_t d = threadIdx.x; d < F; d += blockDim.x) h[(size_t)d * G + g] = sh_hist[d];
}

// One warp per (rel, digit) row: exclusive scan over the G CTA counts in place,
// row total into totals[rel][d].
__global__ void part_scan_rows(uint32_t *hist, uint32_t *totals, uint32_t F, int G) {
    const int lane = threadIdx.x & 31;
    const uint64_t row = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= 2ull * F) return;
    uint32_t *h = hist + row * G;
    uint32_t carry = 0;
    for (int base = 0; base < G; base += 32) {
        int g = base + lane;
        uint32_t v = g < G ? h[g] : 0;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (g < G) h[g] = carry + x - v;
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
    if (lane == 0) totals[row] = carry;
}

// One block per relation: exclusive scan of the F digit totals -> starts.
__global__ void part_scan_totals(const uint32_t *totals, uint64_t *starts, uint32_t F) {
    __shared__ uint32_t tmp[32];
    __shared__ uint64_t carry;
    const int rel = blockIdx.x;
    const uint32_t *t = totals + (size_t)rel * F;
    uint64_t *s = starts + (size_t)rel * (F + 1);
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < F; base += blockDim.x) {
        uint32_t d = base + threadIdx.x;
        uint32_t v = d < F ? t[d] : 0;
        uint32_t tot;
        uint32_t ex = block_exclusive_scan(v, tmp, &tot);
        if (d < F) s[d] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) s[F] = carry;
}

// Shared memory of part_scatter: cursor[F] u64-free u32 offsets relative to the
// relation, tile counters/offsets [F] each, staging [kScatterTile] u64.
__host__ __device__ __forceinline__ size_t scatter_smem(uint32_t F) {
    return (size_t)kScatterTile * 8 + (size_t)F * 4 * 3 + 32 * 4;
}

__global__ void __launch_bounds__(kPartThreads)
part_scatter(RelPair rp, DigitFn df, const uint32_t *hist_off, const uint64_t *starts, int G) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t F = df.mask + 1;
    uint64_t *stage = reinterpret_cast<uint64_t *>(smem);
    uint32_t *cursor = reinterpret_cast<uint32_t *>(smem + (size_t)kScatterTile * 8);
    uint32_t *tcnt = cursor + F;
    uint32_t *toff = tcnt + F;
    uint32_t *scan_tmp = toff + F;

    const int rel = blockIdx.y, g = blockIdx.x;
    const uint64_t n = rel ? rp.n[1] : rp.n[0];
    const uint64_t chunk = chunk_of(n, G);
    const uint64_t b = (uint64_t)g * chunk;
    const uint64_t e = min(n, b + chunk);
    if (b >= e) return;   // whole block exits together
    const uint32_t *ho = hist_off + (size_t)rel * F * G;
    const uint64_t *st = starts + (size_t)rel * (F + 1);
    // relation sizes are < 2^32 (checked on the host), so u32 cursors suffice
    for (uint32_t d = threadIdx.x; d < F; d += blockDim.x)
        cursor[d] = (uint32_t)st[d] + ho[(size_t)d * G + g];
    const uint64_t *in = rel ? rp.in[1] : rp.in[0];
    uint64_t *out = rel ? rp.out[1] : rp.out[0];
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    constexpr int PER = kScatterTile / kPartThreads;   // tuples per thread per tile (8)

    for (uint64_t t0 = b; t0 < e; t0 += kScatterTile) {
        const uint32_t tn = (uint32_t)min((uint64_t)kScatterTile, e - t0);
        for (uint32_t d = threadIdx.x; d < F; d += blockDim.x) tcnt[d] = 0;
        __syncthreads();
        uint64_t w[PER];
        uint32_t rk[PER];
        // element k of this thread: index k*blockDim + tid (coalesced per k)
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const uint32_t i = k * blockDim.x + threadIdx.x;
            const bool ok = i < tn;
            w[k] = ok ? ld_stream(in + t0 + i) : 0;
            const uint32_t d = ok ? df(tkey(w[k])) : 0xFFFFFFFFu;
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            const int leader = __ffs(peers) - 1;
            uint32_t base = 0;
            if (ok && lane == leader) base = atomicAdd(&tcnt[d], (uint32_t)__popc(peers));
            base = __shfl_sync(0xffffffffu, base, leader);
            rk[k] = base + __popc(peers & lt_mask);
        }
        __syncthreads();
        // exclusive scan of the F tile counters (contiguous segment per thread)
        {
            const uint32_t per = (F + blockDim.x - 1) / blockDim.x;
            const uint32_t d0 = threadIdx.x * per;
            uint32_t loc = 0;
            for (uint32_t d = d0; d < min(F, d0 + per); d++) loc += tcnt[d];
            uint32_t tot;
            uint32_t ex = block_exclusive_scan(loc, scan_tmp, &tot);
            for (uint32_t d = d0; d < min(F, d0 + per); d++) { toff[d] = ex; ex += tcnt[d]; }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const uint32_t i = k * blockDim.x + threadIdx.x;
            if (i < tn) stage[toff[df(tkey(w[k]))] + rk[k]] = w[k];
        }
        __syncthreads();
        for (uint32_t j = threadIdx.x; j < tn; j += blockDim.x) {
            const uint64_t v = stage[j];
            const uint32_t d = df(tkey(v));
            out[(uint64_t)cursor[d] + (j - toff[d])] = v;
        }
        __syncthreads();
        for (uint32_t d = threadIdx.x; d < F; d += blockDim.x) cursor[d] += tcnt[d];
        // next iteration's first __syncthreads orders these updates
    }
}

}  // namespace adb
