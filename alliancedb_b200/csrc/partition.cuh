// partition.cuh -- digit functions and the small scans shared by the
// partitioned joins (paged.cuh does the partitioning itself).
// The digit is (key >> shift) & (F - 1): the low-bit radix of PRO
// (HASH_BIT_MODULO, hashing/joins/parallel_radix_join.cpp:68), shift = the bits
// an earlier pass consumed.  The sort-merge joins partition on the same low
// bits (equal keys still meet in one partition; the reference's range split of
// the high bits, sorting/joins/sortmergejoin_multiway.cpp:475-487, is not needed
// for that).
#pragma once

#include "adb_common.cuh"

namespace adb {

__device__ __forceinline__ uint64_t ld_stream(const uint64_t *p) {
    return __ldcs(reinterpret_cast<const unsigned long long *>(p));
}

// Bulk prefetch of [p, p + bytes) into L2 (p 16-byte aligned, bytes a multiple of 16).
__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

struct DigitFn {
    uint32_t shift;
    uint32_t mask;      // F - 1
    bool hashed = false;   // the pass applies it to key * kFibMul (flat passes only)
    __host__ __device__ __forceinline__ uint32_t operator()(uint32_t key) const { return (key >> shift) & mask; }
};

__host__ __device__ __forceinline__ uint64_t chunk_of(uint64_t n, int G) {
    uint64_t c = (n + G - 1) / G;
    return (c + 1) & ~1ULL;                     // even -> 16-byte aligned chunk starts
}

// One warp per (rel, digit) row: exclusive scan over the G CTA counts in place,
// row total into totals[rel][d].
static __global__ void part_scan_rows(uint32_t *hist, uint32_t *totals, uint32_t F, int G) {
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
static __global__ void part_scan_totals(const uint32_t *totals, uint64_t *starts, uint32_t F) {
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

}  // namespace adb
