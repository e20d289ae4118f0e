// adb_common.cuh -- shared device/host definitions of the B200 join library.
//
// Tuple layout: the reference's tuple_t {int32 payloadID @0; int32 key @4}
// (hashing/utils/types.h:67-70).  On the device a tuple is handled as one
// little-endian 64-bit word  w = (u64)key << 32 | payload,  so sorting words
// sorts by key, then payload (the order of sorting/joins/avxsort.cpp:209-223).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/adb/adb_join.h"

namespace adb {

constexpr int kNumSMs = 148;          // B200: 2 dies x 74 SMs
constexpr int kWarp = 32;
constexpr uint32_t kFibMul = 0x9E3779B1u;   // 2^32 / golden ratio: Fibonacci hashing (Knuth, TAOCP 6.4)

__host__ __device__ __forceinline__ uint32_t tkey(uint64_t w) { return (uint32_t)(w >> 32); }
__host__ __device__ __forceinline__ uint32_t tpay(uint64_t w) { return (uint32_t)w; }
__host__ __device__ __forceinline__ uint64_t tword(uint32_t key, uint32_t pay) {
    return ((uint64_t)key << 32) | pay;
}

// SplitMix64 finalizer (Steele, Lea, Flood, "Fast splittable pseudorandom
// number generators", OOPSLA 2014).
__host__ __device__ __forceinline__ uint64_t fmix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// Checksum term of one matched pair (contract of adb_join.h).  The S-side
// half fmix64(b) depends only on the probe tuple, so probe loops compute it
// once per S tuple and call pair_hash_pre per match.
__host__ __device__ __forceinline__ uint64_t s_half(uint32_t key, uint32_t s_pay) {
    return fmix64(((uint64_t)s_pay << 32) | key);
}
__host__ __device__ __forceinline__ uint64_t pair_hash_pre(uint32_t key, uint32_t r_pay, uint64_t sh) {
    return fmix64((((uint64_t)key << 32) | r_pay) ^ sh);
}
__host__ __device__ __forceinline__ uint64_t pair_hash(uint32_t key, uint32_t r_pay, uint32_t s_pay) {
    return pair_hash_pre(key, r_pay, s_half(key, s_pay));
}

// Count + checksum accumulator; sums are exact mod 2^64 and order-independent.
struct Acc {
    uint64_t count = 0;
    uint64_t sum = 0;
};

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide reduction of an Acc into out[0] (count) and out[1] (checksum)
// with one 64-bit atomicAdd each per block.  `red` needs 2*32 u64 of shared
// memory.  Every thread of the block must call it.
__device__ __forceinline__ void block_flush(Acc a, unsigned long long *out, uint64_t *red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    uint64_t c = warp_sum_u64(a.count), s = warp_sum_u64(a.sum);
    if (lane == 0) { red[wid] = c; red[32 + wid] = s; }
    __syncthreads();
    if (wid == 0) {
        c = lane < nw ? red[lane] : 0;
        s = lane < nw ? red[32 + lane] : 0;
        c = warp_sum_u64(c);
        s = warp_sum_u64(s);
        if (lane == 0 && (c | s)) {
            atomicAdd(out, (unsigned long long)c);
            atomicAdd(out + 1, (unsigned long long)s);
        }
    }
    __syncthreads();
}

// Exclusive scan of one value per thread across the block; returns the prefix
// and writes the block total to *total.  `tmp` needs 32 u32 of shared memory.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *tmp, uint32_t *total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) tmp[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t t = lane < nw ? tmp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        tmp[lane] = t;   // inclusive prefix of warp totals
    }
    __syncthreads();
    uint32_t warp_base = wid ? tmp[wid - 1] : 0;
    *total = tmp[nw - 1];
    __syncthreads();
    return warp_base + x - v;
}

__host__ __device__ __forceinline__ uint32_t ceil_log2_u64(uint64_t v) {
    uint32_t b = 0;
    while ((1ULL << b) < v) b++;
    return b;
}

}  // namespace adb
