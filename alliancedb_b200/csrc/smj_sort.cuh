// smj_sort.cuh -- sorting building blocks shared by the sort-merge joins:
//   chunk_sort        sort up to 8192 tuples by key inside one CTA's shared memory
//   block_sort_kernel sort consecutive blocks of a global array (one CTA per block)
//   merge_kernel      merge-path merge of two sorted global arrays
//   merge_join_kernel merge-path join of two sorted global arrays
// They restate avxsort_tuples (sorting/joins/avxsort.cpp:209-223), the merges of
// avx_merge_tuples / avx_multiway_merge (sorting/joins/merge.cpp:105-171,
// avx_multiway_merge.cpp:200-340) and merge_join (sorting/joins/
// common_functions.cpp:298-372) for the device.
#pragma once

#include "adb_common.cuh"

namespace adb {

constexpr uint32_t kSmjBucketBits = 12;

// Sorts src[0..n) by key into dst (both shared memory).  cnt holds 2^12 + 1
// counters; red holds 64 scratch words.  All threads call it.
__device__ __forceinline__ void chunk_sort(const uint64_t *src, uint32_t n, uint64_t *dst, uint32_t *cnt, uint32_t *red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    // key bits that differ within the chunk
    uint32_t a = 0xFFFFFFFFu, o = 0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t k = tkey(src[i]);
        a &= k;
        o |= k;
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        a &= __shfl_xor_sync(0xffffffffu, a, s);
        o |= __shfl_xor_sync(0xffffffffu, o, s);
    }
    if (lane == 0) { red[wid] = a; red[32 + wid] = o; }
    __syncthreads();
    a = 0xFFFFFFFFu;
    o = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) { a &= red[w]; o |= red[32 + w]; }
    const uint32_t vary = a ^ o;
    __syncthreads();
    if (vary == 0) {   // one key value: already sorted
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
        __syncthreads();
        return;
    }
    const uint32_t hi = 31 - __clz(vary);
    const uint32_t nbits = hi + 1 < kSmjBucketBits ? hi + 1 : kSmjBucketBits;
    const uint32_t shift = hi + 1 - nbits;
    const uint32_t nb = 1u << nbits, bmask = nb - 1;
    for (uint32_t d = threadIdx.x; d < nb; d += blockDim.x) cnt[d] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) atomicAdd(&cnt[(tkey(src[i]) >> shift) & bmask], 1u);
    __syncthreads();
    {   // exclusive scan of the bucket counts, contiguous buckets per thread
        const uint32_t per = (nb + blockDim.x - 1) / blockDim.x;
        const uint32_t d0 = threadIdx.x * per, d1 = min(nb, d0 + per);
        uint32_t loc = 0;
        for (uint32_t d = d0; d < d1; d++) loc += cnt[d];
        uint32_t tot;
        uint32_t ex = block_exclusive_scan(loc, red, &tot);
        for (uint32_t d = d0; d < d1; d++) {
            const uint32_t c = cnt[d];
            cnt[d] = ex;
            ex += c;
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint64_t v = src[i];
        dst[atomicAdd(&cnt[(tkey(v) >> shift) & bmask], 1u)] = v;
    }
    __syncthreads();
    // cnt[d] is now the end of bucket d.  Buckets of more than 128 tuples
    // (keys clustered below the bucket bits) would make the insertion sort
    // quadratic: then the whole chunk is bitonic-sorted on the 64-bit word
    // instead, padded with all-ones words that sort last.
    if (shift) {
        int big = 0;
        for (uint32_t d = threadIdx.x; d < nb; d += blockDim.x)
            if (cnt[d] - (d ? cnt[d - 1] : 0u) > 128) big = 1;
        if (__syncthreads_or(big)) {
            uint32_t m = 1;
            while (m < n) m <<= 1;
            for (uint32_t i = n + threadIdx.x; i < m; i += blockDim.x) dst[i] = ~0ULL;
            __syncthreads();
            for (uint32_t k = 2; k <= m; k <<= 1) {
                for (uint32_t jj = k >> 1; jj > 0; jj >>= 1) {
                    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
                        const uint32_t l = i ^ jj;
                        if (l > i) {
                            const uint64_t x = dst[i], y = dst[l];
                            const bool up = (i & k) == 0;
                            if ((x > y) == up) { dst[i] = y; dst[l] = x; }
                        }
                    }
                    __syncthreads();
                }
            }
            return;
        }
        for (uint32_t d = threadIdx.x; d < nb; d += blockDim.x) {
            const uint32_t b = d ? cnt[d - 1] : 0u, e = cnt[d];
            for (uint32_t i = b + 1; i < e; i++) {
                const uint64_t v = dst[i];
                const uint32_t k = tkey(v);
                uint32_t j = i;
                while (j > b && tkey(dst[j - 1]) > k) {
                    dst[j] = dst[j - 1];
                    j--;
                }
                dst[j] = v;
            }
        }
        __syncthreads();
    }
}


constexpr uint32_t kSortBlock = 8192;                 // tuples a CTA sorts in shared memory
constexpr size_t kBlockSortSmem = (size_t)kSortBlock * 8 * 2 + ((size_t)(1u << kSmjBucketBits) + 4) * 4 + 1024;

// Sorts each kSortBlock-tuple block of in[0..n) into out (same positions).
static __global__ void __launch_bounds__(1024, 1) block_sort_kernel(const uint64_t *in, uint64_t n, uint64_t *out) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t *X = reinterpret_cast<uint64_t *>(smem);
    uint64_t *Y = X + kSortBlock;
    uint32_t *cnt = reinterpret_cast<uint32_t *>(Y + kSortBlock);
    uint32_t *red = cnt + (1u << kSmjBucketBits) + 4;
    const uint64_t b = (uint64_t)blockIdx.x * kSortBlock;
    if (b >= n) return;
    const uint32_t m = (uint32_t)min((uint64_t)kSortBlock, n - b);
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) X[i] = in[b + i];
    __syncthreads();
    chunk_sort(X, m, Y, cnt, red);
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) out[b + i] = Y[i];
}

// Number of A elements among the first k elements of merge(A, B), A first on
// equal keys.
__device__ __forceinline__ uint64_t merge_path(const uint64_t *A, uint64_t na, const uint64_t *B, uint64_t nb,
                                               uint64_t k) {
    uint64_t lo = k > nb ? k - nb : 0, hi = k < na ? k : na;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (tkey(A[mid]) <= tkey(B[k - mid - 1])) lo = mid + 1; else hi = mid;
    }
    return lo;
}

constexpr uint32_t kMergeSeg = 64;   // merged elements per thread

// Merges sorted pairs of runs: run pair q covers in[q * 2 * run .. ) as
// A = [q*2*run, q*2*run + run) and B = the next run (shorter at the end).
static __global__ void merge_pass_kernel(const uint64_t *in, uint64_t n, uint64_t run, uint64_t *out) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t k0 = t * kMergeSeg;
    if (k0 >= n) return;
    const uint64_t pair = k0 / (2 * run);
    const uint64_t base = pair * 2 * run;
    const uint64_t na = min(run, n - base);
    const uint64_t nb = min(run, n - base - na);
    const uint64_t *A = in + base, *B = A + na;
    const uint64_t kk0 = k0 - base, kk1 = min(na + nb, kk0 + kMergeSeg);
    uint64_t i = merge_path(A, na, B, nb, kk0), j = kk0 - i;
    for (uint64_t k = kk0; k < kk1; k++) {
        if (j >= nb || (i < na && tkey(A[i]) <= tkey(B[j]))) out[base + k] = A[i++];
        else out[base + k] = B[j++];
    }
}

// Merges two sorted arrays into out.
static __global__ void merge_kernel(const uint64_t *A, uint64_t na, const uint64_t *B, uint64_t nb, uint64_t *out) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t k0 = t * kMergeSeg;
    if (k0 >= na + nb) return;
    const uint64_t k1 = min(na + nb, k0 + kMergeSeg);
    uint64_t i = merge_path(A, na, B, nb, k0), j = k0 - i;
    for (uint64_t k = k0; k < k1; k++) {
        if (j >= nb || (i < na && tkey(A[i]) <= tkey(B[j]))) out[k] = A[i++];
        else out[k] = B[j++];
    }
}

// Joins sorted R (A) with sorted S (B): every S tuple meets the run of equal
// R keys just before its merge position.  r_is_a selects which side A is,
// for the checksum's (r_payload, s_payload) order.
static __global__ void merge_join_kernel(const uint64_t *A, uint64_t na, const uint64_t *B, uint64_t nb, int a_is_r,
                                  unsigned long long *acc) {
    __shared__ uint64_t red[64];
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t k0 = t * kMergeSeg;
    Acc ac;
    if (k0 < na + nb) {
        const uint64_t k1 = min(na + nb, k0 + kMergeSeg);
        uint64_t i = merge_path(A, na, B, nb, k0), j = k0 - i;
        for (uint64_t k = k0; k < k1; k++) {
            if (j >= nb || (i < na && tkey(A[i]) <= tkey(B[j]))) {
                i++;
            } else {
                const uint64_t b = B[j++];
                const uint32_t key = tkey(b);
                for (int64_t q = (int64_t)i - 1; q >= 0 && tkey(A[q]) == key; q--) {
                    ac.count++;
                    ac.sum += a_is_r ? pair_hash(key, tpay(A[q]), tpay(b)) : pair_hash(key, tpay(b), tpay(A[q]));
                }
            }
        }
    }
    block_flush(ac, acc, red);
}

}  // namespace adb
