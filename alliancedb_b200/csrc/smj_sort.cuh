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

// Bitonic sort of dst[0..n) on the whole 64-bit word, padded to a power of
// two with all-ones words (which sort last); dst must hold that many words.
__device__ __forceinline__ void bitonic_words(uint64_t *dst, uint32_t n) {
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
}

// Sorts src[0..n) into dst (both shared memory, dst with room for n rounded
// up to a power of two) by key; tuples with key 0xFFFFFFFF are also ordered
// by payload, so all-ones words come last.  cnt holds 2^12 + 2 counters; red
// holds 64 scratch words.  All threads call it.
//
// MSD counting sort on the (at most) 12 highest key bits that differ within
// the chunk, all-ones words in a bucket of their own behind the rest (they
// pad callers' page slots, so they are kept out of the bit analysis); then an
// insertion sort inside each bucket when the buckets are wider than one key.
// A bucket of more than 128 tuples that needs sorting makes the whole chunk
// take the bitonic path instead.
__device__ __forceinline__ void chunk_sort(const uint64_t *src, uint32_t n, uint64_t *dst, uint32_t *cnt, uint32_t *red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    // key bits that differ within the chunk (all-ones words left out)
    uint32_t a = 0xFFFFFFFFu, o = 0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint64_t v = src[i];
        if (v != ~0ULL) {
            a &= tkey(v);
            o |= tkey(v);
        }
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
    __syncthreads();
    const uint32_t vary = (a & ~o) ? 0u : a ^ o;   // a & ~o != 0: no word counted (a stays all ones)
    const uint32_t hi = vary ? 31 - __clz(vary) : 0u;
    const uint32_t nbits = vary == 0 ? 0u : (hi + 1 < kSmjBucketBits ? hi + 1 : kSmjBucketBits);
    const uint32_t shift = vary == 0 ? 0u : hi + 1 - nbits;
    const uint32_t nb = 1u << nbits, bmask = nb - 1;   // bucket nb: all-ones words
    auto bucket = [&](uint64_t v) { return v == ~0ULL ? nb : (tkey(v) >> shift) & bmask; };
    for (uint32_t d = threadIdx.x; d <= nb; d += blockDim.x) cnt[d] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) atomicAdd(&cnt[bucket(src[i])], 1u);
    __syncthreads();
    {   // exclusive scan of the bucket counts, contiguous buckets per thread
        const uint32_t per = (nb + 1 + blockDim.x - 1) / blockDim.x;
        const uint32_t d0 = threadIdx.x * per, d1 = min(nb + 1, d0 + per);
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
        dst[atomicAdd(&cnt[bucket(v)], 1u)] = v;
    }
    __syncthreads();
    // cnt[d] is now the end of bucket d.  With shift == 0 a bucket is one key
    // value: only the bucket of key 0xFFFFFFFF (the last one, if the chunk's
    // common bits are all ones) needs its payloads ordered.  With shift > 0
    // every bucket is insertion-sorted by whole word.  The all-ones bucket is
    // one word value.
    const uint32_t d_first = shift == 0 ? ((a | bmask) == 0xFFFFFFFFu ? bmask : nb) : 0u;
    int big = 0;
    for (uint32_t d = d_first + threadIdx.x; d < nb; d += blockDim.x)
        if (cnt[d] - (d ? cnt[d - 1] : 0u) > 128) big = 1;
    if (__syncthreads_or(big)) {
        bitonic_words(dst, n);
        return;
    }
    for (uint32_t d = d_first + threadIdx.x; d < nb; d += blockDim.x) {
        const uint32_t b = d ? cnt[d - 1] : 0u, e = cnt[d];
        for (uint32_t i = b + 1; i < e; i++) {
            const uint64_t v = dst[i];
            uint32_t j = i;
            while (j > b && dst[j - 1] > v) {
                dst[j] = dst[j - 1];
                j--;
            }
            dst[j] = v;
        }
    }
    __syncthreads();
}


constexpr uint32_t kDualBucketBits = 11;

// Shared-memory words of dual_chunk_sort's counters: two sides of 2^11 + 1
// 16-bit counters each, packed two per 32-bit word.
constexpr uint32_t kDualCntWords = ((1u << kDualBucketBits) + 2);

// Insertion sort of dst[b..e) by whole word (one thread).
__device__ __forceinline__ void insertion_words(uint64_t *dst, uint32_t b, uint32_t e) {
    for (uint32_t i = b + 1; i < e; i++) {
        const uint64_t v = dst[i];
        uint32_t j = i;
        while (j > b && dst[j - 1] > v) {
            dst[j] = dst[j - 1];
            j--;
        }
        dst[j] = v;
    }
}

// Bucket function and outcome of dual_chunk_sort.
struct DualSort {
    uint32_t shift, bmask, nb;   // bucket(v) = v == ~0 ? nb : (key >> shift) & bmask
    bool bitonic;                // a side took the bitonic path: bucket ends are not valid
    bool max_key;                // a word other than all-ones has key 0xFFFFFFFF
    bool y_single;               // every Y word but its ypads all-ones pads has key y_key
                                 // (< 0xFFFFFFFF): Y is left unsorted in place, ey is not set
    uint32_t y_key;
    uint32_t all_and, vary;      // AND of all keys; key bits that differ (0: none)
    uint32_t onesx, onesy;       // all-ones words in X / Y (pads included)
    const uint16_t *ex, *ey;     // end of bucket d of Xo / Yo: ex[d], ey[d] (unless bitonic)
    __device__ __forceinline__ uint32_t bucket(uint64_t v) const {
        return v == ~0ULL ? nb : (tkey(v) >> shift) & bmask;
    }
};

// Adds 1 to 16-bit counter d of a packed array and returns its old value
// (counts stay below 2^16: a chunk holds at most 8192 words).
__device__ __forceinline__ uint32_t inc16(uint32_t *w, uint32_t d) {
    const uint32_t sh = (d & 1u) << 4;
    return (atomicAdd(&w[d >> 1], 1u << sh) >> sh) & 0xFFFFu;
}

// Scratch words of red[] that dual_chunk_sort uses: [0, 224) the analysis,
// [0, 32) the scan.
constexpr uint32_t kDualRedWords = 224;

// First half of dual_chunk_sort: the bucket function of X[0..nx) and
// Y[0..ny) (the (at most) 11 highest key bits that differ within both) and
// whether Y is a single key.  Also zeroes the counters.  Ends with a barrier
// after which every thread holds the result; red is still being read (the
// next barrier frees it).
__device__ __forceinline__ DualSort dual_analyze(const uint64_t *X, uint32_t nx, const uint64_t *Y, uint32_t ny,
                                                 uint32_t *cnt, uint32_t *red, uint32_t ypads) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (int)(blockDim.x >> 5);
    uint32_t a = 0xFFFFFFFFu, o = 0, mk = 0, ay = 0xFFFFFFFFu, oy = 0, onesy = 0, onesx = 0;
    for (uint32_t i = threadIdx.x; i < nx + ny; i += blockDim.x) {
        const uint64_t v = i < nx ? X[i] : Y[i - nx];
        if (v != ~0ULL) {
            a &= tkey(v);
            o |= tkey(v);
            mk |= tkey(v) == 0xFFFFFFFFu;
            if (i >= nx) {
                ay &= tkey(v);
                oy |= tkey(v);
            }
        } else if (i >= nx) {
            onesy++;
        } else {
            onesx++;
        }
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        a &= __shfl_xor_sync(0xffffffffu, a, s);
        o |= __shfl_xor_sync(0xffffffffu, o, s);
        mk |= __shfl_xor_sync(0xffffffffu, mk, s);
        ay &= __shfl_xor_sync(0xffffffffu, ay, s);
        oy |= __shfl_xor_sync(0xffffffffu, oy, s);
        onesy += __shfl_xor_sync(0xffffffffu, onesy, s);
        onesx += __shfl_xor_sync(0xffffffffu, onesx, s);
    }
    if (lane == 0) {
        red[wid] = a; red[32 + wid] = o; red[64 + wid] = mk;
        red[96 + wid] = ay; red[128 + wid] = oy; red[160 + wid] = onesy; red[192 + wid] = onesx;
    }
    for (uint32_t d = threadIdx.x; d < kDualCntWords; d += blockDim.x) cnt[d] = 0;
    __syncthreads();
    a = lane < nw ? red[lane] : 0xFFFFFFFFu;
    o = lane < nw ? red[32 + lane] : 0u;
    mk = lane < nw ? red[64 + lane] : 0u;
    ay = lane < nw ? red[96 + lane] : 0xFFFFFFFFu;
    oy = lane < nw ? red[128 + lane] : 0u;
    onesy = lane < nw ? red[160 + lane] : 0u;
    onesx = lane < nw ? red[192 + lane] : 0u;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        a &= __shfl_xor_sync(0xffffffffu, a, s);
        o |= __shfl_xor_sync(0xffffffffu, o, s);
        mk |= __shfl_xor_sync(0xffffffffu, mk, s);
        ay &= __shfl_xor_sync(0xffffffffu, ay, s);
        oy |= __shfl_xor_sync(0xffffffffu, oy, s);
        onesy += __shfl_xor_sync(0xffffffffu, onesy, s);
        onesx += __shfl_xor_sync(0xffffffffu, onesx, s);
    }
    DualSort r;
    r.onesx = onesx;
    r.onesy = onesy;
    // Y of one key: ay == oy over its non-pad words, none of them all-ones
    // beyond the pads (so no real key-0xFFFFFFFF tuple hides among the pads)
    r.y_single = ny > onesy && ay == oy && ay != 0xFFFFFFFFu && onesy == ypads;
    r.y_key = ay;
    const uint32_t vary = (a & ~o) ? 0u : a ^ o;
    const uint32_t hi = vary ? 31 - __clz(vary) : 0u;
    const uint32_t nbits = vary == 0 ? 0u : (hi + 1 < kDualBucketBits ? hi + 1 : kDualBucketBits);
    r.shift = vary == 0 ? 0u : hi + 1 - nbits;
    r.nb = 1u << nbits;
    r.bmask = r.nb - 1;
    r.max_key = mk != 0;
    r.all_and = a;
    r.vary = vary;
    r.bitonic = false;
    const uint32_t W = r.nb + 1;
    r.ex = reinterpret_cast<const uint16_t *>(cnt);
    r.ey = reinterpret_cast<const uint16_t *>(cnt + (W + 1) / 2);
    return r;
}

// Second half of dual_chunk_sort (every thread calls it right after
// dual_analyze, with the same arguments): counts, one scan of both sides'
// counters, scatter, then the order inside buckets that hold several keys.
// sort_y = false (block-uniform) sorts X only: Y is neither counted nor moved
// and ey is not set, for a caller that needs only Y's bucket of each word.
__device__ __forceinline__ void dual_sort_rest(DualSort &r, const uint64_t *X, uint32_t nx, uint64_t *Xo,
                                               const uint64_t *Y, uint32_t ny, uint64_t *Yo, uint32_t *cnt,
                                               uint32_t *red, bool sort_y = true) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (int)(blockDim.x >> 5);
    const uint32_t nb = r.nb, W = nb + 1;   // counters per side; [nb] = all-ones words
    uint32_t *wx = cnt, *wy = cnt + (W + 1) / 2;   // packed counter words of each side
    uint16_t *cx = reinterpret_cast<uint16_t *>(wx), *cy = reinterpret_cast<uint16_t *>(wy);
    const uint32_t nyc = r.y_single || !sort_y ? 0u : ny;   // Y words counted and placed
    for (uint32_t i = threadIdx.x; i < nx + nyc; i += blockDim.x) {
        if (i < nx) inc16(wx, r.bucket(X[i]));
        else inc16(wy, r.bucket(Y[i - nx]));
    }
    __syncthreads();   // also: every thread has read red
    {   // exclusive scan of both sides' counters, contiguous counters per thread;
        // every warp scans the warp totals itself, so one barrier suffices
        const uint32_t per = (2 * W + blockDim.x - 1) / blockDim.x;
        const uint32_t d0 = threadIdx.x * per, d1 = min(2 * W, d0 + per);
        uint32_t loc = 0;
        for (uint32_t d = d0; d < d1; d++) loc += d < W ? cx[d] : cy[d - W];
        uint32_t x = loc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) red[wid] = x;
        __syncthreads();
        uint32_t t = lane < nw ? red[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        const uint32_t before = __shfl_sync(0xffffffffu, t, wid > 0 ? wid - 1 : 0);   // warps 0 .. wid - 1
        uint32_t ex = (wid ? before : 0u) + x - loc;
        for (uint32_t d = d0; d < d1; d++) {
            uint16_t &c = d < W ? cx[d] : cy[d - W];
            const uint32_t v = c;
            c = (uint16_t)(d < W ? ex : ex - nx);
            ex += v;
        }
    }
    __syncthreads();   // red[0..32) is not written again before the next analysis
    // X first: Yo may be X's own buffer
    for (uint32_t i = threadIdx.x; i < nx; i += blockDim.x) {
        const uint64_t v = X[i];
        Xo[inc16(wx, r.bucket(v))] = v;
    }
    __syncthreads();
    if (nyc) {   // block-uniform
        for (uint32_t i = threadIdx.x; i < nyc; i += blockDim.x) {
            const uint64_t v = Y[i];
            Yo[inc16(wy, r.bucket(v))] = v;
        }
        __syncthreads();
    }
    // cx / cy[d] = end of bucket d.  Buckets that need whole-word order: all of
    // them when lower key bits vary; else only the bucket that can hold key
    // 0xFFFFFFFF (the last one, if every key bit outside the buckets is one).
    const bool single = (r.vary & ((1u << r.shift) - 1u)) == 0;
    const uint32_t d_first = single ? ((r.all_and | (r.bmask << r.shift)) == 0xFFFFFFFFu ? r.bmask : nb) : 0u;
    bool bigx = false, bigy = false;
    if (d_first < nb) {   // (block-uniform) some bucket may hold several keys
        int big = 0;
        for (uint32_t d = d_first + threadIdx.x; d < nb; d += blockDim.x) {
            if (cx[d] - (d ? cx[d - 1] : 0u) > 128) big |= 1;
            if (nyc && cy[d] - (d ? cy[d - 1] : 0u) > 128) big |= 2;
        }
        bigx = __syncthreads_or(big & 1);
        bigy = __syncthreads_or(big & 2);
    }
    if ((!bigx || !bigy) && d_first < nb) {
        const uint32_t sides = (bigx ? 0u : 1u) | (bigy || !nyc ? 0u : 2u);
        for (uint32_t t = d_first + threadIdx.x; t < 2 * nb; t += blockDim.x) {
            if (t < nb) {
                if (sides & 1) insertion_words(Xo, t ? cx[t - 1] : 0u, cx[t]);
            } else if (t - nb >= d_first && (sides & 2)) {
                const uint32_t d = t - nb;
                insertion_words(Yo, d ? cy[d - 1] : 0u, cy[d]);
            }
        }
        __syncthreads();
    }
    if (bigx) bitonic_words(Xo, nx);
    if (bigy) bitonic_words(Yo, ny);
    r.bitonic = bigx || bigy;
}

// chunk_sort of two chunks at once with one bucket function: X[0..nx) -> Xo
// and Y[0..ny) -> Yo (nx, ny <= 8192), in the same order rules, with about
// half the barriers of two calls.  Yo may be X's
// buffer; Xo, X and Y must be distinct.  cnt holds kDualCntWords words:
// afterwards the result's ex[d] / ey[d] is the end of bucket d of Xo / Yo
// (unless bitonic).  red holds kDualRedWords scratch words.  ypads = all-ones
// pad words among Y's.
//
// A Y chunk of one key (a hot key's block under skew: every increment would hit
// one shared counter) is not sorted at all: y_single reports it, and the caller
// pairs its words with X's run of that key.
//
// The buckets are the (at most) 11 highest key bits that differ within the two
// chunks.  When no lower key bit differs, every bucket holds one key value and
// needs no further order (ties stay in arbitrary order, which merge_join does
// not depend on), except for payload order among key 0xFFFFFFFF tuples.
__device__ __forceinline__ DualSort dual_chunk_sort(const uint64_t *X, uint32_t nx, uint64_t *Xo, const uint64_t *Y,
                                                    uint32_t ny, uint64_t *Yo, uint32_t *cnt, uint32_t *red,
                                                    uint32_t ypads) {
    DualSort r = dual_analyze(X, nx, Y, ny, cnt, red, ypads);
    dual_sort_rest(r, X, nx, Xo, Y, ny, Yo, cnt, red);
    return r;
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
