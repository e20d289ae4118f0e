// datagen.cuh -- seeded, counter-based synthetic relations.
//
// Stands in for the reference's generator (hashing/utils/generator.cpp:
// parallel_create_relation :420-516, knuth_shuffle :85-94, create_relation_zipf
// :851-869, duplicate :518-542; hashing/utils/genzipf.cpp:101-207), which
// draws from glibc rand() and cannot express "R unique, S Zipf over R's keys"
// (create_relation with -d 2 makes both sides Zipf).  Every element here is a
// pure function of (seed, index), so the host and the device produce the same
// arrays and any sub-range can be generated alone.
#pragma once

#include <cmath>
#include <cstdint>

#include "adb_common.cuh"

namespace adb {

__host__ __device__ __forceinline__ uint64_t mix3(uint64_t seed, uint64_t stream, uint64_t i) {
    return fmix64(fmix64(seed + stream * 0x632BE59BD9B4E019ULL) ^ (i * 0x9E3779B97F4A7C15ULL + 1));
}

__host__ __device__ __forceinline__ uint64_t mulhi64(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// uniform integer in [0, n)
__host__ __device__ __forceinline__ uint64_t uniform_below(uint64_t seed, uint64_t stream, uint64_t i, uint64_t n) {
    return mulhi64(mix3(seed, stream, i), n);
}

// uniform double in (0, 1]
__host__ __device__ __forceinline__ double uniform01(uint64_t seed, uint64_t stream, uint64_t i) {
    return ((mix3(seed, stream, i) >> 11) + 1) * (1.0 / 9007199254740992.0);
}

// Bijection on [0, n): 4-round Feistel network over the smallest even bit
// width covering n, cycle-walked back into range (Black & Rogaway 2002).
struct Perm {
    uint64_t n;
    uint32_t half;
    uint64_t hmask;
    uint64_t k[4];
    __host__ __device__ Perm(uint64_t n_, uint64_t seed) : n(n_) {
        uint32_t bits = 2;
        while (bits < 64 && (1ULL << bits) < n_) bits++;
        bits = (bits + 1) & ~1u;
        half = bits / 2;
        hmask = (1ULL << half) - 1;
        for (int r = 0; r < 4; r++) k[r] = mix3(seed, 1000 + r, 0);
    }
    __host__ __device__ __forceinline__ uint64_t round_trip(uint64_t x) const {
        uint64_t L = x >> half, R = x & hmask;
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const uint64_t t = R;
            R = L ^ (fmix64(k[r] ^ R) & hmask);
            L = t;
        }
        return (L << half) | R;
    }
    __host__ __device__ __forceinline__ uint64_t operator()(uint64_t i) const {
        uint64_t x = round_trip(i);
        while (x >= n) x = round_trip(x);
        return x;
    }
};

// Zipf(theta) rank in [0, n) by rejection-inversion (W. Hormann and
// G. Derflinger, "Rejection-inversion to generate variates from monotone
// discrete distributions", ACM TOMACS 6(3), 1996), for theta > 0.
struct Zipf {
    double s, n, hx1, hn, sq;
    __host__ __device__ static double helper1(double x) {   // log1p(x)/x
        return fabs(x) > 1e-8 ? log1p(x) / x : 1.0 - x * (0.5 - x * (1.0 / 3.0 - 0.25 * x));
    }
    __host__ __device__ static double helper2(double x) {   // expm1(x)/x
        return fabs(x) > 1e-8 ? expm1(x) / x : 1.0 + x * 0.5 * (1.0 + x * (1.0 / 3.0) * (1.0 + 0.25 * x));
    }
    __host__ __device__ double h(double x) const { return exp(-s * log(x)); }
    __host__ __device__ double hint(double x) const {
        const double lx = log(x);
        return helper2((1.0 - s) * lx) * lx;
    }
    __host__ __device__ double hinv(double x) const {
        double t = x * (1.0 - s);
        if (t < -1.0) t = -1.0;
        return exp(helper1(t) * x);
    }
    __host__ __device__ Zipf(uint64_t n_, double theta) : s(theta), n((double)n_) {
        hx1 = hint(1.5) - 1.0;
        hn = hint(n + 0.5);
        sq = 2.0 - hinv(hint(2.5) - h(2.0));
    }
    // rank in [0, n): 0 is the most frequent
    __host__ __device__ uint64_t sample(uint64_t seed, uint64_t j) const {
        for (uint32_t attempt = 0; attempt < 64; attempt++) {
            const double u = hn + uniform01(seed, 7, j * 64 + attempt) * (hx1 - hn);
            const double x = hinv(u);
            double kd = floor(x + 0.5);
            if (kd < 1.0) kd = 1.0;
            if (kd > n) kd = n;
            if (kd - x <= sq || u >= hint(kd + 0.5) - h(kd)) return (uint64_t)kd - 1;
        }
        return 0;
    }
};

// ---- device generation kernels (grid-stride) ----
static __global__ void gen_pk_kernel(uint64_t *R, uint64_t n, Perm perm) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        R[i] = tword((uint32_t)(1 + perm(i)), (uint32_t)i);
}

static __global__ void gen_fk_kernel(uint64_t *S, uint64_t nS, const uint64_t *R, uint64_t nR, double theta,
                              uint64_t seed, uint32_t *idx_out, Perm rank_perm, Zipf z) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nS; j += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t idx = theta > 0 ? rank_perm(z.sample(seed, j)) : uniform_below(seed, 3, j, nR);
        S[j] = tword(tkey(R[idx]), (uint32_t)j);
        if (idx_out) idx_out[j] = (uint32_t)idx;
    }
}

static __global__ void gen_uniform_kernel(uint64_t *T, uint64_t n, uint64_t range, uint64_t seed) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        T[i] = tword((uint32_t)(1 + uniform_below(seed, 5, i, range)), (uint32_t)i);
}

}  // namespace adb
