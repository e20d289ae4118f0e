// npo_join.cuh -- no-partitioning hash join (NPO, NPO_st) on one global table.
//
// Replaces hashing/joins/no_partitioning_join.cpp:112-476 (NPO_st, npo_thread,
// np_distribute, NPO) and its table code in hashing/joins/common_functions.cpp
// (allocate_hashtable :75-102, build_hashtable_mt :350-400, probe_hashtable
// :221-280).  The reference chains 32-byte buckets of two tuples behind
// per-bucket latches; on the GPU the table is an open-addressing array of
// 8-byte tuple slots (the tuple word itself is the slot content), claimed with
// one 64-bit atomicCAS, probed linearly within and across 32-byte sectors.
// With 2 slots per build tuple (load <= 0.5) a probe touches one sector on
// average; a table of up to ~60 MB stays resident in the 126 MB L2.
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
    return log2n ? (uint32_t)((key * 0x9E3779B1u) >> (32 - log2n)) : 0u;
}

// static: each translation unit that includes this header gets its own copy
static __global__ void npo_build(const uint64_t *__restrict__ R, uint64_t nR, uint64_t *__restrict__ table,
                          uint32_t log2n, unsigned long long *sentinel_cnt, int *err) {
    const uint64_t mask = (1ULL << log2n) - 1;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nR; i += stride) {
        const uint64_t w = R[i];
        if (w == kEmpty) { atomicAdd(sentinel_cnt, 1ull); continue; }
        uint64_t slot = npo_hash(tkey(w), log2n);
        uint64_t tries = 0;
        while (true) {
            const unsigned long long prev =
                atomicCAS(reinterpret_cast<unsigned long long *>(table + slot), (unsigned long long)kEmpty,
                          (unsigned long long)w);
            if (prev == kEmpty) break;
            slot = (slot + 1) & mask;
            if (++tries > mask) { atomicExch(err, 2); break; }   // table full: cannot happen at load <= 0.5
        }
    }
}

template <bool kMaterialize>
__global__ void npo_probe(const uint64_t *__restrict__ S, uint64_t nS, const uint64_t *__restrict__ table,
                          uint32_t log2n, const unsigned long long *sentinel_cnt, unsigned long long *acc,
                          uint64_t *mat, unsigned long long *mat_n, uint64_t mat_cap) {
    __shared__ uint64_t red[64];
    const uint64_t mask = (1ULL << log2n) - 1;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t nsent = *sentinel_cnt;
    Acc a;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nS; i += stride) {
        const uint64_t s = __ldcs(reinterpret_cast<const unsigned long long *>(S) + i);
        const uint32_t key = tkey(s);
        const uint64_t sh = s_half(key, tpay(s));
        uint64_t slot = npo_hash(key, log2n);
        for (uint64_t tries = 0; tries <= mask; tries++) {
            const uint64_t v = table[slot];
            if (v == kEmpty) break;
            if (tkey(v) == key) {
                a.count++;
                a.sum += pair_hash_pre(key, tpay(v), sh);
                if (kMaterialize) {
                    const unsigned long long k = atomicAdd(mat_n, 1ull);
                    if (k < mat_cap) mat[k] = s;
                }
            }
            slot = (slot + 1) & mask;
        }
        if (key == 0xFFFFFFFFu && nsent) {
            a.count += nsent;
            a.sum += nsent * pair_hash_pre(key, 0xFFFFFFFFu, sh);
            if (kMaterialize)
                for (uint64_t t = 0; t < nsent; t++) {
                    const unsigned long long k = atomicAdd(mat_n, 1ull);
                    if (k < mat_cap) mat[k] = s;
                }
        }
    }
    block_flush(a, acc, red);
}

}  // namespace adb
