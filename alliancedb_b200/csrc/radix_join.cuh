// radix_join.cuh -- per-partition build/probe of the partitioned hash joins.
//
// Replaces, per partition pair (R_p, S_p) produced by partition.cuh:
//   bucket_chaining_join   hashing/joins/parallel_radix_join.cpp:291-354   (PRO, RJ_st)
//   histogram_join         hashing/joins/parallel_radix_join.cpp:373-432   (PRH, PRHO)
// and the task-queue loop of prj_thread (:1409-1416) with a persistent kernel
// that steals work items from a global counter.  A work item is
// (partition p, R chunk, S chunk): the R chunk (<= kRCap tuples) is loaded into
// shared memory with bulk async copies (cp.async.bulk global->shared, completion
// on an mbarrier), a table is built there, and the S chunk is streamed from
// global memory and probed.  Partitions whose R side exceeds kRCap (duplicate
// or skewed build keys) are covered by several R chunks; skewed S partitions
// by several S chunks, so no item is larger than kRCap x kSChunk.
#pragma once

#include "adb_common.cuh"
#include "partition.cuh"

namespace adb {

constexpr int kJoinThreads = 1024;
constexpr uint32_t kRCap = 8192;       // R tuples per item held in shared memory
constexpr uint32_t kSChunk = 16384;    // S tuples per item

// Work items of a partitioned join: items_off[p] = first item of partition p.
__global__ void make_items(const uint64_t *starts, uint32_t F, uint32_t *items_off,
                           uint32_t *n_items, uint32_t rcap, uint32_t schunk) {
    __shared__ uint32_t tmp[32];
    __shared__ uint32_t carry;
    const uint64_t *sR = starts, *sS = starts + (F + 1);
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < F; base += blockDim.x) {
        const uint32_t p = base + threadIdx.x;
        uint32_t v = 0;
        if (p < F) {
            const uint64_t nr = sR[p + 1] - sR[p], ns = sS[p + 1] - sS[p];
            if (nr && ns) v = (uint32_t)(((nr + rcap - 1) / rcap) * ((ns + schunk - 1) / schunk));
        }
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan(v, tmp, &tot);
        if (p < F) items_off[p] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) { items_off[F] = carry; *n_items = carry; }
}

__device__ __forceinline__ uint32_t find_part(const uint32_t *items_off, uint32_t F, uint32_t item) {
    // largest p with items_off[p] <= item (items_off is non-decreasing)
    uint32_t lo = 0, hi = F;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (items_off[mid] <= item) lo = mid; else hi = mid;
    }
    return lo;
}

// --- bulk async copy helpers (sm_90+ PTX) -----------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst_smem, const void *src_gmem, uint32_t bytes, uint64_t *bar) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst_smem);
    const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d),
        "l"(src_gmem), "r"(bytes), "r"(b)
        : "memory");
}
// Bounded wait on the mbarrier phase; returns false when the bound runs out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t phase) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    for (uint32_t it = 0; it < (1u << 22); it++) {
        uint32_t done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(a), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

enum class TableKind { Chain = 0, Hist = 1 };

// Shared memory: raw[kRCap + 2] u64 (the R chunk as copied, from the 16-byte
// boundary at or before its first tuple) | tup2[kRCap] u64 | aux[kRCap] u32 |
// heads[kRCap + 2] u32 | mbarrier, reduction and item slots.
constexpr size_t kJoinSmem = ((size_t)kRCap + 2) * 8 + (size_t)kRCap * 8 + (size_t)kRCap * 4 +
                             ((size_t)kRCap + 2) * 4 + 1024;

struct JoinArgs {
    const uint64_t *R;       // partitioned R
    const uint64_t *S;       // partitioned S
    const uint64_t *starts;  // [2][F+1]
    const uint32_t *items_off;
    const uint32_t *n_items;
    uint32_t *work_counter;
    unsigned long long *acc;  // [2] count, checksum
    int *err;                 // set on a timed-out wait
    uint32_t F;
    uint32_t bits;           // radix bits consumed by the partitioning (hash skips them)
    // optional materialisation: <S-key, S-payload> per match
    uint64_t *mat;
    unsigned long long *mat_n;
    uint64_t mat_cap;
};

template <TableKind K>
__global__ void __launch_bounds__(kJoinThreads, 1)
radix_join_items(JoinArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t *raw = reinterpret_cast<uint64_t *>(smem);                  // R chunk as copied
    uint64_t *tup2 = raw + kRCap + 2;                                    // reordered (Hist)
    uint32_t *aux = reinterpret_cast<uint32_t *>(tup2 + kRCap);          // next[] / ranks
    uint32_t *heads = aux + kRCap;                                       // bucket heads / hist
    uint64_t *bar = reinterpret_cast<uint64_t *>(heads + kRCap + 2);
    uint64_t *red = bar + 2;                                             // 64 u64
    uint32_t *item_sh = reinterpret_cast<uint32_t *>(red + 64);

    const uint32_t n_items = *a.n_items;
    if (threadIdx.x == 0) mbar_init(bar, 1);
    __syncthreads();
    uint32_t phase = 0;
    Acc acc;
    const uint32_t F = a.F;
    const uint64_t *sR = a.starts, *sS = a.starts + (F + 1);

    while (true) {
        if (threadIdx.x == 0) item_sh[0] = atomicAdd(a.work_counter, 1u);
        __syncthreads();
        const uint32_t item = item_sh[0];
        if (item >= n_items) break;
        const uint32_t p = find_part(a.items_off, F, item);
        const uint64_t r0 = sR[p], nr = sR[p + 1] - r0;
        const uint64_t s0 = sS[p], ns = sS[p + 1] - s0;
        const uint32_t sch = (uint32_t)((ns + kSChunk - 1) / kSChunk);
        const uint32_t local = item - a.items_off[p];
        const uint32_t rc = local / sch, sc = local % sch;
        const uint64_t rb = r0 + (uint64_t)rc * kRCap;
        const uint32_t nrc = (uint32_t)min((uint64_t)kRCap, nr - (uint64_t)rc * kRCap);
        const uint64_t sb = s0 + (uint64_t)sc * kSChunk;
        const uint32_t nsc = (uint32_t)min((uint64_t)kSChunk, ns - (uint64_t)sc * kSChunk);

        // --- load the R chunk with one bulk async copy.  The copy starts at the
        //     16-byte boundary at or before the chunk (o = 0 or 1 tuple early)
        //     and is rounded up to 16 bytes; the partition buffers carry two
        //     tuples of slack so both ends stay inside the allocation.
        const uint64_t *src = a.R + rb;
        const uint32_t o = (uint32_t)((reinterpret_cast<uintptr_t>(src) & 15) >> 3);
        const uint32_t copy_bytes = ((o + nrc) * 8 + 15) & ~15u;
        const uint64_t *tup = raw + o;
        if (threadIdx.x == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(bar, copy_bytes);
            bulk_g2s(raw, src - o, copy_bytes, bar);
        }
        uint32_t nb;   // buckets
        if (K == TableKind::Chain) {
            nb = 1;
            while (nb < nrc) nb <<= 1;                      // NEXT_POW_2(|R_i|)
        } else {
            nb = 1;
            while (nb < nrc) nb <<= 1;
            nb >>= 2;
            if (nb < 4) nb = 4;                             // get_hist_size
        }
        const uint32_t bmask = nb - 1;
        for (uint32_t i = threadIdx.x; i < nb + 2; i += blockDim.x) heads[i] = 0;
        if (!mbar_wait(bar, phase)) atomicExch(a.err, 1);
        phase ^= 1;
        __syncthreads();

        if (K == TableKind::Chain) {
            // build: next[i] = bucket[idx]; bucket[idx] = i + 1
            for (uint32_t i = threadIdx.x; i < nrc; i += blockDim.x) {
                const uint32_t h = (tkey(tup[i]) >> a.bits) & bmask;
                aux[i] = atomicExch(&heads[h], i + 1);
            }
            __syncthreads();
        } else {
            // histogram + prefix + reorder into tup2 (bucket-contiguous)
            for (uint32_t i = threadIdx.x; i < nrc; i += blockDim.x) {
                const uint32_t h = (tkey(tup[i]) >> a.bits) & bmask;
                aux[i] = atomicAdd(&heads[h + 1], 1u);
            }
            __syncthreads();
            {
                const uint32_t per = (nb + blockDim.x - 1) / blockDim.x;
                const uint32_t d0 = threadIdx.x * per;
                uint32_t loc = 0;
                for (uint32_t d = d0; d < min(nb, d0 + per); d++) loc += heads[d + 1];
                uint32_t tot;
                uint32_t ex = block_exclusive_scan(loc, item_sh + 4, &tot);
                __syncthreads();
                for (uint32_t d = d0; d < min(nb, d0 + per); d++) {
                    const uint32_t c = heads[d + 1];
                    heads[d + 1] = ex;     // heads[h+1] = start of bucket h
                    ex += c;
                }
                if (threadIdx.x == 0) heads[nb + 1] = tot;
            }
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < nrc; i += blockDim.x) {
                const uint32_t h = (tkey(tup[i]) >> a.bits) & bmask;
                tup2[heads[h + 1] + aux[i]] = tup[i];
            }
            __syncthreads();
        }

        // --- probe the S chunk
        const uint64_t *S = a.S + sb;
        for (uint32_t j = threadIdx.x; j < nsc; j += blockDim.x) {
            const uint64_t s = ld_stream(S + j);
            const uint32_t key = tkey(s);
            const uint32_t h = (key >> a.bits) & bmask;
            uint64_t sh = 0;
            bool have_sh = false;
            if (K == TableKind::Chain) {
                for (uint32_t hit = heads[h]; hit; hit = aux[hit - 1]) {
                    const uint64_t r = tup[hit - 1];
                    if (tkey(r) == key) {
                        if (!have_sh) { sh = s_half(key, tpay(s)); have_sh = true; }
                        acc.count++;
                        acc.sum += pair_hash_pre(key, tpay(r), sh);
                        if (a.mat) {
                            const unsigned long long slot = atomicAdd(a.mat_n, 1ull);
                            if (slot < a.mat_cap) a.mat[slot] = s;
                        }
                    }
                }
            } else {
                const uint32_t e = heads[h + 2];
                for (uint32_t t = heads[h + 1]; t < e; t++) {
                    const uint64_t r = tup2[t];
                    if (tkey(r) == key) {
                        if (!have_sh) { sh = s_half(key, tpay(s)); have_sh = true; }
                        acc.count++;
                        acc.sum += pair_hash_pre(key, tpay(r), sh);
                        if (a.mat) {
                            const unsigned long long slot = atomicAdd(a.mat_n, 1ull);
                            if (slot < a.mat_cap) a.mat[slot] = s;
                        }
                    }
                }
            }
        }
        __syncthreads();   // table is rebuilt by the next item
    }
    block_flush(acc, a.acc, red);
}

}  // namespace adb
