// smj.cu -- sort-merge joins (m-way, m-pass, m-way+skew).
//
// Reference: sortmergejoin_multiway (sorting/joins/sortmergejoin_multiway.cpp:55-700):
// partitioning_phase (MSB radix into PARTFANOUT partitions, :435-497),
// sorting_phase (AVX sort of each partition, :499-567), multiwaymerge_phase
// (:569-660) and mergejoin_phase -> merge_join (sorting/joins/common_functions.cpp
// :298-372), which joins two sorted runs including the cross product of
// duplicate keys.  m-pass (sortmergejoin_multipass.cpp) differs only in merging
// pairwise.
//
// On the device both names run one pipeline:
//   1. the paged partitioning front end (radix.cu) on the low key bits: equal
//      keys meet in one partition, as the reference's range partition
//      guarantees for its key ranges;
//   2. smj_items, a persistent work-stealing kernel: per work item it copies an
//      R chunk (<= 8192 tuples) into shared memory with bulk async copies, sorts
//      it, loads and sorts the item's S block, and merge-joins the two sorted
//      runs with merge-path partitioning across the CTA's threads.
// The per-chunk sort is an MSD counting sort on the (at most) 12 highest key
// bits that differ within the chunk, followed by an insertion sort inside
// each bucket: the bits above those are equal across the chunk, so the result
// is fully sorted by key.  Ties between equal keys stay in arbitrary order,
// which merge_join does not depend on.
#include "joins.cuh"
#include "paged.cuh"
#include "radix_join.cuh"
#include "smj_sort.cuh"

namespace adb {

constexpr uint32_t kSmjCap = 8192;                  // tuples per R chunk and per S block
constexpr uint32_t kSmjChunkW = kSmjCap - kPageTuples;
constexpr uint32_t kSmjSPages = kSmjCap / kPageTuples;   // 128 pages <= 8192 tuples
constexpr uint32_t kSmjMaxPages = 272;              // weight floor 32: <= 8192 / 32 + 1 pages per chunk
constexpr uint32_t kSmjThreads = 1024;

// A | B | C tuple buffers, bucket counters, R and S page tables, barrier and scratch.
constexpr size_t kSmjSmem = (size_t)kSmjCap * 8 * 3 + ((size_t)(1u << kDualBucketBits) + 2) * 4 * 2 +
                            ((size_t)kSmjMaxPages + 1) * 4 * 2 + ((size_t)kSmjSPages + 1) * 4 * 2 + 1024;
static_assert(kSmjSmem <= 232448, "smj_items exceeds the 227 KB shared-memory limit");
static_assert(kSmjMaxPages + kSmjSPages <= kSmjThreads, "one page-table entry per thread");

struct SmjArgs {
    const uint64_t *Rpages, *Spages;
    const uint8_t *Rcount, *Scount;
    const uint32_t *Rlist, *Slist;
    const uint64_t *pstart;          // [2][F+1]
    const uint32_t *items_off, *chunk_off;
    const uint64_t *cstart;
    const uint32_t *n_items;
    uint32_t *work_counter;
    unsigned long long *acc;
    int *err;
    uint32_t F;
    uint64_t *mat;
    unsigned long long *mat_n;
    uint64_t mat_cap;
};

__global__ void __launch_bounds__(kSmjThreads, 1)
smj_items(SmjArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t *A = reinterpret_cast<uint64_t *>(smem);
    uint64_t *B = A + kSmjCap;
    uint64_t *C = B + kSmjCap;
    uint32_t *cnt = reinterpret_cast<uint32_t *>(C + kSmjCap);
    uint32_t *pdst = cnt + 2 * ((1u << kDualBucketBits) + 2);   // R page table
    uint32_t *pcnt = pdst + kSmjMaxPages + 1;
    uint32_t *sdst = pcnt + kSmjMaxPages + 1;                // S page table
    uint32_t *scnt = sdst + kSmjSPages + 1;
    uint64_t *bar = reinterpret_cast<uint64_t *>(scnt + kSmjSPages + 1);
    uint64_t *red = bar + 2;                                 // 64 u64 (96 u32 of sort scratch)
    uint32_t *slots = reinterpret_cast<uint32_t *>(red + 64);   // [0..3) next item, [4..36) scan scratch

    const uint32_t n_items = *a.n_items;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int kWarps = kSmjThreads / 32;
    if (threadIdx.x == 0) mbar_init(bar, 1);
    if (warp == 0) take_item(a.work_counter, a.items_off, a.F, n_items, nullptr, 0, slots, lane);
    __syncthreads();
    uint32_t phase = 0;
    Acc acc;
    const uint32_t F = a.F;
    const uint64_t *pR = a.pstart, *pS = a.pstart + (F + 1);

    while (true) {
        const uint32_t item = slots[0];
        if (item >= n_items) break;
        const uint32_t p = slots[1];
        const uint64_t r0 = pR[p], nrp = pR[p + 1] - r0;
        const uint64_t s0 = pS[p], nsp = pS[p + 1] - s0;
        const uint32_t sch = (uint32_t)((nsp + kSmjSPages - 1) / kSmjSPages);
        const uint32_t local = item - a.items_off[p];
        const uint32_t rc = local / sch, sc = local % sch;
        const uint32_t cid = a.chunk_off[p] + rc;
        const uint64_t rb = a.cstart[cid];
        const uint64_t re = rc + 1 < a.chunk_off[p + 1] - a.chunk_off[p] ? a.cstart[cid + 1] : r0 + nrp;
        const uint32_t nrpg = (uint32_t)(re - rb);
        const uint64_t sb = s0 + (uint64_t)sc * kSmjSPages;
        const uint32_t nspg = (uint32_t)min((uint64_t)kSmjSPages, nsp - (uint64_t)sc * kSmjSPages);

        // --- R chunk -> A and S block -> C, one bulk copy per page, page slots
        //     16-byte aligned (a page takes its count rounded up to even); the
        //     pad slot behind an odd page is set to the all-ones word afterwards,
        //     which sorts last and is cut off by count
        uint32_t rslots, sslots, rpad, spad;
        {
            const uint32_t k = threadIdx.x;   // one page per thread: R pages, then S pages
            const bool isr = k < nrpg, iss = !isr && k < nrpg + nspg;
            uint32_t c = 0;
            if (isr) c = a.Rcount[a.Rlist[rb + k]];
            else if (iss) c = a.Scount[a.Slist[sb + (k - nrpg)]];
            const uint32_t e = (c + 1) & ~1u;
            uint32_t tot;
            const uint32_t ex = block_exclusive_scan(isr ? e : (e << 16), slots + 4, &tot);   // R | S << 16
            rslots = tot & 0xFFFFu;
            sslots = tot >> 16;
            if (isr) { pdst[k] = ex & 0xFFFFu; pcnt[k] = c; }
            if (iss) { sdst[k - nrpg] = (ex >> 16); scnt[k - nrpg] = c; }
            if (threadIdx.x == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                mbar_expect_tx(bar, (rslots + sslots) * 8);
            }
            rpad = __syncthreads_count(isr && (c & 1));
            spad = __syncthreads_count(iss && (c & 1));
        }
        for (uint32_t k = threadIdx.x; k < nrpg + nspg; k += blockDim.x) {
            const bool isr = k < nrpg;
            const uint32_t kk = isr ? k : k - nrpg;
            const uint32_t c = isr ? pcnt[kk] : scnt[kk];
            if (c) {
                const uint32_t pg = isr ? a.Rlist[rb + kk] : a.Slist[sb + kk];
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                bulk_g2s(isr ? A + pdst[kk] : C + sdst[kk], (isr ? a.Rpages : a.Spages) + (uint64_t)pg * kPageTuples,
                         ((c + 1) & ~1u) * 8, bar);
            }
        }
        if (!mbar_wait(bar, phase)) atomicExch(a.err, 1);
        phase ^= 1;
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < nrpg + nspg; k += blockDim.x) {
            const bool isr = k < nrpg;
            const uint32_t kk = isr ? k : k - nrpg;
            const uint32_t c = isr ? pcnt[kk] : scnt[kk];
            if (c & 1) (isr ? A + pdst[kk] : C + sdst[kk])[c] = ~0ULL;
        }
        __syncthreads();
        // sorted R (+ pads) in B, sorted S (+ pads) in A; the pads are the last
        // words of each run and a real all-ones tuple is the same word, so
        // dropping as many words as there are pads is exact
        const DualSort ds = dual_chunk_sort(A, rslots, B, C, sslots, A, cnt, reinterpret_cast<uint32_t *>(red));
        const uint32_t nr = rslots - rpad, ns = sslots - spad;
        const uint64_t *Rs = B, *Ss = A;

        // --- merge-join of the sorted runs; warp 0 first takes the next item
        if (warp == 0) take_item(a.work_counter, a.items_off, F, n_items, nullptr, 0, slots, lane);
        auto emit = [&](uint64_t s, uint64_t r, uint64_t &sh, bool &have) {
            const uint32_t key = tkey(s);
            if (!have) { sh = s_half(key, tpay(s)); have = true; }
            acc.count++;
            acc.sum += pair_hash_pre(key, tpay(r), sh);
            if (a.mat) {
                const unsigned long long m = atomicAdd(a.mat_n, 1ull);
                if (m < a.mat_cap) a.mat[m] = s;
            }
        };
        // all-ones words beyond the pads: real tuples with key 0xFFFFFFFF
        const bool ones = !ds.bitonic && (rslots - (ds.nb ? cnt[ds.nb - 1] : 0u) != rpad ||
                                          sslots - (ds.nb ? cnt[2 * ds.nb] : 0u) != spad);
        if (!ds.bitonic && !ds.max_key && !ones) {
            // both runs are ordered by the same buckets: S bucket d meets R bucket
            // d, whose sorted range [cnt[d - 1], cnt[d]) holds every R tuple that
            // can have the S tuple's key; no key is 0xFFFFFFFF, so no pad matches
            const uint32_t *cx = cnt;
            for (uint32_t j = threadIdx.x; j < ns; j += blockDim.x) {
                const uint64_t s = Ss[j];
                const uint32_t key = tkey(s);
                const uint32_t d = ds.bucket(s);
                uint64_t sh = 0;
                bool have = false;
                for (uint32_t t = d ? cx[d - 1] : 0u, e = cx[d]; t < e; t++) {
                    const uint64_t r = Rs[t];
                    if (tkey(r) > key) break;
                    if (tkey(r) == key) emit(s, r, sh, have);
                }
            }
        } else {
            // merge path over the whole runs; R first on equal keys
            const uint32_t total = nr + ns;
            const uint32_t L = (total + blockDim.x - 1) / blockDim.x;
            const uint32_t k0 = min(total, threadIdx.x * L), k1 = min(total, k0 + L);
            uint32_t lo = k0 > ns ? k0 - ns : 0u, hi = k0 < nr ? k0 : nr;
            while (lo < hi) {   // number of R tuples among the first k0 merged
                const uint32_t mid = (lo + hi) >> 1;
                if (tkey(Rs[mid]) <= tkey(Ss[k0 - mid - 1])) lo = mid + 1; else hi = mid;
            }
            uint32_t i = lo, j = k0 - lo;
            for (uint32_t k = k0; k < k1; k++) {
                if (j >= ns || (i < nr && tkey(Rs[i]) <= tkey(Ss[j]))) {
                    i++;
                } else {
                    const uint64_t s = Ss[j];
                    const uint32_t key = tkey(s);
                    uint64_t sh = 0;
                    bool have = false;
                    for (int t = (int)i - 1; t >= 0 && tkey(Rs[t]) == key; t--) emit(s, Rs[t], sh, have);
                    j++;
                }
            }
        }
        __syncthreads();
    }
    block_flush(acc, a.acc, red);
}

static void smj_bits(uint64_t nR, int part_fanout, uint32_t *b1, uint32_t *b2) {
    int bits;
    if (part_fanout > 1) {
        bits = (int)ceil_log2_u64((uint64_t)part_fanout);
    } else {
        bits = (int)ceil_log2_u64((nR + 4095) / 4096);   // R partitions of about half a chunk
    }
    if (bits < 1) bits = 1;
    if (bits > 16) bits = 16;
    if (bits <= (int)kSmallPassBits) {
        *b1 = bits;
        *b2 = 0;
    } else {
        *b1 = bits / 2;
        *b2 = bits - bits / 2;
    }
}

size_t smj_scratch(uint64_t nR, uint64_t nS, int part_fanout, int num_sms) {
    uint32_t b1, b2;
    smj_bits(nR, part_fanout, &b1, &b2);
    const uint64_t F = 1ull << (b1 + b2);
    const uint64_t pages = paged_final_pool_pages(nR, nS, b1, b2, num_sms);
    return paged_partition_scratch(nR, nS, b1, b2, num_sms) + Workspace::need(F, 4) * 2 +
           Workspace::need(F + 1, 4) * 2 + Workspace::need(pages * kPageTuples / kSmjChunkW + F + 1, 8) +
           Workspace::need(2, 4);
}

int run_smj(Context *ctx, const DevJoin &j, int part_fanout, bool /*multipass*/, unsigned long long *acc) {
    cudaStream_t st = ctx->stream;
    uint32_t b1, b2;
    smj_bits(j.nR, part_fanout, &b1, &b2);
    const DigitFn d1{0u, 0u, (1u << b1) - 1};
    const DigitFn d2{0u, b1, (1u << b2) - 1};
    PartOut po;
    ADB_TRY(run_paged_partition(ctx, j, d1, b2 ? &d2 : nullptr, &po, acc));
    ADB_CK(cudaEventRecord(ctx->ev[1], st));

    const uint32_t F = po.Fout;
    uint32_t *rch = ctx->ws.take<uint32_t>(F);
    uint32_t *sch = ctx->ws.take<uint32_t>(F);
    uint32_t *items_off = ctx->ws.take<uint32_t>(F + 1);
    uint32_t *chunk_off = ctx->ws.take<uint32_t>(F + 1);
    uint64_t *cstart = ctx->ws.take<uint64_t>(po.pool_pages * kPageTuples / kSmjChunkW + F + 1);
    uint32_t *ctr = ctx->ws.take<uint32_t>(2);
    ADB_CK(cudaMemsetAsync(ctr, 0, 2 * sizeof(uint32_t), st));
    part_rslots<<<(F + 7) / 8, 256, 0, st>>>(po.pstart, po.R.plist, po.R.pcount, F, kSmjChunkW, kSmjSPages, rch,
                                             sch);
    make_items_paged<<<1, 1024, 0, st>>>(rch, sch, F, items_off, chunk_off, ctr);
    part_rchunks<<<(F + 7) / 8, 256, 0, st>>>(po.pstart, po.R.plist, po.R.pcount, F, kSmjChunkW, chunk_off, cstart);
    ADB_CK(cudaGetLastError());
    ADB_CK(cudaEventRecord(ctx->ev[2], st));
    ADB_CK(cudaEventRecord(ctx->ev[3], st));

    SmjArgs a;
    a.Rpages = po.R.pages; a.Spages = po.S.pages;
    a.Rcount = po.R.pcount; a.Scount = po.S.pcount;
    a.Rlist = po.R.plist; a.Slist = po.S.plist;
    a.pstart = po.pstart; a.items_off = items_off; a.chunk_off = chunk_off; a.cstart = cstart;
    a.n_items = ctr; a.work_counter = ctr + 1;
    a.acc = acc; a.err = reinterpret_cast<int *>(acc + 2);
    a.F = F;
    a.mat = j.mat; a.mat_n = acc + 3; a.mat_cap = j.mat_cap;
    smj_items<<<ctx->num_sms, kSmjThreads, kSmjSmem, st>>>(a);
    ADB_CK(cudaGetLastError());
    ctx->kernels += 4;
    return ADB_OK;
}

int smj_set_attrs() {
    ADB_CK(cudaFuncSetAttribute(smj_items, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmjSmem));
    return ADB_OK;
}

}  // namespace adb
