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
//      R chunk (<= 4096 tuples) and the item's S block into shared memory with
//      bulk async copies, sorts R, and joins S bucket by bucket against R's
//      sorted buckets (S is bucketed by the same key bits, not moved); only
//      keys 0xFFFFFFFF, or an R chunk that needed the bitonic fallback, sort S
//      as well and merge the two sorted runs with merge-path partitioning.
// The per-chunk sort is an MSD counting sort on the (at most) 11 highest key
// bits that differ within the chunk, followed by an insertion sort inside
// each bucket: the bits above those are equal across the chunk, so the result
// is fully sorted by key.  Ties between equal keys stay in arbitrary order,
// which merge_join does not depend on.
#include "joins.cuh"
#include "paged.cuh"
#include "radix_join.cuh"
#include "smj_sort.cuh"

namespace adb {

constexpr uint32_t kSmjCap = 4096;                  // tuples per R chunk and per S block
constexpr uint32_t kSmjChunkW = kSmjCap - kPageTuples;
constexpr uint32_t kSmjSPages = kSmjCap / kPageTuples;   // 64 pages <= 4096 tuples
constexpr uint32_t kSmjMaxPages = kSmjCap / kMinPageW + 16;   // pages of one R chunk (weight floor 32)
constexpr uint32_t kSmjThreads = 512;
constexpr int kSmjBlocks = 2;                       // CTAs per SM: one's barriers and copies hide behind the other

// A | B | C tuple buffers, bucket counters, two page tables (R pages then S
// pages: page id, dst << 8 | count), barrier, scratch and two item records.
constexpr uint32_t kSmjTabEntries = kSmjMaxPages + kSmjSPages + 1;
constexpr size_t kSmjSmem = (size_t)kSmjCap * 8 * 3 + (size_t)kDualCntWords * 4 + (size_t)kSmjTabEntries * 4 * 2 * 2 +
                            1024;
static_assert(kSmjBlocks * (kSmjSmem + 1024) <= 233472, "smj_items CTAs exceed the SM's shared memory");
static_assert(((size_t)kDualCntWords + (size_t)kSmjTabEntries * 4) % 2 == 0, "mbarrier must be 8-byte aligned");

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
    int waits_run_out;               // ADB_TEST_WAITS_RUN_OUT: report completed waits as run out
    uint32_t F;
    uint64_t *mat;
    unsigned long long *mat_n;
    uint64_t mat_cap;
};

// One work item as the control warp publishes it.
struct SmjRec {
    uint64_t rb, sb;                 // first page-list index of the R chunk / S block
    uint32_t item, nrpg, nspg;       // item (>= n_items: none), pages of each side
    uint32_t rslots, sslots;         // shared-memory slots of each side (pages rounded up to even)
    uint32_t rpad, spad;             // odd pages of each side (one all-ones pad word each)
    uint32_t pad_;
};

static_assert(16 + 8 * 112 + 2 * sizeof(SmjRec) <= 1024 && kDualRedWords <= 224,
              "barrier, scratch and records exceed the tail");

// Items are pipelined as in radix_join_items: while item i is merge-joined by
// warps 0 .. 30, the last warp builds the page table of item i + 1 and takes
// item i + 2, so no dependent global load sits between two items.
__global__ void __launch_bounds__(kSmjThreads, kSmjBlocks)
smj_items(SmjArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t *A = reinterpret_cast<uint64_t *>(smem);
    uint64_t *B = A + kSmjCap;
    uint64_t *C = B + kSmjCap;
    uint32_t *cnt = reinterpret_cast<uint32_t *>(C + kSmjCap);
    uint32_t *ptab = cnt + kDualCntWords;                    // [2] x {pg[kSmjTabEntries], dst << 8 | count []}
    uint64_t *bar = reinterpret_cast<uint64_t *>(ptab + 4 * kSmjTabEntries);
    uint64_t *red = bar + 2;                                 // 112 u64 (224 u32 of sort scratch)
    SmjRec *rec = reinterpret_cast<SmjRec *>(red + 112);     // [2]
    __shared__ uint32_t runn[2];   // length of R's run of a single S key, per item parity

    const uint32_t n_items = *a.n_items;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int kWarps = kSmjThreads / 32;
    constexpr int kCtl = kWarps - 1;
    constexpr uint32_t kWork = kSmjThreads - 32;             // threads of the merge join
    const uint32_t F = a.F;

    // control warp: take the next item into r
    auto take = [&](SmjRec *r) {
        uint32_t item = 0;
        if (lane == 0) item = atomicAdd(a.work_counter, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        uint32_t p = 0;
        if (item < n_items) p = warp_find(a.items_off, F, item, lane);
        if (lane == 0) {
            r->item = item;
            if (item < n_items) {
                const ItemGeo g = item_geo(a, item, p, kSmjSPages);
                r->rb = g.rb;
                r->sb = g.sb;
                r->nrpg = g.nrpg;
                r->nspg = g.nspg;
            }
        }
        __syncwarp();
    };
    // control warp: page table of item r (R pages to A, S pages to C, 16-byte
    // aligned slots), its slot and pad counts, and the mbarrier's expected bytes
    auto table = [&](SmjRec *r, uint32_t *pt) {
        if (r->item >= n_items) return;
        uint32_t *tpg = pt, *tpk = pt + kSmjTabEntries;
        uint32_t slots_of[2] = {0, 0}, pads_of[2] = {0, 0};
        constexpr int U = 4;
#pragma unroll
        for (int side = 0; side < 2; side++) {
            const uint32_t n = side ? r->nspg : r->nrpg;
            const uint64_t b0 = side ? r->sb : r->rb;
            const uint32_t *list = side ? a.Slist : a.Rlist;
            const uint8_t *count = side ? a.Scount : a.Rcount;
            const uint32_t k0 = side ? r->nrpg : 0u;
            uint32_t carry = 0, pads = 0;
            for (uint32_t base = 0; base < n; base += 32 * U) {
                uint32_t pg[U], c[U];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const uint32_t k = base + 32 * u + lane;
                    pg[u] = k < n ? list[b0 + k] : kNone;
                }
#pragma unroll
                for (int u = 0; u < U; u++) c[u] = pg[u] != kNone ? count[pg[u]] : 0u;
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const uint32_t k = base + 32 * u + lane;
                    const uint32_t e = (c[u] + 1) & ~1u;
                    const uint32_t inc = warp_incl_scan(e, lane);
                    if (k < n) {
                        tpg[k0 + k] = pg[u];
                        tpk[k0 + k] = ((carry + inc - e) << 8) | c[u];
                    }
                    carry += __shfl_sync(0xffffffffu, inc, 31);
                    pads += __popc(__ballot_sync(0xffffffffu, c[u] & 1u));
                }
            }
            slots_of[side] = carry;
            pads_of[side] = pads;
        }
        if (lane == 0) {
            r->rslots = slots_of[0];
            r->sslots = slots_of[1];
            r->rpad = pads_of[0];
            r->spad = pads_of[1];
            // the item's copies are issued after the next barrier, in its phase
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(bar, (slots_of[0] + slots_of[1]) * 8);
        }
        __syncwarp();
    };

    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        runn[0] = runn[1] = 0;
    }
    if (warp == kCtl) {
        take(&rec[0]);
        table(&rec[0], ptab);
        take(&rec[1]);
    }
    __syncthreads();
    uint32_t phase = 0;
    int cur = 0;
    Acc acc;

    while (true) {
        const SmjRec cr = rec[cur];
        if (cr.item >= n_items) break;
        const uint32_t *tpg = ptab + cur * 2 * kSmjTabEntries;
        const uint32_t *tpk = tpg + kSmjTabEntries;
        const uint32_t nrpg = cr.nrpg, np = cr.nrpg + cr.nspg;
        const uint32_t rslots = cr.rslots, sslots = cr.sslots, rpad = cr.rpad, spad = cr.spad;
        if (threadIdx.x == 0) runn[cur ^ 1] = 0;   // the next item's (this item's was zeroed the same way)

        // --- R chunk -> A and S block -> C, one bulk copy per page, page slots
        //     16-byte aligned (a page takes its count rounded up to even); the
        //     pad slot behind an odd page arrives holding the all-ones word (the
        //     partition pass wrote it there), which sorts last and is cut off
        //     by count
        for (uint32_t k = threadIdx.x; k < np; k += blockDim.x) {
            const uint32_t v = tpk[k], c = v & 0xFFu;
            if (c) {
                const bool isr = k < nrpg;
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                bulk_g2s((isr ? A : C) + (v >> 8), (isr ? a.Rpages : a.Spages) + (uint64_t)tpg[k] * kPageTuples,
                         ((c + 1) & ~1u) * 8, bar);
            }
        }
        // every thread waits on the mbarrier itself, which makes the copied
        // words visible to it: no block barrier before the analysis
        if (!mbar_wait(bar, phase) || a.waits_run_out) atomicExch(a.err, 1);
        phase ^= 1;
        // sorted R (+ pads) in B; sorted S (+ pads) in A where the merge path
        // needs it, else S stays in C and is only bucketed.  The pads are the
        // last words of each sorted run and a real all-ones tuple is the same
        // word, so dropping as many words as there are pads is exact.  An S
        // block of one key K is not sorted, and neither is R: R's run of K is
        // gathered into B.
        uint32_t *red32 = reinterpret_cast<uint32_t *>(red);
        DualSort ds = dual_analyze(A, rslots, C, sslots, cnt, red32, spad);
        // all-ones words beyond the pads: real tuples with key 0xFFFFFFFF
        const bool ones = ds.onesx != rpad || ds.onesy != spad;
        // the S block needs an order only for the merge path (keys 0xFFFFFFFF);
        // the bucket path meets each S word with R's sorted bucket of the
        // same index, so there S is only bucketed, not moved (block-uniform)
        const bool sort_s = ds.max_key || ones;
        if (ds.y_single) {
            for (uint32_t i = threadIdx.x; i < rslots; i += blockDim.x) {
                const uint64_t v = A[i];   // pads are all-ones words: K < 0xFFFFFFFF never meets them
                if (tkey(v) == ds.y_key) B[atomicAdd(&runn[cur], 1u)] = v;
            }
            __syncthreads();
        } else {
            dual_sort_rest(ds, A, rslots, B, C, sslots, A, cnt, red32, sort_s);
            if (ds.bitonic && !sort_s) {   // R took the bitonic path: the merge path needs S sorted too
                for (uint32_t i = threadIdx.x; i < sslots; i += blockDim.x) A[i] = C[i];
                __syncthreads();
                bitonic_words(A, sslots);
            }
        }
        const uint32_t nr = rslots - rpad, ns = sslots - spad;
        const uint64_t *Rs = B, *Ss = A;

        // --- merge-join of the sorted runs by warps 0 .. 30; the control warp
        //     prepares the next item and takes the one after it (rec[cur] is
        //     free: every thread copied it at the top of the item)
        if (warp == kCtl) {
            table(&rec[cur ^ 1], ptab + (cur ^ 1) * 2 * kSmjTabEntries);
            take(&rec[cur]);
        }
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
        if (ds.y_single) {
            // the S block is one key K (a hot key under skew), left unsorted in C
            // with its pads: every S word but the pads meets R's run of K, B[0..runn[cur])
            const uint32_t nrun = runn[cur];
            for (uint32_t j = threadIdx.x; j < sslots && warp != kCtl && nrun; j += kWork) {
                const uint64_t s = C[j];
                if (s == ~0ULL) continue;   // a pad
                uint64_t sh = 0;
                bool have = false;
                for (uint32_t t = 0; t < nrun; t++) emit(s, Rs[t], sh, have);
            }
        } else if (!ds.bitonic && !sort_s) {
            // S word s in bucket d meets R bucket d, whose sorted range
            // [ex[d - 1], ex[d]) holds every R tuple that can have s's key; no
            // key is 0xFFFFFFFF, so the all-ones words in the unsorted S block
            // are exactly its pads and are skipped
            const uint16_t *cx = ds.ex;
            for (uint32_t j = threadIdx.x; j < sslots && warp != kCtl; j += kWork) {
                const uint64_t s = C[j];
                if (s == ~0ULL) continue;   // a pad
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
        } else if (warp != kCtl) {
            // merge path over the whole runs; R first on equal keys
            const uint32_t total = nr + ns;
            const uint32_t L = (total + kWork - 1) / kWork;
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
        __syncthreads();   // the next item overwrites the buffers; rec / page tables published
        cur ^= 1;
    }
    block_flush(acc, a.acc, red);
}

static void smj_bits(uint64_t nR, int part_fanout, uint32_t *b1, uint32_t *b2) {
    int bits;
    if (part_fanout > 1) {
        bits = (int)ceil_log2_u64((uint64_t)part_fanout);
    } else {
        bits = (int)ceil_log2_u64((nR + kSmjCap / 2 - 1) / (kSmjCap / 2));   // R partitions of about half a chunk
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
    const DigitFn d1{0u, (1u << b1) - 1};
    const DigitFn d2{b1, (1u << b2) - 1};
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
    a.waits_run_out = j.test_flags & ADB_TEST_WAITS_RUN_OUT;
    a.F = F;
    a.mat = j.mat; a.mat_n = acc + 3; a.mat_cap = j.mat_cap;
    smj_items<<<ctx->num_sms * kSmjBlocks, kSmjThreads, kSmjSmem, st>>>(a);
    ADB_CK(cudaGetLastError());
    ctx->kernels += 4;
    return ADB_OK;
}

int smj_set_attrs() {
    ADB_CK(cudaFuncSetAttribute(smj_items, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmjSmem));
    return ADB_OK;
}

}  // namespace adb
