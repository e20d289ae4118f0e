// radix_join.cuh -- per-partition build/probe of the partitioned hash joins.
//
// Replaces, per partition pair (R_p, S_p) produced by paged.cuh:
//   bucket_chaining_join   hashing/joins/parallel_radix_join.cpp:291-354   (PRO, RJ_st)
//   histogram_join         hashing/joins/parallel_radix_join.cpp:373-432   (PRH, PRHO)
// and the task-queue loop of prj_thread (:1409-1416) with a persistent kernel
// that takes work items from a global counter (work stealing).  A work item is
// (partition p, R chunk, S chunk): an R chunk is a run of R_p's pages packed
// greedily up to kRSlots tuples (part_rchunks), copied into shared memory with
// one bulk async copy per page
// (cp.async.bulk global->shared, completion counted on an mbarrier), the table
// is built there, and up to kSPages pages of S_p are streamed from global
// memory and probed, one warp per page.  Large R partitions (duplicate or
// skewed build keys, or |R| beyond 2^12 * 16K) take several R chunks; large S
// partitions (skewed probe keys) several S chunks.
#pragma once

#include "adb_common.cuh"
#include "paged.cuh"

namespace adb {

constexpr int kJoinThreads = 1024;
constexpr int kJoinMinBlocks = 1;                          // CTAs per SM
constexpr uint32_t kRSlots = 17408;                        // R tuples a CTA holds (136 KB)
constexpr uint32_t kChunkW = kRSlots - kPageTuples;        // chunk weight budget
constexpr uint32_t kMinPageW = 32;                         // weight floor of a page
constexpr uint32_t kRMaxPages = kChunkW / kMinPageW + 16;  // pages of one R chunk (bound)
constexpr int kProbeWarps = kJoinThreads / 32 - 1;        // the last warp is the control warp
constexpr uint32_t kSPages = kProbeWarps * 32;             // S pages per item: <= 32 per probing warp (one per lane)
constexpr uint32_t kMaxHeads = kRSlots >= 16384 ? 8192 : 4096;   // Chain: bucket heads (~2 slots each)
constexpr uint32_t kMaxHist = kMaxHeads / 4;               // Hist: buckets

__device__ __forceinline__ uint32_t page_weight(uint32_t cnt) {
    const uint32_t e = (cnt + 1) & ~1u;                    // slots a page occupies (16-byte copies)
    return e > kMinPageW ? e : kMinPageW;
}

// Per partition: R chunk count (greedy by page weight, chunk_w per chunk) and
// S chunk count (s_pages pages per chunk).  One warp per partition.
static __global__ void part_rslots(const uint64_t *pstart, const uint32_t *Rlist, const uint8_t *Rcount, uint32_t F,
                            uint32_t chunk_w, uint32_t s_pages, uint32_t *rch, uint32_t *sch) {
    const int lane = threadIdx.x & 31;
    const uint32_t p = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (p >= F) return;
    const uint64_t *pR = pstart, *pS = pstart + (F + 1);
    const uint64_t r0 = pR[p], r1 = pR[p + 1];
    uint64_t wsum = 0, wlast = 0;
    for (uint64_t k = r0 + lane; k < r1; k += 32) {
        const uint32_t w = page_weight(Rcount[Rlist[k]]);
        wsum += w;
        if (k == r1 - 1) wlast = w;
    }
    wsum = warp_sum_u64(wsum);
    wlast = warp_sum_u64(wlast);
    if (lane == 0) {
        const uint64_t nS = pS[p + 1] - pS[p];
        rch[p] = r1 > r0 ? (uint32_t)((wsum - wlast) / chunk_w + 1) : 0u;
        sch[p] = (uint32_t)((nS + s_pages - 1) / s_pages);
    }
}

// Work items (R chunk x S chunk) and R chunk offsets: items_off[p], chunk_off[p].
static __global__ void make_items_paged(const uint32_t *rch, const uint32_t *sch, uint32_t F, uint32_t *items_off,
                                 uint32_t *chunk_off, uint32_t *n_items) {
    __shared__ uint32_t tmp[32];
    __shared__ uint32_t carry[2];
    if (threadIdx.x == 0) carry[0] = carry[1] = 0;
    __syncthreads();
    for (uint32_t base = 0; base < F; base += blockDim.x) {
        const uint32_t p = base + threadIdx.x;
        uint32_t vi = 0, vc = 0;
        if (p < F) {
            vc = rch[p];
            vi = (vc && sch[p]) ? vc * sch[p] : 0u;
        }
        uint32_t ti, tc;
        const uint32_t ei = block_exclusive_scan(vi, tmp, &ti);
        const uint32_t ec = block_exclusive_scan(vc, tmp, &tc);
        if (p < F) {
            items_off[p] = carry[0] + ei;
            chunk_off[p] = carry[1] + ec;
        }
        __syncthreads();
        if (threadIdx.x == 0) { carry[0] += ti; carry[1] += tc; }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        items_off[F] = carry[0];
        chunk_off[F] = carry[1];
        *n_items = carry[0];
    }
}

// First page (page-list index) of every R chunk: chunk c of partition p starts
// at the first page whose preceding weight in p reaches c * chunk_w.  One warp
// per partition.
static __global__ void part_rchunks(const uint64_t *pstart, const uint32_t *Rlist, const uint8_t *Rcount, uint32_t F,
                             uint32_t chunk_w, const uint32_t *chunk_off, uint64_t *cstart) {
    const int lane = threadIdx.x & 31;
    const uint32_t p = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (p >= F) return;
    const uint64_t r0 = pstart[p], r1 = pstart[p + 1];
    uint64_t carry = 0;                 // weight before this round
    uint32_t prev_chunk = 0xFFFFFFFFu;  // chunk of the page before this round
    for (uint64_t base = r0; base < r1; base += 32) {
        const uint64_t k = base + lane;
        const uint32_t w = k < r1 ? page_weight(Rcount[Rlist[k]]) : 0u;
        uint32_t x = w;                 // inclusive warp scan
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        const uint64_t before = carry + x - w;
        const uint32_t c = (uint32_t)(before / chunk_w);
        uint32_t cprev = __shfl_up_sync(0xffffffffu, c, 1);
        if (lane == 0) cprev = prev_chunk;
        if (k < r1 && c != cprev) cstart[chunk_off[p] + c] = k;
        carry += __shfl_sync(0xffffffffu, x, 31);
        prev_chunk = __shfl_sync(0xffffffffu, c, 31);
    }
}

__device__ __forceinline__ uint32_t find_part(const uint32_t *items_off, uint32_t F, uint32_t item) {
    uint32_t lo = 0, hi = F;   // largest p with items_off[p] <= item
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (items_off[mid] <= item) lo = mid; else hi = mid;
    }
    return lo;
}

// The same search by one warp, 32 probes per round: the largest i in [0, n)
// with off[i] <= v (off non-decreasing, off[0] <= v).  Three dependent rounds
// for 2^14 entries instead of fourteen.
__device__ __forceinline__ uint32_t warp_find(const uint32_t *off, uint32_t n, uint32_t v, int lane) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint32_t step = (hi - lo + 31) / 32;
        const uint32_t idx = lo + (uint32_t)lane * step;
        const bool le = idx < hi && off[idx] <= v;
        const uint32_t m = __ballot_sync(0xffffffffu, le);
        lo += (31u - __clz(m)) * step;   // lane 0 always qualifies
        hi = min(hi, lo + step);
    }
    return lo;
}

// Warp 0 takes the next work item: slots[0] = item, slots[1] = its partition,
// slots[2] = the window of that partition (batched windows, else 0).
__device__ __forceinline__ void take_item(uint32_t *work_counter, const uint32_t *items_off, uint32_t F,
                                          uint32_t n_items, const uint32_t *wbase, uint32_t nwin,
                                          volatile uint32_t *slots, int lane) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(work_counter, 1u);
    item = __shfl_sync(0xffffffffu, item, 0);
    uint32_t p = 0, w = 0;
    if (item < n_items) {
        p = warp_find(items_off, F, item, lane);
        if (wbase) w = warp_find(wbase, nwin, p, lane);
    }
    if (lane == 0) {
        slots[0] = item;
        slots[1] = p;
        slots[2] = w;
    }
}

// Page ranges of one work item (R chunk pages [rb, rb + nrpg) and S pages
// [sb, sb + nspg) of its partition's page lists), kept in shared memory so the
// whole CTA reads them once warp 0 has taken the item.
struct ItemGeo {
    uint64_t rb, sb;
    uint32_t nrpg, nspg;
};

template <typename Args>
__device__ __forceinline__ ItemGeo item_geo(const Args &a, uint32_t item, uint32_t p, uint32_t s_pages) {
    const uint64_t *pR = a.pstart, *pS = a.pstart + (a.F + 1);
    const uint64_t r0 = pR[p], nrp = pR[p + 1] - r0;
    const uint64_t s0 = pS[p], nsp = pS[p + 1] - s0;
    const uint32_t sch = (uint32_t)((nsp + s_pages - 1) / s_pages);
    const uint32_t local = item - a.items_off[p];
    const uint32_t rc = local / sch, sc = local % sch;
    const uint32_t cid = a.chunk_off[p] + rc;
    ItemGeo g;
    g.rb = a.cstart[cid];
    const uint64_t re = rc + 1 < a.chunk_off[p + 1] - a.chunk_off[p] ? a.cstart[cid + 1] : r0 + nrp;
    g.nrpg = (uint32_t)(re - g.rb);
    g.sb = s0 + (uint64_t)sc * s_pages;
    g.nspg = (uint32_t)min((uint64_t)s_pages, nsp - (uint64_t)sc * s_pages);
    return g;
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
// Bounded wait on an mbarrier phase; false when the bound runs out.
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

// Shared memory: tup[kRSlots] u64 | aux[kRSlots] u16 | X | two page tables
// {pg[kRMaxPages + 1] u32, dst << 8 | count [kRMaxPages + 1] u32} | mbarrier,
// reduction, two item records and scan scratch.
// X holds the Chain heads (kMaxHeads u32) or the Hist permutation (kRSlots u16)
// followed by its bucket starts (kMaxHist + 2 u32).
constexpr size_t kXBytes = ((size_t)kRSlots * 2 + ((size_t)kMaxHist + 2) * 4) > (size_t)kMaxHeads * 4
                               ? ((size_t)kRSlots * 2 + ((size_t)kMaxHist + 2) * 4 + 15) & ~(size_t)15
                               : (size_t)kMaxHeads * 4;
constexpr size_t kPageTabBytes = ((size_t)kRMaxPages + 1) * 4 * 2;
constexpr size_t kJoinSmem = (size_t)kRSlots * 8 + (size_t)kRSlots * 2 + kXBytes + 2 * kPageTabBytes + 1024;
static_assert(((size_t)kRSlots * 10 + kXBytes + 2 * kPageTabBytes) % 8 == 0, "mbarrier must be 8-byte aligned");
static_assert(kJoinMinBlocks * (kJoinSmem + 1024) <= 233472, "join CTAs exceed the SM's shared memory");
static_assert(kRSlots < (1u << 24) && kRMaxPages < (uint32_t)kJoinThreads, "page table packing");

struct JoinArgs {
    const uint64_t *Rpages, *Spages;
    const uint8_t *Rcount, *Scount;
    const uint32_t *Rlist, *Slist;   // page lists grouped by digit
    const uint64_t *pstart;          // [2][F+1] page-list starts
    const uint32_t *items_off;
    const uint32_t *chunk_off;       // [F+1] first R chunk of each partition
    const uint64_t *cstart;          // first page-list index of each R chunk
    const uint32_t *n_items;
    uint32_t *work_counter;
    unsigned long long *acc;         // [0] count, [1] checksum
    int *err;
    int waits_run_out;               // ADB_TEST_WAITS_RUN_OUT: report completed waits as run out
    uint32_t F;
    uint32_t bits;                   // bits the partitioning consumed (the hash skips them)
    uint64_t *mat;                   // optional <S-key, S-payload> output
    unsigned long long *mat_n;
    uint64_t mat_cap;
    // batched windows: partition p belongs to window w with wbase[w] <= p < wbase[w + 1];
    // each item's count and checksum go to wacc[2w], wacc[2w + 1] (null: to acc)
    const uint32_t *wbase;
    const uint8_t *wbits;            // fan-out bits of each window (its in-partition hash skips them)
    uint32_t nwin;
    unsigned long long *wacc;
};

// One work item as the control warp publishes it.
struct ItemRec {
    uint64_t rb, sb;          // first page-list index of the R chunk / S chunk
    uint32_t item, p, win;    // item (>= n_items: none), partition, window
    uint32_t nrpg, nspg;      // pages of the R chunk / S chunk
    uint32_t rslots;          // R chunk slots in shared memory (pages rounded up to even counts)
};

// The items of one CTA form a pipeline run by its last warp (the control
// warp), so that no dependent global load sits between two items:
//   while item i is probed, the control warp builds the page table of item
//   i + 1 (page ids, 16-byte aligned shared-memory destinations) and takes
//   item i + 2 from the work counter; the probing warps load their S page ids
//   of item i + 1.
// Per item: one bulk async copy per R page (cp.async.bulk global -> shared,
// completion counted on an mbarrier with a bounded wait), the table build by
// all warps, then the probe by warps 0 .. kProbeWarps - 1, each holding two S
// pages in flight ahead of the one it probes.
template <TableKind K>
__global__ void __launch_bounds__(kJoinThreads, kJoinMinBlocks)
radix_join_items(JoinArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t *tup = reinterpret_cast<uint64_t *>(smem);
    uint16_t *aux = reinterpret_cast<uint16_t *>(tup + kRSlots);        // next[] (Chain) / rank (Hist)
    unsigned char *xr = reinterpret_cast<unsigned char *>(aux + kRSlots);
    uint16_t *perm = reinterpret_cast<uint16_t *>(xr);                   // Hist: bucket-ordered slots
    uint32_t *heads = K == TableKind::Chain ? reinterpret_cast<uint32_t *>(xr)      // Chain: heads
                                            : reinterpret_cast<uint32_t *>(perm + kRSlots);  // Hist: starts
    uint32_t *ptab = reinterpret_cast<uint32_t *>(xr + kXBytes);         // [2] x {pg[], dst << 8 | cnt []}
    uint64_t *bar = reinterpret_cast<uint64_t *>(ptab + 4 * (kRMaxPages + 1));
    uint64_t *red = bar + 2;
    ItemRec *rec = reinterpret_cast<ItemRec *>(red + 64);                // [2]
    uint32_t *scan = reinterpret_cast<uint32_t *>(rec + 2);              // 32 u32

    const uint32_t n_items = *a.n_items;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int kWarps = kJoinThreads / 32;
    constexpr int kCtl = kWarps - 1;
    const uint32_t F = a.F;

    // control warp: take the next item from the work counter into r
    auto take = [&](ItemRec *r) {
        uint32_t item = 0;
        if (lane == 0) item = atomicAdd(a.work_counter, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        uint32_t p = 0, w = 0;
        if (item < n_items) {
            p = warp_find(a.items_off, F, item, lane);
            if (a.wacc) w = warp_find(a.wbase, a.nwin, p, lane);
        }
        if (lane == 0) {
            r->item = item;
            if (item < n_items) {
                const ItemGeo g = item_geo(a, item, p, kSPages);
                r->p = p;
                r->win = w;
                r->rb = g.rb;
                r->sb = g.sb;
                r->nrpg = g.nrpg;
                r->nspg = g.nspg;
            }
        }
        __syncwarp();
    };
    // control warp: page table of item r (page ids, packed destination and
    // count) and the mbarrier's expected bytes for its copies.  (No bulk L2
    // prefetch of the pages: one cp.async.bulk.prefetch per 512-byte page
    // occupies the SM's bulk-copy unit for tens of cycles and delays the
    // item's own copies.)
    auto table = [&](ItemRec *r, uint32_t *pt) {
        if (r->item >= n_items) return;
        const uint64_t rb = r->rb;
        const uint32_t nrpg = r->nrpg;
        uint32_t *tpg = pt, *tpk = pt + kRMaxPages + 1;
        uint32_t carry = 0;
        constexpr int U = 4;
        for (uint32_t base = 0; base < nrpg; base += 32 * U) {
            uint32_t pg[U], cnt[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const uint32_t k = base + 32 * u + lane;
                pg[u] = k < nrpg ? a.Rlist[rb + k] : kNone;
            }
#pragma unroll
            for (int u = 0; u < U; u++) cnt[u] = pg[u] != kNone ? a.Rcount[pg[u]] : 0u;
#pragma unroll
            for (int u = 0; u < U; u++) {
                const uint32_t k = base + 32 * u + lane;
                const uint32_t e = (cnt[u] + 1) & ~1u;
                const uint32_t inc = warp_incl_scan(e, lane);
                if (k < nrpg) {
                    tpg[k] = pg[u];
                    tpk[k] = ((carry + inc - e) << 8) | cnt[u];
                }
                carry += __shfl_sync(0xffffffffu, inc, 31);
            }
        }
        if (lane == 0) {
            r->rslots = carry;
            // the item's copies are issued after the next barrier; the barrier
            // is in the item's phase already (the previous item's copies landed)
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(bar, carry * 8);
        }
        __syncwarp();
    };

    if (threadIdx.x == 0) mbar_init(bar, 1);
    if (warp == kCtl) {
        take(&rec[0]);
        table(&rec[0], ptab);
        take(&rec[1]);
    }
    __syncthreads();

    // S page ids of a probing warp for item r: lane i holds page warp + kProbeWarps * i
    auto s_ids = [&](const ItemRec &r, uint32_t &pg, uint32_t &cnt) {
        pg = 0;
        cnt = 0;
        if (warp < kProbeWarps && r.item < n_items) {
            const uint32_t i = (uint32_t)warp + (uint32_t)kProbeWarps * lane;
            if (i < r.nspg) {
                pg = a.Slist[r.sb + i];
                cnt = a.Scount[pg];
            }
        }
    };
    uint32_t my_pg, my_cnt;
    s_ids(rec[0], my_pg, my_cnt);

    uint32_t phase = 0;
    int cur = 0;
    Acc acc;
    while (true) {
        const ItemRec C = rec[cur];
        if (C.item >= n_items) break;
        const uint32_t *tpg = ptab + cur * 2 * (kRMaxPages + 1);
        const uint32_t *tpk = tpg + kRMaxPages + 1;
        const uint32_t shift = a.wacc ? a.wbits[C.win] : a.bits;
        const uint32_t nrpg = C.nrpg, nspg = C.nspg;

        // --- R chunk: one bulk copy per page from the page table (the
        //     control warp announced the bytes when it built the table)
        for (uint32_t k = threadIdx.x; k < nrpg; k += blockDim.x) {
            const uint32_t v = tpk[k], cnt = v & 0xFFu;
            if (cnt) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                bulk_g2s(tup + (v >> 8), a.Rpages + (uint64_t)tpg[k] * kPageTuples, ((cnt + 1) & ~1u) * 8, bar);
            }
        }

        // --- the probing warp's first two S pages (ids loaded during the previous item)
        const uint32_t npw = warp < kProbeWarps && (uint32_t)warp < nspg
                                 ? (nspg - warp + kProbeWarps - 1) / kProbeWarps : 0u;
        auto load_page = [&](uint32_t i, uint64_t &x0, uint64_t &x1, uint32_t &cn) {
            const uint32_t pgi = __shfl_sync(0xffffffffu, my_pg, i & 31);
            cn = __shfl_sync(0xffffffffu, my_cnt, i & 31);
            if (i >= npw) cn = 0;
            const uint64_t *Sp = a.Spages + (uint64_t)pgi * kPageTuples;
            x0 = lane < (int)cn ? ld_stream(Sp + lane) : 0;
            x1 = lane + 32 < (int)cn ? ld_stream(Sp + lane + 32) : 0;
        };
        uint64_t c0 = 0, c1 = 0, n0 = 0, n1 = 0;
        uint32_t ccnt = 0, ncnt = 0;
        if (warp < kProbeWarps) {
            load_page(0, c0, c1, ccnt);
            load_page(1, n0, n1, ncnt);
        }

        uint32_t nb = 1;
        while (nb < C.rslots) nb <<= 1;
        if (K == TableKind::Chain) {
            nb >>= 1;                                  // about two slots per head
            if (nb > kMaxHeads) nb = kMaxHeads;
        } else {
            nb >>= 2;                                  // get_hist_size: |R_i| / 4 buckets
            if (nb > kMaxHist) nb = kMaxHist;
        }
        if (nb < 1) nb = 1;
        const uint32_t bmask = nb - 1;
        for (uint32_t i = threadIdx.x; i < nb + 2; i += blockDim.x) heads[i] = 0;
        if (!mbar_wait(bar, phase) || a.waits_run_out) atomicExch(a.err, 1);
        phase ^= 1;
        __syncthreads();

        // --- build (warp per page, two tuples per lane)
        if (K == TableKind::Chain) {
            for (uint32_t k = warp; k < nrpg; k += kWarps) {
                const uint32_t v = tpk[k], c = v & 0xFFu, base = v >> 8;
                for (uint32_t l = lane; l < c; l += 32) {
                    const uint32_t s = base + l;
                    const uint32_t h = (tkey(tup[s]) >> shift) & bmask;
                    aux[s] = (uint16_t)atomicExch(&heads[h], s + 1);
                }
            }
            __syncthreads();
        } else {
            for (uint32_t k = warp; k < nrpg; k += kWarps) {
                const uint32_t v = tpk[k], c = v & 0xFFu, base = v >> 8;
                for (uint32_t l = lane; l < c; l += 32) {
                    const uint32_t s = base + l;
                    const uint32_t h = (tkey(tup[s]) >> shift) & bmask;
                    aux[s] = (uint16_t)atomicAdd(&heads[h + 1], 1u);
                }
            }
            __syncthreads();
            {   // bucket starts: heads[h + 1] = start of bucket h, heads[nb + 1] = total
                const uint32_t per = (nb + blockDim.x - 1) / blockDim.x;
                const uint32_t d0 = threadIdx.x * per, d1 = min(nb, d0 + per);
                uint32_t loc = 0;
                for (uint32_t d = d0; d < d1; d++) loc += heads[d + 1];
                uint32_t tot;
                uint32_t ex = block_exclusive_scan(loc, scan, &tot);
                for (uint32_t d = d0; d < d1; d++) {
                    const uint32_t c = heads[d + 1];
                    heads[d + 1] = ex;
                    ex += c;
                }
                __syncthreads();
                if (threadIdx.x == 0) heads[nb + 1] = tot;
            }
            __syncthreads();
            for (uint32_t k = warp; k < nrpg; k += kWarps) {
                const uint32_t v = tpk[k], c = v & 0xFFu, base = v >> 8;
                for (uint32_t l = lane; l < c; l += 32) {
                    const uint32_t s = base + l;
                    const uint32_t h = (tkey(tup[s]) >> shift) & bmask;
                    perm[heads[h + 1] + aux[s]] = (uint16_t)s;
                }
            }
            __syncthreads();
        }

        if (warp == kCtl) {
            // the next item's page table and prefetches, then the item after it
            // (rec[cur] is free: every thread copied it before the barriers above)
            table(&rec[cur ^ 1], ptab + (cur ^ 1) * 2 * (kRMaxPages + 1));
            take(&rec[cur]);
        } else {
            // the next item's S page ids, in flight during this probe
            uint32_t nx_pg, nx_cnt;
            s_ids(rec[cur ^ 1], nx_pg, nx_cnt);
            // --- probe; page i + 2 is loaded before page i is probed
            for (uint32_t i = 0; i < npw; i++) {
                uint64_t m0 = 0, m1 = 0;
                uint32_t mcnt = 0;
                if (i + 2 < npw) load_page(i + 2, m0, m1, mcnt);
#pragma unroll
                for (int half = 0; half < 2; half++) {
                    if (lane + 32 * half >= (int)ccnt) continue;
                    const uint64_t s = half ? c1 : c0;
                    const uint32_t key = tkey(s);
                    const uint32_t h = (key >> shift) & bmask;
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
                                    const unsigned long long m = atomicAdd(a.mat_n, 1ull);
                                    if (m < a.mat_cap) a.mat[m] = s;
                                }
                            }
                        }
                    } else {
                        const uint32_t e = heads[h + 2];
                        for (uint32_t t = heads[h + 1]; t < e; t++) {
                            const uint64_t r = tup[perm[t]];
                            if (tkey(r) == key) {
                                if (!have_sh) { sh = s_half(key, tpay(s)); have_sh = true; }
                                acc.count++;
                                acc.sum += pair_hash_pre(key, tpay(r), sh);
                                if (a.mat) {
                                    const unsigned long long m = atomicAdd(a.mat_n, 1ull);
                                    if (m < a.mat_cap) a.mat[m] = s;
                                }
                            }
                        }
                    }
                }
                c0 = n0; c1 = n1; ccnt = ncnt;
                n0 = m0; n1 = m1; ncnt = mcnt;
            }
            my_pg = nx_pg;
            my_cnt = nx_cnt;
        }
        if (a.wacc) {   // batched windows: this item's sums to its window
            block_flush(acc, a.wacc + 2 * C.win, red);
            acc = Acc();
        }
        __syncthreads();   // the next item rebuilds the table; rec / page tables published
        cur ^= 1;
    }
    block_flush(acc, a.acc, red);
}

}  // namespace adb
