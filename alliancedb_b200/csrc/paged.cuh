// paged.cuh -- radix/range partitioning of R and S into pages, one or two passes.
//
// Replaces the reference's partitioning passes
//   parallel_radix_partition (+ _optimized, software write-combining)
//                         hashing/joins/parallel_radix_join.cpp:739-806, 877-970
//   serial_radix_partition / radix_cluster          :688-729, :573-614
//   partition_relation_optimized / radix_cluster_optimized
//                         sorting/joins/partition.cpp:152-218, 327-350
// Like the reference, large fan-outs take two passes (its NUM_PASSES = 2,
// prj_params.h:19-21); unlike it, no pass needs a histogram pass first:
//   * output goes to 512-byte pages (64 tuples) taken from a per-CTA pool, a
//     partition's pages chained through the CTA's page log, so partitions
//     need not be contiguous and their sizes need not be known in advance;
//   * each tile of 4096 tuples is counting-sorted by digit in shared memory
//     (the role of the reference's software write-combining buffers, its
//     _optimized partitioner), then copied out so that each partition's
//     tuples form one contiguous stream through its pages: warps store
//     contiguous runs, and the partial sectors at the ends of a tile's run are
//     completed in L2 by the stream's next tile, so DRAM sees whole lines;
//   * pass 2 reads the pages of pass 1 in work units of up to unit_pages pages
//     that never cross a pass-1 partition, so skewed partitions are split
//     over many CTAs;
//   * page_place turns the per-CTA page logs into one page list per partition.
// Traffic per pass: 8 bytes read + 8 bytes written per tuple, plus about 5
// bytes of page-list and count metadata per 64 tuples.
#pragma once

#include "adb_common.cuh"
#include "partition.cuh"

namespace adb {

constexpr int kPageTuples = 64;                 // 512-byte pages
constexpr int kPTile = 4096;                    // tuples per tile
constexpr int kPassThreads = 512;               // threads per CTA of a pass
constexpr int kPassMinBlocks = 2;               // CTAs per SM the registers are sized for
constexpr uint32_t kMaxPassBits = 9;            // <= 512 partitions per pass
constexpr uint32_t kSmallPassBits = 8;          // sort-merge: one pass up to 2^8 partitions
constexpr uint32_t kMaxUnitPages = 2048;        // pass-2 work unit: <= 128K tuples
constexpr uint32_t kMinUnitPages = kPTile / 64;  // one tile
constexpr uint32_t kNone = 0xFFFFFFFFu;

// Pages written by one pass for one relation.
struct PageSet {
    uint64_t *pages;     // pool pages x 64 tuples
    uint32_t *log;       // output digit of each pool page
    uint8_t *pcount;     // tuples in each pool page
    uint32_t *nlog;      // [G] pages used by each CTA
    uint32_t *plist;     // page list grouped by output digit (filled by page_place)
    uint64_t *pstart;    // [Fout + 1] page-list starts
};

// Result of the paged partitioning front end: both relations' final pages,
// page lists per output partition, pstart = [2][Fout + 1] list starts.
struct PartOut {
    PageSet R, S;
    uint32_t Fout;
    uint64_t *pstart;
    uint64_t pool_pages;
};

struct PassIn {
    // flat input (pass 1): the relation
    const uint64_t *in;
    uint64_t n;
    // paged input (pass 2): the previous pass's pages, grouped by its digit
    const uint64_t *pages;
    const uint8_t *pcount;
    const uint32_t *plist;
    const uint64_t *pstart;   // [F1 + 1]
    const uint32_t *uoff;     // [F1 + 1] first work unit of each input partition (segments: of each segment)
    // segmented flat input (batched windows): segment w is in[seg_off[w] .. seg_off[w+1]),
    // partitioned 2^seg_bits[w] ways into output partitions seg_dbase[w] + d
    const uint64_t *seg_off;
    const uint8_t *seg_bits;
    const uint32_t *seg_dbase;
    const uint32_t *unit_pool;   // segmented input: first pool page of each unit ([G + 1])
};

struct PassArgs {
    PassIn in[2];
    PageSet out[2];
    DigitFn df;          // this pass's digit (F = df.mask + 1 <= 512)
    uint32_t F1;         // input partitions (1 for flat input)
    int G;               // CTAs per relation: flat chunks, or the bound on work units
    uint32_t pool_cap;   // pages per CTA pool
    uint32_t unit_pages; // paged input: pages per work unit
    uint64_t unit_tuples;// segmented input: tuples per work unit
    int paged;           // 0 = flat input, 1 = paged input, 2 = segmented flat input
    uint32_t *seg_totals;// segmented input: [2][Dtot] pages per output partition (atomic sums)
    uint32_t Dtot;
    uint32_t *npd;       // [2][F][G] pages per (this pass's digit, CTA)
    int *err;
};

__host__ __device__ __forceinline__ uint32_t flat_pool_cap(uint64_t n, int G, uint32_t F) {
    return (uint32_t)((chunk_of(n, G) + kPageTuples - 1) / kPageTuples + F + 1);
}
__host__ __device__ __forceinline__ uint32_t unit_pool_cap(uint32_t F, uint32_t unit_pages) { return unit_pages + F + 1; }

// Pass-2 work-unit size: about four waves of the resident CTAs over both
// relations (units never cross a pass-1 partition, so there are a few more).
__host__ __device__ __forceinline__ uint32_t unit_pages_for(uint64_t pages1_both, int num_sms) {
    uint64_t u = pages1_both / (4ull * kPassMinBlocks * num_sms) + 1;
    if (u < kMinUnitPages) u = kMinUnitPages;
    if (u > kMaxUnitPages) u = kMaxUnitPages;
    return (uint32_t)u;
}

// Shared memory of one pass:
//   stage[kPTile] u64 | inbuf[kPTile] u64 | cnt[2][F] | toff[F] | lim[2][F] | b1[2][F] | b2[2][F]
//   | npos[F] u32 | misc[48] u32 | paged input only: upage[kMaxUnitPages] u32 | ucnt[kMaxUnitPages] u8
__host__ __device__ __forceinline__ size_t pass_smem(uint32_t F, bool paged) {
    return (size_t)kPTile * 8 * 2 + (size_t)F * 4 * 10 + 48 * 4 + (paged ? (size_t)kMaxUnitPages * 5 : 0);
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// Warps that compute a tile's digit runs (step B): one per 128 digits.
__host__ __device__ __forceinline__ uint32_t pass_b_warps(uint32_t F) { return F > 128 ? (F + 127) / 128 : 1u; }

// Asynchronous global -> shared copies of one thread (cp.async, completion by
// cp.async.wait_group of the same thread); src_bytes < 16 zero-fills the rest.
__device__ __forceinline__ void cp_async16(void *sdst, const void *gsrc, uint32_t src_bytes) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(gsrc), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async8(void *sdst, const void *gsrc) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// One pass over one input unit (a flat chunk, a unit of input pages, or a
// unit of a segment).  Per tile of up to kPTile tuples:
//   L  every thread copies its own slots of the tile from global memory into
//      the input buffer (cp.async, 16 bytes at a time), one tile ahead;
//   A  every thread reads its slots back and ranks its tuples within their
//      digit (shared atomics on cnt[tile parity][d]);
//   B  the B warps (one per 128 digits, up to four digits per lane) turn the
//      counts into the tile's digit runs (toff), take the pages each digit's
//      stream needs from the CTA's pool, and advance the streams (npos = next
//      free slot of the digit's current page, kNone when there is none);
//      lim / b1 / b2 of the tile's parity say where its stage slots go: slot i
//      of digit d goes to i + b1[d] while i < lim[d] (the rest of the current
//      page), else to i + b2[d] (the pages taken in B, consecutive in the pool);
//   C  every thread puts its tuples into the stage, grouped by digit;
//   D  threads copy stage slots to their pages, two adjacent slots with one
//      16-byte store when their destinations are adjacent and 16-byte aligned;
//      the thread that writes a page's first slot also writes the page's log
//      entry.
// The steps are pipelined over tiles: while the B warps compute tile t's runs,
// the other warps scatter tile t - 1 (its lim, b1, b2 and size sit in the other
// parity; the stage is free again before C of tile t), and every thread's
// copies of tile t + 1 are in flight from the start of the iteration until A
// of tile t + 1 at its end.  A tile costs two block barriers; no warp waits on
// the run computation.  Consecutive stage slots of a digit go to consecutive
// addresses, so warps store contiguous runs; a run's partial first and last
// 32-byte sectors are completed by the neighbouring tiles of the same stream
// while the line is still in L2.  kMode: 0 flat input, 1 paged input (pass 2),
// 2 segmented flat input (batched windows).
template <int kMode, int kThreads>
__global__ void __launch_bounds__(kThreads, kPassMinBlocks)
partition_pass(PassArgs a) {
    constexpr bool kPaged = kMode == 1;
    constexpr int kPer = kPTile / kThreads;
    static_assert(kPer % 2 == 0 && kThreads % 32 == 0 && (kPTile / kPageTuples) % (kThreads / 32) == 0, "tile shape");
    static_assert((1u << kMaxPassBits) <= 4u * 128u && kThreads / 32 > 4, "step B: at most four B warps, one left for D");
    extern __shared__ __align__(16) unsigned char smem[];
    const int relidx = blockIdx.y, g = blockIdx.x;
    const PassIn &in = relidx ? a.in[1] : a.in[0];

    // ---- this CTA's input: a flat chunk, a unit of input pages, or a unit of a segment
    uint64_t b = 0, e = 0;        // flat / segmented: tuple range; paged: page-list range
    uint32_t p1 = 0;              // paged: input partition; segmented: segment
    DigitFn df = a.df;
    if (kMode == 0) {
        const uint64_t chunk = chunk_of(in.n, a.G);
        b = (uint64_t)g * chunk;
        e = min(in.n, b + chunk);
    } else if ((uint32_t)g < in.uoff[a.F1]) {
        uint32_t lo = 0, hi = a.F1;   // largest p with uoff[p] <= g
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (in.uoff[mid] <= (uint32_t)g) lo = mid; else hi = mid;
        }
        p1 = lo;
        if (kMode == 1) {
            b = in.pstart[p1] + (uint64_t)(g - in.uoff[p1]) * a.unit_pages;
            e = min(in.pstart[p1 + 1], b + a.unit_pages);
        } else {
            b = in.seg_off[p1] + (uint64_t)(g - in.uoff[p1]) * a.unit_tuples;
            e = min(in.seg_off[p1 + 1], b + a.unit_tuples);
            df = DigitFn{0u, (1u << in.seg_bits[p1]) - 1u};
        }
    }
    const uint32_t F = df.mask + 1;
    uint64_t *stage = reinterpret_cast<uint64_t *>(smem);              // [kPTile]
    uint64_t *inbuf = stage + kPTile;                                   // [kPTile]
    uint32_t *cnt = reinterpret_cast<uint32_t *>(inbuf + kPTile);       // [2][F]
    uint32_t *toff = cnt + 2 * F;
    uint32_t *lim = toff + F;           // [2][F]
    uint32_t *b1 = lim + 2 * F;         // [2][F]
    uint32_t *b2 = b1 + 2 * F;          // [2][F]
    uint32_t *npos = b2 + 2 * F;
    uint32_t *misc = npos + F;          // [0] pool pages taken, [2 + parity] stage slots of the tile,
                                        // [8..12) per-B-warp totals of the digit scan
    uint32_t *upage = misc + 48;        // paged input: this unit's pages
    uint8_t *ucnt = reinterpret_cast<uint8_t *>(upage + kMaxUnitPages);

    const PageSet &o = relidx ? a.out[1] : a.out[0];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t pool_base = kMode == 2 ? in.unit_pool[g] : (uint32_t)g * a.pool_cap;
    const uint32_t pool_cap = kMode == 2 ? in.unit_pool[g + 1] - pool_base : a.pool_cap;
    const uint32_t dbase = kMode == 2 ? in.seg_dbase[p1] : p1 * F;   // output digit = dbase + d
    const uint32_t nbw = pass_b_warps(F);                             // B warps
    const uint32_t q = (F + 32 * nbw - 1) / (32 * nbw);               // digits per B lane (<= 4)

    for (uint32_t d = tid; d < F; d += kThreads) {
        cnt[d] = 0;
        cnt[F + d] = 0;
        npos[d] = kNone;
    }
    if (tid == 0) misc[0] = 0;
    if (kPaged)
        for (uint64_t i = b + tid; i < e; i += kThreads) {
            const uint32_t pg = in.plist[i];
            upage[i - b] = pg;
            ucnt[i - b] = in.pcount[pg];
        }
    __syncthreads();

    // ---- tiles: kPTile flat tuples, or kPTile / 64 input pages
    constexpr uint64_t kStep = kPaged ? (uint64_t)(kPTile / kPageTuples) : (uint64_t)kPTile;
    const bool vec = !kPaged && ((reinterpret_cast<uintptr_t>(in.in + b) & 15) == 0);
    // Slots of this thread: pair k = input-buffer slots s(k), s(k) + 1 with
    //   flat input:  s = 2 (k kThreads + tid), tuples t0 + s, t0 + s + 1;
    //   paged input: s = 64 pg + 2 (tid % 32), pg = k (kThreads / 32) + tid / 32,
    //                the tile's pg-th page, its slots 2 (tid % 32), + 1.
    auto pair_slot = [&](int k) -> uint32_t {
        return kPaged ? ((uint32_t)k * (kThreads / 32) + (uint32_t)(tid / 32)) * kPageTuples + 2u * (uint32_t)lane
                      : 2u * ((uint32_t)k * kThreads + (uint32_t)tid);
    };
    auto pair_count = [&](uint64_t t0, int k) -> uint32_t {   // tuples of pair k present (0, 1, 2)
        if (kPaged) {
            const uint64_t li = t0 + (uint64_t)k * (kThreads / 32) + tid / 32;
            const uint32_t c = li < e ? ucnt[li - b] : 0u, s2 = 2u * (uint32_t)lane;
            return c > s2 + 1 ? 2u : (c > s2 ? 1u : 0u);
        }
        const uint64_t i = t0 + pair_slot(k);
        return i + 1 < e ? 2u : (i < e ? 1u : 0u);
    };
    // L. this thread's copies of the tile at t0 into its input-buffer slots
    auto copy_tile = [&](uint64_t t0) {
#pragma unroll
        for (int k = 0; k < kPer / 2; k++) {
            const uint32_t n = pair_count(t0, k), s = pair_slot(k);
            if (!n) continue;
            const uint64_t *src = kPaged ? in.pages + (uint64_t)upage[t0 + (uint64_t)k * (kThreads / 32) + tid / 32 - b] *
                                                          kPageTuples + 2u * (uint32_t)lane
                                         : in.in + t0 + s;
            if (kPaged || vec) {
                cp_async16(inbuf + s, src, n * 8);
            } else {   // relation not 16-byte aligned: 8-byte copies
                cp_async8(inbuf + s, src);
                if (n == 2) cp_async8(inbuf + s + 1, src + 1);
            }
        }
        cp_async_commit();
    };

    // L2 prefetch of a whole flat tile (one bulk prefetch; paged input is not
    // prefetched: one bulk prefetch per 512-byte page costs the SM's bulk-copy
    // unit more than the latency it hides)
    auto prefetch_tile = [&](uint64_t t0) {
        if (t0 >= e) return;
        if (!kPaged && vec && tid == 0) {
            const uint64_t n = min(kStep, e - t0) & ~1ull;   // 16-byte multiple
            if (n) prefetch_l2(in.in + t0, (uint32_t)(n * 8));
        }
    };

    // A. read this thread's slots of the tile at t0 (after its copies landed)
    //    and rank each tuple within its digit (counters of parity par)
    uint64_t w[kPer];
    uint32_t valid = 0;      // bit k: w[k] holds a tuple
    uint32_t rk[kPer / 2];   // two 16-bit ranks per word
    auto rank_tile = [&](uint64_t t0, uint32_t par) {
        cp_async_wait_all();
        valid = 0;
#pragma unroll
        for (int k = 0; k < kPer / 2; k++) {
            const uint32_t n = pair_count(t0, k);
            const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(inbuf + pair_slot(k));
            w[2 * k] = v.x;
            w[2 * k + 1] = v.y;
            valid |= ((n >= 1 ? 1u : 0u) | (n == 2 ? 2u : 0u)) << (2 * k);
        }
        uint32_t *c = cnt + par * F;
#pragma unroll
        for (int k = 0; k < kPer; k++) {
            const uint32_t r = (valid >> k) & 1 ? atomicAdd(&c[df(tkey(w[k]))], 1u) : 0u;
            if (k & 1) rk[k / 2] |= r << 16; else rk[k / 2] = r;
        }
    };

    // B. digit runs of the tile of parity par, its pages and stream positions
    //    (B warps only; lane l of B warp bw owns digits (bw * 32 + l) * q ..
    //    + q - 1; the B warps' totals are combined through misc and a named
    //    barrier).  New pages get their log entry in D, from the thread that
    //    writes their first slot.
    auto run_tile = [&](uint32_t par) {
        uint32_t *c = cnt + par * F;
        uint32_t *lm = lim + par * F, *p1b = b1 + par * F, *p2b = b2 + par * F;
        auto pages_for = [&](uint32_t L, uint32_t p) {
            const uint32_t room = p == kNone ? 0u : kPageTuples - (p & (kPageTuples - 1));
            return L > room ? (L - room + kPageTuples - 1) / kPageTuples : 0u;
        };
        constexpr int kQ = 4;
        uint32_t Ls[kQ], Ps[kQ], sumL = 0, sumN = 0;
#pragma unroll
        for (int j = 0; j < kQ; j++) {
            const uint32_t d = ((uint32_t)warp * 32 + lane) * q + j;
            Ls[j] = 0;
            Ps[j] = kNone;
            if ((uint32_t)j < q && d < F) {
                Ls[j] = c[d];
                Ps[j] = npos[d];
                sumL += Ls[j];
                sumN += pages_for(Ls[j], Ps[j]);
            }
        }
        const uint32_t v = sumL | (sumN << 16);   // L <= kPTile per tile, pages < 2^16
        const uint32_t inc = warp_incl_scan(v, lane);
        const uint32_t pool0 = misc[0];
        uint32_t before = 0, all = __shfl_sync(0xffffffffu, inc, 31);
        if (nbw > 1) {
            if (lane == 31) misc[8 + warp] = inc;
            asm volatile("bar.sync 1, %0;" ::"r"(nbw * 32) : "memory");   // B warps only
            all = 0;
            for (uint32_t k = 0; k < nbw; k++) {
                const uint32_t tv = misc[8 + k];
                if (k < (uint32_t)warp) before += tv;
                all += tv;
            }
        }
        uint32_t off = (before + inc - v) & 0xFFFFu, first = pool0 + ((before + inc - v) >> 16);
#pragma unroll
        for (int j = 0; j < kQ; j++) {
            const uint32_t d = ((uint32_t)warp * 32 + lane) * q + j;
            if ((uint32_t)j < q && d < F) {
                const uint32_t L = Ls[j], p = Ps[j];
                const uint32_t room = p == kNone ? 0u : kPageTuples - (p & (kPageTuples - 1));
                c[d] = 0;
                toff[d] = off;
                lm[d] = off + (L < room ? L : room);
                p1b[d] = p - off;
                uint32_t np = p + L;
                if (L > room) {
                    const uint32_t need = (L - room + kPageTuples - 1) / kPageTuples;
                    uint32_t f = first;
                    if (f + need > pool_cap) {   // cannot happen: the pool covers the input
                        atomicExch(a.err, 3);
                        f = pool_cap - need;
                    }
                    const uint32_t nx = (pool_base + f) * kPageTuples - room;
                    p2b[d] = nx - off;
                    np = nx + L;
                    first += need;
                }
                if (L && (np & (kPageTuples - 1)) == 0) np = kNone;   // page exactly full
                npos[d] = np;
                off += L;
            }
        }
        if (nbw > 1) asm volatile("bar.sync 1, %0;" ::"r"(nbw * 32) : "memory");   // every B warp read misc
        if (warp == 0 && lane == 0) {
            misc[0] = pool0 + (all >> 16);
            misc[2 + par] = all & 0xFFFFu;
        }
    };

    // C. stage the register tuples grouped by digit
    auto stage_tile = [&]() {
#pragma unroll
        for (int k = 0; k < kPer; k++)
            if ((valid >> k) & 1)
                stage[toff[df(tkey(w[k]))] + ((rk[k / 2] >> ((k & 1) * 16)) & 0xFFFFu)] = w[k];
    };

    // D. stage slots to their pages (lim, b1, b2, size of parity par), by
    //    threads t .. t + nt - 1
    auto scatter_tile = [&](uint32_t par, uint32_t t, uint32_t nt) {
        const uint32_t *lm = lim + par * F, *p1b = b1 + par * F, *p2b = b2 + par * F;
        const uint32_t n = misc[2 + par];
        auto dest = [&](uint32_t i, uint64_t v, uint32_t &d) {
            d = df(tkey(v));
            return i + (i < lm[d] ? p1b[d] : p2b[d]);
        };
        auto page_head = [&](uint32_t dst, uint32_t d) {
            if ((dst & (kPageTuples - 1)) == 0) {   // first slot of a page taken in B
                o.log[dst / kPageTuples] = dbase + d;
                o.pcount[dst / kPageTuples] = kPageTuples;
            }
        };
        for (uint32_t i = 2 * t; i < n; i += 2 * nt) {
            // slot i + 1 may be stale when i + 1 == n (n < kPTile then): not used
            const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(stage + i);
            uint32_t d0, d1 = 0;
            const uint32_t x0 = dest(i, v.x, d0);
            if (i + 1 < n) {
                const uint32_t x1 = dest(i + 1, v.y, d1);
                if (x1 == x0 + 1 && (x0 & 1) == 0) {
                    *reinterpret_cast<ulonglong2 *>(o.pages + x0) = v;
                } else {
                    o.pages[x0] = v.x;
                    o.pages[x1] = v.y;
                }
                page_head(x1, d1);
            } else {
                o.pages[x0] = v.x;
            }
            page_head(x0, d0);
        }
    };

    if (b < e) {
        copy_tile(b);
        prefetch_tile(b + kStep);
        rank_tile(b, 0);
    }
    __syncthreads();
    uint32_t par = 0;
    for (uint64_t t0 = b; t0 < e; t0 += kStep, par ^= 1) {
        const bool more = t0 + kStep < e;
        if (more) {   // the next tile's copies: in flight until its ranks at the end of this iteration
            copy_tile(t0 + kStep);
            prefetch_tile(t0 + 2 * kStep);
        }
        if ((uint32_t)warp < nbw) run_tile(par);
        else if (t0 != b) scatter_tile(par ^ 1, tid - nbw * 32, kThreads - nbw * 32);
        __syncthreads();   // runs of this tile known; the previous tile scattered
        stage_tile();
        if (more) rank_tile(t0 + kStep, par ^ 1);
        __syncthreads();   // this tile staged; the next tile ranked
    }
    if (b < e) scatter_tile(par ^ 1, tid, kThreads);   // the last tile
    __syncthreads();
    // E. fill of each digit's last page
    for (uint32_t d = tid; d < F; d += kThreads) {
        const uint32_t p = npos[d];
        if (p != kNone && (p & (kPageTuples - 1))) o.pcount[p / kPageTuples] = (uint8_t)(p & (kPageTuples - 1));
    }
    // F. pages per digit of this CTA (its log was written by this block)
    const uint32_t used = misc[0];
    for (uint32_t d = tid; d < F; d += kThreads) toff[d] = 0;
    __syncthreads();
    for (uint32_t k = tid; k < used; k += kThreads) atomicAdd(&toff[o.log[pool_base + k] - dbase], 1u);
    __syncthreads();
    if (kMode == 2) {
        uint32_t *tot = a.seg_totals + (size_t)relidx * a.Dtot;
        for (uint32_t d = tid; d < F; d += kThreads)
            if (toff[d]) atomicAdd(&tot[dbase + d], toff[d]);
    } else {
        uint32_t *npd = a.npd + (size_t)relidx * F * a.G;
        for (uint32_t d = tid; d < F; d += kThreads) npd[(size_t)d * a.G + g] = toff[d];
    }
    if (tid == 0) o.nlog[g] = used;
}

// Work units of a paged pass: uoff[p] = first unit of input partition p.
static __global__ void make_units(const uint64_t *pstart0, const uint64_t *pstart1, uint32_t F1, uint32_t unit_pages,
                           uint32_t *uoff0, uint32_t *uoff1) {
    __shared__ uint32_t tmp[32];
    __shared__ uint32_t carry;
    const uint64_t *ps = blockIdx.x ? pstart1 : pstart0;
    uint32_t *uo = blockIdx.x ? uoff1 : uoff0;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < F1; base += blockDim.x) {
        const uint32_t p = base + threadIdx.x;
        const uint32_t v = p < F1 ? (uint32_t)((ps[p + 1] - ps[p] + unit_pages - 1) / unit_pages) : 0u;
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan(v, tmp, &tot);
        if (p < F1) uo[p] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) uo[F1] = carry;
}

// Output-partition totals of a pass: pages of output digit D = p1 * F + d.
// rowoff[rel][d][u] is the exclusive scan of npd over the units u; the units
// of input partition p1 are [uoff[p1], uoff[p1 + 1]).
static __global__ void pass_totals(const uint32_t *rowoff, const uint32_t *rowtot, const uint32_t *uoff0,
                            const uint32_t *uoff1, uint32_t F, uint32_t F1, int G, uint32_t *totals) {
    const uint32_t rel = blockIdx.y;
    const uint32_t *uoff = rel ? uoff1 : uoff0;
    const uint32_t Fout = F * F1;
    for (uint32_t D = blockIdx.x * blockDim.x + threadIdx.x; D < Fout; D += gridDim.x * blockDim.x) {
        const uint32_t p1 = D / F, d = D % F;
        const uint32_t *row = rowoff + ((size_t)rel * F + d) * G;
        const uint32_t u0 = uoff ? uoff[p1] : 0u, u1 = uoff ? uoff[p1 + 1] : (uint32_t)G;   // flat: one unit row
        const uint32_t end = u1 < (uint32_t)G ? row[u1] : rowtot[(size_t)rel * F + d];
        const uint32_t beg = u0 < (uint32_t)G ? row[u0] : rowtot[(size_t)rel * F + d];
        totals[(size_t)rel * Fout + D] = end - beg;
    }
}

// Groups the CTAs' page logs into one page list per output digit:
// plist[pstart[D] + (rowoff[d][g] - rowoff[d][first unit of p1]) + i] = the
// i-th page of digit D written by CTA g.
static __global__ void __launch_bounds__(1024)
page_place(PassArgs a, const uint32_t *rowoff, const uint32_t *uoff0, const uint32_t *uoff1) {
    extern __shared__ uint32_t cnt[];
    const uint32_t F = a.df.mask + 1;
    const int relidx = blockIdx.y, g = blockIdx.x;
    const PageSet &o = relidx ? a.out[1] : a.out[0];
    const uint32_t *ro = rowoff + (size_t)relidx * F * a.G;
    for (uint32_t d = threadIdx.x; d < F; d += blockDim.x) cnt[d] = 0;
    __syncthreads();
    const uint32_t used = o.nlog[g];
    if (!used) return;
    const uint32_t pool_base = (uint32_t)g * a.pool_cap;
    const uint32_t D0 = o.log[pool_base];
    const uint32_t p1 = D0 / F;
    const uint32_t u0 = a.paged ? (relidx ? uoff1 : uoff0)[p1] : 0u;
    for (uint32_t k = threadIdx.x; k < used; k += blockDim.x) {
        const uint32_t D = o.log[pool_base + k];
        const uint32_t d = D % F;
        const uint32_t i = atomicAdd(&cnt[d], 1u);
        o.plist[o.pstart[D] + (ro[(size_t)d * a.G + g] - ro[(size_t)d * a.G + u0]) + i] = pool_base + k;
    }
}

}  // namespace adb
