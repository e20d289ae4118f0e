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
constexpr uint32_t kHotRun = kPTile / 2;        // a digit above this many tuples of a tile is hot
constexpr uint32_t kHotWord = 40;               // misc[] word of the hot digit

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
//   stage[kPTile] u64 | cnt[2][F] | toff[F] | lim[F] | b1[F] | b2[F] | npos[F] u32 | misc[48] u32
//   | paged input only: upage[kMaxUnitPages] u32 | ucnt[kMaxUnitPages] u8
__host__ __device__ __forceinline__ size_t pass_smem(uint32_t F, bool paged) {
    return (size_t)kPTile * 8 + (size_t)F * 4 * 7 + 48 * 4 + (paged ? (size_t)kMaxUnitPages * 5 : 0);
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// One pass over one input unit (a flat chunk, a unit of input pages, or a
// unit of a segment).  Per tile of up to kPTile tuples:
//   A  every thread ranks its tuples within their digit (shared atomics on
//      cnt[tile parity][d]);
//   B  warp 0 (up to 32 digits, one per lane) or warps 0 .. F/32 - 1 (one
//      digit per lane) turn the counts into the tile's digit runs (toff), take
//      the pages each digit's stream needs from the CTA's pool, and advance
//      the streams (npos = next free slot of the digit's current page, kNone
//      when there is none);
//   C  every thread puts its tuples into the stage, grouped by digit;
//   D  every thread copies stage slots to their pages: slot i of digit d goes
//      to i + b1[d] while i < lim[d] (the rest of the current page), else to
//      i + b2[d] (the pages taken in B, consecutive in the pool); the thread
//      that writes a page's first slot also writes the page's log entry.
// Consecutive stage slots of a digit go to consecutive addresses, so warps
// store contiguous runs; a run's partial first and last 32-byte sectors are
// completed by the neighbouring tiles of the same stream while the line is
// still in L2.  Three barriers per tile (four above 32 digits); the next
// tile's loads are in flight during D.  kMode: 0 flat input, 1 paged input
// (pass 2), 2 segmented flat input (batched windows).  kHashed: the digit is
// taken from key * kFibMul instead of the key (the table regions of NPO).
template <int kMode, int kThreads, bool kHashed = false>
__global__ void __launch_bounds__(kThreads, kPassMinBlocks)
partition_pass(PassArgs a) {
    constexpr bool kPaged = kMode == 1;
    constexpr int kPer = kPTile / kThreads;
    static_assert(kPer % 2 == 0 && kThreads % 32 == 0 && (kPTile / kPageTuples) % (kThreads / 32) == 0, "tile shape");
    static_assert((1u << kMaxPassBits) <= (uint32_t)kThreads, "one digit per thread in step B");
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
    auto dig = [&](uint64_t w) { return df(kHashed ? tkey(w) * kFibMul : tkey(w)); };
    uint64_t *stage = reinterpret_cast<uint64_t *>(smem);
    uint32_t *cnt = reinterpret_cast<uint32_t *>(stage + kPTile);   // [2][F]
    uint32_t *toff = cnt + 2 * F;
    uint32_t *lim = toff + F;
    uint32_t *b1 = lim + F;
    uint32_t *b2 = b1 + F;
    uint32_t *npos = b2 + F;
    uint32_t *misc = npos + F;          // [0] pool pages taken, [1] tuples in the tile,
                                        // [8..24) per-warp totals of the digit scan,
                                        // [kHotWord] hot digit
    uint32_t *upage = misc + 48;        // paged input: this unit's pages
    uint8_t *ucnt = reinterpret_cast<uint8_t *>(upage + kMaxUnitPages);

    const PageSet &o = relidx ? a.out[1] : a.out[0];
    const int tid = threadIdx.x, lane = tid & 31;
    const uint32_t pool_base = kMode == 2 ? in.unit_pool[g] : (uint32_t)g * a.pool_cap;
    const uint32_t pool_cap = kMode == 2 ? in.unit_pool[g + 1] - pool_base : a.pool_cap;
    const uint32_t dbase = kMode == 2 ? in.seg_dbase[p1] : p1 * F;   // output digit = dbase + d

    for (uint32_t d = tid; d < F; d += kThreads) {
        cnt[d] = 0;
        cnt[F + d] = 0;
        npos[d] = kNone;
    }
    if (tid == 0) {
        misc[0] = 0;
        misc[kHotWord] = kNone;
    }
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
    uint64_t w[kPer];
    uint32_t valid = 0;   // bit k: w[k] holds a tuple
    auto load_tile = [&](uint64_t t0) {
        valid = 0;
        if (kPaged) {
            // tuple pair k of this thread: slots 2 (tid % 32), +1 of the tile's page k * (kThreads / 32) + tid / 32
            const uint32_t slot = 2 * (tid & 31);
#pragma unroll
            for (int k = 0; k < kPer / 2; k++) {
                const uint64_t li = t0 + (uint64_t)k * (kThreads / 32) + tid / 32;
                const uint32_t c = li < e ? ucnt[li - b] : 0u;
                if (slot + 1 < c) {
                    const ulonglong2 v = __ldcs(reinterpret_cast<const ulonglong2 *>(
                        in.pages + (uint64_t)upage[li - b] * kPageTuples + slot));
                    w[2 * k] = v.x;
                    w[2 * k + 1] = v.y;
                    valid |= 3u << (2 * k);
                } else {
                    const bool ok = slot < c;
                    w[2 * k] = ok ? ld_stream(in.pages + (uint64_t)upage[li - b] * kPageTuples + slot) : 0;
                    w[2 * k + 1] = 0;
                    valid |= (ok ? 1u : 0u) << (2 * k);
                }
            }
        } else if (vec) {
#pragma unroll
            for (int k = 0; k < kPer / 2; k++) {
                const uint64_t i = t0 + 2 * ((uint64_t)k * kThreads + tid);
                if (i + 1 < e) {
                    const ulonglong2 v = __ldcs(reinterpret_cast<const ulonglong2 *>(in.in + i));
                    w[2 * k] = v.x;
                    w[2 * k + 1] = v.y;
                    valid |= 3u << (2 * k);
                } else {
                    w[2 * k] = i < e ? ld_stream(in.in + i) : 0;
                    w[2 * k + 1] = 0;
                    valid |= (i < e ? 1u : 0u) << (2 * k);
                }
            }
        } else {
#pragma unroll
            for (int k = 0; k < kPer; k++) {
                const uint64_t i = t0 + (uint64_t)k * kThreads + tid;
                w[k] = i < e ? ld_stream(in.in + i) : 0;
                valid |= (i < e ? 1u : 0u) << k;
            }
        }
    };

    // L2 prefetch of a tile: flat input one bulk prefetch of the whole tile;
    // paged input one 128-byte line prefetch per thread, four per page (a bulk
    // prefetch per 512-byte page costs the SM's bulk-copy unit more than the
    // latency it hides)
    auto prefetch_tile = [&](uint64_t t0) {
        if (t0 >= e) return;
        if (!kPaged && vec && tid == 0) {
            const uint64_t n = min(kStep, e - t0) & ~1ull;   // 16-byte multiple
            if (n) prefetch_l2(in.in + t0, (uint32_t)(n * 8));
        }
        if (kPaged && tid < (int)(kStep * 4)) {
            const uint64_t li = t0 + (uint64_t)(tid >> 2);
            if (li < e) {
                const uint64_t *line = in.pages + (uint64_t)upage[li - b] * kPageTuples + (tid & 3) * 16;
                asm volatile("prefetch.global.L2 [%0];" ::"l"(line));
            }
        }
    };

    if (b < e) {
        prefetch_tile(b + kStep);
        load_tile(b);
    }
    uint32_t par = 0;
    for (uint64_t t0 = b; t0 < e; t0 += kStep, par ^= F) {
        uint32_t *c = cnt + par;
        // A. rank each tuple within its digit.  A digit that held more than
        //    half of the previous tile (a hot key under skew) takes its ranks
        //    from one atomic per warp and tuple slot, by ballot: its increments
        //    would otherwise serialise on one shared counter.
        uint32_t rk[kPer / 2];   // two 16-bit ranks per word
        const uint32_t hot = misc[kHotWord];   // block-uniform
        if (hot == kNone) {
#pragma unroll
            for (int k = 0; k < kPer; k++) {
                const uint32_t r = (valid >> k) & 1 ? atomicAdd(&c[dig(w[k])], 1u) : 0u;
                if (k & 1) rk[k / 2] |= r << 16; else rk[k / 2] = r;
            }
        } else {
            uint32_t lt;
            asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
#pragma unroll
            for (int k = 0; k < kPer; k++) {
                const bool ok = (valid >> k) & 1;
                const uint32_t d = ok ? dig(w[k]) : kNone;
                const uint32_t m = __ballot_sync(0xffffffffu, d == hot);
                uint32_t r = 0;
                if (d == hot) r = (uint32_t)__popc(m & lt);
                else if (ok) r = atomicAdd(&c[d], 1u);
                if (m) {   // warp-uniform
                    const int leader = __ffs(m) - 1;
                    uint32_t base = 0;
                    if (lane == leader) base = atomicAdd(&c[hot], (uint32_t)__popc(m));
                    base = __shfl_sync(0xffffffffu, base, leader);
                    if (d == hot) r += base;
                }
                if (k & 1) rk[k / 2] |= r << 16; else rk[k / 2] = r;
            }
        }
        __syncthreads();
        // B. digit runs of the tile, pages, stream positions.  Up to 32 digits
        //    warp 0 alone, one per lane; above that warp w < F / 32 takes digits
        //    32w .. 32w + 31, one per lane, and the warps' totals are combined
        //    through shared memory (one extra barrier, which costs less than warp
        //    0 walking 2 or 4 digits per lane while the CTA waits: at 2^27 both
        //    passes of PRO gain, pass 2 1.232 -> 1.170 ms).  New pages get their
        //    log entry in D, from the thread that writes their first slot.
        auto run_digit = [&](uint32_t d, uint32_t L, uint32_t p, uint32_t off, uint32_t first) {
            const uint32_t room = p == kNone ? 0u : kPageTuples - (p & (kPageTuples - 1));
            c[d] = 0;
            toff[d] = off;
            lim[d] = off + (L < room ? L : room);
            b1[d] = p - off;
            uint32_t np = p + L;
            if (L > room) {
                const uint32_t need = (L - room + kPageTuples - 1) / kPageTuples;
                if (first + need > pool_cap) {   // cannot happen: the pool covers the input
                    atomicExch(a.err, 3);
                    first = pool_cap - need;
                }
                const uint32_t nx = (pool_base + first) * kPageTuples - room;
                b2[d] = nx - off;
                np = nx + L;
            }
            if (L && (np & (kPageTuples - 1)) == 0) np = kNone;   // page exactly full
            npos[d] = np;
        };
        auto pages_for = [&](uint32_t L, uint32_t p) {
            const uint32_t room = p == kNone ? 0u : kPageTuples - (p & (kPageTuples - 1));
            return L > room ? (L - room + kPageTuples - 1) / kPageTuples : 0u;
        };
        if (F <= 32) {
            constexpr int kQ = 1;   // digits per lane
            const uint32_t q = (F + 31) / 32;
            if (tid < 32) {
                uint32_t Ls[kQ], Ps[kQ], sumL = 0, sumN = 0;
#pragma unroll
                for (int j = 0; j < kQ; j++) {
                    const uint32_t d = (uint32_t)lane * q + j;
                    Ls[j] = 0;
                    Ps[j] = kNone;
                    if ((uint32_t)j < q && d < F) {
                        Ls[j] = c[d];
                        Ps[j] = npos[d];
                        sumL += Ls[j];
                        sumN += pages_for(Ls[j], Ps[j]);
                    }
                }
                const uint32_t v = sumL | (sumN << 16);   // L <= kPTile, pages < 2^16
                const uint32_t inc = warp_incl_scan(v, lane);
                const uint32_t all = __shfl_sync(0xffffffffu, inc, 31);
                const uint32_t pool0 = misc[0];
                uint32_t off = (inc - v) & 0xFFFFu, first = pool0 + ((inc - v) >> 16);
#pragma unroll
                for (int j = 0; j < kQ; j++) {
                    const uint32_t d = (uint32_t)lane * q + j;
                    if ((uint32_t)j < q && d < F) {
                        run_digit(d, Ls[j], Ps[j], off, first);
                        off += Ls[j];
                        first += pages_for(Ls[j], Ps[j]);
                    }
                }
                // the largest run (one digit per lane here): the next tile's hot digit
                const uint32_t mx = __reduce_max_sync(0xffffffffu, (Ls[0] << 16) | (uint32_t)lane);
                __syncwarp();
                if (lane == 0) {
                    misc[0] = pool0 + (all >> 16);
                    misc[1] = all & 0xFFFFu;
                    misc[kHotWord] = (mx >> 16) > kHotRun ? (mx & 0xFFFFu) : kNone;
                }
            }
        } else {
            const uint32_t nbw = (F + 31) / 32;                 // B warps
            const int bw = tid >> 5;
            const uint32_t d = (uint32_t)tid;                   // this lane's digit
            uint32_t L = 0, p = kNone, need = 0, inc = 0, pool0 = 0, mx = 0;
            if (bw < (int)nbw) {
                if (d < F) {
                    L = c[d];
                    p = npos[d];
                    need = pages_for(L, p);
                }
                inc = warp_incl_scan(L | (need << 16), lane);   // L <= kPTile, pages of 32 digits < 2^16
                mx = __reduce_max_sync(0xffffffffu, (L << 16) | d);   // this warp's largest run, its digit
                pool0 = misc[0];
                if (lane == 31) misc[8 + bw] = inc;
                if (tid == 0) misc[kHotWord] = kNone;   // all of this tile's readers are past step A
            }
            __syncthreads();   // every B warp has read misc[0] and written its total
            if (bw < (int)nbw) {
                // totals of the warps before this one, and of all of them
                uint32_t before_t = 0, before_p = 0, all_t = 0, all_p = 0;
                for (uint32_t k = 0; k < nbw; k++) {
                    const uint32_t tv = misc[8 + k];
                    if ((int)k < bw) { before_t += tv & 0xFFFFu; before_p += tv >> 16; }
                    all_t += tv & 0xFFFFu;
                    all_p += tv >> 16;
                }
                const uint32_t ex = inc - (L | (need << 16));
                if (d < F) run_digit(d, L, p, before_t + (ex & 0xFFFFu), pool0 + before_p + (ex >> 16));
                if (bw == 0 && lane == 0) {   // warp 0 read misc[0] before the shuffle above
                    misc[0] = pool0 + all_p;
                    misc[1] = all_t;
                }
                // the next tile's hot digit: a run above half a tile (at most one)
                if (lane == 0 && (mx >> 16) > kHotRun) misc[kHotWord] = mx & 0xFFFFu;
            }
        }
        __syncthreads();
        // C. stage the tile grouped by digit
#pragma unroll
        for (int k = 0; k < kPer; k++)
            if ((valid >> k) & 1)
                stage[toff[dig(w[k])] + ((rk[k / 2] >> ((k & 1) * 16)) & 0xFFFFu)] = w[k];
        const uint32_t tile_n = misc[1];
        if (t0 + kStep < e) {   // in flight during D; the tile after that into L2
            prefetch_tile(t0 + 2 * kStep);
            load_tile(t0 + kStep);
        }
        __syncthreads();
        // D. stage slots to their pages
        for (uint32_t i = tid; i < tile_n; i += kThreads) {
            const uint64_t v = stage[i];
            const uint32_t d = dig(v);
            const uint32_t dst = i + (i < lim[d] ? b1[d] : b2[d]);
            o.pages[dst] = v;
            if ((dst & (kPageTuples - 1)) == 0) {   // first slot of a page taken in B
                o.log[dst / kPageTuples] = dbase + d;
                o.pcount[dst / kPageTuples] = kPageTuples;
            }
        }
        // the next tile's A uses the other counter array and registers only;
        // its B / C run after the next barrier, when every thread is past D
    }
    __syncthreads();
    // E. fill of each digit's last page; an odd fill gets the all-ones word in
    //    its next slot, so that a 16-byte multiple copy of the page carries a
    //    pad that sorts last (every other page of a stream is full)
    for (uint32_t d = tid; d < F; d += kThreads) {
        const uint32_t p = npos[d];
        if (p != kNone && (p & (kPageTuples - 1))) {
            o.pcount[p / kPageTuples] = (uint8_t)(p & (kPageTuples - 1));
            if (p & 1) o.pages[p] = ~0ULL;
        }
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
