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
//   * each tile of 8192 tuples is counting-sorted by digit in shared memory;
//     a partition's tuples then form a stream whose whole 128-byte lines are
//     written with 16-byte stores by 8 adjacent threads; the 0-15 tuples past
//     the last whole line wait in a per-partition line buffer in shared
//     memory for the next tile (software write-combining, as in the
//     reference's _optimized partitioner), so memory sees whole-line writes;
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
constexpr int kLineTuples = 16;                 // 128-byte lines
constexpr int kPTile = 8192;                    // tuples per tile
constexpr uint32_t kMaxPassBits = 9;            // <= 512 partitions per pass (1024 threads)
constexpr uint32_t kSmallPassBits = 8;          // <= 256 partitions: 512 threads, two CTAs per SM
constexpr uint32_t kMaxUnitPages = 2048;        // pass-2 work unit: <= 128K tuples
constexpr uint32_t kMinUnitPages = 128;         // one tile
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

// Pass-2 work-unit size: about four waves of two CTAs per SM over both
// relations (units never cross a pass-1 partition, so there are a few more).
__host__ __device__ __forceinline__ uint32_t unit_pages_for(uint64_t pages1_both, int num_sms) {
    uint64_t u = pages1_both / (8ull * num_sms) + 1;
    if (u < kMinUnitPages) u = kMinUnitPages;
    if (u > kMaxUnitPages) u = kMaxUnitPages;
    return (uint32_t)u;
}

// Whole lines a tile can hold: every digit may complete one line from its
// waiting tuples plus the tile's own 8192 tuples.
__host__ __device__ __forceinline__ uint32_t max_tile_lines(uint32_t F) { return kPTile / kLineTuples + F; }

// stage[kPTile] u64 | carry[F][16] u64 | toff[F+1] | loff[F+1] | pos[F] | nxt[F] u32 |
// linedig[max lines] u16 | cc[F] u8 | misc
__host__ __device__ __forceinline__ size_t pass_smem(uint32_t F) {
    return (size_t)kPTile * 8 + (size_t)F * kLineTuples * 8 + ((size_t)F + 1) * 4 * 2 + (size_t)F * 4 * 2 +
           (size_t)max_tile_lines(F) * 2 + (size_t)F + 256;
}

__device__ __forceinline__ void st16(uint64_t *dst, uint64_t a, uint64_t b) {
    *reinterpret_cast<ulonglong2 *>(dst) = make_ulonglong2(a, b);
}

// One pass.  Per digit d of this CTA:
//   pos[d]  global tuple index of the next free line in the current page (a
//           multiple of 16), or kNone when that page is full or absent;
//   cc[d]   tuples waiting in carry[d][0..cc), stream positions 0..cc of the
//           next tile;
//   nxt[d]  per tile: tuple index of stream position 0 in the freshly taken
//           pages minus the room left in the current page.
// Stream position q of a tile (waiting tuples first, then the tile's tuples in
// sorted order) lands at pos + q while q < room = 64 - pos % 64, else nxt + q.
// kThreads threads hold kPTile / kThreads tuples each; thread d < F owns digit d.
// kMode: 0 flat input, 1 paged input (pass 2), 2 segmented flat input (batched windows).
template <int kMode, int kThreads>
__global__ void __launch_bounds__(kThreads, kThreads == 512 ? 2 : 1)
partition_pass(PassArgs a) {
    constexpr bool kPaged = kMode == 1;
    constexpr int kPer = kPTile / kThreads;
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
            df = DigitFn{0u, 0u, (1u << in.seg_bits[p1]) - 1u};
        }
    }
    const uint32_t F = df.mask + 1;
    uint64_t *stage = reinterpret_cast<uint64_t *>(smem);
    uint64_t *carry = stage + kPTile;                                    // [F][16]
    uint32_t *toff = reinterpret_cast<uint32_t *>(carry + (size_t)F * kLineTuples);
    uint32_t *loff = toff + F + 1;
    uint32_t *pos = loff + F + 1;
    uint32_t *nxt = pos + F;
    uint16_t *linedig = reinterpret_cast<uint16_t *>(nxt + F);           // digit of each whole line
    uint8_t *cc = reinterpret_cast<uint8_t *>(linedig + max_tile_lines(F));
    uint32_t *misc = reinterpret_cast<uint32_t *>((reinterpret_cast<uintptr_t>(cc + F) + 15) & ~(uintptr_t)15);
    uint32_t *pool_next = misc;        // [0]
    uint32_t *scan_tmp = misc + 4;     // [4..36)

    const PageSet &o = relidx ? a.out[1] : a.out[0];
    const int tid = threadIdx.x;
    const uint32_t pool_base = kMode == 2 ? in.unit_pool[g] : (uint32_t)g * a.pool_cap;
    const uint32_t pool_cap = kMode == 2 ? in.unit_pool[g + 1] - pool_base : a.pool_cap;
    const uint32_t dbase = kMode == 2 ? in.seg_dbase[p1] : p1 * F;   // output digit = dbase + d

    for (uint32_t d = tid; d < F; d += kThreads) {
        pos[d] = kNone;
        cc[d] = 0;
        toff[d] = 0;
    }
    if (tid == 0) *pool_next = 0;
    __syncthreads();

    // ---- tiles: flat tiles of 8192 tuples, or 128 input pages
    constexpr uint64_t kStep = kPaged ? (uint64_t)(kPTile / kPageTuples) : (uint64_t)kPTile;
    uint64_t w[kPer];
    uint32_t valid = 0;   // bit k: w[k] holds a tuple
    auto load_tile = [&](uint64_t t0) {
        valid = 0;
        if (!kPaged) {
#pragma unroll
            for (int k = 0; k < kPer; k++) {
                const uint64_t i = t0 + (uint64_t)k * kThreads + tid;
                w[k] = i < e ? ld_stream(in.in + i) : 0;
                valid |= (i < e ? 1u : 0u) << k;
            }
        } else {
            // tuple k of this thread: slot tid % 64 of the tile's page k * (kThreads / 64) + tid / 64
            const uint32_t slot = tid & (kPageTuples - 1);
            uint32_t pg[kPer];
#pragma unroll
            for (int k = 0; k < kPer; k++) {
                const uint64_t li = t0 + (uint64_t)k * (kThreads / kPageTuples) + tid / kPageTuples;
                pg[k] = li < e ? in.plist[li] : kNone;
            }
#pragma unroll
            for (int k = 0; k < kPer; k++) {
                const bool ok = pg[k] != kNone && slot < in.pcount[pg[k] == kNone ? 0 : pg[k]];
                w[k] = ok ? ld_stream(in.pages + (uint64_t)pg[k] * kPageTuples + slot) : 0;
                valid |= (ok ? 1u : 0u) << k;
            }
        }
    };
    auto room_of = [&](uint32_t p) -> uint32_t { return p == kNone ? 0u : kPageTuples - (p & (kPageTuples - 1)); };

    if (b < e) load_tile(b);
    for (uint64_t t0 = b; t0 < e; t0 += kStep) {
        // A. rank each tuple within its digit (toff[] is zero here)
        uint32_t rk[(kPer + 1) / 2];   // two 16-bit ranks per word
#pragma unroll
        for (int k = 0; k < kPer; k++) {
            const uint32_t r = (valid >> k) & 1 ? atomicAdd(&toff[df(tkey(w[k]))], 1u) : 0u;
            if (k & 1) rk[k / 2] |= r << 16; else rk[k / 2] = r;
        }
        __syncthreads();
        // B. per digit (owner = thread d): tile offset, whole lines, new pages
        uint32_t L = 0, c = 0, full = 0, my_toff = 0;
        {
            uint32_t lines = 0;
            if (tid < (int)F) {
                L = toff[tid];
                c = cc[tid];
                lines = (c + L) / kLineTuples;
                full = lines * kLineTuples;
            }
            uint32_t tot;
            const uint32_t ex = block_exclusive_scan(L | (lines << 16), scan_tmp, &tot);   // L <= 8192 < 2^16
            if (tid < (int)F) {
                const uint32_t d = tid;
                my_toff = ex & 0xFFFFu;
                toff[d] = my_toff;
                loff[d] = ex >> 16;
                for (uint32_t k = 0; k < lines; k++) linedig[(ex >> 16) + k] = (uint16_t)d;
                const uint32_t room = room_of(pos[d]);
                if (full > room) {
                    const uint32_t need = (full - room + kPageTuples - 1) / kPageTuples;
                    uint32_t nf = atomicAdd(pool_next, need);
                    if (nf + need > pool_cap) {   // cannot happen: the pool covers the input
                        atomicExch(a.err, 3);
                        nf = pool_cap - need;
                    }
                    for (uint32_t k = 0; k < need; k++) {
                        o.log[pool_base + nf + k] = dbase + d;
                        o.pcount[pool_base + nf + k] = kPageTuples;
                    }
                    nxt[d] = (pool_base + nf) * kPageTuples - room;
                }
            }
            if (tid == 0) {
                toff[F] = tot & 0xFFFFu;
                loff[F] = tot >> 16;
            }
        }
        __syncthreads();
        // C. stage the tile sorted by digit
#pragma unroll
        for (int k = 0; k < kPer; k++)
            if ((valid >> k) & 1)
                stage[toff[df(tkey(w[k]))] + ((rk[k / 2] >> ((k & 1) * 16)) & 0xFFFFu)] = w[k];
        const uint64_t tnext = t0 + kStep;
        __syncthreads();
        if (tnext < e) load_tile(tnext);   // prefetch: in flight during the writes
        // D. whole lines: 8 threads per line, 16 bytes each
        {
            const uint32_t nlines = loff[F];
            for (uint32_t li = tid / 8; li < nlines; li += kThreads / 8) {
                const uint32_t d = linedig[li];
                const uint32_t q = (li - loff[d]) * kLineTuples + (tid & 7) * 2;
                const uint32_t cd = cc[d];
                const uint32_t td = toff[d];
                const uint64_t v0 = q < cd ? carry[d * kLineTuples + q] : stage[td + q - cd];
                const uint64_t v1 = q + 1 < cd ? carry[d * kLineTuples + q + 1] : stage[td + q + 1 - cd];
                const uint32_t p = pos[d];
                const uint32_t dst = q < room_of(p) ? p + q : nxt[d] + q;
                st16(o.pages + dst, v0, v1);
            }
        }
        __syncthreads();
        // E. owner: the rest of the stream (< 16 tuples) to the line buffer,
        //    page state, and a zero counter for the next tile
        if (tid < (int)F) {
            const uint32_t d = tid;
            if (L) {
                const uint32_t total = c + L;
                // positions [max(full, c), total) come from the stage; when
                // full == 0 the waiting tuples [0, c) stay where they are
                for (uint32_t q = full > c ? full : c; q < total; q++)
                    carry[d * kLineTuples + (q - full)] = stage[my_toff + q - c];
                if (full) {
                    const uint32_t room = room_of(pos[d]);
                    uint32_t np = full <= room ? pos[d] + full : nxt[d] + full;
                    if ((np & (kPageTuples - 1)) == 0) np = kNone;   // page exactly full
                    pos[d] = np;
                }
                cc[d] = (uint8_t)(total - full);
            }
            toff[d] = 0;
        }
        __syncthreads();
    }
    // F. flush the waiting tuples; record the fill of each digit's last page
    if (tid < (int)F) {
        const uint32_t d = tid;
        const uint32_t c = cc[d];
        uint32_t p = pos[d];
        if (c) {
            if (p == kNone) {
                uint32_t nf = atomicAdd(pool_next, 1u);
                if (nf + 1 > pool_cap) { atomicExch(a.err, 3); nf = pool_cap - 1; }
                o.log[pool_base + nf] = dbase + d;
                p = (pool_base + nf) * kPageTuples;
            }
            for (uint32_t k = 0; k < c; k++) o.pages[(uint64_t)p + k] = carry[d * kLineTuples + k];
        }
        if (p != kNone && ((p & (kPageTuples - 1)) || c))
            o.pcount[p / kPageTuples] = (uint8_t)((p & (kPageTuples - 1)) + c);
    }
    __syncthreads();
    // G. pages per digit of this CTA (its log was written by this block)
    const uint32_t used = *pool_next;
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
