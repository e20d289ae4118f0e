// npo.cu -- launch sequence of the no-partitioning hash join (NPO, NPO_st).
// Reference: NPO hashing/joins/no_partitioning_join.cpp:383-476 (allocate
// the table for |R|/BUCKET_SIZE buckets, build with all threads, barrier,
// probe S chunks).
//
// The table is one global open-addressing array of 2^l2 slots (npo_join.cuh),
// as the reference's is one shared bucket array.  Up to 256 MB (|R| <= 2^24)
// the join is: clear the table, one build launch, one probe launch over the
// relations as they are.
//
// A larger table (8 B x 2 |R|: 2 GiB at |R| = 2^27) is 16x the L2, and build
// and probe in input order would each touch a random DRAM sector per tuple.
// There the table is cut into 2^rb regions of 2^21 slots (16 MB): region g
// holds the slots whose index has top bits g, i.e. the keys whose top rb bits
// of key * kFibMul are g.  One paged partition pass (paged.cuh, hashed digit)
// groups R and S by region, and build and probe walk the page lists in region
// order, each warp taking a few adjacent pages at a time and every warp of the
// grid sweeping the same stretch of the list.  At any time the grid inserts into or probes one or two regions,
// so the atomics and the sector reads hit L2; in the build each page of
// region g also prefetches its share of region g + 1's table lines into L2,
// so the next region arrives by line reads instead of random sector misses.
// At |R| = |S| = 2^27 this takes NPO from 10.9 ms (build 6.94, probe 3.89)
// to 4.26 ms (grouping 1.06, build 1.95, probe 1.19).
// Matches, count and checksum are the same as in input order.
#include "joins.cuh"
#include "npo_join.cuh"
#include "paged.cuh"

namespace adb {

// 2 slots per build tuple, at least 4 (the probe's first read is a four-slot window)
static uint32_t npo_log2(uint64_t nR) {
    uint32_t l = ceil_log2_u64(2 * (nR ? nR : 1));
    return l < 2 ? 2 : l;
}

constexpr uint32_t kNpoRegionLog2 = 21;     // slots per table region (16 MB)
// Tables up to 2^25 slots (256 MB) are not grouped.  Measured (whole join,
// |R| = |S|, grouped / not): 2^23 0.66 / 0.58 ms, 2^24 2.08 / 1.47 ms,
// 2^25 1.25 / 2.45 ms, 2^26 2.48 / 5.28 ms, 2^27 4.80 / 10.9 ms.  The grouped
// build runs at 68-69 G inserts/s from 2^25 up but at 11-23 G/s at 2^23 and
// 2^24 (tables of 1-2x the L2), whatever the region size; the cause is not
// known.
constexpr uint32_t kNpoUngroupedLog2 = 25;

// Table-region bits: 0 (no grouping) up to a 256 MB table, else regions of
// 2^21 slots.  requested > 0 forces that many bits, < 0 no grouping; at
// most 2^9 regions (one partition pass) of at least 16 slots (one L2 line).
uint32_t npo_region_bits(uint64_t nR, int requested) {
    const uint32_t l2 = npo_log2(nR);
    if (requested < 0) return 0;
    int rb = requested > 0 ? requested : (l2 > kNpoUngroupedLog2 ? (int)(l2 - kNpoRegionLog2) : 0);
    if (rb > (int)kMaxPassBits) rb = (int)kMaxPassBits;
    if (rb > (int)l2 - 4) rb = (int)l2 - 4;
    return rb < 0 ? 0u : (uint32_t)rb;
}

size_t npo_scratch(uint64_t nR, uint64_t nS, int region_bits, int num_sms) {
    const uint32_t rb = npo_region_bits(nR, region_bits);
    return Workspace::need(1ULL << npo_log2(nR), 8) + Workspace::need(1, 8) +
           (rb ? paged_partition_scratch(nR, nS, rb, 0, num_sms) : 0);
}

// One relation's pages grouped by table region (the paged pass's output).
struct NpoPages {
    const uint64_t *pages;
    const uint8_t *pcount;
    const uint32_t *plist;     // page list in region order
    const uint32_t *plog;      // region of each pool page
    const uint64_t *pstart;    // [F + 1] page-list start of each region
    uint32_t F;
};

// The share of the next region's table lines that page k of the list (pool
// page pg) prefetches: region g's pages split region g + 1's 128-byte lines
// evenly among them.  n = 0 for the last region.
__device__ __forceinline__ void npo_next_lines(const NpoPages &P, uint64_t k, uint32_t pg, const uint64_t *table,
                                               uint32_t log2n, uint32_t rb, uint64_t &l0, uint64_t &n,
                                               const char *&base) {
    l0 = 0;
    n = 0;
    base = reinterpret_cast<const char *>(table);
    const uint32_t g = P.plog[pg];
    if (g + 1 >= P.F) return;
    const uint64_t p0 = P.pstart[g], np = P.pstart[g + 1] - p0, i = k - p0;
    const uint32_t rlog = log2n - rb;                      // log2 slots per region (>= 4)
    const uint64_t lines = 1ULL << (rlog - 4);             // 128-byte lines per region
    l0 = i * lines / np;
    n = (i + 1) * lines / np - l0;
    base = reinterpret_cast<const char *>(table + ((uint64_t)(g + 1) << rlog));
}

constexpr int kNpoThreads = 256;

// Build over R's pages in region order: one warp per four adjacent pages of
// the list, two tuples of each page per lane, so that a lane has eight
// compare-and-swaps in flight; lanes 0-3 look up their page's share of the
// next region's lines and the warp issues them as L2 prefetches.  (Measured at
// |R| = 2^27: one page per warp with two CAS per lane 4.48 ms, four pages
// without the prefetch 4.29 ms, with it 1.98 ms.)
__global__ void __launch_bounds__(kNpoThreads)
npo_build_pages(NpoPages P, uint64_t *__restrict__ table, uint32_t log2n, uint32_t rb,
                unsigned long long *sentinel_cnt, int *err) {
    const uint64_t mask = (1ULL << log2n) - 1;
    const int lane = threadIdx.x & 31;
    const uint64_t npg = P.pstart[P.F];
    const uint64_t W = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t k0 = 4 * ((uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)); k0 < npg; k0 += 4 * W) {
        const uint64_t kl = k0 + (lane & 3);
        uint32_t pgl = 0, cl = 0;
        uint64_t pl0 = 0, pn = 0;
        const char *pb = reinterpret_cast<const char *>(table);
        if (kl < npg) {
            pgl = P.plist[kl];
            cl = P.pcount[pgl];
            if (lane < 4) npo_next_lines(P, kl, pgl, table, log2n, rb, pl0, pn, pb);
        }
        uint64_t w[8], slot[8];
        unsigned long long prev[8];
        bool v[8];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint32_t pg = __shfl_sync(0xffffffffu, pgl, q), c = __shfl_sync(0xffffffffu, cl, q);
            const uint64_t *src = P.pages + (uint64_t)pg * kPageTuples;
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const int u = 2 * q + j;
                v[u] = (uint32_t)(lane + 32 * j) < c;
                w[u] = v[u] ? ld_stream(src + lane + 32 * j) : kEmpty;
            }
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint64_t l0 = __shfl_sync(0xffffffffu, pl0, q), n = __shfl_sync(0xffffffffu, pn, q);
            const char *b = reinterpret_cast<const char *>(
                __shfl_sync(0xffffffffu, reinterpret_cast<uintptr_t>(pb), q));
            for (uint64_t l = lane; l < n; l += 32) asm volatile("prefetch.global.L2 [%0];" ::"l"(b + (l0 + l) * 128));
        }
#pragma unroll
        for (int u = 0; u < 8; u++)
            if (v[u] && w[u] == kEmpty) {
                atomicAdd(sentinel_cnt, 1ull);
                v[u] = false;
            }
#pragma unroll
        for (int u = 0; u < 8; u++) {
            slot[u] = npo_hash(tkey(w[u]), log2n);
            prev[u] = v[u] ? atomicCAS(reinterpret_cast<unsigned long long *>(table + slot[u]),
                                       (unsigned long long)kEmpty, (unsigned long long)w[u])
                           : (unsigned long long)kEmpty;
        }
#pragma unroll
        for (int u = 0; u < 8; u++)
            if (prev[u] != kEmpty) npo_insert_from(table, mask, (slot[u] + 1) & mask, w[u], err);
    }
}

// Probe over S's pages in region order: one warp per pair of adjacent pages,
// four probes (window loads) in flight per lane.  No prefetch here: the
// region's lines come in by the probes' own reads (at |S| = 2^27, with the
// sector-first probe: 1.75 ms without the next-region prefetch, 2.26 ms with
// it, 2.53 ms with loads two regions ahead).
template <bool kMaterialize>
__global__ void __launch_bounds__(kNpoThreads, 4)
npo_probe_pages(NpoPages P, const uint64_t *__restrict__ table, uint32_t log2n,
                const unsigned long long *sentinel_cnt, unsigned long long *acc, uint64_t *mat,
                unsigned long long *mat_n, uint64_t mat_cap) {
    __shared__ uint64_t red[64];
    const uint64_t mask = (1ULL << log2n) - 1;
    const int lane = threadIdx.x & 31;
    const uint64_t nsent = *sentinel_cnt;
    const uint64_t npg = P.pstart[P.F];
    const uint64_t W = (uint64_t)gridDim.x * (blockDim.x >> 5);
    NpoSink<kMaterialize> sink{Acc(), mat, mat_n, mat_cap};
    for (uint64_t k0 = 2 * ((uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)); k0 < npg; k0 += 2 * W) {
        uint64_t s[4], slot[4];
        ulonglong2 lo[4], hi[4];
        bool ok[4];
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const uint64_t k = k0 + q;
            uint32_t c = 0, pg = 0;
            if (k < npg) {
                pg = P.plist[k];
                c = P.pcount[pg];
            }
            const uint64_t *src = P.pages + (uint64_t)pg * kPageTuples;
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const int u = 2 * q + j;
                ok[u] = (uint32_t)(lane + 32 * j) < c;
                s[u] = ok[u] ? ld_stream(src + lane + 32 * j) : 0ULL;
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {   // the windows: all loads issued before any is used
            slot[u] = npo_hash(tkey(s[u]), log2n);
            if (ok[u]) npo_window(table, mask, slot[u], lo[u], hi[u]);
        }
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (ok[u]) npo_probe_one(sink, table, mask, s[u], slot[u], lo[u], hi[u], nsent);
    }
    block_flush(sink.a, acc, red);
}

// Phases (ms_phase): 0 grouping by region (0 without), 1 build (with the
// table's clearing), 2 -, 3 probe.
int run_npo(Context *ctx, const DevJoin &j, int region_bits, unsigned long long *acc) {
    cudaStream_t st = ctx->stream;
    const uint32_t l2 = npo_log2(j.nR);
    const uint32_t rb = npo_region_bits(j.nR, region_bits);
    PartOut po{};
    if (rb) ADB_TRY(run_paged_partition(ctx, j, DigitFn{32u - rb, (1u << rb) - 1u, true}, nullptr, &po, acc));
    ADB_CK(cudaEventRecord(ctx->ev[1], st));
    uint64_t *table = ctx->ws.take<uint64_t>(1ULL << l2);
    unsigned long long *sent = ctx->ws.take<unsigned long long>(1);
    ADB_CK(cudaMemsetAsync(table, 0xFF, (1ULL << l2) * 8, st));
    ADB_CK(cudaMemsetAsync(sent, 0, 8, st));
    int *err = reinterpret_cast<int *>(acc + 2);
    if (rb) {
        const NpoPages PR{po.R.pages, po.R.pcount, po.R.plist, po.R.log, po.pstart, po.Fout};
        const NpoPages PS{po.S.pages, po.S.pcount, po.S.plist, po.S.log, po.pstart + (po.Fout + 1), po.Fout};
        // every CTA resident at once, so that the grid's warps sweep the page
        // list together (a second wave would return to earlier regions)
        int nb = 0, np = 0;
        ADB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, npo_build_pages, kNpoThreads, 0));
        if (j.mat)
            ADB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&np, npo_probe_pages<true>, kNpoThreads, 0));
        else
            ADB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&np, npo_probe_pages<false>, kNpoThreads, 0));
        nb = nb < 1 ? 1 : nb;
        np = np < 1 ? 1 : np;
        npo_build_pages<<<ctx->num_sms * nb, kNpoThreads, 0, st>>>(PR, table, l2, rb, sent, err);
        ADB_CK(cudaEventRecord(ctx->ev[2], st));
        ADB_CK(cudaEventRecord(ctx->ev[3], st));
        if (j.mat)
            npo_probe_pages<true><<<ctx->num_sms * np, kNpoThreads, 0, st>>>(PS, table, l2, sent, acc, j.mat,
                                                                              acc + 3, j.mat_cap);
        else
            npo_probe_pages<false><<<ctx->num_sms * np, kNpoThreads, 0, st>>>(PS, table, l2, sent, acc, nullptr,
                                                                               nullptr, 0);
    } else {
        const int threads = 256;
        auto blocks = [&](uint64_t n) {
            uint64_t b = (n + threads - 1) / threads;
            const uint64_t cap = (uint64_t)ctx->num_sms * 8;
            return (int)(b < 1 ? 1 : (b > cap ? cap : b));
        };
        npo_build<<<blocks(j.nR), threads, 0, st>>>(j.R, j.nR, table, l2, sent, err);
        ADB_CK(cudaEventRecord(ctx->ev[2], st));
        ADB_CK(cudaEventRecord(ctx->ev[3], st));
        if (j.mat)
            npo_probe<true><<<blocks(j.nS), threads, 0, st>>>(j.S, j.nS, table, l2, sent, acc, j.mat, acc + 3,
                                                              j.mat_cap);
        else
            npo_probe<false><<<blocks(j.nS), threads, 0, st>>>(j.S, j.nS, table, l2, sent, acc, nullptr, nullptr, 0);
    }
    ADB_CK(cudaGetLastError());
    ctx->kernels += 2;
    return ADB_OK;
}

}  // namespace adb
