// batch.cu -- batched windows: many independent R/S window pairs joined by one
// launch sequence (adb_batch_join_device), with the fan-out of each window
// picked per window-size bucket by a measured table (adb_batch_autotune).
//
// The reference joins one window per call (benchmark.cpp:244-247 calls the join
// once per relation pair); a batch of W windows there is W sequential calls,
// each spawning and joining its threads.  On the device, mode 1 reproduces that
// (one launch sequence per window); mode 0 joins all windows together:
//   1. partition_pass in segmented mode: work units of up to kBatchUnit tuples
//      inside one window, window w partitioned 2^bits[w] ways into output
//      partitions wbase[w] .. wbase[w + 1];
//   2. device-wide scans and atomic page placement build one page list per
//      output partition of every window;
//   3. the persistent work-stealing join kernel of the partitioned hash join
//      takes (partition, R chunk, S chunk) items of all windows, so small and
//      large windows share the SMs, and adds each item into its window's count
//      and checksum.
#include <algorithm>
#include <vector>

#include "datagen.cuh"
#include "joins.cuh"
#include "paged.cuh"
#include "radix_join.cuh"

namespace adb {

constexpr uint64_t kBatchUnit = 131072;       // tuples per work unit (2^17)
constexpr uint32_t kScanBlock = 8192;         // elements per block of the device-wide scan

// ---- device-wide exclusive scan (reduce, scan of block sums, apply) --------
template <class T>
__global__ void dscan_reduce(const uint32_t *in, uint32_t n, T *bsum) {
    __shared__ uint32_t tmp[32];
    const uint64_t b = (uint64_t)blockIdx.x * kScanBlock;
    T loc = 0;
    for (uint32_t i = threadIdx.x; i < kScanBlock; i += blockDim.x)
        if (b + i < n) loc += in[b + i];
    // warp + block sum (T = u32 or u64)
    for (int o = 16; o > 0; o >>= 1) loc += __shfl_xor_sync(0xffffffffu, loc, o);
    __shared__ T part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = loc;
    __syncthreads();
    if (threadIdx.x == 0) {
        T s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += part[w];
        bsum[blockIdx.x] = s;
    }
    (void)tmp;
}

template <class T>
__global__ void dscan_bsums(T *bsum, uint32_t nb, T *total) {
    // one thread: the number of blocks is small (n / 8192)
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        T s = 0;
        for (uint32_t b = 0; b < nb; b++) {
            const T v = bsum[b];
            bsum[b] = s;
            s += v;
        }
        *total = s;
    }
}

template <class T>
__global__ void dscan_apply(const uint32_t *in, uint32_t n, const T *bsum, T *out) {
    __shared__ uint32_t tmp[32];
    __shared__ T carry;
    const uint64_t b = (uint64_t)blockIdx.x * kScanBlock;
    if (threadIdx.x == 0) carry = bsum[blockIdx.x];
    __syncthreads();
    for (uint32_t base = 0; base < kScanBlock; base += blockDim.x) {
        const uint64_t i = b + base + threadIdx.x;
        const uint32_t v = i < n ? in[i] : 0u;
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan(v, tmp, &tot);
        if (i < n) out[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
}

// out[0..n) = exclusive scan of in, out[n] = total.  bsum needs ceil(n / 8192) + 1 slots.
template <class T>
static void dscan(cudaStream_t st, const uint32_t *in, uint32_t n, T *out, T *bsum) {
    const uint32_t nb = (n + kScanBlock - 1) / kScanBlock;
    if (nb == 0) {
        cudaMemsetAsync(out, 0, sizeof(T), st);
        return;
    }
    dscan_reduce<T><<<nb, 1024, 0, st>>>(in, n, bsum);
    dscan_bsums<T><<<1, 32, 0, st>>>(bsum, nb, out + n);
    dscan_apply<T><<<nb, 1024, 0, st>>>(in, n, bsum, out);
}

// items per partition (R chunks x S chunks) next to the R chunk counts
__global__ void items_per_part(const uint32_t *rch, const uint32_t *sch, uint32_t n, uint32_t *items) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        items[p] = (rch[p] && sch[p]) ? rch[p] * sch[p] : 0u;
}

__global__ void copy_last_u32(const uint32_t *src, uint32_t *dst) { *dst = *src; }

// Places each unit's pages into its partitions' page lists (positions by atomics).
__global__ void page_place_atomic(PassArgs a, uint32_t *fill0, uint32_t *fill1) {
    const int relidx = blockIdx.y, g = blockIdx.x;
    const PageSet &o = relidx ? a.out[1] : a.out[0];
    uint32_t *fill = relidx ? fill1 : fill0;
    const uint32_t used = o.nlog[g];
    const uint32_t pool_base = (relidx ? a.in[1] : a.in[0]).unit_pool[g];
    for (uint32_t k = threadIdx.x; k < used; k += blockDim.x) {
        const uint32_t D = o.log[pool_base + k];
        o.plist[o.pstart[D] + atomicAdd(&fill[D], 1u)] = pool_base + k;
    }
}

// ---- fan-out per window-size bucket -----------------------------------------
// bucket = ceil(log2(max(|R_w|, |S_w|))); default: R partitions of about 8K tuples
static int default_bits(uint32_t bucket) {
    const int b = (int)bucket - 13;
    return b < 0 ? 0 : (b > (int)kMaxPassBits ? (int)kMaxPassBits : b);
}

static int8_t g_tune[33] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1,
                            -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1};

static int bits_for_window(uint64_t nr, uint64_t ns) {
    const uint32_t bucket = ceil_log2_u64(std::max<uint64_t>(std::max(nr, ns), 1));
    const int t = bucket < 33 ? g_tune[bucket] : -1;
    return t >= 0 ? t : default_bits(bucket);
}

// ---- mode 0: all windows in one launch sequence -----------------------------
// Enqueues the whole batch on ctx->stream; the per-window sums (count, checksum
// pairs) and the device-side error word land in the pinned host buffer h_out
// (2 W + 8 words) once the stream reaches that point.
int batch_launch(Context *ctx, const uint64_t *dR, const uint64_t *r_off, const uint64_t *dS, const uint64_t *s_off,
                 uint32_t W, unsigned long long *h_out) {
    cudaStream_t st = ctx->stream;
    // host plan: per-window fan-out, partition bases, work units
    std::vector<uint8_t> bits(W);
    std::vector<uint32_t> wbase(W + 1), uoffR(W + 1), uoffS(W + 1);
    std::vector<uint64_t> segR(W + 1), segS(W + 1);
    uint64_t D = 0, uR = 0, uS = 0;
    for (uint32_t w = 0; w < W; w++) {
        const uint64_t nr = r_off[w + 1] - r_off[w], ns = s_off[w + 1] - s_off[w];
        bits[w] = (uint8_t)bits_for_window(nr, ns);
        wbase[w] = (uint32_t)D;
        uoffR[w] = (uint32_t)uR;
        uoffS[w] = (uint32_t)uS;
        segR[w] = r_off[w] - r_off[0];
        segS[w] = s_off[w] - s_off[0];
        D += 1ull << bits[w];
        uR += (nr + kBatchUnit - 1) / kBatchUnit;
        uS += (ns + kBatchUnit - 1) / kBatchUnit;
    }
    wbase[W] = (uint32_t)D;
    uoffR[W] = (uint32_t)uR;
    uoffS[W] = (uint32_t)uS;
    segR[W] = r_off[W] - r_off[0];
    segS[W] = s_off[W] - s_off[0];
    const uint64_t nR = segR[W], nS = segS[W];
    if (D >= (1ull << 31) || uR + uS >= (1ull << 31)) {
        set_error("batch too large: %llu partitions", (unsigned long long)D);
        return ADB_ERR_ARG;
    }
    const uint32_t Dt = (uint32_t)D;
    const int G = (int)std::max<uint64_t>(std::max(uR, uS), 1);
    // each unit's page pool: its tuples in pages plus one partial page per partition
    std::vector<uint32_t> upool[2] = {std::vector<uint32_t>(G + 1), std::vector<uint32_t>(G + 1)};
    uint64_t pages_rel[2] = {0, 0};
    for (int r = 0; r < 2; r++) {
        const uint64_t *off = r ? s_off : r_off;
        uint64_t tot = 0;
        uint32_t g = 0;
        for (uint32_t w = 0; w < W; w++) {
            const uint64_t n = off[w + 1] - off[w];
            for (uint64_t u = 0; u * kBatchUnit < n; u++) {
                upool[r][g++] = (uint32_t)tot;
                const uint64_t nu = std::min(kBatchUnit, n - u * kBatchUnit);
                tot += (nu + kPageTuples - 1) / kPageTuples + (1ull << bits[w]) + 1;
                if (tot >= (1ull << 32)) break;
            }
        }
        for (; g <= (uint32_t)G; g++) upool[r][g] = (uint32_t)std::min<uint64_t>(tot, 0xFFFFFFFFull);
        pages_rel[r] = tot;
    }
    const uint64_t pages = std::max(pages_rel[0], pages_rel[1]);
    const uint32_t pool_cap = 0;   // per unit (unit_pool)
    if (pages * kPageTuples >= (uint64_t)kNone) {
        set_error("batch too large for 32-bit page indices (%llu tuples)", (unsigned long long)(nR + nS));
        return ADB_ERR_ARG;
    }
    const uint32_t nbs = Dt / kScanBlock + 2;
    const size_t meta = Workspace::need(W, 1) + 3 * Workspace::need(W + 1, 4) + 2 * Workspace::need(W + 1, 8) +
                        2 * Workspace::need(G + 1, 4);
    const size_t bytes = meta + 2 * (Workspace::need(pages * kPageTuples, 8) + 2 * Workspace::need(pages, 4) +
                                     Workspace::need(pages, 1) + Workspace::need(G, 4)) +
                         4 * Workspace::need(2ull * Dt + 2, 4) + 2 * Workspace::need(2ull * (Dt + 1), 8) +
                         2 * Workspace::need(nbs, 8) + 4 * Workspace::need(Dt + 1, 4) +
                         Workspace::need(pages * kPageTuples / kChunkW + Dt + 1, 8) + Workspace::need(2 * W + 8, 8);
    ADB_TRY(ctx->ws.reserve(bytes + 8192));

    // the plan (window bits, partition bases, unit offsets, segments, unit pools):
    // laid out in the pinned staging buffer exactly as in the workspace, one copy
    const size_t plan_off = ctx->ws.off;
    uint8_t *d_bits = ctx->ws.take<uint8_t>(W);
    uint32_t *d_wbase = ctx->ws.take<uint32_t>(W + 1);
    uint32_t *d_uoff[2] = {ctx->ws.take<uint32_t>(W + 1), ctx->ws.take<uint32_t>(W + 1)};
    uint64_t *d_seg[2] = {ctx->ws.take<uint64_t>(W + 1), ctx->ws.take<uint64_t>(W + 1)};
    uint32_t *d_upool[2] = {ctx->ws.take<uint32_t>(G + 1), ctx->ws.take<uint32_t>(G + 1)};
    const size_t plan_bytes = ctx->ws.off - plan_off;
    ADB_TRY(pinned_reserve(&ctx->h_stage, &ctx->h_stage_cap, plan_bytes));   // the last plan's copy is done
    char *h = ctx->h_stage;
    auto put = [&](const void *dev_at, const void *src, size_t n) {
        memcpy(h + (reinterpret_cast<const char *>(dev_at) - (ctx->ws.base + plan_off)), src, n);
    };
    put(d_bits, bits.data(), W);
    put(d_wbase, wbase.data(), (W + 1) * 4);
    put(d_uoff[0], uoffR.data(), (W + 1) * 4);
    put(d_uoff[1], uoffS.data(), (W + 1) * 4);
    put(d_seg[0], segR.data(), (W + 1) * 8);
    put(d_seg[1], segS.data(), (W + 1) * 8);
    put(d_upool[0], upool[0].data(), (G + 1) * 4);
    put(d_upool[1], upool[1].data(), (G + 1) * 4);
    ADB_CK(cudaMemcpyAsync(ctx->ws.base + plan_off, h, plan_bytes, cudaMemcpyHostToDevice, st));

    PassArgs a{};
    for (int r = 0; r < 2; r++) {
        PassIn &in = a.in[r];
        in.in = r ? dS : dR;
        in.n = r ? nS : nR;
        in.uoff = d_uoff[r];
        in.seg_off = d_seg[r];
        in.seg_bits = d_bits;
        in.seg_dbase = d_wbase;
        in.unit_pool = d_upool[r];
        PageSet &o = a.out[r];
        o.pages = ctx->ws.take<uint64_t>(pages * kPageTuples);
        o.log = ctx->ws.take<uint32_t>(pages);
        o.pcount = ctx->ws.take<uint8_t>(pages);
        o.nlog = ctx->ws.take<uint32_t>(G);
        o.plist = ctx->ws.take<uint32_t>(pages);
    }
    a.df = DigitFn{0u, 0u};
    a.F1 = W;
    a.G = G;
    a.pool_cap = pool_cap;
    a.unit_tuples = kBatchUnit;
    a.paged = 2;
    a.Dtot = Dt;
    unsigned long long *wacc = ctx->ws.take<unsigned long long>(2 * W + 8);
    unsigned long long *acc = wacc + 2 * W;   // err word at acc[2]
    a.err = reinterpret_cast<int *>(acc + 2);
    uint32_t *tot = ctx->ws.take<uint32_t>(2ull * Dt + 2);
    uint32_t *fill = ctx->ws.take<uint32_t>(2ull * Dt + 2);
    a.seg_totals = tot;
    uint64_t *pstart = ctx->ws.take<uint64_t>(2ull * (Dt + 1));
    a.out[0].pstart = pstart;
    a.out[1].pstart = pstart + (Dt + 1);
    uint64_t *bsum64 = ctx->ws.take<uint64_t>(nbs);
    uint32_t *bsum32 = reinterpret_cast<uint32_t *>(ctx->ws.take<uint64_t>(nbs));
    uint32_t *rch = ctx->ws.take<uint32_t>(Dt + 1);
    uint32_t *sch = ctx->ws.take<uint32_t>(Dt + 1);
    uint32_t *items = ctx->ws.take<uint32_t>(2ull * Dt + 2);
    uint32_t *items_off = ctx->ws.take<uint32_t>(Dt + 1);
    uint32_t *chunk_off = ctx->ws.take<uint32_t>(Dt + 1);
    uint64_t *cstart = ctx->ws.take<uint64_t>(pages * kPageTuples / kChunkW + Dt + 1);
    uint32_t *ctr = ctx->ws.take<uint32_t>(2);

    ADB_CK(cudaMemsetAsync(wacc, 0, (2 * W + 8) * 8, st));
    ADB_CK(cudaMemsetAsync(tot, 0, (2ull * Dt + 2) * 4, st));
    ADB_CK(cudaMemsetAsync(fill, 0, (2ull * Dt + 2) * 4, st));
    ADB_CK(cudaMemsetAsync(ctr, 0, 8, st));
    ADB_CK(cudaEventRecord(ctx->ev[0], st));
    partition_pass<2, kPassThreads><<<dim3(G, 2), kPassThreads, pass_smem(1u << kMaxPassBits, false), st>>>(a);
    ADB_CK(cudaGetLastError());
    ADB_CK(cudaEventRecord(ctx->ev[1], st));
    dscan<uint64_t>(st, tot, Dt, pstart, bsum64);
    dscan<uint64_t>(st, tot + Dt, Dt, pstart + (Dt + 1), bsum64);
    page_place_atomic<<<dim3(G, 2), 256, 0, st>>>(a, fill, fill + Dt);
    part_rslots<<<(Dt + 7) / 8, 256, 0, st>>>(pstart, a.out[0].plist, a.out[0].pcount, Dt, kChunkW, kSPages, rch,
                                             sch);
    items_per_part<<<(Dt + 255) / 256, 256, 0, st>>>(rch, sch, Dt, items);
    dscan<uint32_t>(st, items, Dt, items_off, bsum32);
    dscan<uint32_t>(st, rch, Dt, chunk_off, bsum32);
    copy_last_u32<<<1, 1, 0, st>>>(items_off + Dt, ctr);
    part_rchunks<<<(Dt + 7) / 8, 256, 0, st>>>(pstart, a.out[0].plist, a.out[0].pcount, Dt, kChunkW, chunk_off,
                                              cstart);
    ADB_CK(cudaGetLastError());
    ADB_CK(cudaEventRecord(ctx->ev[2], st));
    JoinArgs ja;
    ja.Rpages = a.out[0].pages; ja.Spages = a.out[1].pages;
    ja.Rcount = a.out[0].pcount; ja.Scount = a.out[1].pcount;
    ja.Rlist = a.out[0].plist; ja.Slist = a.out[1].plist;
    ja.pstart = pstart; ja.items_off = items_off;
    ja.chunk_off = chunk_off; ja.cstart = cstart;
    ja.n_items = ctr; ja.work_counter = ctr + 1;
    ja.acc = acc; ja.err = reinterpret_cast<int *>(acc + 2);
    ja.waits_run_out = 0;
    ja.F = Dt;
    ja.bits = 0;   // per-window fan-out: the kernel reads each window's bits
    ja.mat = nullptr; ja.mat_n = nullptr; ja.mat_cap = 0;
    ja.wbase = d_wbase; ja.wbits = d_bits; ja.nwin = W; ja.wacc = wacc;
    radix_join_items<TableKind::Chain><<<ctx->num_sms * kJoinMinBlocks, kJoinThreads, kJoinSmem, st>>>(ja);
    ADB_CK(cudaGetLastError());
    ADB_CK(cudaEventRecord(ctx->ev[3], st));
    ctx->kernels += 14;
    ADB_CK(cudaMemcpyAsync(h_out, wacc, (2 * W + 8) * 8, cudaMemcpyDeviceToHost, st));
    return ADB_OK;
}

static int batch_join_all(Context *ctx, const uint64_t *dR, const uint64_t *r_off, const uint64_t *dS,
                          const uint64_t *s_off, uint32_t W, uint64_t *counts, uint64_t *sums) {
    ADB_TRY(pinned_reserve(&ctx->h_out, &ctx->h_out_cap, (2 * (size_t)W + 8) * 8));
    unsigned long long *h = reinterpret_cast<unsigned long long *>(ctx->h_out);
    int s = batch_launch(ctx, dR, r_off, dS, s_off, W, h);
    if (s == ADB_OK) {
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) {
            set_error("batched join: %s", cudaGetErrorString(e));
            s = ADB_ERR_DEVICE;
        } else if (h[2 * W + 2]) {
            set_error("device-side check failed in the batched join (code %llu)", h[2 * W + 2]);
            s = ADB_ERR_DEVICE;
        } else {
            for (uint32_t w = 0; w < W; w++) {
                counts[w] = h[2 * w];
                sums[w] = h[2 * w + 1];
            }
        }
    }
    return s;
}

int batch_set_attrs() {
    ADB_CK(cudaFuncSetAttribute(partition_pass<2, kPassThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)pass_smem(1u << kMaxPassBits, false)));
    return ADB_OK;
}

}  // namespace adb

using namespace adb;

extern "C" int adb_batch_join_device(const adb_tuple *dR, const uint64_t *r_off, const adb_tuple *dS,
                                     const uint64_t *s_off, uint32_t n_windows, int mode, uint64_t *counts,
                                     uint64_t *checksums, float *ms_device, void *stream) {
    if (!r_off || !s_off || !counts || !checksums || n_windows == 0) {
        set_error("adb_batch_join_device: bad arguments");
        return ADB_ERR_ARG;
    }
    for (uint32_t w = 0; w < n_windows; w++) {
        if (r_off[w + 1] < r_off[w] || s_off[w + 1] < s_off[w]) {
            set_error("window offsets must not decrease (window %u)", w);
            return ADB_ERR_ARG;
        }
        if (r_off[w + 1] - r_off[w] >= (1ULL << 32) || s_off[w + 1] - s_off[w] >= (1ULL << 32)) {
            set_error("window %u holds 2^32 tuples or more", w);
            return ADB_ERR_ARG;
        }
    }
    if ((r_off[n_windows] > r_off[0] && !dR) || (s_off[n_windows] > s_off[0] && !dS)) {
        set_error("NULL relation");
        return ADB_ERR_ARG;
    }
    int s;
    CtxLock held_ = ctx_acquire(&s);
    Context *ctx = held_.ctx;
    if (!ctx) return s;
    cudaStream_t saved = ctx->stream;
    if (stream) ctx->stream = (cudaStream_t)stream;
    ctx->kernels = 0;
    cudaEvent_t e0 = ctx->ev[8], e1 = ctx->ev[9];
    cudaEventRecord(e0, ctx->stream);
    if (mode == 0) {
        s = batch_join_all(ctx, reinterpret_cast<const uint64_t *>(dR) + r_off[0], r_off,
                           reinterpret_cast<const uint64_t *>(dS) + s_off[0], s_off, n_windows, counts, checksums);
    } else {
        s = ADB_OK;
        for (uint32_t w = 0; w < n_windows && s == ADB_OK; w++) {
            adb_join_result r;
            s = adb_join_device("PRO", dR + r_off[w], r_off[w + 1] - r_off[w], dS + s_off[w],
                                s_off[w + 1] - s_off[w], nullptr, &r, ctx->stream);
            counts[w] = r.count;
            checksums[w] = r.checksum;
        }
    }
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    if (ms_device) {
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        *ms_device = ms;
    }
    ctx->stream = saved;
    return s;
}

// Times the batched join for each window-size bucket at the default fan-out and
// one bit either side, on seeded FK windows, and keeps the fastest; buckets
// lo..hi (log2 of the window size).  bits_out (33 entries, may be NULL)
// receives the table.
extern "C" int adb_batch_autotune(int lo, int hi, int *bits_out) {
    if (lo < 1 || hi > 30 || lo > hi) {
        set_error("adb_batch_autotune: buckets must satisfy 1 <= lo <= hi <= 30");
        return ADB_ERR_ARG;
    }
    int s;
    CtxLock held_ = ctx_acquire(&s);
    Context *ctx = held_.ctx;
    if (!ctx) return s;
    for (int bucket = lo; bucket <= hi; bucket++) {
        const uint64_t n = 1ull << bucket;
        // enough windows of this size for about 2^24 tuples per side
        const uint32_t W = (uint32_t)std::max<uint64_t>(1, (1ull << 24) / n);
        void *dR = nullptr, *dS = nullptr;
        ADB_TRY(adb_device_alloc(&dR, W * n * 8));
        s = adb_device_alloc(&dS, W * n * 8);
        if (s) { adb_device_free(dR); return s; }
        s = adb_gen_uniform((adb_tuple *)dR, W * n, 4 * n, 101 + bucket, 1);
        if (!s) s = adb_gen_uniform((adb_tuple *)dS, W * n, 4 * n, 202 + bucket, 1);
        std::vector<uint64_t> off(W + 1), cnt(W), sum(W);
        for (uint32_t w = 0; w <= W; w++) off[w] = (uint64_t)w * n;
        const int def = default_bits((uint32_t)bucket);
        float best_ms = 1e30f;
        int best = def;
        for (int b = std::max(0, def - 1); b <= std::min((int)kMaxPassBits, def + 1) && !s; b++) {
            g_tune[bucket] = (int8_t)b;
            float ms = 0, tot = 0;
            for (int rep = 0; rep < 3 && !s; rep++) {
                s = adb_batch_join_device((adb_tuple *)dR, off.data(), (adb_tuple *)dS, off.data(), W, 0, cnt.data(),
                                          sum.data(), &ms, nullptr);
                if (rep) tot += ms;
            }
            if (!s && tot < best_ms) { best_ms = tot; best = b; }
        }
        g_tune[bucket] = (int8_t)best;
        adb_device_free(dR);
        adb_device_free(dS);
        if (s) return s;
    }
    if (bits_out)
        for (int b = 0; b < 33; b++) bits_out[b] = g_tune[b] >= 0 ? g_tune[b] : default_bits(b);
    return ADB_OK;
}

extern "C" int adb_batch_set_tuning(const int *bits) {
    if (!bits) {   // back to the built-in rule
        for (int b = 0; b < 33; b++) g_tune[b] = -1;
        return ADB_OK;
    }
    for (int b = 0; b < 33; b++) {
        if (bits[b] > (int)kMaxPassBits) {
            set_error("fan-out bits must be <= %u", kMaxPassBits);
            return ADB_ERR_ARG;
        }
    }
    for (int b = 0; b < 33; b++) g_tune[b] = (int8_t)(bits[b] < 0 ? -1 : bits[b]);
    return ADB_OK;
}
