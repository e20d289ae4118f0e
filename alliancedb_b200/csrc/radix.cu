// radix.cu -- launch sequence of the partitioned hash joins (PRO, RJ_st, PRH, PRHO).
//
// Reference flow: join_init_run (hashing/joins/parallel_radix_join.cpp:1488-1701)
// spawns prj_thread (:981-1473): parallel pass-1 partitioning, task-queued
// pass-2 partitioning, then a task-queued join per partition pair.  Here one
// partition pass (fan-out 2^bits, chosen so an R partition fits a CTA's shared
// memory) is followed by one persistent work-stealing join launch.
#include "joins.cuh"
#include "partition.cuh"
#include "radix_join.cuh"

namespace adb {

static int part_ctas(uint64_t nR, uint64_t nS, int num_sms) {
    const uint64_t n = nR > nS ? nR : nS;
    uint64_t g = (n + kScatterTile - 1) / kScatterTile;
    if (g < 1) g = 1;
    if (g > (uint64_t)num_sms) g = num_sms;
    return (int)g;
}

int radix_bits_for(uint64_t nR, int requested) {
    if (requested > 0) return requested < 1 ? 1 : (requested > 13 ? 13 : requested);
    // aim at R partitions of about kRCap/2 tuples
    int b = (int)ceil_log2_u64((nR + kRCap / 2 - 1) / (kRCap / 2));
    if (b < 1) b = 1;
    if (b > 11) b = 11;
    return b;
}

size_t radix_scratch(uint64_t nR, uint64_t nS, int bits, int num_sms) {
    const uint64_t F = 1ULL << bits;
    const int G = part_ctas(nR, nS, num_sms);
    return Workspace::need(nR + 2, 8) + Workspace::need(nS + 2, 8) + Workspace::need(2 * F * G, 4) +
           Workspace::need(2 * F, 4) + Workspace::need(2 * (F + 1), 8) + Workspace::need(F + 1, 4) +
           Workspace::need(2, 4);
}

int run_radix(Context *ctx, const DevJoin &j, bool hist_table, int bits, unsigned long long *acc) {
    cudaStream_t st = ctx->stream;
    const uint32_t F = 1u << bits;
    const int G = part_ctas(j.nR, j.nS, ctx->num_sms);
    uint64_t *pR = ctx->ws.take<uint64_t>(j.nR + 2);
    uint64_t *pS = ctx->ws.take<uint64_t>(j.nS + 2);
    uint32_t *hist = ctx->ws.take<uint32_t>((size_t)2 * F * G);
    uint32_t *totals = ctx->ws.take<uint32_t>((size_t)2 * F);
    uint64_t *starts = ctx->ws.take<uint64_t>((size_t)2 * (F + 1));
    uint32_t *items_off = ctx->ws.take<uint32_t>(F + 1);
    uint32_t *ctr = ctx->ws.take<uint32_t>(2);   // [0] n_items, [1] work counter

    RelPair rp;
    rp.in[0] = j.R; rp.in[1] = j.S;
    rp.n[0] = j.nR; rp.n[1] = j.nS;
    rp.out[0] = pR; rp.out[1] = pS;
    DigitFn df{0u, 0u, F - 1};

    ADB_CK(cudaMemsetAsync(ctr, 0, 2 * sizeof(uint32_t), st));
    part_hist<<<dim3(G, 2), kPartThreads, F * 4, st>>>(rp, df, hist, G);
    part_scan_rows<<<(2 * F + 7) / 8, 256, 0, st>>>(hist, totals, F, G);
    part_scan_totals<<<2, 1024, 0, st>>>(totals, starts, F);
    ADB_CK(cudaEventRecord(ctx->ev[1], st));
    part_scatter<<<dim3(G, 2), kPartThreads, scatter_smem(F), st>>>(rp, df, hist, starts, G);
    ADB_CK(cudaGetLastError());
    ADB_CK(cudaEventRecord(ctx->ev[2], st));

    make_items<<<1, 1024, 0, st>>>(starts, F, items_off, ctr, kRCap, kSChunk);
    ADB_CK(cudaEventRecord(ctx->ev[3], st));
    JoinArgs a;
    a.R = pR; a.S = pS; a.starts = starts; a.items_off = items_off;
    a.n_items = ctr; a.work_counter = ctr + 1;
    a.acc = acc; a.err = reinterpret_cast<int *>(acc + 2);
    a.F = F; a.bits = (uint32_t)bits;
    a.mat = j.mat; a.mat_n = acc + 3; a.mat_cap = j.mat_cap;
    if (hist_table)
        radix_join_items<TableKind::Hist><<<ctx->num_sms, kJoinThreads, kJoinSmem, st>>>(a);
    else
        radix_join_items<TableKind::Chain><<<ctx->num_sms, kJoinThreads, kJoinSmem, st>>>(a);
    ADB_CK(cudaGetLastError());
    ctx->kernels += 6;
    return ADB_OK;
}

int radix_set_attrs() {
    ADB_CK(cudaFuncSetAttribute(part_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)scatter_smem(1u << 13)));
    ADB_CK(cudaFuncSetAttribute(radix_join_items<TableKind::Chain>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kJoinSmem));
    ADB_CK(cudaFuncSetAttribute(radix_join_items<TableKind::Hist>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kJoinSmem));
    return ADB_OK;
}

}  // namespace adb
