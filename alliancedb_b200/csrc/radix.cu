// radix.cu -- paged partitioning front end and the partitioned hash joins
// (PRO, RJ_st, PRH, PRHO).
//
// Reference flow: join_init_run (hashing/joins/parallel_radix_join.cpp:1488-1701)
// spawns prj_thread (:981-1473): parallel pass-1 partitioning, task-queued
// pass-2 partitioning, then a task-queued join per partition pair.  Here:
//   pass 1        partition_pass (flat input)  + page lists
//   pass 2        partition_pass (paged input, work units) + page lists  [fan-out > 2^9]
//   R chunks      part_rslots, make_items_paged, part_rchunks
//   join          radix_join_items: persistent, work-stealing build + probe
// The fan-out 2^bits is chosen so an R partition fills about one CTA's
// shared-memory table (17408 tuples).
#include "joins.cuh"
#include "paged.cuh"
#include "radix_join.cuh"

namespace adb {

// CTAs of a flat pass: one per tile up to the CTAs resident at once.
static int flat_ctas(uint64_t nR, uint64_t nS, int num_sms, uint32_t /*F*/) {
    const uint64_t n = nR > nS ? nR : nS;
    const uint64_t cap = (uint64_t)num_sms * kPassMinBlocks;
    uint64_t g = (n + kPTile - 1) / kPTile;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}

// Launches one partition pass (both relations: grid.y = relation).
static void launch_pass(const PassArgs &a, uint32_t F, int G, bool paged, cudaStream_t st) {
    const dim3 grid(G, 2);
    const size_t smem = pass_smem(F, paged);
    if (paged) partition_pass<1, kPassThreads><<<grid, kPassThreads, smem, st>>>(a);
    else if (a.df.hashed) partition_pass<0, kPassThreads, true><<<grid, kPassThreads, smem, st>>>(a);
    else partition_pass<0, kPassThreads><<<grid, kPassThreads, smem, st>>>(a);
}

int radix_bits_for(uint64_t nR, int requested) {
    if (requested > 0) return requested > 14 ? 14 : requested;
    // one pass (<= 9 bits) leaves up to one partial page per CTA in every
    // partition, so it aims at half a join chunk; two passes at a full chunk
    constexpr uint64_t kTarget = kRSlots >= 16384 ? 16384 : 8192;   // power of two <= kRSlots
    int b = (int)ceil_log2_u64((nR + kTarget / 2 - 1) / (kTarget / 2));
    if (b > (int)kMaxPassBits) b = (int)ceil_log2_u64((nR + kTarget - 1) / kTarget);
    if (b < 1) b = 1;
    if (b > 14) b = 14;
    return b;
}

// ---------------------------------------------------------------------------
// Paged partitioning front end
// ---------------------------------------------------------------------------
struct PartPlan {
    int passes;
    uint32_t F1, F2, Fout;
    int G1, G2;
    uint32_t pool1, pool2;
    uint32_t unit_pages;       // pass-2 work unit
    uint64_t pages1, pages2;   // pool pages per relation
};

static PartPlan plan_partition(uint64_t nR, uint64_t nS, uint32_t b1, uint32_t b2, int num_sms) {
    PartPlan p{};
    p.passes = b2 ? 2 : 1;
    p.F1 = 1u << b1;
    p.F2 = b2 ? 1u << b2 : 1u;
    p.Fout = p.F1 * p.F2;
    p.G1 = flat_ctas(nR, nS, num_sms, p.F1);
    const uint32_t a = flat_pool_cap(nR, p.G1, p.F1), b = flat_pool_cap(nS, p.G1, p.F1);
    p.pool1 = a > b ? a : b;
    p.pages1 = (uint64_t)p.G1 * p.pool1;
    if (b2) {
        // units from the tuples actually present (the pass-1 pool has slack)
        const uint64_t pages_in = (nR + kPageTuples - 1) / kPageTuples + (nS + kPageTuples - 1) / kPageTuples;
        p.unit_pages = unit_pages_for(pages_in, num_sms);
        p.G2 = (int)((p.pages1 + p.unit_pages - 1) / p.unit_pages + p.F1);
        p.pool2 = unit_pool_cap(p.F2, p.unit_pages);
        p.pages2 = (uint64_t)p.G2 * p.pool2;
    }
    return p;
}

uint64_t paged_final_pool_pages(uint64_t nR, uint64_t nS, uint32_t b1, uint32_t b2, int num_sms) {
    const PartPlan p = plan_partition(nR, nS, b1, b2, num_sms);
    return p.passes == 2 ? p.pages2 : p.pages1;
}

static size_t pageset_bytes(uint64_t pages, uint32_t G, uint32_t Fout) {
    return Workspace::need(pages * kPageTuples, 8) + Workspace::need(pages, 4) + Workspace::need(pages, 1) +
           Workspace::need(G, 4) + Workspace::need(pages, 4);
}

size_t paged_partition_scratch(uint64_t nR, uint64_t nS, uint32_t b1, uint32_t b2, int num_sms) {
    const PartPlan p = plan_partition(nR, nS, b1, b2, num_sms);
    size_t s = 2 * pageset_bytes(p.pages1, p.G1, p.F1) + Workspace::need(2ull * p.F1 * p.G1, 4) +
               Workspace::need(2ull * p.F1, 4) * 2 + Workspace::need(2ull * (p.F1 + 1), 8);
    if (p.passes == 2)
        s += 2 * pageset_bytes(p.pages2, p.G2, p.Fout) + Workspace::need(2ull * p.F2 * p.G2, 4) +
             Workspace::need(2ull * p.F2, 4) + Workspace::need(2ull * p.Fout, 4) +
             Workspace::need(2ull * (p.Fout + 1), 8) + 2 * Workspace::need(p.F1 + 1, 4);
    return s;
}

static void take_pageset(Context *ctx, PageSet &ps, uint64_t pages, int G) {
    ps.pages = ctx->ws.take<uint64_t>(pages * kPageTuples);
    ps.log = ctx->ws.take<uint32_t>(pages);
    ps.pcount = ctx->ws.take<uint8_t>(pages);
    ps.nlog = ctx->ws.take<uint32_t>(G);
    ps.plist = ctx->ws.take<uint32_t>(pages);
}

// Partitions R and S by d1 (and then d2) into page lists per output partition
// D = p1 * F2 + p2.  out->pstart = [2][Fout + 1] page-list starts.
int run_paged_partition(Context *ctx, const DevJoin &j, DigitFn d1, const DigitFn *d2, PartOut *out,
                        unsigned long long *acc) {
    cudaStream_t st = ctx->stream;
    const uint32_t b1 = ceil_log2_u64((uint64_t)d1.mask + 1), b2 = d2 ? ceil_log2_u64((uint64_t)d2->mask + 1) : 0;
    const PartPlan p = plan_partition(j.nR, j.nS, b1, b2, ctx->num_sms);
    const uint64_t maxpages = p.passes == 2 ? p.pages2 : p.pages1;
    if (p.pages1 * kPageTuples >= (uint64_t)kNone || maxpages * kPageTuples >= (uint64_t)kNone) {
        set_error("relation too large for one partitioned join (%llu pool pages)", (unsigned long long)maxpages);
        return ADB_ERR_ARG;
    }
    int *err = reinterpret_cast<int *>(acc + 2);

    // ---- pass 1
    PassArgs a1{};
    for (int r = 0; r < 2; r++) {
        a1.in[r].in = r ? j.S : j.R;
        a1.in[r].n = r ? j.nS : j.nR;
        take_pageset(ctx, a1.out[r], p.pages1, p.G1);
    }
    a1.df = d1;
    a1.F1 = 1;
    a1.G = p.G1;
    a1.pool_cap = p.pool1;
    a1.paged = 0;
    a1.npd = ctx->ws.take<uint32_t>(2ull * p.F1 * p.G1);
    a1.err = err;
    uint32_t *rowtot1 = ctx->ws.take<uint32_t>(2ull * p.F1);
    uint32_t *totals1 = ctx->ws.take<uint32_t>(2ull * p.F1);
    uint64_t *pstart1 = ctx->ws.take<uint64_t>(2ull * (p.F1 + 1));
    a1.out[0].pstart = pstart1;
    a1.out[1].pstart = pstart1 + (p.F1 + 1);

    launch_pass(a1, p.F1, p.G1, false, st);
    part_scan_rows<<<(2 * p.F1 + 7) / 8, 256, 0, st>>>(a1.npd, rowtot1, p.F1, p.G1);
    pass_totals<<<dim3((p.F1 + 255) / 256, 2), 256, 0, st>>>(a1.npd, rowtot1, nullptr, nullptr, p.F1, 1, p.G1,
                                                             totals1);
    part_scan_totals<<<2, 1024, 0, st>>>(totals1, pstart1, p.F1);
    page_place<<<dim3(p.G1, 2), 1024, p.F1 * 4, st>>>(a1, a1.npd, nullptr, nullptr);
    ADB_CK(cudaGetLastError());
    ADB_CK(cudaEventRecord(ctx->ev[1], st));   // end of pass 1 (callers may re-record)
    ctx->kernels += 5;
    if (p.passes == 1) {
        out->R = a1.out[0];
        out->S = a1.out[1];
        out->Fout = p.F1;
        out->pstart = pstart1;
        out->pool_pages = p.pages1;
        return ADB_OK;
    }

    // ---- pass 2: work units over pass-1 partitions
    PassArgs a2{};
    uint32_t *uoff0 = ctx->ws.take<uint32_t>(p.F1 + 1);
    uint32_t *uoff1 = ctx->ws.take<uint32_t>(p.F1 + 1);
    make_units<<<2, 1024, 0, st>>>(pstart1, pstart1 + (p.F1 + 1), p.F1, p.unit_pages, uoff0, uoff1);
    for (int r = 0; r < 2; r++) {
        PassIn &in = a2.in[r];
        in.pages = a1.out[r].pages;
        in.pcount = a1.out[r].pcount;
        in.plist = a1.out[r].plist;
        in.pstart = a1.out[r].pstart;
        in.uoff = r ? uoff1 : uoff0;
        take_pageset(ctx, a2.out[r], p.pages2, p.G2);
    }
    a2.df = *d2;
    a2.F1 = p.F1;
    a2.G = p.G2;
    a2.pool_cap = p.pool2;
    a2.unit_pages = p.unit_pages;
    a2.paged = 1;
    a2.npd = ctx->ws.take<uint32_t>(2ull * p.F2 * p.G2);
    a2.err = err;
    uint32_t *rowtot2 = ctx->ws.take<uint32_t>(2ull * p.F2);
    uint32_t *totals2 = ctx->ws.take<uint32_t>(2ull * p.Fout);
    uint64_t *pstart2 = ctx->ws.take<uint64_t>(2ull * (p.Fout + 1));
    a2.out[0].pstart = pstart2;
    a2.out[1].pstart = pstart2 + (p.Fout + 1);

    launch_pass(a2, p.F2, p.G2, true, st);
    part_scan_rows<<<(2 * p.F2 + 7) / 8, 256, 0, st>>>(a2.npd, rowtot2, p.F2, p.G2);
    pass_totals<<<dim3((p.Fout + 255) / 256, 2), 256, 0, st>>>(a2.npd, rowtot2, uoff0, uoff1, p.F2, p.F1, p.G2,
                                                               totals2);
    part_scan_totals<<<2, 1024, 0, st>>>(totals2, pstart2, p.Fout);
    page_place<<<dim3(p.G2, 2), 1024, p.F2 * 4, st>>>(a2, a2.npd, uoff0, uoff1);
    ADB_CK(cudaGetLastError());
    ctx->kernels += 6;
    out->R = a2.out[0];
    out->S = a2.out[1];
    out->Fout = p.Fout;
    out->pstart = pstart2;
    out->pool_pages = p.pages2;
    return ADB_OK;
}

static void split_bits(int bits, uint32_t *b1, uint32_t *b2) {
    // one pass up to 2^9 partitions; two passes of at most 2^7 each above
    if (bits <= (int)kMaxPassBits) {
        *b1 = bits;
        *b2 = 0;
    } else {
        *b1 = bits / 2;
        *b2 = bits - bits / 2;
    }
}

// ---------------------------------------------------------------------------
// Partitioned hash joins
// ---------------------------------------------------------------------------
size_t radix_scratch(uint64_t nR, uint64_t nS, int bits, int num_sms) {
    uint32_t b1, b2;
    split_bits(bits, &b1, &b2);
    const PartPlan p = plan_partition(nR, nS, b1, b2, num_sms);
    const uint64_t pagesR = p.passes == 2 ? p.pages2 : p.pages1;
    const uint64_t F = p.Fout;
    return paged_partition_scratch(nR, nS, b1, b2, num_sms) + Workspace::need(F, 4) * 2 +
           Workspace::need(F + 1, 4) * 2 + Workspace::need(pagesR * kPageTuples / kChunkW + F + 1, 8) +
           Workspace::need(2, 4);
}

int run_radix(Context *ctx, const DevJoin &j, bool hist_table, int bits, unsigned long long *acc) {
    cudaStream_t st = ctx->stream;
    uint32_t b1, b2;
    split_bits(bits, &b1, &b2);
    const DigitFn d1{0u, (1u << b1) - 1};
    const DigitFn d2{b1, (1u << b2) - 1};
    PartOut po;
    ADB_TRY(run_paged_partition(ctx, j, d1, b2 ? &d2 : nullptr, &po, acc));
    ADB_CK(cudaEventRecord(ctx->ev[2], st));   // phases: pass 1 | pass 2 | work list | join

    const uint32_t F = po.Fout;
    uint32_t *rch = ctx->ws.take<uint32_t>(F);
    uint32_t *sch = ctx->ws.take<uint32_t>(F);
    uint32_t *items_off = ctx->ws.take<uint32_t>(F + 1);
    uint32_t *chunk_off = ctx->ws.take<uint32_t>(F + 1);
    uint64_t *cstart = ctx->ws.take<uint64_t>(po.pool_pages * kPageTuples / kChunkW + F + 1);
    uint32_t *ctr = ctx->ws.take<uint32_t>(2);   // [0] n_items, [1] work counter
    ADB_CK(cudaMemsetAsync(ctr, 0, 2 * sizeof(uint32_t), st));
    part_rslots<<<(F + 7) / 8, 256, 0, st>>>(po.pstart, po.R.plist, po.R.pcount, F, kChunkW, kSPages, rch, sch);
    make_items_paged<<<1, 1024, 0, st>>>(rch, sch, F, items_off, chunk_off, ctr);
    part_rchunks<<<(F + 7) / 8, 256, 0, st>>>(po.pstart, po.R.plist, po.R.pcount, F, kChunkW, chunk_off, cstart);
    ADB_CK(cudaGetLastError());
    ADB_CK(cudaEventRecord(ctx->ev[3], st));

    JoinArgs a;
    a.Rpages = po.R.pages; a.Spages = po.S.pages;
    a.Rcount = po.R.pcount; a.Scount = po.S.pcount;
    a.Rlist = po.R.plist; a.Slist = po.S.plist;
    a.pstart = po.pstart; a.items_off = items_off;
    a.chunk_off = chunk_off; a.cstart = cstart;
    a.n_items = ctr; a.work_counter = ctr + 1;
    a.acc = acc; a.err = reinterpret_cast<int *>(acc + 2);
    a.waits_run_out = j.test_flags & ADB_TEST_WAITS_RUN_OUT;
    a.F = F; a.bits = (uint32_t)bits;
    a.mat = j.mat; a.mat_n = acc + 3; a.mat_cap = j.mat_cap;
    a.wbase = nullptr; a.wbits = nullptr; a.nwin = 0; a.wacc = nullptr;
    const int grid = ctx->num_sms * kJoinMinBlocks;
    if (hist_table)
        radix_join_items<TableKind::Hist><<<grid, kJoinThreads, kJoinSmem, st>>>(a);
    else
        radix_join_items<TableKind::Chain><<<grid, kJoinThreads, kJoinSmem, st>>>(a);
    ADB_CK(cudaGetLastError());
    ctx->kernels += 4;
    return ADB_OK;
}

int radix_set_attrs() {
    ADB_CK(cudaFuncSetAttribute(partition_pass<0, kPassThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)pass_smem(1u << kMaxPassBits, false)));
    ADB_CK(cudaFuncSetAttribute(partition_pass<0, kPassThreads, true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pass_smem(1u << kMaxPassBits, false)));
    ADB_CK(cudaFuncSetAttribute(partition_pass<1, kPassThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)pass_smem(1u << kMaxPassBits, true)));
    ADB_CK(cudaFuncSetAttribute(radix_join_items<TableKind::Chain>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kJoinSmem));
    ADB_CK(cudaFuncSetAttribute(radix_join_items<TableKind::Hist>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kJoinSmem));
    return ADB_OK;
}

}  // namespace adb
