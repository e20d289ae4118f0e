// npo.cu -- launch sequence of the no-partitioning hash join (NPO, NPO_st).
// Reference: NPO hashing/joins/no_partitioning_join.cpp:383-476 (allocate
// the table for |R|/BUCKET_SIZE buckets, build with all threads, barrier,
// probe S chunks).  Here: clear the table, one build launch, one probe launch.
#include "joins.cuh"
#include "npo_join.cuh"

namespace adb {

// 2 slots per build tuple, at least 4 (one 32-byte sector: the probe reads whole sectors)
static uint32_t npo_log2(uint64_t nR) {
    uint32_t l = ceil_log2_u64(2 * (nR ? nR : 1));
    return l < 2 ? 2 : l;
}

size_t npo_scratch(uint64_t nR) {
    return Workspace::need(1ULL << npo_log2(nR), 8) + Workspace::need(1, 8);
}

int run_npo(Context *ctx, const DevJoin &j, unsigned long long *acc) {
    cudaStream_t st = ctx->stream;
    const uint32_t l2 = npo_log2(j.nR);
    uint64_t *table = ctx->ws.take<uint64_t>(1ULL << l2);
    unsigned long long *sent = ctx->ws.take<unsigned long long>(1);
    ADB_CK(cudaMemsetAsync(table, 0xFF, (1ULL << l2) * 8, st));
    ADB_CK(cudaMemsetAsync(sent, 0, 8, st));
    const int threads = 256;
    auto blocks = [&](uint64_t n) {
        uint64_t b = (n + threads - 1) / threads;
        const uint64_t cap = (uint64_t)ctx->num_sms * 8;
        return (int)(b < 1 ? 1 : (b > cap ? cap : b));
    };
    npo_build<<<blocks(j.nR), threads, 0, st>>>(j.R, j.nR, table, l2, sent, reinterpret_cast<int *>(acc + 2));
    ADB_CK(cudaEventRecord(ctx->ev[1], st));
    ADB_CK(cudaEventRecord(ctx->ev[2], st));
    ADB_CK(cudaEventRecord(ctx->ev[3], st));
    if (j.mat)
        npo_probe<true><<<blocks(j.nS), threads, 0, st>>>(j.S, j.nS, table, l2, sent, acc, j.mat, acc + 3, j.mat_cap);
    else
        npo_probe<false><<<blocks(j.nS), threads, 0, st>>>(j.S, j.nS, table, l2, sent, acc, nullptr, nullptr, 0);
    ADB_CK(cudaGetLastError());
    ctx->kernels += 2;
    return ADB_OK;
}

}  // namespace adb
