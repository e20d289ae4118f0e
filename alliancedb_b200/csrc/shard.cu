// shard.cu -- the split step of one join sharded over several GPUs.
//
// The lazy joins shard naturally with one exchange step: every rank splits
// its share of R and S by the destination rank of each key, one all-to-all
// moves every tuple to its destination, each rank joins what it received, and
// one all-reduce adds the (count, checksum) pairs (exact: both are sums mod
// 2^64).  adb_shard_split is the device half of the first step; the exchange
// and the reduction are NCCL collectives issued by the caller
// (alliancedb_b200/dist.py), so this file holds no communication code.
//
// The destination of a key is the high bits of a multiplicative hash,
// part = (key * 0x9E3779B1 mod 2^32) * parts / 2^32, so it does not depend on
// the low key bits that the local partitioned join splits on: the received
// tuples spread over all of a rank's partitions.
//
// Kernels (HBM-bound byte work): a per-block count of destinations over
// contiguous chunks (read 8 B per tuple), one small scan, and a scatter that
// re-reads the chunk and writes each tuple to its destination's run (read 8 B
// + write 8 B); order inside a destination's run is not kept (the join does
// not depend on it).
#include <algorithm>

#include "engine.cuh"

namespace adb {

constexpr int kShardThreads = 256;
constexpr uint32_t kMaxShardParts = 32;

// On the device the high word comes from __umulhi: the widened form
// ((uint64_t)h * parts) >> 32, used as the index of the shared-memory atomics
// below, built (nvcc 12.9, sm_100a, ptxas at its default optimisation level)
// into kernels that counted every key in part 0; the same source was right
// at -Xptxas -O0 and with __umulhi, a masked index or global atomics.
__host__ __device__ __forceinline__ uint32_t shard_of(uint32_t key, uint32_t parts) {
#ifdef __CUDA_ARCH__
    return __umulhi(key * 0x9E3779B1u, parts);
#else
    return (uint32_t)(((uint64_t)(key * 0x9E3779B1u) * parts) >> 32);
#endif
}

__host__ __device__ __forceinline__ uint64_t shard_chunk(uint64_t n, uint32_t blocks) {
    return (n + blocks - 1) / blocks;
}

// hist[b * parts + p] = tuples of block b's chunk bound for part p.
static __global__ void __launch_bounds__(kShardThreads)
shard_count(const uint64_t *__restrict__ in, uint64_t n, uint32_t parts, uint32_t *hist) {
    __shared__ uint32_t c[kMaxShardParts];
    for (uint32_t p = threadIdx.x; p < parts; p += blockDim.x) c[p] = 0;
    __syncthreads();
    const uint64_t chunk = shard_chunk(n, gridDim.x);
    const uint64_t b = (uint64_t)blockIdx.x * chunk, e = min(n, b + chunk);
    for (uint64_t i = b + threadIdx.x; i < e; i += blockDim.x) atomicAdd(&c[shard_of(tkey(in[i]), parts)], 1u);
    __syncthreads();
    for (uint32_t p = threadIdx.x; p < parts; p += blockDim.x) hist[(size_t)blockIdx.x * parts + p] = c[p];
}

// In place: hist[b][p] = first output slot of block b's part-p tuples; tot[p]
// = tuples of part p.  One warp per part (parts <= 32), then the part bases.
static __global__ void shard_scan(uint32_t *hist, uint32_t blocks, uint32_t parts, unsigned long long *tot) {
    __shared__ unsigned long long base[kMaxShardParts];
    const int lane = threadIdx.x & 31;
    const uint32_t p = threadIdx.x >> 5;
    unsigned long long carry = 0;
    if (p < parts) {
        for (uint32_t b0 = 0; b0 < blocks; b0 += 32) {
            const uint32_t b = b0 + lane;
            const uint32_t v = b < blocks ? hist[(size_t)b * parts + p] : 0u;
            uint32_t x = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (b < blocks) hist[(size_t)b * parts + p] = (uint32_t)carry + x - v;
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
        if (lane == 0) tot[p] = carry;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long s = 0;
        for (uint32_t k = 0; k < parts; k++) {
            base[k] = s;
            s += tot[k];
        }
    }
    __syncthreads();
    if (p < parts)
        for (uint32_t b = lane; b < blocks; b += 32) hist[(size_t)b * parts + p] += (uint32_t)base[p];
}

// Every tuple of block b's chunk to its part's run, at the block's offsets.
static __global__ void __launch_bounds__(kShardThreads)
shard_scatter(const uint64_t *__restrict__ in, uint64_t n, uint32_t parts, const uint32_t *off,
              uint64_t *__restrict__ out) {
    __shared__ uint32_t cur[kMaxShardParts];
    for (uint32_t p = threadIdx.x; p < parts; p += blockDim.x) cur[p] = off[(size_t)blockIdx.x * parts + p];
    __syncthreads();
    const uint64_t chunk = shard_chunk(n, gridDim.x);
    const uint64_t b = (uint64_t)blockIdx.x * chunk, e = min(n, b + chunk);
    for (uint64_t i = b + threadIdx.x; i < e; i += blockDim.x) {
        const uint64_t w = in[i];
        out[atomicAdd(&cur[shard_of(tkey(w), parts)], 1u)] = w;
    }
}

}  // namespace adb

using namespace adb;

extern "C" int adb_shard_split(const adb_tuple *dIn, uint64_t n, uint32_t parts, adb_tuple *dOut, uint64_t *counts,
                               void *stream) {
    if (!counts || (n && (!dIn || !dOut))) { set_error("adb_shard_split: NULL pointer"); return ADB_ERR_ARG; }
    if (parts < 1 || parts > kMaxShardParts) {
        set_error("adb_shard_split: parts must be 1 .. %u (got %u)", kMaxShardParts, parts);
        return ADB_ERR_ARG;
    }
    if (n >= (1ULL << 32)) { set_error("adb_shard_split: at most 2^32 - 1 tuples"); return ADB_ERR_ARG; }
    int s;
    CtxLock held_ = ctx_acquire(&s);
    Context *ctx = held_.ctx;
    if (!ctx) return s;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    const uint32_t blocks =
        (uint32_t)std::min<uint64_t>((uint64_t)ctx->num_sms * 4, std::max<uint64_t>(1, n / 2048 + 1));
    ADB_TRY(ctx->ws.reserve(Workspace::need((size_t)blocks * parts, 4) + Workspace::need(kMaxShardParts, 8) + 4096));
    uint32_t *hist = ctx->ws.take<uint32_t>((size_t)blocks * parts);
    unsigned long long *tot = ctx->ws.take<unsigned long long>(kMaxShardParts);
    const uint64_t *in = reinterpret_cast<const uint64_t *>(dIn);
    shard_count<<<blocks, kShardThreads, 0, st>>>(in, n, parts, hist);
    shard_scan<<<1, 1024, 0, st>>>(hist, blocks, parts, tot);
    shard_scatter<<<blocks, kShardThreads, 0, st>>>(in, n, parts, hist, reinterpret_cast<uint64_t *>(dOut));
    ADB_CK(cudaGetLastError());
    ADB_CK(cudaMemcpyAsync(ctx->h_res, tot, parts * 8, cudaMemcpyDeviceToHost, st));
    ADB_CK(cudaStreamSynchronize(st));
    for (uint32_t p = 0; p < parts; p++) counts[p] = ctx->h_res[p];
    ctx->kernels += 3;
    return ADB_OK;
}
