// npo_noalloc.cu -- NPO join that allocates nothing (adb_npo_join_noalloc).
//
// Who needs it: callers that must not allocate device memory while they run,
// such as a host engine that budgets every byte of HBM up front, or code
// running where cudaMalloc is unavailable or forbidden (inside a
// memory-capped sandbox, or a stream-ordered pipeline that must never
// synchronise on an allocator).  adb_join() cannot serve them: it grows a
// cached workspace with cudaMalloc on first use.
//
// This entry point runs the same NPO build and probe kernels as adb_join("NPO")
// (npo_join.cuh), but its hash table and result words live in a file-scope
// __device__ array of fixed size: kNoAllocTableSlots 8-byte slots (32 MiB) for
// the table plus 4 result words.  The array exists on every GPU that loads
// this library, for as long as the process lives.  The largest build side it
// accepts is kNoAllocMaxBuild tuples (table load <= 0.5); larger calls return
// ADB_ERR_ARG.
//
// Host code cannot pass the array's name to a kernel: on the host that name
// is only a stand-in symbol, not a device address.  The device address is
// looked up once per device with cudaGetSymbolAddress, by the first call made
// while that device is current, and cached.  Make that first call before any
// stream capture.  The cached address belongs to the device's primary context:
// after cudaDeviceReset (or anything else that destroys that context) the
// library must be reloaded before this entry point is used again.
//
// Every call on a device shares the one array and leaves the last call's
// contents behind; each call clears the table part it uses and the result
// words before building.  Calls that overlap on the GPU (different streams or
// threads at the same time) race on the array: serialise them.
#include <mutex>

#include "engine.cuh"
#include "npo_join.cuh"

namespace adb {

constexpr uint64_t kNoAllocTableSlots = 1ULL << 22;                 // 32 MiB of slots
constexpr uint64_t kNoAllocMaxBuild = kNoAllocTableSlots / 2;       // 2^21 build tuples
// A table of 2^ceil(log2(2 nR)) <= kNoAllocTableSlots slots is at most half
// full, so every insert finds an empty slot before it has tried them all and
// npo_build never sets its table-full error word: the two result words are the
// whole outcome of a call.
static_assert(2 * kNoAllocMaxBuild <= kNoAllocTableSlots, "the fixed table must stay at most half full");

// [0, kNoAllocTableSlots) table slots, then count, checksum, error word,
// sentinel counter.
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocTableSlots + 4];

static std::mutex g_noalloc_mu;
static unsigned long long *g_noalloc_addr[64];

static int noalloc_scratch_ptr(unsigned long long **out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        set_error("adb_npo_join_noalloc: no current CUDA device (%s)", cudaGetErrorString(e));
        return ADB_ERR_NO_DEVICE;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            set_error("adb_npo_join_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
                      cudaGetErrorString(e));
            return ADB_ERR_DEVICE;
        }
        g_noalloc_addr[dev] = static_cast<unsigned long long *>(p);
    }
    *out = g_noalloc_addr[dev];
    return ADB_OK;
}

// Copies the accumulated count and checksum into the caller's output words.
__global__ void noalloc_emit(const unsigned long long *acc, uint64_t *out) {
    if (threadIdx.x == 0) {
        out[0] = acc[0];
        out[1] = acc[1];
    }
}

}  // namespace adb

using namespace adb;

extern "C" int adb_npo_join_noalloc(const adb_tuple *dR, uint64_t nR, const adb_tuple *dS, uint64_t nS,
                                    uint64_t *d_out, void *stream) {
    if (!d_out || (nR && !dR) || (nS && !dS)) {
        set_error("adb_npo_join_noalloc: NULL pointer");
        return ADB_ERR_ARG;
    }
    if (nR > kNoAllocMaxBuild) {
        set_error("adb_npo_join_noalloc: build side of %llu tuples exceeds the fixed table's limit of %llu",
                  (unsigned long long)nR, (unsigned long long)kNoAllocMaxBuild);
        return ADB_ERR_ARG;
    }
    if (nS >= (1ULL << 32)) {
        set_error("adb_npo_join_noalloc: probe side must hold fewer than 2^32 tuples");
        return ADB_ERR_ARG;
    }
    unsigned long long *scratch = nullptr;
    ADB_TRY(noalloc_scratch_ptr(&scratch));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint32_t l2 = ceil_log2_u64(2 * (nR ? nR : 1));
    if (l2 < 2) l2 = 2;   // at least four slots (the probe's first read is a four-slot window)
    uint64_t *table = reinterpret_cast<uint64_t *>(scratch);
    unsigned long long *acc = scratch + kNoAllocTableSlots;   // count, checksum, err, sentinel
    ADB_CK(cudaMemsetAsync(table, 0xFF, (1ULL << l2) * sizeof(uint64_t), st));
    ADB_CK(cudaMemsetAsync(acc, 0, 4 * sizeof(unsigned long long), st));
    if (nR && nS) {
        const int threads = 256;
        auto blocks = [&](uint64_t n) {
            const uint64_t b = (n + threads - 1) / threads;
            return (int)(b < 1 ? 1 : (b > (uint64_t)kNumSMs * 8 ? (uint64_t)kNumSMs * 8 : b));
        };
        npo_build<<<blocks(nR), threads, 0, st>>>(reinterpret_cast<const uint64_t *>(dR), nR, table, l2, acc + 3,
                                                  reinterpret_cast<int *>(acc + 2));
        npo_probe<false><<<blocks(nS), threads, 0, st>>>(reinterpret_cast<const uint64_t *>(dS), nS, table, l2,
                                                         acc + 3, acc, nullptr, nullptr, 0);
    }
    noalloc_emit<<<1, 32, 0, st>>>(acc, d_out);
    ADB_CK(cudaGetLastError());
    return ADB_OK;
}
