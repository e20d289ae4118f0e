// engine.cuh -- host-side context of the join library: device, stream, events,
// a grow-only device workspace, and the status/error plumbing of the C ABI.
#pragma once

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "adb_common.cuh"

namespace adb {

struct Context;

void set_error(const char *fmt, ...);
// Grows the pinned host buffer *buf to at least `bytes` (its old contents are lost).
int pinned_reserve(char **buf, size_t *cap, size_t bytes);
// Host -> device copy of `bytes` from src to dst (device), ordered before the
// work queued on st after it and, with after_st, after the work queued on st
// before it (without: dst is not in use there, and the copy overlaps that
// work).  Pinned sources and copies under 16 MiB are one cudaMemcpyAsync;
// larger pageable sources go through pinned slots filled by host worker
// threads, so that the host-side copy runs on several cores and overlaps the
// DMA.  src must stay unchanged until st has passed the copy.
int h2d_copy(Context *ctx, void *dst, const void *src, size_t bytes, cudaStream_t st, bool after_st = true);

#define ADB_CK(call)                                                                      \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            ::adb::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),      \
                             __FILE__, __LINE__);                                         \
            return e_ == cudaErrorMemoryAllocation ? ADB_ERR_OOM : ADB_ERR_DEVICE;        \
        }                                                                                 \
    } while (0)

#define ADB_TRY(expr)                      \
    do {                                   \
        int s_ = (expr);                   \
        if (s_ != ADB_OK) return s_;       \
    } while (0)

// Bump allocator over one cached device buffer.  reserve() grows the buffer
// (free + malloc) only when a call needs more than the current capacity, so
// repeated joins of one size allocate nothing.
struct Workspace {
    char *base = nullptr;
    size_t cap = 0;
    size_t off = 0;
    int reserve(size_t bytes);
    void reset() { off = 0; }
    template <class T>
    T *take(size_t count) {
        size_t bytes = (count * sizeof(T) + 255) & ~(size_t)255;
        T *p = reinterpret_cast<T *>(base + off);
        off += bytes;
        return p;
    }
    static size_t need(size_t count, size_t elem) { return (count * elem + 255) & ~(size_t)255; }
    void release();
};

// Stream tuples per side whose timestamp order adb_stream_join checks on the
// host; longer streams are checked on the device after their copy.
constexpr uint64_t kHostOrderCheck = 1ull << 16;

struct Context {
    int device = -1;
    int num_sms = kNumSMs;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[12] = {};
    Workspace ws;
    unsigned long long *h_res = nullptr;   // pinned: [0] count [1] checksum [2] err [3] mat_n ...
    // pinned, grow-only host buffers of the batched path: the per-call plan (one
    // host -> device copy) and the per-window results (one copy back); growing
    // one needs its previous use finished
    char *h_stage = nullptr;
    size_t h_stage_cap = 0;
    char *h_out = nullptr;
    size_t h_out_cap = 0;
    // staged host -> device copies of pageable memory (h2d_copy): per worker a
    // stream, two pinned slots and an event per slot; made on first use
    static constexpr int kCopyWorkers = 8;
    static constexpr size_t kCopyChunk = 4u << 20;
    cudaStream_t copy_st[kCopyWorkers] = {};
    cudaEvent_t copy_ev[kCopyWorkers][2] = {};
    cudaEvent_t copy_start = nullptr, copy_done = nullptr;
    unsigned char *h_copy = nullptr;       // kCopyWorkers x 2 x kCopyChunk
    bool attrs_set = false;
    int kernels = 0;                       // kernels launched by the current call
    std::recursive_mutex mu;               // held by the call that uses this context
};

// The per-device context, locked for the holder's scope: calls from several
// host threads on one device are serialised, each owning the context's
// stream, events and workspace while it runs.  (Recursive: a batched call
// may run per-window joins on the same context.)
struct CtxLock {
    Context *ctx = nullptr;
    std::unique_lock<std::recursive_mutex> lk;
};
CtxLock ctx_acquire(int *status);

// The per-device context (created on first use).  Returns nullptr and sets
// the error if no device is usable.
Context *ctx_get(int *status);
// A separate context on device `dev` (own stream, events and workspace), for
// work that runs beside the default context; released with ctx_destroy.
Context *ctx_create(int dev, int *status);
void ctx_destroy(Context *c);

}  // namespace adb
