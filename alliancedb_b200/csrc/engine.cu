// engine.cu -- context, workspace, algorithm registry and the C ABI of
// libadb_b200.so (declared in include/adb/adb_join.h).
//
// The registry mirrors the reference's name -> function tables
// (hashing/main.cpp:306-338, sorting/main.cpp:481-486).  Each name maps to a
// GPU pipeline; names whose reference code is a stub or unfinished are listed
// as not provided and return ADB_ERR_UNSUPPORTED.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <thread>
#include <vector>

#include "datagen.cuh"
#include "joins.cuh"

namespace adb {

int radix_set_attrs();
int smj_set_attrs();
int eager_set_attrs();
int batch_set_attrs();

static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

int Workspace::reserve(size_t bytes) {
    off = 0;
    if (bytes <= cap) return ADB_OK;
    if (base) cudaFree(base);
    base = nullptr;
    cap = 0;
    size_t want = bytes + (bytes >> 3);   // headroom for slightly larger calls
    cudaError_t e = cudaMalloc(&base, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        e = cudaMalloc(&base, bytes);
        want = bytes;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        base = nullptr;
        set_error("device workspace of %zu bytes: %s", bytes, cudaGetErrorString(e));
        return ADB_ERR_OOM;
    }
    cap = want;
    return ADB_OK;
}

int pinned_reserve(char **buf, size_t *cap, size_t bytes) {
    if (bytes <= *cap) return ADB_OK;
    if (*buf) cudaFreeHost(*buf);
    *buf = nullptr;
    *cap = 0;
    const size_t want = bytes + (bytes >> 2);
    if (cudaMallocHost(reinterpret_cast<void **>(buf), want) != cudaSuccess) {
        cudaGetLastError();
        *buf = nullptr;
        set_error("pinned host buffer of %zu bytes", want);
        return ADB_ERR_OOM;
    }
    *cap = want;
    return ADB_OK;
}

static int copy_init(Context *ctx) {
    if (ctx->copy_done) return ADB_OK;
    constexpr int T = Context::kCopyWorkers;
    for (int t = 0; t < T; t++) {
        ADB_CK(cudaStreamCreateWithFlags(&ctx->copy_st[t], cudaStreamNonBlocking));
        for (auto &e : ctx->copy_ev[t]) ADB_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    ADB_CK(cudaEventCreateWithFlags(&ctx->copy_start, cudaEventDisableTiming));
    ADB_CK(cudaEventCreateWithFlags(&ctx->copy_done, cudaEventDisableTiming));
    return ADB_OK;
}

int h2d_copy(Context *ctx, void *dst, const void *src, size_t bytes, cudaStream_t st, bool after_st) {
    if (!bytes) return ADB_OK;
    cudaPointerAttributes at{};
    const bool pinned = cudaPointerGetAttributes(&at, src) == cudaSuccess && at.type == cudaMemoryTypeHost;
    cudaGetLastError();
    constexpr int T = Context::kCopyWorkers;
    constexpr size_t K = Context::kCopyChunk;
    const unsigned hw = std::thread::hardware_concurrency();
    const int workers = (int)std::min<unsigned>(T, hw > 1 ? hw / 2 : 1u);
    if (pinned || bytes < (16u << 20) || workers < 2) {
        if (after_st) {
            ADB_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
            return ADB_OK;
        }
        ADB_TRY(copy_init(ctx));
        ADB_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->copy_st[0]));
        ADB_CK(cudaEventRecord(ctx->copy_done, ctx->copy_st[0]));
        ADB_CK(cudaStreamWaitEvent(st, ctx->copy_done, 0));
        return ADB_OK;
    }
    ADB_TRY(copy_init(ctx));
    if (!ctx->h_copy && cudaMallocHost(reinterpret_cast<void **>(&ctx->h_copy), (size_t)T * 2 * K) != cudaSuccess) {
        cudaGetLastError();
        ctx->h_copy = nullptr;
        set_error("pinned staging buffer of %zu bytes", (size_t)T * 2 * K);
        return ADB_ERR_OOM;
    }
    if (after_st) {   // the copies start after the work already queued on st (dst may be in use there)
        ADB_CK(cudaEventRecord(ctx->copy_start, st));
        for (int t = 0; t < workers; t++) ADB_CK(cudaStreamWaitEvent(ctx->copy_st[t], ctx->copy_start, 0));
    }
    const size_t chunks = (bytes + K - 1) / K;
    std::vector<cudaError_t> errs(workers, cudaSuccess);
    auto work = [&](int t) {
        cudaError_t e = cudaSetDevice(ctx->device);
        int k = 0;
        for (size_t c = t; c < chunks && e == cudaSuccess; c += workers, k ^= 1) {
            unsigned char *slot = ctx->h_copy + ((size_t)t * 2 + k) * K;
            e = cudaEventSynchronize(ctx->copy_ev[t][k]);   // the slot's previous copy is done
            if (e != cudaSuccess) break;
            const size_t off = c * K, len = std::min(K, bytes - off);
            memcpy(slot, static_cast<const unsigned char *>(src) + off, len);
            e = cudaMemcpyAsync(static_cast<unsigned char *>(dst) + off, slot, len, cudaMemcpyHostToDevice,
                                ctx->copy_st[t]);
            if (e == cudaSuccess) e = cudaEventRecord(ctx->copy_ev[t][k], ctx->copy_st[t]);
        }
        errs[t] = e;
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < workers; t++) pool.emplace_back(work, t);
    work(0);
    for (auto &th : pool) th.join();
    for (int t = 0; t < workers; t++) {
        ADB_CK(errs[t]);
        for (auto &e : ctx->copy_ev[t]) ADB_CK(cudaStreamWaitEvent(st, e, 0));   // work after this waits
    }
    return ADB_OK;
}

void Workspace::release() {
    if (base) cudaFree(base);
    base = nullptr;
    cap = off = 0;
}

static std::mutex g_ctx_mu;
static Context *g_ctx[64];

// Creates a context on the current device (stream, events, pinned result
// words, kernel attributes); not registered as the device's default context.
Context *ctx_create(int dev, int *status) {
    Context *c = new Context();
    c->device = dev;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        cudaGetLastError();
        set_error("cudaGetDeviceProperties failed");
        *status = ADB_ERR_DEVICE;
        delete c;
        return nullptr;
    }
    if (prop.major != 10) {
        set_error("device %d is sm_%d%d; this library is built for sm_100a only", dev, prop.major, prop.minor);
        *status = ADB_ERR_NO_DEVICE;
        delete c;
        return nullptr;
    }
    c->num_sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) goto fail;
    for (auto &e : c->ev)
        if (cudaEventCreate(&e) != cudaSuccess) goto fail;
    if (cudaMallocHost(&c->h_res, 64 * sizeof(unsigned long long)) != cudaSuccess) goto fail;
    {
        int s = radix_set_attrs();
        if (s == ADB_OK) s = smj_set_attrs();
        if (s == ADB_OK) s = eager_set_attrs();
        if (s == ADB_OK) s = batch_set_attrs();
        if (s != ADB_OK) {
            *status = s;
            delete c;
            return nullptr;
        }
    }
    *status = ADB_OK;
    return c;
fail:
    set_error("context creation failed: %s", cudaGetErrorString(cudaGetLastError()));
    *status = ADB_ERR_DEVICE;
    delete c;
    return nullptr;
}

void ctx_destroy(Context *c) {
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->ws.release();
    for (auto &e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->h_res) cudaFreeHost(c->h_res);
    if (c->h_stage) cudaFreeHost(c->h_stage);
    if (c->h_out) cudaFreeHost(c->h_out);
    for (int t = 0; t < Context::kCopyWorkers; t++) {
        if (c->copy_st[t]) cudaStreamSynchronize(c->copy_st[t]);
        if (c->copy_st[t]) cudaStreamDestroy(c->copy_st[t]);
        for (auto &e : c->copy_ev[t])
            if (e) cudaEventDestroy(e);
    }
    if (c->copy_start) cudaEventDestroy(c->copy_start);
    if (c->copy_done) cudaEventDestroy(c->copy_done);
    if (c->h_copy) cudaFreeHost(c->h_copy);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

Context *ctx_get(int *status) {
    int dev = 0;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_error("no CUDA device available");
        *status = ADB_ERR_NO_DEVICE;
        return nullptr;
    }
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        set_error("cudaGetDevice failed");
        *status = ADB_ERR_DEVICE;
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    if (g_ctx[dev]) {
        *status = ADB_OK;
        return g_ctx[dev];
    }
    Context *c = ctx_create(dev, status);
    if (c) g_ctx[dev] = c;
    return c;
}

CtxLock ctx_acquire(int *status) {
    CtxLock l;
    l.ctx = ctx_get(status);
    if (l.ctx) l.lk = std::unique_lock<std::recursive_mutex>(l.ctx->mu);
    return l;
}

// --------------------------------------------------------------------------
// Algorithm registry
// --------------------------------------------------------------------------
struct AlgoEntry {
    const char *name;
    Family fam;
    int model;        // eager distribution model, or variant
    bool provided;
};

// eager models: the reference's fetcher/shuffler combinations
enum { M_JM_NP = 0, M_JM_P = 1, M_JB_NP = 2, M_JB_P = 3, M_JBCR_NP = 4, M_JBCR_P = 5, M_HS_NP = 6, M_ST = 7 };

static const AlgoEntry kAlgos[] = {
    // hashing/main.cpp:306-338
    {"PRO", Family::Radix, 0, true},
    {"RJ_st", Family::Radix, 1, true},
    {"PRH", Family::RadixHist, 0, true},
    {"PRHO", Family::RadixHist, 1, true},
    {"NPO", Family::Npo, 0, true},
    {"NPO_st", Family::Npo, 1, true},
    {"SHJ_st", Family::Shj, M_ST, true},
    {"SHJ_JM_P", Family::Shj, M_JM_P, true},
    {"SHJ_JM_NP", Family::Shj, M_JM_NP, true},
    {"SHJ_JB_NP", Family::Shj, M_JB_NP, true},
    {"SHJ_JBCR_NP", Family::Shj, M_JBCR_NP, true},
    {"SHJ_JBCR_P", Family::Shj, M_JBCR_P, true},
    {"SHJ_HS_NP", Family::Shj, M_HS_NP, true},
    {"PMJ_st", Family::Pmj, M_ST, true},
    {"PMJ_JM_NP", Family::Pmj, M_JM_NP, true},
    {"PMJ_JM_P", Family::Pmj, M_JM_P, true},
    {"PMJ_JB_NP", Family::Pmj, M_JB_NP, true},
    {"PMJ_JB_P", Family::Pmj, M_JB_P, true},    // onlinejoins.cpp:405-423 (not in algos[])
    {"PMJ_JBCR_NP", Family::Pmj, M_JBCR_NP, true},
    {"PMJ_JBCR_P", Family::Pmj, M_JBCR_P, true},
    {"PMJ_HS_NP", Family::Pmj, M_HS_NP, true},
    // ripple joins are marked unfinished in the reference (hashing/main.cpp:331)
    {"RPJ_st", Family::Unsupported, 0, false},
    {"RPJ_JM_NP", Family::Unsupported, 0, false},
    {"RPJ_JB_NP", Family::Unsupported, 0, false},
    {"RPJ_JBCR_NP", Family::Unsupported, 0, false},
    {"RPJ_HS_NP", Family::Unsupported, 0, false},
    // sorting/main.cpp:481-486
    {"m-way", Family::SortMerge, 0, true},
    {"m-pass", Family::SortMerge, 1, true},
    {"m-way+skew", Family::SortMerge, 2, true},
    // sortmergejoin_mpsm.cpp:38-42 prints "excluded" and exits
    {"mpsm", Family::Unsupported, 0, false},
};
static const int kNumAlgos = sizeof(kAlgos) / sizeof(kAlgos[0]);

static const AlgoEntry *find_algo(const char *name) {
    if (!name) return nullptr;
    for (int i = 0; i < kNumAlgos; i++)
        if (strcmp(kAlgos[i].name, name) == 0) return &kAlgos[i];
    return nullptr;
}

static uint64_t eager_batch(const adb_join_params *p) {
    if (p && p->batch_tuples > 0) return (uint64_t)p->batch_tuples;
    // one millisecond of each stream: step_size tuples per interval ms
    if (p && p->step_size_r > 0 && p->interval > 0)
        return std::max<uint64_t>(1, (uint64_t)p->step_size_r / (uint64_t)p->interval);
    return 1600;   // 1.6M tuples/s
}

static size_t scratch_for(const AlgoEntry *a, uint64_t nR, uint64_t nS, const adb_join_params *p, int num_sms) {
    switch (a->fam) {
        case Family::Radix:
        case Family::RadixHist:
            return radix_scratch(nR, nS, radix_bits_for(nR, p ? p->radix_bits : 0), num_sms);
        case Family::Npo: return npo_scratch(nR, nS, p ? p->radix_bits : 0, num_sms);
        case Family::SortMerge: return smj_scratch(nR, nS, p ? p->part_fanout : 0, num_sms);
        case Family::Shj:
        case Family::Pmj:
            return eager_scratch(nR, nS, a->fam, a->model, p && p->nthreads ? (int)p->nthreads : 1,
                                 p ? p->group_size : 0);
        default: return 0;
    }
}

static int dispatch(Context *ctx, const AlgoEntry *a, const DevJoin &j, const adb_join_params *p,
                    unsigned long long *acc) {
    switch (a->fam) {
        case Family::Radix:
            return run_radix(ctx, j, false, radix_bits_for(j.nR, p ? p->radix_bits : 0), acc);
        case Family::RadixHist:
            return run_radix(ctx, j, true, radix_bits_for(j.nR, p ? p->radix_bits : 0), acc);
        case Family::Npo: return run_npo(ctx, j, p ? p->radix_bits : 0, acc);
        case Family::SortMerge: return run_smj(ctx, j, p ? p->part_fanout : 0, a->model == 1, acc);
        case Family::Shj:
        case Family::Pmj:
            return run_eager(ctx, j, a->fam, a->model, eager_batch(p), p && p->nthreads ? (int)p->nthreads : 0,
                             p ? p->group_size : 0, p && p->progressive_step > 0 ? p->progressive_step : 1,
                             p ? p->seed : 0, acc);
        default: set_error("algorithm %s is not provided", a->name); return ADB_ERR_UNSUPPORTED;
    }
}

// Runs one join on device-resident inputs; inputs may live inside the workspace
// region [0, pre) that the caller already reserved.
static int join_device_core(Context *ctx, const AlgoEntry *a, DevJoin j, const adb_join_params *p,
                            adb_join_result *out, size_t pre_bytes) {
    cudaStream_t st = ctx->stream;
    ctx->kernels = 0;
    ctx->ws.off = pre_bytes;
    unsigned long long *acc = ctx->ws.take<unsigned long long>(4);
    ADB_CK(cudaMemsetAsync(acc, 0, 4 * sizeof(unsigned long long), st));
    // phase events: ev[0] start; drivers record ev[1..3] at their phase
    // boundaries (radix: after histograms, after scatter, before the join
    // kernel); ev[6] end.  Unrecorded boundaries collapse onto the start.
    for (int k = 0; k < 4; k++) ADB_CK(cudaEventRecord(ctx->ev[k], st));
    if (j.nR && j.nS) ADB_TRY(dispatch(ctx, a, j, p, acc));
    ADB_CK(cudaEventRecord(ctx->ev[6], st));
    ADB_CK(cudaMemcpyAsync(ctx->h_res, acc, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    ADB_CK(cudaStreamSynchronize(st));
    float t[4] = {0, 0, 0, 0}, tot = 0;
    ADB_CK(cudaEventElapsedTime(&tot, ctx->ev[0], ctx->ev[6]));
    for (int k = 0; k < 3; k++) ADB_CK(cudaEventElapsedTime(&t[k], ctx->ev[k], ctx->ev[k + 1]));
    ADB_CK(cudaEventElapsedTime(&t[3], ctx->ev[3], ctx->ev[6]));
    out->count = ctx->h_res[0];
    out->checksum = ctx->h_res[1];
    out->materialized = std::min<uint64_t>(ctx->h_res[3], j.mat_cap);
    for (int k = 0; k < 4; k++) out->ms_phase[k] = t[k];
    out->ms_device = tot;
    out->kernels = ctx->kernels;
    if (ctx->h_res[2]) {
        set_error("a bounded device wait ran out (error word %llu)", ctx->h_res[2]);
        return ADB_ERR_TIMEOUT;
    }
    return ADB_OK;
}

static int check_sizes(uint64_t nR, uint64_t nS) {
    if (nR >= (1ULL << 32) || nS >= (1ULL << 32)) {
        set_error("relations must hold fewer than 2^32 tuples (got %llu, %llu)", (unsigned long long)nR,
                  (unsigned long long)nS);
        return ADB_ERR_ARG;
    }
    return ADB_OK;
}

}  // namespace adb

using namespace adb;

// ==========================================================================
// C ABI
// ==========================================================================
extern "C" {

void adb_params_default(adb_join_params *p) {
    if (!p) return;
    memset(p, 0, sizeof *p);
    // hashing/main.cpp:340-390 defaultParam
    p->nthreads = 1;
    p->window_size = 1000;
    p->step_size_r = 1600;
    p->step_size_s = 1600;
    p->interval = 1;
    p->group_size = 2;
    p->progressive_step = 1;
    p->merge_step = 2;
}

const char *adb_last_error(void) { return g_err; }
const char *adb_version(void) { return "adb_b200 1.0 (sm_100a)"; }

int adb_algo_count(void) { return kNumAlgos; }

const char *adb_algo_name(int i, int *provided) {
    if (i < 0 || i >= kNumAlgos) return nullptr;
    if (provided) *provided = kAlgos[i].provided ? 1 : 0;
    return kAlgos[i].name;
}

int adb_join_device(const char *algo, const adb_tuple *dR, uint64_t nR, const adb_tuple *dS, uint64_t nS,
                    const adb_join_params *p, adb_join_result *out, void *stream) {
    if (!out) { set_error("out is NULL"); return ADB_ERR_ARG; }
    memset(out, 0, sizeof *out);
    const AlgoEntry *a = find_algo(algo);
    if (!a) { set_error("unknown algorithm '%s'", algo ? algo : "(null)"); return out->status = ADB_ERR_ARG; }
    if (!a->provided) { set_error("algorithm %s is not provided", a->name); return out->status = ADB_ERR_UNSUPPORTED; }
    if ((nR && !dR) || (nS && !dS)) { set_error("NULL relation"); return out->status = ADB_ERR_ARG; }
    int s = check_sizes(nR, nS);
    if (s) return out->status = s;
    CtxLock held_ = ctx_acquire(&s);
    Context *ctx = held_.ctx;
    if (!ctx) return out->status = s;
    cudaStream_t saved = ctx->stream;
    if (stream) ctx->stream = (cudaStream_t)stream;
    s = ctx->ws.reserve(scratch_for(a, nR, nS, p, ctx->num_sms) + 4096);
    if (s == ADB_OK) {
        DevJoin j{reinterpret_cast<const uint64_t *>(dR), nR, reinterpret_cast<const uint64_t *>(dS), nS};
        j.test_flags = p ? p->test_flags : 0;
        s = join_device_core(ctx, a, j, p, out, 0);
    }
    ctx->stream = saved;
    return out->status = s;
}

int adb_join_materialize_device(const char *algo, const adb_tuple *dR, uint64_t nR, const adb_tuple *dS,
                                uint64_t nS, const adb_join_params *p, adb_tuple *dOut, uint64_t cap,
                                adb_join_result *out, void *stream) {
    if (!out) { set_error("out is NULL"); return ADB_ERR_ARG; }
    memset(out, 0, sizeof *out);
    const AlgoEntry *a = find_algo(algo);
    if (!a) { set_error("unknown algorithm '%s'", algo ? algo : "(null)"); return out->status = ADB_ERR_ARG; }
    if (!(a->fam == Family::Radix || a->fam == Family::RadixHist || a->fam == Family::Npo ||
          a->fam == Family::SortMerge)) {
        set_error("materialisation is provided for the lazy joins (PRO, RJ_st, PRH, PRHO, NPO, NPO_st, m-way, m-pass)");
        return out->status = ADB_ERR_UNSUPPORTED;
    }
    if ((nR && !dR) || (nS && !dS) || (cap && !dOut)) { set_error("NULL pointer"); return out->status = ADB_ERR_ARG; }
    int s = check_sizes(nR, nS);
    if (s) return out->status = s;
    CtxLock held_ = ctx_acquire(&s);
    Context *ctx = held_.ctx;
    if (!ctx) return out->status = s;
    cudaStream_t saved = ctx->stream;
    if (stream) ctx->stream = (cudaStream_t)stream;
    s = ctx->ws.reserve(scratch_for(a, nR, nS, p, ctx->num_sms) + 4096);
    if (s == ADB_OK) {
        DevJoin j{reinterpret_cast<const uint64_t *>(dR), nR, reinterpret_cast<const uint64_t *>(dS), nS,
                  reinterpret_cast<uint64_t *>(dOut), cap};
        j.test_flags = p ? p->test_flags : 0;
        s = join_device_core(ctx, a, j, p, out, 0);
    }
    ctx->stream = saved;
    return out->status = s;
}

int adb_join(const char *algo, const adb_tuple *R, uint64_t nR, const adb_tuple *S, uint64_t nS,
             const adb_join_params *p, adb_join_result *out) {
    if (!out) { set_error("out is NULL"); return ADB_ERR_ARG; }
    memset(out, 0, sizeof *out);
    const AlgoEntry *a = find_algo(algo);
    if (!a) { set_error("unknown algorithm '%s'", algo ? algo : "(null)"); return out->status = ADB_ERR_ARG; }
    if (!a->provided) { set_error("algorithm %s is not provided", a->name); return out->status = ADB_ERR_UNSUPPORTED; }
    if ((nR && !R) || (nS && !S)) { set_error("NULL relation"); return out->status = ADB_ERR_ARG; }
    int s = check_sizes(nR, nS);
    if (s) return out->status = s;
    CtxLock held_ = ctx_acquire(&s);
    Context *ctx = held_.ctx;
    if (!ctx) return out->status = s;
    const size_t in_bytes = Workspace::need(nR + 2, 8) + Workspace::need(nS + 2, 8);
    s = ctx->ws.reserve(in_bytes + scratch_for(a, nR, nS, p, ctx->num_sms) + 4096);
    if (s) return out->status = s;
    uint64_t *dR = ctx->ws.take<uint64_t>(nR + 2);
    uint64_t *dS = ctx->ws.take<uint64_t>(nS + 2);
    cudaStream_t st = ctx->stream;
    ADB_CK(cudaEventRecord(ctx->ev[4], st));
    s = h2d_copy(ctx, dR, R, nR * 8, st);
    if (s == ADB_OK) s = h2d_copy(ctx, dS, S, nS * 8, st);
    if (s) return out->status = s;
    ADB_CK(cudaEventRecord(ctx->ev[5], st));
    DevJoin j{dR, nR, dS, nS};
    j.test_flags = p ? p->test_flags : 0;
    s = join_device_core(ctx, a, j, p, out, ctx->ws.off);
    float th = 0;
    if (cudaEventElapsedTime(&th, ctx->ev[4], ctx->ev[5]) == cudaSuccess) out->ms_h2d = th;
    return out->status = s;
}

int adb_stream_join(const char *algo, const adb_stream_tuple *R, uint64_t nR, const adb_stream_tuple *S,
                    uint64_t nS, const adb_join_params *p, adb_window_result *windows, uint64_t max_windows,
                    uint64_t *n_windows) {
    return adb_stream_join_progress(algo, R, nR, S, nS, p, windows, nullptr, max_windows, n_windows);
}

int adb_stream_join_progress(const char *algo, const adb_stream_tuple *R, uint64_t nR, const adb_stream_tuple *S,
                             uint64_t nS, const adb_join_params *p, adb_window_result *windows,
                             adb_window_progress *progress, uint64_t max_windows, uint64_t *n_windows) {
    if (!n_windows) { set_error("n_windows is NULL"); return ADB_ERR_ARG; }
    *n_windows = 0;
    const AlgoEntry *a = find_algo(algo);
    if (!a) { set_error("unknown algorithm '%s'", algo ? algo : "(null)"); return ADB_ERR_ARG; }
    if (a->fam != Family::Shj && a->fam != Family::Pmj) {
        set_error("%s is not an eager stream join (SHJ_* or PMJ_*)", a->name);
        return ADB_ERR_ARG;
    }
    if ((nR && !R) || (nS && !S) || (max_windows && !windows)) { set_error("NULL pointer"); return ADB_ERR_ARG; }
    // order of short streams checked here (longer ones on the device, after their copy)
    if (nR <= kHostOrderCheck)
        for (uint64_t i = 1; i < nR; i++)
            if (R[i].ts_ms < R[i - 1].ts_ms) { set_error("R is not ordered by timestamp (index %llu)", (unsigned long long)i); return ADB_ERR_ARG; }
    if (nS <= kHostOrderCheck)
        for (uint64_t i = 1; i < nS; i++)
            if (S[i].ts_ms < S[i - 1].ts_ms) { set_error("S is not ordered by timestamp (index %llu)", (unsigned long long)i); return ADB_ERR_ARG; }
    int s;
    CtxLock held_ = ctx_acquire(&s);
    Context *ctx = held_.ctx;
    if (!ctx) return s;
    ctx->kernels = 0;
    return stream_join(ctx, a->fam, a->model, R, nR, S, nS, p, windows, progress, max_windows, n_windows);
}

int adb_device_alloc(void **ptr, size_t bytes) {
    if (!ptr) { set_error("ptr is NULL"); return ADB_ERR_ARG; }
    cudaError_t e = cudaMalloc(ptr, bytes ? bytes : 1);
    if (e != cudaSuccess) { cudaGetLastError(); set_error("cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e)); return ADB_ERR_OOM; }
    return ADB_OK;
}
int adb_device_free(void *ptr) { ADB_CK(cudaFree(ptr)); return ADB_OK; }
int adb_host_alloc_pinned(void **ptr, size_t bytes) {
    if (!ptr) { set_error("ptr is NULL"); return ADB_ERR_ARG; }
    cudaError_t e = cudaMallocHost(ptr, bytes ? bytes : 1);
    if (e != cudaSuccess) { cudaGetLastError(); set_error("cudaMallocHost(%zu): %s", bytes, cudaGetErrorString(e)); return ADB_ERR_OOM; }
    return ADB_OK;
}
int adb_host_free_pinned(void *ptr) { ADB_CK(cudaFreeHost(ptr)); return ADB_OK; }
int adb_memcpy_h2d(void *dst, const void *src, size_t bytes) { ADB_CK(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice)); return ADB_OK; }
int adb_memcpy_d2h(void *dst, const void *src, size_t bytes) { ADB_CK(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost)); return ADB_OK; }
int adb_device_sync(void) { ADB_CK(cudaDeviceSynchronize()); return ADB_OK; }
int adb_release_workspace(void) {
    int s;
    CtxLock held_ = ctx_acquire(&s);
    Context *c = held_.ctx;
    if (!c) return s;
    ADB_CK(cudaStreamSynchronize(c->stream));
    c->ws.release();
    return ADB_OK;
}

}  // extern "C"

// ==========================================================================
// Generators
// ==========================================================================
namespace adb {

template <class F>
static void host_parallel(uint64_t n, F f) {
    unsigned nt = std::thread::hardware_concurrency();
    if (nt == 0) nt = 1;
    if (n < (1u << 16)) nt = 1;
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; t++) {
        const uint64_t b = n * t / nt, e = n * (t + 1) / nt;
        th.emplace_back([=] { for (uint64_t i = b; i < e; i++) f(i); });
    }
    for (auto &x : th) x.join();
}

static Zipf zipf_for(uint64_t nR, double theta) { return Zipf(nR ? nR : 1, theta > 0 ? theta : 1.0); }

}  // namespace adb

extern "C" {

int adb_gen_pk(adb_tuple *R, uint64_t n, uint64_t seed, int on_device) {
    if (n && !R) { set_error("NULL relation"); return ADB_ERR_ARG; }
    if (n >= (1ULL << 32) - 1) { set_error("n too large"); return ADB_ERR_ARG; }
    Perm perm(n ? n : 1, seed);
    uint64_t *w = reinterpret_cast<uint64_t *>(R);
    if (on_device) {
        int s;
        CtxLock held_ = ctx_acquire(&s);
        Context *c = held_.ctx;
        if (!c) return s;
        gen_pk_kernel<<<c->num_sms * 8, 256, 0, c->stream>>>(w, n, perm);
        ADB_CK(cudaGetLastError());
        ADB_CK(cudaStreamSynchronize(c->stream));
        return ADB_OK;
    }
    host_parallel(n, [&](uint64_t i) { w[i] = tword((uint32_t)(1 + perm(i)), (uint32_t)i); });
    return ADB_OK;
}

int adb_gen_fk(adb_tuple *S, uint64_t nS, const adb_tuple *R, uint64_t nR, double theta, uint64_t seed,
               uint32_t *idx, int on_device) {
    if ((nS && !S) || (nS && (!R || nR == 0))) { set_error("NULL or empty relation"); return ADB_ERR_ARG; }
    if (theta < 0 || nR >= (1ULL << 32)) { set_error("bad theta or nR"); return ADB_ERR_ARG; }
    Perm rank_perm(nR, seed ^ 0x5A5A5A5A5A5A5A5AULL);
    Zipf z = zipf_for(nR, theta);
    uint64_t *w = reinterpret_cast<uint64_t *>(S);
    const uint64_t *rw = reinterpret_cast<const uint64_t *>(R);
    if (on_device) {
        int s;
        CtxLock held_ = ctx_acquire(&s);
        Context *c = held_.ctx;
        if (!c) return s;
        gen_fk_kernel<<<c->num_sms * 8, 256, 0, c->stream>>>(w, nS, rw, nR, theta, seed, idx, rank_perm, z);
        ADB_CK(cudaGetLastError());
        ADB_CK(cudaStreamSynchronize(c->stream));
        return ADB_OK;
    }
    host_parallel(nS, [&](uint64_t j) {
        uint64_t i = theta > 0 ? rank_perm(z.sample(seed, j)) : uniform_below(seed, 3, j, nR);
        w[j] = tword(tkey(rw[i]), (uint32_t)j);
        if (idx) idx[j] = (uint32_t)i;
    });
    return ADB_OK;
}

int adb_gen_uniform(adb_tuple *T, uint64_t n, uint64_t key_range, uint64_t seed, int on_device) {
    if ((n && !T) || key_range == 0 || key_range > (1ULL << 32) - 1) { set_error("bad arguments"); return ADB_ERR_ARG; }
    uint64_t *w = reinterpret_cast<uint64_t *>(T);
    if (on_device) {
        int s;
        CtxLock held_ = ctx_acquire(&s);
        Context *c = held_.ctx;
        if (!c) return s;
        gen_uniform_kernel<<<c->num_sms * 8, 256, 0, c->stream>>>(w, n, key_range, seed);
        ADB_CK(cudaGetLastError());
        ADB_CK(cudaStreamSynchronize(c->stream));
        return ADB_OK;
    }
    host_parallel(n, [&](uint64_t i) { w[i] = tword((uint32_t)(1 + uniform_below(seed, 5, i, key_range)), (uint32_t)i); });
    return ADB_OK;
}

}  // extern "C"
