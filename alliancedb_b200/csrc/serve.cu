// serve.cu -- a serving loop for windowed-join requests (adb_serve_run).
//
// Requests arrive open-loop (each with an arrival time); a request is one
// window pair R = PK(n_r, seed), S = FK(n_s over R, seed + 1), generated on
// the device from its descriptor, so arrivals cost no host-to-device bandwidth.
// The loop practises continuous batching:
//   * arrived requests wait in a FIFO until admitted;
//   * admission is bounded by device memory: the inputs of in-flight requests
//     live in a ring arena of budget / 4 bytes (the rest of the budget covers
//     the batches' partitioning scratch), and a request enters a batch only
//     while the arena has room;
//   * `slots` execution slots (each its own stream and workspace) run batches
//     concurrently: whenever a slot is idle, everything admitted so far is
//     generated and joined as one batched launch sequence (batch.cu) while the
//     other slots' batches are still on the device;
//   * a finished batch returns its results, frees its arena range, and its
//     requests' latency (completion - arrival, wall clock) is recorded.
#include <algorithm>
#include <chrono>
#include <deque>
#include <thread>
#include <vector>

#include "datagen.cuh"
#include "joins.cuh"

namespace adb {

int batch_launch(Context *ctx, const uint64_t *dR, const uint64_t *r_off, const uint64_t *dS, const uint64_t *s_off,
                 uint32_t W, unsigned long long *h_out);

struct GenDesc {
    uint64_t r_off, s_off;   // tuple offsets inside the batch's R and S areas
    uint32_t n_r, n_s;
    uint64_t seed;
    Perm perm;               // R's key permutation (PK over 1..n_r)
};

// R of every request of a batch: R_k[i] = {payload i, key 1 + perm_k(i)}.
__global__ void gen_batch_pk(uint64_t *R, const GenDesc *d, uint32_t k, uint64_t total) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = k;   // request of tuple i: largest q with r_off[q] <= i
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (d[mid].r_off <= i) lo = mid; else hi = mid;
        }
        const uint64_t j = i - d[lo].r_off;
        R[i] = tword((uint32_t)(1 + d[lo].perm(j)), (uint32_t)j);
    }
}

// S of every request: S_k[j] = {payload j, key R_k[uniform(seed + 1, j) % n_r].key}.
__global__ void gen_batch_fk(uint64_t *S, const uint64_t *R, const GenDesc *d, uint32_t k, uint64_t total) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = k;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (d[mid].s_off <= i) lo = mid; else hi = mid;
        }
        const uint64_t j = i - d[lo].s_off;
        const uint64_t idx = uniform_below(d[lo].seed + 1, 3, j, d[lo].n_r);
        S[i] = tword(tkey(R[d[lo].r_off + idx]), (uint32_t)j);
    }
}

struct Slot {
    Context *ctx = nullptr;
    bool busy = false;
    std::vector<uint32_t> reqs;           // request ids of the batch in flight
    uint64_t arena_end = 0;               // ring position after this batch's inputs
    unsigned long long *h_out = nullptr;  // pinned per-window sums
    GenDesc *h_desc = nullptr;            // pinned descriptors
    GenDesc *d_desc = nullptr;
    uint32_t cap = 0;                     // most requests per batch
    uint32_t batch_id = 0;
    double admit_ms = 0;
};

}  // namespace adb

using namespace adb;

extern "C" int adb_serve_run(const adb_serve_config *cfg, const adb_serve_request *req, uint32_t n,
                             adb_serve_result *res, adb_serve_stats *stats) {
    if (!cfg || (n && (!req || !res))) {
        set_error("adb_serve_run: NULL argument");
        return ADB_ERR_ARG;
    }
    for (uint32_t i = 0; i < n; i++) {
        if (i && req[i].arrival_us < req[i - 1].arrival_us) {
            set_error("requests must be ordered by arrival time (index %u)", i);
            return ADB_ERR_ARG;
        }
        if (req[i].n_r == 0 && req[i].n_s > 0) {
            set_error("request %u: S is drawn from R's keys, so R must not be empty", i);
            return ADB_ERR_ARG;
        }
    }
    int s;
    CtxLock held_ = ctx_acquire(&s);
    Context *c0 = held_.ctx;
    if (!c0) return s;
    const uint32_t max_batch = cfg->max_batch ? cfg->max_batch : 256;
    const uint32_t nslots = cfg->slots ? std::min<uint32_t>(cfg->slots, 4) : 2;
    size_t free_b = 0, total_b = 0;
    ADB_CK(cudaMemGetInfo(&free_b, &total_b));
    uint64_t budget = cfg->budget_bytes ? cfg->budget_bytes : (uint64_t)free_b / 2;
    budget = std::min<uint64_t>(budget, (uint64_t)free_b * 9 / 10);
    const uint64_t arena_bytes = (budget / 4) & ~(uint64_t)255;
    for (uint32_t i = 0; i < n; i++) {
        const uint64_t need = ((uint64_t)req[i].n_r + req[i].n_s) * 8 + 512;
        if (need > arena_bytes) {
            set_error("request %u needs %llu bytes of inputs, more than the admission budget allows (%llu)", i,
                      (unsigned long long)need, (unsigned long long)arena_bytes);
            return ADB_ERR_BUSY;
        }
    }
    uint64_t *arena = nullptr;
    ADB_CK(cudaMalloc(&arena, arena_bytes));
    std::vector<Slot> slots(nslots);
    s = ADB_OK;
    for (auto &sl : slots) {
        sl.ctx = ctx_create(c0->device, &s);
        if (!sl.ctx) break;
        sl.cap = max_batch;
        // the batches' partitioning scratch: the rest of the budget, split over the slots
        if (sl.ctx->ws.reserve((budget - arena_bytes) / nslots) != ADB_OK) { s = ADB_ERR_OOM; break; }
        if (cudaMallocHost(&sl.h_out, (2ull * max_batch + 8) * 8) != cudaSuccess ||
            cudaMallocHost(&sl.h_desc, sizeof(GenDesc) * max_batch) != cudaSuccess ||
            cudaMalloc(&sl.d_desc, sizeof(GenDesc) * max_batch) != cudaSuccess) {
            set_error("serving slot allocation failed");
            s = ADB_ERR_OOM;
            break;
        }
    }
    auto cleanup = [&]() {
        for (auto &sl : slots) {
            if (sl.ctx) ctx_destroy(sl.ctx);
            if (sl.h_out) cudaFreeHost(sl.h_out);
            if (sl.h_desc) cudaFreeHost(sl.h_desc);
            if (sl.d_desc) cudaFree(sl.d_desc);
        }
        cudaFree(arena);
    };
    if (s != ADB_OK) {
        cleanup();
        return s;
    }

    // Ring arena over [0, arena_bytes), freed in admission order: live holds the
    // (batch, start, end) ranges in use, oldest first; new ranges go after the
    // newest one, or wrap to 0 when they fit before the oldest.
    struct Range { uint32_t batch; uint64_t start, end; };
    std::deque<Range> live;
    std::vector<char> finished;   // per batch id
    uint64_t peak = 0, in_use = 0;
    auto ring_place = [&](uint64_t bytes, uint64_t *off) -> bool {
        if (live.empty()) {
            if (bytes > arena_bytes) return false;
            *off = 0;
            return true;
        }
        const uint64_t tail = live.front().start, head = live.back().end;
        if (head >= tail) {   // not wrapped: room after head, or before tail at the start
            if (head + bytes <= arena_bytes) { *off = head; return true; }
            if (bytes <= tail) { *off = 0; return true; }
            return false;
        }
        if (head + bytes <= tail) { *off = head; return true; }   // wrapped: room between head and tail
        return false;
    };
    auto ring_take = [&](uint32_t batch, uint64_t off, uint64_t bytes) {
        live.push_back(Range{batch, off, off + bytes});
        in_use += bytes;
        peak = std::max(peak, in_use);
    };

    const auto t0 = std::chrono::steady_clock::now();
    auto now_ms = [&]() { return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(); };
    std::deque<uint32_t> pending;
    uint32_t next = 0, completed = 0, batches = 0;
    uint64_t batched_reqs = 0;
    double last_done = 0;
    while (completed < n && s == ADB_OK) {
        const double t = now_ms();
        while (next < n && (!cfg->realtime || req[next].arrival_us / 1000.0 <= t)) pending.push_back(next++);
        bool progressed = false;
        // finished batches
        for (auto &sl : slots) {
            if (!sl.busy) continue;
            const cudaError_t q = cudaEventQuery(sl.ctx->ev[11]);
            if (q == cudaErrorNotReady) continue;
            if (q != cudaSuccess) {
                set_error("serving batch failed: %s", cudaGetErrorString(q));
                s = ADB_ERR_DEVICE;
                break;
            }
            const double tdone = now_ms();
            const uint32_t W = (uint32_t)sl.reqs.size();
            if (sl.h_out[2 * W + 2]) {
                set_error("device-side check failed in serving batch %u", sl.batch_id);
                s = ADB_ERR_DEVICE;
                break;
            }
            for (uint32_t k = 0; k < W; k++) {
                adb_serve_result &r = res[sl.reqs[k]];
                r.count = sl.h_out[2 * k];
                r.checksum = sl.h_out[2 * k + 1];
                const double arr = cfg->realtime ? req[sl.reqs[k]].arrival_us / 1000.0 : 0.0;
                r.latency_ms = (float)(tdone - arr);
                r.queue_ms = (float)(sl.admit_ms - arr);
                r.batch = sl.batch_id;
                r.status = ADB_OK;
            }
            completed += W;
            last_done = tdone;
            if (finished.size() <= sl.batch_id) finished.resize(sl.batch_id + 1, 0);
            finished[sl.batch_id] = 1;
            while (!live.empty() && live.front().batch < finished.size() && finished[live.front().batch]) {
                in_use -= live.front().end - live.front().start;
                live.pop_front();
            }
            sl.busy = false;
            progressed = true;
        }
        if (s != ADB_OK) break;
        // launch a batch of everything admitted on an idle slot
        for (auto &sl : slots) {
            if (sl.busy || pending.empty()) continue;
            std::vector<uint32_t> ids;
            uint64_t tr = 0, ts = 0, off = 0, bytes = 0;
            for (uint32_t q : pending) {
                if (ids.size() >= max_batch) break;
                const uint64_t b2 = ((tr + req[q].n_r + ts + req[q].n_s) * 8 + 16 + 255) & ~(uint64_t)255;
                uint64_t o2;
                if (!ring_place(b2, &o2)) break;   // admission: the inputs must fit the arena
                ids.push_back(q);
                tr += req[q].n_r;
                ts += req[q].n_s;
                off = o2;
                bytes = b2;
            }
            if (ids.empty()) break;   // wait for memory
            for (size_t k = 0; k < ids.size(); k++) pending.pop_front();
            const uint32_t W = (uint32_t)ids.size();
            uint64_t *dR = arena + off / 8;
            uint64_t *dS = dR + tr + (tr & 1);   // keep S 16-byte aligned
            std::vector<uint64_t> r_off(W + 1), s_off(W + 1);
            uint64_t ar = 0, as = 0;
            for (uint32_t k = 0; k < W; k++) {
                const adb_serve_request &q = req[ids[k]];
                r_off[k] = ar;
                s_off[k] = as;
                GenDesc &d = sl.h_desc[k];
                d.r_off = ar;
                d.s_off = as;
                d.n_r = q.n_r;
                d.n_s = q.n_s;
                d.seed = q.seed;
                d.perm = Perm(q.n_r ? q.n_r : 1, q.seed);
                ar += q.n_r;
                as += q.n_s;
            }
            r_off[W] = ar;
            s_off[W] = as;
            cudaStream_t st = sl.ctx->stream;
            sl.admit_ms = now_ms();
            if (cudaMemcpyAsync(sl.d_desc, sl.h_desc, sizeof(GenDesc) * W, cudaMemcpyHostToDevice, st) != cudaSuccess) {
                set_error("descriptor copy failed");
                s = ADB_ERR_DEVICE;
                break;
            }
            const int grid = sl.ctx->num_sms * 8;
            if (ar) gen_batch_pk<<<grid, 256, 0, st>>>(dR, sl.d_desc, W, ar);
            if (as) gen_batch_fk<<<grid, 256, 0, st>>>(dS, dR, sl.d_desc, W, as);
            s = batch_launch(sl.ctx, dR, r_off.data(), dS, s_off.data(), W, sl.h_out);
            if (s != ADB_OK) break;
            if (cudaEventRecord(sl.ctx->ev[11], st) != cudaSuccess) {
                s = ADB_ERR_DEVICE;
                break;
            }
            sl.busy = true;
            sl.reqs = ids;
            sl.batch_id = batches++;
            batched_reqs += W;
            ring_take(sl.batch_id, off, bytes);
            progressed = true;
        }
        if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
    for (auto &sl : slots)
        if (sl.busy) cudaStreamSynchronize(sl.ctx->stream);
    if (stats && s == ADB_OK) {
        std::vector<float> lat(n);
        uint64_t tuples = 0;
        for (uint32_t i = 0; i < n; i++) {
            lat[i] = res[i].latency_ms;
            tuples += (uint64_t)req[i].n_r + req[i].n_s;
        }
        std::sort(lat.begin(), lat.end());
        auto pct = [&](double p) -> double {
            if (lat.empty()) return 0.0;
            size_t k = (size_t)std::ceil(p * lat.size()) ;
            k = k ? k - 1 : 0;
            return lat[std::min(k, lat.size() - 1)];
        };
        stats->requests = n;
        stats->tuples = tuples;
        stats->batches = batches;
        stats->makespan_ms = last_done;
        stats->tuples_per_s = last_done > 0 ? tuples / (last_done / 1e3) : 0.0;
        stats->p50_ms = pct(0.50);
        stats->p99_ms = pct(0.99);
        stats->p999_ms = pct(0.999);
        stats->mean_batch = batches ? (double)batched_reqs / batches : 0.0;
        stats->peak_arena_bytes = peak;
        (void)in_use;
        stats->arena_bytes = arena_bytes;
    }
    cleanup();
    return s;
}
