/*
 * adb_join.h -- C ABI of the B200 join library (libadb_b200.so).
 *
 * This is the drop-in boundary for AllianceDB's join hot path.  The reference
 * dispatches joins through a name -> function table:
 *   hashing:  algo_t{name, result_t *(*)(relation_t *, relation_t *, param_t)}
 *             (hashing/benchmark.h:53-57, table hashing/main.cpp:306-338,
 *              called at hashing/benchmark.cpp:244-247)
 *   sorting:  algo_t{name, result_t *(*)(relation_t *, relation_t *, joinconfig_t *,
 *                    int exp_id, int window_size, int gap)}
 *             (sorting/main.cpp:420-425, table :481-486, called at :752-758)
 * adb_join() takes the same algorithm names and the same relations (arrays of
 * 8-byte {payload @0, key @4} tuples, hashing/utils/types.h:67-70) and returns
 * the reference's result (the match count, result_t.totalresults,
 * hashing/utils/types.h:98-102) plus an order-independent 64-bit checksum over
 * the matched (key, r_payload, s_payload) triples:
 *     a = (u64)key << 32 | r_payload,  b = (u64)s_payload << 32 | key,
 *     H = fmix64(a ^ fmix64(b)),  checksum = sum of H mod 2^64,
 * fmix64 being the SplitMix64 finalizer.
 *
 * Differences from the reference, all deliberate:
 *  - inputs are never modified (the reference's PRO overwrites R and S,
 *    hashing/joins/parallel_radix_join.cpp:1176-1181);
 *  - errors are status codes, never exit() (the reference exits on malloc or
 *    barrier failure, :47-64);
 *  - keys are unsigned 32-bit and every value, 0 and 0xFFFFFFFF included, is a
 *    valid key.
 *
 * All functions are thread-compatible, not thread-safe: one host thread per
 * library context (the library keeps one context per device).
 */
#ifndef ADB_JOIN_H
#define ADB_JOIN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* hashing/utils/types.h:67-70 and sorting/utils/types.h:63-67 */
typedef struct adb_tuple {
    uint32_t payload;
    uint32_t key;
} adb_tuple;

/* Timestamped stream tuple (the reference keeps ts in relation_payload_t,
 * hashing/utils/types.h:83-88; here it travels beside the tuple). */
typedef struct adb_stream_tuple {
    uint64_t ts_ms;
    adb_tuple t;
} adb_stream_tuple;

typedef enum adb_status {
    ADB_OK = 0,
    ADB_ERR_ARG = 1,         /* bad argument: NULL pointer, unknown algorithm, size out of range */
    ADB_ERR_OOM = 2,         /* device or pinned-host allocation failed */
    ADB_ERR_DEVICE = 3,      /* a CUDA call failed; the message says which */
    ADB_ERR_TIMEOUT = 4,     /* a bounded device wait ran out */
    ADB_ERR_UNSUPPORTED = 5, /* name known to the reference but not provided (adb_algo_name reports which) */
    ADB_ERR_BUSY = 6,        /* admission refused: over the device-memory budget */
    ADB_ERR_NO_DEVICE = 7    /* no CUDA device, or the kernels were not built for it */
} adb_status;

/* Subset of the reference's param_t (hashing/benchmark.h:59-112) that the join
 * functions read, plus the GPU tuning knobs.  Zero means "default" for every
 * field; adb_params_default() fills the reference's defaults. */
typedef struct adb_join_params {
    uint32_t nthreads;          /* param_t.nthreads: worker count of the distribution model (JM/JB/JBCR) */
    int32_t window_size;        /* param_t.window_size, ms (eager joins) */
    int32_t step_size_r;        /* param_t.step_sizeR, tuples per interval */
    int32_t step_size_s;        /* param_t.step_sizeS */
    int32_t interval;           /* param_t.interval, ms */
    int32_t group_size;         /* param_t.group_size, JBCR groups (-G) */
    int32_t progressive_step;   /* param_t.progressive_step, PMJ run size in % of each side */
    int32_t merge_step;         /* param_t.merge_step, PMJ runs merged per step */
    int32_t radix_bits;         /* PRO/PRH/RJ fan-out bits; 0 = chosen from |R|.  NPO: bits of the table
                                   regions its inputs are grouped by (up to 9); 0 = chosen from |R|
                                   (none up to a 256 MB table, |R| <= 2^24), < 0 = no grouping */
    int32_t part_fanout;        /* joinconfig_t.PARTFANOUT for m-way/m-pass; 0 = chosen */
    int32_t materialize;        /* 1: also write <S-key, S-payload> per match (JOIN_RESULT_MATERIALIZE) */
    int32_t batch_tuples;       /* eager joins: arrival micro-batch in tuples per side; 0 = 1 ms of stream */
    uint64_t seed;              /* JBCR's random split of S */
    int32_t realtime;           /* adb_stream_join: 1 = release each micro-batch at its timestamp
                                   (wall clock, the reference's WAIT gating, fetcher.cpp:120-190) */
    int32_t test_flags;         /* 0 in normal use.  ADB_TEST_WAITS_RUN_OUT: every bounded device wait
                                   of the partitioned and sort-merge joins, once it has completed,
                                   reports that it ran out, so callers can test their ADB_ERR_TIMEOUT
                                   handling without making a GPU wait for real */
} adb_join_params;

#define ADB_TEST_WAITS_RUN_OUT 1

typedef struct adb_join_result {
    uint64_t count;             /* result_t.totalresults */
    uint64_t checksum;          /* sum of H over the matched pairs, mod 2^64 */
    int32_t status;             /* adb_status */
    int32_t kernels;            /* kernels this call launched */
    float ms_device;            /* device time of the join, CUDA events on the library stream */
    float ms_phase[4];          /* device time per phase; radix: partition pass 1, pass 2 (0 with one pass),
                                   work list, join kernel; NPO: grouping by table region, build, -, probe;
                                   m-way: partitioning,
                                   work list, -, sort + merge-join kernel */
    float ms_h2d;               /* host->device copy time (adb_join only) */
    uint64_t materialized;      /* tuples written to the materialisation buffer */
} adb_join_result;

void adb_params_default(adb_join_params *p);

/* Last error message of this thread (static storage, never NULL). */
const char *adb_last_error(void);
const char *adb_version(void);

/* Number of algorithm names, and the i-th name with its status:
 * 1 = provided, 0 = known to the reference but not provided. */
int adb_algo_count(void);
const char *adb_algo_name(int i, int *provided);

/* Join two host-resident relations: copies R and S to the device (inside the
 * call), joins, and reads back the result.  Replaces the algos[] entry
 * `name`.  R and S are not modified.  Pinned (page-locked) relations are
 * copied by DMA directly; pageable ones of 16 MiB or more go through pinned
 * staging slots that host worker threads fill while earlier slots are in
 * flight (the same for adb_stream_join's streams). */
int adb_join(const char *algo, const adb_tuple *R, uint64_t nR, const adb_tuple *S, uint64_t nS,
             const adb_join_params *p, adb_join_result *out);

/* Join two device-resident relations on `stream` (a cudaStream_t, NULL = the
 * library stream).  Returns after the result is on the host.  The library
 * stream is non-blocking: it is not ordered with the legacy default stream,
 * so a caller whose inputs are produced there (torch's default stream, an
 * NCCL receive that torch orders on it) passes cudaStreamLegacy. */
int adb_join_device(const char *algo, const adb_tuple *dR, uint64_t nR, const adb_tuple *dS,
                    uint64_t nS, const adb_join_params *p, adb_join_result *out, void *stream);

/* Materialising join (JOIN_RESULT_MATERIALIZE, hashing/joins/common_functions.cpp:255-258):
 * writes one <S-key, S-payload> tuple per match into dOut (device, capacity
 * `cap` tuples) in an unspecified order; out->materialized = matches written,
 * out->count = all matches (count > cap means the buffer was too small). */
int adb_join_materialize_device(const char *algo, const adb_tuple *dR, uint64_t nR,
                                const adb_tuple *dS, uint64_t nS, const adb_join_params *p,
                                adb_tuple *dOut, uint64_t cap, adb_join_result *out, void *stream);

/* ---------------------------------------------------------------------- */
/* Eager stream joins (SHJ_* / PMJ_*) over tumbling windows.              */
/* ---------------------------------------------------------------------- */

/* Per-window result of a windowed stream join. */
typedef struct adb_window_result {
    uint64_t window_start_ms;
    uint64_t n_r, n_s;
    uint64_t count, checksum;
    float latency_ms;           /* realtime: close of the window -> result on the host (wall clock);
                                   per-batch form: the last batch -> result (device clock);
                                   throughput form: the window's whole device time (table
                                   reset, joins, result copy) */
    float reserved;
} adb_window_result;

/* Join two timestamp-ordered streams in tumbling windows of p->window_size
 * ms.  Tuples are fed to the device in arrival micro-batches of
 * p->batch_tuples (default: one millisecond of stream) and each batch is
 * joined on arrival against the window's device-resident state (eager
 * join).  Writes up to max_windows results; *n_windows = windows seen.
 * Streams that are not ordered by ts_ms are refused with ADB_ERR_ARG: up to
 * 2^16 tuples per side before the device is touched, longer ones on their
 * device copies (in the throughput form on pinned streams window by window,
 * as each window's tuples arrive while the window before it is joined;
 * results written before the refusal are then not valid). */
int adb_stream_join(const char *algo, const adb_stream_tuple *R, uint64_t nR,
                    const adb_stream_tuple *S, uint64_t nS, const adb_join_params *p,
                    adb_window_result *windows, uint64_t max_windows, uint64_t *n_windows);

/* Progressiveness of one window: the reference's progressive measurement
 * (END_PROGRESSIVE_MEASURE samples every gap-th match with its time and the
 * probing tuple, hashing/timer/t_timer.h:195-212; dump_timing reports the time
 * to 1..50 % of the results and the 95th / 99th tuple latency,
 * hashing/timer/t_timer.cpp:401-452), taken per arrival micro-batch on the
 * device clock.  t_pct[i] = ms from the release of the window's first batch
 * until the results of the batch that brings the window's matches to pct[i] %
 * of its total, pct = {1, 5, 10, 25, 50, 75, 95, 99, 100}; lat_* = percentiles,
 * weighted by each batch's matches, of the ms from a batch's release (its
 * start on the device; with p->realtime, the arrival of its last tuple) to its
 * results. */
typedef struct adb_window_progress {
    float t_pct[9];
    float lat_p50, lat_p95, lat_p99;
    uint32_t batches;
    uint32_t reserved;
} adb_window_progress;

/* adb_stream_join that also fills progress[w] (may be NULL) for the first
 * max_windows windows; each micro-batch adds two one-thread clock kernels. */
int adb_stream_join_progress(const char *algo, const adb_stream_tuple *R, uint64_t nR,
                             const adb_stream_tuple *S, uint64_t nS, const adb_join_params *p,
                             adb_window_result *windows, adb_window_progress *progress,
                             uint64_t max_windows, uint64_t *n_windows);

/* ---------------------------------------------------------------------- */
/* Batched windows: many independent R/S pairs joined in one launch.      */
/* ---------------------------------------------------------------------- */

/* Window w is R[r_off[w] .. r_off[w+1]) joined with S[s_off[w] .. s_off[w+1]),
 * all device-resident (offsets are host arrays of n_windows+1 entries).
 * mode 0 = one persistent launch sequence for all windows (work stealing over
 * (window, partition) items); mode 1 = one launch sequence per window. */
int adb_batch_join_device(const adb_tuple *dR, const uint64_t *r_off, const adb_tuple *dS,
                          const uint64_t *s_off, uint32_t n_windows, int mode,
                          uint64_t *counts, uint64_t *checksums, float *ms_device, void *stream);

/* Batched mode 0 partitions window w 2^b ways, b taken from a table indexed by
 * ceil(log2(max(|R_w|, |S_w|))).  adb_batch_autotune times b = default - 1,
 * default, default + 1 for the window sizes 2^lo .. 2^hi on seeded windows and
 * keeps the fastest; bits_out (33 entries, may be NULL) receives the table.
 * adb_batch_set_tuning installs a table (33 entries, -1 = built-in rule;
 * NULL restores the built-in rule for every size). */
int adb_batch_autotune(int lo, int hi, int *bits_out);
int adb_batch_set_tuning(const int *bits);

/* ---------------------------------------------------------------------- */
/* Serving: open-loop windowed-join requests with continuous batching.    */
/* ---------------------------------------------------------------------- */

/* One request: R = PK(n_r tuples, seed) and S = FK(n_s tuples drawn uniformly
 * from R's keys, seed + 1), as adb_gen_pk / adb_gen_fk define them, generated
 * on the device when the request is admitted.  arrival_us: offered arrival,
 * microseconds after the run starts (requests ordered by it). */
typedef struct adb_serve_request {
    uint64_t arrival_us;
    uint32_t n_r, n_s;
    uint64_t seed;
} adb_serve_request;

typedef struct adb_serve_result {
    uint64_t count, checksum;
    float latency_ms;           /* completion - arrival, wall clock */
    float queue_ms;             /* admission - arrival */
    uint32_t batch;             /* the device batch that served it */
    int32_t status;
} adb_serve_result;

typedef struct adb_serve_config {
    uint64_t budget_bytes;      /* device memory for requests in flight; 0 = half of the free memory */
    uint32_t max_batch;         /* most requests per batch; 0 = 256 */
    int32_t realtime;           /* 1 = admit each request at its arrival time; 0 = all arrived at t = 0 */
    uint32_t slots;             /* batches in flight at once (own stream + workspace each); 0 = 2 */
    uint32_t reserved;
} adb_serve_config;

typedef struct adb_serve_stats {
    uint64_t requests, tuples, batches;
    double makespan_ms;         /* run start -> last completion */
    double tuples_per_s;        /* input tuples of all requests / makespan */
    double p50_ms, p99_ms, p999_ms;
    double mean_batch;          /* requests per batch */
    uint64_t peak_arena_bytes, arena_bytes;
} adb_serve_stats;

/* Runs the serving loop over the n requests: arrived requests are admitted
 * while their inputs fit the device-memory budget (ADB_ERR_BUSY if one never
 * can), batched with whatever else has arrived, and joined by the batched
 * pipeline on one of `slots` concurrent slots.  res[i] receives request i's
 * result; stats (may be NULL) the throughput and latency percentiles. */
int adb_serve_run(const adb_serve_config *cfg, const adb_serve_request *req, uint32_t n,
                  adb_serve_result *res, adb_serve_stats *stats);

/* ---------------------------------------------------------------------- */
/* One join over several GPUs (one process per GPU).                      */
/* ---------------------------------------------------------------------- */

/* The split step of a sharded join (no counterpart in the reference, which
 * runs on one machine): groups the device relation dIn[0..n) by destination
 * rank into dOut (device, n tuples): the tuples of part p (p < parts <= 32)
 * are dOut[off_p .. off_p + counts[p]), off_p = counts[0] + .. + counts[p-1],
 * in no particular order; counts is a host array of `parts` entries.  The
 * destination of a key is (key * 0x9E3779B1 mod 2^32) * parts / 2^32.  After an
 * all-to-all of the parts, every rank holds all tuples of its keys from both
 * relations and joins them alone; the ranks' (count, checksum) pairs add up
 * (mod 2^64) to the join of the whole relations.  Synchronises `stream`
 * (NULL = the library stream) before it returns the counts. */
int adb_shard_split(const adb_tuple *dIn, uint64_t n, uint32_t parts, adb_tuple *dOut, uint64_t *counts,
                    void *stream);

/* ---------------------------------------------------------------------- */
/* Device memory helpers for callers without a CUDA runtime of their own. */
/* ---------------------------------------------------------------------- */
int adb_device_alloc(void **ptr, size_t bytes);
int adb_device_free(void *ptr);
int adb_host_alloc_pinned(void **ptr, size_t bytes);
int adb_host_free_pinned(void *ptr);
int adb_memcpy_h2d(void *dst, const void *src, size_t bytes);
int adb_memcpy_d2h(void *dst, const void *src, size_t bytes);
int adb_device_sync(void);
/* Releases the cached device workspace (it is re-created on the next join). */
int adb_release_workspace(void);

/* ---------------------------------------------------------------------- */
/* Allocation-free NPO join.                                              */
/* ---------------------------------------------------------------------- */

/* No counterpart in the reference: an extra entry point for callers that may
 * not allocate device memory while they run (an engine that budgets all of
 * HBM up front, a memory-capped sandbox, a pipeline that must never wait on an
 * allocator).  It computes exactly what adb_join("NPO", ...) computes, on
 * device-resident R and S, but its hash table lives in a fixed 32 MiB
 * __device__ array inside the library instead of allocated memory, so it
 * calls no cudaMalloc/cudaFree.  Limit: nR <= 2^21 build tuples (larger calls
 * return ADB_ERR_ARG), nS < 2^32.  d_out is a device array of two uint64:
 * count, checksum.  Runs on `stream` (a cudaStream_t, NULL = the default
 * stream) and returns without synchronising.  The first call on each device
 * looks up the array's device address (cudaGetSymbolAddress) and caches it;
 * make that first call before any stream capture.  The cached address does not
 * survive cudaDeviceReset: reload the library after a reset.  All calls on a device
 * share the one array: calls that overlap on the GPU race and must be
 * serialised by the caller. */
int adb_npo_join_noalloc(const adb_tuple *dR, uint64_t nR, const adb_tuple *dS, uint64_t nS,
                         uint64_t *d_out, void *stream);

/* ---------------------------------------------------------------------- */
/* Seeded synthetic relations (the generator of the benchmark configs).   */
/* Counter-based: element i depends only on (seed, i), so host and device */
/* produce identical arrays.  Arrays may be host or device pointers as    */
/* named.                                                                 */
/* ---------------------------------------------------------------------- */

/* R: key = 1 + perm_seed(i) (a permutation of 1..n), payload = i. */
int adb_gen_pk(adb_tuple *R, uint64_t n, uint64_t seed, int on_device);
/* S: payload = j, key = R.key[idx_j] with idx_j Zipf(theta) over 0..nR-1 through a
 * seeded rank permutation (theta = 0: uniform).  idx (may be NULL) receives idx_j. */
int adb_gen_fk(adb_tuple *S, uint64_t nS, const adb_tuple *R, uint64_t nR, double theta,
               uint64_t seed, uint32_t *idx, int on_device);
/* Non-unique: key = 1 + uniform(seed, i) % key_range, payload = i. */
int adb_gen_uniform(adb_tuple *T, uint64_t n, uint64_t key_range, uint64_t seed, int on_device);

/* ---------------------------------------------------------------------- */
/* Relations from text files (host only, no device needed).               */
/* ---------------------------------------------------------------------- */

/* Reads num_tuples records of the text file at path into tuples (and their
 * timestamps into ts, which may be NULL), as the reference's file loader does.
 * Replaces load_relation / read_relation (hashing/utils/generator.cpp:646-666,
 * :900-1027), called from createRelation (hashing/benchmark.cpp:80-83):
 * fields separated by the first ',' or '|' of the file, no header line, key =
 * integer field key_col, timestamp = integer field ts_col (milliseconds) times
 * 2.1e6 when ts_col != 0 (0 otherwise), runs of equal timestamps spread
 * linearly to the next one (smooth, :1050-1067), record i placed round-robin
 * into `partitions` contiguous ranges, payload = its index.  ADB_ERR_ARG when
 * the file cannot be read, has fewer than num_tuples records, or a record lacks
 * the fields (the reference's behaviour is undefined there). */
int adb_load_relation(const char *path, int32_t key_col, int32_t ts_col, uint32_t partitions,
                      uint64_t num_tuples, adb_tuple *tuples, uint64_t *ts);

#ifdef __cplusplus
}
#endif
#endif /* ADB_JOIN_H */
