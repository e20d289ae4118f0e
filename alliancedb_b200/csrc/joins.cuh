// joins.cuh -- device-resident join drivers shared by the C ABI and the
// batched/served paths.  Each driver: scratch size for a call, then the
// launch sequence on ctx->stream.  Results land in acc[0] (count) and acc[1]
// (checksum) of a device accumulator the caller zeroed; acc[2] is the error
// word (a timed-out device wait sets it), acc[3] the materialised count.
#pragma once

#include "engine.cuh"

namespace adb {

struct DevJoin {
    const uint64_t *R;
    uint64_t nR;
    const uint64_t *S;
    uint64_t nS;
    uint64_t *mat = nullptr;      // optional <S-key, S-payload> output
    uint64_t mat_cap = 0;
    int test_flags = 0;           // adb_join_params.test_flags
};

struct JoinTimes {
    float ms[4] = {0, 0, 0, 0};
};

enum class Family { Radix, RadixHist, Npo, SortMerge, Shj, Pmj, Unsupported };

// ---- paged partitioning front end (radix and sort-merge joins), paged.cuh ----
struct PartOut;
struct DigitFn;
size_t paged_partition_scratch(uint64_t nR, uint64_t nS, uint32_t b1, uint32_t b2, int num_sms);
uint64_t paged_final_pool_pages(uint64_t nR, uint64_t nS, uint32_t b1, uint32_t b2, int num_sms);
int run_paged_partition(Context *ctx, const DevJoin &j, DigitFn d1, const DigitFn *d2, PartOut *out,
                        unsigned long long *acc);

// ---- radix (PRO / RJ_st / PRH / PRHO) ----
int radix_bits_for(uint64_t nR, int requested);
size_t radix_scratch(uint64_t nR, uint64_t nS, int bits, int num_sms);
int run_radix(Context *ctx, const DevJoin &j, bool hist_table, int bits, unsigned long long *acc);

// ---- NPO / NPO_st ----
uint32_t npo_region_bits(uint64_t nR, int requested);
size_t npo_scratch(uint64_t nR, uint64_t nS, int region_bits, int num_sms);
int run_npo(Context *ctx, const DevJoin &j, int region_bits, unsigned long long *acc);

// ---- m-way / m-pass ----
size_t smj_scratch(uint64_t nR, uint64_t nS, int part_fanout, int num_sms);
int run_smj(Context *ctx, const DevJoin &j, int part_fanout, bool multipass, unsigned long long *acc);

// ---- eager SHJ / PMJ over one window given as arrival-ordered relations ----
size_t eager_scratch(uint64_t nR, uint64_t nS, Family fam, int model, int nthreads, int group_size);
int run_eager(Context *ctx, const DevJoin &j, Family fam, int model, uint64_t batch, int nthreads,
              int group_size, int progressive_step, uint64_t seed, unsigned long long *acc);
int stream_join(Context *ctx, Family fam, int model, const adb_stream_tuple *R, uint64_t nR,
                const adb_stream_tuple *S, uint64_t nS, const adb_join_params *p, adb_window_result *out,
                adb_window_progress *progress, uint64_t max_windows, uint64_t *n_windows);

}  // namespace adb
