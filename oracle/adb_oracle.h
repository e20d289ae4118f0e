/*
 * adb_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, single-threaded restatement of the AllianceDB join algorithms that
 * the GPU library replaces.  It exists to check the GPU results: only tests,
 * the smoke check and the CPU-baseline leg of bench.py load it.  Nothing in the
 * product library links, includes or calls this file.
 *
 * Every join returns the match count and the order-independent 64-bit checksum
 *     checksum = sum over matched (r, s) of H(key, r.payload, s.payload) mod 2^64
 *     a = (u64)key << 32 | r_payload,  b = (u64)s_payload << 32 | key,
 *     H = fmix(a ^ fmix(b)),  fmix = SplitMix64 finalizer (Steele, Lea, Flood 2014).
 * The reference itself returns only the count (hashing/utils/types.h:98-102);
 * the checksum is added at each of its match sites.
 */
#ifndef ADB_ORACLE_H
#define ADB_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* hashing/utils/types.h:67-70: {payloadID @0, key @4}, 8 bytes */
typedef struct { uint32_t payload; uint32_t key; } ora_tuple;
typedef struct { uint64_t count; uint64_t checksum; } ora_result;

uint64_t ora_fmix64(uint64_t z);
uint64_t ora_pair_hash(uint32_t key, uint32_t r_payload, uint32_t s_payload);

/* PRO / RJ_st: two-pass radix clustering + bucket-chaining join. */
int ora_pro(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS,
            int num_radix_bits, ora_result *out);
/* PRH: radix clustering + histogram (reorder) join. */
int ora_prh(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS,
            int num_radix_bits, ora_result *out);
/* NPO / NPO_st: one bucket-chained hash table of 2-tuple buckets. */
int ora_npo(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS, ora_result *out);
/* m-way / m-pass: sort both relations by the 64-bit word, then merge_join. */
int ora_smj(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS, ora_result *out);
/* SHJ_*: symmetric hash join, R and S tuples interleaved one at a time. */
int ora_shj(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS, ora_result *out);
/* PMJ_*: progressive merge join with runs of step_r / step_s tuples. */
int ora_pmj(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS,
            uint64_t step_r, uint64_t step_s, ora_result *out);
/* Independent truth: sort both by key, multiply run lengths, enumerate pairs. */
int ora_truth(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS, ora_result *out);

/* Truth for R with unique keys by direct addressing on the key (no
 * partitioning, hashing or sorting).  Returns -1 when R repeats a key, -2 when
 * R's largest key exceeds 8 |R| + 2^20 (no direct table), -3 out of memory. */
int ora_pk_truth(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS, ora_result *out);

/* Result materialisation: writes <S-key, S-payload> per match (the reference's
 * JOIN_RESULT_MATERIALIZE output), sorted as 64-bit words; returns the count. */
uint64_t ora_materialize_sorted(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS,
                                ora_tuple *out, uint64_t cap);

#ifdef __cplusplus
}
#endif
#endif
