/*
 * checksum.h -- TEST INFRASTRUCTURE ONLY: force-included (g++ -include) into
 * the reference sources that oracle/ref/ref_tree.py prepared, whose match sites
 * call ADB_REF_MATCH(key, r_payload, s_payload) next to their match counter.
 *
 * The checksum is the library's result contract:
 *     a = (u64)key << 32 | r_payload,  b = (u64)s_payload << 32 | key,
 *     H = fmix64(a ^ fmix64(b)),  checksum = sum of H mod 2^64,
 * fmix64 being the SplitMix64 finalizer (Steele, Lea, Flood 2014).
 *
 * Each thread adds into its own accumulator (no shared cache line on the match
 * path); a thread's accumulator is added to adb_ref_checksum_total when the
 * thread exits, so after the reference has joined its worker threads the
 * call's checksum is adb_ref_checksum_total plus the calling thread's own
 * accumulator (the single-threaded joins run on the calling thread).
 *
 * With ADB_REF_NO_CK defined the sites compile to nothing (the build that the
 * CPU baseline times).
 */
#ifndef ADB_REF_CHECKSUM_H
#define ADB_REF_CHECKSUM_H

#include <stdint.h>

#if defined(__cplusplus) && defined(ADB_REF_NO_CK)
/* timing build: the match sites compile to the reference's code alone */
#define ADB_REF_MATCH(key, rp, sp) ((void)0)
static bool adb_ref_probe_r;
#elif defined(__cplusplus)
struct AdbRefAcc {
    uint64_t sum = 0;
    ~AdbRefAcc();
};
extern thread_local AdbRefAcc adb_ref_acc;
extern thread_local bool adb_ref_probe_r;   /* PMJ: the tuple of the current sweepArea::query is R */
extern uint64_t adb_ref_checksum_total;

static inline uint64_t adb_ref_fmix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

static inline uint64_t adb_ref_pair_hash(uint32_t key, uint32_t r_payload, uint32_t s_payload) {
    const uint64_t a = ((uint64_t)key << 32) | r_payload;
    const uint64_t b = ((uint64_t)s_payload << 32) | key;
    return adb_ref_fmix64(a ^ adb_ref_fmix64(b));
}

#define ADB_REF_MATCH(key, rp, sp) \
    (adb_ref_acc.sum += adb_ref_pair_hash((uint32_t)(key), (uint32_t)(rp), (uint32_t)(sp)))
#endif

#endif
