// reference_shim.cpp -- the reference's join functions, with their exact names
// and signatures, implemented on libadb_b200.so.
//
// This file is the reference-side binding: a maintainer adds it to AllianceDB's
// hashing/ build in place of joins/parallel_radix_join.cpp,
// joins/no_partitioning_join.cpp and joins/onlinejoins.cpp, and links
// libadb_b200.so.  It compiles against the reference's own headers (include
// path: the hashing/ directory) and the C ABI (include/adb/adb_join.h).
//
// Contract kept (hashing/joins/parallel_radix_join.h:37-85,
// no_partitioning_join.h, onlinejoins.h:33-213; caller hashing/benchmark.cpp:244-256):
//   result_t *NAME(relation_t *relR, relation_t *relS, param_t cmd_params)
//   * the callee mallocs the result_t and the caller frees it with free(); the
//     result is the head of a larger malloc'd block that also carries the
//     checksum (adb_shim_checksum reads it);
//   * result_t.totalresults = match count; resultlist is NULL (the reference
//     leaves it unset without JOIN_RESULT_MATERIALIZE);
//   * relR/relS are read only (the reference's PRO overwrites them,
//     parallel_radix_join.cpp:1176-1181; nothing may rely on that);
//   * on failure the reference calls exit() or returns NULL; the shim prints
//     the library's message to stderr and returns NULL.
// The eager joins (SHJ_*, PMJ_*) take the tuples in array order as their arrival
// order; the per-window stream form with timestamps is adb_stream_join.
#include <cstdio>
#include <cstdlib>

#include "joins/no_partitioning_join.h"
#include "joins/onlinejoins.h"
#include "joins/parallel_radix_join.h"

#include "adb/adb_join.h"

static_assert(sizeof(tuple_t) == sizeof(adb_tuple), "tuple layout {payload @0, key @4}");

namespace {

struct ShimResult {
    result_t base;  // first member: free(result_t *) releases the whole block
    uint64_t checksum;
};

result_t *run(const char *name, const relation_t *R, const relation_t *S, const param_t &cp) {
    adb_join_params p;
    adb_params_default(&p);
    if (cp.nthreads) p.nthreads = cp.nthreads;
    if (cp.window_size) p.window_size = cp.window_size;
    if (cp.step_sizeR) p.step_size_r = cp.step_sizeR;
    if (cp.step_sizeS) p.step_size_s = cp.step_sizeS;
    if (cp.interval) p.interval = cp.interval;
    if (cp.group_size) p.group_size = cp.group_size;
    if (cp.progressive_step) p.progressive_step = cp.progressive_step;
    if (cp.merge_step) p.merge_step = cp.merge_step;
    adb_join_result r;
    const int st = adb_join(name, reinterpret_cast<const adb_tuple *>(R->tuples), R->num_tuples,
                            reinterpret_cast<const adb_tuple *>(S->tuples), S->num_tuples, &p, &r);
    if (st != ADB_OK) {
        fprintf(stderr, "[adb] %s failed: %s\n", name, adb_last_error());
        return nullptr;
    }
    auto *out = static_cast<ShimResult *>(calloc(1, sizeof(ShimResult)));
    if (!out) return nullptr;
    out->base.totalresults = static_cast<int64_t>(r.count);
    out->base.resultlist = nullptr;
    out->base.nthreads = static_cast<int>(cp.nthreads);
    out->checksum = r.checksum;
    return &out->base;
}

}  // namespace

// The checksum of a result returned by one of the functions below.
extern "C" uint64_t adb_shim_checksum(const result_t *res) {
    return reinterpret_cast<const ShimResult *>(res)->checksum;
}

#define ADB_SHIM_JOIN(NAME) \
    result_t *NAME(relation_t *relR, relation_t *relS, param_t cmd_params) { return run(#NAME, relR, relS, cmd_params); }

// hashing/main.cpp:306-338, the algos[] table
ADB_SHIM_JOIN(PRO)
ADB_SHIM_JOIN(RJ_st)
ADB_SHIM_JOIN(PRH)
ADB_SHIM_JOIN(PRHO)
ADB_SHIM_JOIN(NPO)
ADB_SHIM_JOIN(NPO_st)
ADB_SHIM_JOIN(SHJ_st)
ADB_SHIM_JOIN(SHJ_JM_P)
ADB_SHIM_JOIN(SHJ_JM_NP)
ADB_SHIM_JOIN(SHJ_JB_NP)
ADB_SHIM_JOIN(SHJ_JBCR_NP)
ADB_SHIM_JOIN(SHJ_JBCR_P)
ADB_SHIM_JOIN(SHJ_HS_NP)
ADB_SHIM_JOIN(PMJ_st)
ADB_SHIM_JOIN(PMJ_JM_NP)
ADB_SHIM_JOIN(PMJ_JM_P)
ADB_SHIM_JOIN(PMJ_JB_NP)
ADB_SHIM_JOIN(PMJ_JB_P)
ADB_SHIM_JOIN(PMJ_JBCR_NP)
ADB_SHIM_JOIN(PMJ_JBCR_P)
ADB_SHIM_JOIN(PMJ_HS_NP)
// ripple joins are unfinished in the reference (hashing/main.cpp:331); the
// library reports them as unsupported and these return NULL
ADB_SHIM_JOIN(RPJ_st)
ADB_SHIM_JOIN(RPJ_JM_NP)
ADB_SHIM_JOIN(RPJ_JB_NP)
ADB_SHIM_JOIN(RPJ_JBCR_NP)
ADB_SHIM_JOIN(RPJ_HS_NP)
