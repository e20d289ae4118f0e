// reference_shim_sort.cpp -- the reference's sort-merge join functions, with
// their exact names and signatures, implemented on libadb_b200.so.
//
// The sorting/ counterpart of reference_shim.cpp: a maintainer adds this file
// to AllianceDB's sorting/ build in place of joins/sortmergejoin_multiway.cpp,
// joins/sortmergejoin_multipass.cpp, joins/sortmergejoin_multiway_skewhandling.cpp
// and joins/sortmergejoin_mpsm.cpp, and links libadb_b200.so.  It compiles
// against the reference's own sorting/ headers (include path: the sorting/
// directory) and the C ABI (include/adb/adb_join.h).
//
// Contract kept (sorting/joins/sortmergejoin_multiway.h:27,
// sortmergejoin_multipass.h:29, sortmergejoin_multiway_skewhandling.h:26,
// sortmergejoin_mpsm.h:25; table sorting/main.cpp:481-486, caller :752-758):
//   result_t *NAME(relation_t *relR, relation_t *relS, joinconfig_t *joincfg,
//                  int exp_id, int window_size, int gap)
//   * joincfg->PARTFANOUT becomes adb_join_params.part_fanout (the library's
//     partitioning fan-out); NTHREADS, the scalar/AVX switches, the merge
//     buffer size and the NUMA strategy select CPU code paths and have no
//     GPU counterpart; exp_id, window_size and gap only name the reference's
//     timing output;
//   * the callee mallocs the result_t, the caller frees it with free(); the
//     result heads a larger block that also carries the checksum
//     (adb_shim_sort_checksum reads it);
//   * result_t.totalresults = match count, resultlist = NULL;
//   * relR/relS are read only (the reference sorts and partitions copies, but
//     callers must not rely on either);
//   * unlike the reference, any thread count is accepted (the reference needs a
//     power of two, sortmergejoin_multiway.cpp:59) and |R| need not be a
//     multiple of it;
//   * on failure the shim prints the library's message to stderr and returns
//     NULL; mpsm is excluded in the reference (it prints "excluded" and exits,
//     sortmergejoin_mpsm.cpp:38-42) and returns NULL here.
#include <cstdio>
#include <cstdlib>

#include "joins/sortmergejoin_mpsm.h"
#include "joins/sortmergejoin_multipass.h"
#include "joins/sortmergejoin_multiway.h"
#include "joins/sortmergejoin_multiway_skewhandling.h"

#include "adb/adb_join.h"

static_assert(sizeof(tuple_t) == sizeof(adb_tuple), "tuple layout {payload @0, key @4}");

namespace {

struct ShimSortResult {
    result_t base;  // first member: free(result_t *) releases the whole block
    uint64_t checksum;
};

result_t *run(const char *name, const relation_t *R, const relation_t *S, const joinconfig_t *cfg) {
    adb_join_params p;
    adb_params_default(&p);
    if (cfg && cfg->PARTFANOUT > 0) p.part_fanout = cfg->PARTFANOUT;
    adb_join_result r;
    const int st = adb_join(name, reinterpret_cast<const adb_tuple *>(R->tuples), R->num_tuples,
                            reinterpret_cast<const adb_tuple *>(S->tuples), S->num_tuples, &p, &r);
    if (st != ADB_OK) {
        fprintf(stderr, "[adb] %s failed: %s\n", name, adb_last_error());
        return nullptr;
    }
    auto *out = static_cast<ShimSortResult *>(calloc(1, sizeof(ShimSortResult)));
    if (!out) return nullptr;
    out->base.totalresults = static_cast<int64_t>(r.count);
    out->base.resultlist = nullptr;
    out->base.nthreads = cfg ? cfg->NTHREADS : 1;
    out->checksum = r.checksum;
    return &out->base;
}

}  // namespace

// The checksum of a result returned by one of the functions below.
extern "C" uint64_t adb_shim_sort_checksum(const result_t *res) {
    return reinterpret_cast<const ShimSortResult *>(res)->checksum;
}

// sorting/main.cpp:481-486, the algos[] table
result_t *sortmergejoin_multiway(relation_t *relR, relation_t *relS, joinconfig_t *joincfg, int, int, int) {
    return run("m-way", relR, relS, joincfg);
}
result_t *sortmergejoin_multipass(relation_t *relR, relation_t *relS, joinconfig_t *joincfg, int, int, int) {
    return run("m-pass", relR, relS, joincfg);
}
result_t *sortmergejoin_multiway_skewhandling(relation_t *relR, relation_t *relS, joinconfig_t *joincfg, int, int,
                                              int) {
    return run("m-way+skew", relR, relS, joincfg);
}
result_t *sortmergejoin_mpsm(relation_t *relR, relation_t *relS, joinconfig_t *joincfg, int, int, int) {
    return run("mpsm", relR, relS, joincfg);
}
