// smj.cu -- sort-merge joins (m-way, m-pass, m-way+skew).
#include "joins.cuh"

namespace adb {
size_t smj_scratch(uint64_t, uint64_t, int) { return 0; }
int run_smj(Context *, const DevJoin &, int, bool, unsigned long long *) {
    set_error("m-way is not built yet");
    return ADB_ERR_UNSUPPORTED;
}
int smj_set_attrs() { return ADB_OK; }
}  // namespace adb
