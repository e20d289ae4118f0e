// eager.cu -- eager stream joins (SHJ_*, PMJ_*).
#include "joins.cuh"

namespace adb {
size_t eager_scratch(uint64_t, uint64_t, Family, uint64_t) { return 0; }
int run_eager(Context *, const DevJoin &, Family, int, uint64_t, int, int, int, uint64_t, unsigned long long *) {
    set_error("eager joins are not built yet");
    return ADB_ERR_UNSUPPORTED;
}
int eager_set_attrs() { return ADB_OK; }
}  // namespace adb

extern "C" int adb_stream_join(const char *, const adb_stream_tuple *, uint64_t, const adb_stream_tuple *, uint64_t,
                               const adb_join_params *, adb_window_result *, uint64_t, uint64_t *) {
    adb::set_error("stream joins are not built yet");
    return ADB_ERR_UNSUPPORTED;
}
