// batch.cu -- batched windows.
#include "joins.cuh"

extern "C" int adb_batch_join_device(const adb_tuple *, const uint64_t *, const adb_tuple *, const uint64_t *,
                                     uint32_t, int, uint64_t *, uint64_t *, float *, void *) {
    adb::set_error("batched windows are not built yet");
    return ADB_ERR_UNSUPPORTED;
}
