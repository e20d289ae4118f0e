// read_harness.cpp -- TEST INFRASTRUCTURE ONLY.  Runs the reference's own file
// loader, load_relation / read_relation / smooth (hashing/utils/generator.cpp
// :646-666, :900-1067, compiled unmodified by oracle/Makefile), and writes what
// it produced, so tests/golden/make_loader_golden.py can pin the library's
// adb_load_relation against it.
//
// Usage: adb_ref_read <file> <key_col> <ts_col> <partitions> <num_tuples> <out.bin>
// out.bin: num_tuples 8-byte {payload, key} tuples, then num_tuples uint64
// timestamps (only meaningful when ts_col != 0; the reference leaves them
// unset otherwise).
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "utils/generator.h"
#include "utils/genzipf.h"

// symbols generator.cpp references for code paths the loader does not take
int get_cpu_id(int thread_id) { return thread_id; }
item_t *gen_zipf(unsigned int, unsigned int, double, item_t **) { return nullptr; }
int32_t *gen_zipf_ts(unsigned int, unsigned int, double) { return nullptr; }

int main(int argc, char **argv) {
    if (argc < 7) {
        fprintf(stderr, "usage: %s <file> <key_col> <ts_col> <partitions> <num_tuples> <out.bin>\n", argv[0]);
        return 2;
    }
    const uint64_t n = strtoull(argv[5], nullptr, 10);
    relation_t rel;
    relation_payload_t pl;
    memset(&rel, 0, sizeof rel);
    memset(&pl, 0, sizeof pl);
    pl.num_tuples = n;
    pl.ts = (uint64_t *)calloc(n ? n : 1, sizeof(uint64_t));
    if (load_relation(&rel, &pl, atoi(argv[2]), atoi(argv[3]), argv[1], n, (uint32_t)atoi(argv[4])) != 0) return 1;
    FILE *f = fopen(argv[6], "wb");
    if (!f) return 1;
    fwrite(rel.tuples, sizeof(tuple_t), n, f);
    fwrite(pl.ts, sizeof(uint64_t), n, f);
    fclose(f);
    return 0;
}
