// loader.cu -- relations read from text files, the reference's file loader.
//
// Restates load_relation / read_relation / smooth
// (hashing/utils/generator.cpp:646-666, :900-1027, :1050-1067), which the
// reference's driver uses when a relation is given as a file
// (createRelation, hashing/benchmark.cpp:80-83):
//   * the field delimiter is the first ',' or '|' in the file (:918-936);
//   * every line is a record, from the first one on (the reference does not
//     skip a header), until num_tuples records are read (:979);
//   * key = std::stoi of field key_col (:981, :990); timestamp = std::stol of
//     field ts_col times 2.1 and times 1E6 (milliseconds in ticks of a
//     2.1 GHz clock, :985, :994), converted to uint64;
//   * smooth: a run of equal timestamps is spread linearly up to the next
//     distinct timestamp, in double arithmetic; the last run stays (:1050-1067);
//   * record i goes to partition i % partitions, where partition p owns the
//     index range [p * q, (p + 1) * q), q = num_tuples / partitions, the last
//     partition up to num_tuples; a full partition's records go to the last
//     one (:1005-1021); payload = the record's index in the relation.
// Host code only: no device is needed.  Differences on inputs where the
// reference's behaviour is undefined: a file with fewer than num_tuples
// records, a missing field or a field that is not a number is an error
// (ADB_ERR_ARG) instead of uninitialised tuples or an uncaught exception;
// without a timestamp column (ts_col == 0) the timestamps are 0 instead of
// uninitialised memory.
#include <cerrno>
#include <climits>
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "engine.cuh"

namespace adb {

// Field `col` of a line split at `delim` (every delimiter starts a new field,
// empty fields included), or false when the line has fewer fields.
static bool field_of(const std::string &line, char delim, int32_t col, std::string *out) {
    size_t start = 0;
    for (int32_t f = 0; f < col; f++) {
        const size_t pos = line.find(delim, start);
        if (pos == std::string::npos) return false;
        start = pos + 1;
    }
    const size_t end = line.find(delim, start);
    *out = line.substr(start, end == std::string::npos ? std::string::npos : end - start);
    return true;
}

// std::stol / std::stoi semantics: leading white space, optional sign, base-10
// digits, anything after them ignored; false when no digit is read or the
// value is out of range of the target type.
static bool parse_long(const std::string &s, long lo, long hi, long *v) {
    errno = 0;
    char *end = nullptr;
    const long x = std::strtol(s.c_str(), &end, 10);
    if (end == s.c_str() || errno == ERANGE || x < lo || x > hi) return false;
    *v = x;
    return true;
}

// The reference's smooth(): a maximal run ts[b, i) of equal values that is
// followed by a different value ts[i] is spread towards it: ts[b + k] becomes
// (uint64)((double)ts[b + k] + k * d) with d = (double)(ts[i] - ts[b]) / len,
// the difference taken in uint64 and the run length an int.  The k = 0 term
// is kept: above 2^53 the round trip through double changes the value.  A
// run at the end of the array stays as it is.
static void smooth_ts(uint64_t *ts, uint64_t n) {
    uint64_t b = 0;                      // start of the current run
    for (uint64_t i = 1; i < n; i++) {
        if (ts[i] == ts[b]) continue;
        const int len = (int)(i - b);
        const double d = (double)(ts[i] - ts[b]) / (double)len;
        for (int k = 0; k < len; k++) ts[b + k] = (uint64_t)((double)ts[b + k] + k * d);
        b = i;
    }
}

static int load_relation(const char *path, int32_t key_col, int32_t ts_col, uint32_t partitions,
                         uint64_t num_tuples, adb_tuple *tuples, uint64_t *ts) {
    if (!path || !tuples || key_col < 0 || ts_col < 0 || partitions == 0) {
        set_error("adb_load_relation: path and tuples must be given, columns >= 0, partitions >= 1");
        return ADB_ERR_ARG;
    }
    if (num_tuples / partitions > (uint64_t)INT_MAX) {
        set_error("adb_load_relation: num_tuples / partitions must fit an int (the reference's per-thread count)");
        return ADB_ERR_ARG;
    }
    std::ifstream in(path, std::ios::binary);
    if (!in.is_open()) {
        set_error("adb_load_relation: cannot open %s", path);
        return ADB_ERR_ARG;
    }
    char delim = 0;
    for (char c; !delim && in.get(c);)
        if (c == ',' || c == '|') delim = c;
    if (!delim) {
        set_error("adb_load_relation: %s has neither ',' nor '|' fields", path);
        return ADB_ERR_ARG;
    }
    in.clear();
    in.seekg(0);

    std::vector<uint32_t> key(num_tuples);
    std::vector<uint64_t> ret(num_tuples, 0);
    std::string line, fld;
    uint64_t i = 0;
    while (i < num_tuples && std::getline(in, line)) {
        long v;
        if (!field_of(line, delim, key_col, &fld) || !parse_long(fld, INT_MIN, INT_MAX, &v)) {
            set_error("adb_load_relation: record %llu of %s has no integer field %d", (unsigned long long)i, path,
                      key_col);
            return ADB_ERR_ARG;
        }
        key[i] = (uint32_t)(int32_t)v;
        if (ts_col != 0) {
            if (!field_of(line, delim, ts_col, &fld) || !parse_long(fld, LONG_MIN, LONG_MAX, &v) || v < 0) {
                set_error("adb_load_relation: record %llu of %s has no non-negative integer field %d",
                          (unsigned long long)i, path, ts_col);
                return ADB_ERR_ARG;
            }
            ret[i] = (uint64_t)((double)v * 2.1 * 1E6);
        }
        i++;
    }
    if (i < num_tuples) {
        set_error("adb_load_relation: %s holds %llu records, fewer than the %llu asked for", path,
                  (unsigned long long)i, (unsigned long long)num_tuples);
        return ADB_ERR_ARG;
    }
    smooth_ts(ret.data(), num_tuples);

    const uint64_t q = num_tuples / partitions;
    std::vector<uint64_t> fill(partitions, 0);
    for (uint64_t r = 0; r < num_tuples; r++) {
        uint32_t p = (uint32_t)(r % partitions);
        const uint64_t start = q * p, end = p + 1 == partitions ? num_tuples : q * (p + 1);
        if (start + fill[p] == end) p = partitions - 1;   // full: to the last partition
        const uint64_t at = q * p + fill[p]++;
        tuples[at].payload = (uint32_t)at;
        tuples[at].key = key[r];
        if (ts) ts[at] = ret[r];
    }
    return ADB_OK;
}

}  // namespace adb

extern "C" int adb_load_relation(const char *path, int32_t key_col, int32_t ts_col, uint32_t partitions,
                                 uint64_t num_tuples, adb_tuple *tuples, uint64_t *ts) {
    return adb::load_relation(path, key_col, ts_col, partitions, num_tuples, tuples, ts);
}
