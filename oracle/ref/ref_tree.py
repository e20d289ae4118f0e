"""TEST INFRASTRUCTURE ONLY: prepares the reference's own sources for the checker.

    python oracle/ref/ref_tree.py <AllianceDB source tree> <output dir> [--wait]

copies the reference's hashing/ and sorting/ directories into <output dir>
(oracle/_ref/src, git-ignored) and makes these edits in the copy, each found by
a pattern whose number of matches is checked, so a different reference version
fails here instead of building something else:

  build switches (the survey's recipe for running the reference on a machine
  without Intel PCM, NUMA libraries or the authors' /data1 directory)
    hashing/utils/perf_counters.h     PERF_COUNTERS off
    hashing/joins/common_functions.h  OVERVIEW, PROFILE_TOPDOWN, PROFILE_MEMORY_CONSUMPTION off;
                                      WAIT off (throughput; kept with --wait)
    sorting/joins/common_functions.h  TIMING -> NO_TIMING; the same three profiling switches off
    */cpu_mapping.cpp                 use every online CPU (the "/ 2" that assumes
                                      hyper-threads indexes out of range otherwise)
  checksum at the match sites (the reference returns only the count)
    hashing/joins/parallel_radix_join.cpp  bucket_chaining_join and histogram_join
    hashing/joins/common_functions.cpp     probe_hashtable_single (NPO, SHJ): the
                                           probe side is R when ISTupleR
    hashing/helper/pmj_helper.h            sweepArea::query (PMJ)
    hashing/helper/pmj_helper.cpp          each sweepArea::query call records which
                                           side probes (the call's ISTupleR argument is
                                           not reliable in earlyJoinMergedRuns)
    sorting/joins/common_functions.cpp     merge_join (m-way, m-pass)

Each checksum site calls ADB_REF_MATCH(key, r_payload, s_payload) from
oracle/ref/checksum.h, which the Makefile force-includes into every file.
"""
from __future__ import annotations

import re
import shutil
import sys
from pathlib import Path

PROFILING = r"^#define (OVERVIEW|PROFILE_TOPDOWN|PROFILE_MEMORY_CONSUMPTION)\b.*$"

# (file, regex, replacement, matches expected, index of the match to edit or None for all)
EDITS = [
    ("hashing/utils/perf_counters.h", r"^#define PERF_COUNTERS\s*$", "/* adb: PERF_COUNTERS off */", 1, None),
    ("hashing/joins/common_functions.h", PROFILING, r"/* adb: \1 off */", 3, None),
    ("hashing/utils/cpu_mapping.cpp", r"sysconf\(_SC_NPROCESSORS_ONLN\) */ *2", "sysconf(_SC_NPROCESSORS_ONLN)", 1, None),
    ("sorting/joins/common_functions.h", r"^#define TIMING\b.*$", "#define NO_TIMING", 1, None),
    ("sorting/joins/common_functions.h", PROFILING, r"/* adb: \1 off */", 3, None),
    ("sorting/affinity/cpu_mapping.cpp", r"sysconf\(_SC_NPROCESSORS_ONLN\) */ *2", "sysconf(_SC_NPROCESSORS_ONLN)", 1, None),
    # match sites
    ("hashing/joins/parallel_radix_join.cpp", r"^(\s*)matches\+\+;\s*$",
     r"\1matches++; ADB_REF_MATCH(Stuples[i].key, Rtuples[hit - 1].payloadID, Stuples[i].payloadID);", 1, None),
    ("hashing/joins/parallel_radix_join.cpp", r"^(\s*)\+\+match;\s*$",
     r"\1++match; ADB_REF_MATCH(Stuples[i].key, tmpRtuples[j].payloadID, Stuples[i].payloadID);", 1, None),
    ("hashing/joins/common_functions.cpp", r"^(\s*)\(\*matches\)\+\+;\s*$",
     r"\1(*matches)++; if (ISTupleR) ADB_REF_MATCH(tuple->key, tuple->payloadID, b->tuples[index_ht].payloadID); "
     r"else ADB_REF_MATCH(tuple->key, b->tuples[index_ht].payloadID, tuple->payloadID);", 2, 0),
    ("hashing/helper/pmj_helper.h", r"^(\s*)\(\*matches\)\+\+;\s*$",
     r"\1(*matches)++; if (adb_ref_probe_r) ADB_REF_MATCH(tuple->key, tuple->payloadID, (*it)->payloadID); "
     r"else ADB_REF_MATCH(tuple->key, (*it)->payloadID, tuple->payloadID);", 1, None),
    ("hashing/helper/pmj_helper.cpp", r"\bSM(\[[^\]]*\])?\.query\(", r"(adb_ref_probe_r = true, SM\1).query(", 2, None),
    ("hashing/helper/pmj_helper.cpp", r"\bRM(\[[^\]]*\])?\.query\(", r"(adb_ref_probe_r = false, RM\1).query(", 2, None),
    ("sorting/joins/common_functions.cpp", r"^(\s*)matches\+\+;\s*$",
     r"\1matches++; ADB_REF_MATCH(rtuples[i].key, rtuples[i].payloadID, stuples[jj].payloadID);", 2, 0),
]
WAIT_EDIT = ("hashing/joins/common_functions.h", r"^#define WAIT\b.*$", "/* adb: WAIT off */", 1, None)


def apply(root: Path, edit) -> None:
    rel, pat, rep, want, which = edit
    f = root / rel
    text = f.read_text()
    rx = re.compile(pat, re.M)
    found = list(rx.finditer(text))
    if len(found) != want:
        raise SystemExit(f"{rel}: pattern {pat!r} matched {len(found)} times, expected {want}")
    if which is None:
        text = rx.sub(rep, text)
    else:
        m = found[which]
        text = text[:m.start()] + m.expand(rep) + text[m.end():]
    f.write_text(text)


def main(argv: list[str]) -> int:
    if len(argv) < 3:
        print(__doc__)
        return 2
    src, out = Path(argv[1]), Path(argv[2])
    keep_wait = "--wait" in argv[3:]
    if out.exists():
        shutil.rmtree(out)
    out.mkdir(parents=True)
    for tree in ("hashing", "sorting"):
        shutil.copytree(src / tree, out / tree, ignore=shutil.ignore_patterns("scripts", "test", "*.cbp"))
    for e in EDITS + ([] if keep_wait else [WAIT_EDIT]):
        apply(out, e)
    (out / "READY").write_text("reference tree prepared by oracle/ref/ref_tree.py\n")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
