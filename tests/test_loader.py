"""File loader (adb_load_relation) against the reference's own loader.

The fixtures under tests/golden/loader/ hold seeded text files and the
tuples and timestamps that load_relation / read_relation / smooth
(hashing/utils/generator.cpp:646-666, :900-1067), compiled from the reference's
sources, produced for them (tests/golden/make_loader_golden.py).  The loader is
host code: these tests need no GPU.
"""
import json
from pathlib import Path

import numpy as np
import pytest

import alliancedb_b200 as adb

GOLD = Path(__file__).resolve().parent / "golden" / "loader"
CASES = json.loads((GOLD / "cases.json").read_text())


@pytest.mark.parametrize("name", sorted(CASES))
def test_matches_reference_loader(name):
    c = CASES[name]
    want = np.load(GOLD / f"{name}.npy")
    t, ts = adb.load_relation(GOLD / f"{name}.txt", c["rows"], c["key_col"], c["ts_col"], c["partitions"])
    assert np.array_equal(t["payload"], want["payload"])
    assert np.array_equal(t["key"], want["key"])
    if c["ts_col"]:
        assert np.array_equal(ts, want["ts"])   # smoothing in the reference's double arithmetic, bit for bit
    else:
        assert not ts.any()


def test_fewer_rows_than_asked(tmp_path):
    p = tmp_path / "r.csv"
    p.write_text("1,10\n2,11\n")
    with pytest.raises(RuntimeError, match="fewer"):
        adb.load_relation(p, 3, 0, 1)
    t, _ = adb.load_relation(p, 2, 0, 1)      # extra lines beyond num_tuples are ignored
    assert list(t["key"]) == [1, 2]


@pytest.mark.parametrize("text", ["key,ts\n1,10\n", "1,10\n2\n", "1 10\n2 11\n"])
def test_bad_records_are_errors(tmp_path, text):
    """A header line, a missing field or no ',' / '|' separator: the reference's
    behaviour is undefined there (uncaught exception, out-of-range access)."""
    p = tmp_path / "r.txt"
    p.write_text(text)
    with pytest.raises(RuntimeError):
        adb.load_relation(p, 2, 0, 1)


def test_missing_file(tmp_path):
    with pytest.raises(RuntimeError, match="cannot open"):
        adb.load_relation(tmp_path / "none.csv", 1)
