"""Golden fixtures of the file loader: seeded text files and what the
reference's own loader made of them.

Writes tests/golden/loader/<case>.txt (the input) and <case>.npy (a record
array of payload, key, ts) produced by oracle/_ref/adb_ref_read, which runs
load_relation / read_relation / smooth compiled unmodified from the AllianceDB
sources (hashing/utils/generator.cpp:646-666, :900-1067).  Run where those
sources are present, after `make -C oracle read`:

    python tests/golden/make_loader_golden.py

The inputs stand in for the reference's real datasets (not available): rows
of integer fields with a millisecond timestamp that repeats and sometimes
steps back, keys of both signs, blanks before numbers, ',' and '|' separators.
"""
from __future__ import annotations

import json
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "loader"
REF = HERE.parent.parent / "oracle" / "_ref" / "adb_ref_read"
REC = np.dtype([("payload", "<u4"), ("key", "<u4"), ("ts", "<u8")])

# name: (sep, rows, key_col, ts_col, partitions)
CASES = {
    "csv_key0_ts1": (",", 1000, 0, 1, 1),
    "bar_key2_ts1_p4": ("|", 1003, 2, 1, 4),
    "csv_keyonly_p3": (",", 777, 0, 0, 3),
    "csv_tiny_p4": (",", 10, 1, 2, 4),
    "csv_ts_steps_back": (",", 64, 0, 1, 2),
}


def rows_for(name: str, n: int, rng: np.random.Generator) -> list[list[str]]:
    ts = np.cumsum(rng.poisson(0.7, n)).astype(np.int64) + 1000
    if name == "csv_ts_steps_back":
        ts = ts - 3 * (np.arange(n) % 7 == 6)   # every seventh row steps back
    keys = rng.integers(-2**31, 2**31, n, dtype=np.int64)
    out = []
    for i in range(n):
        k = f" {keys[i]}" if i % 5 == 0 else str(keys[i])
        if name == "bar_key2_ts1_p4":
            out.append([str(i), str(ts[i]), k, str(rng.integers(0, 1000))])
        elif name == "csv_keyonly_p3":
            out.append([k, f"name{i}"])
        elif name == "csv_tiny_p4":
            out.append([str(i), k, str(ts[i])])
        else:
            out.append([k, str(ts[i]), "x"])
    return out


def main() -> None:
    OUT.mkdir(exist_ok=True)
    meta = {}
    for idx, (name, (sep, n, kc, tc, parts)) in enumerate(CASES.items()):
        rng = np.random.default_rng(100 + idx)
        text = "\n".join(sep.join(r) for r in rows_for(name, n, rng)) + "\n"
        src = OUT / f"{name}.txt"
        src.write_text(text)
        with tempfile.TemporaryDirectory() as d:
            binf = Path(d) / "out.bin"
            subprocess.run([str(REF), str(src), str(kc), str(tc), str(parts), str(n), str(binf)], check=True,
                           stdout=subprocess.DEVNULL)
            raw = binf.read_bytes()
        tup = np.frombuffer(raw[: 8 * n], dtype=[("payload", "<u4"), ("key", "<u4")])
        ts = np.frombuffer(raw[8 * n:], dtype="<u8")
        rec = np.empty(n, REC)
        rec["payload"], rec["key"] = tup["payload"], tup["key"]
        rec["ts"] = ts if tc else 0          # the reference leaves them unset without a ts column
        np.save(OUT / f"{name}.npy", rec)
        meta[name] = {"rows": n, "key_col": kc, "ts_col": tc, "partitions": parts}
    (OUT / "cases.json").write_text(json.dumps(meta, indent=1) + "\n")


if __name__ == "__main__":
    main()
