"""Build the in-tree native libraries.

libadb_b200.so   the CUDA join library (sm_100a only), from alliancedb_b200/csrc/*.cu
liboracle.so     the CPU checker used by tests (oracle/adb_oracle.c), built beside it

Run as ``python -m alliancedb_b200.build [AllianceDB source tree]`` (or with
ADB_REF_ROOT set) or through ``__graft_entry__.build()``; without a source
tree only the product library and the C restatement are built.
Objects go to _build/ (not committed); the shared libraries stay in the tree
so they travel with the repository snapshot.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "alliancedb_b200"
CSRC = PKG / "csrc"
BUILD = ROOT / "_build"
LIB = PKG / "libadb_b200.so"
ORACLE_LIB = ROOT / "oracle" / "liboracle.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
           "--expt-relaxed-constexpr", "-I", str(ROOT / "include")]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd)}")


def _newer(src: Path, dst: Path, deps: list[Path]) -> bool:
    if not dst.exists():
        return True
    t = dst.stat().st_mtime
    return src.stat().st_mtime > t or any(d.stat().st_mtime > t for d in deps)


def build_cuda(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    headers = sorted(CSRC.glob("*.cuh")) + sorted((ROOT / "include").rglob("*.h"))
    objs = []
    jobs = []
    for src in sources:
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if _newer(src, obj, headers):
            cmd = [NVCC, *ARCH, *NVFLAGS, "-c", str(src), "-o", str(obj)]
            if verbose:
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(_run, jobs))
    if jobs or not LIB.exists():
        tmp = LIB.with_suffix(".so.tmp")
        _run([NVCC, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lpthread"])
        os.replace(tmp, LIB)
    return LIB


def ref_root(explicit: str | None = None) -> Path | None:
    """The AllianceDB source tree (its hashing/ and sorting/ directories), from
    the argument or the ADB_REF_ROOT environment variable; None when neither
    names an existing directory (the reference builds are then skipped)."""
    r = explicit or os.environ.get("ADB_REF_ROOT")
    return Path(r) if r and (Path(r) / "hashing").is_dir() else None


def build_oracle(ref: Path | None = None) -> Path:
    """The CPU checker: the C restatement, and (when the AllianceDB sources are
    given) the reference's own joins under oracle/_ref/."""
    _run(["make", "-s", "-C", str(ROOT / "oracle"), "liboracle.so"])
    if ref is not None:
        _run(["make", "-s", "-j8", "-C", str(ROOT / "oracle"), "ref", "read", "ck", "wait", f"REF_ROOT={ref}"])
    return ORACLE_LIB


def build_shim(ref: Path | None = None) -> None:
    """oracle/_ref/adb_ref_bench_gpu: the reference-side shim (its join
    signatures on libadb_b200.so) under the test harness; needs the
    reference's headers, so only where its sources are given."""
    if ref is not None:
        _run(["make", "-s", "-C", str(ROOT / "oracle"), "shim", "shim-sort", f"REF_ROOT={ref}"])


def build_all(verbose: bool = False, ref: str | None = None) -> None:
    r = ref_root(ref)
    build_oracle(r)
    build_cuda(verbose)
    build_shim(r)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if a != "-v"]
    build_all(verbose="-v" in sys.argv, ref=args[0] if args else None)
    print(LIB)
