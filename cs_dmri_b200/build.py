"""Build recipe for libcsdshore.so, the B200 SHORE fit library.

Compiles the CUDA sources under csrc/ for sm_100a only into an in-tree shared
library with a plain C ABI (include/csd_shore.h).  Run as
``python -m cs_dmri_b200.build`` or through ``__graft_entry__.build()``.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
LIB = HERE / "libcsdshore.so"
SOURCES = [HERE / "csrc" / "csd_shore.cu"]
PEAK_LIB = HERE / "libcsdpeak.so"
PEAK_SOURCES = [HERE / "csrc" / "peak_fp64.cu"]
DEPS = sorted((HERE / "csrc").glob("*.cuh")) + [ROOT / "include" / "csd_shore.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared", "-cudart", "static",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libcsdshore.so")
    return cand


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in SOURCES + DEPS)


def _compile(out: Path, sources: list[Path], verbose: bool, extra: list[str] | None) -> None:
    cmd = [nvcc(), *NVCC_FLAGS, *(extra or []), "-o", str(out), *map(str, sources)]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr:
        print(res.stderr, file=sys.stderr)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    if force or stale():
        _compile(LIB, SOURCES, verbose, extra)
    if force or not PEAK_LIB.exists() or PEAK_SOURCES[0].stat().st_mtime > PEAK_LIB.stat().st_mtime:
        _compile(PEAK_LIB, PEAK_SOURCES, verbose, None)
    return LIB


if __name__ == "__main__":
    force = "--force" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else None
    print(build(force=force, verbose=True, extra=extra))
