"""Compile the native library (``libeulersr.so``) in-tree for sm_100a.

``python -m eulersr_b200._build`` (or ``__graft_entry__.build()``) runs nvcc on
the sources under ``csrc/``; the library is rebuilt only when a source is
newer than it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libeulersr.so"

SOURCES = ["esr_host.cu", "esr_mesh.cpp", "esr_noalloc.cu", "esr_mlp.cu"]
HEADERS = ["esr_device.cuh", "esr_internal.h", "esr_layout.h", "esr_mlp.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libeulersr.so")


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    files = [CSRC / s for s in SOURCES + HEADERS if (CSRC / s).exists()] + [INCLUDE / "eulersr.h", Path(__file__)]
    return any(f.stat().st_mtime > t for f in files)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    if not force and not _stale():
        return LIB
    srcs = [str(CSRC / s) for s in SOURCES if (CSRC / s).exists()]
    cmd = [nvcc_path(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-O3",
           "-I", str(INCLUDE), "-o", str(LIB) + ".tmp", *srcs, *(extra or [])]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed ({r.returncode}):\n{r.stderr[-8000:]}")
    if verbose and r.stderr:
        print(r.stderr[-4000:])
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
    print(LIB)
