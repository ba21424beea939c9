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

SOURCES = ["esr_host.cu", "esr_mesh.cpp", "esr_noalloc.cu", "esr_mlp.cu", "esr_faithful.cu"]
HEADERS = ["esr_device.cuh", "esr_internal.h", "esr_layout.h", "esr_mlp.cuh", "esr_faithful.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# per-source flags: the reference-fidelity kernels round every float32
# product and sum separately, as the reference's float32 arithmetic does
SOURCE_FLAGS = {"esr_faithful.cu": ["-fmad=false"]}
OBJ_DIR = PKG.parent / "_build"


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
    nvcc = nvcc_path()
    OBJ_DIR.mkdir(exist_ok=True)
    common = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3,-ffp-contract=off", "-I", str(INCLUDE)]
    # every translation unit compiles on its own (in parallel), then one link
    jobs, objs = [], []
    for src in SOURCES:
        path = CSRC / src
        if not path.exists():
            continue
        obj = OBJ_DIR / (path.stem + ".o")
        cmd = [nvcc, *common, *SOURCE_FLAGS.get(src, []), "-c", str(path), "-o", str(obj), *(extra or [])]
        if verbose:
            print(" ".join(cmd))
        jobs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
        objs.append(str(obj))
    for cmd, proc in jobs:
        out, err = proc.communicate()
        if proc.returncode != 0:
            raise RuntimeError(f"nvcc failed ({proc.returncode}): {' '.join(cmd)}\n{err[-8000:]}")
        if verbose and err:
            print(err[-4000:])
    link = [nvcc, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(LIB) + ".tmp", *objs]
    if verbose:
        print(" ".join(link))
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({r.returncode}):\n{r.stderr[-8000:]}")
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
    print(LIB)
