"""Builds the in-tree CUDA library implexity_b200/liblbm_b200.so for sm_100a.

Run as ``python -m implexity_b200.build`` (or through ``__graft_entry__.build``).
nvcc cross-compiles without a GPU; the objects are rebuilt only when a
source or header is newer than the library.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "liblbm_b200.so"
MMA_LIB = PKG / "libmma_cpu.so"
MMA_SOURCE = CSRC / "mma_cpu.cpp"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden"]
SOURCES = ["lbm_forward.cu", "lbm_adjoint.cu", "lbm_misc.cu", "lbm_noalloc.cu", "lbm_runtime.cpp"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build liblbm_b200.so")


def _inputs() -> list[Path]:
    files = [CSRC / s for s in SOURCES]
    files += sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))
    return files


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(f.stat().st_mtime <= t for f in _inputs())


def host_cxx() -> str:
    """A host C++ compiler with OpenMP (the distribution g++ first)."""
    for cand in (os.environ.get("MMA_CXX"), "/usr/bin/g++", shutil.which("g++")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("g++ not found: a host C++ compiler with OpenMP is required to build libmma_cpu.so")


def build_mma(force: bool = False, verbose: bool = False) -> Path:
    """The host MMA library (include/mma_cpu.h): C++17 with OpenMP."""
    deps = [MMA_SOURCE, INCLUDE / "mma_cpu.h"]
    if not force and MMA_LIB.exists() and all(d.stat().st_mtime <= MMA_LIB.stat().st_mtime for d in deps):
        return MMA_LIB
    tmp = MMA_LIB.with_suffix(".so.tmp")
    cmd = [host_cxx(), "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-fvisibility=hidden", "-Wall",
           "-o", str(tmp), str(MMA_SOURCE)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, MMA_LIB)
    return MMA_LIB


def build(force: bool = False, verbose: bool = False) -> Path:
    build_mma(force, verbose)
    if not force and up_to_date():
        return LIB
    BUILD.mkdir(exist_ok=True)
    cc = nvcc()

    headers = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))

    def compile_one(src: str) -> Path:
        obj = BUILD / (src + ".o")
        deps = [CSRC / src, *headers]
        if not force and obj.exists() and all(d.stat().st_mtime <= obj.stat().st_mtime for d in deps):
            return obj
        cmd = [cc, *ARCH, *FLAGS, "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        return obj

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [cc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
