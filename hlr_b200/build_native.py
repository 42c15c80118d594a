"""Builds the in-tree native library ``hlr_b200/libhlrc.so`` for sm_100a.

The library holds the host construction (C++/OpenMP), the flattening
planner and the CUDA kernels behind the C ABI declared in ``include/hlrc.h``.
Objects go to ``hlr_b200/_build``; the shared object is written next to this
file so that it travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libhlrc.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("HLRC_CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# x86-64-v3 (AVX2/FMA): the library is built here and runs on the GPU host
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-march=x86-64-v3", "-Wall", "-Wno-unknown-pragmas"]
NVCCFLAGS = ["-O3", "-std=c++17", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-fopenmp", "--expt-relaxed-constexpr"]

CXX_SOURCES = ["common.cpp", "plan.cpp", "host/build.cpp"]
CU_SOURCES = ["hmvm.cu", "measure.cu", "build_gpu.cu"]


def _sources() -> list[Path]:
    files = [p for p in CSRC.rglob("*") if p.suffix in {".cpp", ".cu", ".hpp", ".cuh", ".h"}]
    files += list(INCLUDE.glob("*.h"))
    return files


def _stale(target: Path) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(p.stat().st_mtime > t for p in _sources())


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, file=sys.stderr)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    """Compile and link libhlrc.so if any source is newer than it."""
    if not force and not _stale(LIB):
        return LIB
    BUILD.mkdir(exist_ok=True)
    objs = []
    for src in CXX_SOURCES:
        obj = BUILD / (src.replace("/", "_") + ".o")
        _run([CXX, *CXXFLAGS, f"-I{INCLUDE}", f"-I{CSRC}", "-c", str(CSRC / src), "-o", str(obj)], verbose)
        objs.append(obj)
    for src in CU_SOURCES:
        obj = BUILD / (src.replace("/", "_") + ".o")
        extra = ["-Xptxas", "-v"] if ptxas_info else []
        _run([NVCC, *NVCCFLAGS, *extra, f"-I{INCLUDE}", f"-I{CSRC}", "-c", str(CSRC / src), "-o", str(obj)],
             verbose or ptxas_info)
        objs.append(obj)
    tmp = LIB.with_suffix(".so.tmp")
    _run([NVCC, "-shared", *ARCH, "-o", str(tmp), *map(str, objs), "-Xcompiler", "-fopenmp", "-lgomp"], verbose)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
