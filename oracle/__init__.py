"""ORACLE — test infrastructure only (see oracle.c's header).

Only ``tests/``, ``__graft_entry__.smoke()`` (as the checker) and ``bench.py``'s
CPU-baseline / reference arm import this package.  The product package
``hlr_b200`` never does.

Builds ``oracle/liboracle.so`` from ``oracle.c`` with gcc + OpenMP and
exposes the restated HLR CPU products on the descriptors of ``include/hlrc.h``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
SRC = HERE / "oracle.c"
LIB = HERE / "liboracle.so"
CFLAGS = ["-O3", "-fPIC", "-fopenmp", "-march=x86-64-v3", "-std=c11", "-Wall", "-shared"]

_lib = None


def build(force: bool = False) -> Path:
    if force or not LIB.exists() or LIB.stat().st_mtime < max(SRC.stat().st_mtime,
                                                              (ROOT / "include" / "hlrc.h").stat().st_mtime):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [os.environ.get("HLRC_CC", "gcc"), *CFLAGS, f"-I{ROOT / 'include'}", str(SRC), "-o", str(tmp), "-lm"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"oracle build failed: {' '.join(cmd)}\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        vp, i64, f64, ci = C.c_void_p, C.c_int64, C.c_double, C.c_int
        L.oracle_hmvm_seq.argtypes = [vp, f64, ci, vp, vp]
        L.oracle_hmvm_chunk.argtypes = [vp, f64, ci, vp, vp, ci]
        L.oracle_uniform_mvm.argtypes = [vp, f64, ci, vp, vp, ci]
        L.oracle_h2_mvm.argtypes = [vp, f64, ci, vp, vp]
        L.oracle_h2_mvm_par.argtypes = [vp, f64, ci, vp, vp, ci]
        L.oracle_dense_matvec.argtypes = [ci, i64, vp, vp, f64, f64, f64, ci, vp, vp, ci]
        L.oracle_leaf_max_error.argtypes = [vp, ci, vp, vp, f64, f64, i64]
        L.oracle_leaf_max_error.restype = f64
        for f in ("oracle_hmvm_seq", "oracle_hmvm_chunk", "oracle_uniform_mvm", "oracle_h2_mvm", "oracle_h2_mvm_par",
                  "oracle_dense_matvec"):
            getattr(L, f).restype = ci
        _lib = L
    return _lib


def _p(a: np.ndarray):
    """Address of a float64 array the C code reads or writes as contiguous."""
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise ValueError("oracle vectors must be contiguous float64 arrays")
    return a.ctypes.data


def _check(st: int, name: str) -> None:
    if st != 0:
        raise RuntimeError(f"{name} returned status {st}")


def hmvm_seq(desc, alpha: float, op: int, x: np.ndarray, y: np.ndarray) -> None:
    """y += alpha op(M) x, leaf by leaf in descriptor order (hlr::seq::mul_vec)."""
    _check(lib().oracle_hmvm_seq(C.addressof(desc), alpha, op, _p(x), _p(y)), "oracle_hmvm_seq")


def hmvm_chunk(desc, alpha: float, op: int, x: np.ndarray, y: np.ndarray, nthreads: int = 0) -> None:
    """y += alpha op(M) x with 64-row chunk locks (hlr::tbb::mul_vec)."""
    _check(lib().oracle_hmvm_chunk(C.addressof(desc), alpha, op, _p(x), _p(y), nthreads), "oracle_hmvm_chunk")


def h2_mvm(desc, alpha: float, op: int, x: np.ndarray, y: np.ndarray, nthreads: int = 1) -> int:
    """y += alpha op(M) x for an H^2 matrix (hlr::h2::mul_vec); returns the
    status.  nthreads != 1: the threaded form (0 = all cores), bit-identical."""
    if nthreads == 1:
        return lib().oracle_h2_mvm(C.addressof(desc), alpha, op, _p(x), _p(y))
    return lib().oracle_h2_mvm_par(C.addressof(desc), alpha, op, _p(x), _p(y), nthreads)


def uniform_mvm(desc, alpha: float, op: int, x: np.ndarray, y: np.ndarray, nthreads: int = 0) -> int:
    """y += alpha op(M) x for uniform-H (hlr::tbb::uniform::mul_vec); returns the status."""
    return lib().oracle_uniform_mvm(C.addressof(desc), alpha, op, _p(x), _p(y), nthreads)


def dense_matvec(hm, alpha: float, op: int, x: np.ndarray, y: np.ndarray, nthreads: int = 0) -> None:
    """y += alpha op(A) x with A formed from the kernel function (no compression)."""
    pr = hm.problem
    pts = np.ascontiguousarray(hm.points, dtype=np.float64)
    w = hm.weights if hm.weights is not None else np.zeros(1)
    _check(lib().oracle_dense_matvec(pr.kind, hm.n, _p(pts), _p(w), pr.ell, pr.nugget, alpha, op, _p(x), _p(y),
                                     nthreads), "oracle_dense_matvec")


def leaf_max_error(hm, desc, stride: int = 1) -> float:
    pr = hm.problem
    pts = np.ascontiguousarray(hm.points, dtype=np.float64)
    w = hm.weights if hm.weights is not None else np.zeros(1)
    return lib().oracle_leaf_max_error(C.addressof(desc), pr.kind, _p(pts), _p(w), pr.ell, pr.nugget, stride)
