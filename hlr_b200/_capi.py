"""ctypes binding of the C ABI in ``include/hlrc.h`` (libhlrc.so).

The structures below mirror the header field by field; ``tests/test_abi.py``
checks their sizes against the compiled library's expectations.  Loading
fails loudly when the in-tree library is missing: there is no fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libhlrc.so"

HLRC_OK = 0
STATUS_NAMES = {
    0: "HLRC_OK", 1: "HLRC_ERR_ARG", 2: "HLRC_ERR_SHAPE", 3: "HLRC_ERR_OOM", 4: "HLRC_ERR_CUDA",
    5: "HLRC_ERR_TIMEOUT", 6: "HLRC_ERR_UNSUPPORTED_OP", 7: "HLRC_ERR_NOT_CONVERGED", 8: "HLRC_ERR_INTERNAL",
}

i32, i64, u64, f64 = C.c_int32, C.c_int64, C.c_uint64, C.c_double
pdbl = C.POINTER(C.c_double)


class hlrc_block(C.Structure):
    _fields_ = [("row0", i64), ("nrows", i64), ("col0", i64), ("ncols", i64),
                ("kind", i32), ("rank", i32),
                ("D", pdbl), ("ldd", i64), ("U", pdbl), ("ldu", i64), ("V", pdbl), ("ldv", i64),
                ("sv", pdbl)]


class hlrc_h_desc(C.Structure):
    _fields_ = [("nrows", i64), ("ncols", i64), ("nblocks", i64), ("blocks", C.POINTER(hlrc_block))]


class hlrc_basis(C.Structure):
    _fields_ = [("ofs", i64), ("size", i64), ("rank", i32), ("pad_", i32), ("V", pdbl), ("ldv", i64)]


class hlrc_uniform_block(C.Structure):
    _fields_ = [("row0", i64), ("nrows", i64), ("col0", i64), ("ncols", i64),
                ("kind", i32), ("row_basis", i32), ("col_basis", i32), ("pad_", i32),
                ("S", pdbl), ("lds", i64), ("D", pdbl), ("ldd", i64)]


class hlrc_uniform_desc(C.Structure):
    _fields_ = [("nrows", i64), ("ncols", i64),
                ("nrow_bases", i64), ("row_bases", C.POINTER(hlrc_basis)),
                ("ncol_bases", i64), ("col_bases", C.POINTER(hlrc_basis)),
                ("nblocks", i64), ("blocks", C.POINTER(hlrc_uniform_block))]


class hlrc_h2_cluster(C.Structure):
    _fields_ = [("ofs", i64), ("size", i64), ("son", i32 * 2), ("parent", i32), ("rank", i32),
                ("V", pdbl), ("ldv", i64), ("E", pdbl), ("lde", i64)]


class hlrc_h2_desc(C.Structure):
    _fields_ = [("nrows", i64), ("ncols", i64),
                ("nrow_clusters", i64), ("row_clusters", C.POINTER(hlrc_h2_cluster)),
                ("ncol_clusters", i64), ("col_clusters", C.POINTER(hlrc_h2_cluster)),
                ("nblocks", i64), ("blocks", C.POINTER(hlrc_uniform_block))]


class hlrc_options(C.Structure):
    _fields_ = [("precision", i32), ("max_nrhs", i32), ("mixed_eps", f64), ("device", i32),
                ("finish_slots", i32), ("piece_tiles", i32), ("leaves_on_device", i32), ("near_field", i32),
                ("reserved", i32 * 3)]


class hlrc_info(C.Structure):
    _fields_ = [("n_rows", i64), ("n_cols", i64), ("n_dense", i64), ("n_lowrank", i64),
                ("n_row_tiles", i64), ("n_col_tiles", i64), ("matrix_bytes", i64),
                ("algorithmic_bytes", i64), ("flops", i64), ("workspace_bytes", i64),
                ("device_bytes", i64), ("precision", i32), ("kind", i32), ("max_rank", i32),
                ("launches", i32 * 3), ("scratch_bytes", i64)]


class hlrc_tuning(C.Structure):
    _fields_ = [("nform_warps", i32), ("ttform_warps", i32), ("mr_min_nrhs", i32), ("wide_min_nrhs", i32),
                ("overlap", i32), ("side_at", i32), ("reserved", i32 * 2)]


HLRC_MR_NEVER = 1000000


class hlrc_problem(C.Structure):
    _fields_ = [("kind", i32), ("leaf_size", i32), ("n", i64), ("refine", i32), ("uniform", i32),
                ("seed", u64), ("eta", f64), ("eps", f64), ("ell", f64), ("nugget", f64),
                ("nthreads", i32), ("nested", i32), ("on_device", i32), ("reserved", i32 * 3)]


# name -> (restype, argtypes); every symbol declared in include/hlrc.h
PROTOTYPES = {
    "hlrc_abi_version": (C.c_int, []),
    "hlrc_last_error": (C.c_char_p, []),
    "hlrc_default_options": (None, [C.POINTER(hlrc_options)]),
    "hlrc_upload_h": (C.c_int, [C.POINTER(hlrc_h_desc), C.POINTER(hlrc_options), C.POINTER(C.c_void_p)]),
    "hlrc_upload_uniform": (C.c_int, [C.POINTER(hlrc_uniform_desc), C.POINTER(hlrc_options), C.POINTER(C.c_void_p)]),
    "hlrc_upload_h_batch": (C.c_int, [C.POINTER(hlrc_h_desc), C.c_int, C.POINTER(i64), C.POINTER(hlrc_options),
                                      C.POINTER(C.c_void_p)]),
    "hlrc_plan_info_h": (C.c_int, [C.POINTER(hlrc_h_desc), C.POINTER(hlrc_options), C.POINTER(hlrc_info)]),
    "hlrc_plan_info_uniform": (C.c_int, [C.POINTER(hlrc_uniform_desc), C.POINTER(hlrc_options),
                                         C.POINTER(hlrc_info)]),
    "hlrc_upload_h2": (C.c_int, [C.POINTER(hlrc_h2_desc), C.POINTER(hlrc_options), C.POINTER(C.c_void_p)]),
    "hlrc_plan_info_h2": (C.c_int, [C.POINTER(hlrc_h2_desc), C.POINTER(hlrc_options), C.POINTER(hlrc_info)]),
    "hlrc_row_cuts": (C.c_int, [C.POINTER(hlrc_h_desc), C.c_int, C.POINTER(i64)]),
    "hlrc_mvm": (C.c_int, [C.c_void_p, f64, C.c_int, C.c_void_p, C.c_void_p, C.c_int, i64, i64, C.c_void_p]),
    "hlrc_mvm_host": (C.c_int, [C.c_void_p, f64, C.c_int, C.c_void_p, C.c_void_p, C.c_int, i64, i64]),
    "hlrc_mvm_noalloc": (C.c_int, [C.c_void_p, f64, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "hlrc_get_info": (C.c_int, [C.c_void_p, C.POINTER(hlrc_info)]),
    "hlrc_workspace_create": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "hlrc_mvm_ws": (C.c_int, [C.c_void_p, C.c_void_p, f64, C.c_int, C.c_void_p, C.c_void_p, C.c_int, i64, i64,
                              C.c_void_p]),
    "hlrc_workspace_free": (C.c_int, [C.c_void_p]),
    "hlrc_fp64_peak": (C.c_int, [C.c_int, C.POINTER(f64)]),
    "hlrc_debug_waits": (C.c_int, [C.c_void_p, i64, C.c_int]),
    "hlrc_get_tuning": (C.c_int, [C.c_void_p, C.POINTER(hlrc_tuning)]),
    "hlrc_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(hlrc_tuning)]),
    "hlrc_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "hlrc_last_profile": (C.c_int, [C.c_void_p, C.POINTER(C.c_char_p), C.POINTER(C.c_int), pdbl,
                                    C.POINTER(i64), C.c_int]),
    "hlrc_free": (C.c_int, [C.c_void_p]),
    "hlrc_launch_count": (i64, [C.c_void_p]),
    "hlrc_check_device_error": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "hlrc_build": (C.c_int, [C.POINTER(hlrc_problem), C.POINTER(C.c_void_p)]),
    "hlrc_build_h_desc": (C.c_int, [C.c_void_p, C.POINTER(hlrc_h_desc)]),
    "hlrc_build_uniform_desc": (C.c_int, [C.c_void_p, C.POINTER(hlrc_uniform_desc)]),
    "hlrc_build_h2_desc": (C.c_int, [C.c_void_p, C.POINTER(hlrc_h2_desc)]),
    "hlrc_build_points": (C.c_int, [C.c_void_p, C.POINTER(pdbl), C.POINTER(C.c_int), C.POINTER(i64)]),
    "hlrc_build_weights": (C.c_int, [C.c_void_p, C.POINTER(pdbl)]),
    "hlrc_build_perm": (C.c_int, [C.c_void_p, C.POINTER(C.POINTER(i64))]),
    "hlrc_build_stats": (C.c_int, [C.c_void_p, C.POINTER(f64), C.POINTER(i64), C.POINTER(i32), C.POINTER(i64)]),
    "hlrc_build_free": (C.c_int, [C.c_void_p]),
    "hlrc_build_leaves_on_device": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "hlrc_build_fetch": (C.c_int, [C.c_void_p]),
    "hlrc_build_entry": (f64, [C.c_void_p, i64, i64]),
}

_lib = None


class HLRCError(RuntimeError):
    """Raised for a non-OK hlrc_status; carries the status and the C message."""

    def __init__(self, status: int, func: str, msg: str):
        self.status = status
        super().__init__(f"{func}: {STATUS_NAMES.get(status, status)}: {msg}")


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"native library {LIB_PATH} is missing; run `python -m hlr_b200.build_native` "
                               "(there is no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in PROTOTYPES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int, func: str) -> None:
    if status != HLRC_OK:
        msg = lib().hlrc_last_error()
        raise HLRCError(status, func, msg.decode() if msg else "")
