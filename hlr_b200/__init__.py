"""hlr_b200 — B200-native H-matrix / uniform-H matrix-vector product.

Host-side mirror of HLR's MVM interface:

    hlr::tbb::mul_vec(alpha, op_M, M, x, y)            -> hlr_b200.mul_vec(alpha, op, M, x, y)
    hlr::tbb::uniform::mul_vec(alpha, op_M, M, x, y,
                               rowcb, colcb)           -> hlr_b200.uniform.mul_vec(alpha, op, M, x, y)

``M`` is a :class:`DeviceMatrix` (the flattened, device-resident copy made
once by :func:`upload`), ``x``/``y`` are float64 CUDA tensors (or numpy arrays
for the host-buffer path).  ``y`` is accumulated: ``y += alpha * op(M) x``.

Matrices come either from a caller's own leaf list (:class:`LeafList`,
the shape HLR's block tree flattens to) or from the host construction
:func:`build` (clustering, admissibility, ACA + SVD, uniform bases in C++).
Everything runs through ``libhlrc.so``; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _capi
from ._capi import HLRCError, check, lib

# HLIBpro matop_t
apply_normal = 0
apply_transposed = 1
apply_adjoint = 2

# storage precisions (hlrc_precision)
PREC_F64, PREC_F32, PREC_BF16, PREC_F16, PREC_MIXED, PREC_BFP = 0, 1, 2, 3, 4, 5
PRECISIONS = {"f64": PREC_F64, "f32": PREC_F32, "bf16": PREC_BF16, "f16": PREC_F16, "mixed": PREC_MIXED,
              "bfp": PREC_BFP}

LEAF_DENSE, LEAF_LOWRANK = 0, 1
PROBLEM_LOG1D, PROBLEM_EXP3D, PROBLEM_LAPLACE_SPH = 0, 1, 2


@dataclass
class Problem:
    """A test matrix definition (point set + kernel + H parameters)."""
    kind: int
    n: int = 0
    leaf_size: int = 64
    eta: float = 2.0
    eps: float = 1e-6
    seed: int = 1
    ell: float = 0.1
    nugget: float = 0.0
    refine: int = 6
    uniform: bool = False
    nthreads: int = 0
    nested: bool = False   # also build the H^2 form (nested cluster bases)
    on_device: bool = False  # assemble the leaves on the current CUDA device (H form only)

    @staticmethod
    def log1d(n: int, **kw) -> "Problem":
        """A_ij = log|x_i - x_j|, A_ii = h(log h - 1), x_i ~ U[0,1]."""
        return Problem(kind=PROBLEM_LOG1D, n=n, **kw)

    @staticmethod
    def exp3d(n: int, ell: float = 0.1, nugget: float = 1e-4, **kw) -> "Problem":
        """Exponential covariance exp(-r/ell) (+ nugget) on U[0,1]^3 points."""
        return Problem(kind=PROBLEM_EXP3D, n=n, ell=ell, nugget=nugget, **kw)

    @staticmethod
    def laplace_sphere(refine: int = 6, **kw) -> "Problem":
        """Collocation of 1/(4 pi r) on a refined octahedron sphere mesh."""
        return Problem(kind=PROBLEM_LAPLACE_SPH, refine=refine, **kw)

    def to_c(self) -> _capi.hlrc_problem:
        p = _capi.hlrc_problem()
        p.kind, p.leaf_size, p.n, p.refine = self.kind, self.leaf_size, self.n, self.refine
        p.uniform, p.seed, p.eta, p.eps = int(self.uniform), self.seed, self.eta, self.eps
        p.ell, p.nugget, p.nthreads = self.ell, self.nugget, self.nthreads
        p.nested = int(self.nested)
        p.on_device = int(self.on_device)
        return p


class HostMatrix:
    """Host-built H-matrix (and optionally its uniform-H form) owned by C++."""

    def __init__(self, problem: Problem):
        self.problem = problem
        h = C.c_void_p()
        pc = problem.to_c()
        check(lib().hlrc_build(C.byref(pc), C.byref(h)), "hlrc_build")
        self._h = h
        pts, dim, n = _capi.pdbl(), C.c_int(), C.c_int64()
        check(lib().hlrc_build_points(h, C.byref(pts), C.byref(dim), C.byref(n)), "hlrc_build_points")
        self.n = n.value
        self.dim = dim.value
        self.points = np.ctypeslib.as_array(pts, shape=(self.n * self.dim,)).reshape(self.n, self.dim).copy()
        w = _capi.pdbl()
        check(lib().hlrc_build_weights(h, C.byref(w)), "hlrc_build_weights")
        self.weights = np.ctypeslib.as_array(w, shape=(self.n,)).copy() if bool(w) else None
        perm = C.POINTER(C.c_int64)()
        check(lib().hlrc_build_perm(h, C.byref(perm)), "hlrc_build_perm")
        self.perm_i2e = np.ctypeslib.as_array(perm, shape=(self.n,)).copy()
        secs, nl, mr, by = C.c_double(), C.c_int64(), C.c_int32(), C.c_int64()
        check(lib().hlrc_build_stats(h, C.byref(secs), C.byref(nl), C.byref(mr), C.byref(by)), "hlrc_build_stats")
        self.build_seconds, self.nleaves, self.max_rank, self.bytes = secs.value, nl.value, mr.value, by.value

    @property
    def leaves_on_device(self) -> bool:
        """True while the leaf data of an on_device build is in device memory
        (h_desc() then holds device pointers; upload passes that on)."""
        v = C.c_int(0)
        check(lib().hlrc_build_leaves_on_device(self._h, C.byref(v)), "hlrc_build_leaves_on_device")
        return bool(v.value)

    def fetch(self) -> "HostMatrix":
        """Copies device-resident leaf data to host memory (hlrc_build_fetch);
        afterwards the matrix behaves like a host build.  Returns self."""
        check(lib().hlrc_build_fetch(self._h), "hlrc_build_fetch")
        return self

    def h_desc(self) -> _capi.hlrc_h_desc:
        d = _capi.hlrc_h_desc()
        check(lib().hlrc_build_h_desc(self._h, C.byref(d)), "hlrc_build_h_desc")
        d._owner = self
        return d

    def uniform_desc(self) -> _capi.hlrc_uniform_desc:
        d = _capi.hlrc_uniform_desc()
        check(lib().hlrc_build_uniform_desc(self._h, C.byref(d)), "hlrc_build_uniform_desc")
        d._owner = self
        return d

    def h2_desc(self) -> _capi.hlrc_h2_desc:
        d = _capi.hlrc_h2_desc()
        check(lib().hlrc_build_h2_desc(self._h, C.byref(d)), "hlrc_build_h2_desc")
        d._owner = self
        return d

    def entry(self, i: int, j: int) -> float:
        return lib().hlrc_build_entry(self._h, i, j)

    def close(self) -> None:
        if self._h:
            lib().hlrc_build_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def build(problem: Problem) -> HostMatrix:
    """Host construction: cluster tree, block tree, ACA + SVD (C++, OpenMP)."""
    return HostMatrix(problem)


class LeafList:
    """An H-matrix given as a flat list of leaves (numpy, column-major).

    ``add_dense(row0, col0, D)`` and ``add_lowrank(row0, col0, U, V)`` (M = U V^T)
    mirror dense_matrix / lrmatrix; the list keeps the arrays alive.
    """

    def __init__(self, nrows: int, ncols: int):
        self.nrows, self.ncols = nrows, ncols
        self._keep = []
        self._blocks = []

    def _arr(self, a) -> np.ndarray:
        a = np.asfortranarray(np.asarray(a, dtype=np.float64))
        self._keep.append(a)
        return a

    def add_dense(self, row0: int, col0: int, D) -> None:
        D = self._arr(D)
        b = _capi.hlrc_block()
        b.row0, b.nrows, b.col0, b.ncols = row0, D.shape[0], col0, D.shape[1]
        b.kind, b.rank = LEAF_DENSE, 0
        b.D = D.ctypes.data_as(_capi.pdbl)
        b.ldd = max(1, D.shape[0])
        self._blocks.append(b)

    def add_lowrank(self, row0: int, col0: int, U, V) -> None:
        U, V = self._arr(U), self._arr(V)
        assert U.shape[1] == V.shape[1]
        b = _capi.hlrc_block()
        b.row0, b.nrows, b.col0, b.ncols = row0, U.shape[0], col0, V.shape[0]
        b.kind, b.rank = LEAF_LOWRANK, U.shape[1]
        b.U = U.ctypes.data_as(_capi.pdbl)
        b.ldu = max(1, U.shape[0])
        b.V = V.ctypes.data_as(_capi.pdbl)
        b.ldv = max(1, V.shape[0])
        self._blocks.append(b)

    def h_desc(self) -> _capi.hlrc_h_desc:
        arr = (_capi.hlrc_block * max(1, len(self._blocks)))(*self._blocks)
        d = _capi.hlrc_h_desc()
        d.nrows, d.ncols, d.nblocks = self.nrows, self.ncols, len(self._blocks)
        d.blocks = C.cast(arr, C.POINTER(_capi.hlrc_block))
        d._owner = (self, arr)
        return d


def _on_device(src) -> bool:
    """Whether src's leaf data is in device memory (an on_device build not
    fetched to the host)."""
    return isinstance(src, HostMatrix) and src.leaves_on_device


def _options(precision="f64", max_nrhs: int = 1, mixed_eps: float = 1e-6, device: int = -1, plan=None):
    o = _capi.hlrc_options()
    lib().hlrc_default_options(C.byref(o))
    o.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    o.max_nrhs, o.mixed_eps, o.device = max_nrhs, mixed_eps, device
    plan = plan or {}
    unknown = set(plan) - {"finish_slots", "piece_tiles", "near_field"}
    if unknown:
        raise ValueError(f"unknown plan options {sorted(unknown)}")
    o.finish_slots = int(plan.get("finish_slots", 0))
    o.piece_tiles = int(plan.get("piece_tiles", 0))
    o.near_field = int(plan.get("near_field", 0))
    return o


class DeviceMatrix:
    """Device-resident flattened H / uniform-H matrix (an ``hlrc_hmat``)."""

    def __init__(self, handle: C.c_void_p, uniform: bool):
        self._h = handle
        self.uniform = uniform
        self.h2 = False
        self.plan = {}     # plan-level choices it was uploaded with
        inf = _capi.hlrc_info()
        check(lib().hlrc_get_info(self._h, C.byref(inf)), "hlrc_get_info")
        self.info = {f: getattr(inf, f) for f, _ in _capi.hlrc_info._fields_ if f not in ("reserved", "launches")}
        self.info["launches"] = list(inf.launches)
        self.nrows, self.ncols = inf.n_rows, inf.n_cols

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def set_profiling(self, on: bool = True) -> None:
        check(lib().hlrc_set_profiling(self._h, int(on)), "hlrc_set_profiling")

    def last_profile(self) -> dict:
        """{pass name: (launches, total ms, algorithmic bytes per launch)} since the last read."""
        names = (C.c_char_p * 64)()
        cnt = (C.c_int * 64)()
        ms = (C.c_double * 64)()
        by = (C.c_int64 * 64)()
        k = lib().hlrc_last_profile(self._h, names, cnt, ms, by, 64)
        return {names[i].decode(): (cnt[i], ms[i], by[i]) for i in range(k)}

    @property
    def tuning(self) -> dict:
        """Launch shapes of this handle's products (hlrc_get_tuning):
        nform_warps, ttform_warps (4, 8 or 16), mr_min_nrhs, wide_min_nrhs,
        overlap (programmatic dependent launch of the one-vector kernels) and
        side_at (how many other passes launch before the near field's side
        pass is forked)."""
        t = _capi.hlrc_tuning()
        check(lib().hlrc_get_tuning(self._h, C.byref(t)), "hlrc_get_tuning")
        return {"nform_warps": t.nform_warps, "ttform_warps": t.ttform_warps, "mr_min_nrhs": t.mr_min_nrhs,
                "wide_min_nrhs": t.wide_min_nrhs, "overlap": t.overlap, "side_at": t.side_at}

    def set_tuning(self, **kw) -> None:
        """Changes some launch shapes (hlrc_set_tuning); the others keep their
        values.  Invalid values raise HLRCError (HLRC_ERR_ARG)."""
        cur = self.tuning
        unknown = set(kw) - set(cur)
        if unknown:
            raise ValueError(f"unknown tuning keys {sorted(unknown)}")
        cur.update(kw)
        t = _capi.hlrc_tuning(int(cur["nform_warps"]), int(cur["ttform_warps"]), int(cur["mr_min_nrhs"]),
                              int(cur["wide_min_nrhs"]), int(cur["overlap"]), int(cur["side_at"]))
        check(lib().hlrc_set_tuning(self._h, C.byref(t)), "hlrc_set_tuning")

    def launch_count(self) -> int:
        """Kernels launched by this handle so far (hlrc_launch_count)."""
        return int(lib().hlrc_launch_count(self._h))

    def device_error(self) -> int:
        """Reads and clears the device error word (hlrc_check_device_error):
        0, or the code of a bounded device wait that ran out."""
        code = C.c_int(0)
        check(lib().hlrc_check_device_error(self._h, C.byref(code)), "hlrc_check_device_error")
        return int(code.value)

    def free(self) -> None:
        if self._h:
            lib().hlrc_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Workspace:
    """Caller-owned scratch for one handle's products (``hlrc_workspace``).

    A DeviceMatrix is immutable; all the scratch a product writes lives in a
    workspace.  Products of one handle on several streams run concurrently
    when each passes its own workspace to :func:`mul_vec` — the counterpart
    of calling ``hlr::tbb::mul_vec`` on one matrix from several threads with
    different y (tbb/arith.hh:312-323).  ``max_nrhs > 1`` adds the
    multi-vector kernels' scratch.
    """

    def __init__(self, M: "DeviceMatrix", max_nrhs: int = 1):
        h = C.c_void_p()
        check(lib().hlrc_workspace_create(M.handle, int(max_nrhs), C.byref(h)), "hlrc_workspace_create")
        self._h = h
        self.device_matrix = M

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def free(self) -> None:
        if self._h:
            lib().hlrc_workspace_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def upload(src, precision="f64", uniform: Optional[bool] = None, max_nrhs: int = 1,
           mixed_eps: float = 1e-6, device: int = -1, h2: bool = False, plan: Optional[dict] = None) -> DeviceMatrix:
    """Flatten and upload a matrix: ``src`` is a HostMatrix, LeafList or
    descriptor.  ``h2=True`` uploads the H^2 form (nested cluster bases) of
    a HostMatrix built with ``Problem(..., nested=True)``, or an
    ``hlrc_h2_desc``.  ``plan``: plan-level choices (``finish_slots``,
    ``piece_tiles``; see hlrc_options), e.g. from tune.autotune_plan."""
    if isinstance(src, _capi.hlrc_h2_desc):
        h2 = True
    if uniform is None:
        uniform = (not h2) and isinstance(src, HostMatrix) and src.problem.uniform
    o = _options(precision, max_nrhs, mixed_eps, device, plan)
    o.leaves_on_device = int(_on_device(src))
    h = C.c_void_p()
    if h2:
        d = src.h2_desc() if hasattr(src, "h2_desc") else src
        check(lib().hlrc_upload_h2(C.byref(d), C.byref(o), C.byref(h)), "hlrc_upload_h2")
        M = DeviceMatrix(h, False)
        M.h2 = True
        M.plan = dict(plan or {})
        return M
    if uniform:
        d = src.uniform_desc() if hasattr(src, "uniform_desc") else src
        check(lib().hlrc_upload_uniform(C.byref(d), C.byref(o), C.byref(h)), "hlrc_upload_uniform")
    else:
        d = src.h_desc() if hasattr(src, "h_desc") else src
        check(lib().hlrc_upload_h(C.byref(d), C.byref(o), C.byref(h)), "hlrc_upload_h")
    M = DeviceMatrix(h, uniform)
    M.plan = dict(plan or {})
    return M


def upload_batch(members, precision="f64", max_nrhs: int = 1, pad_to: Optional[int] = None,
                 mixed_eps: float = 1e-6, device: int = -1, plan: Optional[dict] = None) -> DeviceMatrix:
    """Upload many H-matrices as one block-diagonal handle.

    Member i occupies rows/columns [offsets[i], offsets[i] + n_i); with
    ``pad_to`` every member starts at i * pad_to (zero padding between), so
    batched vectors can be viewed as (count, pad_to, nrhs) tensors.  Every
    pass of a product then runs as one launch over all members.
    """
    descs = [m.h_desc() if hasattr(m, "h_desc") else m for m in members]
    sizes = [int(d.nrows) for d in descs]
    if pad_to is not None:
        if max(sizes) > pad_to:
            raise ValueError("pad_to is smaller than the largest member")
        offsets = [i * pad_to for i in range(len(descs) + 1)]
    else:
        offsets = [0]
        for s in sizes:
            offsets.append(offsets[-1] + s)
    arr = (_capi.hlrc_h_desc * len(descs))(*descs)
    offs = (C.c_int64 * len(offsets))(*offsets)
    o = _options(precision, max_nrhs, mixed_eps, device, plan)
    dev = {_on_device(m) for m in members}
    if len(dev) > 1:
        raise ValueError("upload_batch: members with device-resident and host leaves (fetch() the former)")
    o.leaves_on_device = int(dev.pop())
    h = C.c_void_p()
    check(lib().hlrc_upload_h_batch(arr, len(descs), offs, C.byref(o), C.byref(h)), "hlrc_upload_h_batch")
    M = DeviceMatrix(h, False)
    M.plan = dict(plan or {})
    M.offsets = offsets
    M.sizes = sizes
    return M


def plan_info(src, precision="f64", uniform: Optional[bool] = None, max_nrhs: int = 1,
              mixed_eps: float = 1e-6, h2: bool = False, plan: Optional[dict] = None) -> dict:
    """Dry run of :func:`upload`: validates and flattens on the host only."""
    if isinstance(src, _capi.hlrc_h2_desc):
        h2 = True
    if uniform is None:
        uniform = (not h2) and isinstance(src, HostMatrix) and src.problem.uniform
    o = _options(precision, max_nrhs, mixed_eps, -1, plan)
    o.leaves_on_device = int(_on_device(src))
    inf = _capi.hlrc_info()
    if h2:
        d = src.h2_desc() if hasattr(src, "h2_desc") else src
        check(lib().hlrc_plan_info_h2(C.byref(d), C.byref(o), C.byref(inf)), "hlrc_plan_info_h2")
    elif uniform:
        d = src.uniform_desc() if hasattr(src, "uniform_desc") else src
        check(lib().hlrc_plan_info_uniform(C.byref(d), C.byref(o), C.byref(inf)), "hlrc_plan_info_uniform")
    else:
        d = src.h_desc() if hasattr(src, "h_desc") else src
        check(lib().hlrc_plan_info_h(C.byref(d), C.byref(o), C.byref(inf)), "hlrc_plan_info_h")
    out = {f: getattr(inf, f) for f, _ in _capi.hlrc_info._fields_ if f not in ("reserved", "launches")}
    out["launches"] = list(inf.launches)   # one-vector product, per op N / T / C
    return out


def _vec_args(v, n: int):
    """(pointer, nrhs, ld, is_device) for a 1-D (n,) or column-major (n, nrhs) float64 array."""
    if hasattr(v, "data_ptr"):  # torch tensor
        import torch
        if v.dtype != torch.float64:
            raise TypeError("vectors must be float64")
        if v.dim() == 1:
            if v.stride(0) != 1 and v.numel() > 1:
                raise ValueError("vector must be contiguous")
            return v.data_ptr(), 1, max(1, v.shape[0]), v.is_cuda
        # the stride of a dimension of size 1 is arbitrary in torch
        if v.stride(0) != 1 and v.shape[0] > 1:
            raise ValueError("multi-RHS arrays must be column-major (n, nrhs) with stride(0) == 1")
        ld = v.stride(1) if v.shape[1] > 1 else max(1, v.shape[0])
        return v.data_ptr(), v.shape[1], ld, v.is_cuda
    a = v
    if not isinstance(a, np.ndarray) or a.dtype != np.float64:
        raise TypeError("vectors must be float64 numpy arrays or torch tensors")
    if a.ndim == 1:
        if not a.flags.c_contiguous:
            raise ValueError("vector must be contiguous")
        return a.ctypes.data, 1, max(1, a.shape[0]), False
    if not a.flags.f_contiguous:
        raise ValueError("multi-RHS arrays must be Fortran-ordered (n, nrhs)")
    return a.ctypes.data, a.shape[1], a.shape[0], False


def mul_vec(alpha: float, op: int, M: DeviceMatrix, x, y, stream=None, workspace: Optional[Workspace] = None) -> None:
    """y += alpha * op(M) x  (drop-in for hlr::tbb::mul_vec / hlr::seq::mul_vec).

    Device tensors run on ``stream`` (default: torch's current stream) without
    synchronising; numpy arrays take the host-buffer path (copies included).
    With ``workspace`` (device tensors only) the product's scratch is that
    workspace instead of the handle's, so products on other streams with
    other workspaces may run at the same time.
    """
    xp, xn, ldx, xdev = _vec_args(x, 0)
    yp, yn, ldy, ydev = _vec_args(y, 0)
    if xn != yn:
        raise ValueError("x and y have different numbers of right-hand sides")
    if xdev != ydev:
        raise ValueError("x and y must both be device or both be host arrays")
    nx = M.ncols if op == apply_normal else M.nrows
    ny = M.nrows if op == apply_normal else M.ncols
    if (x.shape[0] != nx) or (y.shape[0] != ny):
        raise ValueError(f"shape mismatch: op(M) is {ny}x{nx}, x has {x.shape[0]}, y has {y.shape[0]} rows")
    if xdev:
        if stream is None:
            import torch
            stream = torch.cuda.current_stream(x.device).cuda_stream
        if workspace is not None:
            check(lib().hlrc_mvm_ws(M.handle, workspace.handle, float(alpha), int(op), C.c_void_p(xp),
                                    C.c_void_p(yp), xn, ldx, ldy, C.c_void_p(stream)), "hlrc_mvm_ws")
            return
        check(lib().hlrc_mvm(M.handle, float(alpha), int(op), C.c_void_p(xp), C.c_void_p(yp), xn, ldx, ldy,
                             C.c_void_p(stream)), "hlrc_mvm")
    else:
        if workspace is not None:
            raise ValueError("a workspace serves device vectors; host vectors use the handle's staging")
        check(lib().hlrc_mvm_host(M.handle, float(alpha), int(op), C.c_void_p(xp), C.c_void_p(yp), xn, ldx, ldy),
              "hlrc_mvm_host")


mvm = mul_vec


class h2:  # namespace mirroring hlr::h2
    @staticmethod
    def mul_vec(alpha: float, op: int, M: DeviceMatrix, x, y, stream=None) -> None:
        """y += alpha * op(M) x for an H^2 matrix (op N or adjoint)."""
        if not getattr(M, "h2", False):
            raise ValueError("h2.mul_vec needs an H^2 DeviceMatrix (upload(..., h2=True))")
        mul_vec(alpha, op, M, x, y, stream)


class uniform:  # namespace mirroring hlr::tbb::uniform
    @staticmethod
    def mul_vec(alpha: float, op: int, M: DeviceMatrix, x, y, stream=None) -> None:
        """y += alpha * op(M) x for a uniform-H matrix (op N or adjoint)."""
        if not M.uniform:
            raise ValueError("uniform.mul_vec needs a uniform-H DeviceMatrix")
        mul_vec(alpha, op, M, x, y, stream)


def fp64_peak(device: int = 0) -> float:
    """Measured FP64 tensor-core throughput of ``device`` in TFLOP/s
    (hlrc_fp64_peak: a timed DMMA loop; no clock or other setting changes)."""
    t = C.c_double(0.0)
    check(lib().hlrc_fp64_peak(int(device), C.byref(t)), "hlrc_fp64_peak")
    return float(t.value)


__all__ = [
    "apply_normal", "apply_transposed", "apply_adjoint", "Problem", "HostMatrix", "LeafList", "DeviceMatrix",
    "build", "upload", "mul_vec", "mvm", "uniform", "h2", "HLRCError", "PRECISIONS", "Workspace", "fp64_peak",
]
