"""Batched conjugate gradients with FP64 iterative refinement.

HLR's mixed-precision linear iteration (programs/iterrefine.hh:24-88) keeps
the residual b - A x in FP64 and applies a cheaper inner operator.  Here the
inner solver is CG with a reduced-precision H-matrix product (BF16 / FP16 /
mixed FP32-FP16 storage), the outer residual uses the FP64 product, and all
systems of a batched handle (members x right-hand sides) advance together:
every CG iteration is one batched product with all right-hand sides.

Vectors are (nrhs, count * pad) contiguous float64 CUDA tensors; the
products see their (count * pad, nrhs) column-major transposes, and
per-system reductions view them as (nrhs, count, pad).  Padding rows stay
zero throughout.  Refinement converges when kappa(A) * u_inner < 1 (u_inner
is the inner operator's relative error); systems where it stalls are
reported as not converged.

Preconditioning.  The reference preconditions its linear iteration with an
H-LU factorisation applied by triangular solves (iterrefine.hh:125-184,
matrix/luinv_eval.hh).  Here the inner CG can be preconditioned with a
block-Jacobi operator W = diag(A_kk^-1): the dense inverses of the diagonal
blocks of A (contiguous index ranges of `block` entries, assembled from the
leaves inside them), uploaded as a block-diagonal H-matrix of dense leaves,
so that applying W is one more product with the same kernels.  H-LU itself
(H-matrix arithmetic with recompression) is not built.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from . import LeafList, apply_normal, mul_vec, upload, upload_batch


@dataclass
class CGResult:
    x: torch.Tensor                   # (nrhs, N) solution (padding rows zero)
    rel_residual: torch.Tensor        # (nrhs, count) final ||b - A x|| / ||b|| (FP64 product)
    converged: torch.Tensor           # (nrhs, count) bool
    outer_iterations: int
    inner_iterations: int
    history: list = field(default_factory=list)   # max relative residual after each outer step


def _dots(a, b, count, pad):
    return (a.view(a.shape[0], count, pad) * b.view(b.shape[0], count, pad)).sum(-1)


def _axpy_(y, coef, x, count, pad):
    """y += coef[:, :, None] * x   (per-system coefficients)"""
    y.view(y.shape[0], count, pad).add_(coef[:, :, None] * x.view(x.shape[0], count, pad))


def _leaf_array(ptr, ld, rows, cols):
    """The (rows x cols) column-major matrix behind a leaf pointer (a view)."""
    if rows == 0 or cols == 0:
        return np.zeros((rows, cols))
    a = np.ctypeslib.as_array(ptr, shape=(ld * cols,))
    return a.reshape(cols, ld).T[:rows]


def diagonal_blocks(src, block: int = 256):
    """The dense diagonal blocks A_kk of an H-matrix (HostMatrix, LeafList or
    hlrc_h_desc): index ranges [k block, (k + 1) block), each assembled from
    the parts of the leaves (D, or U V^T) that fall inside it.  Returns a
    list of (first index, dense block)."""
    d = src.h_desc() if hasattr(src, "h_desc") else src
    n = int(d.nrows)
    starts = list(range(0, n, block))
    out = [np.zeros((min(block, n - i0), min(block, n - i0))) for i0 in starts]
    for i in range(int(d.nblocks)):
        b = d.blocks[i]
        r0, nr, c0, nc = int(b.row0), int(b.nrows), int(b.col0), int(b.ncols)
        if nr == 0 or nc == 0:
            continue
        for k in range(max(r0, c0) // block, min(r0 + nr - 1, c0 + nc - 1) // block + 1):
            i0, i1 = starts[k], min(starts[k] + block, n)
            ra, rb = max(r0, i0), min(r0 + nr, i1)
            ca, cb = max(c0, i0), min(c0 + nc, i1)
            if ra >= rb or ca >= cb:
                continue
            if b.kind == 0:
                D = _leaf_array(b.D, int(b.ldd), nr, nc)
                part = D[ra - r0:rb - r0, ca - c0:cb - c0]
            else:
                if b.rank == 0:
                    continue
                U = _leaf_array(b.U, int(b.ldu), nr, int(b.rank))
                V = _leaf_array(b.V, int(b.ldv), nc, int(b.rank))
                part = U[ra - r0:rb - r0] @ V[ca - c0:cb - c0].T
            out[k][ra - i0:rb - i0, ca - i0:cb - i0] += part
    return list(zip(starts, out))


def _zero_offdiagonal(W: LeafList, lo: int, hi: int, block: int) -> None:
    """Rank-0 leaves for the off-diagonal part of [lo, hi)^2, split in halves
    at multiples of `block` down to single diagonal blocks (about two leaves
    per diagonal block), so that the leaves of W cover the whole matrix."""
    nb = (hi - lo + block - 1) // block
    if nb <= 1:
        return
    mid = lo + (nb // 2) * block
    W.add_lowrank(lo, mid, np.zeros((mid - lo, 0)), np.zeros((hi - mid, 0)))
    W.add_lowrank(mid, lo, np.zeros((hi - mid, 0)), np.zeros((mid - lo, 0)))
    _zero_offdiagonal(W, lo, mid, block)
    _zero_offdiagonal(W, mid, hi, block)


def block_jacobi_leaves(src, block: int = 256) -> LeafList:
    """W = diag(A_kk^-1) as a leaf list: dense inverses of the diagonal
    blocks (A_kk symmetric positive definite: inverted through its Cholesky
    factor) and rank-0 leaves elsewhere."""
    d = src.h_desc() if hasattr(src, "h_desc") else src
    n = int(d.nrows)
    W = LeafList(n, n)
    for i0, Akk in diagonal_blocks(d, block):
        L = np.linalg.cholesky(0.5 * (Akk + Akk.T))
        Li = np.linalg.solve(L, np.eye(L.shape[0]))
        W.add_dense(i0, i0, Li.T @ Li)
    _zero_offdiagonal(W, 0, n, block)
    return W


def block_jacobi(src, block: int = 256, precision="f64", max_nrhs: int = 1):
    """The block-Jacobi preconditioner of one H-matrix, uploaded (a
    DeviceMatrix applied with mul_vec)."""
    return upload(block_jacobi_leaves(src, block), precision=precision, max_nrhs=max_nrhs)


def block_jacobi_batch(members, pad: int, block: int = 256, precision="f64", max_nrhs: int = 1):
    """The same for the members of a batched handle uploaded with pad_to=pad."""
    return upload_batch([block_jacobi_leaves(m, block) for m in members], precision=precision, max_nrhs=max_nrhs,
                        pad_to=pad)


class _InnerCG:
    """Static-tensor (preconditioned) CG state so that a block of iterations
    can be captured in a CUDA graph and replayed.  With W (a DeviceMatrix)
    the iteration is PCG with z = W r."""

    def __init__(self, A, nrhs, N, count, pad, device, W=None):
        self.A, self.W, self.count, self.pad = A, W, count, pad
        z = lambda: torch.zeros(nrhs, N, dtype=torch.float64, device=device)
        self.d, self.res, self.p, self.q = z(), z(), z(), z()
        self.z = z() if W is not None else self.res
        zs = lambda: torch.zeros(nrhs, count, dtype=torch.float64, device=device)
        self.rr, self.rz, self.stop = zs(), zs(), zs()
        self.active = torch.zeros(nrhs, count, dtype=torch.bool, device=device)

    def _precondition(self):
        if self.W is not None:
            self.z.zero_()
            mul_vec(1.0, apply_normal, self.W, self.res.T, self.z.T)

    def reset(self, r, rtol):
        self.d.zero_()
        self.res.copy_(r)
        self._precondition()
        self.p.copy_(self.z)
        self.rr.copy_(_dots(r, r, self.count, self.pad))
        self.rz.copy_(_dots(r, self.z, self.count, self.pad))
        self.stop.copy_(rtol * rtol * self.rr)
        self.active.copy_(self.rr > 0)

    def step(self):
        c, p = self.count, self.pad
        self.q.zero_()
        mul_vec(1.0, apply_normal, self.A, self.p.T, self.q.T)
        pq = _dots(self.p, self.q, c, p)
        ok = self.active & (pq > 0)
        a = torch.where(ok, self.rz / torch.where(ok, pq, torch.ones_like(pq)), torch.zeros_like(pq))
        _axpy_(self.d, a, self.p, c, p)
        _axpy_(self.res, -a, self.q, c, p)
        rr_new = _dots(self.res, self.res, c, p)
        self.active &= rr_new > self.stop
        self._precondition()
        rz_new = _dots(self.res, self.z, c, p) if self.W is not None else rr_new
        beta = torch.where(self.active, rz_new / torch.where(self.rz > 0, self.rz, torch.ones_like(self.rz)),
                           torch.zeros_like(rz_new))
        self.p.view(self.p.shape[0], c, p).mul_(beta[:, :, None]).add_(self.z.view(self.z.shape[0], c, p))
        self.rr.copy_(rr_new)
        self.rz.copy_(rz_new)


def cg_refine(A64, Alow, b: torch.Tensor, count: int, pad: int, tol: float = 1e-10, inner_rtol: float = 1e-6,
              max_outer: int = 20, max_inner: int = 20000, check_every: int = 20, use_graph: bool = True,
              precond=None) -> CGResult:
    """Solve A x = b for every member and right-hand side of a batched handle.

    A64: FP64 batched DeviceMatrix (outer residual); Alow: the same matrices
    in reduced precision (inner CG operator; may be A64 itself).  b is
    (nrhs, count * pad).  precond: an optional preconditioner W (a batched
    DeviceMatrix, e.g. block_jacobi_batch) for the inner CG.  Stops when
    every system reaches ||b - A x|| <= tol ||b|| with the FP64 product, or
    when refinement stops improving.
    """
    nrhs, N = b.shape
    dev = b.device
    bnorm = _dots(b, b, count, pad).sqrt()
    x = torch.zeros_like(b)
    r = torch.zeros_like(b)
    cg = _InnerCG(Alow, nrhs, N, count, pad, dev, precond)
    graph = None
    if use_graph:
        # warm up on a side stream, then capture `check_every` iterations
        cg.reset(b, inner_rtol)
        s = torch.cuda.Stream(device=dev)
        s.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(s):
            for _ in range(2):
                cg.step()
        torch.cuda.current_stream(dev).wait_stream(s)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            for _ in range(check_every):
                cg.step()
    inner_total, history = 0, []
    outer = 0
    best = float("inf")
    rel = torch.ones(nrhs, count, dtype=torch.float64, device=dev)
    for outer in range(1, max_outer + 1):
        r.copy_(b)
        mul_vec(-1.0, apply_normal, A64, x.T, r.T)             # r = b - A x in FP64
        rel = _dots(r, r, count, pad).sqrt() / torch.where(bnorm > 0, bnorm, torch.ones_like(bnorm))
        worst = float(rel.max())
        history.append(worst)
        if worst <= tol or worst > 0.5 * best:                 # converged, or refinement stalled
            break
        best = worst
        cg.reset(r, inner_rtol)
        it = 0
        while it < max_inner:
            if graph is not None:
                graph.replay()
            else:
                for _ in range(check_every):
                    cg.step()
            it += check_every
            if not bool(cg.active.any()):
                break
        inner_total += it
        x.add_(cg.d)
    return CGResult(x=x, rel_residual=rel, converged=rel <= tol, outer_iterations=outer,
                    inner_iterations=inner_total, history=history)
