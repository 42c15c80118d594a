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
"""
from __future__ import annotations

from dataclasses import dataclass, field

import torch

from . import apply_normal, mul_vec


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


class _InnerCG:
    """Static-tensor CG state so that a block of iterations can be captured
    in a CUDA graph and replayed."""

    def __init__(self, A, nrhs, N, count, pad, device):
        self.A, self.count, self.pad = A, count, pad
        z = lambda: torch.zeros(nrhs, N, dtype=torch.float64, device=device)
        self.d, self.res, self.p, self.q = z(), z(), z(), z()
        zs = lambda: torch.zeros(nrhs, count, dtype=torch.float64, device=device)
        self.rr, self.stop = zs(), zs()
        self.active = torch.zeros(nrhs, count, dtype=torch.bool, device=device)

    def reset(self, r, rtol):
        self.d.zero_()
        self.res.copy_(r)
        self.p.copy_(r)
        self.rr.copy_(_dots(r, r, self.count, self.pad))
        self.stop.copy_(rtol * rtol * self.rr)
        self.active.copy_(self.rr > 0)

    def step(self):
        c, p = self.count, self.pad
        self.q.zero_()
        mul_vec(1.0, apply_normal, self.A, self.p.T, self.q.T)
        pq = _dots(self.p, self.q, c, p)
        ok = self.active & (pq > 0)
        a = torch.where(ok, self.rr / torch.where(ok, pq, torch.ones_like(pq)), torch.zeros_like(pq))
        _axpy_(self.d, a, self.p, c, p)
        _axpy_(self.res, -a, self.q, c, p)
        rr_new = _dots(self.res, self.res, c, p)
        self.active &= rr_new > self.stop
        beta = torch.where(self.active, rr_new / torch.where(self.rr > 0, self.rr, torch.ones_like(self.rr)),
                           torch.zeros_like(rr_new))
        self.p.view(self.p.shape[0], c, p).mul_(beta[:, :, None]).add_(self.res.view(self.res.shape[0], c, p))
        self.rr.copy_(rr_new)


def cg_refine(A64, Alow, b: torch.Tensor, count: int, pad: int, tol: float = 1e-10, inner_rtol: float = 1e-6,
              max_outer: int = 20, max_inner: int = 20000, check_every: int = 20, use_graph: bool = True) -> CGResult:
    """Solve A x = b for every member and right-hand side of a batched handle.

    A64: FP64 batched DeviceMatrix (outer residual); Alow: the same matrices
    in reduced precision (inner CG operator; may be A64 itself).  b is
    (nrhs, count * pad).  Stops when every system reaches ||b - A x|| <= tol
    ||b|| with the FP64 product, or when refinement stops improving.
    """
    nrhs, N = b.shape
    dev = b.device
    bnorm = _dots(b, b, count, pad).sqrt()
    x = torch.zeros_like(b)
    r = torch.zeros_like(b)
    cg = _InnerCG(Alow, nrhs, N, count, pad, dev)
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
