"""Concurrent products of one immutable handle: each stream passes its own
workspace (hlrc_mvm_ws).  HLR's TBB product may likewise be called from
several threads on one matrix with different y (tbb/arith.hh:312-323, y
updated under per-chunk locks in tbb/detail/arith.hh:95-124).  Every result
is checked against the oracle's FP64 product."""
import numpy as np
import pytest

import hlr_b200 as hlr
import oracle
from hlr_b200 import HLRCError

from conftest import built, relerr

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _oracle_cols(desc, alpha, op, X, uniform=False):
    Y = np.zeros_like(X)
    for j in range(X.shape[1]):
        y = np.zeros(X.shape[0])
        if uniform:
            assert oracle.uniform_mvm(desc, alpha, op, np.ascontiguousarray(X[:, j]), y) == 0
        else:
            oracle.hmvm_seq(desc, alpha, op, np.ascontiguousarray(X[:, j]), y)
        Y[:, j] = y
    return Y


def _colmajor(A):
    return torch.from_numpy(np.ascontiguousarray(A.T)).cuda().T


@pytest.mark.parametrize("nrhs", [1, 8])
def test_two_streams_two_workspaces_one_handle(nrhs):
    hm = built("exp3d_16384", lambda: hlr.build(hlr.Problem.exp3d(16384)))
    M = hlr.upload(hm, max_nrhs=nrhs)
    W = [hlr.Workspace(M, max_nrhs=nrhs), hlr.Workspace(M, max_nrhs=nrhs)]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    rng = np.random.default_rng(11)
    X = [rng.standard_normal((hm.n, nrhs)) for _ in range(2)]
    Xd = [_colmajor(a) for a in X]
    Yd = [_colmajor(np.zeros((hm.n, nrhs))) for _ in range(2)]
    ops, alphas, reps = [0, 2], [1.5, -0.25], 6
    torch.cuda.synchronize()
    for _ in range(reps):
        for k in range(2):
            with torch.cuda.stream(streams[k]):
                xk, yk = (Xd[k][:, 0], Yd[k][:, 0]) if nrhs == 1 else (Xd[k], Yd[k])
                hlr.mul_vec(alphas[k], ops[k], M, xk, yk, workspace=W[k])
    torch.cuda.synchronize()
    d = hm.h_desc()
    for k in range(2):
        ref = _oracle_cols(d, alphas[k] * reps, ops[k], X[k])
        got = Yd[k].cpu().numpy()
        for j in range(nrhs):
            assert relerr(got[:, j], ref[:, j]) <= TOL, (k, j)
    for w in W:
        w.free()
    M.free()


def test_workspace_on_uniform_and_reduced_precision_handles():
    hu = built("sphere5u", lambda: hlr.build(hlr.Problem.laplace_sphere(refine=5, uniform=True)))
    U = hlr.upload(hu)
    Wu = hlr.Workspace(U)
    xh = np.random.default_rng(2).standard_normal(hu.n)
    for op in (0, 2):
        y = torch.zeros(hu.n, dtype=torch.float64, device="cuda")
        hlr.mul_vec(1.0, op, U, torch.from_numpy(xh).cuda(), y, workspace=Wu)
        torch.cuda.synchronize()
        yo = np.zeros(hu.n)
        assert oracle.uniform_mvm(hu.uniform_desc(), 1.0, op, xh, yo) == 0
        assert relerr(y.cpu().numpy(), yo) <= TOL
    Wu.free()
    U.free()
    # mixed FP32/FP16 store, 8 vectors: the workspace carries the 8-vector
    # kernels' scratch; against the handle's own workspace the result is
    # bit-identical (same kernels, same order)
    hm = built("exp3d_16384", lambda: hlr.build(hlr.Problem.exp3d(16384)))
    M = hlr.upload(hm, precision="mixed", max_nrhs=8)
    W = hlr.Workspace(M, max_nrhs=8)
    X = _colmajor(np.random.default_rng(3).standard_normal((hm.n, 8)))
    Y1, Y2 = _colmajor(np.zeros((hm.n, 8))), _colmajor(np.zeros((hm.n, 8)))
    hlr.mul_vec(1.0, 0, M, X, Y1)
    hlr.mul_vec(1.0, 0, M, X, Y2, workspace=W)
    torch.cuda.synchronize()
    assert torch.equal(Y1, Y2)
    W.free()
    M.free()


def test_workspace_too_small_for_another_handle_is_rejected():
    small = built("c1_small", lambda: hlr.build(hlr.Problem.log1d(2048)))
    big = built("exp3d_16384", lambda: hlr.build(hlr.Problem.exp3d(16384)))
    Ms, Mb = hlr.upload(small), hlr.upload(big)
    W = hlr.Workspace(Ms)
    x = torch.ones(big.n, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    with pytest.raises(HLRCError, match="too small"):
        hlr.mul_vec(1.0, 0, Mb, x, y, workspace=W)
    W.free()
    Ms.free()
    Mb.free()
