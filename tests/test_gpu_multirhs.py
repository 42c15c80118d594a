"""Blocked multi-right-hand-side products (matrix streamed once per 8
vectors) against the per-vector oracle, FP64 tolerance 1e-13."""
import numpy as np
import pytest

import hlr_b200 as hlr
import oracle

from conftest import built, relerr

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL = 1e-13


def colmajor_dev(A):
    """(n, k) float64 CUDA tensor with stride (1, n)."""
    return torch.from_numpy(np.ascontiguousarray(A.T)).cuda().T


@pytest.mark.parametrize("nrhs", [2, 8, 13, 32])
@pytest.mark.parametrize("op", [0, 1])
def test_h_multi_rhs(nrhs, op):
    hm = built("exp3d_5000_48", lambda: hlr.build(hlr.Problem.exp3d(5000, leaf_size=48)))
    M = hlr.upload(hm, max_nrhs=32)
    rng = np.random.default_rng(40 + nrhs)
    X = rng.standard_normal((hm.n, nrhs))
    Y0 = rng.standard_normal((hm.n, nrhs))
    Xd, Yd = colmajor_dev(X), colmajor_dev(Y0)
    hlr.mul_vec(0.5, op, M, Xd, Yd)
    torch.cuda.synchronize()
    Y = Yd.cpu().numpy()
    for j in range(nrhs):
        yref = Y0[:, j].copy()
        oracle.hmvm_seq(hm.h_desc(), 0.5, op, X[:, j].copy(), yref)
        assert relerr(Y[:, j] - Y0[:, j], yref - Y0[:, j]) < TOL, (op, j)
    M.free()


def test_h_multi_rhs_padded_leading_dimension(c1):
    M = hlr.upload(c1, max_nrhs=8)
    rng = np.random.default_rng(50)
    ld = c1.n + 7
    Xb = torch.zeros((5, ld), dtype=torch.float64, device="cuda")
    Yb = torch.zeros((5, ld), dtype=torch.float64, device="cuda")
    X = rng.standard_normal((c1.n, 5))
    Xb[:, : c1.n] = torch.from_numpy(X.T.copy()).cuda()
    Xd = Xb.T[: c1.n]  # (n, 5) with stride (1, ld)
    Yd = Yb.T[: c1.n]
    hlr.mul_vec(1.0, 0, M, Xd, Yd)
    torch.cuda.synchronize()
    for j in range(5):
        yref = np.zeros(c1.n)
        oracle.hmvm_seq(c1.h_desc(), 1.0, 0, X[:, j].copy(), yref)
        assert relerr(Yd[:, j].cpu().numpy(), yref) < TOL
    # the padding rows beyond n were not touched
    assert float(Yb[:, c1.n:].abs().max()) == 0.0
    M.free()


@pytest.mark.parametrize("op", [0, 2])
def test_uniform_multi_rhs(op):
    hm = built("sphere5u", lambda: hlr.build(hlr.Problem.laplace_sphere(refine=5, uniform=True)))
    M = hlr.upload(hm, max_nrhs=32)
    rng = np.random.default_rng(60)
    X = rng.standard_normal((hm.n, 32))
    Yd = colmajor_dev(np.zeros((hm.n, 32)))
    hlr.uniform.mul_vec(1.0, op, M, colmajor_dev(X), Yd)
    torch.cuda.synchronize()
    Y = Yd.cpu().numpy()
    for j in (0, 7, 8, 31):
        yref = np.zeros(hm.n)
        assert oracle.uniform_mvm(hm.uniform_desc(), 1.0, op, X[:, j].copy(), yref) == 0
        assert relerr(Y[:, j], yref) < TOL, (op, j)
    M.free()


def test_multi_rhs_host_path():
    hm = built("exp3d_5000_48", lambda: hlr.build(hlr.Problem.exp3d(5000, leaf_size=48)))
    M = hlr.upload(hm, max_nrhs=16)
    rng = np.random.default_rng(70)
    X = np.asfortranarray(rng.standard_normal((hm.n, 16)))
    Y = np.zeros((hm.n, 16), order="F")
    hlr.mul_vec(2.0, 0, M, X, Y)
    for j in (0, 9, 15):
        yref = np.zeros(hm.n)
        oracle.hmvm_seq(hm.h_desc(), 2.0, 0, X[:, j].copy(), yref)
        assert relerr(Y[:, j], yref) < TOL
    M.free()
