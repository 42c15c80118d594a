"""Multi-right-hand-side products of reduced-precision stores (16-bit chunks
and block-floating-point byte planes on FP16 tensor cores, FP32 chunks on
FP64 tensor cores) against the FP64 oracle and against the single-vector
reduced-precision product of the same store.

The tensor-core path splits each vector entry into two 16-bit terms, so it
differs from the single-vector path (FP32 vector) only by about 2^-22
(FP16) or 2^-17 (BF16) relative; layout mistakes would show as O(1)
differences."""
import numpy as np
import pytest

import hlr_b200 as hlr
import oracle

from conftest import built, relerr

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL = {"f32": 1e-6, "mixed": 1e-6, "f16": 2e-3, "bf16": 1.5e-2, "bfp": 1e-6}
# FP16 / BF16 handles uploaded with max_nrhs > 8 take the 64-vector kernels
# for more than 8 vectors, which sum a whole output tile in FP32
SAME_STORE = {"f32": 1e-6, "mixed": 2e-6, "f16": 2e-5, "bf16": 1e-4, "bfp": 1e-6}


def colmajor_dev(A):
    return torch.from_numpy(np.ascontiguousarray(A.T)).cuda().T


def matrices():
    return {
        "exp3d_5000_48": built("exp3d_5000_48", lambda: hlr.build(hlr.Problem.exp3d(5000, leaf_size=48))),
        "exp3d_16384_64": built("exp3d_16384_64", lambda: hlr.build(hlr.Problem.exp3d(16384))),
    }


@pytest.mark.parametrize("name", ["exp3d_5000_48", "exp3d_16384_64"])
@pytest.mark.parametrize("prec", ["mixed", "f16", "bf16", "f32", "bfp"])
@pytest.mark.parametrize("op", [0, 1])
def test_multi_rhs_reduced_precision(name, prec, op):
    hm = matrices()[name]
    M = hlr.upload(hm, precision=prec, max_nrhs=16)
    nrhs = 11
    rng = np.random.default_rng(90 + op)
    X = rng.standard_normal((hm.n, nrhs))
    Yd = colmajor_dev(np.zeros((hm.n, nrhs)))
    l0 = M.launch_count()
    hlr.mul_vec(1.0, op, M, colmajor_dev(X), Yd)
    torch.cuda.synchronize()
    # two blocks of 8 vectors, each a handful of grids (a loop of one-vector
    # products would take 11 times the one-vector launches)
    assert M.launch_count() - l0 <= 2 * 11
    Y = Yd.cpu().numpy()
    for j in (0, 5, 8, 10):
        yref = np.zeros(hm.n)
        oracle.hmvm_seq(hm.h_desc(), 1.0, op, X[:, j].copy(), yref)
        assert relerr(Y[:, j], yref) <= TOL[prec], (prec, op, j)
        ys = torch.zeros(hm.n, dtype=torch.float64, device="cuda")
        hlr.mul_vec(1.0, op, M, torch.from_numpy(X[:, j].copy()).cuda(), ys)
        torch.cuda.synchronize()
        assert relerr(Y[:, j], ys.cpu().numpy()) <= SAME_STORE[prec], (prec, op, j)
    assert M.device_error() == 0
    M.free()


@pytest.mark.parametrize("prec", ["mixed", "f16", "bf16", "bfp"])
def test_each_rhs_is_scaled_on_its_own(prec):
    """Right-hand sides of very different magnitude in one block: each one
    keeps its own relative accuracy (per-vector power-of-two scales on the
    16-bit path; FP32 chunks convert the vector to FP32, so magnitudes stay
    inside its range)."""
    hm = matrices()["exp3d_5000_48"]
    M = hlr.upload(hm, precision=prec, max_nrhs=8)
    rng = np.random.default_rng(95)
    mags = np.array([1.0, 1e-12, 1e9, 3e-25, 1e20, 1.0, 1e-5, 7.0])
    X = rng.standard_normal((hm.n, 8)) * mags
    Yd = colmajor_dev(np.zeros((hm.n, 8)))
    hlr.mul_vec(1.0, 0, M, colmajor_dev(X), Yd)
    torch.cuda.synchronize()
    Y = Yd.cpu().numpy()
    for j in range(8):
        yref = np.zeros(hm.n)
        oracle.hmvm_seq(hm.h_desc(), 1.0, 0, X[:, j].copy(), yref)
        assert np.all(np.isfinite(Y[:, j])), j
        assert relerr(Y[:, j], yref) <= TOL[prec], (prec, j, mags[j])
    M.free()


def test_multi_rhs_exactly_representable_known_answer():
    rng = np.random.default_rng(96)
    n = 40
    ll = hlr.LeafList(n, n)
    h = 24
    D0 = rng.integers(-8, 9, (h, h)).astype(float)
    D1 = rng.integers(-8, 9, (n - h, n - h)).astype(float)
    U = rng.integers(-4, 5, (h, 3)).astype(float)
    V = rng.integers(-4, 5, (n - h, 3)).astype(float)
    U2 = rng.integers(-4, 5, (n - h, 2)).astype(float)
    V2 = rng.integers(-4, 5, (h, 2)).astype(float)
    ll.add_dense(0, 0, D0)
    ll.add_lowrank(0, h, U, V)
    ll.add_lowrank(h, 0, U2, V2)
    ll.add_dense(h, h, D1)
    A = np.zeros((n, n))
    A[:h, :h], A[:h, h:], A[h:, :h], A[h:, h:] = D0, U @ V.T, U2 @ V2.T, D1
    X = rng.integers(-3, 4, (n, 8)).astype(float)
    for prec in ("f16", "bf16", "mixed", "f32", "bfp"):
        M = hlr.upload(ll, precision=prec, max_nrhs=8)
        for op, Aop in ((0, A), (1, A.T)):
            Yd = colmajor_dev(np.zeros((n, 8)))
            hlr.mul_vec(1.0, op, M, colmajor_dev(X), Yd)
            torch.cuda.synchronize()
            np.testing.assert_allclose(Yd.cpu().numpy(), Aop @ X, rtol=0, atol=1e-9, err_msg=f"{prec} op {op}")
        M.free()
