"""Reduced-precision storage on the GPU (FP32, scaled FP16 / BF16, and the
VALR-style mixed FP32/FP16 form) against the FP64 oracle.

Tolerances (relative 2-norm error of y against the FP64 oracle product on
the same matrix, x ~ N(0,1)):
  f32    <= 1e-6   (storage unit roundoff 6e-8)
  mixed  <= 1e-6   (VALR: FP16 only for columns with sigma_l small enough)
  f16    <= 2e-3   (unit roundoff 4.9e-4)
  bf16   <= 1.5e-2 (unit roundoff 3.9e-3)
  bfp    <= 1e-6   (VALR: 16-bit block floating point for columns whose bit
                    rate is at most 15, 24-bit for the rest and the dense leaves)
"""
import numpy as np
import pytest

import hlr_b200 as hlr
import oracle

from conftest import built, relerr

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL = {"f32": 1e-6, "mixed": 1e-6, "f16": 2e-3, "bf16": 1.5e-2, "bfp": 1e-6}


def gpu(M, alpha, op, x, y0):
    y = torch.from_numpy(y0.copy()).cuda()
    hlr.mul_vec(alpha, op, M, torch.from_numpy(x).cuda(), y)
    torch.cuda.synchronize()
    return y.cpu().numpy()


@pytest.mark.parametrize("prec", ["f32", "mixed", "f16", "bf16", "bfp"])
@pytest.mark.parametrize("op", [0, 1])
def test_exp3d_reduced_precision_error(prec, op):
    hm = built("exp3d_16384_64", lambda: hlr.build(hlr.Problem.exp3d(16384)))
    M = hlr.upload(hm, precision=prec)
    assert M.info["precision"] == hlr.PRECISIONS[prec]
    x = np.random.default_rng(12).standard_normal(hm.n)
    y = gpu(M, 1.0, op, x, np.zeros(hm.n))
    yref = np.zeros(hm.n)
    oracle.hmvm_seq(hm.h_desc(), 1.0, op, x, yref)
    err = relerr(y, yref)
    assert err <= TOL[prec], (prec, op, err)
    M.free()


@pytest.mark.parametrize("prec", ["f32", "mixed", "f16", "bfp"])
def test_log1d_reduced_precision_error(c1, prec):
    M = hlr.upload(c1, precision=prec)
    x = np.random.default_rng(13).standard_normal(c1.n)
    y = gpu(M, 2.0, 0, x, np.zeros(c1.n))
    yref = np.zeros(c1.n)
    oracle.hmvm_seq(c1.h_desc(), 2.0, 0, x, yref)
    assert relerr(y, yref) <= TOL[prec]
    M.free()


def test_mixed_is_deterministic_and_accumulates_in_fp64():
    hm = built("exp3d_16384_64", lambda: hlr.build(hlr.Problem.exp3d(16384)))
    M = hlr.upload(hm, precision="mixed")
    x = torch.from_numpy(np.random.default_rng(14).standard_normal(hm.n)).cuda()
    outs = []
    for _ in range(2):
        y = torch.full((hm.n,), 1e8, dtype=torch.float64, device="cuda")
        hlr.mul_vec(1.0, 0, M, x, y)
        torch.cuda.synchronize()
        outs.append(y.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    # y is accumulated in FP64: an FP32 accumulation of 1e8 + O(30) would lose the low digits
    ydelta = outs[0] - 1e8
    y0 = torch.zeros(hm.n, dtype=torch.float64, device="cuda")
    hlr.mul_vec(1.0, 0, M, x, y0)
    assert relerr(ydelta, y0.cpu().numpy()) < 1e-7
    M.free()


def test_exactly_representable_known_answer():
    """Small integers are exact in every format: the reduced-precision product
    equals the FP64 one to rounding of the FP32 chunk sums."""
    rng = np.random.default_rng(15)
    ll = hlr.LeafList(6, 6)
    D0 = rng.integers(-8, 9, (3, 3)).astype(float)
    D1 = rng.integers(-8, 9, (3, 3)).astype(float)
    U = rng.integers(-4, 5, (3, 2)).astype(float)
    V = rng.integers(-4, 5, (3, 2)).astype(float)
    ll.add_dense(0, 0, D0)
    ll.add_lowrank(0, 3, U, V)
    ll.add_lowrank(3, 0, np.zeros((3, 0)), np.zeros((3, 0)))
    ll.add_dense(3, 3, D1)
    A = np.zeros((6, 6))
    A[:3, :3], A[:3, 3:], A[3:, 3:] = D0, U @ V.T, D1
    x = rng.integers(-3, 4, 6).astype(float)
    for prec in ("f32", "f16", "bf16", "mixed", "bfp"):
        M = hlr.upload(ll, precision=prec)
        for op, Aop in ((0, A), (1, A.T)):
            np.testing.assert_allclose(gpu(M, 1.0, op, x, np.zeros(6)), Aop @ x, rtol=0, atol=1e-9)
        M.free()
