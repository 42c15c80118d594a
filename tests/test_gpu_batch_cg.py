"""Batched handles (many matrices, one launch per pass) and the batched CG
with FP64 iterative refinement."""
import numpy as np
import pytest

import hlr_b200 as hlr
import oracle
from hlr_b200.solve import cg_refine

from conftest import built, relerr

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def members():
    return [
        built("b_exp_1000", lambda: hlr.build(hlr.Problem.exp3d(1000, ell=0.1, seed=1000))),
        built("b_exp_1500", lambda: hlr.build(hlr.Problem.exp3d(1500, ell=0.05, seed=1001))),
        built("b_exp_700", lambda: hlr.build(hlr.Problem.exp3d(700, ell=0.2, seed=1002))),
    ]


@pytest.mark.parametrize("pad", [None, 1536])
@pytest.mark.parametrize("op", [0, 1])
def test_batched_product_matches_members(pad, op):
    ms = members()
    B = hlr.upload_batch(ms, max_nrhs=8, pad_to=pad)
    N = B.offsets[-1]
    rng = np.random.default_rng(80)
    nrhs = 3
    X = np.zeros((nrhs, N))
    for i, m in enumerate(ms):
        X[:, B.offsets[i]:B.offsets[i] + m.n] = rng.standard_normal((nrhs, m.n))
    Xd = torch.from_numpy(X).cuda()
    Yd = torch.zeros_like(Xd)
    hlr.mul_vec(1.0, op, B, Xd.T, Yd.T)
    torch.cuda.synchronize()
    Y = Yd.cpu().numpy()
    for i, m in enumerate(ms):
        o = B.offsets[i]
        for j in range(nrhs):
            yref = np.zeros(m.n)
            oracle.hmvm_seq(m.h_desc(), 1.0, op, X[j, o:o + m.n].copy(), yref)
            assert relerr(Y[j, o:o + m.n], yref) < 1e-13, (i, j)
    if pad is not None:  # padding rows untouched
        for i, m in enumerate(ms):
            assert np.all(Y[:, B.offsets[i] + m.n:B.offsets[i + 1]] == 0)
    B.free()


def test_batch_rejects_too_small_padding():
    with pytest.raises(ValueError):
        hlr.upload_batch(members(), pad_to=800)  # 1000 and 1500 do not fit in 800


@pytest.mark.parametrize("inner", ["f64", "mixed"])
def test_cg_refinement_reaches_1e10(inner):
    ms = members()
    pad = 1536
    A64 = hlr.upload_batch(ms, precision="f64", max_nrhs=8, pad_to=pad)
    Alow = A64 if inner == "f64" else hlr.upload_batch(ms, precision=inner, max_nrhs=8, pad_to=pad)
    nrhs, count = 4, len(ms)
    rng = np.random.default_rng(81)
    b = np.zeros((nrhs, count * pad))
    for i, m in enumerate(ms):
        b[:, i * pad:i * pad + m.n] = rng.standard_normal((nrhs, m.n))
    bt = torch.from_numpy(b).cuda()
    res = cg_refine(A64, Alow, bt, count, pad, tol=1e-10, check_every=10)
    assert bool(res.converged.all()), res.history
    assert float(res.rel_residual.max()) <= 1e-10
    # independent check of one system with the oracle's FP64 product
    x = res.x.cpu().numpy()
    m = ms[1]
    o = pad
    r = b[2, o:o + m.n].copy()
    oracle.hmvm_seq(m.h_desc(), -1.0, 0, x[2, o:o + m.n].copy(), r)
    assert np.linalg.norm(r) / np.linalg.norm(b[2, o:o + m.n]) <= 1e-10
    # padding stays zero
    assert np.all(x[:, m.n + o:2 * pad] == 0)


def test_cg_reports_stall_for_too_coarse_inner_operator():
    """BF16 storage (relative error ~2e-3) cannot refine systems with
    kappa * 2e-3 > 1: the solver stops and reports them unconverged instead
    of looping."""
    ms = [built("b_exp_700_ill", lambda: hlr.build(hlr.Problem.exp3d(700, ell=0.3, nugget=1e-6, seed=7)))]
    pad = 704
    A64 = hlr.upload_batch(ms, precision="f64", max_nrhs=8, pad_to=pad)
    Alow = hlr.upload_batch(ms, precision="bf16", max_nrhs=8, pad_to=pad)
    b = torch.zeros((1, pad), dtype=torch.float64, device="cuda")
    b[0, :700] = torch.from_numpy(np.random.default_rng(3).standard_normal(700)).cuda()
    res = cg_refine(A64, Alow, b, 1, pad, tol=1e-10, max_outer=8, max_inner=2000, check_every=10)
    assert res.outer_iterations <= 8
    assert len(res.history) >= 1


@pytest.mark.parametrize("inner", ["f64", "mixed"])
def test_block_jacobi_preconditioned_cg(inner):
    """PCG with the block-Jacobi preconditioner (dense inverses of the
    256 x 256 diagonal blocks, applied by the product kernels): the same
    1e-10 solution as plain CG, in fewer inner iterations."""
    from hlr_b200.solve import block_jacobi_batch
    ms = members()
    pad = 1536
    A64 = hlr.upload_batch(ms, precision="f64", max_nrhs=8, pad_to=pad)
    Alow = A64 if inner == "f64" else hlr.upload_batch(ms, precision=inner, max_nrhs=8, pad_to=pad)
    W = block_jacobi_batch(ms, pad, block=256, precision="f64" if inner == "f64" else "f32", max_nrhs=8)
    nrhs, count = 4, len(ms)
    rng = np.random.default_rng(82)
    b = np.zeros((nrhs, count * pad))
    for i, m in enumerate(ms):
        b[:, i * pad:i * pad + m.n] = rng.standard_normal((nrhs, m.n))
    bt = torch.from_numpy(b).cuda()
    plain = cg_refine(A64, Alow, bt, count, pad, tol=1e-10, check_every=5)
    pre = cg_refine(A64, Alow, bt, count, pad, tol=1e-10, check_every=5, precond=W)
    assert bool(pre.converged.all()), pre.history
    assert float(pre.rel_residual.max()) <= 1e-10
    assert pre.inner_iterations < plain.inner_iterations, (pre.inner_iterations, plain.inner_iterations)
    assert relerr(pre.x.cpu().numpy(), plain.x.cpu().numpy()) <= 1e-8
