"""Shapes the built test matrices do not produce: rectangular operators,
tiny matrices, leaves taller and wider than a tile (split into several
tiles), rank-0 blocks and empty right-hand-side counts, in every storage
precision and on both the single-vector and the 8-vector paths."""
import numpy as np
import pytest

import hlr_b200 as hlr

from conftest import relerr

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-13, "f32": 1e-6, "mixed": 1e-6, "f16": 2e-3, "bf16": 1.5e-2, "bfp": 1e-6}
# the 8-vector BFP kernels accumulate byte-plane products on the FP16 tensor
# cores in FP32 per 32-column stage: about 1e-7 on top of the store's own
# error, which VALR sets near 1e-6 on these random leaves
TOL8 = dict(TOL, bfp=2e-6)


def leaves(nrows, ncols, seed):
    """A 2 x 3 block partition of an nrows x ncols operator: dense leaves,
    low-rank leaves of ranks 0..5 and one leaf wider than a tile."""
    rng = np.random.default_rng(seed)
    r = [0, nrows // 3, nrows]
    c = [0, ncols // 4, ncols // 2, ncols]
    ll = hlr.LeafList(nrows, ncols)
    A = np.zeros((nrows, ncols))
    k = 0
    for i in range(2):
        for j in range(3):
            m, n = r[i + 1] - r[i], c[j + 1] - c[j]
            if m == 0 or n == 0:
                continue
            if (i + j) % 2 == 0:
                D = rng.standard_normal((m, n))
                ll.add_dense(r[i], c[j], D)
                A[r[i]:r[i + 1], c[j]:c[j + 1]] = D
            else:
                rank = k % 6
                U = rng.standard_normal((m, rank))
                V = rng.standard_normal((n, rank))
                ll.add_lowrank(r[i], c[j], U, V)
                A[r[i]:r[i + 1], c[j]:c[j + 1]] = U @ V.T
            k += 1
    return ll, A


@pytest.mark.parametrize("shape", [(1, 1), (3, 7), (70, 33), (200, 130), (130, 200), (257, 257)])
@pytest.mark.parametrize("prec", ["f64", "mixed", "f16", "bf16", "f32", "bfp"])
def test_rectangular_and_tiny(shape, prec):
    nrows, ncols = shape
    ll, A = leaves(nrows, ncols, seed=nrows * 1000 + ncols)
    M = hlr.upload(ll, precision=prec, max_nrhs=8)
    rng = np.random.default_rng(7)
    for op, Aop in ((0, A), (1, A.T)):
        nx, ny = Aop.shape[1], Aop.shape[0]
        x = rng.standard_normal(nx)
        y0 = rng.standard_normal(ny)
        y = torch.from_numpy(y0.copy()).cuda()
        hlr.mul_vec(0.5, op, M, torch.from_numpy(x).cuda(), y)
        torch.cuda.synchronize()
        ref = 0.5 * (Aop @ x)
        assert relerr(y.cpu().numpy() - y0, ref) <= TOL[prec] or np.linalg.norm(ref) == 0, (prec, op)
        # eight vectors at once
        X = rng.standard_normal((nx, 8))
        Xd = torch.from_numpy(np.ascontiguousarray(X.T)).cuda().T
        Yd = torch.zeros((8, ny), dtype=torch.float64, device="cuda").T
        hlr.mul_vec(1.0, op, M, Xd, Yd)
        torch.cuda.synchronize()
        R = Aop @ X
        for j in range(8):
            if np.linalg.norm(R[:, j]) > 0:
                assert relerr(Yd[:, j].cpu().numpy(), R[:, j]) <= TOL8[prec], (prec, op, j)
    assert M.device_error() == 0
    M.free()


def test_zero_vectors_and_alpha_zero_on_multi_rhs():
    ll, A = leaves(130, 200, seed=3)
    M = hlr.upload(ll, precision="mixed", max_nrhs=8)
    X = torch.zeros((8, 200), dtype=torch.float64, device="cuda").T     # column-major (200, 8)
    Y = torch.ones((8, 130), dtype=torch.float64, device="cuda").T
    hlr.mul_vec(1.0, 0, M, X, Y)            # zero input: y unchanged
    hlr.mul_vec(0.0, 0, M, torch.ones((8, 200), dtype=torch.float64, device="cuda").T, Y)   # alpha = 0
    torch.cuda.synchronize()
    assert float((Y - 1.0).abs().max()) == 0.0
    M.free()
