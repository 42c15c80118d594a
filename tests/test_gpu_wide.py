"""One-pass 64-vector products of 16-bit (FP16 / BF16) H-matrix stores on
the tcgen05 tensor cores (kernels_wide.cuh): the matrix is streamed once per
64 right-hand sides, the block apply of lrmatrix::apply_add on a multi-vector
(include/hlr/matrix/lrmatrix.hh:681-746) over all leaves at once.

Checked against the FP64 oracle (to the store's own accuracy), against the
8-vector tensor-core kernels and the one-vector kernels on the same store:
the vector split keeps about 22 bits (FP16) or 16 bits (BF16) and the
full-tile N-form accumulates a whole output tile's run in FP32 (FP64 y), so
the paths agree to 2e-5 / 1e-4, far inside the store's own error (2e-3 /
1.5e-2); a layout mistake shows as an O(1) difference."""
import numpy as np
import pytest

import hlr_b200 as hlr
import oracle
from hlr_b200 import _capi

from conftest import built, relerr

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL = {"f16": 2e-3, "bf16": 1.5e-2}            # against the FP64 oracle
SAME_STORE = {"f16": 2e-5, "bf16": 1e-4}       # against the other kernels on the same store


def colmajor_dev(A):
    return torch.from_numpy(np.ascontiguousarray(A.T)).cuda().T


MATS = {
    # ragged 48-row tiles
    "exp3d_5000_48": lambda: hlr.build(hlr.Problem.exp3d(5000, leaf_size=48)),
    # full 64-row tiles, blocks spanning many column tiles (two-level finish)
    "exp3d_16384_64": lambda: hlr.build(hlr.Problem.exp3d(16384)),
    "log1d_8192": lambda: hlr.build(hlr.Problem.log1d(8192)),
    # 64-row and 32/33-row tiles: the TMA kernels and the cp.async kernels in one product
    "exp3d_8200_64": lambda: hlr.build(hlr.Problem.exp3d(8200)),
}


def _product(M, X, alpha=1.0, y0=None):
    Yd = colmajor_dev(np.zeros_like(X) if y0 is None else y0)
    hlr.mul_vec(alpha, hlr.apply_normal, M, colmajor_dev(X), Yd)
    torch.cuda.synchronize()
    return Yd.cpu().numpy()


def _uses_wide(M, X):
    M.set_profiling(True)
    M.last_profile()
    _product(M, X)
    names = set(M.last_profile())
    M.set_profiling(False)
    return "wide_xsplit" in names


@pytest.mark.parametrize("name", list(MATS))
@pytest.mark.parametrize("prec", ["f16", "bf16"])
@pytest.mark.parametrize("nrhs", [64, 100, 12])
def test_wide_against_oracle_and_other_kernels(name, prec, nrhs):
    hm = built(name, MATS[name])
    M = hlr.upload(hm, precision=prec, max_nrhs=nrhs)
    assert M.tuning["wide_min_nrhs"] == 9
    rng = np.random.default_rng(7 + nrhs)
    X = rng.standard_normal((hm.n, nrhs)) * rng.uniform(0.1, 10.0, nrhs)   # vectors of different scales
    assert _uses_wide(M, X)
    Y0 = rng.standard_normal((hm.n, nrhs))
    Yw = _product(M, X, alpha=-1.5, y0=Y0) - Y0
    M.set_tuning(wide_min_nrhs=_capi.HLRC_MR_NEVER)          # the 8-vector kernels
    assert not _uses_wide(M, X)
    Y8 = _product(M, X, alpha=-1.5, y0=Y0) - Y0
    for j in sorted({0, 1, nrhs // 2, nrhs - 1, min(nrhs - 1, 63)}):
        assert relerr(Yw[:, j], Y8[:, j]) <= SAME_STORE[prec], (name, prec, j, "8-vector")
        yref = np.zeros(hm.n)
        oracle.hmvm_seq(hm.h_desc(), -1.5, 0, X[:, j].copy(), yref)
        assert relerr(Yw[:, j], yref) <= TOL[prec], (name, prec, j, "oracle")
    # one vector on the same store
    ys = torch.zeros(hm.n, dtype=torch.float64, device="cuda")
    hlr.mul_vec(-1.5, 0, M, torch.from_numpy(X[:, 1].copy()).cuda(), ys)
    torch.cuda.synchronize()
    assert relerr(Yw[:, 1], ys.cpu().numpy()) <= SAME_STORE[prec]
    assert M.device_error() == 0
    M.free()


def test_wide_zero_and_tiny_vectors():
    """A zero vector stays zero, and vectors far below 1 keep their accuracy
    (the per-vector scales are powers of two)."""
    hm = built("exp3d_16384_64", MATS["exp3d_16384_64"])
    M = hlr.upload(hm, precision="f16", max_nrhs=64)
    rng = np.random.default_rng(3)
    X = rng.standard_normal((hm.n, 64))
    X[:, 5] = 0.0
    X[:, 6] *= 1e-30
    X[:, 7] *= 1e25
    Y = _product(M, X)
    assert np.all(Y[:, 5] == 0.0)
    for j in (6, 7, 8):
        yref = np.zeros(hm.n)
        oracle.hmvm_seq(hm.h_desc(), 1.0, 0, X[:, j].copy(), yref)
        assert relerr(Y[:, j], yref) <= TOL["f16"], j
    assert M.device_error() == 0
    M.free()


def test_wide_deterministic_graph_host_and_workspace():
    hm = built("exp3d_5000_48", MATS["exp3d_5000_48"])
    M = hlr.upload(hm, precision="f16", max_nrhs=64)
    X = np.random.default_rng(4).standard_normal((hm.n, 64))
    Y1 = _product(M, X)
    Y2 = _product(M, X)
    assert np.array_equal(Y1, Y2)          # fixed order: bit-identical
    # captured in a CUDA graph and replayed
    Xd, Yd = colmajor_dev(X), colmajor_dev(np.zeros_like(X))
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        hlr.mul_vec(1.0, 0, M, Xd, Yd)     # warm-up outside the capture
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    Yd.zero_()
    with torch.cuda.graph(g):
        hlr.mul_vec(1.0, 0, M, Xd, Yd)
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    assert np.array_equal(Yd.cpu().numpy(), 2 * Y1) or relerr(Yd.cpu().numpy(), 2 * Y1) <= 1e-15
    del g
    # host buffers (copies inside)
    Xh = np.asfortranarray(X)
    Yh = np.asfortranarray(np.zeros_like(X))
    hlr.mul_vec(1.0, 0, M, Xh, Yh)
    assert np.array_equal(Yh, Y1)
    # a workspace of its own
    W = hlr.Workspace(M, max_nrhs=64)
    Yw = colmajor_dev(np.zeros_like(X))
    hlr.mul_vec(1.0, 0, M, colmajor_dev(X), Yw, workspace=W)
    torch.cuda.synchronize()
    assert np.array_equal(Yw.cpu().numpy(), Y1)
    W.free()
    assert M.device_error() == 0
    M.free()
