"""The near field of a one-vector product as its own pass on a side stream
(hlrc_options.near_field = 2, the default).

HLR sums every block of a row into y (tbb/detail/arith.hh:95-124); here the
dense leaves' D x is one pass and the low-rank part another, both per row
tile, D x first.  With the split, D x is launched on the workspace's side
stream, forked from the caller's stream at the start of the product and
joined before the pass that adds the low-rank part, so it runs beside the
dependent low-rank passes.  Checked: the split and the fused product against
the oracle and against each other (summation order only); direct launches,
programmatic dependent launch, CUDA graph replays, a workspace of the caller
on another stream and the no-alloc entry point (side stages in line on the
caller's stream) give identical bits; graph replays profile the side pass."""
import ctypes as C

import numpy as np
import pytest

import hlr_b200 as hlr
import oracle
from hlr_b200 import _capi

from conftest import built, relerr

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

CASES = {
    "h": lambda: built("c2_small", lambda: hlr.build(hlr.Problem.exp3d(4096))),
    "uniform": lambda: built("c3_small", lambda: hlr.build(hlr.Problem.laplace_sphere(refine=4, uniform=True))),
    "h2": lambda: built("sphere5_h2", lambda: hlr.build(hlr.Problem.laplace_sphere(refine=5, nested=True))),
}


def _upload(hm, kind, near_field):
    return hlr.upload(hm, uniform=(kind == "uniform"), h2=(kind == "h2"), plan={"near_field": near_field})


def _oracle(hm, kind, alpha, op, x, y0):
    y = y0.copy()
    if kind == "h2":
        assert oracle.h2_mvm(hm.h2_desc(), alpha, op, x, y) == 0
    elif kind == "uniform":
        assert oracle.uniform_mvm(hm.uniform_desc(), alpha, op, x, y) == 0
    else:
        oracle.hmvm_seq(hm.h_desc(), alpha, op, x, y)
    return y


@pytest.mark.parametrize("kind", sorted(CASES))
def test_side_and_fused_near_field_match_the_oracle(kind):
    hm = CASES[kind]()
    M1, M2 = _upload(hm, kind, 1), _upload(hm, kind, 2)
    assert M2.info["launches"][0] == M1.info["launches"][0] + 1   # D x is its own pass
    rng = np.random.default_rng(8)
    for op in (0, 2):
        xh, y0 = rng.standard_normal(hm.n), rng.standard_normal(hm.n)
        x = torch.from_numpy(xh).cuda()
        ys = []
        for M in (M1, M2):
            y = torch.from_numpy(y0.copy()).cuda()
            hlr.mul_vec(1.25, op, M, x, y)
            torch.cuda.synchronize()
            ys.append(y.cpu().numpy() - y0)
        yo = _oracle(hm, kind, 1.25, op, xh, y0) - y0
        for y in ys:
            assert relerr(y, yo) <= 1e-13, (kind, op)
        assert relerr(ys[0], ys[1]) <= 1e-14, (kind, op)
        if op == 2:   # op C has no side stage: the same passes
            assert np.array_equal(ys[0], ys[1])
    M1.free()
    M2.free()


def _noalloc(M, alpha, op, x, y):
    L = _capi.lib()
    st = L.hlrc_mvm_noalloc(M.handle, float(alpha), int(op), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, L.hlrc_last_error().decode()


@pytest.mark.parametrize("kind", ["uniform", "h2", "h"])
def test_side_stream_products_are_bit_identical_on_every_path(kind):
    hm = CASES[kind]()
    M = _upload(hm, kind, 2)
    x = torch.from_numpy(np.random.default_rng(3).standard_normal(hm.n)).cuda()
    alphas = [0.5 + k for k in range(8)]

    def chain(overlap, graph, workspace=None, stream=None):
        M.set_tuning(overlap=overlap)
        y = torch.zeros_like(x)
        st = stream or torch.cuda.current_stream()
        st.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(st):
            if not graph:
                for a in alphas:
                    hlr.mul_vec(a, 0, M, x, y, workspace=workspace)
            else:
                hlr.mul_vec(1.0, 0, M, x, y, workspace=workspace)   # warm-up outside the graph
                torch.cuda.synchronize()
                y.zero_()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):
                    for a in alphas:
                        hlr.mul_vec(a, 0, M, x, y, workspace=workspace)
                g.replay()
                torch.cuda.synchronize()
                del g
        torch.cuda.synchronize()
        return y.cpu().numpy()

    plain = chain(0, False)
    assert np.array_equal(chain(1, False), plain)
    assert np.array_equal(chain(1, True), plain)
    assert np.array_equal(chain(0, True), plain)
    W = hlr.Workspace(M)
    other = torch.cuda.Stream()
    assert np.array_equal(chain(1, False, W, other), plain)
    assert np.array_equal(chain(1, True, W, other), plain)
    # the side pass forked later (after 1..3 other passes, clamped before
    # the pass that joins it): the same kernels in the same order on y
    for k in (1, 2, 3, 16):
        M.set_tuning(side_at=k)
        assert np.array_equal(chain(1, True), plain), k
        assert np.array_equal(chain(1, False, W, other), plain), k
    M.set_tuning(side_at=0)
    # the no-alloc entry point has no side stream: D x runs first in line
    y = torch.zeros_like(x)
    for a in alphas:
        _noalloc(M, a, 0, x, y)
    torch.cuda.synchronize()
    assert np.array_equal(y.cpu().numpy(), plain)
    yo = _oracle(hm, kind, sum(alphas), 0, x.cpu().numpy(), np.zeros(hm.n))
    assert relerr(plain, yo) <= 1e-13
    assert M.device_error() == 0
    W.free()
    M.free()


@pytest.mark.parametrize("kind", ["uniform", "h2"])
def test_graph_replay_profiles_the_side_pass(kind):
    hm = CASES[kind]()
    M = _upload(hm, kind, 0)   # the default: near field on the side stream
    x = torch.from_numpy(np.random.default_rng(4).standard_normal(hm.n)).cuda()
    y = torch.zeros_like(x)
    hlr.mul_vec(1.0, 0, M, x, y)
    torch.cuda.synchronize()
    M.set_profiling(True)
    M.last_profile()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for _ in range(3):
            hlr.mul_vec(1.0, 0, M, x, y)
    g.replay()
    torch.cuda.synchronize()
    prof = M.last_profile()
    M.set_profiling(False)
    side = "h2_Dx" if kind == "h2" else "nform_Dx"
    assert side in prof, sorted(prof)
    for name, (cnt, ms, by) in prof.items():
        assert cnt == 3 and ms > 0 and by > 0, (name, cnt, ms, by)
    del g
    M.free()


@pytest.mark.parametrize("prec", ["f64", "mixed", "bfp"])
def test_side_stream_in_eight_vector_products(prec):
    """With near_field = 2 asked for explicitly, the 8-vector kernels take
    the same split (by default they keep the fused pass): D X on the side
    stream after x is staged, U T after the join.  Against the fused plan the
    result differs by summation order only; against the oracle, by the
    store's precision."""
    hm = CASES["h"]()
    M1 = hlr.upload(hm, precision=prec, max_nrhs=8, plan={"near_field": 1})
    M2 = hlr.upload(hm, precision=prec, max_nrhs=8, plan={"near_field": 2})
    rng = np.random.default_rng(21)
    X = rng.standard_normal((hm.n, 8))
    Xd = torch.from_numpy(np.ascontiguousarray(X.T)).cuda().T
    outs = []
    for M in (M1, M2):
        M.set_profiling(True)
        M.last_profile()
        Yd = torch.zeros((8, hm.n), dtype=torch.float64, device="cuda").T
        hlr.mul_vec(0.75, 0, M, Xd, Yd)
        torch.cuda.synchronize()
        prof = M.last_profile()
        M.set_profiling(False)
        outs.append((Yd.cpu().numpy(), prof))
    assert "nform_Dx" in outs[1][1] and "nform_Dx" not in outs[0][1]
    tol = 1e-13 if prec == "f64" else 2e-6
    for j in range(8):
        yo = _oracle(hm, "h", 0.75, 0, np.ascontiguousarray(X[:, j]), np.zeros(hm.n))
        for Y, _ in outs:
            assert relerr(Y[:, j], yo) <= tol, (prec, j)
        assert relerr(outs[0][0][:, j], outs[1][0][:, j]) <= (1e-14 if prec == "f64" else 1e-6), (prec, j)
    M1.free()
    M2.free()
