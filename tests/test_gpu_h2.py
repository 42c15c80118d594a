"""H^2 products on the GPU against the CPU oracle's restatement of
hlr::h2::mul_vec on the same nested bases: op N and op C, one and eight
vectors, FP64 to 1e-13; op T is rejected as in the reference."""
import numpy as np
import pytest

import hlr_b200 as hlr
import oracle

from conftest import built, relerr

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL = 1e-13

CASES = {
    "sphere4": lambda: hlr.build(hlr.Problem.laplace_sphere(refine=4, nested=True)),
    "sphere5": lambda: hlr.build(hlr.Problem.laplace_sphere(refine=5, nested=True)),
    "log1d_2048": lambda: hlr.build(hlr.Problem.log1d(2048, nested=True)),
    "exp3d_4096": lambda: hlr.build(hlr.Problem.exp3d(4096, nested=True)),
}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("op", [0, 2])
def test_h2_parity(case, op):
    hm = built(case + "_h2", CASES[case])
    M = hlr.upload(hm, h2=True, max_nrhs=8)
    assert M.h2 and M.info["kind"] == 2
    rng = np.random.default_rng(31 + op)
    x = rng.standard_normal(hm.n)
    y0 = rng.standard_normal(hm.n)
    y = torch.from_numpy(y0.copy()).cuda()
    hlr.h2.mul_vec(1.5, op, M, torch.from_numpy(x).cuda(), y)
    torch.cuda.synchronize()
    yref = y0.copy()
    assert oracle.h2_mvm(hm.h2_desc(), 1.5, op, x, yref) == 0
    assert relerr(y.cpu().numpy() - y0, yref - y0) <= TOL
    # eight vectors (op N runs the 8-vector kernels, op C loops)
    X = rng.standard_normal((hm.n, 8))
    Xd = torch.from_numpy(np.ascontiguousarray(X.T)).cuda().T
    Yd = torch.zeros((8, hm.n), dtype=torch.float64, device="cuda").T
    hlr.mul_vec(1.0, op, M, Xd, Yd)
    torch.cuda.synchronize()
    Y = Yd.cpu().numpy()
    for j in range(8):
        yj = np.zeros(hm.n)
        oracle.h2_mvm(hm.h2_desc(), 1.0, op, X[:, j].copy(), yj)
        assert relerr(Y[:, j], yj) <= TOL, j
    assert M.device_error() == 0
    M.free()


def test_h2_rejects_transposed_and_other_precisions():
    hm = built("sphere4_h2", CASES["sphere4"])
    M = hlr.upload(hm, h2=True)
    x = torch.zeros(hm.n, dtype=torch.float64, device="cuda")
    with pytest.raises(hlr.HLRCError) as e:
        hlr.mul_vec(1.0, hlr.apply_transposed, M, x, x.clone())
    assert e.value.status == 6
    M.free()
    with pytest.raises(hlr.HLRCError):
        hlr.upload(hm, h2=True, precision="mixed")


@pytest.mark.parametrize("op", [0, 2])
def test_h2_tree_sweeps(op):
    """The sphere with 8192 triangles has 32 clusters at level 5 and three
    levels below them: the one-vector product sweeps those levels of each
    tree in one launch (one cluster of CTAs per subtree), the 8-vector
    product runs them level by level, and both match the oracle."""
    hm = built("sphere5_h2", CASES["sphere5"])
    M = hlr.upload(hm, h2=True, max_nrhs=8)
    M.set_profiling(True)
    M.last_profile()
    rng = np.random.default_rng(77 + op)
    x = rng.standard_normal(hm.n)
    y = torch.zeros(hm.n, dtype=torch.float64, device="cuda")
    hlr.mul_vec(-0.5, op, M, torch.from_numpy(x).cuda(), y)
    torch.cuda.synchronize()
    prof = M.last_profile()
    assert prof["h2_fwd_tree"][0] == 1 and prof["h2_bwd_tree"][0] == 1
    # the forward transfer into level 4 keeps its own pass; the backward
    # transfer into the subtree roots is the first level of their sweep
    assert prof["h2_fwd_transfer"][0] == 1 and "h2_bwd_transfer" not in prof
    # op N: the near field on the side stream (the default for H2)
    assert ("h2_Dx" in prof) == (op == 0)
    yref = np.zeros(hm.n)
    oracle.h2_mvm(hm.h2_desc(), -0.5, op, x, yref)
    assert relerr(y.cpu().numpy(), yref) <= TOL
    # the level passes of the multi-vector product give the same result
    X = np.stack([x, rng.standard_normal(hm.n)], axis=1)
    Xd = torch.from_numpy(np.ascontiguousarray(X.T)).cuda().T
    Yd = torch.zeros((2, hm.n), dtype=torch.float64, device="cuda").T
    hlr.mul_vec(-0.5, op, M, Xd, Yd)
    torch.cuda.synchronize()
    prof = M.last_profile()
    if op == 0:   # op C loops the one-vector product (unit T-form coupling)
        assert "h2_fwd_tree" not in prof and prof["h2_fwd_transfer"][0] == 3   # parents at levels 4-6
    assert relerr(Yd[:, 0].cpu().numpy(), yref) <= TOL
    assert M.device_error() == 0
    M.free()


def test_plan_info_launches_match_upload():
    """The dry run's launch counts equal those of the uploaded handle."""
    cases = [(built("sphere5_h2", CASES["sphere5"]), dict(h2=True)),
             (built("log1d_2048_h", lambda: hlr.build(hlr.Problem.log1d(2048))), dict(precision="f64")),
             (built("log1d_2048_h", lambda: hlr.build(hlr.Problem.log1d(2048))), dict(precision="mixed")),
             (built("log1d_2048_h", lambda: hlr.build(hlr.Problem.log1d(2048))), dict(precision="bfp"))]
    for hm, kw in cases:
        M = hlr.upload(hm, **kw)
        assert hlr.plan_info(hm, **kw)["launches"] == M.info["launches"], kw
        M.free()


@pytest.mark.parametrize("op", [0, 2])
def test_h2_tree_sweeps_high_rank(op):
    """3D exponential kernel, n = 16384: cluster ranks up to about 110, so
    transfer matrices span two 64-row pieces, segments are 64 rows tall (two
    32-row blocks per half-warp) and the shared-memory budget puts the
    subtree roots below the first level with 32 clusters."""
    hm = built("exp3d_16384_h2", lambda: hlr.build(hlr.Problem.exp3d(16384, nested=True)))
    assert hm.h2_desc().nrow_clusters > 0
    M = hlr.upload(hm, h2=True)
    M.set_profiling(True)
    M.last_profile()
    rng = np.random.default_rng(90 + op)
    x = rng.standard_normal(hm.n)
    y0 = rng.standard_normal(hm.n)
    y = torch.from_numpy(y0.copy()).cuda()
    hlr.mul_vec(0.5, op, M, torch.from_numpy(x).cuda(), y)
    torch.cuda.synchronize()
    prof = M.last_profile()
    assert prof["h2_fwd_tree"][0] == 1 and prof["h2_bwd_tree"][0] == 1
    yref = y0.copy()
    assert oracle.h2_mvm(hm.h2_desc(), 0.5, op, x, yref) == 0
    assert relerr(y.cpu().numpy() - y0, yref - y0) <= TOL
    assert M.device_error() == 0
    M.free()


SWEEP_CASES = {
    "exp3d_2048_leaf16": lambda: hlr.Problem.exp3d(2048, nested=True, leaf_size=16),
    "log1d_4096_leaf32": lambda: hlr.Problem.log1d(4096, nested=True, leaf_size=32),
}


@pytest.mark.parametrize("case", sorted(SWEEP_CASES))
@pytest.mark.parametrize("op", [0, 2])
def test_h2_sweeps_small_leaves(case, op):
    """Tree sweeps over segments of 2 to 56 rows (ranks 6 to 55) match the
    oracle to 1e-13."""
    hm = built(case + "_h2", lambda: hlr.build(SWEEP_CASES[case]()))
    M = hlr.upload(hm, h2=True)
    M.set_profiling(True)
    M.last_profile()
    rng = np.random.default_rng(120 + op)
    x = rng.standard_normal(hm.n)
    y = torch.zeros(hm.n, dtype=torch.float64, device="cuda")
    hlr.mul_vec(1.0, op, M, torch.from_numpy(x).cuda(), y)
    torch.cuda.synchronize()
    prof = M.last_profile()
    assert "h2_fwd_tree" in prof and "h2_bwd_tree" in prof
    yref = np.zeros(hm.n)
    assert oracle.h2_mvm(hm.h2_desc(), 1.0, op, x, yref) == 0
    assert relerr(y.cpu().numpy(), yref) <= TOL
    assert M.device_error() == 0
    M.free()
