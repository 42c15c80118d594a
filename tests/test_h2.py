"""H^2 (nested cluster bases) on the host: the construction reproduces the
kernel matrix to the construction accuracy, the oracle's op N and op C agree
with the dense products, the transfer structure is nested, and the planner
validates descriptors (no GPU)."""
import ctypes as C

import numpy as np
import pytest

import hlr_b200 as hlr
import oracle

from conftest import built, relerr


@pytest.fixture(scope="module")
def sphere_h2():
    return built("sphere4_h2", lambda: hlr.build(hlr.Problem.laplace_sphere(refine=4, nested=True)))


@pytest.fixture(scope="module")
def log1d_h2():
    return built("log1d_2048_h2", lambda: hlr.build(hlr.Problem.log1d(2048, nested=True)))


@pytest.mark.parametrize("fixture", ["sphere_h2", "log1d_h2"])
@pytest.mark.parametrize("op", [0, 2])
def test_h2_oracle_matches_dense(request, fixture, op):
    hm = request.getfixturevalue(fixture)
    x = np.random.default_rng(3).standard_normal(hm.n)
    y = np.zeros(hm.n)
    assert oracle.h2_mvm(hm.h2_desc(), 1.5, op, x, y) == 0
    yd = np.zeros(hm.n)
    oracle.dense_matvec(hm, 1.5, op, x, yd)
    assert relerr(y, yd) < 2e-6          # construction accuracy eps = 1e-6


def test_h2_rejects_transposed(sphere_h2):
    x = np.zeros(sphere_h2.n)
    y = np.zeros(sphere_h2.n)
    assert oracle.h2_mvm(sphere_h2.h2_desc(), 1.0, 1, x, y) == 6   # HLRC_ERR_UNSUPPORTED_OP


def test_h2_bases_are_nested(sphere_h2):
    """V_parent = [V_son0 E_son0; V_son1 E_son1] has orthonormal columns when
    the leaf bases and the stacked transfer matrices do."""
    d = sphere_h2.h2_desc()
    cl = d.row_clusters

    def explicit(t):
        c = cl[t]
        if c.son[0] < 0 and c.son[1] < 0:
            return np.ctypeslib.as_array(c.V, shape=(c.rank * c.ldv,)).reshape(c.rank, c.ldv).T[:c.size] if c.rank else np.zeros((c.size, 0))
        parts = []
        for s in c.son:
            if s < 0:
                continue
            cs = cl[s]
            Vs = explicit(s)
            E = (np.ctypeslib.as_array(cs.E, shape=(c.rank * cs.lde,)).reshape(c.rank, cs.lde).T[:cs.rank]
                 if cs.rank and c.rank else np.zeros((cs.rank, c.rank)))
            parts.append(Vs @ E)
        return np.vstack(parts)
    # an inner cluster of positive rank (upper levels hold no admissible
    # blocks here and have rank 0)
    t = next(i for i in range(d.nrow_clusters) if cl[i].son[0] >= 0 and cl[i].rank > 0)
    V = explicit(t)
    assert V.shape == (cl[t].size, cl[t].rank)
    assert np.allclose(V.T @ V, np.eye(cl[t].rank), atol=1e-10)


def test_h2_plan_info_and_validation(sphere_h2):
    info = hlr.plan_info(sphere_h2, h2=True)
    assert info["kind"] == 2 and info["matrix_bytes"] > 0 and info["max_rank"] > 0
    d = sphere_h2.h2_desc()
    # a son whose parent link is broken is refused before anything is planned
    clusters = (hlr._capi.hlrc_h2_cluster * d.nrow_clusters)(*[d.row_clusters[i] for i in range(d.nrow_clusters)])
    s0 = clusters[0].son[0]
    clusters[s0].parent = 5 if clusters[s0].parent != 5 else 6
    bad = hlr._capi.hlrc_h2_desc(d.nrows, d.ncols, d.nrow_clusters, C.cast(clusters, C.POINTER(hlr._capi.hlrc_h2_cluster)),
                                 d.ncol_clusters, d.col_clusters, d.nblocks, d.blocks)
    with pytest.raises(hlr.HLRCError) as e:
        hlr.plan_info(bad, h2=True)
    assert e.value.status == 2
    with pytest.raises(hlr.HLRCError):
        hlr.plan_info(sphere_h2, h2=True, precision="mixed")


def test_h2_tree_sweeps_planned():
    """On the sphere with 8192 triangles the one-vector product sweeps the
    transfer levels below the 32 clusters of level 5 in one launch per tree:
    op N is the leaf transform, the forward sweep, the level-4 transfer, the
    couplings, the backward sweep (from the level-5 transfer down) and the
    leaf pass, and by default the near field D x as its own pass on a side
    stream (the planner and its checks of the sweep's arrays run here, on
    the host)."""
    hm = built("sphere5_h2", lambda: hlr.build(hlr.Problem.laplace_sphere(refine=5, nested=True)))
    info = hlr.plan_info(hm, h2=True)
    assert info["launches"][0] == 7
    assert info["launches"][1] == 0   # op T unsupported
    assert hlr.plan_info(hm, h2=True, plan={"near_field": 1})["launches"][0] == 6
    assert hlr.plan_info(hm, h2=True, plan={"near_field": 2})["launches"][0] == 7
    # without levels below the subtree roots there is no sweep: one pass per level
    small = built("sphere4_h2", lambda: hlr.build(hlr.Problem.laplace_sphere(refine=4, nested=True)))
    assert hlr.plan_info(small, h2=True, plan={"near_field": 1})["launches"][0] == 5
    with pytest.raises(hlr.HLRCError):
        hlr.plan_info(small, h2=True, plan={"near_field": 3})


SMALL_TREES = {
    # (problem, launches of the one-vector op N product with the sweeps and
    # the near field fused into the leaf pass; one more with it on the side)
    "exp3d_4096_leaf32": (lambda: hlr.Problem.exp3d(4096, nested=True, leaf_size=32), 6),
    "log1d_4096_leaf32": (lambda: hlr.Problem.log1d(4096, nested=True, leaf_size=32), 10),
    "sphere4_leaf32": (lambda: hlr.Problem.laplace_sphere(refine=4, nested=True, leaf_size=32), 7),
    "exp3d_2048_leaf16": (lambda: hlr.Problem.exp3d(2048, nested=True, leaf_size=16), 6),
}


@pytest.mark.parametrize("case", sorted(SMALL_TREES))
def test_h2_sweeps_planned_for_small_leaves(case):
    """Leaves of 16 or 32 rows give deep trees at small n: the planner builds
    the sweeps where at least two levels lie below the subtree roots (not on
    the 2048-triangle sphere), over segments from 2 to 56 rows tall, and its
    checks of the sweep arrays pass."""
    make, launches = SMALL_TREES[case]
    hm = built(case + "_h2", lambda: hlr.build(make()))
    assert hlr.plan_info(hm, h2=True, plan={"near_field": 1})["launches"][0] == launches
    assert hlr.plan_info(hm, h2=True)["launches"][0] == launches + 1


@pytest.mark.parametrize("op", [0, 2])
@pytest.mark.parametrize("case", ["sphere4", "exp3d_2048_leaf16", "log1d_4096_leaf32"])
def test_h2_threaded_oracle_is_bit_identical(case, op):
    """The threaded oracle (OpenMP tasks over subtrees, couplings per output
    cluster, near field per row group) performs the sequential oracle's
    operations in the same order for every output: identical bits."""
    if case == "sphere4":
        hm = built("sphere4_h2", lambda: hlr.build(hlr.Problem.laplace_sphere(refine=4, nested=True)))
    else:
        make, _ = SMALL_TREES[case]
        hm = built(case + "_h2", lambda: hlr.build(make()))
    rng = np.random.default_rng(3 + op)
    x = rng.standard_normal(hm.n)
    y0 = rng.standard_normal(hm.n)
    ys, yp = y0.copy(), y0.copy()
    assert oracle.h2_mvm(hm.h2_desc(), 1.75, op, x, ys) == 0
    assert oracle.h2_mvm(hm.h2_desc(), 1.75, op, x, yp, nthreads=4) == 0
    assert np.array_equal(ys, yp)
