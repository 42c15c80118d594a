"""Host construction (restated clustering / admissibility / ACA / SVD /
uniform bases): structural and accuracy properties."""
import numpy as np
import pytest

import hlr_b200 as hlr
import oracle


def leaves(hm):
    d = hm.h_desc()
    return d, [d.blocks[i] for i in range(d.nblocks)]


@pytest.mark.parametrize("fixture", ["c1_small", "c2_small", "c3_small"])
def test_leaves_partition_the_matrix(request, fixture):
    hm = request.getfixturevalue(fixture)
    d, bl = leaves(hm)
    n = hm.n
    # coverage count on the leaf-cluster grid: every cell covered exactly once
    cuts = sorted({b.row0 for b in bl} | {b.row0 + b.nrows for b in bl})
    idx = {c: i for i, c in enumerate(cuts)}
    cov = np.zeros((len(cuts) - 1, len(cuts) - 1), dtype=np.int32)
    for b in bl:
        cov[idx[b.row0]:idx[b.row0 + b.nrows], idx[b.col0]:idx[b.col0 + b.ncols]] += 1
    assert cuts[0] == 0 and cuts[-1] == n
    assert (cov == 1).all()
    assert max(b.nrows for b in bl if b.kind == 0) <= 64


@pytest.mark.parametrize("fixture", ["c1_small", "c2_small"])
def test_admissibility_condition(request, fixture):
    hm = request.getfixturevalue(fixture)
    _, bl = leaves(hm)
    P = hm.points

    def box(a, m):
        pts = P[a:a + m]
        return pts.min(0), pts.max(0)

    for b in bl[:: max(1, len(bl) // 400)]:
        (rmin, rmax), (cmin, cmax) = box(b.row0, b.nrows), box(b.col0, b.ncols)
        dr, dc = np.linalg.norm(rmax - rmin), np.linalg.norm(cmax - cmin)
        gap = np.maximum(0, np.maximum(cmin - rmax, rmin - cmax))
        dist = np.linalg.norm(gap)
        adm = min(dr, dc) <= 2.0 * dist
        if b.kind == 1:
            assert adm
        else:
            assert not adm or b.nrows <= 64 or b.ncols <= 64


@pytest.mark.parametrize("fixture", ["c1_small", "c2_small", "c3_small"])
def test_leaf_accuracy(request, fixture):
    hm = request.getfixturevalue(fixture)
    d = hm.h_desc()
    err = oracle.leaf_max_error(hm, d, 5)
    amax = max(abs(hm.entry(0, 0)), abs(hm.entry(1, 2)), 1e-300)
    assert err < 1e-4 * amax


def test_ranks_are_truncated(c2_small):
    _, bl = leaves(c2_small)
    lr = [b for b in bl if b.kind == 1]
    assert lr
    assert all(b.rank < min(b.nrows, b.ncols) for b in lr)
    assert max(b.rank for b in lr) <= 64


def test_points_are_reproducible():
    a = hlr.build(hlr.Problem.exp3d(700, leaf_size=32))
    b = hlr.build(hlr.Problem.exp3d(700, leaf_size=32))
    np.testing.assert_array_equal(a.points, b.points)
    np.testing.assert_array_equal(a.perm_i2e, b.perm_i2e)
    c = hlr.build(hlr.Problem.exp3d(700, leaf_size=32, seed=5))
    assert not np.array_equal(a.points, c.points)
    # internal order is a permutation of the generated points
    assert sorted(a.perm_i2e.tolist()) == list(range(700))


def test_sphere_mesh():
    hm = hlr.build(hlr.Problem.laplace_sphere(refine=3))
    assert hm.n == 8 * 4 ** 3
    assert np.allclose(np.linalg.norm(hm.points, axis=1) <= 1.0, True)
    total = hm.weights.sum()
    assert 0.9 * 4 * np.pi < total < 4 * np.pi


def test_uniform_bases_are_orthonormal(c3_small):
    u = c3_small.uniform_desc()
    for arr, cnt in ((u.row_bases, u.nrow_bases), (u.col_bases, u.ncol_bases)):
        for i in range(cnt):
            b = arr[i]
            if b.rank == 0 or b.size == 0:
                continue
            V = np.ctypeslib.as_array(b.V, shape=(b.rank * b.ldv,)).reshape(b.rank, b.ldv).T[: b.size]
            np.testing.assert_allclose(V.T @ V, np.eye(b.rank), atol=1e-12)


def test_odd_sizes_and_leaf_sizes():
    hm = hlr.build(hlr.Problem.exp3d(1000, leaf_size=48))
    d = hm.h_desc()
    x = np.random.default_rng(0).standard_normal(hm.n)
    y = np.zeros(hm.n)
    oracle.hmvm_seq(d, 1.0, 0, x, y)
    yd = np.zeros(hm.n)
    oracle.dense_matvec(hm, 1.0, 0, x, yd)
    assert np.linalg.norm(y - yd) / np.linalg.norm(yd) < 2e-6


def test_device_build_arguments():
    # the device build assembles the H form only
    with pytest.raises(hlr.HLRCError) as e:
        hlr.build(hlr.Problem.laplace_sphere(2, uniform=True, on_device=True))
    assert e.value.status == 1
    # without a usable GPU it fails with a CUDA status, not a crash
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        with pytest.raises(hlr.HLRCError) as e:
            hlr.build(hlr.Problem.exp3d(500, on_device=True))
        assert e.value.status == 4
    # a host build reports host leaves and fetch() is a no-op
    hm = hlr.build(hlr.Problem.log1d(300))
    assert not hm.leaves_on_device
    assert hm.fetch() is hm and not hm.leaves_on_device
