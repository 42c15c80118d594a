"""Leaf assembly on the GPU (hlrc_problem.on_device): the same cluster and
block trees as the host build, dense leaves evaluated, admissible leaves by
ACA + QR/SVD recompression on the device (approx/aca.hh:328-436,
approx/svd.hh:94-209 restated as CTA-wide kernels).

Checked: ranks within +-1 of the host build leaf by leaf; the product of
the device-built matrix against the dense kernel matrix (to the
approximation accuracy) and against the oracle on the same leaves (to
rounding); FP64 stores gathered on the device from device-resident leaves
equal stores uploaded from host copies of the same leaves; reduced
precisions and batches take device-resident leaves as well."""
import numpy as np
import pytest

import hlr_b200 as hlr
import oracle

from conftest import relerr

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

PROBLEMS = {
    "exp3d_4096": lambda dev: hlr.Problem.exp3d(4096, on_device=dev),
    "log1d_2048": lambda dev: hlr.Problem.log1d(2048, on_device=dev),
    "sphere_r4": lambda dev: hlr.Problem.laplace_sphere(4, on_device=dev),
    "exp3d_3000_48": lambda dev: hlr.Problem.exp3d(3000, leaf_size=48, ell=0.2, on_device=dev),
}


def _blocks(hm):
    d = hm.h_desc()
    return [d.blocks[i] for i in range(d.nblocks)]


@pytest.mark.parametrize("name", list(PROBLEMS))
def test_device_build_matches_host_build(name):
    hd = hlr.build(PROBLEMS[name](True))
    hh = hlr.build(PROBLEMS[name](False))
    assert hd.leaves_on_device and not hh.leaves_on_device
    bd, bh = _blocks(hd), _blocks(hh)
    assert len(bd) == len(bh)
    for a, b in zip(bd, bh):
        assert (a.row0, a.nrows, a.col0, a.ncols, a.kind) == (b.row0, b.nrows, b.col0, b.ncols, b.kind)
        assert abs(a.rank - b.rank) <= 1, (a.row0, a.col0, a.rank, b.rank)
    n = hd.n
    x = np.random.default_rng(4).standard_normal(n)
    # FP64 upload straight from device memory (store gathered on the device)
    M = hlr.upload(hd, precision="f64")
    yd = torch.zeros(n, dtype=torch.float64, device="cuda")
    hlr.mul_vec(1.0, hlr.apply_normal, M, torch.from_numpy(x).cuda(), yd)
    torch.cuda.synchronize()
    y = yd.cpu().numpy()
    # against the dense kernel matrix: the approximation accuracy
    ydense = np.zeros(n)
    oracle.dense_matvec(hh, 1.0, 0, x, ydense)
    assert relerr(y, ydense) <= 2e-6
    # against the oracle on the same (fetched) leaves: rounding only
    hd.fetch()
    assert not hd.leaves_on_device
    yor = np.zeros(n)
    oracle.hmvm_seq(hd.h_desc(), 1.0, 0, x, yor)
    assert relerr(y, yor) <= 1e-13
    # the fetched leaves give the same store, hence the same product
    M2 = hlr.upload(hd, precision="f64")
    y2 = torch.zeros(n, dtype=torch.float64, device="cuda")
    hlr.mul_vec(1.0, hlr.apply_normal, M2, torch.from_numpy(x).cuda(), y2)
    torch.cuda.synchronize()
    assert np.array_equal(y2.cpu().numpy(), y)
    assert M.info["matrix_bytes"] == M2.info["matrix_bytes"]
    M.free()
    M2.free()


def _leaf_data(hm):
    """All leaf entries of a host-resident build, concatenated."""
    parts = []
    for b in _blocks(hm):
        if b.kind == 0:
            parts.append(np.ctypeslib.as_array(b.D, shape=(b.ldd * b.ncols,)).copy())
        elif b.rank > 0:
            parts.append(np.ctypeslib.as_array(b.U, shape=(b.ldu * b.rank,)).copy())
            parts.append(np.ctypeslib.as_array(b.V, shape=(b.ldv * b.rank,)).copy())
    return np.concatenate(parts)


def test_device_build_is_deterministic():
    p = hlr.Problem.exp3d(3500, seed=4, on_device=True)
    a = hlr.build(p).fetch()
    b = hlr.build(p).fetch()
    assert [x.rank for x in _blocks(a)] == [x.rank for x in _blocks(b)]
    da, db = _leaf_data(a), _leaf_data(b)
    assert da.shape == db.shape
    assert np.array_equal(da, db), float(np.abs(da - db).max())


def test_device_leaves_in_reduced_precision_and_batches():
    probs = [hlr.Problem.exp3d(n, seed=s, on_device=True) for n, s in ((2000, 3), (3500, 4))]
    hds = [hlr.build(p) for p in probs]
    hhs = [hlr.build(hlr.Problem.exp3d(p.n, seed=p.seed, on_device=True)).fetch() for p in probs]
    x = np.random.default_rng(6).standard_normal(hds[1].n)
    xt = torch.from_numpy(x).cuda()

    def product(M):
        y = torch.zeros(hds[1].n, dtype=torch.float64, device="cuda")
        hlr.mul_vec(1.0, 0, M, xt, y)
        torch.cuda.synchronize()
        M.free()
        return y.cpu().numpy()

    precs = ("mixed", "f16", "bfp")
    # reduced precisions: the upload makes host copies of the device leaves
    ya = {prec: product(hlr.upload(hds[1], precision=prec)) for prec in precs}
    yb = {prec: product(hlr.upload(hhs[1], precision=prec)) for prec in precs}
    hds[1].fetch()
    for prec in precs:
        # the same leaves copied by the upload or fetched: the same store
        assert np.array_equal(product(hlr.upload(hds[1], precision=prec)), ya[prec]), prec
        # another device build of the same problem
        assert np.array_equal(yb[prec], ya[prec]), prec
    hds[1] = hlr.build(probs[1])
    pad = 3584
    A = hlr.upload_batch(hds, precision="f64", pad_to=pad)
    B = hlr.upload_batch(hhs, precision="f64", pad_to=pad)
    xb = np.random.default_rng(7).standard_normal(2 * pad)
    ya = torch.zeros(2 * pad, dtype=torch.float64, device="cuda")
    yb = torch.zeros_like(ya)
    hlr.mul_vec(1.0, 0, A, torch.from_numpy(xb).cuda(), ya)
    hlr.mul_vec(1.0, 0, B, torch.from_numpy(xb).cuda(), yb)
    torch.cuda.synchronize()
    assert np.array_equal(ya.cpu().numpy(), yb.cpu().numpy())
    with pytest.raises(ValueError):
        hlr.upload_batch([hds[0], hhs[1]], precision="f64", pad_to=pad)
    A.free()
    B.free()
