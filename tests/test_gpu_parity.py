"""GPU parity of the FP64 drop-in product against the CPU oracle
(restated hlr::seq::mul_vec / hlr::uniform::mul_vec) on identical host-built
matrices, through the C ABI.

Tolerances: FP64 GPU vs FP64 oracle ||y - y_ref|| / ||y_ref|| <= 1e-13
(summation order differs, so not bit-exact); vs the dense kernel matrix
<= 2e-6 (the construction accuracy eps = 1e-6)."""
import numpy as np
import pytest

import hlr_b200 as hlr
import oracle
from hlr_b200._capi import HLRCError

from conftest import built, relerr

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL = 1e-13


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def gpu_mvm(M, alpha, op, x, y0):
    y = dev(y0)
    hlr.mul_vec(alpha, op, M, dev(x), y)
    torch.cuda.synchronize()
    return y.cpu().numpy()


@pytest.fixture(scope="module")
def c1_dev(c1):
    return c1, hlr.upload(c1)


@pytest.mark.parametrize("op", [0, 1, 2])
def test_c1_log1d_matches_oracle(c1_dev, op):
    hm, M = c1_dev
    x = np.random.default_rng(2).standard_normal(hm.n)
    y0 = np.random.default_rng(3).standard_normal(hm.n)
    y = gpu_mvm(M, 2.0, op, x, y0)
    yref = y0.copy()
    oracle.hmvm_seq(hm.h_desc(), 2.0, op, x, yref)
    assert relerr(y, yref) < TOL
    yd = y0.copy()
    oracle.dense_matvec(hm, 2.0, op, x, yd)
    assert relerr(y - y0, yd - y0) < 2e-6


@pytest.mark.parametrize("n,leaf", [(16384, 64), (5000, 48), (777, 32)])
@pytest.mark.parametrize("op", [0, 1])
def test_exp3d_matches_oracle(n, leaf, op):
    hm = built(f"exp3d_{n}_{leaf}", lambda: hlr.build(hlr.Problem.exp3d(n, leaf_size=leaf)))
    M = hlr.upload(hm)
    x = np.random.default_rng(5).standard_normal(hm.n)
    y = gpu_mvm(M, -0.75, op, x, np.zeros(hm.n))
    yref = np.zeros(hm.n)
    oracle.hmvm_seq(hm.h_desc(), -0.75, op, x, yref)
    assert relerr(y, yref) < TOL
    M.free()


@pytest.fixture(scope="module")
def sphere_dev():
    hm = built("sphere5u", lambda: hlr.build(hlr.Problem.laplace_sphere(refine=5, uniform=True)))
    return hm, hlr.upload(hm)


@pytest.mark.parametrize("op", [0, 2])
def test_uniform_matches_oracle(sphere_dev, op):
    hm, M = sphere_dev
    assert M.uniform
    x = np.random.default_rng(6).standard_normal(hm.n)
    y0 = np.random.default_rng(7).standard_normal(hm.n)
    y = y0.copy()
    hlr.uniform.mul_vec(1.5, op, M, x, y)  # host-buffer path
    yref = y0.copy()
    assert oracle.uniform_mvm(hm.uniform_desc(), 1.5, op, x, yref) == 0
    assert relerr(y, yref) < TOL
    yg = gpu_mvm(M, 1.5, op, x, y0)
    assert relerr(yg, yref) < TOL


def test_uniform_transposed_is_unsupported(sphere_dev):
    hm, M = sphere_dev
    with pytest.raises(HLRCError) as e:
        gpu_mvm(M, 1.0, 1, np.ones(hm.n), np.zeros(hm.n))
    assert e.value.status == 6


def test_uniform_h_form_of_same_matrix(sphere_dev):
    """The H-matrix and its uniform-H form agree to the basis accuracy."""
    hm, Mu = sphere_dev
    Mh = hlr.upload(hm, uniform=False)
    x = np.random.default_rng(8).standard_normal(hm.n)
    yu = gpu_mvm(Mu, 1.0, 0, x, np.zeros(hm.n))
    yh = gpu_mvm(Mh, 1.0, 0, x, np.zeros(hm.n))
    assert relerr(yu, yh) < 2e-5
    Mh.free()


def test_golden_vectors_on_gpu():
    import json
    from pathlib import Path
    g = Path(__file__).resolve().parent / "golden"
    for meta_path in sorted(g.glob("*.json")):
        meta = json.loads(meta_path.read_text())
        data = np.load(meta_path.with_suffix(".npz"))
        prob = hlr.Problem(**meta["problem"])
        hm = hlr.build(prob)
        M = hlr.upload(hm, h2=prob.nested)   # nested bases: the vectors are H^2 products
        for op in meta["ops"]:
            y = gpu_mvm(M, 1.0, op, data["x"], np.zeros(hm.n))
            assert relerr(y, data[f"y_op{op}"]) < TOL, (meta_path.name, op)
        M.free()


def test_known_answer_tiny():
    ll = hlr.LeafList(7, 7)
    rng = np.random.default_rng(9)
    D0, D1 = rng.standard_normal((3, 3)), rng.standard_normal((4, 4))
    U, V = rng.standard_normal((3, 2)), rng.standard_normal((4, 2))
    ll.add_dense(0, 0, D0)
    ll.add_lowrank(0, 3, U, V)
    ll.add_lowrank(3, 0, np.zeros((4, 0)), np.zeros((3, 0)))
    ll.add_dense(3, 3, D1)
    A = np.zeros((7, 7))
    A[:3, :3], A[:3, 3:], A[3:, 3:] = D0, U @ V.T, D1
    M = hlr.upload(ll)
    x = rng.standard_normal(7)
    for op, Aop in ((0, A), (1, A.T), (2, A.T)):
        y = gpu_mvm(M, 0.5, op, x, np.ones(7))
        np.testing.assert_allclose(y, 1.0 + 0.5 * Aop @ x, rtol=1e-14, atol=1e-14)


def test_alpha_zero_and_nrhs_zero(c1_dev):
    hm, M = c1_dev
    y0 = np.arange(hm.n, dtype=np.float64)
    y = gpu_mvm(M, 0.0, 0, np.ones(hm.n), y0)
    np.testing.assert_array_equal(y, y0)


def test_deterministic_and_accumulating(c1_dev):
    hm, M = c1_dev
    x = dev(np.random.default_rng(10).standard_normal(hm.n))
    ys = []
    for _ in range(2):
        y = torch.zeros(hm.n, dtype=torch.float64, device="cuda")
        hlr.mul_vec(1.0, 0, M, x, y)
        hlr.mul_vec(1.0, 0, M, x, y)
        torch.cuda.synchronize()
        ys.append(y.cpu().numpy())
    assert np.array_equal(ys[0], ys[1])  # bit-identical, no atomics
    y1 = torch.zeros(hm.n, dtype=torch.float64, device="cuda")
    hlr.mul_vec(2.0, 0, M, x, y1)
    assert relerr(ys[0], y1.cpu().numpy()) < TOL


def test_reference_alpha_scaling_check(c1_dev):
    """programs/mvm/mvm.hh:158-212: 50 products with alpha=2 vs one with alpha=100, x = 1."""
    hm, M = c1_dev
    x = torch.ones(hm.n, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    yref = torch.zeros_like(x)
    hlr.mul_vec(100.0, 0, M, x, yref)
    for _ in range(50):
        hlr.mul_vec(2.0, 0, M, x, y)
    assert relerr(y.cpu().numpy(), yref.cpu().numpy()) < 1e-13


def test_multi_rhs_equals_columns(c1_dev):
    hm, M = c1_dev
    X = np.asfortranarray(np.random.default_rng(11).standard_normal((hm.n, 3)))
    Y = np.zeros((hm.n, 3), order="F")
    Xd = torch.from_numpy(X.T.copy()).cuda().T  # (n, 3), stride (1, n)
    Yd = torch.zeros((3, hm.n), dtype=torch.float64, device="cuda").T
    hlr.mul_vec(1.0, 0, M, Xd, Yd)
    hlr.mul_vec(1.0, 0, M, X, Y)  # host path
    for j in range(3):
        yref = np.zeros(hm.n)
        oracle.hmvm_seq(hm.h_desc(), 1.0, 0, X[:, j].copy(), yref)
        assert relerr(Yd[:, j].cpu().numpy(), yref) < TOL
        assert relerr(Y[:, j], yref) < TOL


def test_info_accounting(c1_dev):
    hm, M = c1_dev
    info = M.info
    assert info["n_rows"] == hm.n and info["kind"] == 0 and info["precision"] == 0
    assert info["matrix_bytes"] == hlr.plan_info(hm)["matrix_bytes"]
    assert info["device_bytes"] >= info["matrix_bytes"]
