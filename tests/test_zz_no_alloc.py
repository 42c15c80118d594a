"""hlrc_mvm_noalloc: the product for callers that cannot allocate device
memory while they run (open global-mode stream captures, loops that cannot
take cudaFree's device synchronisation, devices whose memory another
allocator already holds).  Its scratch is a static 8 MiB device array of the
library; the test calls it through the C ABI twice in a row and compares each
result with hlrc_mvm's on the same inputs and with the oracle's FP64 product.

This file is collected last so that a stopping run has executed every other
test first; it also passes on its own in a fresh process."""
import ctypes as C

import numpy as np
import pytest

import hlr_b200 as hlr
import oracle
from hlr_b200 import _capi

from conftest import built, relerr

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL = 1e-13  # same bound as the FP64 parity tests
SCRATCH_BYTES = 8 * 2 ** 20  # the static array


def _noalloc(M, alpha, op, x, y):
    L = _capi.lib()
    st = L.hlrc_mvm_noalloc(M.handle, float(alpha), int(op), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, L.hlrc_last_error().decode()


def _oracle(hm, kind, alpha, op, x, y0):
    """y0 + alpha op(M) x by the oracle (FP64 restatement of HLR's product)."""
    y = y0.copy()
    if kind == "h2":
        assert oracle.h2_mvm(hm.h2_desc(), alpha, op, x, y) == 0
    elif kind == "uniform":
        assert oracle.uniform_mvm(hm.uniform_desc(), alpha, op, x, y) == 0
    else:
        oracle.hmvm_seq(hm.h_desc(), alpha, op, x, y)
    return y


CASES = {
    "c1": (lambda: hlr.build(hlr.Problem.log1d(8192)), "h", [(2.0, 0), (-0.5, 1)]),
    "exp3d_16384": (lambda: hlr.build(hlr.Problem.exp3d(16384)), "h", [(1.0, 0), (3.0, 0)]),
    "sphere5u": (lambda: hlr.build(hlr.Problem.laplace_sphere(refine=5, uniform=True)), "uniform",
                 [(1.5, 0), (1.5, 2)]),
    "sphere5n": (lambda: hlr.build(hlr.Problem.laplace_sphere(refine=5, nested=True)), "h2",
                 [(1.0, 0), (-2.0, 2)]),
}


def _upload(hm, kind):
    return hlr.upload(hm, h2=(kind == "h2"))


@pytest.mark.parametrize("name", list(CASES))
def test_noalloc_matches_mvm_and_oracle_on_two_calls_in_a_row(name):
    factory, kind, calls = CASES[name]
    hm = built(name, factory)
    M = _upload(hm, kind)
    rng = np.random.default_rng(31)
    for alpha, op in calls:
        xh = rng.standard_normal(hm.n)
        x = torch.from_numpy(xh).cuda()
        y0 = rng.standard_normal(hm.n)
        y_ref = torch.from_numpy(y0.copy()).cuda()
        y_new = torch.from_numpy(y0.copy()).cuda()
        hlr.mul_vec(alpha, op, M, x, y_ref)        # existing entry point (hlrc_mvm)
        _noalloc(M, alpha, op, x, y_new)           # static-scratch entry point
        torch.cuda.synchronize()
        a, b = y_new.cpu().numpy() - y0, y_ref.cpu().numpy() - y0
        assert relerr(a, b) <= TOL, (name, alpha, op)
        yo = _oracle(hm, kind, alpha, op, xh, y0) - y0
        assert relerr(a, yo) <= TOL, (name, alpha, op, "oracle")
    M.free()


def test_noalloc_interleaved_handles_leave_no_stale_scratch():
    """Calls on two handles of different layouts, alternating: each call
    finds the other matrix's scratch in the shared array and must still be
    exact."""
    ha = built("c1", CASES["c1"][0])
    hb = built("sphere5n", CASES["sphere5n"][0])
    Ma, Mb = _upload(ha, "h"), _upload(hb, "h2")
    rng = np.random.default_rng(5)
    for rep in range(3):
        for hm, M, kind, op in ((ha, Ma, "h", rep % 2), (hb, Mb, "h2", 2 * (rep % 2))):
            xh = rng.standard_normal(hm.n)
            y = torch.zeros(hm.n, dtype=torch.float64, device="cuda")
            _noalloc(M, 1.25, op, torch.from_numpy(xh).cuda(), y)
            torch.cuda.synchronize()
            yo = _oracle(hm, kind, 1.25, op, xh, np.zeros(hm.n))
            assert relerr(y.cpu().numpy(), yo) <= TOL, (kind, rep, op)
    Ma.free()
    Mb.free()


def test_noalloc_limit_is_the_products_scratch():
    """Accepted exactly when the product's scratch (hlrc_info.scratch_bytes:
    coefficients plus partial sums) fits the 8 MiB array."""
    under = built("exp3d_16384", CASES["exp3d_16384"][0])
    over = built("exp3d_20480", lambda: hlr.build(hlr.Problem.exp3d(20480)))
    L = _capi.lib()
    for hm, fits in ((under, True), (over, False)):
        need = hlr.plan_info(hm)["scratch_bytes"]
        assert (need <= SCRATCH_BYTES) == fits, need
        M = hlr.upload(hm)
        assert M.info["scratch_bytes"] == need
        x = torch.ones(hm.n, dtype=torch.float64, device="cuda")
        y = torch.zeros_like(x)
        st = L.hlrc_mvm_noalloc(M.handle, 1.0, 0, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), None)
        torch.cuda.synchronize()
        if fits:
            assert st == 0, L.hlrc_last_error().decode()
            assert float(y.abs().max()) > 0.0
        else:
            assert st == 2  # HLRC_ERR_SHAPE
            assert b"static scratch" in L.hlrc_last_error()
            assert float(y.abs().max()) == 0.0  # nothing ran
        M.free()
