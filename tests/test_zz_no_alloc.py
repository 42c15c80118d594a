"""hlrc_mvm_noalloc: the product for callers that cannot allocate device
memory while they run (open global-mode stream captures, loops that cannot
take cudaFree's device synchronisation, devices whose memory another
allocator already holds).  Its scratch is a static 8 MiB device array of the
library; the test calls it through the C ABI twice in a row and compares each
result with hlrc_mvm's on the same inputs.

This file is collected last so that a stopping run has executed every other
test first; it also passes on its own in a fresh process."""
import ctypes as C

import numpy as np
import pytest

import hlr_b200 as hlr
from hlr_b200 import _capi

from conftest import built, relerr

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL = 1e-13  # same bound as the FP64 parity tests


def _noalloc(M, alpha, op, x, y):
    L = _capi.lib()
    st = L.hlrc_mvm_noalloc(M.handle, float(alpha), int(op), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, L.hlrc_last_error().decode()


@pytest.mark.parametrize("name,factory,calls", [
    ("c1", lambda: hlr.build(hlr.Problem.log1d(8192)), [(2.0, 0), (-0.5, 1)]),
    ("exp3d_16384", lambda: hlr.build(hlr.Problem.exp3d(16384)), [(1.0, 0), (3.0, 0)]),
    ("sphere5u", lambda: hlr.build(hlr.Problem.laplace_sphere(refine=5, uniform=True)), [(1.5, 0), (1.5, 2)]),
])
def test_noalloc_matches_mvm_on_two_calls_in_a_row(name, factory, calls):
    hm = built(name, factory)
    M = hlr.upload(hm)
    rng = np.random.default_rng(31)
    for alpha, op in calls:
        x = torch.from_numpy(rng.standard_normal(hm.n)).cuda()
        y0 = rng.standard_normal(hm.n)
        y_ref = torch.from_numpy(y0.copy()).cuda()
        y_new = torch.from_numpy(y0.copy()).cuda()
        hlr.mul_vec(alpha, op, M, x, y_ref)        # existing entry point (hlrc_mvm)
        _noalloc(M, alpha, op, x, y_new)           # static-scratch entry point
        torch.cuda.synchronize()
        a, b = y_new.cpu().numpy() - y0, y_ref.cpu().numpy() - y0
        assert relerr(a, b) <= TOL, (name, alpha, op)
    M.free()


def test_noalloc_rejects_matrix_beyond_static_scratch():
    hm = built("exp3d_32768", lambda: hlr.build(hlr.Problem.exp3d(32768)))
    assert hlr.plan_info(hm)["workspace_bytes"] > 8 * 2 ** 20
    M = hlr.upload(hm)
    x = torch.ones(hm.n, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    L = _capi.lib()
    st = L.hlrc_mvm_noalloc(M.handle, 1.0, 0, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), None)
    assert st == 2  # HLRC_ERR_SHAPE
    assert b"static scratch" in L.hlrc_last_error()
    torch.cuda.synchronize()
    assert float(y.abs().max()) == 0.0  # nothing ran
    M.free()
