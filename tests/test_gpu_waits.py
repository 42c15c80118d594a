"""Bounded device waits: a wait that runs out returns an error status that
the host reads, and the context stays usable.  hlrc_debug_waits shortens
the bound and leaves one hand-over undone in every waiting CTA (a flag that
nothing sets), so the wait runs out deterministically: an H^2 tree sweep
announces more bytes on its first level's barrier than its copies deliver,
and the producers of the 64-vector kernels never signal their first stage.
No copy is left in flight, no GPU fault is raised."""
import ctypes as C
import time

import numpy as np
import pytest

import hlr_b200 as hlr
import oracle
from hlr_b200 import _capi

from conftest import built, relerr

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _debug(M, limit_ns, skip):
    L = _capi.lib()
    assert L.hlrc_debug_waits(M.handle, int(limit_ns), int(skip)) == 0, L.hlrc_last_error().decode()


def test_tree_sweep_wait_runs_out_and_recovers():
    hm = built("sphere5n", lambda: hlr.build(hlr.Problem.laplace_sphere(refine=5, nested=True)))
    M = hlr.upload(hm, h2=True)
    x = np.random.default_rng(1).standard_normal(hm.n)
    xd = torch.from_numpy(x).cuda()
    _debug(M, 20_000_000, 1)                    # 20 ms bound, first level never completes
    y = torch.zeros(hm.n, dtype=torch.float64, device="cuda")
    t0 = time.perf_counter()
    hlr.h2.mul_vec(1.0, 0, M, xd, y)
    torch.cuda.synchronize()
    assert time.perf_counter() - t0 < 30.0
    assert M.device_error() & 1                 # bit 0: a copy wait of a tree sweep ran out
    _debug(M, 0, 0)                             # normal waits again: the same handle is exact
    y.zero_()
    hlr.h2.mul_vec(1.0, 0, M, xd, y)
    torch.cuda.synchronize()
    assert M.device_error() == 0
    yo = np.zeros(hm.n)
    assert oracle.h2_mvm(hm.h2_desc(), 1.0, 0, x, yo) == 0
    assert relerr(y.cpu().numpy(), yo) <= 1e-13
    M.free()


def test_wide_kernel_wait_runs_out_and_recovers():
    hm = built("exp3d_16384_64", lambda: hlr.build(hlr.Problem.exp3d(16384)))
    M = hlr.upload(hm, precision="f16", max_nrhs=64)
    X = np.random.default_rng(2).standard_normal((hm.n, 64))
    Xd = torch.from_numpy(np.ascontiguousarray(X.T)).cuda().T
    Yd = torch.zeros((64, hm.n), dtype=torch.float64, device="cuda").T
    _debug(M, 20_000_000, 1)
    t0 = time.perf_counter()
    hlr.mul_vec(1.0, 0, M, Xd, Yd)
    torch.cuda.synchronize()
    assert time.perf_counter() - t0 < 30.0
    assert M.device_error() & 2                 # bit 1: a hand-over of the 64-vector kernels ran out
    _debug(M, 0, 0)
    Yd.zero_()
    hlr.mul_vec(1.0, 0, M, Xd, Yd)
    torch.cuda.synchronize()
    assert M.device_error() == 0
    Y = Yd.cpu().numpy()
    for j in (0, 63):
        yo = np.zeros(hm.n)
        oracle.hmvm_seq(hm.h_desc(), 1.0, 0, X[:, j].copy(), yo)
        assert relerr(Y[:, j], yo) <= 2e-3
    M.free()


def test_debug_waits_rejects_bad_limits():
    hm = built("c1_small", lambda: hlr.build(hlr.Problem.log1d(2048)))
    M = hlr.upload(hm)
    L = _capi.lib()
    assert L.hlrc_debug_waits(M.handle, -1, 0) == 1
    assert L.hlrc_debug_waits(None, 0, 0) == 1
    M.free()


def test_fp64_peak_is_measured():
    L = _capi.lib()
    t = C.c_double()
    assert L.hlrc_fp64_peak(0, C.byref(t)) == 0, L.hlrc_last_error().decode()
    # B200: tens of TFLOP/s of FP64 on the DMMA pipe
    assert 5.0 < t.value < 500.0, t.value
