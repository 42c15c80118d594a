"""Products captured into a CUDA graph: replays give the same y as direct
launches, and with profiling enabled the per-pass events are graph nodes
that every replay records again (the bench times its runs this way)."""
import numpy as np
import pytest

import hlr_b200 as hlr

from conftest import relerr

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["f64", "mixed"])
def test_graph_replay_matches_direct_and_profiles(c2_small, prec):
    M = hlr.upload(c2_small, precision=prec)
    x = torch.from_numpy(np.random.default_rng(1).standard_normal(c2_small.n)).cuda()
    y_direct = torch.zeros_like(x)
    for _ in range(6):
        hlr.mul_vec(2.0, hlr.apply_normal, M, x, y_direct)
    torch.cuda.synchronize()
    per_product = M.launch_count()
    y = torch.zeros_like(x)
    hlr.mul_vec(2.0, hlr.apply_normal, M, x, y)       # warm-up outside the graph
    torch.cuda.synchronize()
    y.zero_()
    M.set_profiling(True)
    M.last_profile()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for _ in range(3):
            hlr.mul_vec(2.0, hlr.apply_normal, M, x, y)
    torch.cuda.synchronize()
    assert float(y.abs().max()) == 0.0                  # capture runs nothing
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    prof = M.last_profile()
    M.set_profiling(False)
    tol = 1e-13 if prec == "f64" else 1e-6
    assert relerr(y.cpu().numpy(), y_direct.cpu().numpy()) <= tol
    assert prof, "no pass timings from the replay"
    for name, (cnt, ms, by) in prof.items():
        assert cnt == 3 and ms > 0 and by > 0, (name, cnt, ms, by)
    assert per_product > 0
    del g
    M.free()


@pytest.mark.parametrize("prec", ["f64", "mixed", "bfp"])
@pytest.mark.parametrize("op", [0, 1])
def test_overlapped_launches_match_plain_launches(c2_small, prec, op):
    """Programmatic dependent launch (tuning overlap = 1, the default) lets
    each one-vector kernel start while its predecessor runs; every kernel
    waits for its predecessor on the device before it reads or writes a
    vector, so chains of products, direct and in a CUDA graph, give exactly
    the plain launches' results (same kernels, same summation order)."""
    M = hlr.upload(c2_small, precision=prec)
    assert M.tuning["overlap"] == 1
    x = torch.from_numpy(np.random.default_rng(3).standard_normal(c2_small.n)).cuda()

    def chain(overlap, graph):
        M.set_tuning(overlap=overlap)
        y = torch.zeros_like(x)
        if not graph:
            for k in range(8):
                hlr.mul_vec(0.5 + k, op, M, x, y)
        else:
            hlr.mul_vec(1.0, op, M, x, y)          # warm-up outside the graph
            torch.cuda.synchronize()
            y.zero_()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                for k in range(8):
                    hlr.mul_vec(0.5 + k, op, M, x, y)
            g.replay()
            torch.cuda.synchronize()
            del g
        torch.cuda.synchronize()
        return y.cpu().numpy()

    plain = chain(0, False)
    assert np.array_equal(chain(1, False), plain)
    assert np.array_equal(chain(1, True), plain)
    assert np.array_equal(chain(0, True), plain)
    with pytest.raises(hlr.HLRCError):
        M.set_tuning(overlap=2)
    assert M.device_error() == 0
    M.free()
