"""Row shards on the GPU: each shard is uploaded as its own rectangular
H-matrix and multiplied on cuda:0 (one GPU: the shards run one after the
other, with no collective); the reassembled products match the oracle to
1e-13 for op N (y slices) and op T (summed full-length partials)."""
import numpy as np
import pytest

import hlr_b200 as hlr
import oracle
from hlr_b200 import dist as hdist

from conftest import built, relerr

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("op", [0, 1, 2])
def test_shards_on_gpu(op):
    hm = built("exp3d_4096", lambda: hlr.build(hlr.Problem.exp3d(4096)))
    cuts = hdist.row_cuts(hm, 3)
    shards = [hdist.upload_shard(hm, cuts, r) for r in range(3)]
    rng = np.random.default_rng(40 + op)
    x = rng.standard_normal(hm.n)
    y0 = rng.standard_normal(hm.n)
    xd = torch.from_numpy(x).cuda()
    y = torch.from_numpy(y0.copy()).cuda()
    for r, M in enumerate(shards):
        a, b = cuts[r], cuts[r + 1]
        assert M.nrows == b - a and M.ncols == hm.n
        if op == 0:
            hlr.mul_vec(-1.25, op, M, xd, y[a:b])
        else:
            part = torch.zeros(hm.n, dtype=torch.float64, device="cuda")
            hlr.mul_vec(-1.25, op, M, xd[a:b].contiguous(), part)
            y += part
    torch.cuda.synchronize()
    yref = y0.copy()
    oracle.hmvm_seq(hm.h_desc(), -1.25, op, x, yref)
    assert relerr(y.cpu().numpy() - y0, yref - y0) <= 1e-13
    for M in shards:
        assert M.device_error() == 0
        M.free()


def test_row_shards_single_rank_on_gpu():
    hm = built("exp3d_4096", lambda: hlr.build(hlr.Problem.exp3d(4096)))
    M = hlr.upload(hm)
    sh = hdist.RowShards([0, hm.n], 0, 1)
    x = torch.randn(hm.n, dtype=torch.float64, device="cuda")
    y = torch.zeros(hm.n, dtype=torch.float64, device="cuda")
    y2 = torch.zeros_like(y)
    sh.mul_vec(0.5, 0, lambda a, op, xx, yy: hlr.mul_vec(a, op, M, xx, yy), x, y)
    hlr.mul_vec(0.5, 0, M, x, y2)
    torch.cuda.synchronize()
    assert torch.equal(y, y2)
    M.free()
