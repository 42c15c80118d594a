"""Row-sharded product (hlr_b200.dist) on CPU: the row cuts, the shard
descriptors against the oracle, and the collectives of the product with two
gloo ranks on 127.0.0.1 (each rank's local product is the oracle's
restatement of hlr::seq::mul_vec on its shard)."""
import os
import socket
import sys

import numpy as np
import pytest

import hlr_b200 as hlr
import oracle
from hlr_b200 import dist as hdist

from conftest import ROOT, built, relerr

torch = pytest.importorskip("torch")


def _log1d():
    return built("log1d_2048", lambda: hlr.build(hlr.Problem.log1d(2048)))


def _exp3d():
    return built("exp3d_4096", lambda: hlr.build(hlr.Problem.exp3d(4096)))


@pytest.mark.parametrize("parts", [1, 2, 3, 4, 8])
def test_row_cuts_do_not_split_leaves(parts):
    hm = _exp3d()
    cuts = hdist.row_cuts(hm, parts)
    assert len(cuts) == parts + 1 and cuts[0] == 0 and cuts[-1] == hm.n
    assert cuts == sorted(cuts)
    d = hm.h_desc()
    for i in range(int(d.nblocks)):
        b = d.blocks[i]
        for c in cuts:
            assert not (b.row0 < c < b.row0 + b.nrows)
    # about equal stored bytes when every shard is non-empty
    sizes = [sum(hdist._block_bytes(b) for b in hdist._blocks(hdist.shard_desc(hm, cuts[r], cuts[r + 1])))
             for r in range(parts)]
    assert sum(sizes) == sum(hdist._block_bytes(b) for b in hdist._blocks(d))
    if parts <= 4:
        assert max(sizes) <= 1.6 * sum(sizes) / parts


@pytest.mark.parametrize("op", [0, 1])
def test_shards_reassemble_the_product(op):
    hm = _exp3d()
    cuts = hdist.row_cuts(hm, 3)
    rng = np.random.default_rng(5 + op)
    x = rng.standard_normal(hm.n)
    yref = np.zeros(hm.n)
    oracle.hmvm_seq(hm.h_desc(), 0.75, op, x, yref)
    y = np.zeros(hm.n)
    for r in range(3):
        a, b = cuts[r], cuts[r + 1]
        sd = hdist.shard_desc(hm, a, b)
        assert sd.nrows == b - a and sd.ncols == hm.n
        if op == 0:
            yr = np.zeros(b - a)
            oracle.hmvm_seq(sd, 0.75, 0, x, yr)
            y[a:b] += yr
        else:   # op T: each shard's A_r^T x_r is a full-length partial
            part = np.zeros(hm.n)
            oracle.hmvm_seq(sd, 0.75, 1, np.ascontiguousarray(x[a:b]), part)
            y += part
    assert relerr(y, yref) < 1e-13


def test_shard_rejects_straddling_range():
    hm = _log1d()
    cuts = hdist.row_cuts(hm, 2)
    with pytest.raises(ValueError):
        hdist.shard_desc(hm, 1, cuts[1])   # row 1 is inside the first leaf
    with pytest.raises(ValueError):
        hdist.RowShards([0, 5, 3], 0, 2)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import datetime

    import torch.distributed as tdist

    import hlr_b200 as h
    import oracle as orc
    from hlr_b200 import dist as hd
    tdist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        hm = h.build(h.Problem.log1d(2048))
        cuts = hd.row_cuts(hm, world)
        sh = hd.RowShards(cuts, rank, world)
        sd = hd.shard_desc(hm, sh.r0, sh.r1)

        def local(alpha, op, x, y):   # the oracle stands in for the device product on CPU
            orc.hmvm_seq(sd, alpha, op, x.contiguous().numpy(), y.numpy())

        res = {}
        for op in (0, 1):
            rng = np.random.default_rng(11 + op)   # same x and y on every rank
            x = torch.from_numpy(rng.standard_normal(hm.n))
            y0 = torch.from_numpy(rng.standard_normal(hm.n))
            y_local = y0[sh.r0:sh.r1].clone()
            sh.mul_vec(2.0, op, local, x[sh.r0:sh.r1].clone(), y_local)
            yref = y0.numpy().copy()
            orc.hmvm_seq(hm.h_desc(), 2.0, op, x.numpy(), yref)
            res[op] = (float(np.linalg.norm(y_local.numpy() - yref[sh.r0:sh.r1])),
                       float(np.linalg.norm(yref[sh.r0:sh.r1])))
        out.put((rank, cuts, res))
    finally:
        tdist.destroy_process_group()


def test_sharded_product_two_gloo_ranks():
    world, port = 2, _free_port()
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    cuts = {tuple(c) for _, c, _ in results}
    assert len(cuts) == 1   # both ranks cut the same way
    (c,) = cuts
    assert 0 < c[1] < c[2]
    for rank, _, res in results:
        for op, (err, ref) in res.items():
            assert err <= 1e-13 * ref, (rank, op)


def test_row_cuts_c_abi_arguments():
    """hlrc_row_cuts refuses a missing descriptor, parts < 1 and leaves
    outside the rows (HLRC_ERR_ARG / HLRC_ERR_SHAPE)."""
    import ctypes as C
    hm = _log1d()
    d = hm.h_desc()
    out = (C.c_int64 * 3)()
    assert hlr.lib().hlrc_row_cuts(None, 2, out) == 1
    assert hlr.lib().hlrc_row_cuts(C.byref(d), 0, out) == 1
    bad = hdist.shard_desc(hm, 0, hm.n)
    bad.nrows = 100   # leaves now reach past the rows
    assert hlr.lib().hlrc_row_cuts(C.byref(bad), 2, out) == 2
    assert hlr.lib().hlrc_row_cuts(C.byref(d), 2, out) == 0
    assert list(out) == hdist.row_cuts(hm, 2)
