"""The multi-rank logic of bench.py on CPU: two gloo ranks on 127.0.0.1.

bench.py --gpus N runs N independent replicas; the only exchange is the
max-over-ranks reduction of each timed region, which every rank performs at
the same point.  The reduction helper is exercised here with world size 2."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from conftest import ROOT  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import datetime

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # ranks report different times; both must see the largest
        got = [bench.max_over_ranks(1.5 + rank, world, torch.device("cpu")) for _ in range(3)]
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert results == {0: [2.5] * 3, 1: [2.5] * 3}


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.25, 1, torch.device("cpu")) == 3.25


def test_l2_label_marks_small_workloads_resident():
    """Products streaming less than twice the 126 MB L2 (C1's 19 MB, the H^2
    form of C3 at 248 MB) are labelled L2-resident; C2's 11 GB is not."""
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.l2_label(19e6).startswith("L2-resident")
    assert bench.l2_label(248e6).startswith("L2-resident")
    assert bench.l2_label(295e6).startswith("inputs larger than L2")
    assert bench.l2_label(11.07e9).startswith("inputs larger than L2")


def test_products_per_graph_gives_several_runs():
    sys.path.insert(0, str(ROOT))
    import bench
    # the driver's 20 timed products run as 5 replays of 4, the default 300 as 6 of 50
    assert bench.products_per_graph(20) == 4
    assert bench.products_per_graph(300) == 50
    for k in (1, 3, 7, 10, 64, 97, 500):
        d = bench.products_per_graph(k)
        assert k % d == 0 and d <= 50 and k // d >= min(k, 5)
