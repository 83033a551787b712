"""CPU: the multi-rank plumbing of bench.py with two gloo ranks (processes started with
spawn, rendezvous on 127.0.0.1): the barrier, the max-over-ranks step time, rank-disjoint
cameras and the whole-job views/s.  The path shards by view with no data-path
collective, so this host logic is all that differs at N > 1."""
import datetime
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import numpy as np
    import torch
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench._barrier(True)
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, torch.device("cpu"), True)
        cams = bench.rank_cameras(3, rank, W=64, H=48)
        value = bench.aggregate_views_per_s(world, 3, 4, ms)
        q.put((rank, ms, value, np.stack([c.viewmatrix for c in cams]).tolist()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    # every rank sees the slowest rank's time
    assert [o[1] for o in out] == [15.0, 15.0]
    # whole-job throughput: 2 ranks x 3 views x 4 steps in 15 ms
    assert all(o[2] == pytest.approx(2 * 3 * 4 / 0.015) for o in out)
    # each rank draws its own cameras
    assert out[0][3] != out[1][3]


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import torch
    import bench
    assert bench.max_over_ranks(7.5, torch.device("cpu"), False) == 7.5
    a, b = bench.rank_cameras(2, 0, W=32, H=32), bench.rank_cameras(2, 0, W=32, H=32)
    assert all((x.viewmatrix == y.viewmatrix).all() for x, y in zip(a, b))
