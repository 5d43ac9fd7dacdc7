"""CPU tests of bench.py's multi-rank plumbing (world size 2 over gloo) and of its
deterministic serving stream. No GPU: the ranks only exercise the host-side logic."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=30))
    try:
        import bench

        got_ws, got_rank, _ = bench.dist_env()
        bench.barrier(ws)
        slowest = bench.max_over_ranks(ws, 1.5 + rank)  # rank 1 is the slow one
        bench.barrier(ws)
        q.put((rank, got_ws, got_rank, slowest))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_barrier_world_size_2():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[0] for r in res] == [0, 1]
    assert all(r[1] == 2 and r[2] == r[0] for r in res)
    assert all(r[3] == 2.5 for r in res)  # every rank reports the max over ranks


def test_single_rank_helpers_are_identity():
    import bench

    assert bench.max_over_ranks(1, 3.25) == 3.25
    bench.barrier(1)


def test_serving_stream_is_deterministic_and_follows_the_mix():
    import bench

    class G:
        def __init__(self, m):
            self.m = m

    graphs = [G(1 << 16), G(1 << 18), G(1 << 20), G(1 << 22)]
    a = bench.serve_stream(graphs, 4000, 1000.0)
    b = bench.serve_stream(graphs, 4000, 1000.0)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(np.asarray(x), np.asarray(y))
    kinds, which, srcs, arrive = a
    frac = np.bincount(kinds, minlength=3) / len(kinds)
    assert abs(frac[0] - 0.70) < 0.03 and abs(frac[1] - 0.25) < 0.03 and abs(frac[2] - 0.05) < 0.02
    assert set(np.unique(which)) == {0, 1, 2, 3}
    assert all(0 <= s < graphs[w].m for s, w in zip(srcs, which))
    gaps = np.diff(arrive)
    assert np.all(gaps >= 0) and abs(gaps.mean() - 1e-3) < 1e-4  # Poisson at 1000 queries/s
    sat = bench.serve_stream(graphs, 10, 0.0)
    assert np.all(sat[3] == 0)
