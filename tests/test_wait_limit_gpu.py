"""Bounded device-side waits: a grid barrier that one block never reaches runs out after
the context's wait limit, every block of the launch returns, the call reports
APSPIE_ERR_TIMEOUT, and the same context then answers correctly. The failure is made by a
block that leaves before arriving (no fault, no trap, no endless loop)."""
import time

import numpy as np
import pytest

import apspie_b200 as ap
import oracle

pytestmark = pytest.mark.gpu


def test_barrier_check_passes_with_every_block_present():
    with ap.Context(0) as c:
        grid = c.grid_barrier_check(rounds=64)
        assert grid > 0


def test_barrier_wait_runs_out_then_context_answers():
    import torch

    g = ap.gen_rmat(12, 16, 1, 3)
    src = ap.max_degree_vertex(g)
    with ap.Context(0) as c:
        c.set_wait_limit(1_000_000)  # 1 ms
        for absent in (0, 1):
            t0 = time.perf_counter()
            with pytest.raises(ap.ApspieError) as ei:
                c.grid_barrier_check(rounds=4, absent_block=absent)
            took = time.perf_counter() - t0
            assert ei.value.name == "APSPIE_ERR_TIMEOUT"
            assert took < 2.0  # the 1 ms bound, not the 4 s default
            c.synchronize()  # nothing left pending on the stream
        dg = ap.DeviceGraph(g)
        np.testing.assert_array_equal(c.bfs(dg, src).cpu().numpy(), oracle.bfs(g.row_ptr, g.col_ind, src))
        np.testing.assert_array_equal(c.sssp(dg, src).cpu().numpy(),
                                      oracle.sssp(g.row_ptr, g.col_ind, g.val, src))
        c.set_wait_limit(0)  # back to the default bound
        assert c.grid_barrier_check(rounds=8) > 0
        torch.cuda.synchronize()
