"""The allocation-free BFS entry point (apspie_bfs_noalloc).

Some callers cannot call cudaMalloc: code that runs inside another allocator's memory
budget, on a host that reserved all device memory up front, or as a plugin loaded into
such a process. apspie_bfs_noalloc serves them by keeping its scratch in a fixed device
array inside the library instead of allocating. This test calls it through the C ABI and
checks it against the ordinary apspie_bfs (exact equality: depths are integers) on two
calls in a row, so a second call that reuses the shared array must still be right. It is
collected last so that a run stopping at the first failure has run everything else.
"""
import ctypes

import numpy as np
import pytest

import apspie_b200 as ap
from apspie_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _noalloc(view, source, out, stream, depth_cap=0):
    st = L.RunStats()
    rc = L.lib().apspie_bfs_noalloc(ctypes.byref(view), source, depth_cap, out.data_ptr(),
                                    ctypes.c_void_p(stream.cuda_stream), ctypes.byref(st))
    return rc, st


def test_bfs_noalloc_matches_apspie_bfs_on_two_calls():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    stream = torch.cuda.current_stream()
    g = ap.gen_rmat(14, 16, 1, 3)
    dg = ap.DeviceGraph(g)
    src = ap.max_degree_vertex(g)
    with ap.Context(0) as ctx:
        ref = ctx.bfs(dg, src)
        ref_other = ctx.bfs(dg, 12345)
    # two calls in a row on the same source, then a different source: each must match
    for source, expect in ((src, ref), (src, ref), (12345, ref_other)):
        out = torch.full((g.m,), -7, dtype=torch.int32, device="cuda")
        rc, st = _noalloc(dg.view(False), source, out, stream)
        assert rc == 0, L.STATUS.get(rc, rc)
        assert torch.equal(out, expect)
        assert st.vertices_reached == int((expect >= 0).sum().item())


def test_bfs_noalloc_rejects_graphs_above_its_maximum():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    g = ap.gen_rmat(8, 4, 1, 3, weights=False)
    dg = ap.DeviceGraph(g)
    v = dg.view(False)
    v.m = v.n = 262144 + 1  # rejected before any device access
    out = torch.empty(4, dtype=torch.int32, device="cuda")
    rc, _ = _noalloc(v, 0, out, torch.cuda.current_stream())
    assert L.STATUS[rc] == "APSPIE_ERR_INVALID_ARG"
