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


def test_bfs_noalloc_at_its_maximum_size_with_depth_cap_on_a_side_stream():
    """A graph of exactly APSPIE_NOALLOC_MAX_VERTICES vertices (R-MAT scale 18), where the
    fixed queues and bitmaps are full-size; then a depth cap, on a stream other than the
    current one, twice in a row."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    g = ap.gen_rmat(18, 4, 11, 3, weights=False)
    assert g.m == 262144
    dg = ap.DeviceGraph(g)
    src = ap.max_degree_vertex(g)
    with ap.Context(0) as ctx:
        ref = ctx.bfs(dg, src)
        ref_cap = ctx.bfs(dg, src, depth_cap=2)
    side = torch.cuda.Stream()
    for cap, expect in ((0, ref), (2, ref_cap), (2, ref_cap), (0, ref)):
        out = torch.full((g.m,), -7, dtype=torch.int32, device="cuda")
        torch.cuda.current_stream().synchronize()
        rc, st = _noalloc(dg.view(True), src, out, side, depth_cap=cap)
        assert rc == 0, L.STATUS.get(rc, rc)
        assert torch.equal(out, expect), cap
    assert int((ref_cap >= 0).sum()) < int((ref >= 0).sum())


_OWN_CONTEXT_SCRIPT = r"""
import ctypes, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import apspie_b200 as ap
from apspie_b200 import _lib as L
import oracle

cu = ctypes.CDLL("libcuda.so.1")
def ok(rc, what):
    if rc != 0:
        raise SystemExit(f"{what}: CUresult {rc}")
ok(cu.cuInit(0), "cuInit")
dev = ctypes.c_int()
ok(cu.cuDeviceGet(ctypes.byref(dev), 0), "cuDeviceGet")
g = ap.gen_rmat(12, 8, 5, 3, weights=False)
src = ap.max_degree_vertex(g)
expect = oracle.bfs(g.row_ptr, g.col_ind, src)
lib = L.lib()

def run_in_current_context():
    bufs = []
    def upload(a):
        p = ctypes.c_uint64()
        ok(cu.cuMemAlloc_v2(ctypes.byref(p), ctypes.c_size_t(a.nbytes)), "cuMemAlloc")
        ok(cu.cuMemcpyHtoD_v2(p, a.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(a.nbytes)), "HtoD")
        bufs.append(p)
        return p.value
    v = L.CSR()
    v.m = v.n = g.m
    v.nnz = g.nnz
    v.val_type = L.VAL_NONE
    v.row_ptr = upload(np.ascontiguousarray(g.row_ptr))
    v.col_ind = upload(np.ascontiguousarray(g.col_ind))
    v.val = None
    v.flags = 1
    out = upload(np.full(g.m, -7, dtype=np.int32))
    for _ in range(2):
        rc = lib.apspie_bfs_noalloc(ctypes.byref(v), src, 0, out, None, None)
        if rc != 0:
            raise SystemExit(f"apspie_bfs_noalloc: {L.STATUS.get(rc, rc)}")
        got = np.empty(g.m, dtype=np.int32)
        ok(cu.cuMemcpyDtoH_v2(got.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint64(out), ctypes.c_size_t(got.nbytes)), "DtoH")
        if not np.array_equal(got, expect):
            raise SystemExit("depths differ from the oracle")
    for p in bufs:
        ok(cu.cuMemFree_v2(p), "cuMemFree")

# a context of the caller's own, made with the driver API, first
own = ctypes.c_void_p()
ok(cu.cuCtxCreate_v2(ctypes.byref(own), 0, dev), "cuCtxCreate")
run_in_current_context()
# then the device's primary context, while the caller's context still exists
primary = ctypes.c_void_p()
ok(cu.cuDevicePrimaryCtxRetain(ctypes.byref(primary), dev), "cuDevicePrimaryCtxRetain")
ok(cu.cuCtxSetCurrent(primary), "cuCtxSetCurrent")
run_in_current_context()
ok(cu.cuCtxSetCurrent(own), "cuCtxSetCurrent")
run_in_current_context()
ok(cu.cuCtxSetCurrent(None), "cuCtxSetCurrent")
ok(cu.cuCtxDestroy_v2(own), "cuCtxDestroy")
ok(cu.cuDevicePrimaryCtxRelease_v2(dev), "cuDevicePrimaryCtxRelease")
print("own-context ok")
"""


def test_bfs_noalloc_in_a_context_the_caller_created():
    """A plugin host may run the library inside a CUDA context it made itself
    (cuCtxCreate): the fixed array then has a separate address in that context and in the
    device's primary context. Calls alternate between the two, both alive, each checked
    against the oracle; a fresh process keeps torch out of the contexts."""
    import os
    import subprocess
    import sys

    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = subprocess.run([sys.executable, "-c", _OWN_CONTEXT_SCRIPT, root], capture_output=True, text=True,
                         timeout=300)
    assert res.returncode == 0 and "own-context ok" in res.stdout, res.stdout[-2000:] + res.stderr[-2000:]
