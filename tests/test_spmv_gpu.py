"""GPU tests of the dense-vector SpMV and PageRank against float64 restatements
(tolerances in each test: float32 accumulation only). PageRank stops at an L1 change of
1e-6, above what float32 ranks resolve (a tol near 1e-9 would run to max_iter)."""
import numpy as np
import pytest

import apspie_b200 as ap
import oracle

pytestmark = pytest.mark.gpu


def _t(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


@pytest.mark.parametrize("shape,dens", [((1, 1), 1.0), ((300, 500), 0.01), ((4000, 4000), 0.002),
                                        ((2000, 3000), 0.05)])
def test_spmv_matches_float64(ctx, shape, dens):
    import scipy.sparse as sp

    m, n = shape
    A = sp.random(m, n, density=dens, format="csr", dtype=np.float32, random_state=np.random.RandomState(m))
    g = ap.HostGraph(m, n, A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float32))
    x = np.random.default_rng(1).uniform(-1, 1, n).astype(np.float32)
    y0 = np.random.default_rng(2).uniform(-1, 1, m).astype(np.float32)
    y = _t(y0)
    ctx.spmv_into(ap.DeviceGraph(g), _t(x), y, 2.0, 0.5)
    ref = 2.0 * oracle.spmv(A.indptr, A.indices, A.data, x) + 0.5 * y0.astype(np.float64)
    bound = 2.0 * oracle.spmv(A.indptr, A.indices, np.abs(A.data), np.abs(x)) + 0.5 * np.abs(y0)
    assert np.all(np.abs(y.cpu().numpy() - ref) <= 1e-5 * bound + 1e-6)


def test_spmv_pattern_counts_degrees(ctx):
    g = ap.gen_rmat(12, 16, 1, 3, weights=False)
    y = _t(np.zeros(g.m))
    ctx.spmv_into(ap.DeviceGraph(g), _t(np.ones(g.m)), y)
    np.testing.assert_array_equal(y.cpu().numpy(), np.diff(g.row_ptr).astype(np.float32))


@pytest.mark.parametrize("key", ["test_pr_d", "test_pr_u", "test_cc_d", "chesapeake_u"])
def test_pagerank_fixtures(ctx, golden, key):
    rp, ci = golden[key + "_row_ptr"], golden[key + "_col_ind"]
    m = rp.shape[0] - 1
    g = ap.HostGraph(m, m, rp, ci, None, key.endswith("_u"))
    r, it = ctx.pagerank(ap.DeviceGraph(g), 0.85, 1e-6, 200)
    ref, rit = oracle.pagerank(rp, ci, 0.85, 1e-6, 200)
    np.testing.assert_allclose(r.cpu().numpy(), ref, rtol=1e-4, atol=1e-7)
    assert abs(it - rit) <= 2
    assert abs(float(r.sum().item()) - 1.0) < 1e-4


@pytest.mark.parametrize("symmetric", [True, False])
def test_pagerank_rmat(ctx, symmetric):
    g = ap.gen_rmat(14, 16, 1, 3, weights=False)
    if not symmetric:
        keep = np.repeat(np.arange(g.m), np.diff(g.row_ptr)) < g.col_ind  # upper triangle: a DAG
        rows = np.repeat(np.arange(g.m), np.diff(g.row_ptr))[keep]
        rp = np.zeros(g.m + 1, dtype=np.int32)
        rp[1:] = np.cumsum(np.bincount(rows, minlength=g.m))
        g = ap.HostGraph(g.m, g.m, rp, g.col_ind[keep].astype(np.int32), None, False)
    r, it = ctx.pagerank(ap.DeviceGraph(g), 0.85, 1e-6, 100)
    ref, _ = oracle.pagerank(g.row_ptr, g.col_ind, 0.85, 1e-6, 100)
    np.testing.assert_allclose(r.cpu().numpy(), ref, rtol=2e-4, atol=1e-8)
