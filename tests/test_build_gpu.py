"""GPU tests of device graph construction: COO -> CSR with the generator's symmetrise /
dedup rules (identical to the host R-MAT CSR), plain COO -> CSR against a numpy
restatement, and CSR transpose against scipy."""
import numpy as np
import pytest

import apspie_b200 as ap

pytestmark = pytest.mark.gpu

SYM, DROP, DEDUP = ap.BUILD_SYMMETRIZE, ap.BUILD_DROP_SELF_LOOPS, ap.BUILD_DEDUP


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("scale", [10, 14, 17])
def test_rmat_edge_list_builds_the_host_generator_csr(ctx, scale):
    src, dst, w = ap.gen_rmat_coo(scale, 16, 1, 3)
    g = ap.gen_rmat(scale, 16, 1, 3)
    C = ctx.build_csr(g.m, _dev(src), _dev(dst), _dev(w), SYM | DROP | DEDUP)
    rp, ci, val = C.to_numpy()
    np.testing.assert_array_equal(rp, g.row_ptr)
    np.testing.assert_array_equal(ci, g.col_ind)
    np.testing.assert_array_equal(val, g.val)


def _ref_build(m, src, dst, val, flags):
    a, b = src.astype(np.int64), dst.astype(np.int64)
    order_in = np.arange(a.shape[0])
    if flags & SYM:
        a, b = np.minimum(a, b), np.maximum(a, b)
    keep = np.ones(a.shape[0], dtype=bool)
    if flags & DROP:
        keep &= a != b
    a, b, val, order_in = a[keep], b[keep], val[keep], order_in[keep]
    o = np.lexsort((order_in, b, a))
    a, b, val, order_in = a[o], b[o], val[o], order_in[o]
    if flags & DEDUP and a.shape[0]:
        first = np.concatenate(([True], (a[1:] != a[:-1]) | (b[1:] != b[:-1])))
        a, b, val, order_in = a[first], b[first], val[first], order_in[first]
    if flags & SYM:
        rows = np.concatenate((b, a))
        cols = np.concatenate((a, b))
        val = np.concatenate((val, val))
        tie = np.concatenate((order_in, order_in))
        o = np.lexsort((tie, cols, rows))
        rows, cols, val = rows[o], cols[o], val[o]
    else:
        rows, cols = a, b
    rp = np.zeros(m + 1, dtype=np.int64)
    rp[1:] = np.cumsum(np.bincount(rows, minlength=m))
    return rp.astype(np.int32), cols.astype(np.int32), val


@pytest.mark.parametrize("flags", [0, DROP, DEDUP, DROP | DEDUP, SYM | DROP, SYM | DROP | DEDUP])
@pytest.mark.parametrize("m", [1, 7, 300, 4096])
def test_coo_build_matches_numpy(ctx, flags, m):
    rng = np.random.default_rng(m * 31 + flags)
    ne = 5 * m + 3
    src = rng.integers(0, m, ne).astype(np.int32)
    dst = rng.integers(0, m, ne).astype(np.int32)
    dup = rng.integers(0, ne, ne // 4)
    src[dup[: len(dup) // 2]] = src[dup[len(dup) // 2:][: len(dup) // 2]]
    dst[dup[: len(dup) // 2]] = dst[dup[len(dup) // 2:][: len(dup) // 2]]
    val = rng.uniform(-1, 1, ne).astype(np.float32)
    C = ctx.build_csr(m, _dev(src), _dev(dst), _dev(val), flags)
    rp, ci, v = C.to_numpy()
    erp, eci, ev = _ref_build(m, src, dst, val, flags)
    np.testing.assert_array_equal(rp, erp)
    np.testing.assert_array_equal(ci, eci)
    np.testing.assert_array_equal(v, ev)


def test_coo_build_without_values_and_empty(ctx):
    import torch

    C = ctx.build_csr(5, torch.empty(0, dtype=torch.int32, device="cuda"),
                      torch.empty(0, dtype=torch.int32, device="cuda"), None, SYM | DROP | DEDUP)
    rp, ci, v = C.to_numpy()
    assert rp.tolist() == [0] * 6 and ci.shape[0] == 0 and v is None
    src = np.array([0, 1, 1, 2], dtype=np.int32)
    dst = np.array([1, 0, 2, 2], dtype=np.int32)
    rp, ci, _ = ctx.build_csr(3, _dev(src), _dev(dst), None, SYM | DROP | DEDUP).to_numpy()
    assert rp.tolist() == [0, 1, 3, 4] and ci.tolist() == [1, 0, 2, 1]


def test_coo_build_rejects_out_of_range_ids(ctx):
    src = np.array([0, 5], dtype=np.int32)
    dst = np.array([1, 1], dtype=np.int32)
    with pytest.raises(ap.ApspieError):
        ctx.build_csr(4, _dev(src), _dev(dst))
    # the context stays usable
    rp, ci, _ = ctx.build_csr(4, _dev(src[:1]), _dev(dst[:1])).to_numpy()
    assert rp.tolist() == [0, 1, 1, 1, 1] and ci.tolist() == [1]


@pytest.mark.parametrize("shape", [(1, 1), (50, 300), (3000, 700), (1 << 14, 1 << 14)])
def test_transpose_matches_scipy(ctx, shape):
    import scipy.sparse as sp

    m, n = shape
    A = sp.random(m, n, density=min(1.0, 8.0 / n), format="csr", dtype=np.float32,
                  random_state=np.random.RandomState(m + n))
    A.sort_indices()
    g = ap.HostGraph(m, n, A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float32))
    T = ctx.transpose(ap.DeviceGraph(g))
    rp, ci, v = T.to_numpy()
    AT = A.T.tocsr()
    AT.sort_indices()
    np.testing.assert_array_equal(rp, AT.indptr)
    np.testing.assert_array_equal(ci, AT.indices)
    np.testing.assert_array_equal(v, AT.data)
    # transposing twice gives A back
    rp2, ci2, v2 = ctx.transpose(T).to_numpy()
    np.testing.assert_array_equal(rp2, A.indptr)
    np.testing.assert_array_equal(ci2, A.indices)
    np.testing.assert_array_equal(v2, A.data)
