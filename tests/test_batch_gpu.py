"""GPU parity tests of the batched multi-source BFS: every row of the batch output must equal
the single-source BFS of that source (and the oracle), bit-exact."""
import numpy as np
import pytest

import apspie_b200 as ap
import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rmat14():
    g = ap.gen_rmat(14, 16, 1, 3)
    return g, ap.DeviceGraph(g)


def _srcs(g, n, seed=6):
    import torch

    return torch.from_numpy(ap.lcc_sample(g, n, seed)).cuda()


@pytest.mark.parametrize("nq", [1, 5, 32, 33, 100, 512])
def test_batch_rows_equal_single_bfs(ctx, rmat14, nq):
    g, dg = rmat14
    s = _srcs(g, nq)
    out = ctx.bfs_batch(dg, s).cpu().numpy()
    for q, src in enumerate(s.cpu().numpy().tolist()):
        np.testing.assert_array_equal(out[q], ctx.bfs(dg, src).cpu().numpy(), err_msg=f"query {q}")
    for q in (0, nq - 1):
        np.testing.assert_array_equal(out[q], oracle.bfs(g.row_ptr, g.col_ind, int(s[q])))


@pytest.mark.parametrize("frac", [0.0, 1e9])
def test_batch_push_only_and_pull_only(ctx, rmat14, frac):
    import torch

    g, dg = rmat14
    s = _srcs(g, 64, 9)
    ctx.set_batch_push_frac(frac)
    try:
        out = torch.empty((64, g.m), dtype=torch.int32, device="cuda")
        st = ctx.bfs_batch_into(dg, s, out, stats=True)
    finally:
        ctx.set_batch_push_frac(0.05)
    if frac == 0.0:
        assert st["push_iterations"] == 0
    else:
        assert st["pull_iterations"] == 0
    out = out.cpu().numpy()
    for q in range(0, 64, 7):
        np.testing.assert_array_equal(out[q], oracle.bfs(g.row_ptr, g.col_ind, int(s[q])))


def test_batch_duplicate_sources_and_chunking(ctx, rmat14):
    import torch

    g, dg = rmat14
    base = ap.lcc_sample(g, 300, 3)
    srcs = np.concatenate([base, base[:300], base[:13]]).astype(np.int32)  # 613 -> two launches
    out = ctx.bfs_batch(dg, torch.from_numpy(srcs).cuda()).cpu().numpy()
    for q in (0, 299, 300, 599, 612):
        np.testing.assert_array_equal(out[q], oracle.bfs(g.row_ptr, g.col_ind, int(srcs[q])))
    np.testing.assert_array_equal(out[0], out[300])


def test_batch_depth_cap(ctx, rmat14):
    g, dg = rmat14
    s = _srcs(g, 40)
    out = ctx.bfs_batch(dg, s, depth_cap=3).cpu().numpy()
    for q in range(0, 40, 9):
        full = oracle.bfs(g.row_ptr, g.col_ind, int(s[q]))
        np.testing.assert_array_equal(out[q], np.where((full >= 0) & (full < 3), full, -1))


def test_batch_directed_graph(ctx, golden):
    import torch

    rp, ci = golden["chesapeake_d_row_ptr"], golden["chesapeake_d_col_ind"]
    g = ap.HostGraph(rp.shape[0] - 1, rp.shape[0] - 1, rp, ci)
    out = ctx.bfs_batch(ap.DeviceGraph(g), torch.arange(g.m, dtype=torch.int32, device="cuda")).cpu().numpy()
    np.testing.assert_array_equal(out, golden["chesapeake_d_bfs"])


def test_batch_rmat22_full_size(ctx):
    """R-MAT scale 22 (the batched config): 128 LCC sources, rows checked against the oracle."""
    import torch

    g = ap.gen_rmat(22, 16, 1, 3, weights=False)
    dg = ap.DeviceGraph(g)
    s = torch.from_numpy(ap.lcc_sample(g, 128, 6)).cuda()
    out = ctx.bfs_batch(dg, s)
    for q in (0, 63, 127):
        np.testing.assert_array_equal(out[q].cpu().numpy(), oracle.bfs(g.row_ptr, g.col_ind, int(s[q])))


# ------------------------------------------------------------------ batched SSSP
@pytest.mark.parametrize("groups", [0, 3, 64, -1])
@pytest.mark.parametrize("nq", [1, 7, 32, 100, 512])
def test_sssp_batch_rows_equal_single_sssp(ctx, rmat14, nq, groups):
    """groups 0 (the default) and -1: the multi-query kernel; 3 / 64: that many query
    groups (64 > 7 queries leaves groups idle)."""
    g, dg = rmat14
    s = _srcs(g, nq, 4)
    ctx.set_sssp_batch_groups(groups)
    try:
        out = ctx.sssp_batch(dg, s).cpu().numpy()
        st = ctx.sssp_batch_into(dg, s, torch_empty_like_rows(nq, g.m), stats=True)
    finally:
        ctx.set_sssp_batch_groups(0)
    assert st["edges_expanded"] > 0
    for q in sorted({0, nq // 2, nq - 1}):
        np.testing.assert_array_equal(out[q], oracle.sssp(g.row_ptr, g.col_ind, g.val, int(s[q])), err_msg=f"q{q}")
    for q in range(0, nq, max(1, nq // 8)):
        np.testing.assert_array_equal(out[q], ctx.sssp(dg, int(s[q])).cpu().numpy())


def torch_empty_like_rows(nq, m):
    import torch

    return torch.empty((nq, m), dtype=torch.int32, device="cuda")


def test_sssp_batch_duplicates_and_unreached(ctx, golden):
    import torch

    rp, ci = golden["test_cc_u_row_ptr"], golden["test_cc_u_col_ind"]
    w = golden["test_cc_u_w"]
    g = ap.HostGraph(rp.shape[0] - 1, rp.shape[0] - 1, rp, ci, w, True)
    srcs = torch.tensor([0, 3, 3, 9, 0], dtype=torch.int32, device="cuda")
    out = ctx.sssp_batch(ap.DeviceGraph(g), srcs).cpu().numpy()
    for q, s in enumerate(srcs.cpu().numpy().tolist()):
        np.testing.assert_array_equal(out[q], golden["test_cc_u_sssp"][s])


def test_sssp_batch_rmat20_full_size(ctx):
    import torch

    g = ap.gen_rmat(20, 16, 2, 3)
    dg = ap.DeviceGraph(g)
    s = torch.from_numpy(ap.lcc_sample(g, 64, 6)).cuda()
    out = ctx.sssp_batch(dg, s)
    for q in (0, 17, 63):
        np.testing.assert_array_equal(out[q].cpu().numpy(), oracle.sssp(g.row_ptr, g.col_ind, g.val, int(s[q])))


def _chain(weights):
    """Undirected path 0 - 1 - ... - k with the given edge weights."""
    k = len(weights)
    rows = [[] for _ in range(k + 1)]
    for i, w in enumerate(weights):
        rows[i].append((i + 1, w))
        rows[i + 1].append((i, w))
    rp = np.zeros(k + 2, dtype=np.int32)
    ci, wt = [], []
    for i, r in enumerate(sorted(x) for x in rows):
        for c, w in r:
            ci.append(c)
            wt.append(w)
        rp[i + 1] = len(ci)
    return ap.HostGraph(k + 1, k + 1, rp, np.array(ci, dtype=np.int32), np.array(wt, dtype=np.int32), True)


@pytest.mark.parametrize("groups", [0, 2])
@pytest.mark.parametrize("weights,what", [([5, -3, 2], "negative"), ([1 << 30, 1 << 30, 1], "overflow")])
def test_sssp_batch_bad_weights_reported_and_context_reusable(ctx, weights, what, groups):
    """A negative weight, or a distance that leaves int32, is reported as an error (never
    a hang or a wrong answer), and the context answers the next call correctly."""
    import torch

    g = _chain(weights)
    dg = ap.DeviceGraph(g)
    srcs = torch.tensor([0, 3, 1], dtype=torch.int32, device="cuda")
    out = torch.empty((3, g.m), dtype=torch.int32, device="cuda")
    ctx.set_sssp_batch_groups(groups)
    try:
        with pytest.raises(ap.ApspieError):
            ctx.sssp_batch_into(dg, srcs, out, stats=True)
        good = _chain([5, 3, 2])
        got = ctx.sssp_batch(ap.DeviceGraph(good), srcs).cpu().numpy()
    finally:
        ctx.set_sssp_batch_groups(0)
    for q, s in enumerate([0, 3, 1]):
        np.testing.assert_array_equal(got[q], oracle.sssp(good.row_ptr, good.col_ind, good.val, s))


def test_sssp_single_source_overflow_reported(ctx):
    import torch

    g = _chain([1 << 30, 1 << 30, 1])
    out = torch.empty(g.m, dtype=torch.int32, device="cuda")
    with pytest.raises(ap.ApspieError):
        ctx.sssp_into(ap.DeviceGraph(g), 0, out, stats=True)
    g2 = _chain([(1 << 30) - 1, (1 << 30) - 1])  # 2^31 - 2 is the largest distance allowed
    np.testing.assert_array_equal(ctx.sssp(ap.DeviceGraph(g2), 0).cpu().numpy(),
                                  oracle.sssp(g2.row_ptr, g2.col_ind, g2.val, 0))


@pytest.mark.parametrize("kind,groups", [("bfs", 0), ("sssp", 0), ("sssp", 2)])
@pytest.mark.parametrize("bad", [-1, "m"])
def test_batch_source_out_of_range_reported(ctx, rmat14, kind, groups, bad):
    """Sources live in device memory, so the kernels range-check them: an out-of-range
    source is reported as an invalid argument (nothing is written for it) and the context
    answers the next call."""
    import torch

    g, dg = rmat14
    b = g.m if bad == "m" else bad
    srcs = torch.tensor([0, b, 5], dtype=torch.int32, device="cuda")
    out = torch.empty((3, g.m), dtype=torch.int32, device="cuda")
    ctx.set_sssp_batch_groups(groups)
    try:
        with pytest.raises(ap.ApspieError):
            if kind == "bfs":
                ctx.bfs_batch_into(dg, srcs, out, stats=True)
            else:
                ctx.sssp_batch_into(dg, srcs, out, stats=True)
        good = torch.tensor([0, 5], dtype=torch.int32, device="cuda")
        got = (ctx.bfs_batch(dg, good) if kind == "bfs" else ctx.sssp_batch(dg, good)).cpu().numpy()
    finally:
        ctx.set_sssp_batch_groups(0)
    for q, s in enumerate([0, 5]):
        ref = oracle.bfs(g.row_ptr, g.col_ind, s) if kind == "bfs" else oracle.sssp(g.row_ptr, g.col_ind, g.val, s)
        np.testing.assert_array_equal(got[q], ref)
