"""GPU parity tests of the SpMSpV traversals (BFS, SSSP, MIS) through the C ABI.

Bit-exact against golden vectors from the reference's own CPU code (small fixtures, all
sources) and against the oracle on generated R-MAT graphs up to the benchmark's full
size (scale 20)."""
import numpy as np
import pytest

import apspie_b200 as ap
import oracle

pytestmark = pytest.mark.gpu


def _dev(golden, key, with_w=False):
    rp, ci = golden[key + "_row_ptr"], golden[key + "_col_ind"]
    val = golden[key + "_w"] if with_w else None
    g = ap.HostGraph(rp.shape[0] - 1, rp.shape[0] - 1, rp, ci, val, symmetric=key.endswith("_u"))
    return g, ap.DeviceGraph(g)


@pytest.fixture(scope="module")
def rmat14():
    g = ap.gen_rmat(14, 16, 1, 3)
    return g, ap.DeviceGraph(g), ap.max_degree_vertex(g)


@pytest.fixture(scope="module")
def rmat20():
    g = ap.gen_rmat(20, 16, 2, 3)
    return g, ap.DeviceGraph(g), ap.max_degree_vertex(g)


# ------------------------------------------------------------------------------- BFS
def test_bfs_fixtures_all_sources(ctx, golden, fixture_keys):
    for key in fixture_keys:
        g, dg = _dev(golden, key)
        for s in range(g.m):
            got = ctx.bfs(dg, s).cpu().numpy()
            np.testing.assert_array_equal(got, golden[key + "_bfs"][s], err_msg=f"{key} src {s}")


@pytest.mark.parametrize("alpha", [0.0, 14.0, 1e6])
def test_bfs_rmat12_golden_all_directions(ctx, golden, alpha):
    g = ap.gen_rmat(12, 16, 1, 3)
    src = int(golden["rmat12_meta"][2])
    dg = ap.DeviceGraph(g)
    ctx.set_bfs_tuning(alpha, 24.0)
    try:
        d = ctx.bfs(dg, src).cpu().numpy()
    finally:
        ctx.set_bfs_tuning(14.0, 24.0)
    np.testing.assert_array_equal(d, golden["rmat12_bfs"])


def test_bfs_rmat14_many_sources_vs_oracle(ctx, rmat14):
    g, dg, src = rmat14
    rng = np.random.default_rng(0)
    for s in [src] + rng.integers(0, g.m, 12).tolist():
        np.testing.assert_array_equal(ctx.bfs(dg, int(s)).cpu().numpy(), oracle.bfs(g.row_ptr, g.col_ind, int(s)))


def test_bfs_push_and_pull_paths_both_taken(ctx, rmat14):
    import torch

    g, dg, src = rmat14
    out = torch.empty(g.m, dtype=torch.int32, device="cuda")
    st = ctx.bfs_into(dg, src, out, stats=True)
    assert st["push_iterations"] >= 1 and st["pull_iterations"] >= 1, st
    ref = oracle.bfs(g.row_ptr, g.col_ind, src)
    np.testing.assert_array_equal(out.cpu().numpy(), ref)
    reached = ref >= 0
    assert st["vertices_reached"] == int(reached.sum())
    assert st["edges_component"] == int(g.degrees()[reached].sum())
    assert st["iterations"] == int(ref.max()) + 1


def test_bfs_depth_cap(ctx, rmat14):
    g, dg, src = rmat14
    full = oracle.bfs(g.row_ptr, g.col_ind, src)
    for cap in (1, 2, 3):
        got = ctx.bfs(dg, src, depth_cap=cap).cpu().numpy()
        np.testing.assert_array_equal(got, np.where((full >= 0) & (full < cap), full, -1))


def test_bfs_rmat20_full_size(ctx, rmat20):
    g, dg, src = rmat20
    np.testing.assert_array_equal(ctx.bfs(dg, src).cpu().numpy(), oracle.bfs(g.row_ptr, g.col_ind, src))


def test_bfs_isolated_source_and_empty_rows(ctx):
    # vertices 0..3 isolated, a path 4-5-6, vertex 7 isolated
    rp = np.array([0, 0, 0, 0, 0, 1, 3, 4, 4], dtype=np.int32)
    ci = np.array([5, 4, 6, 5], dtype=np.int32)
    g = ap.HostGraph(8, 8, rp, ci, symmetric=True)
    dg = ap.DeviceGraph(g)
    for s in range(8):
        np.testing.assert_array_equal(ctx.bfs(dg, s).cpu().numpy(), oracle.bfs(rp, ci, s))


# ------------------------------------------------------------------------------ SSSP
def test_sssp_fixtures_all_sources(ctx, golden, fixture_keys):
    for key in fixture_keys:
        if key + "_sssp" not in golden:
            continue
        g, dg = _dev(golden, key, with_w=True)
        for s in range(g.m):
            np.testing.assert_array_equal(ctx.sssp(dg, s).cpu().numpy(), golden[key + "_sssp"][s], err_msg=f"{key} {s}")


def test_sssp_rmat12_golden(ctx, golden):
    g = ap.gen_rmat(12, 16, 1, 3)
    np.testing.assert_array_equal(ctx.sssp(ap.DeviceGraph(g), int(golden["rmat12_meta"][2])).cpu().numpy(),
                                  golden["rmat12_sssp"])


def test_sssp_rmat14_vs_oracle(ctx, rmat14):
    import torch

    g, dg, src = rmat14
    out = torch.empty(g.m, dtype=torch.int32, device="cuda")
    st = ctx.sssp_into(dg, src, out, stats=True)
    ref = oracle.sssp(g.row_ptr, g.col_ind, g.val, src)
    np.testing.assert_array_equal(out.cpu().numpy(), ref)
    assert st["vertices_reached"] == int((ref >= 0).sum())


def test_sssp_rmat20_full_size(ctx, rmat20):
    g, dg, src = rmat20
    np.testing.assert_array_equal(ctx.sssp(dg, src).cpu().numpy(), oracle.sssp(g.row_ptr, g.col_ind, g.val, src))


def test_sssp_zero_weights_and_repeated_calls(ctx, rmat14):
    g, _, src = rmat14
    w = g.val.copy()
    w[::3] = 0
    h = ap.HostGraph(g.m, g.n, g.row_ptr, g.col_ind, w, symmetric=True)
    dg = ap.DeviceGraph(h)
    ref = oracle.sssp(h.row_ptr, h.col_ind, h.val, src)
    for _ in range(3):
        np.testing.assert_array_equal(ctx.sssp(dg, src).cpu().numpy(), ref)


# ------------------------------------------------------------------------------- MIS
def test_mis_fixtures(ctx, golden, fixture_keys):
    import torch

    for key in fixture_keys:
        if key + "_mis" not in golden:
            continue
        g, dg = _dev(golden, key)
        prio = torch.from_numpy(golden["mt19937_seed4"][: g.m].astype(np.uint32).view(np.int32)).cuda()
        got = ctx.mis(dg, prio).cpu().numpy()
        np.testing.assert_array_equal(got, golden[key + "_mis"], err_msg=key)


def _prio(m):
    import torch

    return torch.from_numpy(ap.mt19937_u32(4, m).view(np.int32)).cuda()


def test_mis_rmat12_golden(ctx, golden):
    g = ap.gen_rmat(12, 16, 1, 3)
    got = ctx.mis(ap.DeviceGraph(g), _prio(g.m)).cpu().numpy()
    np.testing.assert_array_equal(got, golden["rmat12_mis"])


def test_mis_rmat20_full_size(ctx, rmat20):
    g, dg, _ = rmat20
    pr = ap.mt19937_u32(4, g.m)
    got = ctx.mis(dg, _prio(g.m)).cpu().numpy()
    ref = oracle.mis_greedy(g.row_ptr, g.col_ind, pr)
    np.testing.assert_array_equal(got, ref)
    assert oracle.mis_check(g.row_ptr, g.col_ind, got) == 0


def test_mis_priority_ties_broken_by_id(ctx, rmat14):
    import torch

    g, dg, _ = rmat14
    pr = (ap.mt19937_u32(9, g.m) % 4).astype(np.uint32)  # heavy ties
    got = ctx.mis(dg, torch.from_numpy(pr.view(np.int32)).cuda()).cpu().numpy()
    np.testing.assert_array_equal(got, oracle.mis_greedy(g.row_ptr, g.col_ind, pr))


# ----------------------------------------------------------------- SpMSpV (one hop)
def test_spmspv_bool_matches_mis_check_semantics(ctx, rmat14):
    import torch

    g, dg, _ = rmat14
    x = (np.arange(g.m) % 7 == 0).astype(np.int32)
    y = torch.empty(g.m, dtype=torch.int32, device="cuda")
    ctx.spmspv_bool_into(dg, torch.from_numpy(x).cuda(), y)
    exp = np.zeros(g.m, dtype=np.int32)
    for u in np.flatnonzero(x):
        exp[g.col_ind[g.row_ptr[u]:g.row_ptr[u + 1]]] = 1
    np.testing.assert_array_equal(y.cpu().numpy(), exp)


# ------------------------------------------------------------------------ errors
def test_invalid_arguments_rejected(ctx, rmat14):
    import torch

    g, dg, src = rmat14
    out = torch.empty(g.m, dtype=torch.int32, device="cuda")
    with pytest.raises(ap.ApspieError) as e:
        ctx.bfs_into(dg, g.m, out)
    assert e.value.name == "APSPIE_ERR_INVALID_ARG"
    with pytest.raises(ap.ApspieError):
        ctx.bfs_into(dg, -1, out)
    with pytest.raises(ap.ApspieError):  # SSSP needs int32 weights
        ctx.sssp_into(ap.DeviceGraph(ap.HostGraph(g.m, g.n, g.row_ptr, g.col_ind, None)), src, out)
    # the context stays usable
    np.testing.assert_array_equal(ctx.bfs(dg, src).cpu().numpy(), oracle.bfs(g.row_ptr, g.col_ind, src))


def test_poisoned_csr_caught_by_validation(ctx, rmat14):
    g, _, src = rmat14
    bad = g.col_ind.copy()
    bad[123] = g.m + 5  # column out of range
    dg = ap.DeviceGraph(ap.HostGraph(g.m, g.n, g.row_ptr, bad, g.val, symmetric=True))
    with pytest.raises(ap.ApspieError):
        ctx.validate(dg)
    ctx.set_validate(True)
    try:
        with pytest.raises(ap.ApspieError) as e:
            ctx.bfs(dg, src)
        assert "column index out of range" in str(e.value)
        rp = g.row_ptr.copy()
        rp[5], rp[6] = rp[6], rp[5]
        dg2 = ap.DeviceGraph(ap.HostGraph(g.m, g.n, rp, g.col_ind, g.val))
        with pytest.raises(ap.ApspieError):
            ctx.sssp(dg2, src)
    finally:
        ctx.set_validate(False)
    good = ap.DeviceGraph(g)
    np.testing.assert_array_equal(ctx.bfs(good, src).cpu().numpy(), oracle.bfs(g.row_ptr, g.col_ind, src))


def test_negative_weight_reported_not_hung(ctx):
    rp = np.array([0, 1, 2], dtype=np.int32)
    ci = np.array([1, 0], dtype=np.int32)
    w = np.array([-3, -3], dtype=np.int32)
    dg = ap.DeviceGraph(ap.HostGraph(2, 2, rp, ci, w))
    import torch

    out = torch.empty(2, dtype=torch.int32, device="cuda")
    with pytest.raises(ap.ApspieError):
        ctx.sssp_into(dg, 0, out, stats=True)


def test_bfs_directed_graph_never_pulls(ctx, golden):
    """A directed pattern must be expanded top-down only: pull would follow in-edges."""
    import torch

    g, dg = _dev(golden, "chesapeake_d")
    assert not dg.symmetric
    out = torch.empty(g.m, dtype=torch.int32, device="cuda")
    for s in range(g.m):
        st = ctx.bfs_into(dg, s, out, stats=True)
        assert st["pull_iterations"] == 0
        np.testing.assert_array_equal(out.cpu().numpy(), golden["chesapeake_d_bfs"][s])


@pytest.mark.parametrize("delta", [1, 7, 64, 100000])
def test_sssp_bucket_width_does_not_change_result(ctx, rmat14, delta):
    g, dg, src = rmat14
    ref = oracle.sssp(g.row_ptr, g.col_ind, g.val, src)
    ctx.set_sssp_delta(delta)
    try:
        np.testing.assert_array_equal(ctx.sssp(dg, src).cpu().numpy(), ref)
    finally:
        ctx.set_sssp_delta(0)


@pytest.mark.parametrize("band", [-1, 1, 4096, 0, 1 << 40])
@pytest.mark.parametrize("delta", [0, 64])
def test_sssp_band_does_not_change_result(ctx, rmat14, band, delta):
    """The distance band only orders the work: band 1 expands one histogram bin per
    iteration (deferring almost the whole frontier every time), -1 and 2^40 never defer."""
    g, dg, src = rmat14
    ref = oracle.sssp(g.row_ptr, g.col_ind, g.val, src)
    ctx.set_sssp_band(band)
    ctx.set_sssp_delta(delta)
    try:
        out = ctx.sssp(dg, src)
        st = ctx.sssp_into(dg, src, out, stats=True)
        np.testing.assert_array_equal(out.cpu().numpy(), ref)
        assert st["edges_expanded"] >= st["edges_component"]
    finally:
        ctx.set_sssp_band(0)
        ctx.set_sssp_delta(0)


def test_sssp_band_cuts_rework(ctx, rmat14):
    """With the default band, re-expansion stays near one pass over the component's edges
    (a whole-frontier Bellman-Ford pass expands several times more)."""
    g, dg, src = rmat14
    out = ctx.sssp(dg, src)
    banded = ctx.sssp_into(dg, src, out, stats=True)
    ctx.set_sssp_band(-1)
    ctx.set_sssp_delta(1 << 20)
    try:
        whole = ctx.sssp_into(dg, src, out, stats=True)
    finally:
        ctx.set_sssp_band(0)
        ctx.set_sssp_delta(0)
    assert banded["edges_expanded"] < whole["edges_expanded"]


@pytest.mark.skipif(not oracle.ref_available(), reason="reference CPU driver not built")
@pytest.mark.parametrize("band", [1, 0, -1])
def test_sssp_f32_band_matches_reference_ssspCPU(ctx, rmat14, band):
    import torch

    g, _, src = rmat14
    rows = np.repeat(np.arange(g.m), np.diff(g.row_ptr))
    lo, hi = np.minimum(rows, g.col_ind), np.maximum(rows, g.col_ind)
    w = (((lo * 7919 + hi * 104729) % 1000) / 9700.0 + 0.0001).astype(np.float32)
    dg = ap.DeviceGraph(ap.HostGraph(g.m, g.n, g.row_ptr, g.col_ind, w, True))
    out = torch.empty(g.m, dtype=torch.float32, device="cuda")
    ctx.set_sssp_band(band)
    try:
        ctx.sssp_f32_into(dg, src, out, unreached=-1.0)
    finally:
        ctx.set_sssp_band(0)
    ref, _ = oracle.ref_sssp_f32(g.row_ptr, g.col_ind, w, src)
    np.testing.assert_array_equal(out.cpu().numpy(), ref)


@pytest.mark.parametrize("blocks", [1, 3, 148])
def test_grid_size_does_not_change_results(ctx, rmat14, blocks):
    import torch

    g, dg, src = rmat14
    ctx.set_max_grid(blocks)
    try:
        np.testing.assert_array_equal(ctx.bfs(dg, src).cpu().numpy(), oracle.bfs(g.row_ptr, g.col_ind, src))
        np.testing.assert_array_equal(ctx.sssp(dg, src).cpu().numpy(), oracle.sssp(g.row_ptr, g.col_ind, g.val, src))
        pr = ap.mt19937_u32(4, g.m)
        got = ctx.mis(dg, torch.from_numpy(pr.view(np.int32)).cuda()).cpu().numpy()
        np.testing.assert_array_equal(got, oracle.mis_greedy(g.row_ptr, g.col_ind, pr))
    finally:
        ctx.set_max_grid(0)


# ------------------------------------------------------------ float SSSP / int32 MIS
def test_sssp_f32_integral_weights_match_golden(ctx, golden):
    import torch

    for key in ("chesapeake_u", "test_mesh_u", "test_cc_u"):
        rp, ci = golden[key + "_row_ptr"], golden[key + "_col_ind"]
        w = golden[key + "_w"].astype(np.float32)
        dg = ap.DeviceGraph(ap.HostGraph(rp.shape[0] - 1, rp.shape[0] - 1, rp, ci, w, True))
        out = torch.empty(rp.shape[0] - 1, dtype=torch.float32, device="cuda")
        for s in range(rp.shape[0] - 1):
            ctx.sssp_f32_into(dg, s, out, unreached=-1.0)
            np.testing.assert_array_equal(out.cpu().numpy(), golden[key + "_sssp"][s].astype(np.float32))


@pytest.mark.skipif(not oracle.ref_available(), reason="reference CPU driver not built")
def test_sssp_f32_fractional_weights_match_reference_ssspCPU(ctx, rmat14):
    """Non-integral float weights: the fixed point of float min-plus relaxation does not
    depend on the order relaxations land, so the GPU result equals the reference's own
    ssspCPU (label-correcting priority queue, src/testSssp.cpp:33-115) bit for bit."""
    import torch

    g, _, src = rmat14
    rows = np.repeat(np.arange(g.m), np.diff(g.row_ptr))
    lo, hi = np.minimum(rows, g.col_ind), np.maximum(rows, g.col_ind)
    w = (((lo * 7919 + hi * 104729) % 1000) / 97.0 + 0.01).astype(np.float32)  # symmetric
    dg = ap.DeviceGraph(ap.HostGraph(g.m, g.n, g.row_ptr, g.col_ind, w, True))
    out = torch.empty(g.m, dtype=torch.float32, device="cuda")
    ctx.sssp_f32_into(dg, src, out, unreached=-1.0)
    ref, _ = oracle.ref_sssp_f32(g.row_ptr, g.col_ind, w, src)
    np.testing.assert_array_equal(out.cpu().numpy(), ref)


def test_sssp_f32_unreached_value(ctx):
    import torch

    rp = np.array([0, 1, 2, 2], dtype=np.int32)
    ci = np.array([1, 0], dtype=np.int32)
    w = np.array([0.5, 0.5], dtype=np.float32)
    dg = ap.DeviceGraph(ap.HostGraph(3, 3, rp, ci, w, True))
    out = torch.empty(3, dtype=torch.float32, device="cuda")
    ctx.sssp_f32_into(dg, 0, out, unreached=1.70141e38)
    np.testing.assert_array_equal(out.cpu().numpy(), np.array([0.0, 0.5, 1.70141e38], dtype=np.float32))


def test_mis_int32_layout(ctx, rmat14):
    import torch

    g, dg, _ = rmat14
    pr = ap.mt19937_u32(4, g.m)
    out = torch.empty(g.m, dtype=torch.int32, device="cuda")
    ctx.mis_int32_into(dg, torch.from_numpy(pr.view(np.int32)).cuda(), out)
    np.testing.assert_array_equal(out.cpu().numpy(), oracle.mis_greedy(g.row_ptr, g.col_ind, pr).astype(np.int32))
