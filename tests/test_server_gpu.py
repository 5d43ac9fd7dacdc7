"""GPU tests of the query server: answers identical to the plain path alone and in a mix,
continuous batching actually folds requests, and the memory budget is enforced."""
import numpy as np
import pytest

import apspie_b200 as ap
from apspie_b200 import _lib as L

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def graphs():
    return [ap.gen_rmat(s, 16, 20 + s, 3) for s in (10, 12, 14)]


def _plain(ctx, g, kind, src):
    import torch

    dg = ap.DeviceGraph(g)
    if kind == L.QUERY_BFS:
        return ctx.bfs(dg, src).cpu().numpy()
    if kind == L.QUERY_SSSP:
        return ctx.sssp(dg, src).cpu().numpy()
    pr = torch.from_numpy(ap.mt19937_u32(4, g.m).view(np.int32)).cuda()
    return ctx.mis(dg, pr).cpu().numpy()


def _out(g, kind):
    import torch

    return torch.empty(g.m, dtype=torch.uint8 if kind == L.QUERY_MIS else torch.int32, device="cuda")


@pytest.mark.parametrize("sssp_fold,sssp_min,bfs_min", [(1, 0, 6), (64, 2, 1), (512, 0, 1000)])
def test_server_mix_matches_plain_path_alone_and_in_mix(ctx, graphs, sssp_fold, sssp_min, bfs_min):
    """sssp_fold 1: each SSSP request runs the single-source kernel; 64 with sssp_min 2:
    SSSP requests are folded into the batched kernel whenever two or more wait; 512 with
    0: the defaults (minimum by graph size). bfs_min 1: every BFS launch uses the batched
    kernel; 1000: none does."""
    srv = ap.Server(0, budget_bytes=8 << 30, slots=2, max_batch=512)
    gids = [srv.add_graph(g) for g in graphs]
    srv.set_sssp_fold(sssp_fold)
    srv.set_sssp_min_batch(sssp_min)
    srv.set_bfs_min_batch(bfs_min)
    srv.start()
    rng = np.random.default_rng(7)
    kinds = rng.choice([L.QUERY_BFS, L.QUERY_SSSP, L.QUERY_MIS], size=400, p=[0.7, 0.25, 0.05])
    which = rng.integers(0, len(graphs), 400)
    srcs = [int(rng.integers(0, graphs[w].m)) for w in which]
    # one request alone
    k0, w0, s0 = int(kinds[0]), int(which[0]), srcs[0]
    alone = _out(graphs[w0], k0)
    srv.wait(srv.submit(gids[w0], k0, s0, alone))
    # all of them in a burst (the first one again, now in the mix)
    outs, tickets = [], []
    for k, w, s in zip(kinds, which, srcs):
        o = _out(graphs[w], int(k))
        outs.append(o)
        tickets.append(srv.submit(gids[w], int(k), s, o))
    lat = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    assert st["completed"] == 401 and st["failed"] == 0
    assert st["launches"] < st["completed"]  # requests were folded into shared launches
    assert st["max_batch_seen"] > 1
    cache = {}
    for k, w, s, o in zip(kinds, which, srcs, outs):
        key = (int(k), int(w), s if k != L.QUERY_MIS else -1)
        if key not in cache:
            cache[key] = _plain(ctx, graphs[w], int(k), s)
        np.testing.assert_array_equal(o.cpu().numpy(), cache[key], err_msg=str(key))
    np.testing.assert_array_equal(alone.cpu().numpy(), outs[0].cpu().numpy())
    assert min(lat) > 0


def test_server_budget_enforced(graphs):
    g = graphs[2]
    need = (g.m + 1) * 4 + g.nnz * 8 + g.m * 4
    with pytest.raises(ap.ApspieError):
        srv = ap.Server(0, budget_bytes=need // 2, slots=1)
        try:
            srv.add_graph(g)
        finally:
            srv.close()


def test_server_tight_budget_shrinks_batches_but_answers_stay_exact(ctx, graphs):
    g = graphs[2]
    # A one-query server reserves the graph plus the arena of a BFS engine with one word
    # (32 query slots). 64 KB more than that lets the tight server's arena grow to a
    # one-word engine but not to the two-word one (12 bytes per vertex more) that 64 waiting
    # sources would ask for; the engine then serves them 32 at a time.
    probe = ap.Server(0, budget_bytes=4 << 30, slots=1, max_batch=1)
    probe.add_graph(g)
    probe.start()
    resident = probe.stats()["resident_bytes"]
    probe.close()
    budget = resident + (64 << 10)
    assert 12 * g.m > 2 * (64 << 10)
    srv = ap.Server(0, budget_bytes=budget, slots=1, max_batch=512)
    gid = srv.add_graph(g)
    srv.start()
    srcs = ap.lcc_sample(g, 64, 5)
    outs = [_out(g, L.QUERY_BFS) for _ in srcs]
    ts = [srv.submit(gid, L.QUERY_BFS, int(s), o) for s, o in zip(srcs, outs)]
    for t in ts:
        srv.wait(t)
    st = srv.stats()
    srv.close()
    assert st["peak_bytes"] <= budget
    assert st["max_batch_seen"] < 64
    for s, o in zip(srcs, outs):
        np.testing.assert_array_equal(o.cpu().numpy(), _plain(ctx, g, L.QUERY_BFS, int(s)))


def test_server_rejects_bad_requests(graphs):
    import torch

    srv = ap.Server(0, budget_bytes=2 << 30, slots=1)
    gid = srv.add_graph(ap.HostGraph(graphs[0].m, graphs[0].n, graphs[0].row_ptr, graphs[0].col_ind, None, True))
    srv.start()
    o = torch.empty(graphs[0].m, dtype=torch.int32, device="cuda")
    with pytest.raises(ap.ApspieError):
        srv.submit(gid, L.QUERY_BFS, graphs[0].m, o)  # source out of range
    with pytest.raises(ap.ApspieError):
        srv.submit(gid, L.QUERY_SSSP, 0, o)  # no weights on this graph
    with pytest.raises(ap.ApspieError):
        srv.submit(gid + 1, L.QUERY_BFS, 0, o)
    srv.close()


def test_server_bfs_arrivals_join_the_running_engine(ctx):
    """Bursts of BFS requests arrive while the graph's engine is on the GPU: they are posted
    into the running launch (joined_running > 0) and every answer equals the plain path's,
    including sources without edges (answered without a traversal)."""
    import time

    g = ap.gen_rmat(16, 16, 5, 3)
    srv = ap.Server(0, budget_bytes=8 << 30, slots=1, max_batch=256)
    gid = srv.add_graph(g)
    srv.start()
    import torch

    rng = np.random.default_rng(11)
    srcs = [int(x) for x in rng.integers(0, g.m, 600)]
    # every other output row starts 4 bytes past a 16-byte boundary (scalar fill path)
    spare = torch.empty(300 * (g.m + 4), dtype=torch.int32, device="cuda")
    outs, tickets = [], []
    for burst in range(12):
        for s in srcs[burst * 50:(burst + 1) * 50]:
            k = len(outs)
            o = _out(g, L.QUERY_BFS) if k % 2 == 0 else spare[(k // 2) * (g.m + 4) + 1:][:g.m]
            outs.append(o)
            tickets.append(srv.submit(gid, L.QUERY_BFS, s, o))
        time.sleep(0.0005)
    done = {}
    while len(done) < len(tickets):
        for t, status, lat in srv.take_completed():
            assert status == 0
            done[t] = lat
    st = srv.stats()
    srv.close()
    assert st["completed"] == 600 and st["failed"] == 0
    assert st["joined_running"] > 0
    assert st["trivial"] == sum(1 for s in srcs if g.row_ptr[s + 1] == g.row_ptr[s])
    dg = ap.DeviceGraph(g)
    for s, o in zip(srcs, outs):
        np.testing.assert_array_equal(o.cpu().numpy(), ctx.bfs(dg, s).cpu().numpy(), err_msg=str(s))


def test_server_take_completed_reports_each_request_once(ctx, graphs):
    g = graphs[1]
    srv = ap.Server(0, budget_bytes=2 << 30, slots=2, max_batch=64)
    gid = srv.add_graph(g)
    srv.start()
    outs = [_out(g, k) for k in (L.QUERY_BFS, L.QUERY_SSSP, L.QUERY_MIS) for _ in range(20)]
    kinds = [k for k in (L.QUERY_BFS, L.QUERY_SSSP, L.QUERY_MIS) for _ in range(20)]
    tickets = [srv.submit(gid, k, (7 * i) % g.m, o) for i, (k, o) in enumerate(zip(kinds, outs))]
    seen = []
    while len(seen) < len(tickets):
        seen += [t for t, status, _ in srv.take_completed(cap=7) if status == 0]
    assert sorted(seen) == sorted(tickets)
    with pytest.raises(ap.ApspieError):
        srv.wait(tickets[0], timeout_ms=10)  # already reported
    srv.close()


def test_server_submit_many_matches_single_submits(ctx, graphs):
    """A mixed batch submitted in one call: every answer equals the plain path's; a batch
    holding one invalid request is rejected whole (nothing of it runs)."""
    g = graphs[1]
    srv = ap.Server(0, budget_bytes=2 << 30, slots=2, max_batch=64)
    gid = srv.add_graph(g)
    srv.start()
    kinds = [L.QUERY_BFS] * 40 + [L.QUERY_SSSP] * 10 + [L.QUERY_MIS] * 3
    srcs = [(13 * i + 5) % g.m for i in range(len(kinds))]
    outs = [_out(g, k) for k in kinds]
    bad = list(srcs)
    bad[7] = g.m  # out of range
    with pytest.raises(ap.ApspieError):
        srv.submit_many([gid] * len(kinds), kinds, bad, outs)
    tickets = srv.submit_many([gid] * len(kinds), kinds, srcs, outs)
    assert len(set(tickets.tolist())) == len(kinds)
    done = set()
    while len(done) < len(kinds):
        for t, status, _ in srv.take_completed():
            assert status == 0
            done.add(t)
    st = srv.stats()
    srv.close()
    assert done == set(tickets.tolist())
    assert st["submitted"] == len(kinds) and st["completed"] == len(kinds)
    for k, s_, o in zip(kinds, srcs, outs):
        np.testing.assert_array_equal(o.cpu().numpy(), _plain(ctx, g, k, int(s_)), err_msg=f"{k} {s_}")


def test_server_sources_without_edges_any_row_alignment(ctx):
    """Sources without edges are answered by the side kernel (every entry -1 but the
    source's 0): rows of a length that is not a multiple of 4, rows that start off a
    16-byte boundary, and sources at every position of a 4-entry group."""
    import torch

    m = 1001
    rng = np.random.default_rng(5)
    edges = {(int(a), int(b)) for a, b in rng.integers(0, 500, (800, 2)) if a != b}  # 500..1000 isolated
    rows = [[] for _ in range(m)]
    for a, b in edges:
        rows[a].append(b)
        rows[b].append(a)
    rp = np.zeros(m + 1, dtype=np.int32)
    for v in range(m):
        rp[v + 1] = rp[v] + len(set(rows[v]))
    ci = np.concatenate([np.array(sorted(set(r)), dtype=np.int32) for r in rows if r] or [np.zeros(0, np.int32)])
    g = ap.HostGraph(m, m, rp, ci, None, True)
    srv = ap.Server(0, budget_bytes=1 << 30, slots=1)
    gid = srv.add_graph(g)
    srv.start()
    srcs = [996, 997, 998, 999, 1000] + [600, 601, 602, 603, 1000]
    big = torch.empty(5 * (m + 1) + 4, dtype=torch.int32, device="cuda")
    outs = [big[1 + k * (m + 1):1 + k * (m + 1) + m] for k in range(5)]  # views off a 16-byte boundary
    outs += [torch.empty(m, dtype=torch.int32, device="cuda") for _ in range(5)]  # aligned rows
    tickets = [srv.submit(gid, L.QUERY_BFS, s_, o) for s_, o in zip(srcs, outs)]
    for t in tickets:
        srv.wait(t)
    st = srv.stats()
    srv.close()
    assert st["trivial"] == len(srcs)
    for s_, o in zip(srcs, outs):
        want = np.full(m, -1, dtype=np.int32)
        want[s_] = 0
        np.testing.assert_array_equal(o.cpu().numpy(), want, err_msg=str(s_))

