"""CPU tests of the oracle itself: each restatement is pinned against golden vectors made
by the reference's own CPU code (tests/golden/make_golden.py) or, where the reference has
no CPU implementation, against an independent brute-force computation."""
import json
import os

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))


def _graph(golden, key):
    return golden[key + "_row_ptr"], golden[key + "_col_ind"]


def test_bfs_restatement_matches_reference_bfsCPU(golden, fixture_keys):
    for key in fixture_keys:
        rp, ci = _graph(golden, key)
        m = rp.shape[0] - 1
        for s in range(m):
            np.testing.assert_array_equal(oracle.bfs(rp, ci, s), golden[key + "_bfs"][s], err_msg=f"{key} src {s}")


def test_bfs_stop_cap_matches_reference_semantics(golden):
    rp, ci = _graph(golden, "chesapeake_u")
    full = oracle.bfs(rp, ci, 0)
    for stop in range(0, int(full.max()) + 2):
        capped = oracle.bfs(rp, ci, 0, stop)
        exp = np.where(full <= stop, full, -1)
        np.testing.assert_array_equal(capped, exp)


def test_sssp_restatement_matches_reference_ssspCPU(golden, fixture_keys):
    for key in fixture_keys:
        if key + "_sssp" not in golden:
            continue
        rp, ci = _graph(golden, key)
        w = golden[key + "_w"]
        for s in range(rp.shape[0] - 1):
            np.testing.assert_array_equal(oracle.sssp(rp, ci, w, s), golden[key + "_sssp"][s], err_msg=f"{key} src {s}")


def _dijkstra_py(rp, ci, w, s):
    import heapq

    m = rp.shape[0] - 1
    d = [-1] * m
    d[s] = 0
    pq = [(0, s)]
    while pq:
        dv, v = heapq.heappop(pq)
        if dv != d[v]:
            continue
        for e in range(rp[v], rp[v + 1]):
            u, nd = int(ci[e]), dv + int(w[e])
            if d[u] == -1 or nd < d[u]:
                d[u] = nd
                heapq.heappush(pq, (nd, u))
    return np.array(d, dtype=np.int32)


def test_sssp_restatement_matches_plain_dijkstra_on_rmat12(golden):
    import apspie_b200 as ap

    g = ap.gen_rmat(12, 16, 1, 3)
    src = int(golden["rmat12_meta"][2])
    got = oracle.sssp(g.row_ptr, g.col_ind, g.val, src)
    np.testing.assert_array_equal(got, golden["rmat12_sssp"])
    np.testing.assert_array_equal(got, _dijkstra_py(g.row_ptr, g.col_ind, g.val, src))


def test_mt19937_restatement_matches_reference(golden):
    np.testing.assert_array_equal(oracle.mt19937(4, 1000), golden["mt19937_seed4"])


def _mis_bruteforce_greedy(rp, ci, prio):
    m = rp.shape[0] - 1
    order = sorted(range(m), key=lambda v: (int(prio[v]), v), reverse=True)
    state = [0] * m
    for v in order:
        if state[v] == 0:
            state[v] = 1
            for e in range(rp[v], rp[v + 1]):
                if ci[e] != v and state[ci[e]] == 0:
                    state[ci[e]] = 2
    return np.array([1 if s == 1 else 0 for s in state], dtype=np.uint8)


def _luby_rounds_py(rp, ci, prio):
    """Round-synchronous restatement of spmspvMis (src/spmspvMis.cuh:232-318) with the
    threshold lowered to 0 (all undecided are candidates) and (prio, id) keys."""
    m = rp.shape[0] - 1
    st = [-1] * m
    while -1 in st:
        best = {}
        cand = [v for v in range(m) if st[v] == -1]
        for v in cand:
            for e in range(rp[v], rp[v + 1]):
                u = int(ci[e])
                if u != v:
                    k = (int(prio[v]), v)
                    best[u] = max(best.get(u, (-1, -1)), k)
        sel = [v for v in cand if (int(prio[v]), v) > best.get(v, (-1, -1))]
        for v in sel:
            st[v] = 1
        for v in sel:
            for e in range(rp[v], rp[v + 1]):
                u = int(ci[e])
                if st[u] == -1:
                    st[u] = 0
    return np.array(st, dtype=np.uint8)


def test_mis_restatement_is_luby_fixed_point_and_valid(golden, fixture_keys):
    for key in fixture_keys:
        if key + "_mis" not in golden:
            continue
        rp, ci = _graph(golden, key)
        prio = golden["mt19937_seed4"][: rp.shape[0] - 1]
        got = oracle.mis_greedy(rp, ci, prio)
        np.testing.assert_array_equal(got, golden[key + "_mis"])
        np.testing.assert_array_equal(got, _mis_bruteforce_greedy(rp, ci, prio))
        np.testing.assert_array_equal(got, _luby_rounds_py(rp, ci, prio))
        assert oracle.mis_check(rp, ci, got) == 0
        # the reference's vertex-order MIS passes the same validity check
        ref = golden[key + "_misref"].astype(np.uint8)
        assert oracle.mis_check(rp, ci, ref) == 0
        np.testing.assert_array_equal(oracle.mis_vertex_order(rp, ci, 0).astype(np.uint8), ref)


def test_mis_check_flags_planted_violations(golden):
    rp, ci = _graph(golden, "test_mesh_u")
    good = golden["test_mesh_u_mis"].copy()
    bad = good.copy()
    v = int(np.flatnonzero(good)[0])
    bad[ci[rp[v]]] = 1  # a neighbour of a set vertex joins: not independent
    assert oracle.mis_check(rp, ci, bad) > 0
    bad2 = good.copy()
    bad2[v] = 0  # drop a member: not maximal
    assert oracle.mis_check(rp, ci, bad2) > 0


def _spgemm_dense(m, n, arp, aci, aval, brp, bci, bval):
    A = np.zeros((m, n), dtype=np.float64)
    B = np.zeros((n, n), dtype=np.float64)
    for i in range(m):
        for e in range(arp[i], arp[i + 1]):
            A[i, aci[e]] += aval[e]
    for i in range(n):
        for e in range(brp[i], brp[i + 1]):
            B[i, bci[e]] += bval[e]
    P = (A != 0).astype(np.int64) @ (B != 0).astype(np.int64)
    return A @ B, P


def test_spgemm_restatement_matches_dense_product(golden):
    import apspie_b200 as ap

    for vt in (ap.VAL_F32, ap.VAL_I32):
        e = ap.gen_er(64, 4, 5, vt)
        crp, cci, cval = oracle.spgemm(e.m, e.n, e.row_ptr, e.col_ind, e.val, e.row_ptr, e.col_ind, e.val)
        C, P = _spgemm_dense(e.m, e.n, e.row_ptr, e.col_ind, e.val, e.row_ptr, e.col_ind, e.val)
        tag = "f32" if vt == ap.VAL_F32 else "i32"
        np.testing.assert_array_equal(crp, golden[f"spgemm_er64_{tag}_row_ptr"])
        np.testing.assert_array_equal(cci, golden[f"spgemm_er64_{tag}_col_ind"])
        np.testing.assert_array_equal(cval, golden[f"spgemm_er64_{tag}_val"])
        for i in range(e.m):
            cols = cci[crp[i]:crp[i + 1]]
            assert np.all(np.diff(cols) > 0)
            np.testing.assert_array_equal(cols, np.flatnonzero(P[i]))
            np.testing.assert_allclose(cval[crp[i]:crp[i + 1]], C[i, cols], rtol=1e-5, atol=1e-6)


def test_tc_restatement_matches_bruteforce(golden, fixture_keys):
    import itertools

    for key in fixture_keys:
        if key + "_tc" not in golden:
            continue
        rp, ci = _graph(golden, key)
        m = rp.shape[0] - 1
        adj = [set(int(c) for c in ci[rp[i]:rp[i + 1]] if c != i) for i in range(m)]
        brute = sum(1 for a, b, c in itertools.combinations(range(m), 3) if b in adj[a] and c in adj[a] and c in adj[b])
        assert int(golden[key + "_tc"][0]) == brute, key


def test_tc_restatement_matches_reference_formulation():
    """sum((U*L) .* U) over CSC arrays (the reference's TC, test/tc/main.cu:243-249 with
    ewiseMultTc tc.cuh:168-199) equals the oracle's sum over L of |L(i,:) n L(k,:)|."""
    import apspie_b200 as ap

    g = ap.gen_rmat(9, 8, 11, 3, weights=False)
    m = g.m
    A = np.zeros((m, m), dtype=np.int64)
    for i in range(m):
        A[i, g.col_ind[g.row_ptr[i]:g.row_ptr[i + 1]]] = 1
    Lw = np.tril(A, -1)
    Uw = np.triu(A, 1)
    ref_count = int(((Uw @ Lw) * Uw).sum())
    L = ap.strict_lower(g)
    assert oracle.tc(L.row_ptr, L.col_ind) == ref_count
    assert ref_count == int(np.trace(np.linalg.matrix_power(A, 3)) // 6)


def test_golden_manifest_consistent(golden):
    with open(os.path.join(HERE, "golden", "golden.json")) as f:
        man = json.load(f)
    for fx in man["fixtures"]:
        assert golden[fx["key"] + "_row_ptr"].shape[0] == fx["m"] + 1
        assert golden[fx["key"] + "_col_ind"].shape[0] == fx["nnz"]


@pytest.mark.skipif(not oracle.ref_available(), reason="reference CPU driver not built")
def test_reference_driver_agrees_on_rmat14():
    import apspie_b200 as ap

    g = ap.gen_rmat(14, 16, 1, 3)
    src = ap.max_degree_vertex(g)
    np.testing.assert_array_equal(oracle.ref_bfs(g.row_ptr, g.col_ind, src)[0], oracle.bfs(g.row_ptr, g.col_ind, src))
    np.testing.assert_array_equal(oracle.ref_sssp(g.row_ptr, g.col_ind, g.val, src)[0],
                                  oracle.sssp(g.row_ptr, g.col_ind, g.val, src))


def test_oracle_pagerank_and_spmv_sanity():
    # a directed 4-cycle: every vertex has rank 1/4; a star's centre collects the most rank
    rp = np.array([0, 1, 2, 3, 4]); ci = np.array([1, 2, 3, 0])
    r, it = oracle.pagerank(rp, ci, 0.85, 1e-12, 100)
    np.testing.assert_allclose(r, 0.25)
    rp = np.array([0, 1, 2, 3, 3]); ci = np.array([3, 3, 3])  # three leaves -> sink 3 (dangling)
    r, _ = oracle.pagerank(rp, ci, 0.85, 1e-12, 500)
    assert abs(r.sum() - 1.0) < 1e-12 and r[3] > r[0]
    np.testing.assert_allclose(oracle.spmv(np.array([0, 2, 3]), np.array([0, 1, 1]), np.array([1.0, 2.0, 3.0]),
                                           np.array([1.0, 10.0])), [21.0, 30.0])


def test_oracle_spmspv_against_dense_product():
    """The oracle's sparse-vector product equals x^T A computed densely (int32, exact)."""
    rng = np.random.default_rng(5)
    n = 40
    dense = (rng.random((n, n)) < 0.15) * rng.integers(1, 9, (n, n))
    rp = np.concatenate([[0], np.cumsum((dense != 0).sum(1))]).astype(np.int32)
    ci = np.nonzero(dense)[1].astype(np.int32)
    val = dense[dense != 0].astype(np.int32)
    x_ind = rng.integers(0, n, 12).astype(np.int32)
    x_val = rng.integers(-3, 4, 12).astype(np.int32)
    xd = np.zeros(n, dtype=np.int64)
    np.add.at(xd, x_ind, x_val)
    y = xd @ dense
    hit = (np.abs(dense[np.unique(x_ind)]).sum(0) > 0)
    yi, yv = oracle.spmspv(rp, ci, val, n, x_ind, x_val)
    np.testing.assert_array_equal(yi, np.nonzero(hit)[0])
    np.testing.assert_array_equal(yv, y[hit])
