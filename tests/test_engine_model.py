"""A CPU model of the server's BFS engine protocol (msbfs_kernel with SERVE = true): query
slots, per-level retirement of queries whose frontier died, admission of waiting requests
into swept slots (while at most 1/admit_frac of the slots are in flight -- the kernel uses
1/64: queries run in generations), depths relative to each query's start level. Requests arrive at random
levels; every completed row must equal the oracle's BFS from its source, each request
must complete exactly once, and models with a planted mistake must fail. No GPU."""
import numpy as np
import pytest

import oracle
from test_batch_sssp_model import _random_graph

Q = 32  # one word of query slots


def _run_engine(rp, ci, arrivals, sweep=True, check_alive=True, max_levels=10_000, gate=True, admit_frac=32):
    """arrivals: list of (level, source). Returns {request index: (completion level, row)}."""
    n = len(rp) - 1
    full = (1 << Q) - 1
    vis = [0] * n
    fr = [0] * n
    act = dirty = sweeping = 0
    alive_prev = 0
    rows = {}
    slot_req = {}
    slot_row = {}  # the row a slot writes into (kept after retirement, as on the device)
    start = {}
    done = {}
    waiting = []
    nxt_arrival = 0
    order = sorted(range(len(arrivals)), key=lambda i: arrivals[i][0])
    for L in range(max_levels):
        while nxt_arrival < len(order) and arrivals[order[nxt_arrival]][0] <= L:
            waiting.append(order[nxt_arrival])
            nxt_arrival += 1
        # admin: retire, admit, decide on a sweep
        if L > 0:
            ret = act & ~alive_prev if check_alive else act
            act &= ~ret
            dirty = (dirty & ~sweeping) | ret
            sweeping = 0
            b = ret
            while b:
                s = (b & -b).bit_length() - 1
                b &= b - 1
                r = slot_req.pop(s)
                done[r] = (L, list(rows[r]))  # what the host reads at completion
        free = ~(act | dirty) & full if sweep else ~act & full
        if gate and bin(act).count("1") * admit_frac > Q:
            free = 0  # a generation is still running: arrivals wait for it to drain
        while waiting and free:
            s = (free & -free).bit_length() - 1
            free &= free - 1
            r = waiting.pop(0)
            src = arrivals[r][1]
            slot_req[s] = r
            start[s] = L
            rows[r] = [-1] * n
            rows[r][src] = 0
            slot_row[s] = rows[r]
            vis[src] |= 1 << s
            fr[src] |= 1 << s
            act |= 1 << s
        ndirty = bin(dirty).count("1")
        nfree = bin(~(act | dirty) & full).count("1")
        pending = bool(waiting) or nxt_arrival < len(order)
        do_sweep = sweep and ndirty > 0 and (4 * ndirty >= Q or (pending and nfree == 0))
        sweeping = dirty if do_sweep else 0
        if act == 0 and not pending and not do_sweep:
            return done
        # first phase: the sweep
        if sweeping:
            for v in range(n):
                vis[v] &= ~sweeping
        # expansion + finalize
        nxt = [0] * n
        for u in range(n):
            if fr[u]:
                for e in range(rp[u], rp[u + 1]):
                    v = int(ci[e])
                    nxt[v] |= fr[u] & ~vis[v]
        alive = 0
        for v in range(n):
            nb = nxt[v] & ~vis[v]
            if nb:
                vis[v] |= nb
                alive |= nb
                b = nb
                while b:
                    s = (b & -b).bit_length() - 1
                    b &= b - 1
                    slot_row[s][v] = L + 1 - start[s]
            nxt[v] = nb
        fr = nxt
        alive_prev = alive
    raise AssertionError("engine did not finish")


def _stream(rng, n, count, spread):
    return [(int(rng.integers(0, spread)), int(rng.integers(0, n))) for _ in range(count)]


@pytest.mark.parametrize("gate,admit_frac", [(True, 32), (True, 8), (False, 32)])
@pytest.mark.parametrize("seed", range(6))
def test_engine_rows_equal_single_source_bfs(seed, gate, admit_frac):
    rng = np.random.default_rng(100 + seed)
    rp, ci, _ = _random_graph(rng, int(rng.integers(20, 60)), int(rng.integers(1, 4)))
    n = len(rp) - 1
    arrivals = _stream(rng, n, 90, 25)  # more requests than slots, arriving over 25 levels
    done = _run_engine(rp, ci, arrivals, gate=gate, admit_frac=admit_frac)
    assert sorted(done) == list(range(len(arrivals)))
    for r, (lvl, row) in done.items():
        ref = oracle.bfs(rp, ci, arrivals[r][1])
        np.testing.assert_array_equal(np.array(row), ref, err_msg=str(r))
        # it completes at the level after its last frontier: start + eccentricity + 1 at the earliest
        assert lvl >= arrivals[r][0] + int(ref.max()) + 1


@pytest.mark.parametrize("mistake", ["no_sweep", "retire_without_alive_check"])
def test_engine_planted_mistakes_are_caught(mistake):
    bad = 0
    for seed in range(6):
        rng = np.random.default_rng(200 + seed)
        rp, ci, _ = _random_graph(rng, 40, 3)
        n = len(rp) - 1
        arrivals = _stream(rng, n, 120, 30)
        done = _run_engine(rp, ci, arrivals, sweep=mistake != "no_sweep",
                           check_alive=mistake != "retire_without_alive_check")
        for r, (_, row) in done.items():
            if not np.array_equal(np.array(row), oracle.bfs(rp, ci, arrivals[r][1])):
                bad += 1
                break
    assert bad > 0
