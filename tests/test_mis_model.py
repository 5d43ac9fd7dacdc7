"""A CPU model of the MIS kernel's round protocol under random interleavings: it reaches
the oracle's set (the greedy MIS in descending (priority, id) order) on every schedule, and
models with a planted mistake do not.

Modelled at the level that matters for correctness (mis_kernel): each undecided vertex keeps
a scan position (the neighbour blocking it). Phase A re-checks the blocker; a vertex whose
blocker went out (or that has none yet) scans the rest of its row. In phase B the vertices
that joined last round write "out" into their neighbours while, interleaved at random with
those writes, the scans read their neighbours' states in tiles of 1-3 edges, each tile
flushing the least stop it saw into the vertex's `first` after its own reads. Phase C lets a
scanned vertex with no stop join and gives one with a stop its new blocker. No GPU is
involved."""
import numpy as np
import pytest

import oracle
from test_batch_sssp_model import _random_graph

UNDECIDED, IN, OUT, SCAN = 0, 1, 2, 3
INF = 1 << 60


def _outranks(pu, u, pv, v):
    return pu > pv or (pu == pv and u > v)


def _run_model(rp, ci, prio, rng, mistake=None):
    n = len(rp) - 1
    state = np.full(n, UNDECIDED)
    pos = np.array([int(rp[v]) - 1 for v in range(n)], dtype=np.int64)
    first = np.full(n, INF, dtype=np.int64)
    queue = [(v, False) for v in range(n)]  # (vertex, joined last round)
    for _ in range(n + 3):
        if not queue:
            return state
        # phase A
        segs = []
        for v, joined in queue:
            r0, r1 = int(rp[v]), int(rp[v + 1])
            if joined:
                segs.append((v, True, r0, r1))
                continue
            p = int(pos[v])
            scan = p < r0 or state[int(ci[p])] == OUT
            if mistake == "skip_undecided_blocker" and p >= r0 and state[int(ci[p])] == UNDECIDED:
                scan = True
            if scan:
                state[v] = SCAN
                segs.append((v, False, p + 1, r1))
        # phase B: push writes and scan tiles, interleaved at random
        events = []
        tiles = []
        for v, joined, e0, e1 in segs:
            e = e0
            while e < e1:
                k = int(rng.integers(1, 4))
                edges = list(range(e, min(e + k, e1)))
                e += k
                if joined:
                    for x in edges:
                        events.append(("push", v, x))
                else:
                    tiles.append([v, edges, INF])
                    t = len(tiles) - 1
                    events.append(("read", t, None))
                    events.append(("flush", t, None))
        pending = set()
        done_read = set()
        for k in rng.permutation(len(events)):
            kind, a, b = events[k]
            if kind == "push":
                u = int(ci[b])
                if u != a:
                    state[u] = OUT
            elif kind == "read":
                v, edges, _ = tiles[a]
                for x in edges:
                    u = int(ci[x])
                    if u != v and state[u] != OUT and _outranks(prio[u], u, prio[v], v):
                        tiles[a][2] = min(tiles[a][2], x)
                done_read.add(a)
                if a in pending:
                    pending.discard(a)
                    first[v] = min(first[v], tiles[a][2])
            elif a in done_read:
                first[tiles[a][0]] = min(first[tiles[a][0]], tiles[a][2])
            else:
                pending.add(a)
        # phase C
        nxt = []
        for v, joined in queue:
            if joined:
                continue
            if state[v] == UNDECIDED:
                nxt.append((v, False))
            elif state[v] == SCAN:
                if first[v] == INF or mistake == "join_despite_stop":
                    state[v] = IN
                    nxt.append((v, True))
                else:
                    pos[v] = first[v]
                    first[v] = INF
                    state[v] = UNDECIDED
                    nxt.append((v, False))
        queue = nxt
    raise AssertionError("no fixed point")


@pytest.mark.parametrize("seed", range(16))
def test_round_protocol_reaches_the_greedy_mis(seed):
    rng = np.random.default_rng(seed)
    rp, ci, _ = _random_graph(rng, int(rng.integers(6, 50)), int(rng.integers(1, 5)))
    n = len(rp) - 1
    prio = rng.integers(0, 6, n).astype(np.uint32)  # few values: many ties, broken by id
    state = _run_model(rp, ci, prio, rng)
    got = (state == IN).astype(np.uint8)
    np.testing.assert_array_equal(got, oracle.mis_greedy(rp, ci, prio))


@pytest.mark.parametrize("mistake", ["skip_undecided_blocker", "join_despite_stop"])
def test_planted_mistakes_break_the_set(mistake):
    """Planted mistakes: a vertex scans past a blocker that is still undecided, or joins
    although its scan found a stop; some schedule then puts two neighbours in the set."""
    bad = 0
    for seed in range(20):
        rng = np.random.default_rng(3000 + seed)
        rp, ci, _ = _random_graph(rng, 30, 3)
        prio = rng.integers(0, 1000, len(rp) - 1).astype(np.uint32)
        state = _run_model(rp, ci, prio, rng, mistake=mistake)
        got = (state == IN).astype(np.uint8)
        bad += int(not np.array_equal(got, oracle.mis_greedy(rp, ci, prio)))
    assert bad > 0
