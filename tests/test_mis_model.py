"""A CPU model of the MIS kernel's round protocol under random interleavings: it reaches
the oracle's set (the greedy MIS in descending (priority, id) order) on every schedule, and
a model with a planted mistake does not.

Modelled at the level that matters for correctness (mis_kernel): each round's edge pass
reads the state of every undecided vertex's neighbours while other warps of the same pass
already mark vertices "out" (a vertex with a neighbour in the set); a row may be split
over several tiles, each flushing its own flags (out, or blocked in this round). The
vertex pass then lets every undecided vertex that is neither out nor blocked join. No GPU
is involved."""
import numpy as np
import pytest

import oracle
from test_batch_sssp_model import _random_graph

UNDECIDED, IN, OUT = 0, 1, 2


def _outranks(pu, u, pv, v):
    return pu > pv or (pu == pv and u > v)


def _run_model(rp, ci, prio, rng, join_when_blocked=False):
    n = len(rp) - 1
    state = np.full(n, UNDECIDED)
    blocked = np.zeros(n, dtype=np.int64)
    queue = list(range(n))
    for rnd in range(1, n + 3):
        if not queue:
            return state
        # edge pass: each row cut into tiles of 1-3 edges; a tile's reads happen at random
        # times, its flag flush happens after its own reads
        tiles = []
        for v in queue:
            e, e1 = int(rp[v]), int(rp[v + 1])
            while e < e1:
                k = int(rng.integers(1, 4))
                tiles.append((v, list(range(e, min(e + k, e1)))))
                e += k
        events = [(t, "read") for t in range(len(tiles))] + [(t, "flush") for t in range(len(tiles))]
        flags = [0] * len(tiles)
        read = [False] * len(tiles)
        waiting = set()
        for k in rng.permutation(len(events)):
            t, kind = events[k]
            if kind == "read":
                v, edges = tiles[t]
                for e in edges:
                    u = int(ci[e])
                    if u == v:
                        continue
                    if state[u] == IN:
                        flags[t] |= 1
                    elif state[u] == UNDECIDED and _outranks(prio[u], u, prio[v], v):
                        flags[t] |= 2
                read[t] = True
                if t in waiting:
                    waiting.discard(t)
                    _flush(tiles[t][0], flags[t], state, blocked, rnd)
            elif read[t]:
                _flush(tiles[t][0], flags[t], state, blocked, rnd)
            else:
                waiting.add(t)
        # vertex pass
        nxt = []
        for v in queue:
            if state[v] == UNDECIDED:
                if blocked[v] != rnd or join_when_blocked:
                    state[v] = IN
                else:
                    nxt.append(v)
        queue = nxt
    raise AssertionError("no fixed point")


def _flush(v, f, state, blocked, rnd):
    if f & 1:
        state[v] = OUT
    elif f & 2:
        blocked[v] = rnd


@pytest.mark.parametrize("seed", range(16))
def test_round_protocol_reaches_the_greedy_mis(seed):
    rng = np.random.default_rng(seed)
    rp, ci, _ = _random_graph(rng, int(rng.integers(6, 50)), int(rng.integers(1, 5)))
    n = len(rp) - 1
    prio = rng.integers(0, 6, n).astype(np.uint32)  # few values: many ties, broken by id
    state = _run_model(rp, ci, prio, rng)
    got = (state == IN).astype(np.uint8)
    np.testing.assert_array_equal(got, oracle.mis_greedy(rp, ci, prio))


def test_joining_while_blocked_breaks_independence():
    """Planted mistake: a blocked vertex joins anyway; some schedule then puts two
    neighbours in the set."""
    bad = 0
    for seed in range(20):
        rng = np.random.default_rng(3000 + seed)
        rp, ci, _ = _random_graph(rng, 30, 3)
        prio = rng.integers(0, 1000, len(rp) - 1).astype(np.uint32)
        state = _run_model(rp, ci, prio, rng, join_when_blocked=True)
        got = (state == IN).astype(np.uint8)
        bad += int(not np.array_equal(got, oracle.mis_greedy(rp, ci, prio)))
    assert bad > 0
