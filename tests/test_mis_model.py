"""A CPU model of the MIS kernel's round protocol under random interleavings: it reaches
the oracle's set (the greedy MIS in descending (priority, id) order) on every schedule, and
models with a planted mistake do not.

Modelled at the level that matters for correctness (mis_kernel): vertices without
neighbours join at once; each undecided vertex keeps a scan position (the neighbour
blocking it). A round first lets the vertices that joined last round write "out" into their
neighbours (phase P, complete before the scans start); then every undecided vertex, in
steps interleaved at random with every other vertex's steps: leaves if it is out, waits if
its blocker is still undecided (or in), else scans the rest of its row in chunks of 1-3
neighbours, stopping at the first that outranks it and is not out, and then decides at
once -- joining (state in, read by the others' later steps) when it found no stop. Scans may
read stale states (as through L1); blocker checks read current ones. No GPU is involved."""
import numpy as np
import pytest

import oracle
from test_batch_sssp_model import _random_graph

UNDECIDED, IN, OUT = 0, 1, 2


def _outranks(pu, u, pv, v):
    return pu > pv or (pu == pv and u > v)


def _run_model(rp, ci, prio, rng, mistake=None):
    n = len(rp) - 1
    state = np.full(n, UNDECIDED)
    pos = np.array([int(rp[v]) - 1 for v in range(n)], dtype=np.int64)
    queue = []
    for v in range(n):
        if rp[v + 1] > rp[v]:
            queue.append((v, False))
        else:
            state[v] = IN
    snaps = [state.copy()]  # states at the start of earlier rounds (what an L1 may still hold)
    for _ in range(4 * n + 8):
        if not queue:
            return state
        snaps = (snaps + [state.copy()])[-3:]
        # phase P
        for v, joined in queue:
            if joined:
                for e in range(int(rp[v]), int(rp[v + 1])):
                    if int(ci[e]) != v:
                        state[int(ci[e])] = OUT
        # phase S: each undecided vertex is a generator of steps; run them interleaved
        def steps(v):
            if state[v] != UNDECIDED:
                yield None
                return
            r0, r1 = int(rp[v]), int(rp[v + 1])
            p = int(pos[v])
            if p >= r0 and state[int(ci[p])] != OUT and mistake != "skip_undecided_blocker":
                nxt.append((v, False))  # still blocked
                yield None
                return
            e = p + 1
            stop = -1
            while e < r1 and stop < 0:
                k = int(rng.integers(1, 4))
                for x in range(e, min(e + k, r1)):
                    u = int(ci[x])
                    # scans may read a stale state (through L1): the current one or one from
                    # the start of this or an earlier round
                    su = state[u] if rng.random() < 0.5 else snaps[int(rng.integers(0, len(snaps)))][u]
                    if u != v and su != OUT and _outranks(prio[u], u, prio[v], v):
                        stop = x
                        break
                e += k
                yield None
            if stop >= 0 and mistake != "join_despite_stop":
                pos[v] = stop
                nxt.append((v, False))
            else:
                state[v] = IN
                nxt.append((v, True))
            yield None

        nxt = []
        gens = [steps(v) for v, joined in queue if not joined]
        while gens:
            k = int(rng.integers(0, len(gens)))
            try:
                next(gens[k])
            except StopIteration:
                gens.pop(k)
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
