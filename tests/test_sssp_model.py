"""A CPU model of the single-source SSSP kernel's queue protocol, run under random
interleavings and random distance bands: it reaches the oracle's distances on every
schedule, and a model with a planted ordering mistake does not.

Modelled at the level that matters for correctness (sssp_kernel, phases A and B):
  * a vertex is queued at most once: its "queued" bit is set by whoever appends it;
  * phase A reads each queued vertex's distance (coherent read). A vertex above this
    iteration's band stays queued (re-appended, bit kept); the least queued distance
    always expands. Every other vertex clears its bit and expands only if its distance
    changed since it last expanded (`last`), relaxing with the distance read here;
  * phase B relaxes each expanded row's edges as a read event (the target's distance) and
    a later write event: atomicMin when the candidate beats the distance READ earlier
    (the kernel does not wait for the atomic's old value), then the target is appended
    unless its queued bit was already set.
No GPU is involved."""
import numpy as np
import pytest

import oracle
from test_batch_sssp_model import _random_graph

INF = 1 << 40


def _run_model(rp, ci, wt, src, rng, clear_bits_late=False):
    """clear_bits_late: the planted mistake, clearing queued bits after phase B instead of
    in phase A (an improvement made during phase B then finds the bit still set, is not
    appended, and its bit is cleared afterwards)."""
    n = len(rp) - 1
    dist = np.full(n, INF, dtype=np.int64)
    dist[src] = 0
    last = np.full(n, -1, dtype=np.int64)
    queued = np.zeros(n, dtype=bool)
    queued[src] = True
    queue = [src]
    for _ in range(8 * n + 16):
        if not queue:
            return dist
        # phase A
        dmin = min(dist[v] for v in queue)
        finite = sorted({int(dist[v]) for v in queue})
        cut = finite[int(rng.integers(0, len(finite)))]  # a random band edge at or above the min
        nxt, expand = [], []
        for v in queue:
            d = dist[v]
            if d > cut and d != dmin:
                nxt.append(v)  # deferred: stays queued, bit kept
                continue
            if not clear_bits_late:
                queued[v] = False
            if last[v] != d:
                last[v] = d
                expand.append((v, d))
        # phase B: (edge) read events and write events, randomly interleaved
        tasks = [(u, du, int(ci[e]), int(wt[e])) for u, du in expand for e in range(rp[u], rp[u + 1])]
        events = [(t, "r") for t in range(len(tasks))] + [(t, "w") for t in range(len(tasks))]
        reads, deferred = {}, set()
        for k in rng.permutation(len(events)):
            t, kind = events[k]
            if kind == "r":
                reads[t] = dist[tasks[t][2]]
                if t in deferred:
                    deferred.discard(t)
                    _write(tasks[t], reads[t], dist, queued, nxt)
            elif t in reads:
                _write(tasks[t], reads[t], dist, queued, nxt)
            else:
                deferred.add(t)
        if clear_bits_late:
            for v, _ in expand:
                queued[v] = False
        queue = nxt
    raise AssertionError("no fixed point")


def _write(task, cd, dist, queued, nxt):
    _, du, v, w = task
    nd = du + w
    if nd < cd:
        dist[v] = min(dist[v], nd)  # atomicMin, old value not awaited
        if not queued[v]:  # atomicOr on the queued bit returned 0
            queued[v] = True
            nxt.append(v)


@pytest.mark.parametrize("seed", range(16))
def test_queue_protocol_reaches_oracle_distances(seed):
    rng = np.random.default_rng(seed)
    rp, ci, wt = _random_graph(rng, int(rng.integers(8, 48)), int(rng.integers(1, 4)))
    src = int(rng.integers(0, len(rp) - 1))
    dist = _run_model(rp, ci, wt, src, rng)
    got = np.where(dist >= INF, -1, dist)
    np.testing.assert_array_equal(got, oracle.sssp(rp, ci, wt, src).astype(np.int64))


def test_late_bit_clearing_loses_updates_on_some_schedule():
    failures = 0
    for seed in range(40):
        rng = np.random.default_rng(2000 + seed)
        rp, ci, wt = _random_graph(rng, 30, 3)
        dist = _run_model(rp, ci, wt, 0, rng, clear_bits_late=True)
        got = np.where(dist >= INF, -1, dist)
        failures += int(not np.array_equal(got, oracle.sssp(rp, ci, wt, 0).astype(np.int64)))
    assert failures > 0
