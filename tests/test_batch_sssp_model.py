"""A CPU model of the batched SSSP kernel's relaxation protocol, run under random
interleavings: the protocol reaches the oracle's distances on every schedule, and a model
with a planted mistake (labels read from a stale copy) does not.

The model follows sssp_batch_kernel step for step at the level that matters for
correctness: phase A takes each queued entry's changed-query mask and clears it; phase B
relaxes every (edge, changed query) pair as two events that other pairs may interleave
with: a read of both labels (coherent: the current values), then a write that lowers the
target label (atomicMin) and, when the candidate beat the label READ earlier (not the
label at write time: the kernel does not wait for the atomic's old value), sets the
query's bit in the target's next changed mask. No GPU is involved."""
import numpy as np
import pytest

import oracle

INF = 1 << 40


def _random_graph(rng, n, deg):
    """Undirected weighted graph as sorted CSR (int32 weights 1..20)."""
    pairs = {}
    for u in range(n):
        for v in rng.integers(0, n, deg):
            if u != v:
                a, b = min(u, int(v)), max(u, int(v))
                pairs.setdefault((a, b), int(rng.integers(1, 21)))
    rows = [[] for _ in range(n)]
    for (a, b), w in pairs.items():
        rows[a].append((b, w))
        rows[b].append((a, w))
    rp = np.zeros(n + 1, dtype=np.int32)
    ci, wt = [], []
    for u in range(n):
        for v, w in sorted(rows[u]):
            ci.append(v)
            wt.append(w)
        rp[u + 1] = len(ci)
    return rp, np.array(ci, dtype=np.int32), np.array(wt, dtype=np.int32)


def _run_model(rp, ci, wt, sources, rng, stale_reads=False):
    """stale_reads: source labels come from the copy taken at the start of the PREVIOUS
    iteration (what a non-coherent cache line kept across a grid barrier would hold)."""
    n, nq = len(rp) - 1, len(sources)
    lab = np.full((n, nq), INF, dtype=np.int64)  # vertex-major, as in the kernel
    chg = [set() for _ in range(n)]
    queue = []
    for q, s in enumerate(sources):
        lab[s, q] = 0
        if not chg[s]:
            queue.append(s)
        chg[s].add(q)
    older = lab.copy()
    for _ in range(4 * n + 8):
        if not queue:
            return lab
        # phase A: take and clear each entry's changed mask
        taken = {}
        for u in queue:
            taken[u] = chg[u]
            chg[u] = set()
        stale, older = older, lab.copy()  # labels as of the previous iteration's start
        nxt = [set() for _ in range(n)]
        # phase B: every (edge, changed query) as a read event then a write event
        tasks = [(u, int(ci[e]), int(wt[e]), q) for u, qs in taken.items()
                 for e in range(rp[u], rp[u + 1]) for q in qs]
        reads = {}
        pending = list(range(len(tasks)))
        events = [(t, "r") for t in pending] + [(t, "w") for t in pending]
        order = rng.permutation(len(events))
        done_read = set()
        deferred = []
        for k in order:
            t, kind = events[k]
            if kind == "w" and t not in done_read:
                deferred.append(t)  # a write waits for its own read
                continue
            if kind == "r":
                u, v, w, q = tasks[t]
                src = stale if stale_reads else lab
                reads[t] = (src[u, q], lab[v, q])
                done_read.add(t)
                # writes that were waiting for this read may now run, in random order
                if t in deferred:
                    deferred.remove(t)
                    _write(tasks[t], reads[t], lab, nxt)
            else:
                _write(tasks[t], reads[t], lab, nxt)
        for t in deferred:
            _write(tasks[t], reads[t], lab, nxt)
        queue = [v for v in range(n) if nxt[v]]
        for v in queue:
            chg[v] = nxt[v]
    raise AssertionError("no fixed point")


def _write(task, read, lab, nxt):
    u, v, w, q = task
    du, dv = read
    if du >= INF:
        return
    nd = du + w
    if nd < dv:  # improvement over the label read earlier
        lab[v, q] = min(lab[v, q], nd)  # atomicMin, old value not awaited
        nxt[v].add(q)


@pytest.mark.parametrize("seed", range(12))
def test_protocol_reaches_oracle_distances_on_random_schedules(seed):
    rng = np.random.default_rng(seed)
    rp, ci, wt = _random_graph(rng, int(rng.integers(8, 40)), int(rng.integers(1, 4)))
    n = len(rp) - 1
    sources = [int(x) for x in rng.integers(0, n, int(rng.integers(1, 6)))]
    lab = _run_model(rp, ci, wt, sources, rng)
    for q, s in enumerate(sources):
        ref = oracle.sssp(rp, ci, wt, s).astype(np.int64)
        got = np.where(lab[:, q] >= INF, -1, lab[:, q])
        np.testing.assert_array_equal(got, ref, err_msg=f"seed {seed} query {q}")


def test_stale_label_reads_lose_updates_on_some_schedule():
    """Planted mistake: phase B reads the source label from a copy taken at the start of
    the previous iteration. A label lowered during that iteration is expanded now with its
    old value while its change bit is consumed, so the lower value is never propagated."""
    failures = 0
    for seed in range(40):
        rng = np.random.default_rng(1000 + seed)
        rp, ci, wt = _random_graph(rng, 30, 3)
        sources = [0, 7]
        lab = _run_model(rp, ci, wt, sources, rng, stale_reads=True)
        for q, s in enumerate(sources):
            ref = oracle.sssp(rp, ci, wt, s).astype(np.int64)
            got = np.where(lab[:, q] >= INF, -1, lab[:, q])
            failures += int(not np.array_equal(got, ref))
    assert failures > 0
