"""Benchmark: single-source SSSP (min-plus SpMSpV) on R-MAT scale 20 -- the
configuration the headline metric (BFS/SSSP GTEPS & % of HBM roofline) is quoted on --
plus BFS on R-MAT scale 14 and MIS on R-MAT scale 20 as extra lines of the same JSON.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one complete SSSP query from the max-degree vertex on the HBM-resident graph.
`value` is device time (CUDA events on the library's stream, max over ranks); `e2e`
goes through the C ABI with host buffers: every step uploads the CSR and weights from
pinned host memory, runs the query and reads the distances back. Multi-GPU runs are
independent replicas (a single-source query does not shard), so scaling is weak.
`--impl reference` times the reference's own CPU SSSP (ssspCPU, compiled from the
reference sources into oracle/_ref) on the same graph and source, one query per worker
process per step on every host core it may use.
"""
from __future__ import annotations

import argparse
import collections
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "BFS/SSSP GTEPS & % HBM roofline; batched/served queries/s + p50/p99 vs plain"
WORKLOAD = ("SSSP (min-plus SpMSpV) from the max-degree vertex on undirected R-MAT scale 20 "
            "(1,048,576 vertices, edge factor 16, a/b/c/d .57/.19/.19/.05, seed 2, symmetrised, "
            "deduplicated, int32 CSR), int32 weights uniform [1,255] from seed 3; int32 distances")
FALLBACK_HBM_GBS = 6650.0


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.5)  # let the sampler come up before the timed region
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def build_graph(scale, seed):
    import apspie_b200 as ap

    g = ap.gen_rmat(scale, 16, seed, 3)
    return g, ap.max_degree_vertex(g)


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(ws, x: float) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist

    # nccl reduces device tensors; gloo (the CPU test backend) host tensors
    dev = "cpu" if dist.get_backend() == "gloo" else "cuda"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def time_steps(stream, fn, steps):
    """Runs fn() `steps` times between events on `stream`; returns (total_ms, per_step_ms list)."""
    import torch

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record(stream)
    for i in range(steps):
        starts[i].record(stream)
        fn()
        ends[i].record(stream)
    t1.record(stream)
    torch.cuda.synchronize()
    return t0.elapsed_time(t1), [s.elapsed_time(e) for s, e in zip(starts, ends)]


def traffic_from_profile(kernel: str):
    """DRAM bytes per launch recorded by an ncu capture summarised under profiles/."""
    p = os.path.join(ROOT, "profiles", f"{kernel}.md")
    try:
        with open(p) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------------
def ref_worker_count():
    n = os.cpu_count() or 1
    try:
        n = len(os.sched_getaffinity(0))
    except Exception:
        pass
    return max(1, min(n, 32))


def run_reference_sssp(g, src, workers, tmpdir):
    """One step: `workers` concurrent reference ssspCPU processes on the same query.
    Returns (max CPU ms over workers, distances of worker 0)."""
    import oracle

    gpath = os.path.join(tmpdir, "g.csr")
    if not os.path.exists(gpath):
        oracle._write_csr(gpath, g.row_ptr, g.col_ind, g.val)

    def one(i):
        out = os.path.join(tmpdir, f"d{i}.bin")
        res = subprocess.run([oracle.REF_BIN, "sssp", gpath, str(src), out], capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(res.stderr[-300:])
        for line in res.stdout.splitlines():
            if line.startswith("APSPIE_REF "):
                return json.loads(line[11:])["ms"]
        raise RuntimeError("no timing line")

    with ThreadPoolExecutor(max_workers=workers) as ex:
        ms = list(ex.map(one, range(workers)))
    return max(ms), np.fromfile(os.path.join(tmpdir, "d0.bin"), dtype=np.int32)


def main_reference(args, ws, rank):
    import oracle

    if rank != 0:
        return 0
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/apspie_ref (the reference CPU "
                          "code compiled from its sources) was not built"}))
        return 0
    # the input comes from the oracle's serial restatement of the generator (the same CSR
    # as the product's generator, pinned by tests/test_host.py), so this arm loads nothing
    # of the product library
    g = oracle.gen_rmat(20, 16, 2, 3)
    src = g.max_degree_vertex()
    comp_edges = int(g.degrees()[oracle.sssp(g.row_ptr, g.col_ind, g.val, src) >= 0].sum())
    workers = ref_worker_count()
    with tempfile.TemporaryDirectory() as d:
        for _ in range(args.warmup):
            run_reference_sssp(g, src, workers, d)
        times = []
        for _ in range(args.steps):
            ms, _ = run_reference_sssp(g, src, workers, d)
            times.append(ms)
    ms_step = float(np.mean(times))
    value = workers * comp_edges / (ms_step * 1e-3) / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "parallelism": f"{workers} concurrent CPU queries"},
        "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": workers, "kind": "reference",
                         "sample": f"per step, {workers} concurrent runs of the reference ssspCPU "
                                   "(src/testSssp.cpp:117, compiled from the reference sources) on the "
                                   "full scale-20 query; CPU time inside each process"},
        "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------
def main_ours(args, ws, rank, local):
    import torch

    import apspie_b200 as ap

    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    if args.only_extra:
        # one extra leg alone (for profiling a kernel without the rest of the run)
        ctx = ap.Context(local)
        if args.only_extra == "traversal":
            res = extras_traversal(ctx, args, ws, local)
        elif args.only_extra == "spgemm_tc":
            res = extras_spgemm_tc(ctx, args, ws, local)
        elif args.only_extra == "build":
            res = extras_build(ctx, args, ws, local)
        else:
            g22 = ap.gen_rmat(22, 16, 1, 3)
            res = extras_batched(ctx, args, ws, local, g22) if args.only_extra == "batched" \
                else extras_serving(ctx, args, local, g22)
        ctx.close()
        if rank == 0:
            print(json.dumps({"extra": res}))
        return 0
    g, src = build_graph(20, 2)
    ctx = ap.Context(local)
    stream = ctx.stream
    dg = ap.DeviceGraph(g, dev)
    out = torch.empty(g.m, dtype=torch.int32, device=dev)
    ctx.reserve(g.m, g.nnz)

    for _ in range(args.warmup):
        ctx.sssp_into(dg, src, out)
    st = ctx.sssp_into(dg, src, out, stats=True)
    comp_edges, reached = st["edges_component"], st["vertices_reached"]

    sampler = ClockSampler(local)
    sampler.start()
    barrier(ws)
    total_ms, per = time_steps(stream, lambda: ctx.sssp_into(dg, src, out), args.steps)
    barrier(ws)
    clocks = sampler.stop()
    ctx.synchronize()
    ms_step = max_over_ranks(ws, total_ms / args.steps)
    launch_ms = max_over_ranks(ws, float(np.mean(per)))
    value = ws * comp_edges / (ms_step * 1e-3) / 1e9

    # e2e through the C ABI with host buffers
    h_rp = torch.from_numpy(g.row_ptr).pin_memory()
    h_ci = torch.from_numpy(g.col_ind).pin_memory()
    h_w = torch.from_numpy(g.val).pin_memory()
    h_out = torch.empty(g.m, dtype=torch.int32).pin_memory()
    d_rp = torch.empty_like(h_rp, device=dev)
    d_ci = torch.empty_like(h_ci, device=dev)
    d_w = torch.empty_like(h_w, device=dev)
    e2e_graph = ap.DeviceGraph.from_tensors(g.m, g.n, d_rp, d_ci, d_w, ap.VAL_I32)

    def e2e_step():
        with torch.cuda.stream(stream):
            d_rp.copy_(h_rp, non_blocking=True)
            d_ci.copy_(h_ci, non_blocking=True)
            d_w.copy_(h_w, non_blocking=True)
        ctx.sssp_into(e2e_graph, src, out)
        with torch.cuda.stream(stream):
            h_out.copy_(out, non_blocking=True)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    barrier(ws)
    e2e_total, _ = time_steps(stream, e2e_step, args.steps)
    barrier(ws)
    e2e_ms = max_over_ranks(ws, e2e_total / args.steps)
    h2d = (g.m + 1) * 4 + g.nnz * 8
    d2h = g.m * 4

    # correctness of what was timed
    import oracle

    ref = None
    if rank == 0:
        ref = oracle.sssp(g.row_ptr, g.col_ind, g.val, src)
        assert np.array_equal(h_out.numpy(), ref), "timed SSSP result differs from the oracle"

    peak, peak_kind = hbm_peak()
    alg_bytes = 8 * comp_edges + 8 * reached + 4 * g.m
    achieved = alg_bytes / (launch_ms * 1e-3) / 1e9

    line = {
        "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                   "l2": "inputs larger than L2 (CSR + weights 256 MB > 126 MB)",
                   "source": int(src), "vertices_reached": int(reached), "edges_component": int(comp_edges),
                   "iterations": st["iterations"], "edges_relaxed": st["edges_expanded"]},
        "e2e": {"value": ws * comp_edges / (e2e_ms * 1e-3) / 1e9, "unit": "GTEPS",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic_from_profile("sssp_kernel_rmat20"),
                     "kernel": "sssp_kernel", "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                     if peak_kind == "measured" else "fallback 6650 GB/s",
                     "alg_bytes_per_launch": alg_bytes, "launch_ms": launch_ms},
        "clocks": clocks,
    }

    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(g, src, comp_edges)
    if not args.no_extra:
        line["extra"] = extras(ctx, args, ws, local)
    ctx.close()
    if rank == 0:
        print(json.dumps(line))
    return 0


def cpu_baseline(g, src, comp_edges):
    import oracle

    if oracle.ref_available():
        _, info = oracle.ref_sssp(g.row_ptr, g.col_ind, g.val, src)
        ms, kind = info["ms"], "reference"
        sample = "one full scale-20 SSSP query by the reference ssspCPU (src/testSssp.cpp:117) compiled from its sources"
    else:
        t0 = time.perf_counter()
        oracle.sssp(g.row_ptr, g.col_ind, g.val, src)
        ms, kind = (time.perf_counter() - t0) * 1e3, "port"
        sample = "one full scale-20 SSSP query by the oracle's C restatement"
    return {"value": comp_edges / (ms * 1e-3) / 1e9, "unit": "GTEPS", "cores": 1, "kind": kind,
            "sample": sample, "ms": ms}


def extras(ctx, args, ws, local):
    """Every extra leg: traversal kernels, SpGEMM / TC, device construction, batched
    traversal and serving."""
    import apspie_b200 as ap

    _progress("extra: traversal")
    res = extras_traversal(ctx, args, ws, local)
    _progress("extra: spgemm / tc")
    res.update(extras_spgemm_tc(ctx, args, ws, local))
    _progress("extra: device construction")
    res.update(extras_build(ctx, args, ws, local))
    g22 = ap.gen_rmat(22, 16, 1, 3)  # weights for the serving leg; BFS ignores them
    _progress("extra: batched traversal")
    res.update(extras_batched(ctx, args, ws, local, g22))
    if ws == 1:
        res.update(extras_serving(ctx, args, local, g22))
    return res


def extras_traversal(ctx, args, ws, local):
    """BFS on R-MAT scale 14 (seed 1), MIS and BFS on R-MAT scale 20 (seed 2), same timing
    rules; MIS and BFS at scale 20 with their algorithmic-bytes roofline."""
    import torch

    import apspie_b200 as ap
    import oracle

    dev = f"cuda:{local}"
    res = {}
    g14, s14 = build_graph(14, 1)
    d14 = ap.DeviceGraph(g14, dev)
    o14 = torch.empty(g14.m, dtype=torch.int32, device=dev)
    for _ in range(max(3, args.warmup)):
        ctx.bfs_into(d14, s14, o14)
    st = ctx.bfs_into(d14, s14, o14, stats=True)
    steps = max(args.steps, 50)
    tot, per = time_steps(ctx.stream, lambda: ctx.bfs_into(d14, s14, o14), steps)
    ms = max_over_ranks(ws, tot / steps)
    res["bfs_rmat14"] = {"GTEPS": ws * st["edges_component"] / (ms * 1e-3) / 1e9, "us_per_bfs": ms * 1e3,
                         "levels": st["iterations"], "push_levels": st["push_iterations"],
                         "pull_levels": st["pull_iterations"], "edges_component": st["edges_component"],
                         "source": int(s14), "steps": steps,
                         "exact": bool(np.array_equal(o14.cpu().numpy(), oracle.bfs(g14.row_ptr, g14.col_ind, s14))),
                         "note": "whole CSR (1.8 MB) is L2-resident: launch/latency bound"}
    if oracle.ref_available():
        _, info = oracle.ref_bfs(g14.row_ptr, g14.col_ind, s14)
        res["bfs_rmat14"]["cpu_reference_ms"] = info["ms"]

    g20, _ = build_graph(20, 2)
    d20 = ap.DeviceGraph(g20, dev)
    pr = ap.mt19937_u32(4, g20.m)
    prio = torch.from_numpy(pr.view(np.int32)).to(dev)
    mem = torch.empty(g20.m, dtype=torch.uint8, device=dev)
    for _ in range(max(2, args.warmup)):
        ctx.mis_into(d20, prio, mem)
    st = ctx.mis_into(d20, prio, mem, stats=True)
    steps = max(5, min(args.steps, 20))
    tot, _ = time_steps(ctx.stream, lambda: ctx.mis_into(d20, prio, mem), steps)
    ms = max_over_ranks(ws, tot / steps)
    peak, peak_kind = hbm_peak()
    alg = 4 * g20.nnz + 13 * g20.m
    res["mis_rmat20"] = {"ms": ms, "rounds": st["iterations"], "set_size": st["vertices_reached"],
                         "edges_scanned": st["edges_expanded"], "alg_GBps": alg / (ms * 1e-3) / 1e9,
                         "frac": alg / (ms * 1e-3) / 1e9 / peak, "peak": f"{peak} GB/s ({peak_kind})",
                         "exact": bool(np.array_equal(mem.cpu().numpy(), oracle.mis_greedy(g20.row_ptr, g20.col_ind, pr)))}
    # BFS at scale 20 for the roofline of the BFS kernel on an HBM-sized graph
    s20 = ap.max_degree_vertex(g20)
    o20 = torch.empty(g20.m, dtype=torch.int32, device=dev)
    for _ in range(3):
        ctx.bfs_into(d20, s20, o20)
    st = ctx.bfs_into(d20, s20, o20, stats=True)
    steps = max(args.steps, 20)
    tot, _ = time_steps(ctx.stream, lambda: ctx.bfs_into(d20, s20, o20), steps)
    ms = max_over_ranks(ws, tot / steps)
    alg = 4 * st["edges_component"] + 8 * st["vertices_reached"] + 4 * g20.m
    res["bfs_rmat20"] = {"GTEPS": ws * st["edges_component"] / (ms * 1e-3) / 1e9, "ms": ms,
                         "levels": st["iterations"], "push_levels": st["push_iterations"],
                         "pull_levels": st["pull_iterations"], "alg_GBps": alg / (ms * 1e-3) / 1e9,
                         "frac": alg / (ms * 1e-3) / 1e9 / peak,
                         "exact": bool(np.array_equal(o20.cpu().numpy(), oracle.bfs(g20.row_ptr, g20.col_ind, s20)))}
    del d20, o20, mem, prio
    return res


def extras_build(ctx, args, ws, local):
    """Device graph construction: the R-MAT scale-20 edge list (seed 2, 16.8M generated
    edges with self-loops and repeats) -> symmetrised, deduplicated, weighted CSR; and the
    transpose of the ER n=2^20 matrix. Checked against the host generator's CSR."""
    import torch

    import apspie_b200 as ap

    dev = f"cuda:{local}"
    src, dst, w = ap.gen_rmat_coo(20, 16, 2, 3)
    ds, dd, dw = (torch.from_numpy(x).to(dev) for x in (src, dst, w))
    flags = ap.BUILD_SYMMETRIZE | ap.BUILD_DROP_SELF_LOOPS | ap.BUILD_DEDUP
    for _ in range(2):
        C = ctx.build_csr(1 << 20, ds, dd, dw, flags)
        C.free()
    steps = 5
    # outputs are callee-allocated (inside the timed call); they are freed after timing
    outs = []
    tot, _ = time_steps(ctx.stream, lambda: outs.append(ctx.build_csr(1 << 20, ds, dd, dw, flags)), steps)
    for o in outs:
        o.free()
    ms = max_over_ranks(ws, tot / steps)
    C = ctx.build_csr(1 << 20, ds, dd, dw, flags)
    rp, ci, val = C.to_numpy()
    g = ap.gen_rmat(20, 16, 2, 3)
    exact = bool(np.array_equal(rp, g.row_ptr) and np.array_equal(ci, g.col_ind) and np.array_equal(val, g.val))
    res = {"csr_build_rmat20": {"ms": ms, "edges_in": int(src.shape[0]), "nnz_out": int(C.nnz),
                                "Gedges_per_s": src.shape[0] / (ms * 1e-3) / 1e9, "exact": exact}}
    C.free()
    e = ap.gen_er(1 << 20, 8, 5, ap.VAL_F32)
    A = ap.DeviceGraph(e, dev)
    for _ in range(2):
        ctx.transpose(A).free()
    outs = []
    tot, _ = time_steps(ctx.stream, lambda: outs.append(ctx.transpose(A)), steps)
    for o in outs:
        o.free()
    res["transpose_er20"] = {"ms": max_over_ranks(ws, tot / steps), "nnz": e.nnz,
                             "note": "includes allocating the callee-owned output"}
    return res


def extras_spgemm_tc(ctx, args, ws, local):
    """C = A*A on ER n=2^20, 8 nnz/row (seed 5), f32 and i32; TC on R-MAT scale 18 (seed 1)."""
    import torch

    import apspie_b200 as ap
    import oracle

    res = {}
    peak, _ = hbm_peak()
    for vt, tag in ((ap.VAL_F32, "f32"), (ap.VAL_I32, "i32")):
        e = ap.gen_er(1 << 20, 8, 5, vt)
        A = ap.DeviceGraph(e, f"cuda:{local}")
        for _ in range(2):
            rp, ci, cv = ctx.spgemm_two_step(A, A)
        steps = 5
        tot, _ = time_steps(ctx.stream, lambda: ctx.spgemm_two_step(A, A), steps)
        ms = max_over_ranks(ws, tot / steps)
        nnz = int(ci.shape[0])
        alg = (4 * (e.m + 1) + 8 * e.nnz) + (4 * (e.m + 1) + 8 * nnz)
        orp, oci, ocv = oracle.spgemm(e.m, e.n, e.row_ptr, e.col_ind, e.val, e.row_ptr, e.col_ind, e.val)
        exact = (np.array_equal(rp.cpu().numpy(), orp) and np.array_equal(ci.cpu().numpy(), oci)
                 and np.array_equal(cv.cpu().numpy(), ocv))
        res[f"spgemm_er20_{tag}"] = {"ms": ms, "nnz_C": nnz, "products": 64 * e.m, "alg_GBps": alg / (ms * 1e-3) / 1e9,
                                     "frac_of_hbm": alg / (ms * 1e-3) / 1e9 / peak, "exact": bool(exact),
                                     "note": "symbolic + numeric into caller-owned C, two host syncs per call"}
        del A, rp, ci, cv
    g = ap.gen_rmat(18, 16, 1, 3, weights=False)
    Lh = ap.strict_lower(g)
    Ld = ap.DeviceGraph(Lh, f"cuda:{local}")
    for _ in range(2):
        count = ctx.tc(Ld)
    steps = 5
    tot, _ = time_steps(ctx.stream, lambda: ctx.tc(Ld), steps)
    ms = max_over_ranks(ws, tot / steps)
    wedges = int(np.diff(Lh.row_ptr)[Lh.col_ind].sum())
    alg = 4 * (Lh.m + 1) + 4 * Lh.nnz + 4 * wedges
    res["tc_rmat18"] = {"ms": ms, "triangles": count, "nnz_L": Lh.nnz, "wedges": wedges,
                        "alg_GBps": alg / (ms * 1e-3) / 1e9, "frac_of_hbm": alg / (ms * 1e-3) / 1e9 / peak,
                        "exact": bool(count == oracle.tc(Lh.row_ptr, Lh.col_ind))}
    return res


def extras_batched(ctx, args, ws, local, g):
    """Batched BFS and SSSP on R-MAT scale 22 (seed 1, int32 weights from seed 3): batches
    of 32/128/512 LCC sources (seed 6) against the plain path looping one source at a time
    over the same sources."""
    import torch

    import apspie_b200 as ap
    import oracle

    dev = f"cuda:{local}"
    dg = ap.DeviceGraph(g, dev)
    srcs = ap.lcc_sample(g, 512, 6)
    one = torch.empty(g.m, dtype=torch.int32, device=dev)
    for x in srcs[:3]:
        ctx.bfs_into(dg, int(x), one)
    tot, _ = time_steps(ctx.stream, lambda: [ctx.bfs_into(dg, int(x), one) for x in srcs[:64]], 1)
    plain_ms = max_over_ranks(ws, tot / 64)
    res = {"plain_bfs_rmat22": {"ms_per_query": plain_ms, "queries_per_s": ws * 1e3 / plain_ms}}
    # every batched row is compared with the plain path's answer for its source (row hashes),
    # and row 0 with the oracle
    ref = RowHasher(ctx, g.m, 512, dev)
    for q, x in enumerate(srcs):
        ctx.bfs_into(dg, int(x), one)
        ref.put_now(q, one)
    ref_h = ref.result()
    for nq in (32, 128, 512):
        s = torch.from_numpy(srcs[:nq]).to(dev)
        out = torch.empty((nq, g.m), dtype=torch.int32, device=dev)
        ctx.bfs_batch_into(dg, s, out)
        tot, per = time_steps(ctx.stream, lambda: ctx.bfs_batch_into(dg, s, out), 3)
        ms = max_over_ranks(ws, tot / 3)
        h = RowHasher(ctx, g.m, nq, dev, ref.coef)
        for q in range(nq):
            h.put(q, out[q])
        same = int((h.result() == ref_h[:nq]).sum())
        exact = same == nq and np.array_equal(out[0].cpu().numpy(), oracle.bfs(g.row_ptr, g.col_ind, int(srcs[0])))
        res[f"batched_bfs_rmat22_B{nq}"] = {"ms_per_batch": ms, "queries_per_s": ws * nq * 1e3 / ms,
                                            "x_plain": plain_ms * nq / ms, "rows_checked": nq,
                                            "rows_equal_plain": same, "exact": bool(exact)}
        del out
    # SSSP: the plain loop over 16 sources (each query takes milliseconds), then the batches
    for x in srcs[:2]:
        ctx.sssp_into(dg, int(x), one)
    tot, _ = time_steps(ctx.stream, lambda: [ctx.sssp_into(dg, int(x), one) for x in srcs[:16]], 1)
    plain_ms = max_over_ranks(ws, tot / 16)
    res["plain_sssp_rmat22"] = {"ms_per_query": plain_ms, "queries_per_s": ws * 1e3 / plain_ms}
    ref = RowHasher(ctx, g.m, 512, dev)
    for q, x in enumerate(srcs):
        ctx.sssp_into(dg, int(x), one)
        ref.put_now(q, one)
    ref_h = ref.result()
    for nq in (32, 128, 512):
        s = torch.from_numpy(srcs[:nq]).to(dev)
        out = torch.empty((nq, g.m), dtype=torch.int32, device=dev)
        ctx.sssp_batch_into(dg, s, out)
        reps = 3 if nq < 512 else 1
        tot, per = time_steps(ctx.stream, lambda: ctx.sssp_batch_into(dg, s, out), reps)
        ms = max_over_ranks(ws, tot / reps)
        h = RowHasher(ctx, g.m, nq, dev, ref.coef)
        for q in range(nq):
            h.put(q, out[q])
        same = int((h.result() == ref_h[:nq]).sum())
        exact = same == nq and np.array_equal(out[0].cpu().numpy(),
                                              oracle.sssp(g.row_ptr, g.col_ind, g.val, int(srcs[0])))
        res[f"batched_sssp_rmat22_B{nq}"] = {"ms_per_batch": ms, "queries_per_s": ws * nq * 1e3 / ms,
                                             "x_plain": plain_ms * nq / ms, "rows_checked": nq,
                                             "rows_equal_plain": same, "exact": bool(exact)}
        del out
    return res


SERVE_QUERIES = 100_000  # the serving stream's full length
SERVE_SLOTS = 2
SERVE_MAX_BATCH = 512
POOL_ROWS = 1536  # output rows per graph a stream keeps in flight (int32 rows; MIS: 64)


class RowHasher:
    """A 64-bit linear checksum of each result row, computed on the device by the library
    (apspie_row_checksums) without a host sync: h = sum_i row[i] * c[i] (int32 products,
    int64 sum; exact, so order-independent) with per-position coefficients drawn once.
    Equal rows give equal checksums; a differing row collides only with probability about
    2^-32. Rows are checksummed in groups of up to 128 per launch, on the given context's
    stream; put_now() checksums a row at once (for a buffer that is about to be reused)."""

    def __init__(self, ctx, m_max, n, dev, coef=None):
        import torch

        self.ctx = ctx
        if coef is None:
            g = torch.Generator(device="cpu").manual_seed(12345)
            coef = torch.randint(-(1 << 31), (1 << 31) - 1, (m_max,), generator=g, dtype=torch.int64)
            coef = coef.to(torch.int32).to(dev)
        self.coef = coef
        self.out = torch.zeros(n, dtype=torch.int64, device=dev)
        self.rows, self.slots = [], []

    def put(self, i, row):
        self.rows.append(row)
        self.slots.append(i)
        if len(self.rows) >= 128:
            self.flush()

    def put_now(self, i, row):
        self.put(i, row)
        self.flush()

    def flush(self):
        groups = {}
        for r, i in zip(self.rows, self.slots):
            groups.setdefault((r.shape[0], r.element_size()), ([], []))
            groups[(r.shape[0], r.element_size())][0].append(r)
            groups[(r.shape[0], r.element_size())][1].append(i)
        for rows, slots in groups.values():
            self.ctx.row_checksums(rows, slots, self.coef, self.out)
        self.rows, self.slots = [], []

    def result(self):
        self.flush()
        return self.out.cpu().numpy()


def serve_stream(graphs, n, rate_qps, seed=7):
    """The request stream: from mt19937(seed) words, per query a kind (70 % BFS, 25 % SSSP,
    5 % MIS), a graph (uniform), a source (uniform in that graph) and a Poisson arrival
    (exponential gaps at rate_qps; rate 0 = all at t=0). Kinds, graphs and sources do not
    depend on the rate."""
    import apspie_b200 as ap

    u = ap.mt19937_u32(seed, 4 * n).astype(np.float64).reshape(n, 4)
    r = u[:, 0] % 100
    kinds = np.where(r < 70, 0, np.where(r < 95, 1, 2)).astype(int)
    which = (u[:, 1] % len(graphs)).astype(int)
    srcs = (u[:, 2] % np.array([g.m for g in graphs])[which]).astype(np.int64)
    if rate_qps > 0:
        gaps = -np.log1p(-u[:, 3] / 4294967296.0) / rate_qps
        arrive = np.cumsum(gaps) - gaps[0]
    else:
        arrive = np.zeros(n)
    return kinds, which, srcs, arrive


def _progress(msg):
    """One progress line on stderr (the JSON result goes to stdout)."""
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def _pct(lat):
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "p99.9_ms": float(np.percentile(lat, 99.9))}


def serve_plain(ctx, dgs, prios, stream, dev, hasher=None):
    """One query at a time through the plain entry points, FIFO in arrival order; latency
    from arrival to completion. With a hasher, every answer's hash is recorded (on the
    library's stream, after the latency is taken)."""
    import torch

    kinds, which, srcs, arrive = stream
    outs = [torch.empty(d.m, dtype=torch.int32, device=dev) for d in dgs]
    mis_out = [torch.empty(d.m, dtype=torch.uint8, device=dev) for d in dgs]
    lat = np.zeros(len(kinds))
    t0 = time.perf_counter()
    for i in range(len(kinds)):
        k, w, s = int(kinds[i]), int(which[i]), int(srcs[i])
        now = time.perf_counter() - t0
        if now < arrive[i]:
            time.sleep(arrive[i] - now)
        if k == 0:
            ctx.bfs_into(dgs[w], s, outs[w])
        elif k == 1:
            ctx.sssp_into(dgs[w], s, outs[w])
        else:
            ctx.mis_into(dgs[w], prios[w], mis_out[w])
        ctx.synchronize()
        lat[i] = (time.perf_counter() - t0 - arrive[i]) * 1e3
        if i % 20000 == 19999:
            _progress(f"plain: {i + 1} done")
        if hasher is not None:  # on the library's stream, before the buffer is reused
            hasher.put_now(i, mis_out[w] if k == 2 else outs[w])
    total = time.perf_counter() - t0
    torch.cuda.synchronize()
    return lat, total


def serve_server(graphs, stream, dev, hasher, slots=None, max_batch=None, pool_rows=None, side_room=True):
    """The same stream through apspie_server (40 GB budget): the main thread submits at the
    arrival times from a pool of output rows per graph and, whenever a pool runs dry or
    while it waits for the next arrival, takes completed requests in bulk, hashes their
    rows on the device and returns the rows to the pools. Latency = server latency (submit
    to completion) + how late the submit was after the arrival. pool_rows: int32 output
    rows per graph (default POOL_ROWS each)."""
    import torch

    import apspie_b200 as ap

    kinds, which, srcs, arrive = stream
    srv = ap.Server(int(dev.split(":")[1]), budget_bytes=40 << 30, slots=slots or SERVE_SLOTS,
                    max_batch=max_batch or SERVE_MAX_BATCH)
    srv.set_side_room(side_room)
    gids = [srv.add_graph(g) for g in graphs]
    srv.start()
    pool_rows = pool_rows or [POOL_ROWS] * len(graphs)
    pools = [[torch.empty(g.m, dtype=torch.int32, device=dev) for _ in range(k)] for g, k in zip(graphs, pool_rows)]
    mpools = [[torch.empty(g.m, dtype=torch.uint8, device=dev) for _ in range(64)] for g in graphs]
    # warm-up: a burst of every (graph, kind) before the clock starts
    warm = []
    for gi, g in enumerate(graphs):
        for kind in (0, 1, 2):
            for k in range(min(16, len(pools[gi]))):
                o = (mpools if kind == 2 else pools)[gi][k]
                warm.append(srv.submit(gids[gi], kind, (k * 7919 + 1) % g.m, o))
    for t in warm:
        srv.wait(t)
    n = len(kinds)
    owner = {}  # ticket -> (query index, row tensor, pool)
    late = np.zeros(n)
    lat = np.zeros(n)
    hashed = []  # rows whose checksums are queued but not yet launched as a group
    checks = collections.deque()  # (event after a group's checksums, its (row, pool) pairs)
    # where the client's time goes: submit calls, waits for completions (blocking takes),
    # hashing the completed rows, and waits for checksums before their rows are reused
    client = {"submit_s": 0.0, "wait_s": 0.0, "check_s": 0.0, "check_wait_s": 0.0, "blocking_takes": 0,
              "pool_empty": 0}

    def recycle(wait):
        """Rows whose checksums have run go back to their pools (wait: for the oldest group)."""
        back = 0
        while checks and (wait or checks[0][0].query()):
            ev, done = checks.popleft()
            if wait:
                t_w = time.perf_counter()
                ev.synchronize()
                client["check_wait_s"] += time.perf_counter() - t_w
                wait = False
            for row, pool in done:
                pool.append(row)
            back += len(done)
        return back

    def drain(block):
        got = []
        if owner:
            t_w = time.perf_counter()
            try:
                got = srv.take_completed(cap=4096, timeout_ms=-1 if block else 0)
            except ap.ApspieError as e:
                if e.name != "APSPIE_ERR_TIMEOUT":
                    raise
            if block:
                client["wait_s"] += time.perf_counter() - t_w
                client["blocking_takes"] += 1
        t_c = time.perf_counter()
        for t, status, ms in got:
            i, row, pool = owner.pop(t)
            if status != 0:
                raise RuntimeError(f"request {i} failed with status {status}")
            lat[i] = ms + late[i]
            hasher.put(i, row)
            hashed.append((row, pool))
        if hashed and (block or len(hashed) >= 256):
            # the rows return to their pools once the event after their checksums has passed
            hasher.flush()
            ev = torch.cuda.Event()
            ev.record(torch.cuda.current_stream())
            checks.append((ev, list(hashed)))
            hashed.clear()
        recycle(False)
        client["check_s"] += time.perf_counter() - t_c
        return len(got)

    gid_of = np.asarray(gids, dtype=np.int32)[np.asarray(which, dtype=np.int64)]
    t0 = time.perf_counter()
    i = 0
    next_note = 20000
    while i < n:
        now = time.perf_counter() - t0
        if arrive[i] > now:
            if drain(False) == 0:
                time.sleep(min(2e-4, max(0.0, arrive[i] - now)))
            continue
        # every request that has arrived and has an output row, in arrival order, is
        # submitted in one call
        batch, rows, bpools = [], [], []
        while i < n and arrive[i] <= now and len(batch) < 4096:
            pool = mpools[int(which[i])] if int(kinds[i]) == 2 else pools[int(which[i])]
            if not pool:
                break
            rows.append(pool.pop())
            bpools.append(pool)
            batch.append(i)
            i += 1
        if not batch:
            client["pool_empty"] += 1
            if not recycle(False):
                if owner:
                    drain(True)
                else:
                    drain(True)  # nothing at the server: launch the queued rows' checksums
                    recycle(True)
            continue
        t_s = time.perf_counter()
        late[batch] = (t_s - t0 - np.asarray(arrive)[batch]) * 1e3
        tickets = srv.submit_many(gid_of[batch], np.asarray(kinds)[batch], np.asarray(srcs)[batch], rows)
        for t, j, row, pool in zip(tickets.tolist(), batch, rows, bpools):
            owner[t] = (j, row, pool)
        client["submit_s"] += time.perf_counter() - t_s
        if i >= next_note:
            _progress(f"server: {i} submitted, {i - len(owner)} completed")
            next_note += 20000
    while owner:
        drain(True)
    drain(True)
    while checks:
        recycle(True)
    total = time.perf_counter() - t0
    torch.cuda.synchronize()
    st = srv.stats()
    srv.close()
    st["client"] = {k: round(v, 4) if isinstance(v, float) else v for k, v in client.items()}
    return lat, total, st


def extras_serving(ctx, args, local, g22):
    """Serving on 4 resident R-MAT graphs (scales 16/18/20/22, edge factor 16, int32
    weights [1,255]; seeds 16/18/2/1) under a 40 GB budget: the 100,000-query 70/25/5
    BFS/SSSP/MIS stream (mt19937 seed 7), first all at once (saturation), then with Poisson
    arrivals at 0.8x and 2x the plain path's saturated rate; and a BFS-only stream on the
    scale-22 graph. The plain path runs each stream one query at a time, FIFO. Every answer
    of every server run is compared with the plain path's answer to the same query (a
    64-bit hash of each row, computed on the device)."""
    import apspie_b200 as ap
    import torch

    dev = f"cuda:{local}"
    graphs = [ap.gen_rmat(16, 16, 16, 3), ap.gen_rmat(18, 16, 18, 3), ap.gen_rmat(20, 16, 2, 3), g22]
    dgs = [ap.DeviceGraph(g, dev) for g in graphs]
    prios = [torch.from_numpy(ap.mt19937_u32(4, g.m).view(np.int32)).to(dev) for g in graphs]
    n = args.serve_queries
    m_max = max(g.m for g in graphs)
    legs = set(args.serve_legs.split(","))
    hctx = ap.Context(local)  # the server leg's checksums run on torch's current stream
    res = {"serving": {
        "workload": "4 graphs R-MAT s16/s18/s20/s22, 70/25/5 BFS/SSSP/MIS, 40 GB budget, 100,000 queries",
        "slots": args.serve_slots, "max_batch": SERVE_MAX_BATCH, "queries": n}}
    coef = None
    if legs & {"mixed", "poisson"}:
        sat = serve_stream(graphs, n, 0.0)
        serve_plain(ctx, dgs, prios, serve_stream(graphs, 50, 0.0), dev)  # warm-up
        ref = RowHasher(ctx, m_max, n, dev)
        coef = ref.coef
        _progress(f"serving: plain path, {n} queries")
        lat_p, tot_p = serve_plain(ctx, dgs, prios, sat, dev, ref)
        ref_h = ref.result()
        plain_qps = n / tot_p

        def run_server(stream):
            _progress("serving: server")
            h = RowHasher(hctx, m_max, n, dev, ref.coef)
            lat_s, tot_s, st = serve_server(graphs, stream, dev, h, slots=args.serve_slots,
                                            side_room=not args.serve_no_side_room)
            return lat_s, tot_s, st, int((h.result() == ref_h).sum())

    if "mixed" in legs:
        lat_s, tot_s, st, same = run_server(sat)
        res["serving"].update({
            "plain_qps": plain_qps, "server_qps": n / tot_s, "x_plain": tot_p / tot_s,
            "saturated": {"server": _pct(lat_s), "plain": _pct(lat_p)},
            "launches": st["launches"], "joined_running": st["joined_running"], "trivial": st["trivial"],
            "engine_launches": st["engine_launches"], "engine_levels": st["engine_levels"],
            "client": st["client"],
            "max_batch_seen": st["max_batch_seen"], "peak_bytes": st["peak_bytes"],
            "exact_checked": n, "exact_equal": same, "exact": same == n})
    for mult in ((0.8, 2.0) if "poisson" in legs else ()):
        rate = mult * plain_qps
        stream = serve_stream(graphs, n, rate)
        lat_s, tot_s, st, same = run_server(stream)
        _progress(f"serving: plain path at {rate:.0f} queries/s")
        lat_p, tot_p = serve_plain(ctx, dgs, prios, stream, dev)
        res["serving"][f"poisson_{mult}x_plain_rate"] = {
            "rate_qps": rate, "server": dict(_pct(lat_s), qps=n / tot_s),
            "plain": dict(_pct(lat_p), qps=n / tot_p), "joined_running": st["joined_running"],
            "exact_checked": n, "exact": same == n}
    if "bfs" not in legs:
        hctx.close()
        return res
    # BFS-only stream on the scale-22 graph: the batched-serving target
    words = ap.mt19937_u32(8, n).astype(np.int64)
    bstream = (np.zeros(n, dtype=int), np.full(n, 3), words % graphs[3].m, np.zeros(n))
    bref = RowHasher(ctx, m_max, n, dev, coef)
    _progress("serving: BFS-only stream, plain path")
    lat_p, tot_p = serve_plain(ctx, dgs, prios, bstream, dev, bref)
    _progress("serving: BFS-only stream, server")
    bref_h = bref.result()
    h = RowHasher(hctx, m_max, n, dev, bref.coef)
    pool = [0] * (len(graphs) - 1) + [args.serve_pool]  # only the scale-22 graph is queried
    lat_s, tot_s, st = serve_server(graphs, bstream, dev, h, slots=args.serve_slots, pool_rows=pool,
                                    side_room=not args.serve_no_side_room)
    same = int((h.result() == bref_h).sum())
    hctx.close()
    res["serving"]["bfs_only_rmat22_saturated"] = {
        "queries": n, "plain_qps": n / tot_p, "server_qps": n / tot_s, "x_plain": tot_p / tot_s,
        "server": _pct(lat_s), "plain": _pct(lat_p), "launches": st["launches"],
        "joined_running": st["joined_running"], "trivial": st["trivial"], "max_batch_seen": st["max_batch_seen"],
        "engine_launches": st["engine_launches"], "engine_levels": st["engine_levels"],
        "client": st["client"], "pool_rows": args.serve_pool, "side_room": not args.serve_no_side_room,
        "exact_checked": n, "exact": same == n}
    return res


def main():
    ap_ = argparse.ArgumentParser()
    ap_.add_argument("--gpus", type=int, default=1)
    ap_.add_argument("--steps", type=int, default=100)
    ap_.add_argument("--warmup", type=int, default=3)
    ap_.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap_.add_argument("--no-extra", action="store_true")
    ap_.add_argument("--no-cpu-baseline", action="store_true")
    ap_.add_argument("--serve-queries", type=int, default=SERVE_QUERIES,
                     help="length of the serving streams (default: the config's 100,000)")
    ap_.add_argument("--serve-slots", type=int, default=SERVE_SLOTS, help="server execution slots")
    ap_.add_argument("--serve-pool", type=int, default=4096,
                     help="output rows the BFS-only serving leg keeps in flight")
    ap_.add_argument("--serve-no-side-room", action="store_true",
                     help="serving: let a slot's persistent grid fill the device when it runs alone")
    ap_.add_argument("--serve-legs", default="mixed,poisson,bfs",
                     help="serving legs to run (comma list of mixed, poisson, bfs)")
    ap_.add_argument("--only-extra", choices=["traversal", "spgemm_tc", "build", "batched", "serving"], default=None,
                     help="run one extra leg alone and print its JSON (no headline line)")
    args = ap_.parse_args()
    ws, rank, local = dist_env()
    if ws > 1 and args.impl == "ours":
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.impl == "reference":
            return main_reference(args, ws, rank)
        return main_ours(args, ws, rank, local)
    finally:
        if ws > 1 and args.impl == "ours":
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
