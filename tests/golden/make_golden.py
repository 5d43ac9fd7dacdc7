"""Generates tests/golden/golden.npz from the REFERENCE's own CPU code.

Run here, where the reference tree and oracle/_ref/apspie_ref (built by `make -C oracle`)
exist:  python tests/golden/make_golden.py REF_DIR   (or REF_DIR in the environment)

Contents, per small Matrix Market fixture of the reference (dataset/small/*.mtx) and
both load modes (directed / undirected = makeSymmetric):
  <name>_<u|d>_{row_ptr,col_ind}   CSR exactly as the reference loader builds it
                                   (readEdge/readMtx/makeSymmetric, buildMatrix order)
  <name>_<u|d>_bfs                 [m, m] depth from every source: bfsCPU (testBfs.cpp:75)
  <name>_<u|d>_w                   int32 weights (deterministic, symmetric in (u,v))
  <name>_<u|d>_sssp                [m, m] distances from every source: ssspCPU
                                   (testSssp.cpp:117) on those weights, -1 unreached
  <name>_u_misref                  misCPU (test/mis/main.cu:90) set from source 0
  <name>_u_mis                     greedy (priority, id) MIS, priorities mt19937(4)
                                   (oracle restatement: the reference has no CPU Luby MIS)
  <name>_u_tc                      triangle count of the strict lower triangle (oracle)
  mt19937_seed4                    first 1000 outputs of init_genrand(4)/genrand_int32
  rmat12_*                         R-MAT scale 12, edge factor 16, seed 1, weight seed 3:
                                   bfs/sssp from the max-degree vertex (reference code),
                                   mis (oracle) and a digest of the CSR so tests can
                                   regenerate the same graph with the library generator.
  spgemm_*                         C = A*A for the test_spgemm fixture and a small ER
                                   matrix (oracle restatement; the reference's own check
                                   was the removed cuSPARSE csrgemm).
"""
from __future__ import annotations

import glob
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
import apspie_b200 as ap  # noqa: E402


def weights_for(rp, ci):
    """Deterministic int32 weights in [1, 9], equal for (u,v) and (v,u)."""
    m = rp.shape[0] - 1
    rows = np.repeat(np.arange(m, dtype=np.int64), np.diff(rp))
    lo = np.minimum(rows, ci)
    hi = np.maximum(rows, ci)
    return (1 + (lo * 31 + hi * 17) % 9).astype(np.int32)


def csr_digest(rp, ci, val=None):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(rp, dtype=np.int32).tobytes())
    h.update(np.ascontiguousarray(ci, dtype=np.int32).tobytes())
    if val is not None:
        h.update(np.ascontiguousarray(val).tobytes())
    return h.hexdigest()


def main(ref_dir=None):
    ref_dir = ref_dir or os.environ.get("REF_DIR")
    if not ref_dir or not os.path.isdir(os.path.join(ref_dir, "dataset")):
        raise SystemExit("give the reference source tree: make_golden.py REF_DIR")
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/apspie_ref missing: run `make -C oracle REF_DIR=...` first")
    out = {}
    manifest = {"fixtures": []}
    for path in sorted(glob.glob(os.path.join(ref_dir, "dataset", "small", "*.mtx"))):
        name = os.path.splitext(os.path.basename(path))[0]
        for und in (0, 1):
            key = f"{name}_{'u' if und else 'd'}"
            rp, ci, val = oracle.ref_load_mtx(path, und)
            m = rp.shape[0] - 1
            out[key + "_row_ptr"] = rp
            out[key + "_col_ind"] = ci
            out[key + "_val"] = val
            bfs = np.stack([oracle.ref_bfs(rp, ci, s)[0] for s in range(m)])
            out[key + "_bfs"] = bfs
            if und:
                w = weights_for(rp, ci)
                out[key + "_w"] = w
                out[key + "_sssp"] = np.stack([oracle.ref_sssp(rp, ci, w, s)[0] for s in range(m)])
                out[key + "_misref"] = oracle.ref_mis_vertex_order(rp, ci, 0)[0]
                prio = oracle.ref_mt19937(4, m)
                out[key + "_mis"] = oracle.mis_greedy(rp, ci, prio)
                lrp = [0]
                lci = []
                for i in range(m):
                    row = [int(c) for c in ci[rp[i]:rp[i + 1]] if c < i]
                    lci += sorted(row)
                    lrp.append(len(lci))
                out[key + "_tc"] = np.array([oracle.tc(np.array(lrp), np.array(lci, dtype=np.int32))],
                                            dtype=np.int64)
            manifest["fixtures"].append({"key": key, "file": os.path.basename(path), "undirected": und,
                                         "m": int(m), "nnz": int(ci.shape[0])})
    out["mt19937_seed4"] = oracle.ref_mt19937(4, 1000)

    g = ap.gen_rmat(12, 16, 1, 3)
    src = ap.max_degree_vertex(g)
    out["rmat12_meta"] = np.array([g.m, g.nnz, src], dtype=np.int64)
    out["rmat12_bfs"] = oracle.ref_bfs(g.row_ptr, g.col_ind, src)[0]
    out["rmat12_sssp"] = oracle.ref_sssp(g.row_ptr, g.col_ind, g.val, src)[0]
    out["rmat12_mis"] = oracle.mis_greedy(g.row_ptr, g.col_ind, ap.mt19937_u32(4, g.m))
    manifest["rmat12_digest"] = csr_digest(g.row_ptr, g.col_ind, g.val)

    rp, ci = out["test_spgemm_d_row_ptr"], out["test_spgemm_d_col_ind"]
    ones = np.ones(ci.shape[0], dtype=np.float32)
    crp, cci, cval = oracle.spgemm(rp.shape[0] - 1, rp.shape[0] - 1, rp, ci, ones, rp, ci, ones)
    out["spgemm_fixture_row_ptr"], out["spgemm_fixture_col_ind"], out["spgemm_fixture_val"] = crp, cci, cval
    for vt, tag in ((ap.VAL_F32, "f32"), (ap.VAL_I32, "i32")):
        e = ap.gen_er(64, 4, 5, vt)
        crp, cci, cval = oracle.spgemm(e.m, e.n, e.row_ptr, e.col_ind, e.val, e.row_ptr, e.col_ind, e.val)
        out[f"spgemm_er64_{tag}_row_ptr"] = crp
        out[f"spgemm_er64_{tag}_col_ind"] = cci
        out[f"spgemm_er64_{tag}_val"] = cval
        manifest[f"er64_{tag}_digest"] = csr_digest(e.row_ptr, e.col_ind, e.val)

    here = os.path.dirname(os.path.abspath(__file__))
    np.savez_compressed(os.path.join(here, "golden.npz"), **out)
    with open(os.path.join(here, "golden.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    print(f"wrote {len(out)} arrays")


if __name__ == "__main__":
    main(*sys.argv[1:])
