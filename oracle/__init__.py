"""CPU oracle for apspie_b200 -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference legs may import this package, and only as the checker or the timed CPU
baseline. Two layers:

* ``liboracle.so`` (``oracle.c``): plain-C restatements of the reference algorithms
  (BFS src/testBfs.cpp:6-72, SSSP src/testSssp.cpp:33-115, MIS greedy fixed point of
  src/spmspvMis.cuh:54-78, vertex-order MIS test/mis/main.cu:25-88, SpGEMM/TC
  restatements), built by ``make -C oracle``;
* ``_ref/apspie_ref``: the reference's OWN CPU code (loader, bfsCPU, ssspCPU, misCPU,
  uncompareResults, MT19937) compiled from its sources by the same Makefile; it runs as a
  subprocess and is used to pin the restatements and as the reference CPU baseline.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "apspie_ref")

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE, "_build/liboracle.so"], check=True,
                           stdout=subprocess.DEVNULL)
        _lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        I = ctypes.c_int
        sig = {
            "oracle_bfs": (I, [I, P, P, I, I, P]),
            "oracle_sssp": (I, [I, P, P, P, I, P]),
            "oracle_mis_greedy": (None, [I, P, P, P, P]),
            "oracle_mis_vertex_order": (None, [I, P, P, I, P]),
            "oracle_mis_check": (ctypes.c_longlong, [I, P, P, P]),
            "oracle_spgemm_row_nnz": (ctypes.c_longlong, [I, I, P, P, P, P, P]),
            "oracle_spgemm_fill": (None, [I, I, I, P, P, P, P, P, P, P, P, P]),
            "oracle_tc": (ctypes.c_longlong, [I, P, P]),
            "oracle_mt19937": (None, [ctypes.c_uint, ctypes.c_longlong, P]),
            "oracle_spmspv": (I, [I, I, I, P, P, P, I, P, P, P, P]),
            "oracle_gen_rmat": (ctypes.c_longlong, [I, I, ctypes.c_uint, ctypes.c_uint, ctypes.c_double,
                                                    ctypes.c_double, ctypes.c_double, ctypes.c_longlong, P, P, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


# ---------------------------------------------------------------------------------
# restatements
# ---------------------------------------------------------------------------------
def bfs(row_ptr, col_ind, source, stop=1 << 30):
    rp, ci = _i32(row_ptr), _i32(col_ind)
    m = rp.shape[0] - 1
    out = np.empty(m, dtype=np.int32)
    lib().oracle_bfs(m, _p(rp), _p(ci), int(source), int(stop), _p(out))
    return out


def sssp(row_ptr, col_ind, weights, source):
    rp, ci, w = _i32(row_ptr), _i32(col_ind), _i32(weights)
    m = rp.shape[0] - 1
    out = np.empty(m, dtype=np.int32)
    rc = lib().oracle_sssp(m, _p(rp), _p(ci), _p(w), int(source), _p(out))
    if rc != 0:
        raise ValueError(f"oracle_sssp failed ({rc})")
    return out


def mis_greedy(row_ptr, col_ind, prio):
    rp, ci = _i32(row_ptr), _i32(col_ind)
    pr = np.ascontiguousarray(prio, dtype=np.uint32)
    m = rp.shape[0] - 1
    out = np.empty(m, dtype=np.uint8)
    lib().oracle_mis_greedy(m, _p(rp), _p(ci), _p(pr), _p(out))
    return out


def mis_vertex_order(row_ptr, col_ind, source=0):
    rp, ci = _i32(row_ptr), _i32(col_ind)
    m = rp.shape[0] - 1
    out = np.empty(m, dtype=np.int32)
    lib().oracle_mis_vertex_order(m, _p(rp), _p(ci), int(source), _p(out))
    return out


def mis_check(row_ptr, col_ind, member):
    rp, ci = _i32(row_ptr), _i32(col_ind)
    mem = np.ascontiguousarray(member, dtype=np.uint8)
    return int(lib().oracle_mis_check(rp.shape[0] - 1, _p(rp), _p(ci), _p(mem)))


def spgemm(m, n, arp, aci, aval, brp, bci, bval):
    """C = A*B (CSR, sorted columns; values float32 / int32 / None)."""
    arp, aci, brp, bci = _i32(arp), _i32(aci), _i32(brp), _i32(bci)
    crp = np.empty(m + 1, dtype=np.int32)
    nnz = int(lib().oracle_spgemm_row_nnz(m, n, _p(arp), _p(aci), _p(brp), _p(bci), _p(crp)))
    cci = np.empty(max(nnz, 1), dtype=np.int32)
    if aval is None:
        vt, cval = 0, None
        av = bv = None
    elif np.asarray(aval).dtype == np.float32:
        vt = 1
        av = np.ascontiguousarray(aval, dtype=np.float32)
        bv = np.ascontiguousarray(bval, dtype=np.float32)
        cval = np.empty(max(nnz, 1), dtype=np.float32)
    else:
        vt = 2
        av = np.ascontiguousarray(aval, dtype=np.int32)
        bv = np.ascontiguousarray(bval, dtype=np.int32)
        cval = np.empty(max(nnz, 1), dtype=np.int32)
    lib().oracle_spgemm_fill(m, n, vt, _p(arp), _p(aci), None if av is None else _p(av),
                             _p(brp), _p(bci), None if bv is None else _p(bv), _p(crp),
                             _p(cci), None if cval is None else _p(cval))
    return crp, cci[:nnz], None if cval is None else cval[:nnz]


def spmspv(row_ptr, col_ind, val, n, x_ind, x_val):
    """y = x^T A (sparse in, sparse out); returns (y_ind, y_val)."""
    rp, ci = _i32(row_ptr), _i32(col_ind)
    vt = 1 if np.asarray(val).dtype == np.float32 else 2
    dt = np.float32 if vt == 1 else np.int32
    av = np.ascontiguousarray(val, dtype=dt)
    xi = _i32(x_ind)
    xv = np.ascontiguousarray(x_val, dtype=dt)
    y_ind = np.empty(max(1, n), dtype=np.int32)
    y_val = np.empty(max(1, n), dtype=dt)
    k = lib().oracle_spmspv(rp.shape[0] - 1, n, vt, _p(rp), _p(ci), _p(av), xi.shape[0], _p(xi), _p(xv),
                            _p(y_ind), _p(y_val))
    return y_ind[:k].copy(), y_val[:k].copy()


def tc(row_ptr_l, col_ind_l):
    rp, ci = _i32(row_ptr_l), _i32(col_ind_l)
    return int(lib().oracle_tc(rp.shape[0] - 1, _p(rp), _p(ci)))


def spmv(row_ptr, col_ind, val, x):
    """y = A x in float64 (val None: a pattern of 1.0s); the dense-vector product of
    cuspmv (src/tc.cuh:17-59) and SpmvCsrBinary (src/bfs.cuh:11-14)."""
    rp = np.asarray(row_ptr, dtype=np.int64)
    rows = np.repeat(np.arange(rp.shape[0] - 1), np.diff(rp))
    a = np.ones(rows.shape[0]) if val is None else np.asarray(val, dtype=np.float64)
    y = np.zeros(rp.shape[0] - 1)
    np.add.at(y, rows, a * np.asarray(x, dtype=np.float64)[np.asarray(col_ind, dtype=np.int64)])
    return y


def pagerank(row_ptr, col_ind, damping=0.85, tol=1e-6, max_iter=100):
    """Power iteration in float64: r = 1/n, r' = (1 - d)/n + d (sum over in-edges of
    r[u]/outdeg(u) + dangling mass / n), until sum |r' - r| < tol. Returns (r, iterations)."""
    rp = np.asarray(row_ptr, dtype=np.int64)
    n = rp.shape[0] - 1
    deg = np.diff(rp)
    rows = np.repeat(np.arange(n), deg)
    cols = np.asarray(col_ind, dtype=np.int64)
    r = np.full(n, 1.0 / n)
    it = 0
    while it < max_iter:
        x = np.where(deg > 0, r / np.maximum(deg, 1), 0.0)
        y = np.zeros(n)
        np.add.at(y, cols, x[rows])
        nr = (1.0 - damping) / n + damping * (y + r[deg == 0].sum() / n)
        diff = np.abs(nr - r).sum()
        r = nr
        it += 1
        if diff < tol:
            break
    return r, it


class Csr:
    """A host CSR (row_ptr, col_ind, val) from the oracle's generator."""

    def __init__(self, row_ptr, col_ind, val):
        self.row_ptr, self.col_ind, self.val = row_ptr, col_ind, val
        self.m = self.n = row_ptr.shape[0] - 1
        self.nnz = col_ind.shape[0]

    def degrees(self):
        return np.diff(self.row_ptr)

    def max_degree_vertex(self):
        return int(np.argmax(self.degrees()))  # argmax takes the first (smallest id) maximum


def gen_rmat(scale, edge_factor, seed, weight_seed, a=0.57, b=0.19, c=0.19, weights=True):
    """Serial restatement of the undirected R-MAT input (oracle/gen.cpp states the spec)."""
    m = 1 << scale
    rp = np.empty(m + 1, dtype=np.int32)
    args = (scale, edge_factor, seed, weight_seed, a, b, c)
    need = lib().oracle_gen_rmat(*args, 0, _p(rp), None, None)
    if need < 0:
        raise ValueError("oracle_gen_rmat: bad arguments")
    ci = np.empty(need, dtype=np.int32)
    w = np.empty(need, dtype=np.int32) if weights else None
    got = lib().oracle_gen_rmat(*args, need, _p(rp), _p(ci), _p(w) if weights else None)
    assert got == need
    return Csr(rp, ci, w)


def mt19937(seed, count):
    out = np.empty(count, dtype=np.uint32)
    lib().oracle_mt19937(int(seed), int(count), _p(out))
    return out


# ---------------------------------------------------------------------------------
# the reference's own CPU code (oracle/_ref/apspie_ref)
# ---------------------------------------------------------------------------------
def ref_available() -> bool:
    return os.path.exists(REF_BIN)


def _run_ref(args):
    res = subprocess.run([REF_BIN] + [str(a) for a in args], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"apspie_ref {args[0]} failed ({res.returncode}): {res.stderr[-400:]}")
    for line in res.stdout.splitlines():
        if line.startswith("APSPIE_REF "):
            return json.loads(line[len("APSPIE_REF "):])
    raise RuntimeError("apspie_ref printed no result line")


def _write_csr(path, row_ptr, col_ind, val=None, n=None):
    rp, ci = _i32(row_ptr), _i32(col_ind)
    m = rp.shape[0] - 1
    vt = 0 if val is None else (1 if np.asarray(val).dtype == np.float32 else 2)
    with open(path, "wb") as f:
        np.array([m, m if n is None else n, ci.shape[0], vt], dtype=np.int32).tofile(f)
        rp.tofile(f)
        ci.tofile(f)
        if val is not None:
            np.ascontiguousarray(val).tofile(f)


def ref_load_mtx(path, undirected):
    """(row_ptr, col_ind, val float32) as the reference's readMtx/makeSymmetric build them."""
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "g.csr")
        _run_ref(["load", path, int(bool(undirected)), out])
        raw = np.fromfile(out, dtype=np.int32)
    m, _n, nnz = int(raw[0]), int(raw[1]), int(raw[2])
    rp = raw[4:5 + m].copy()
    ci = raw[5 + m:5 + m + nnz].copy()
    val = raw[5 + m + nnz:5 + m + 2 * nnz].view(np.float32).copy()
    return rp, ci, val


def _ref_vertex_cmd(cmd, row_ptr, col_ind, val, source):
    with tempfile.TemporaryDirectory() as d:
        g = os.path.join(d, "g.csr")
        out = os.path.join(d, "out.bin")
        _write_csr(g, row_ptr, col_ind, val)
        info = _run_ref([cmd, g, int(source), out])
        res = np.fromfile(out, dtype=np.int32)
    return res, info


def ref_bfs(row_ptr, col_ind, source):
    """bfsCPU (src/testBfs.cpp:75). Returns (depth, info with CPU ms)."""
    return _ref_vertex_cmd("bfs", row_ptr, col_ind, None, source)


def ref_sssp(row_ptr, col_ind, weights, source):
    """ssspCPU (src/testSssp.cpp:117) on float(weights). Returns (dist, info)."""
    return _ref_vertex_cmd("sssp", row_ptr, col_ind, _i32(weights), source)


def ref_sssp_f32(row_ptr, col_ind, weights_f32, source):
    """ssspCPU on float32 weights; float32 distances (-1 unreached). Returns (dist, info)."""
    with tempfile.TemporaryDirectory() as d:
        g = os.path.join(d, "g.csr")
        out = os.path.join(d, "out.bin")
        _write_csr(g, row_ptr, col_ind, np.ascontiguousarray(weights_f32, dtype=np.float32))
        info = _run_ref(["ssspf", g, int(source), out])
        res = np.fromfile(out, dtype=np.float32)
    return res, info


def ref_mis_vertex_order(row_ptr, col_ind, source=0):
    """misCPU (test/mis/main.cu:90). Returns (set 1/0, info)."""
    return _ref_vertex_cmd("mis", row_ptr, col_ind, None, source)


def ref_mis_check(row_ptr, col_ind, member):
    """The reference's one-hop + uncompareResults validity check; returns its error count."""
    with tempfile.TemporaryDirectory() as d:
        g = os.path.join(d, "g.csr")
        mp = os.path.join(d, "m.u8")
        _write_csr(g, row_ptr, col_ind)
        np.ascontiguousarray(member, dtype=np.uint8).tofile(mp)
        return int(_run_ref(["mischeck", g, mp])["errors"])


def ref_mt19937(seed, count):
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "mt.bin")
        _run_ref(["mt", int(seed), int(count), out])
        return np.fromfile(out, dtype=np.uint32)
