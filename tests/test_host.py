"""CPU tests of the product's host side: the C-ABI library loads and exports every
declared symbol, the graph generators follow their stated specification, and the Matrix
Market loader builds exactly the reference loader's CSR. No device calls."""
import glob
import hashlib
import json
import os
import re

import numpy as np
import pytest

import apspie_b200 as ap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# The reference's small Matrix Market fixtures, read in place where its source tree is
# present (REF_DIR in the environment, else the build machine's checkout).
REF_SMALL = os.path.join(os.environ.get("REF_DIR", "/root/reference"), "dataset", "small")


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"\b(apspie_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = ap.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_signatures_cover_declarations():
    from apspie_b200 import _lib

    assert declared_functions() <= set(_lib.SIGNATURES)


def test_library_is_sm100a_only():
    import subprocess

    import shutil

    tool = shutil.which("cuobjdump") or os.path.join(os.environ.get("CUDA_HOME", ""), "bin", "cuobjdump")
    if not os.path.exists(tool):
        pytest.skip("cuobjdump unavailable")
    out = subprocess.run([tool, "--list-elf", ap.LIB_PATH], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    arches = set(re.findall(r"sm_(\d+a?)", out.stdout))
    assert arches == {"100a"}, arches


def test_mt19937_matches_reference(golden):
    np.testing.assert_array_equal(ap.mt19937_u32(4, 1000), golden["mt19937_seed4"])


def test_rmat_generator_is_deterministic_and_symmetric(golden):
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        man = json.load(f)
    g = ap.gen_rmat(12, 16, 1, 3)
    h = hashlib.sha256()
    for a in (g.row_ptr, g.col_ind, g.val):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest() == man["rmat12_digest"]
    meta = golden["rmat12_meta"]
    assert (g.m, g.nnz, ap.max_degree_vertex(g)) == tuple(int(x) for x in meta)
    m = g.m
    rows = np.repeat(np.arange(m), np.diff(g.row_ptr))
    assert np.all(rows != g.col_ind)  # no self-loops
    for i in range(0, m, 97):
        r = g.col_ind[g.row_ptr[i]:g.row_ptr[i + 1]]
        assert np.all(np.diff(r) > 0)  # sorted, no duplicates
    fwd = {(int(a), int(b)): int(w) for a, b, w in zip(rows, g.col_ind, g.val)}
    for (a, b), w in list(fwd.items())[:5000]:
        assert fwd[(b, a)] == w  # symmetric structure and weights
    assert g.val.min() >= 1 and g.val.max() <= 255


def test_rmat14_matches_published_probe_shape():
    g = ap.gen_rmat(14, 16, 1, 3, weights=False)
    assert (g.m, g.nnz, int(g.degrees().max())) == (16384, 426598, 3688)
    assert g.val is None


def test_er_generator():
    for vt, lo, hi in ((ap.VAL_F32, -1.0, 1.0), (ap.VAL_I32, 1, 8)):
        e = ap.gen_er(1000, 8, 5, vt)
        assert e.nnz == 8000 and np.all(np.diff(e.row_ptr) == 8)
        for i in range(e.m):
            assert np.all(np.diff(e.col_ind[8 * i:8 * i + 8]) > 0)
        assert e.val.min() >= lo and e.val.max() <= hi
    a = ap.gen_er(1000, 8, 5, ap.VAL_F32)
    b = ap.gen_er(1000, 8, 5, ap.VAL_I32)
    np.testing.assert_array_equal(a.col_ind, b.col_ind)  # same structure for both value runs


def test_lcc_sample_distinct_and_in_component():
    g = ap.gen_rmat(10, 4, 7, 3, weights=False)
    s = ap.lcc_sample(g, 64, 6)
    assert len(set(s.tolist())) == 64
    import oracle

    src = ap.max_degree_vertex(g)
    reach = oracle.bfs(g.row_ptr, g.col_ind, int(s[0]))
    assert np.all(reach[s] >= 0)
    assert reach[src] >= 0
    np.testing.assert_array_equal(s, ap.lcc_sample(g, 64, 6))


def test_strict_lower():
    g = ap.gen_rmat(8, 8, 2, 3, weights=False)
    L = ap.strict_lower(g)
    rows = np.repeat(np.arange(L.m), np.diff(L.row_ptr))
    assert np.all(L.col_ind < rows)
    assert L.nnz * 2 == g.nnz


@pytest.mark.skipif(not os.path.isdir(REF_SMALL), reason="reference fixtures absent")
def test_mtx_loader_matches_reference_loader(golden):
    for path in sorted(glob.glob(os.path.join(REF_SMALL, "*.mtx"))):
        name = os.path.splitext(os.path.basename(path))[0]
        for und in (0, 1):
            key = f"{name}_{'u' if und else 'd'}"
            g = ap.load_mtx(path, bool(und))
            np.testing.assert_array_equal(g.row_ptr, golden[key + "_row_ptr"], err_msg=key)
            np.testing.assert_array_equal(g.col_ind, golden[key + "_col_ind"], err_msg=key)
            np.testing.assert_array_equal(g.val, golden[key + "_val"], err_msg=key)


def test_mtx_loader_rejects_missing_file():
    with pytest.raises(ap.ApspieError):
        ap.load_mtx("/nonexistent/graph.mtx", False)


def test_mtx_loader_weighted_and_comments(tmp_path):
    p = tmp_path / "w.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real general\n% comment\n3 3 3\n2 1 0.5\n3 1 2.25\n1 3 4\n")
    g = ap.load_mtx(str(p), False)
    # (first, second) = (column, row): row 0 holds columns 1 and 2, row 2 holds column 0
    np.testing.assert_array_equal(g.row_ptr, [0, 2, 2, 3])
    np.testing.assert_array_equal(g.col_ind, [1, 2, 0])
    np.testing.assert_allclose(g.val, [0.5, 2.25, 4.0])


def _write_mtx(path, m, n, rows, cols, vals=None, comments=("%%MatrixMarket matrix coordinate real general",)):
    with open(path, "w") as f:
        for c in comments:
            f.write(c + "\n")
        f.write(f"{m} {n} {len(rows)}\n")
        for k in range(len(rows)):
            if vals is None:
                f.write(f"{cols[k] + 1} {rows[k] + 1}\n")
            else:
                f.write(f"{cols[k] + 1} {rows[k] + 1} {vals[k]:.6g}\n")


@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("undirected", [False, True])
def test_parallel_mtx_loader_equals_serial(tmp_path, weighted, undirected):
    rng = np.random.default_rng(11 + weighted + 2 * undirected)
    m = 3000
    ne = 40000
    rows = rng.integers(0, m, ne)
    cols = rng.integers(0, m, ne)
    rows[:500] = cols[:500]  # self-loops
    rows[500:1500], cols[500:1500] = rows[2000:3000], cols[2000:3000]  # repeated pairs
    vals = rng.uniform(-2, 2, ne) if weighted else None
    p = tmp_path / "g.mtx"
    _write_mtx(p, m, m, rows, cols, vals, comments=("%%MatrixMarket matrix coordinate real general", "% a", "%b"))
    ref = ap.load_mtx(str(p), undirected)
    for threads in (1, 2, 7, 0):
        got = ap.load_mtx(str(p), undirected, threads=threads)
        assert got.m == ref.m and got.n == ref.n
        np.testing.assert_array_equal(got.row_ptr, ref.row_ptr)
        np.testing.assert_array_equal(got.col_ind, ref.col_ind)
        np.testing.assert_array_equal(got.val, ref.val)


def test_parallel_mtx_loader_short_file_and_errors(tmp_path):
    p = tmp_path / "short.mtx"
    with open(p, "w") as f:
        f.write("%%MatrixMarket\n4 4 10\n1 2\n2 3\n")  # fewer entries than promised
    a, b = ap.load_mtx(str(p), False), ap.load_mtx(str(p), False, threads=3)
    np.testing.assert_array_equal(a.row_ptr, b.row_ptr)
    np.testing.assert_array_equal(a.col_ind, b.col_ind)
    with pytest.raises(ap.ApspieError):
        ap.load_mtx(str(tmp_path / "missing.mtx"), False, threads=2)


def test_rmat_generation_and_lcc_sample_are_independent_of_thread_count():
    """The generator splits the mt19937 stream into chunks decoded by worker threads and
    builds the CSR with per-thread offsets, and the component sample runs a parallel
    union-find: one thread and many give the same bytes."""
    import subprocess
    import sys

    code = ("import hashlib, numpy as np, apspie_b200 as ap\n"
            "g = ap.gen_rmat(16, 16, 5, 9)\n"
            "s, d, w = ap.gen_rmat_coo(15, 16, 5, 9)\n"
            "h = hashlib.sha256()\n"
            "smp = ap.lcc_sample(g, 64, 6)\n"
            "for a in (g.row_ptr, g.col_ind, g.val, s, d, w, smp): h.update(np.ascontiguousarray(a).tobytes())\n"
            "print(h.hexdigest())\n")
    digests = set()
    for threads in ("1", "3", "8"):
        env = dict(os.environ, OMP_NUM_THREADS=threads)
        out = subprocess.run([sys.executable, "-c", code], env=env, cwd=ROOT, capture_output=True, text=True,
                             timeout=300)
        assert out.returncode == 0, out.stderr
        digests.add(out.stdout.strip())
    assert len(digests) == 1


def test_integration_guide_covers_every_declared_function():
    """Every C-ABI function a header declares is named in the integration guide."""
    guide = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    missing = sorted(n for n in declared_functions() if n not in guide)
    assert not missing, missing


@pytest.mark.parametrize("scale,seed", [(10, 7), (12, 1), (14, 1)])
def test_rmat_generator_equals_oracle_restatement(scale, seed):
    """The product's parallel generator and the oracle's serial restatement of the same
    spec build the same CSR, weights included (the bench's reference arm builds its input
    with the oracle's)."""
    import oracle

    g = ap.gen_rmat(scale, 16, seed, 3)
    o = oracle.gen_rmat(scale, 16, seed, 3)
    np.testing.assert_array_equal(o.row_ptr, g.row_ptr)
    np.testing.assert_array_equal(o.col_ind, g.col_ind)
    np.testing.assert_array_equal(o.val, g.val)
    assert o.max_degree_vertex() == ap.max_degree_vertex(g)


def test_oracle_rmat_matches_committed_digest():
    import oracle

    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        man = json.load(f)
    o = oracle.gen_rmat(12, 16, 1, 3)
    h = hashlib.sha256()
    for a in (o.row_ptr, o.col_ind, o.val):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest() == man["rmat12_digest"]
