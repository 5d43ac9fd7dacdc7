"""The C++ drop-in header include/apspie/compat.hpp: a program written against the
reference's entry points compiles (CPU) and, on a GPU, produces the oracle's answers."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER_SRC = os.path.join(ROOT, "tests", "compat_driver.cpp")


def _build(tmp_path):
    exe = os.path.join(str(tmp_path), "compat_driver")
    cmd = ["g++", "-std=c++14", "-O1", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
           DRIVER_SRC, "-o", exe, "-L", os.path.join(ROOT, "apspie_b200", "lib"), "-lapspie",
           "-L", "/usr/local/cuda/lib64", "-lcudart",
           "-Wl,-rpath," + os.path.join(ROOT, "apspie_b200", "lib"), "-Wl,-rpath,/usr/local/cuda/lib64"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-2000:]
    return exe


def test_compat_header_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_compat_driver_matches_oracle(tmp_path):
    import apspie_b200 as ap
    import oracle

    exe = _build(tmp_path)
    outdir = str(tmp_path)
    res = subprocess.run([exe, outdir], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    g = ap.gen_rmat(12, 16, 1, 3)
    src = ap.max_degree_vertex(g)
    rd = lambda name, dt: np.fromfile(os.path.join(outdir, name), dtype=dt)
    ref_bfs = oracle.bfs(g.row_ptr, g.col_ind, src)
    np.testing.assert_array_equal(rd("bfs.i32", np.int32), ref_bfs)
    np.testing.assert_array_equal(rd("spmspvbfs.i32", np.int32), ref_bfs)
    ref_sssp = oracle.sssp(g.row_ptr, g.col_ind, g.val, src)
    np.testing.assert_array_equal(rd("sssp.i32", np.int32), ref_sssp)
    f = rd("sssp.f32", np.float32)
    np.testing.assert_array_equal(f, np.where(ref_sssp < 0, np.float32(1.70141e38), ref_sssp).astype(np.float32))
    prf = rd("mis_prio.f32", np.float32)
    mis = rd("mis.i32", np.int32)
    np.testing.assert_array_equal(mis, oracle.mis_greedy(g.row_ptr, g.col_ind, prf.view(np.uint32)).astype(np.int32))
    assert oracle.mis_check(g.row_ptr, g.col_ind, mis.astype(np.uint8)) == 0
    hop = rd("hop.i32", np.int32)
    np.testing.assert_array_equal(mis + hop, np.ones(g.m, dtype=np.int32))  # uncompareResults
    vals = g.val.astype(np.float32)
    orp, oci, ocv = oracle.spgemm(g.m, g.m, g.row_ptr, g.col_ind, vals, g.row_ptr, g.col_ind, vals)
    np.testing.assert_array_equal(rd("spgemm_rp.i32", np.int32), orp)
    np.testing.assert_array_equal(rd("spgemm_ci.i32", np.int32), oci)
    np.testing.assert_allclose(rd("spgemm_v.f32", np.float32), ocv, rtol=1e-5)
    er = ap.gen_er(g.m, 8, 9, ap.VAL_F32)
    orp, oci, ocv = oracle.spgemm(g.m, g.m, er.row_ptr, er.col_ind, er.val, g.row_ptr, g.col_ind, vals)
    np.testing.assert_array_equal(rd("mxm_rp.i32", np.int32), orp)  # mXm: CSC of R^T * E^T = CSR of E * R
    np.testing.assert_array_equal(rd("mxm_ci.i32", np.int32), oci)
    # rows of E*R reach hundreds of signed products: the f32 bar is |got - ref| <= 1e-5 * sum|a*b|
    _, _, mag = oracle.spgemm(g.m, g.m, er.row_ptr, er.col_ind, np.abs(er.val), g.row_ptr, g.col_ind, vals)
    assert np.all(np.abs(rd("mxm_v.f32", np.float32) - ocv) <= 1e-5 * mag)
    xi = (7 * np.arange(64)) % g.m
    xi[63] = 0
    xv = (0.5 + np.arange(64) / 64.0).astype(np.float32)
    oi, ov = oracle.spmspv(g.row_ptr, g.col_ind, vals, g.m, xi, xv)
    np.testing.assert_array_equal(rd("mxv_i.i32", np.int32), oi)  # mXv: bit-exact, same summation order
    np.testing.assert_array_equal(rd("mxv_v.f32", np.float32), ov)
    L = ap.strict_lower(g)
    assert int(open(os.path.join(outdir, "tc.txt")).read()) == oracle.tc(L.row_ptr, L.col_ind)
