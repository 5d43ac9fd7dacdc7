"""GPU parity tests of the row-binned hash SpGEMM and the masked-SpGEMM triangle count.

int32 values and structures are compared bit-exact with the oracle (row-wise Gustavson).
FP32: rows with at most 128 products (the warp tier: every ER row of the benchmark) are
summed in the oracle's order and compared bit-exact; longer rows accumulate in any order
and are compared within |got - ref| <= 1e-5 * sum(|a_ik * b_kj|) + 1e-30."""
import numpy as np
import pytest

import apspie_b200 as ap
import oracle

pytestmark = pytest.mark.gpu


def _abs_bound(Ah, Bh, crp, cci):
    """sum over products of |a*b| for every output entry (float64)."""
    m = Ah.m
    out = np.zeros(cci.shape[0], dtype=np.float64)
    for i in range(m):
        acc = {}
        for ea in range(Ah.row_ptr[i], Ah.row_ptr[i + 1]):
            k = Ah.col_ind[ea]
            for eb in range(Bh.row_ptr[k], Bh.row_ptr[k + 1]):
                j = int(Bh.col_ind[eb])
                acc[j] = acc.get(j, 0.0) + abs(float(Ah.val[ea]) * float(Bh.val[eb]))
        for p in range(crp[i], crp[i + 1]):
            out[p] = acc[int(cci[p])]
    return out


def _check(ctx, Ah, Bh, exact_f32=True):
    A, B = ap.DeviceGraph(Ah), ap.DeviceGraph(Bh)
    rp, ci, cv = ctx.spgemm(A, B)
    orp, oci, ocv = oracle.spgemm(Ah.m, Bh.n, Ah.row_ptr, Ah.col_ind, Ah.val, Bh.row_ptr, Bh.col_ind, Bh.val)
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(ci, oci)
    if Ah.val.dtype == np.int32 or exact_f32:
        np.testing.assert_array_equal(cv, ocv)
    else:
        bound = _abs_bound(Ah, Bh, orp, oci)
        assert np.all(np.abs(cv.astype(np.float64) - ocv) <= 1e-5 * bound + 1e-30)
    return rp, ci, cv


def test_spgemm_golden_fixture(ctx, golden):
    rp, ci = golden["test_spgemm_d_row_ptr"], golden["test_spgemm_d_col_ind"]
    g = ap.HostGraph(rp.shape[0] - 1, rp.shape[0] - 1, rp, ci, np.ones(ci.shape[0], dtype=np.float32))
    crp, cci, cv = ctx.spgemm(ap.DeviceGraph(g), ap.DeviceGraph(g))
    np.testing.assert_array_equal(crp, golden["spgemm_fixture_row_ptr"])
    np.testing.assert_array_equal(cci, golden["spgemm_fixture_col_ind"])
    np.testing.assert_array_equal(cv, golden["spgemm_fixture_val"])


@pytest.mark.parametrize("vt", [ap.VAL_F32, ap.VAL_I32])
def test_spgemm_er64_golden(ctx, golden, vt):
    e = ap.gen_er(64, 4, 5, vt)
    tag = "f32" if vt == ap.VAL_F32 else "i32"
    rp, ci, cv = ctx.spgemm(ap.DeviceGraph(e), ap.DeviceGraph(e))
    np.testing.assert_array_equal(rp, golden[f"spgemm_er64_{tag}_row_ptr"])
    np.testing.assert_array_equal(ci, golden[f"spgemm_er64_{tag}_col_ind"])
    np.testing.assert_array_equal(cv, golden[f"spgemm_er64_{tag}_val"])


@pytest.mark.parametrize("vt", [ap.VAL_F32, ap.VAL_I32])
def test_spgemm_er_exact(ctx, vt):
    e = ap.gen_er(1 << 14, 8, 5, vt)  # every row: 64 products -> warp tier
    _check(ctx, e, e, exact_f32=True)


def _skewed(n, seed, vt, scale_rows=True):
    """Rows of very different lengths so every bin (warp/block/global) is exercised."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, 4, n)
    lens[rng.choice(n, 8, replace=False)] = rng.integers(40, 300, 8)
    lens[rng.choice(n, 3, replace=False)] = [1500, 2200, 3000]
    rp = np.zeros(n + 1, dtype=np.int32)
    rp[1:] = np.cumsum(lens)
    ci = np.concatenate([np.sort(rng.choice(n, int(l), replace=False)) for l in lens]).astype(np.int32)
    if vt == ap.VAL_F32:
        val = rng.uniform(-1, 1, ci.shape[0]).astype(np.float32)
    else:
        val = rng.integers(1, 9, ci.shape[0]).astype(np.int32)
    return ap.HostGraph(n, n, rp, ci, val)


@pytest.mark.parametrize("vt", [ap.VAL_F32, ap.VAL_I32])
def test_spgemm_all_bins(ctx, vt):
    A = _skewed(6000, 1, vt)
    B = _skewed(6000, 2, vt)
    _check(ctx, A, B, exact_f32=False)
    _check(ctx, B, A, exact_f32=False)


def test_spgemm_rectangular_and_empty(ctx):
    rng = np.random.default_rng(3)
    m, k, n = 300, 50, 700
    ra = np.sort(rng.integers(0, 4, m))
    rpa = np.zeros(m + 1, dtype=np.int32)
    rpa[1:] = np.cumsum(ra)
    cia = np.concatenate([np.sort(rng.choice(k, int(x), replace=False)) for x in ra]).astype(np.int32)
    rb = rng.integers(0, 9, k)
    rb[:5] = 0  # empty rows of B
    rpb = np.zeros(k + 1, dtype=np.int32)
    rpb[1:] = np.cumsum(rb)
    cib = np.concatenate([np.sort(rng.choice(n, int(x), replace=False)) for x in rb]).astype(np.int32)
    A = ap.HostGraph(m, k, rpa, cia, rng.integers(1, 9, cia.shape[0]).astype(np.int32))
    B = ap.HostGraph(k, n, rpb, cib, rng.integers(1, 9, cib.shape[0]).astype(np.int32))
    _check(ctx, A, B)


def test_spgemm_two_step_matches(ctx):
    e = ap.gen_er(4096, 8, 7, ap.VAL_I32)
    A = ap.DeviceGraph(e)
    rp, ci, cv = ctx.spgemm_two_step(A, A)
    orp, oci, ocv = oracle.spgemm(e.m, e.n, e.row_ptr, e.col_ind, e.val, e.row_ptr, e.col_ind, e.val)
    np.testing.assert_array_equal(rp.cpu().numpy(), orp)
    np.testing.assert_array_equal(ci.cpu().numpy(), oci)
    np.testing.assert_array_equal(cv.cpu().numpy(), ocv)


def test_spgemm_er_full_size_properties(ctx):
    """ER n=2^20, 8/row, C = A*A (the benchmark size): structure vs the oracle, f32 exact."""
    e = ap.gen_er(1 << 20, 8, 5, ap.VAL_F32)
    _check(ctx, e, e, exact_f32=True)


def test_spgemm_rejects_mismatch(ctx):
    e = ap.gen_er(64, 4, 5, ap.VAL_F32)
    f = ap.gen_er(64, 4, 5, ap.VAL_I32)
    with pytest.raises(ap.ApspieError):
        ctx.spgemm(ap.DeviceGraph(e), ap.DeviceGraph(f))


# --------------------------------------------------------------------------- TC
def test_tc_fixtures(ctx, golden, fixture_keys):
    for key in fixture_keys:
        if key + "_tc" not in golden:
            continue
        rp, ci = golden[key + "_row_ptr"], golden[key + "_col_ind"]
        A = ap.DeviceGraph(ap.HostGraph(rp.shape[0] - 1, rp.shape[0] - 1, rp, ci, None, True))
        Lg = ctx.strict_lower(A)
        assert ctx.tc(Lg) == int(golden[key + "_tc"][0]), key
        Lg.free()


@pytest.mark.parametrize("scale,ef", [(10, 16), (14, 16)])
def test_tc_rmat_vs_oracle(ctx, scale, ef):
    g = ap.gen_rmat(scale, ef, 1, 3, weights=False)
    Lh = ap.strict_lower(g)
    ref = oracle.tc(Lh.row_ptr, Lh.col_ind)
    assert ctx.tc(ap.DeviceGraph(Lh)) == ref
    Ld = ctx.strict_lower(ap.DeviceGraph(g))
    lrp, lci, _ = Ld.to_numpy()
    np.testing.assert_array_equal(lrp, Lh.row_ptr)
    np.testing.assert_array_equal(lci, Lh.col_ind)
    assert ctx.tc(Ld) == ref


def test_tc_rmat18_full_size(ctx):
    g = ap.gen_rmat(18, 16, 1, 3, weights=False)
    Lh = ap.strict_lower(g)
    assert ctx.tc(ap.DeviceGraph(Lh)) == oracle.tc(Lh.row_ptr, Lh.col_ind)


def test_tc_dense_clique_uses_block_and_global_tiers(ctx):
    # a 3000-clique: every row of L up to 2999 long -> block and global tiers
    n = 3000
    rows = [np.arange(i, dtype=np.int32) for i in range(n)]
    rp = np.zeros(n + 1, dtype=np.int32)
    rp[1:] = np.cumsum([len(r) for r in rows])
    ci = np.concatenate(rows)
    assert ctx.tc(ap.DeviceGraph(ap.HostGraph(n, n, rp, ci))) == n * (n - 1) * (n - 2) // 6
