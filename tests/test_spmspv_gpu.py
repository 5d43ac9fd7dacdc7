"""Valued sparse-in / sparse-out SpMSpV (apspie_spmspv, the reference's mXv<T>,
src/mXv.cuh:249-389) against the oracle's sequential restatement: indices exact, values
bit-exact (int32 and f32: both sum each column in x's entry order, then row order)."""
import numpy as np
import pytest

import apspie_b200 as ap
import oracle

pytestmark = pytest.mark.gpu


def _graph(kind, vt):
    if kind == "rmat":
        g = ap.gen_rmat(12, 16, 4, 3)
        val = g.val.astype(np.float32) / 7.0 if vt == ap.VAL_F32 else g.val
        return ap.HostGraph(g.m, g.n, g.row_ptr, g.col_ind, np.ascontiguousarray(val), True), val
    g = ap.gen_er(1 << 14, 8, 5, vt)
    return g, g.val


@pytest.mark.parametrize("kind", ["rmat", "er"])
@pytest.mark.parametrize("vt", [ap.VAL_F32, ap.VAL_I32])
@pytest.mark.parametrize("nx", [1, 37, 2000])
def test_spmspv_matches_oracle(ctx, kind, vt, nx):
    import torch

    g, val = _graph(kind, vt)
    rng = np.random.default_rng(nx * 7 + vt)
    x_ind = rng.integers(0, g.m, nx).astype(np.int32)  # repeats allowed: their products add
    if vt == ap.VAL_F32:
        x_val = rng.uniform(-1, 1, nx).astype(np.float32)
    else:
        x_val = rng.integers(-5, 6, nx).astype(np.int32)
    dg = ap.DeviceGraph(g)
    yi, yv = ctx.spmspv(dg, torch.from_numpy(x_ind).cuda(), torch.from_numpy(x_val).cuda())
    oi, ov = oracle.spmspv(g.row_ptr, g.col_ind, val, g.n, x_ind, x_val)
    np.testing.assert_array_equal(yi.cpu().numpy(), oi)
    np.testing.assert_array_equal(yv.cpu().numpy().view(np.uint32), ov.view(np.uint32))


def test_spmspv_empty_vector_and_empty_rows(ctx):
    import torch

    g, val = _graph("rmat", ap.VAL_I32)
    dg = ap.DeviceGraph(g)
    yi, yv = ctx.spmspv(dg, torch.empty(0, dtype=torch.int32, device="cuda"),
                        torch.empty(0, dtype=torch.int32, device="cuda"))
    assert yi.numel() == 0 and yv.numel() == 0
    deg = np.diff(g.row_ptr)
    iso = np.nonzero(deg == 0)[0][:5].astype(np.int32)  # rows with no entries
    assert iso.size > 0
    yi, _ = ctx.spmspv(dg, torch.from_numpy(iso).cuda(), torch.ones(iso.size, dtype=torch.int32, device="cuda"))
    assert yi.numel() == 0


def test_spmspv_rejects_index_out_of_range_and_context_survives(ctx):
    import torch

    g, val = _graph("er", ap.VAL_I32)
    dg = ap.DeviceGraph(g)
    bad = torch.tensor([0, g.m], dtype=torch.int32, device="cuda")
    with pytest.raises(ap.ApspieError) as ei:
        ctx.spmspv(dg, bad, torch.ones(2, dtype=torch.int32, device="cuda"))
    assert ei.value.name == "APSPIE_ERR_INVALID_ARG"
    x = np.array([3, 1, 3], dtype=np.int32)
    xv = np.array([1, 2, 3], dtype=np.int32)
    yi, yv = ctx.spmspv(dg, torch.from_numpy(x).cuda(), torch.from_numpy(xv).cuda())
    oi, ov = oracle.spmspv(g.row_ptr, g.col_ind, val, g.n, x, xv)
    np.testing.assert_array_equal(yi.cpu().numpy(), oi)
    np.testing.assert_array_equal(yv.cpu().numpy(), ov)


def test_row_checksums_match_a_torch_computation(ctx):
    """apspie_row_checksums equals sum(row * coef) computed by torch (int32 products,
    int64 sum), for int32 and uint8 rows, several rows per launch and more than one launch."""
    import torch

    m = 100_003
    g = torch.Generator().manual_seed(3)
    coef = torch.randint(-(1 << 31), (1 << 31) - 1, (m,), generator=g, dtype=torch.int64).to(torch.int32).cuda()
    rows = [torch.randint(-1, 40, (m,), generator=g, dtype=torch.int32).cuda() for _ in range(300)]
    out = torch.zeros(310, dtype=torch.int64, device="cuda")
    slots = list(range(5, 305))
    ctx.row_checksums(rows, slots, coef, out)
    ref = torch.stack([torch.sum(r * coef, dtype=torch.int64) for r in rows])
    assert torch.equal(out[5:305], ref) and int(out[:5].abs().sum()) == 0
    u8 = [torch.randint(0, 2, (m,), generator=g, dtype=torch.uint8).cuda() for _ in range(3)]
    o8 = torch.zeros(3, dtype=torch.int64, device="cuda")
    ctx.row_checksums(u8, [0, 1, 2], coef, o8)
    assert torch.equal(o8, torch.stack([torch.sum(r.to(torch.int32) * coef, dtype=torch.int64) for r in u8]))
    # int32 rows starting off a 16-byte boundary (views at 4-byte offsets) take the scalar path
    big = torch.randint(-1, 40, (m + 3,), generator=g, dtype=torch.int32).cuda()
    views = [big[k:k + m] for k in (1, 2, 3)]
    ov = torch.zeros(3, dtype=torch.int64, device="cuda")
    ctx.row_checksums(views, [0, 1, 2], coef, ov)
    assert torch.equal(ov, torch.stack([torch.sum(r * coef, dtype=torch.int64) for r in views]))
