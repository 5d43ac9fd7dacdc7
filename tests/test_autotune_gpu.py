"""GPU tests of the autotuner: every candidate a tuner may pick gives the oracle's answer,
the tuner records its choice per (kind, shape bucket), later calls on that bucket use it,
and the table survives a save / load round trip."""
import numpy as np
import pytest

import apspie_b200 as ap
import oracle
from test_spgemm_tc_gpu import _check, _skewed

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rmat12():
    g = ap.gen_rmat(12, 16, 1, 3)
    return g, ap.DeviceGraph(g), ap.max_degree_vertex(g)


@pytest.fixture
def fresh_ctx():
    c = ap.Context(0)
    yield c
    c.close()


def _knobs_of_other_kinds_unchanged(before, after, kind):
    mine = {ap.TUNE_BFS: {"bfs_alpha", "bfs_beta"}, ap.TUNE_SSSP: {"sssp_band", "sssp_delta"},
            ap.TUNE_BFS_BATCH: {"batch_push_frac"}, ap.TUNE_SPGEMM: {"spgemm_reg_max", "spgemm_block_max"},
            ap.TUNE_TC: {"tc_task_work", "tc_orient"}}[kind]
    for k in before:
        if k not in mine:
            assert before[k] == after[k], k


def test_autotune_bfs_and_sssp_record_and_keep_results(fresh_ctx, rmat12):
    ctx = fresh_ctx
    g, dg, src = rmat12
    defaults = ctx.get_params()
    for kind in (ap.TUNE_BFS, ap.TUNE_SSSP):
        best, ms = ctx.autotune(kind, dg, sources=[src], reps=2)
        assert ms > 0
        _knobs_of_other_kinds_unchanged(defaults, best, kind)
        got, found = ctx.tune_lookup(kind, dg)
        assert found and got == best
    assert ctx.tune_entries() == 2
    assert ctx.get_params() == defaults  # the context's own knobs are restored
    np.testing.assert_array_equal(ctx.bfs(dg, src).cpu().numpy(), oracle.bfs(g.row_ptr, g.col_ind, src))
    np.testing.assert_array_equal(ctx.sssp(dg, src).cpu().numpy(),
                                  oracle.sssp(g.row_ptr, g.col_ind, g.val, src))


def test_autotune_bfs_batch(fresh_ctx, rmat12):
    import torch

    ctx = fresh_ctx
    g, dg, _ = rmat12
    srcs = ap.lcc_sample(g, 40, 6)
    best, _ = ctx.autotune(ap.TUNE_BFS_BATCH, dg, sources=list(srcs), reps=1)
    assert ctx.tune_lookup(ap.TUNE_BFS_BATCH, dg)[1]
    out = ctx.bfs_batch(dg, torch.from_numpy(srcs).cuda())
    for q in (0, 17, 39):
        np.testing.assert_array_equal(out[q].cpu().numpy(), oracle.bfs(g.row_ptr, g.col_ind, int(srcs[q])))


def test_autotune_spgemm_and_tc(fresh_ctx):
    ctx = fresh_ctx
    e = ap.gen_er(1 << 12, 8, 5, ap.VAL_I32)
    A = ap.DeviceGraph(e)
    best, _ = ctx.autotune(ap.TUNE_SPGEMM, A, A, reps=1)
    assert best["spgemm_reg_max"] in (0, 32, 64, 128) and best["spgemm_block_max"] in (256, 1024)
    _check(ctx, e, e)
    g = ap.gen_rmat(12, 16, 1, 3, weights=False)
    Lh = ap.strict_lower(g)
    Ld = ap.DeviceGraph(Lh)
    best, _ = ctx.autotune(ap.TUNE_TC, Ld, reps=1)
    assert best["tc_orient"] in (0, 1)
    assert ctx.tc(Ld) == oracle.tc(Lh.row_ptr, Lh.col_ind)


@pytest.mark.parametrize("reg_max", [0, 32, 64, 128])
@pytest.mark.parametrize("block_max", [0, 256, 1024])
def test_every_spgemm_tier_split_is_exact(ctx, reg_max, block_max):
    """block_max 0 sends every row above the register tiers to global-memory tables."""
    ctx.set_params(spgemm_reg_max=reg_max, spgemm_block_max=block_max)
    try:
        A = _skewed(3000, 1, ap.VAL_I32)
        B = _skewed(3000, 2, ap.VAL_I32)
        _check(ctx, A, B)
        e = ap.gen_er(1 << 11, 8, 5, ap.VAL_F32)
        _check(ctx, e, e, exact_f32=reg_max >= 64)
    finally:
        ctx.set_params(spgemm_reg_max=128, spgemm_block_max=1024)


@pytest.mark.parametrize("orient", [0, 1])
@pytest.mark.parametrize("task_work", [256, 1024, 65536])
def test_every_tc_setting_counts_the_same(ctx, orient, task_work):
    ctx.set_params(tc_orient=orient, tc_task_work=task_work)
    try:
        g = ap.gen_rmat(13, 16, 2, 3, weights=False)
        Lh = ap.strict_lower(g)
        assert ctx.tc(ap.DeviceGraph(Lh)) == oracle.tc(Lh.row_ptr, Lh.col_ind)
    finally:
        ctx.set_params(tc_orient=1, tc_task_work=4096)


def test_tc_input_that_is_not_strictly_lower_is_counted_as_given(ctx):
    """A full symmetric pattern is not a strict lower triangle: the count is
    sum((A*A) .* A) = 6 x triangles, with or without the orientation knob."""
    g = ap.gen_rmat(10, 8, 3, 3, weights=False)
    Lh = ap.strict_lower(g)
    tri = oracle.tc(Lh.row_ptr, Lh.col_ind)
    full = ap.DeviceGraph(ap.HostGraph(g.m, g.n, g.row_ptr, g.col_ind))
    assert ctx.tc(full) == 6 * tri


def test_tuning_table_save_load_and_off_switch(fresh_ctx, rmat12, tmp_path):
    ctx = fresh_ctx
    g, dg, src = rmat12
    best, _ = ctx.autotune(ap.TUNE_SSSP, dg, sources=[src], reps=1)
    path = tmp_path / "tune.txt"
    ctx.tune_save(path)
    other = ap.Context(0)
    try:
        assert other.tune_entries() == 0
        other.tune_load(path)
        got, found = other.tune_lookup(ap.TUNE_SSSP, dg)
        assert found and got["sssp_band"] == best["sssp_band"]
        other.set_autotune(False)
        own, found = other.tune_lookup(ap.TUNE_SSSP, dg)
        assert found and own["sssp_band"] == other.get_params()["sssp_band"]
        np.testing.assert_array_equal(other.sssp(dg, src).cpu().numpy(),
                                      oracle.sssp(g.row_ptr, g.col_ind, g.val, src))
    finally:
        other.close()
    bad = tmp_path / "bad.txt"
    bad.write_text("not a tuning file\n")
    with pytest.raises(ap.ApspieError):
        ctx.tune_load(bad)


def test_set_params_rejects_out_of_range(ctx):
    for knobs in ({"spgemm_reg_max": 48}, {"spgemm_block_max": 4096}, {"tc_task_work": 10},
                  {"tc_orient": 2}, {"bfs_beta": 0.0}):
        with pytest.raises(ap.ApspieError):
            ctx.set_params(**knobs)
    assert ctx.get_params()["spgemm_reg_max"] == 128
