"""Autotuned launch geometry: the table round-trips through the C ABI, bad
entries are rejected, results stay exact under the smallest and the largest
grid caps, and the committed table is well formed."""
import numpy as np
import pytest

import gswitch_b200 as gs
import oracle
from gswitch_b200.autotune import load_table

pytestmark = pytest.mark.gpu


def test_table_round_trip_and_validation(ctx):
    t = np.arange(gs.TUNE_ENTRIES, dtype=np.int32) % 17
    ctx.tune_load(t)
    assert np.array_equal(ctx.tune_save(), t)
    bad = t.copy()
    bad[3] = 65
    with pytest.raises(gs.GswError):
        ctx.tune_load(bad)
    ctx.tune_load(None)
    assert not ctx.tune_save().any()


@pytest.mark.parametrize("quarters", [1, 64])
def test_results_exact_under_extreme_grids(ctx, quarters):
    h = oracle.rmat(13, 16, seed=6)
    hw = oracle.add_weights(h, 3, 64)
    root = int(oracle.roots(h, 4, 1)[0])
    g = ctx.upload(hw.off, hw.col, hw.w)
    ctx.tune_load(np.full(gs.TUNE_ENTRIES, quarters, dtype=np.int32))
    try:
        ref = oracle.bfs(h, root)
        dref = oracle.sssp_dijkstra(hw, root)
        for cfg in ["", "Push-Queue-WM", "Push-Queue-STRICT-Fused", "Pull-Bitmap-TM", "Push-Bitmap-TWC",
                    "Pull-Queue-CM"]:
            lv, _ = g.bfs(root, cfg)
            assert np.array_equal(lv, ref), (quarters, cfg)
            d, _ = g.sssp(root, cfg)
            assert np.array_equal(d, dref), (quarters, cfg)
        lv, _ = g.bfs(root, gs.RunOpts(captured=True))
        assert np.array_equal(lv, ref)
    finally:
        ctx.tune_load(None)


def test_committed_table_is_well_formed():
    t = load_table()
    assert t is not None and t.shape == (gs.TUNE_ENTRIES,)
    assert np.all((t >= 0) & (t <= 64))


def test_shape_table_round_trip_and_validation(ctx):
    """Shapes exist only for the STRICT variants (3 tiles), the thread-mapped
    push (3 CTA sizes) and the thread-mapped pull (3 candidates-per-thread
    counts x 3 CTA sizes); anything else is rejected."""
    s = np.zeros(gs.TUNE_ENTRIES, dtype=np.int32)
    s[gs.Context.tune_index("Push", "Queue", "STRICT")] = 2
    s[gs.Context.tune_index("Pull", "Bitmap", "TM")] = 8
    s[gs.Context.tune_index("Push", "Queue", "TM", True)] = 2
    ctx.tune_load_shapes(s)
    assert np.array_equal(ctx.tune_save_shapes(), s)
    for bad in ((gs.Context.tune_index("Push", "Queue", "WM"), 1), (gs.Context.tune_index("Pull", "Bitmap", "STRICT"), 3),
                (gs.Context.tune_index("Pull", "Bitmap", "TM"), 9), (gs.Context.tune_index("Push", "Bitmap", "TM"), 3)):
        b = s.copy()
        b[bad[0]] = bad[1]
        with pytest.raises(gs.GswError):
            ctx.tune_load_shapes(b)
    ctx.tune_load_shapes(None)
    assert not ctx.tune_save_shapes().any()


@pytest.mark.parametrize("shape", [1, 2, 3, 4, 5, 6, 7, 8])
def test_results_exact_under_every_shape(ctx, shape):
    """Every STRICT tile, every thread-mapped CTA size and every pull
    candidates-per-thread count gives the oracle's BFS, SSSP and PageRank."""
    h = oracle.rmat(14, 16, seed=7)
    hw = oracle.add_weights(h, 3, 64)
    root = int(oracle.roots(h, 4, 1)[0])
    g = ctx.upload(hw.off, hw.col, hw.w)
    gu = ctx.upload(h.off, h.col)
    s = np.zeros(gs.TUNE_ENTRIES, dtype=np.int32)
    for d in ("Push", "Pull"):
        for f in ("Queue", "Bitmap"):
            for fused in ((False, True) if d == "Push" else (False,)):
                s[gs.Context.tune_index(d, f, "STRICT", fused)] = shape % 3
                s[gs.Context.tune_index("Push", f, "TM", fused)] = shape % 3
            s[gs.Context.tune_index("Pull", f, "TM")] = shape
    ctx.tune_load_shapes(s)
    try:
        ref, dref = oracle.bfs(h, root), oracle.sssp_dijkstra(hw, root)
        for cfg in ["Push-Queue-STRICT", "Pull-Bitmap-STRICT", "Push-Queue-STRICT-Fused", "Pull-Bitmap-TM",
                    "Pull-Queue-TM", "Push-Queue-TM", "Push-Bitmap-TM", "Push-Queue-TM-Fused", ""]:
            lv, _ = gu.bfs(root, gs.RunOpts.from_config(cfg, persistent=False))
            assert np.array_equal(lv, ref), (shape, cfg)
            d, _ = g.sssp(root, gs.RunOpts.from_config(cfg, persistent=False))
            assert np.array_equal(d, dref), (shape, cfg)
        from test_gpu_apps import _pr_l1
        for cfg in ["Pull-Bitmap-STRICT", "Pull-Bitmap-TM"]:
            pr, _ = gu.pagerank(iters=20, eps=0.0, opts=cfg)
            assert _pr_l1(pr, h)[0] <= 1e-6, (shape, cfg)
    finally:
        ctx.tune_load_shapes(None)
