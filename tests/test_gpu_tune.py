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
