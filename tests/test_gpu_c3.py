"""Config C3 at full size: the 4096 x 4096 grid with 1% long-range edges
(weights U[1, 1000]) against the oracle, and RMAT scale 26 (67 M vertices,
about 2.1 B arcs, int64 row offsets) through size-independent properties.

BC on the grid: path counts are int32 in the reference (bc.cu:26-29) and
overflow on large grids; the engine keeps the reference's wrapping, so path
counts are compared bit for bit with the oracle's int32 restatement, and
dependencies are compared with the FP64 oracle (1e-5 relative) where no
count overflowed; the number of overflowed vertices is reported."""
import numpy as np
import pytest

import gswitch_b200 as gs
import oracle
from gswitch_b200.selector_train import load_fusion_model, load_model

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c3grid(ctx):
    h = oracle.grid(4096, 4096, 100, seed=1)
    hw = oracle.add_weights(h, 5, 1000)
    g = ctx.upload(hw.off, hw.col, hw.w)
    root = int(oracle.roots(h, 3, 1)[0])
    yield h, hw, g, root
    g.close()


def test_c3_grid_device_generator_matches_oracle(ctx, c3grid):
    h, _, _, _ = c3grid
    g = ctx.grid(4096, 4096, 100, seed=1)
    off, col, _ = g.download()
    assert np.array_equal(off, h.off) and np.array_equal(col, h.col)
    g.close()


def test_c3_grid_bfs(ctx, c3grid):
    h, _, g, root = c3grid
    ref = oracle.bfs(h, root)
    model, conf = load_model()
    ctx.mlp_load(model, conf)
    for o in (gs.RunOpts(), gs.RunOpts(selector="mlp"), gs.RunOpts(selector="mlp", captured=True),
              gs.RunOpts.from_config("Push-Queue-STRICT"), gs.RunOpts.from_config("Pull-Bitmap-TM-Standalone")):
        lv, st = g.bfs(root, o)
        assert np.array_equal(lv, ref)
        assert st.edges == oracle.traversed_edges(h, ref)
    ctx.mlp_load(None)


def test_c3_grid_sssp(ctx, c3grid):
    _, hw, g, root = c3grid
    ref = oracle.sssp_dijkstra(hw, root)
    for cfg in ("", "Push-Queue-STRICT", "Push-Queue-WM-Fused"):
        d, _ = g.sssp(root, cfg)
        assert np.array_equal(d, ref), cfg
    # the learned level selector and fused/standalone decision
    model, conf = load_model()
    fmodel, fconf = load_fusion_model()
    ctx.mlp_load(model, conf)
    ctx.mlp_load_fusion(fmodel, fconf)
    d, _ = g.sssp(root, gs.RunOpts(selector="mlp"))
    assert np.array_equal(d, ref)
    ctx.mlp_load_fusion(None)
    ctx.mlp_load(None)


def test_c3_grid_bc(ctx, c3grid):
    h, _, g, root = c3grid
    nsp, dep, _ = g.bc(root)
    ref_nsp, _ = oracle.bc_f32(h, root)
    assert np.array_equal(nsp, ref_nsp)
    n64, d64, _ = oracle.bc_f64(h, root)
    overflow = n64 > np.iinfo(np.int32).max
    print(f"BC grid: {int(overflow.sum())} of {h.n} vertices have > 2^31 shortest paths")
    if not overflow.any():
        rel = np.abs(dep.astype(np.float64) - d64) / np.maximum(np.abs(d64), 1.0)
        assert rel.max() <= 1e-5


def _bfs_properties(off, col, lv, root, chunk=1 << 22):
    """Levels are a BFS of the graph: root at 0, every edge joins levels that
    differ by at most one (or two unreached vertices), and every reached
    vertex but the root has a neighbour one level closer."""
    n = len(off) - 1
    assert lv[root] == 0
    has_parent = np.zeros(n, dtype=bool)
    for v0 in range(0, n, chunk):
        v1 = min(n, v0 + chunk)
        a, b = off[v0], off[v1]
        src = np.repeat(np.arange(v0, v1, dtype=np.int64), np.diff(off[v0:v1 + 1]))
        ls, ld = lv[src], lv[col[a:b]]
        assert np.all((ls < 0) == (ld < 0)), "an edge leaves the reached set"
        ok = ls >= 0
        assert np.all(np.abs(ls[ok] - ld[ok]) <= 1)
        par = ok & (ld == ls - 1)
        has_parent[src[par]] = True
    reached = lv >= 0
    reached[root] = False
    assert np.all(has_parent[reached]), "a reached vertex has no neighbour one level closer"


def test_c3_rmat26_bfs_properties(ctx):
    g = ctx.rmat(26, 16, 0.57, 0.19, 0.19, seed=1)
    assert g.m > 2**30  # 2.1 B arcs: row offsets are int64
    model, conf = load_model()
    ctx.mlp_load(model, conf)
    root = int(g.roots(1000, 1)[0])
    lv, st = g.bfs(root, gs.RunOpts(selector="mlp"))
    off, col, _ = g.download()
    _bfs_properties(off, col, lv, root)
    deg = np.diff(off)
    assert st.edges == int(deg[lv >= 0].sum()) // 2
    # a second root through the captured loop: the same properties
    root2 = int(g.roots(1001, 1)[0])
    lv2, _ = g.bfs(root2, gs.RunOpts(selector="mlp", captured=True))
    _bfs_properties(off, col, lv2, root2)
    ctx.mlp_load(None)
    g.close()
