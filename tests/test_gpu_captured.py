"""Captured level loop: the whole inspect -> select -> filter -> expand loop
as one CUDA graph with device-side selection and termination.

Results must be bit-exact with the oracle (BFS) or within the PageRank
tolerance (L1 of normalised vectors <= 1e-6 after 20 iterations), and the
device selector must take the host selector's decisions level for level."""
import numpy as np
import pytest

import gswitch_b200 as gs
import oracle
from conftest import golden_names, load_golden
from test_gpu_apps import ALL_VARIANTS, STANDALONE_VARIANTS, _pr_l1

pytestmark = pytest.mark.gpu


def cap(cfg="", **kw):
    return gs.RunOpts.from_config(cfg, captured=True, **kw)


@pytest.fixture(scope="module")
def graphs():
    out = {}
    for name, g in [("rmat14", oracle.rmat(14, 16, seed=1)), ("grid64", oracle.grid(64, 64, 100, seed=2)),
                    ("er20k", oracle.er(20000, 80000, seed=3))]:
        root = 0 if name.startswith("rmat") else int(oracle.roots(g, 9, 1)[0])
        out[name] = (g, root)
    return out


@pytest.mark.parametrize("name", golden_names())
def test_captured_bfs_goldens_every_variant(ctx, name):
    d = load_golden(name)
    g = ctx.upload(d["off"], d["col"])
    for cfg in ALL_VARIANTS:
        lv, st = g.bfs(int(d["root"]), cap(cfg))
        assert np.array_equal(lv, d["lvl"]), (name, cfg)
        assert st.device_error == 0
        # one trace entry per level, except that a persistent launch of
        # fused levels is one entry for all the levels it ran
        if any(st.level_persistent):
            assert st.levels >= len(st.trace)
        else:
            assert st.levels == len(st.trace)
        _, host = g.bfs(int(d["root"]), gs.RunOpts.from_config(cfg))
        assert st.levels == host.levels, (name, cfg)


@pytest.mark.parametrize("name", ["rmat14", "grid64", "er20k"])
def test_captured_bfs_large(ctx, graphs, name):
    h, root = graphs[name]
    ref = oracle.bfs(h, root)
    g = ctx.upload(h.off, h.col)
    for cfg in ALL_VARIANTS:
        lv, st = g.bfs(root, cap(cfg, sorted_queue=(len(cfg) % 2 == 0)))
        assert np.array_equal(lv, ref), (name, cfg)
        assert st.edges == oracle.traversed_edges(h, ref)


@pytest.mark.parametrize("name", ["rmat14", "grid64", "er20k"])
def test_captured_selector_takes_host_decisions(ctx, graphs, name):
    """Standalone levels: same variant and frontier size at every level as
    the host-driven loop (forced standalone keeps the host loop's
    wall-clock fusion rule out of the comparison)."""
    h, root = graphs[name]
    g = ctx.upload(h.off, h.col)
    for cfg in ["x-x-x-Standalone", "Push-x-x-Standalone", "Pull-x-x-Standalone", "x-Queue-x-Standalone"]:
        _, host = g.bfs(root, gs.RunOpts.from_config(cfg, persistent=False))
        _, dev = g.bfs(root, cap(cfg))
        assert dev.trace == host.trace, (name, cfg)
        assert dev.levels == host.levels


@pytest.mark.parametrize("name", ["rmat14", "er20k", "grid64"])
def test_captured_persistent_fused_levels(ctx, graphs, name):
    """Fused levels of the captured loop run as the host loop's persistent
    launch (the cooperative multi-level kernel inside the graph): exact
    results, the same levels and variants as the host loop, the persistent
    entries reporting the load balance the kernel ran, and per-launch fused
    levels when persistent launches are off."""
    h, root = graphs[name]
    g = ctx.upload(h.off, h.col)
    ref = oracle.bfs(h, root)
    for cfg in ["", "Push-Queue-WM-Fused", "Push-Queue-STRICT-Fused", "Push-Queue-TWC-Fused", "Push-Queue-CM-Fused"]:
        _, host = g.bfs(root, gs.RunOpts.from_config(cfg))
        for _ in range(2):
            lv, st = g.bfs(root, cap(cfg))
            assert np.array_equal(lv, ref), (name, cfg)
            assert st.device_error == 0
            assert st.levels == host.levels, (name, cfg, st.levels, host.levels)
            assert [t[:4] for t in st.trace] == [t[:4] for t in host.trace], (name, cfg)
            assert st.level_persistent == host.level_persistent, (name, cfg)
        if cfg:
            assert any(st.level_persistent), (name, cfg)
        lv, st = g.bfs(root, cap(cfg, persistent=False))
        assert np.array_equal(lv, ref), (name, cfg)
        assert not any(st.level_persistent)


def test_captured_graph_reused_across_roots_and_rebuilt_per_graph(ctx, graphs):
    for name in ["rmat14", "er20k"]:
        h, _ = graphs[name]
        g = ctx.upload(h.off, h.col)
        for r in oracle.roots(h, 11, 4):
            lv, _ = g.bfs(int(r), cap())
            assert np.array_equal(lv, oracle.bfs(h, int(r))), (name, r)


def test_captured_bfs_accounting_matches_host(ctx, graphs):
    h, root = graphs["rmat14"]
    g = ctx.upload(h.off, h.col)
    cfg = "Push-Queue-WM-Standalone"
    _, host = g.bfs(root, gs.RunOpts.from_config(cfg, account=True, persistent=False))
    _, dev = g.bfs(root, cap(cfg, account=True))
    assert dev.level_edges == host.level_edges
    assert sum(dev.level_edges) > 0


@pytest.mark.parametrize("name", ["rmat10", "grid24_lr", "er1500", "path10", "twocomp_isolated"])
def test_captured_pagerank_20_iterations(ctx, name):
    d = load_golden(name)
    h = oracle.Csr(d["off"], d["col"])
    g = ctx.upload(d["off"], d["col"])
    for cfg in STANDALONE_VARIANTS + ["x-x-TWOD"]:
        pr, st = g.pagerank(iters=20, eps=0.0, opts=cap(cfg))
        l1, mrel = _pr_l1(pr, h)
        assert l1 <= 1e-6, (name, cfg, l1, mrel)
        assert st.levels == 20


def test_captured_pagerank_fixpoint(ctx, graphs):
    h, _ = graphs["rmat14"]
    g = ctx.upload(h.off, h.col)
    pr, st = g.pagerank(iters=0, eps=0.01, opts=cap())
    assert oracle.pagerank_check(h, pr) < 0
    assert st.levels > 1


@pytest.mark.parametrize("name", golden_names())
def test_captured_cc_goldens(ctx, name):
    """Captured CC (edge-centric inspection, on-device stop and format
    choice, hooking and pointer jumping in one graph): the reference's labels."""
    d = load_golden(name)
    g = ctx.upload(d["off"], d["col"])
    lab, st = g.cc(cap())
    assert np.array_equal(lab, d["cc"])
    assert st.device_error == 0


@pytest.mark.parametrize("name", ["rmat14", "grid64", "er20k"])
def test_captured_cc_large(ctx, graphs, name):
    h, _ = graphs[name]
    g = ctx.upload(h.off, h.col)
    ref = oracle.cc(h)
    lab_h, st_h = g.cc()
    # hooking races (atomicMin from many edges), so the number of rounds may
    # differ from run to run; the labels may not
    for _ in range(2):  # the second run reuses the cached graph
        lab, st = g.cc(cap())
        assert np.array_equal(lab, ref)
        assert st.levels >= 1 and st.device_error == 0
        assert st.trace[0][1] == "Bitmap"  # every edge active at the first level: the bitmap form
    assert np.array_equal(lab_h, ref)


@pytest.mark.parametrize("name", golden_names())
def test_captured_sssp_goldens(ctx, name):
    """Captured SSSP: the stepping window lives in device memory, the exit
    probe runs inside the graph when a level finds no input, and the loop
    restarts on the next window until no value lies outside it: the
    reference's distances, standalone and fused levels."""
    d = load_golden(name)
    g = ctx.upload(d["off"], d["col"], d["w"])
    for cfg in ["", "Push-Queue-WM-Standalone", "Push-Queue-WM-Fused", "Push-Queue-STRICT-Fused", "Pull-Bitmap-TM"]:
        dist, st = g.sssp(int(d["root"]), cap(cfg))
        assert np.array_equal(dist, d["dist"]), (name, cfg)
        assert st.device_error == 0


@pytest.mark.parametrize("name", ["rmat14", "grid64", "er20k"])
def test_captured_sssp_large(ctx, graphs, name):
    h, root = graphs[name]
    hw = oracle.add_weights(h, 5, 1000 if name.startswith("grid") else 64)
    g = ctx.upload(hw.off, hw.col, hw.w)
    ref = oracle.sssp_dijkstra(hw, root)
    from gswitch_b200.selector_train import load_fusion_model, load_model
    model, conf = load_model()
    ctx.mlp_load(model, conf)
    fm, fc = load_fusion_model()
    ctx.mlp_load_fusion(fm, fc)
    try:
        for o in (cap(), cap(selector="mlp"), cap("Push-Queue-TWC-Fused"), cap("Push-Bitmap-CM-Standalone")):
            for _ in range(2):  # the second run reuses the cached graph
                dist, st = g.sssp(root, o)
                assert np.array_equal(dist, ref), (name, vars(o))
                assert st.device_error == 0
    finally:
        ctx.mlp_load_fusion(None)
        ctx.mlp_load(None)


@pytest.mark.parametrize("name", golden_names())
def test_captured_gc_goldens(ctx, name):
    """Graph colouring through the captured loop (rule trees on the device):
    the reference's level colouring bit for bit, the host loop's levels."""
    d = load_golden(name)
    h = oracle.Csr(d["off"], d["col"])
    g = ctx.upload(d["off"], d["col"])
    ref = oracle.gc_levels(h)
    for cfg in ["", "Push-Queue-WM-Standalone", "Pull-Bitmap-TM-Standalone", "Push-Bitmap-STRICT-Standalone"]:
        _, host = g.gc(gs.RunOpts.from_config(cfg))
        for _ in range(2):  # the second run reuses the cached graph
            col, st = g.gc(cap(cfg))
            assert np.array_equal(col, ref), (name, cfg)
            assert oracle.gc_check(h, col) < 0
            assert st.levels == host.levels, (name, cfg)


def test_captured_gc_large(ctx, graphs):
    for name in ("rmat14", "grid64"):
        h, _ = graphs[name]
        g = ctx.upload(h.off, h.col)
        col, st = g.gc(cap())
        assert np.array_equal(col, oracle.gc_levels(h)), name
        assert st.device_error == 0


@pytest.mark.parametrize("name", ["rmat10", "grid24_lr", "er1500", "path10", "twocomp_isolated"])
def test_captured_delta_pagerank(ctx, name):
    """Delta-PageRank through the captured loop: the oracle's fixed point
    within the delta tolerance, the host loop's values, level count and work
    up to the order of FP32 atomic sums (which moves a vertex across its
    activation threshold now and then); an iteration cap stops both loops at
    the same level."""
    d = load_golden(name)
    h = oracle.Csr(d["off"], d["col"])
    ref = oracle.pagerank(h, 400, 0.85)
    g = ctx.upload(d["off"], d["col"])
    for cfg in ["", "Push-Queue-WM-Standalone", "Pull-Bitmap-TM-Standalone"]:
        hp, hst = g.pagerank_delta(eps=1e-5, max_levels=2000, opts=cfg)
        for _ in range(2):
            pr, st = g.pagerank_delta(eps=1e-5, max_levels=2000, opts=cap(cfg))
            l1 = np.abs(pr / pr.sum() - ref / ref.sum()).sum()
            assert l1 <= 1e-5 / 0.15 + 1e-5, (name, cfg, l1)
            assert np.allclose(pr, hp, rtol=5e-4, atol=1e-6), (name, cfg)
            assert abs(st.levels - hst.levels) <= 1, (name, cfg, st.levels, hst.levels)
            assert st.edges > 0 and "Fused" not in {t[3] for t in st.trace}
        _, c5 = g.pagerank_delta(eps=1e-5, max_levels=5, opts=cap(cfg))
        _, h5 = g.pagerank_delta(eps=1e-5, max_levels=5, opts=cfg)
        assert c5.levels == h5.levels == 5, (name, cfg, c5.levels, h5.levels)
        assert abs(c5.edges - h5.edges) <= 0.01 * h5.edges, (name, cfg, c5.edges, h5.edges)


def test_captured_rejected_where_unsupported(ctx, graphs):
    h, root = graphs["er20k"]
    g = ctx.upload(h.off, h.col)
    with pytest.raises(gs.GswError) as e:
        g.bc(root, cap())
    assert gs.STATUS[e.value.code] == "UNSUPPORTED"


# ---------------------------------------------------------------------------
# batched instances: a batch of G(n, m) graphs as one disjoint union, every
# instance's BFS in one level loop (host-driven, captured) and CC over all
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def er_batch(ctx):
    g, voff = ctx.er_batch(48, seed=21, nlo=500, nhi=20000, dlo=4.0, dhi=32.0)
    parts = oracle.er_batch(21, 48, nlo=500, nhi=20000, dlo=4.0, dhi=32.0)
    yield g, voff, parts
    g.close()


def test_er_batch_union_matches_instances(er_batch):
    g, voff, parts = er_batch
    off, col, _ = g.download()
    assert len(voff) == len(parts) + 1 and voff[-1] == g.n
    for i, h in enumerate(parts):
        a, b = voff[i], voff[i + 1]
        assert b - a == h.n
        seg = off[a:b + 1] - off[a]
        assert np.array_equal(seg, h.off), i
        assert np.array_equal(col[off[a]:off[b]] - a, h.col), i


@pytest.mark.parametrize("opts", [dict(), dict(selector="mlp"), dict(captured=True), dict(persistent=False),
                                  dict(fusion=1)])
def test_er_batch_bfs_every_instance_in_one_loop(ctx, er_batch, opts):
    g, voff, parts = er_batch
    if opts.get("selector") == "mlp":
        from gswitch_b200.selector_train import load_model
        model, conf = load_model()
        ctx.mlp_load(model, conf)
    roots = [int(voff[i] + oracle.roots(h, 5 + i, 1)[0]) for i, h in enumerate(parts)]
    lv, st = g.bfs_multi(roots, gs.RunOpts(**opts))
    for i, h in enumerate(parts):
        ref = oracle.bfs(h, roots[i] - int(voff[i]))
        assert np.array_equal(lv[voff[i]:voff[i + 1]], ref), (i, opts)
    assert st.edges == sum(oracle.traversed_edges(h, oracle.bfs(h, roots[i] - int(voff[i])))
                           for i, h in enumerate(parts))
    ctx.mlp_load(None)


def test_er_batch_cc_labels_per_instance(er_batch):
    g, voff, parts = er_batch
    lab, _ = g.cc()
    for i, h in enumerate(parts):
        assert np.array_equal(lab[voff[i]:voff[i + 1]] - voff[i], oracle.cc(h)), i
