"""GPU parity of the seven applications through the C ABI.

Expected values: the golden vectors produced by the reference's own CPU
validators (tests/golden) and the oracle restatement on larger seeded
graphs.  Integer results (BFS levels, SSSP distances, CC labels, BC path
counts, GC colours, MBFS levels) must match bit for bit under every forced
variant and under the selector.  Tolerances for floating point:
  * PageRank, 20 iterations: L1 distance of the normalised FP32 vector to
    the normalised FP64 oracle <= 1e-6;
  * BC dependencies: |gpu - fp64| / max(|fp64|, 1) <= 1e-5 per vertex.
"""
import itertools

import numpy as np
import pytest

import gswitch_b200 as gs
import oracle
from conftest import golden_names, load_golden

pytestmark = pytest.mark.gpu

DIRS = ["Push", "Pull"]
FMTS = ["Queue", "Bitmap"]
LBS = ["TM", "WM", "CM", "STRICT", "TWC"]
FUS = ["Standalone", "Fused"]
ALL_VARIANTS = ["-".join(v) for v in itertools.product(DIRS, FMTS, LBS, FUS)] + [""]
STANDALONE_VARIANTS = ["-".join(v) for v in itertools.product(DIRS, FMTS, LBS, ["Standalone"])] + [""]


@pytest.fixture(scope="module")
def big():
    """Seeded graphs larger than the fixtures, with oracle answers."""
    out = {}
    for name, g in [("rmat14", oracle.rmat(14, 16, seed=1)), ("grid64", oracle.grid(64, 64, 100, seed=2)),
                    ("er20k", oracle.er(20000, 80000, seed=3))]:
        gw = oracle.add_weights(g, 5, 1000 if name.startswith("grid") else 64)
        root = 0 if name.startswith("rmat") else int(oracle.roots(g, 9, 1)[0])
        out[name] = (g, gw, root)
    return out


@pytest.mark.parametrize("name", golden_names())
def test_bfs_reference_goldens_every_variant(ctx, name):
    d = load_golden(name)
    g = ctx.upload(d["off"], d["col"])
    for cfg in ALL_VARIANTS:
        lv, st = g.bfs(int(d["root"]), cfg)
        assert np.array_equal(lv, d["lvl"]), (name, cfg)
        assert st.device_error == 0


@pytest.mark.parametrize("name", ["rmat14", "grid64", "er20k"])
def test_bfs_large_every_variant(ctx, big, name):
    h, _, root = big[name]
    ref = oracle.bfs(h, root)
    g = ctx.upload(h.off, h.col)
    for cfg in ALL_VARIANTS:
        lv, st = g.bfs(root, gs.RunOpts.from_config(cfg, sorted_queue=(len(cfg) % 2 == 0)))
        assert np.array_equal(lv, ref), (name, cfg)
        assert st.edges == oracle.traversed_edges(h, ref)


@pytest.mark.parametrize("name", golden_names())
def test_sssp_reference_goldens(ctx, name):
    d = load_golden(name)
    g = ctx.upload(d["off"], d["col"], d["w"])
    for cfg in ALL_VARIANTS:
        dist, _ = g.sssp(int(d["root"]), cfg)
        assert np.array_equal(dist, d["dist"]), (name, cfg)


@pytest.mark.parametrize("name", ["rmat14", "grid64", "er20k"])
def test_sssp_large(ctx, big, name):
    _, hw, root = big[name]
    ref = oracle.sssp_dijkstra(hw, root)
    g = ctx.upload(hw.off, hw.col, hw.w)
    for cfg in ["", "Push-Queue-WM", "Push-Queue-STRICT", "Push-Queue-TWC", "Push-Bitmap-CM",
                "Push-Queue-TM-Fused", "Push-Queue-WM-Fused", "Pull-Bitmap-TM", "Pull-Bitmap-WM"]:
        dist, _ = g.sssp(root, cfg)
        assert np.array_equal(dist, ref), (name, cfg)


@pytest.mark.parametrize("name", golden_names())
def test_cc_reference_goldens(ctx, name):
    d = load_golden(name)
    g = ctx.upload(d["off"], d["col"])
    for cfg in ["", "x-Queue", "x-Bitmap"]:
        lab, _ = g.cc(cfg)
        assert np.array_equal(lab, d["cc"]), (name, cfg)


@pytest.mark.parametrize("name", ["rmat14", "grid64", "er20k"])
def test_cc_large(ctx, big, name):
    h, _, _ = big[name]
    g = ctx.upload(h.off, h.col)
    lab, st = g.cc()
    assert np.array_equal(lab, oracle.cc(h))


def _bc_check(nsp, dep, h, root):
    ref_nsp, ref_dep = oracle.bc_f32(h, root)
    _, d64, _ = oracle.bc_f64(h, root)
    assert np.array_equal(nsp, ref_nsp)
    rel = np.abs(dep.astype(np.float64) - d64) / np.maximum(np.abs(d64), 1.0)
    assert rel.max() <= 1e-5, rel.max()


@pytest.mark.parametrize("name", golden_names())
def test_bc_reference_goldens(ctx, name):
    d = load_golden(name)
    h = oracle.Csr(d["off"], d["col"])
    g = ctx.upload(d["off"], d["col"])
    for cfg in ALL_VARIANTS:
        nsp, dep, _ = g.bc(int(d["root"]), cfg)
        assert np.array_equal(nsp, d["bc_nsp"]), (name, cfg)
        _bc_check(nsp, dep, h, int(d["root"]))


@pytest.mark.parametrize("name", ["rmat14", "grid64", "er20k"])
def test_bc_large(ctx, big, name):
    h, _, root = big[name]
    g = ctx.upload(h.off, h.col)
    for cfg in ["", "Push-Queue-WM", "Push-Queue-TWC", "Pull-Bitmap-TM", "Push-Queue-WM-Fused"]:
        nsp, dep, _ = g.bc(root, cfg)
        _bc_check(nsp, dep, h, root)


def _pr_l1(pr_over_od, h, iters=20):
    od = h.degrees().astype(np.float64)
    pr = np.where(od > 0, pr_over_od.astype(np.float64) * od, pr_over_od.astype(np.float64))
    ref = oracle.pagerank(h, iters)
    return np.abs(pr / pr.sum() - ref / ref.sum()).sum(), np.max(np.abs(pr - ref) / ref)


@pytest.mark.parametrize("name", ["rmat10", "grid24_lr", "er1500", "path10", "twocomp_isolated"])
def test_pagerank_20_iterations(ctx, name):
    d = load_golden(name)
    h = oracle.Csr(d["off"], d["col"])
    g = ctx.upload(d["off"], d["col"])
    for cfg in STANDALONE_VARIANTS:
        pr, st = g.pagerank(iters=20, eps=0.0, opts=cfg)
        l1, mrel = _pr_l1(pr, h)
        assert l1 <= 1e-6, (name, cfg, l1, mrel)
        assert st.levels == 20


@pytest.mark.parametrize("name", ["rmat14", "er20k"])
def test_pagerank_large_and_fixpoint(ctx, big, name):
    h, _, _ = big[name]
    g = ctx.upload(h.off, h.col)
    for cfg in ["", "Pull-Bitmap-TM", "Pull-Bitmap-WM", "Push-Bitmap-WM", "Pull-Bitmap-STRICT", "Pull-Bitmap-TWC"]:
        pr, _ = g.pagerank(iters=20, eps=0.0, opts=cfg)
        l1, _ = _pr_l1(pr, h)
        assert l1 <= 1e-6, (cfg, l1)
    # reference termination (per-vertex 1% test) passes the reference's own
    # fix-point validation (application/pagerank.cu:44-79)
    pr, _ = g.pagerank(iters=0, eps=0.01)
    assert oracle.pagerank_check(h, pr) < 0


@pytest.mark.parametrize("name", golden_names())
def test_gc_reference_goldens(ctx, name):
    d = load_golden(name)
    h = oracle.Csr(d["off"], d["col"])
    g = ctx.upload(d["off"], d["col"])
    ref = oracle.gc_levels(h)
    for cfg in STANDALONE_VARIANTS:
        col, _ = g.gc(cfg)
        assert np.array_equal(col, ref), (name, cfg)
        assert oracle.gc_check(h, col) < 0


@pytest.mark.parametrize("name", ["rmat14", "grid64"])
def test_gc_large(ctx, big, name):
    h, _, _ = big[name]
    g = ctx.upload(h.off, h.col)
    col, _ = g.gc()
    assert np.array_equal(col, oracle.gc_levels(h))


@pytest.mark.parametrize("nsrc", [1, 5, 64, 100])
def test_mbfs_batched_and_sequential(ctx, big, nsrc):
    h, _, _ = big["rmat14"]
    g = ctx.upload(h.off, h.col)
    roots = oracle.roots(h, 11, nsrc)
    ref = oracle.mbfs(h, roots)
    lv, st = g.mbfs(roots, batched=True)
    assert np.array_equal(lv, ref)
    assert st.edges == sum(oracle.traversed_edges(h, ref[i]) for i in range(nsrc))
    if nsrc <= 5:
        lv2, _ = g.mbfs(roots, batched=False)
        assert np.array_equal(lv2, ref)


def test_device_generators_match_oracle(ctx):
    for dev, host in [(ctx.rmat(12, 16, seed=1, wmax=64, wseed=11), oracle.add_weights(oracle.rmat(12, 16, seed=1), 11, 64)),
                      (ctx.grid(40, 33, 100, seed=3, wmax=1000, wseed=2),
                       oracle.add_weights(oracle.grid(40, 33, 100, seed=3), 2, 1000)),
                      (ctx.er(3000, 9000, seed=5), oracle.er(3000, 9000, seed=5))]:
        off, col, w = dev.download()
        assert np.array_equal(off, host.off) and np.array_equal(col, host.col)
        if host.w is not None:
            assert np.array_equal(w, host.w)
        # integer-valued sums are exact; the Gini / Hoover terms are summed
        # per degree value on the device side, equal up to rounding
        a, b = dev.attr(), oracle.degree_attr(host)
        assert np.array_equal(a[:4], b[:4])
        assert np.allclose(a[4:], b[4:], rtol=1e-9, atol=1e-12)


def test_errors_are_status_codes(ctx):
    d = load_golden("path10")
    g = ctx.upload(d["off"], d["col"])
    with pytest.raises(gs.GswError) as e:
        g.bfs(10**6)
    assert e.value.code == 1
    with pytest.raises(gs.GswError) as e:
        g.sssp(0)  # no weights
    assert e.value.code == 1
    with pytest.raises(gs.GswError):
        ctx.upload(np.array([0, 5], dtype=np.int64), np.array([0], dtype=np.int32))


def test_upload_rejects_a_bad_csr(ctx):
    """A caller's CSR is checked before any kernel indexes with it: a column
    index outside [0, n) (too large or negative, undirected or directed) and
    offsets that decrease are INVALID_ARG, and the context keeps working."""
    off = np.array([0, 2, 3, 4], dtype=np.int64)
    good = np.array([1, 2, 0, 0], dtype=np.int32)
    for col, directed in (([1, 3, 0, 0], False), ([1, -1, 0, 0], False), ([1, 2, 0, 7], True)):
        with pytest.raises(gs.GswError) as e:
            ctx.upload(off, np.array(col, dtype=np.int32), directed=directed)
        assert e.value.code == 1, (col, directed)
        assert "column" in str(e.value)
    with pytest.raises(gs.GswError) as e:
        ctx.upload(np.array([0, 3, 1, 4], dtype=np.int64), good)
    assert e.value.code == 1 and "offsets" in str(e.value)
    g = ctx.upload(off, good)
    lv, _ = g.bfs(0)
    assert list(lv) == [0, 1, 1]
    g.close()


def test_graphs_without_edges(ctx):
    """One vertex and no arcs, and many vertices and no arcs: every
    application answers for the root (or every vertex) alone."""
    for n in (1, 1000):
        off = np.zeros(n + 1, dtype=np.int64)
        col = np.zeros(0, dtype=np.int32)
        g = ctx.upload(off, col)
        root = n // 2
        ref = np.full(n, -1, dtype=np.int32)
        ref[root] = 0
        for o in (gs.RunOpts(), gs.RunOpts(selector="mlp"), gs.RunOpts(captured=True), "Push-Queue-STRICT-Fused",
                  "Pull-Bitmap-TM-Standalone"):
            lv, st = g.bfs(root, o)
            assert np.array_equal(lv, ref), (n, o)
            assert st.edges == 0
        lab, _ = g.cc()
        assert np.array_equal(lab, np.arange(n))
        col_, _ = g.gc()
        assert oracle.gc_check(oracle.Csr(off, col), col_) < 0
        nsp, dep, _ = g.bc(root)
        assert nsp[root] == 1 and not dep.any()
        lv2, _ = g.mbfs([root, 0], batched=True)
        assert lv2[0][root] == 0 and lv2[1][0] == 0
        gw = ctx.upload(off, col, np.zeros(0, dtype=np.int32))
        d, _ = gw.sssp(root)
        assert d[root] == 0 and (n == 1 or d[(root + 1) % n] > 10**8)
        g.close()
        gw.close()


@pytest.mark.parametrize("persistent", [True, False])
def test_fused_levels_persistent_and_per_launch(ctx, big, persistent):
    """Fused levels run either in one grid-wide launch with a level barrier or
    one launch per level; both give the oracle's results, including the
    high-diameter grid (pruning BFS: one barrier per level; SSSP: visited bits
    cleared between levels, two barriers per level)."""
    for name in ["grid64", "rmat14", "er20k"]:
        h, hw, root = big[name]
        g = ctx.upload(h.off, h.col)
        gw = ctx.upload(hw.off, hw.col, hw.w)
        for lb in ["WM", "TM", "CM", "STRICT", "TWC"]:
            lv, st = g.bfs(root, gs.RunOpts.from_config(f"Push-Queue-{lb}-Fused", persistent=persistent))
            assert np.array_equal(lv, oracle.bfs(h, root)), (name, lb, persistent)
            assert st.levels == int(lv.max()) + 1 or st.levels == int(lv.max()) + 2
            check_fused_kernels(st, lb, persistent)
            dist, st = gw.sssp(root, gs.RunOpts.from_config(f"Push-Queue-{lb}-Fused", persistent=persistent))
            assert np.array_equal(dist, oracle.sssp_dijkstra(hw, root)), (name, lb, persistent)
            check_fused_kernels(st, lb, persistent)


def check_fused_kernels(st, lb, persistent):
    """Every fused level ran the forced load balance; in persistent mode the
    LB is the one the launched kernel reported back, so a kernel that ran
    another LB's body shows up here."""
    fused = [(t, p) for t, p in zip(st.trace, st.level_persistent) if t[3] == "Fused"]
    assert fused
    for t, p in fused:
        assert t[2] == lb, (t, lb)
        assert p == persistent, (t, p, persistent)


def test_path_graph_many_levels_persistent(ctx):
    h = oracle.csr_from_pairs(5000, np.arange(4999), np.arange(1, 5000))
    g = ctx.upload(h.off, h.col)
    lv, st = g.bfs(0, gs.RunOpts.from_config("Push-Queue-WM-Fused", persistent=True))
    assert np.array_equal(lv, np.arange(5000))
    lv, st = g.bfs(2500)
    assert np.array_equal(lv, np.abs(np.arange(5000) - 2500))


def test_level_barrier_timeout_is_reported_and_context_survives(ctx):
    """Failure path of the grid-wide level barrier: one block leaves without
    arriving, the others' bounded wait expires, the call returns TIMEOUT, and
    the same context then runs normally."""
    h = oracle.grid(40, 40, 100, seed=2)
    g = ctx.upload(h.off, h.col)
    with pytest.raises(gs.GswError) as e:
        g.bfs(0, gs.RunOpts.from_config("Push-Queue-WM-Fused", persistent=True, barrier_test=True))
    assert e.value.code == 4
    lv, _ = g.bfs(0, gs.RunOpts.from_config("Push-Queue-WM-Fused", persistent=True))
    assert np.array_equal(lv, oracle.bfs(h, 0))


@pytest.mark.parametrize("name", ["rmat14", "grid64", "er20k"])
def test_twod_partition_pagerank_and_gc(ctx, big, name):
    """2D-partition expand (heavy tile pairs staged in shared memory, light
    edges gathered): PageRank within the FP32 tolerance, GC colours exact."""
    h, _, _ = big[name]
    g = ctx.upload(h.off, h.col)
    pr, st = g.pagerank(iters=20, eps=0.0, opts="x-x-TWOD")
    l1, _ = _pr_l1(pr, h)
    assert l1 <= 1e-6, l1
    assert st.levels == 20
    col, _ = g.gc("x-x-TWOD")
    assert np.array_equal(col, oracle.gc_levels(h))


def test_twod_heavy_blocks_on_dense_tiles(ctx):
    """A graph dense enough that (tile, tile) pairs reach the heavy threshold."""
    h = oracle.er(6000, 6000 * 900, seed=8)
    g = ctx.upload(h.off, h.col)
    pr, _ = g.pagerank(iters=20, eps=0.0, opts="x-x-TWOD")
    l1, _ = _pr_l1(pr, h)
    assert l1 <= 1e-6, l1


@pytest.mark.parametrize("name", ["rmat14", "grid64", "er20k"])
def test_inspection_counters_match_reference_definition(ctx, big, name):
    """The six counters of one inspection, including the reference's
    per-block sums of per-thread maximum degrees (inspector.cuh:39-110), for
    every level of a BFS and for random states, against the oracle."""
    h, _, root = big[name]
    g = ctx.upload(h.off, h.col)
    lv = oracle.bfs(h, root)
    for level in range(0, int(lv.max()) + 2):
        assert np.array_equal(g.bfs_inspect(lv, level), oracle.inspect_bfs(h, lv, level)), (name, level)
    rng = np.random.default_rng(4)
    for _ in range(3):
        st = rng.integers(-1, 3, h.n).astype(np.int32)
        assert np.array_equal(g.bfs_inspect(st, 1), oracle.inspect_bfs(h, st, 1))


def test_inspection_counters_on_multi_step_sizes(ctx):
    """Sizes where every virtual thread takes several steps (both halves of a
    CTA, a ragged last word): RMAT 2^19 and G(n, m) with n = 700,001."""
    for h in (oracle.rmat(19, 8, seed=3), oracle.er(700001, 2000000, seed=5)):
        g = ctx.upload(h.off, h.col)
        root = int(oracle.roots(h, 2, 1)[0])
        lv = oracle.bfs(h, root)
        for level in (0, 1, 2, 3, 5):
            assert np.array_equal(g.bfs_inspect(lv, level), oracle.inspect_bfs(h, lv, level)), (h.n, level)
        g.close()


def test_graph_blocks_reused_across_uploads(ctx, big):
    """Destroyed graphs hand their device blocks to the next upload of a
    fitting size; stale contents of a reused block must not leak into the
    next graph's results."""
    h, hw, root = big["rmat14"]
    ref = oracle.bfs(h, root)
    for _ in range(3):
        g = ctx.upload(h.off, h.col)
        lv, _ = g.bfs(root)
        assert np.array_equal(lv, ref)
        g.close()
    # a slightly smaller graph reuses the larger one's blocks (within a quarter)
    sub = oracle.er(h.n - 100, int(h.m // 2 * 0.9), seed=11)
    r2 = int(oracle.roots(sub, 4, 1)[0])
    g = ctx.upload(sub.off, sub.col)
    lv, _ = g.bfs(r2)
    assert np.array_equal(lv, oracle.bfs(sub, r2))
    d, _ = ctx.upload(hw.off, hw.col, hw.w).sssp(root)
    assert np.array_equal(d, oracle.sssp_dijkstra(hw, root))
    g.close()


@pytest.mark.parametrize("hub_path", [gs.HUB_SCALAR, gs.HUB_VECTOR, gs.HUB_STAGED])
def test_hub_paths_of_the_tiered_push(ctx, big, hub_path):
    """The CTA tier of the tiered push reads a hub's columns with 4-byte
    loads, int4 loads of the aligned body, or shared-memory chunks filled by
    TMA bulk copies (ragged ends with plain loads): BFS and SSSP stay exact,
    standalone, per-launch fused and persistent fused, on graphs whose hubs
    span many chunks (RMAT 2^14 ef 16 and a denser G(n, m) with lists of
    every alignment)."""
    graphs = [big["rmat14"], (oracle.er(3000, 3000 * 400, seed=6), None, 7)]
    for h, hw, root in graphs:
        hw = hw if hw is not None else oracle.add_weights(h, 5, 64)
        g = ctx.upload(h.off, h.col)
        gw = ctx.upload(hw.off, hw.col, hw.w)
        ref, dref = oracle.bfs(h, root), oracle.sssp_dijkstra(hw, root)
        for cfg, persistent in (("Push-Queue-TWC-Standalone", None), ("Push-Queue-TWC-Fused", False),
                                ("Push-Queue-TWC-Fused", True), ("Push-Bitmap-TWC-Standalone", None)):
            o = gs.RunOpts.from_config(cfg, persistent=persistent, hub_path=hub_path)
            lv, st = g.bfs(root, o)
            assert np.array_equal(lv, ref), (cfg, persistent, hub_path)
            assert st.device_error == 0
            d, st = gw.sssp(root, o)
            assert np.array_equal(d, dref), (cfg, persistent, hub_path)
            assert st.device_error == 0
        g.close()
        gw.close()


def hub_frontier_graph():
    """Vertex 0 joined to six hubs whose lists hold 256 (the smallest hub),
    8,191, 8,192, 8,193, 30,001 and 70,000 leaves (pieces of 8,192 columns
    with ragged ends, lists at every alignment); the hubs share some leaves
    and a chain hangs off the last leaf, so level 2 is the six hubs alone."""
    degs = [256, 8191, 8192, 8193, 30001, 70000]
    src, dst, nxt = [], [], 7
    for i, d in enumerate(degs, start=1):
        src.append(0)
        dst.append(i)
        leaves = np.arange(nxt, nxt + d)
        src += [i] * d
        dst += list(leaves)
        nxt += d // 2  # half of each list is shared with the next hub
    n = int(leaves[-1]) + 41
    chain = np.arange(int(leaves[-1]), n - 1)
    src += list(chain)
    dst += list(chain + 1)
    return oracle.csr_from_pairs(n, np.array(src), np.array(dst))


@pytest.mark.parametrize("hub_path", [gs.HUB_SCALAR, gs.HUB_VECTOR, gs.HUB_STAGED])
def test_tiered_push_hub_list_spreads_a_hub_frontier(ctx, hub_path):
    """A per-launch tiered push lists the frontier's hubs in pieces of at most
    8,192 columns and a second kernel sweeps one piece per CTA: on a level
    that is six hubs, BFS and SSSP stay exact, every edge is counted once,
    and the persistent form (hubs swept in their tile) agrees."""
    h = hub_frontier_graph()
    hw = oracle.add_weights(h, 3, 64)
    ref, dref = oracle.bfs(h, 0), oracle.sssp_dijkstra(hw, 0)
    per_level = [int(x) for x in np.bincount(ref[ref >= 0], weights=h.degrees()[ref >= 0])]
    g, gw = ctx.upload(h.off, h.col), ctx.upload(hw.off, hw.col, hw.w)
    for cfg, persistent in (("Push-Queue-TWC-Standalone", None), ("Push-Queue-TWC-Fused", False),
                            ("Push-Queue-TWC-Fused", True), ("Push-Bitmap-TWC-Standalone", None)):
        o = gs.RunOpts.from_config(cfg, persistent=persistent, hub_path=hub_path, account=True)
        for _ in range(2):  # the list's count is back at 0 for the next run
            lv, st = g.bfs(0, o)
            assert np.array_equal(lv, ref), (cfg, persistent)
            assert st.device_error == 0
            if cfg == "Push-Queue-TWC-Standalone":  # the queue's size (fused levels do not count it)
                assert st.trace[1][-1] == 6  # level 2: the hubs
            if persistent is not True:  # the hubs' level and the next: every arc examined once
                assert st.level_edges[1:3] == per_level[1:3], (cfg, persistent, st.level_edges[:3])
        d, st = gw.sssp(0, o)
        assert np.array_equal(d, dref), (cfg, persistent)
        assert st.device_error == 0
    g.close()
    gw.close()


@pytest.mark.parametrize("name,nsrc", [("rmat14", 1), ("rmat14", 32), ("rmat14", 45), ("grid64", 40), ("er20k", 33)])
def test_bc_batch_every_source(ctx, big, name, nsrc):
    """Batched BC (bit-sliced levels, then per-level forward / backward passes
    over a batch of up to 32 sources): per source, path counts equal the
    reference's int32 counts bit for bit and dependencies are within 1e-5 of
    the FP64 oracle, for one source, a full batch, and batches with a
    partial tail; hubs of RMAT spread over many adjacency chunks."""
    h, _, _ = big[name]
    g = ctx.upload(h.off, h.col)
    roots = oracle.roots(h, 23, nsrc)
    nsp, dep, st = g.bc_batch(roots)
    assert nsp.shape == (nsrc, h.n) and dep.shape == (nsrc, h.n)
    edges = 0
    for i, r in enumerate(roots):
        _bc_check(nsp[i], dep[i], h, int(r))
        edges += oracle.traversed_edges(h, oracle.bfs(h, int(r)))
    assert st.edges == edges
    g.close()


def test_bc_batch_matches_single_source_runs(ctx, big):
    h, _, _ = big["rmat14"]
    g = ctx.upload(h.off, h.col)
    roots = oracle.roots(h, 29, 8)
    nsp, dep, _ = g.bc_batch(roots)
    for i, r in enumerate(roots):
        n1, d1, _ = g.bc(int(r))
        assert np.array_equal(nsp[i], n1)
        assert np.allclose(dep[i], d1, rtol=1e-5, atol=1e-5)
    g.close()


@pytest.mark.parametrize("persistent", [True, False])
def test_batched_sources_persistent_and_per_level(ctx, big, persistent):
    """Batched MBFS and batched BC give the same answers whether all levels
    run in one cooperative launch (grid barriers, direction chosen on the
    device) or one launch per level / pass."""
    h, _, _ = big["rmat14"]
    g = ctx.upload(h.off, h.col)
    roots = oracle.roots(h, 31, 70)
    lv, _ = g.mbfs(roots, batched=True, opts=gs.RunOpts(persistent=persistent))
    assert np.array_equal(lv, oracle.mbfs(h, roots))
    nsp, dep, _ = g.bc_batch(roots[:40], opts=gs.RunOpts(persistent=persistent))
    for i, r in enumerate(roots[:40]):
        _bc_check(nsp[i], dep[i], h, int(r))
    g.close()


@pytest.mark.parametrize("selector", ["rules", "mlp"])
def test_select_entry_point_reproduces_the_loop_choices(ctx, big, selector):
    """gsw_select, given one level's inspection counters and the graph's
    degree statistics, picks the standalone variant the BFS loop itself
    picked at that level (standalone levels forced, so no fusion history)."""
    from gswitch_b200.selector_train import load_model

    if selector == "mlp":
        model, conf = load_model()
        ctx.mlp_load(model, conf)
        saved, c2 = ctx.mlp_save()
        assert np.array_equal(saved, model) and c2 == pytest.approx(conf)
    try:
        for name in ("rmat14", "grid64", "er20k"):
            h, _, root = big[name]
            g = ctx.upload(h.off, h.col)
            lv = oracle.bfs(h, root)
            _, st = g.bfs(root, gs.RunOpts(fusion=gs.STANDALONE, selector=selector))
            attr = g.attr()
            for i, t in enumerate(st.trace):
                s = gs.LevelStats()
                s.nvertexs, s.nedges = h.n, h.m
                for k in range(6):
                    s.attr[k] = attr[k]
                s.pattern, s.level = 0, i
                if i == 0:
                    s.first_level, s.active, s.root_degree = 1, 1, int(h.degrees()[root])
                else:
                    state = np.where((lv >= 0) & (lv <= i), lv, -1).astype(np.int32)
                    c = g.bfs_inspect(state, i)
                    (s.active, s.inactive, s.push_workload, s.pull_workload, s.max_push,
                     s.max_pull) = (int(x) for x in c)
                choice, done = ctx.select(s, selector)
                assert not done
                assert choice == tuple(t[:3]), (name, i, choice, t)
            g.close()
    finally:
        ctx.mlp_load(None)
