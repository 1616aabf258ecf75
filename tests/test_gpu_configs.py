"""Parity at the configurations the bench measures: the same graphs, roots,
weights, iteration counts and batch seeds as its lines, checked against the
oracle.

  C1  BFS on RMAT scale 16 ef 16 seed 1 from vertex 0: every variant, the
      learned selector and the captured loop, bit-exact.
  C2  RMAT scale 24 ef 16 seed 1 (16.8 M vertices, 521 M arcs), the headline
      graph: BFS from the bench's first timed roots (switched forms, and every
      fixed variant from one root), SSSP on the weighted copy (weights
      U[1, 64], seed 2) from the bench's SSSP root, CC, and 20 PageRank
      iterations in FP32 against the FP64 oracle: the L1 distance of the
      normalised vectors must be <= 1e-6 under x-x-TWOD, Pull-Bitmap-STRICT
      and the selectors; the max relative error is reported beside it.
  C4  256-source batched BFS on RMAT scale 22 (the bench's sources), every
      source exact; the 512-instance G(n, m) batch (the bench's seed): one
      BFS per instance in one level loop (host-driven and captured) and CC
      over the union, exact per instance.

The device builds each graph with its own generator; the tests first check
that it equals the oracle's, then compare results.  The oracle runs on host
threads while the GPU works (ctypes releases the GIL).  With
GSW_PARITY_REPORT=<file>, each PageRank case appends its errors there as a
JSON line."""
import json
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import gswitch_b200 as gs
import oracle
from gswitch_b200.autotune import load_into
from gswitch_b200.selector_train import load_fusion_model, load_model
from test_gpu_apps import ALL_VARIANTS

pytestmark = pytest.mark.gpu

POOL = ThreadPoolExecutor(max_workers=max(4, os.cpu_count() or 4))
BENCH_ROOT_SEED = 1000   # bench.py: roots = g.roots(1000 + rank, W + K)
PR_TOL = 1e-6


def report(**kw):
    path = os.environ.get("GSW_PARITY_REPORT")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(kw) + "\n")


@pytest.fixture(scope="module")
def bctx():
    """A context set up as the bench sets it up: tuned grids and shapes, the learned
    selector and the fusion network loaded."""
    c = gs.Context(0)
    load_into(c)
    model, conf = load_model()
    if model is not None:
        c.mlp_load(model, conf)
    fmodel, fconf = load_fusion_model()
    if fmodel is not None:
        c.mlp_load_fusion(fmodel, fconf)
    yield c
    c.close()


def same_graph(dev, host):
    off, col, w = dev.download()
    assert np.array_equal(off, host.off)
    assert np.array_equal(col, host.col)
    if host.w is not None:
        assert np.array_equal(w, host.w)


def pr_errors(pr_over_od, h, ref):
    od = h.degrees().astype(np.float64)
    pr = np.where(od > 0, pr_over_od.astype(np.float64) * od, pr_over_od.astype(np.float64))
    return float(np.abs(pr / pr.sum() - ref / ref.sum()).sum()), float(np.max(np.abs(pr - ref) / ref))


# ---------------------------------------------------------------------------
# C1
# ---------------------------------------------------------------------------
def test_c1_bfs_rmat16_root0_every_variant(bctx):
    h = oracle.rmat(16, 16, seed=1)
    g = bctx.rmat(16, 16, seed=1)
    same_graph(g, h)
    ref = oracle.bfs(h, 0)
    for cfg in ALL_VARIANTS:
        lv, st = g.bfs(0, cfg)
        assert np.array_equal(lv, ref), cfg
        assert st.device_error == 0
    for o in (gs.RunOpts(selector="mlp"), gs.RunOpts(captured=True), gs.RunOpts(selector="mlp", captured=True),
              gs.RunOpts(persistent=False)):
        lv, st = g.bfs(0, o)
        assert np.array_equal(lv, ref), vars(o)
    assert st.edges == oracle.traversed_edges(h, ref)
    g.close()


# ---------------------------------------------------------------------------
# C2: the headline graph
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def c2(bctx):
    h = oracle.rmat(24, 16, seed=1)
    g = bctx.rmat(24, 16, seed=1)
    same_graph(g, h)
    roots = [int(r) for r in oracle.roots(h, BENCH_ROOT_SEED, 8)]
    assert np.array_equal(g.roots(BENCH_ROOT_SEED, 8), roots)
    # the bench's timed roots start after its warm-up roots (3 by default)
    timed = roots[3:8]
    hw = oracle.add_weights(h, 2, 64)
    jobs = {("bfs", r): POOL.submit(oracle.bfs, h, r) for r in timed}
    jobs["cc"] = POOL.submit(oracle.cc_linear, h)
    jobs["pr"] = POOL.submit(oracle.pagerank, h, 20)
    jobs["sssp"] = POOL.submit(oracle.sssp_dial, hw, timed[0], 64)
    yield dict(h=h, hw=hw, g=g, timed=timed, jobs=jobs)
    g.close()


def test_c2_bfs_switched_forms_from_the_bench_roots(c2):
    g, h = c2["g"], c2["h"]
    for r in c2["timed"]:
        ref = c2["jobs"][("bfs", r)].result()
        for o in (gs.RunOpts(selector="mlp"), gs.RunOpts(), gs.RunOpts(selector="mlp", captured=True)):
            lv, st = g.bfs(r, o)
            assert np.array_equal(lv, ref), (r, vars(o))
            assert st.device_error == 0
        assert st.edges == oracle.traversed_edges(h, ref)


def test_c2_bfs_every_fixed_variant(c2):
    g, r = c2["g"], c2["timed"][0]
    ref = c2["jobs"][("bfs", r)].result()
    for cfg in ALL_VARIANTS:
        lv, _ = g.bfs(r, cfg)
        assert np.array_equal(lv, ref), cfg


def test_c2_sssp_weights_1_64(c2, bctx):
    gw = bctx.rmat(24, 16, seed=1, wmax=64, wseed=2)
    same_graph(gw, c2["hw"])
    r = c2["timed"][0]
    ref = c2["jobs"]["sssp"].result()
    cfgs = [gs.RunOpts(selector="mlp"), gs.RunOpts()] + [gs.RunOpts.from_config(c) for c in (
        "Push-Queue-STRICT-Standalone", "Push-Queue-WM-Standalone", "Push-Bitmap-TWC-Standalone",
        "Pull-Bitmap-TM-Standalone", "Push-Queue-WM-Fused", "Push-Queue-STRICT-Fused", "Push-Queue-TM-Fused")]
    for o in cfgs:
        dist, st = gw.sssp(r, o)
        assert np.array_equal(dist, ref), vars(o)
        assert st.device_error == 0
    gw.close()


def test_c2_cc(c2):
    ref = c2["jobs"]["cc"].result()
    for cfg in ("", "x-Queue", "x-Bitmap"):
        lab, st = c2["g"].cc(cfg)
        assert np.array_equal(lab, ref), cfg
        assert st.device_error == 0


@pytest.mark.parametrize("cfg", ["x-x-TWOD", "Pull-Bitmap-STRICT", "rules", "mlp", "Pull-Bitmap-TM",
                                 "Push-Bitmap-WM"])
def test_c2_pagerank_20_iterations_fp32_vs_fp64(c2, cfg):
    opts = gs.RunOpts(selector=cfg) if cfg in ("rules", "mlp") else cfg
    pr, st = c2["g"].pagerank(iters=20, eps=0.0, opts=opts)
    assert st.levels == 20
    l1, mrel = pr_errors(pr, c2["h"], c2["jobs"]["pr"].result())
    report(case="c2_pagerank20", cfg=cfg, l1_normalised=l1, max_rel=mrel)
    assert l1 <= PR_TOL, (cfg, l1, mrel)


# ---------------------------------------------------------------------------
# C4: batched forms
# ---------------------------------------------------------------------------
def test_c4_mbfs_256_sources_rmat22_every_source(bctx):
    h = oracle.rmat(22, 16, seed=1)
    g = bctx.rmat(22, 16, seed=1)
    same_graph(g, h)
    src = g.roots(77, 256)  # the bench's sources
    assert np.array_equal(src, oracle.roots(h, 77, 256))
    lv, st = g.mbfs(src, batched=True)
    assert lv.shape == (256, h.n)
    edges = 0
    step = 32  # oracle answers in flight at once (17 MB each)
    for c0 in range(0, 256, step):
        jobs = [POOL.submit(oracle.bfs, h, int(s)) for s in src[c0:c0 + step]]
        for i, j in enumerate(jobs, start=c0):
            ref = j.result()
            assert np.array_equal(lv[i], ref), (i, int(src[i]))
            edges += oracle.traversed_edges(h, ref)
    assert st.edges == edges
    g.close()


def test_c4_er_batch_512_instances(bctx):
    gb, voff = bctx.er_batch(512, seed=7, nlo=1000, nhi=200000, dlo=4.0, dhi=32.0)  # the bench's batch
    parts = oracle.er_batch(7, 512, nlo=1000, nhi=200000, dlo=4.0, dhi=32.0)
    off, col, _ = gb.download()
    assert len(voff) == 513 and voff[-1] == gb.n
    for i, h in enumerate(parts):
        a, b = int(voff[i]), int(voff[i + 1])
        assert b - a == h.n, i
        assert np.array_equal(off[a:b + 1] - off[a], h.off), i
        assert np.array_equal(col[off[a]:off[b]] - a, h.col), i
    del off, col
    roots = [int(oracle.roots(h, 11 + i, 1)[0]) for i, h in enumerate(parts)]  # bench: h.roots(11 + i, 1)
    bfs_jobs = [POOL.submit(oracle.bfs, h, r) for h, r in zip(parts, roots)]
    cc_jobs = [POOL.submit(oracle.cc_linear, h) for h in parts]
    groots = [int(voff[i]) + r for i, r in enumerate(roots)]
    for o in (gs.RunOpts(selector="mlp"), gs.RunOpts(selector="mlp", captured=True)):
        lv, st = gb.bfs_multi(groots, o)
        edges = 0
        for i, j in enumerate(bfs_jobs):
            ref = j.result()
            assert np.array_equal(lv[voff[i]:voff[i + 1]], ref), (i, vars(o))
            edges += oracle.traversed_edges(parts[i], ref)
        assert st.edges == edges
    lab, _ = gb.cc()
    for i, j in enumerate(cc_jobs):
        assert np.array_equal(lab[voff[i]:voff[i + 1]] - voff[i], j.result()), i
    gb.close()
