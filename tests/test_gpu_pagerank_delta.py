"""Delta-PageRank (gsw_pagerank_delta) against the oracle's FP64 fixed point
of the reference's unnormalised PageRank (pr = (1-d) + d * sum pr[u]/od[u],
application/pagerank.cu:19-32, iterated to convergence).  Every change a
vertex accumulates is positive and a vertex holds back less than eps times
its value, so the result approaches the fixed point from below and the
normalised L1 distance is at most eps / (1 - d); the tolerance adds 1e-5 for
FP32 accumulation."""
import itertools

import numpy as np
import pytest

import oracle
from conftest import golden_names, load_golden

pytestmark = pytest.mark.gpu

D = 0.85
VARIANTS = ["", "Push-Queue-TM-Standalone", "Push-Queue-WM-Standalone", "Push-Queue-CM-Standalone",
            "Push-Queue-STRICT-Standalone", "Push-Queue-TWC-Standalone", "Push-Bitmap-WM-Standalone",
            "Pull-Bitmap-TM-Standalone", "Pull-Queue-WM-Standalone", "Pull-Bitmap-STRICT-Standalone"]


def _fixpoint(h):
    return oracle.pagerank(h, 400, D)


def _check(pr, ref, eps):
    pr = pr.astype(np.float64)
    l1 = np.abs(pr / pr.sum() - ref / ref.sum()).sum()
    assert l1 <= eps / (1 - D) + 1e-5, l1
    # approached from below (FP32 rounding aside)
    assert np.all(pr <= ref * (1 + 1e-4) + 1e-6)
    return l1


@pytest.mark.parametrize("name", ["rmat10", "grid24_lr", "er1500", "path10", "twocomp_isolated"])
def test_delta_pagerank_goldens_every_variant(ctx, name):
    d = load_golden(name)
    h = oracle.Csr(d["off"], d["col"])
    ref = _fixpoint(h)
    g = ctx.upload(d["off"], d["col"])
    for cfg in VARIANTS:
        pr, st = g.pagerank_delta(eps=1e-5, max_levels=2000, opts=cfg)
        _check(pr, ref, 1e-5)
        assert 1 < st.levels < 2000, (cfg, st.levels)
        assert "Fused" not in {t[3] for t in st.trace}


@pytest.mark.parametrize("scale_eps", [(14, 1e-4), (16, 1e-5)])
def test_delta_pagerank_rmat_and_work(ctx, scale_eps):
    scale, eps = scale_eps
    h = oracle.rmat(scale, 16, seed=3)
    ref = _fixpoint(h)
    g = ctx.upload(h.off, h.col)
    pr, st = g.pagerank_delta(eps=eps, max_levels=2000)
    _check(pr, ref, eps)
    assert st.levels < 2000
    # the work: out-edges of the vertices that sent, at least one full sweep
    # (level 0) -- reported beside the sweeps Jacobi needs for the same L1
    # bound (d^k <= eps / (1 - d)); the per-vertex relative threshold is the
    # stricter criterion, so the delta form is not always cheaper
    jacobi_iters = int(np.ceil(np.log(eps / (1 - D)) / np.log(D)))
    assert st.edges >= h.m
    print(f"delta-PR RMAT s{scale} eps {eps}: {st.edges / h.m:.1f} sweeps of edges, Jacobi {jacobi_iters}")


def test_delta_pagerank_level_cap_and_bad_args(ctx):
    h = oracle.grid(64, 64, 100, seed=2)
    g = ctx.upload(h.off, h.col)
    _, st = g.pagerank_delta(eps=1e-6, max_levels=3)
    assert st.levels == 3
    import gswitch_b200 as gs
    with pytest.raises(gs.GswError):
        g.pagerank_delta(eps=0.0)
    # activation needs a whole level's sum: fused levels are refused
    with pytest.raises(gs.GswError):
        g.pagerank_delta(eps=1e-4, opts="Push-Queue-WM-Fused")
