"""Learned selector: the training kernels' gradient against an FP64 CPU
reference, the warp-level inference against the same forward pass in FP64,
training on a learnable synthetic task, the per-level label generator, exact
results under the network's choices, and the gain of the committed model
over the rule-based selector."""
import numpy as np
import pytest

import gswitch_b200 as gs
import oracle
from gswitch_b200.selector_train import load_model, regret
from test_gpu_apps import _pr_l1

pytestmark = pytest.mark.gpu

H, K, F = 32, gs.MLP_CLASSES, gs.MLP_FEATURES


def unpack(model):
    m = np.asarray(model, dtype=np.float64)
    o = 0
    W1 = m[o:o + H * F].reshape(H, F); o += H * F
    b1 = m[o:o + H]; o += H
    W2 = m[o:o + H * H].reshape(H, H); o += H * H
    b2 = m[o:o + H]; o += H
    W3 = m[o:o + K * H].reshape(K, H); o += K * H
    b3 = m[o:o + K]; o += K
    mean = m[o:o + F]; o += F
    inv = m[o:o + F]
    return W1, b1, W2, b2, W3, b3, mean, inv


def soft_labels(T, tau):
    T = np.asarray(T, dtype=np.float64)
    tmin = np.where(T > 0, T, np.inf).min(axis=1, keepdims=True)
    q = np.where(T > 0, np.exp(-(T / tmin - 1.0) / tau), 0.0)
    return q / q.sum(axis=1, keepdims=True)


def ref_loss_grad(model, X, T, tau):
    """FP64 forward and backward pass of the mean soft-label cross entropy."""
    W1, b1, W2, b2, W3, b3, mean, inv = unpack(model)
    x = (np.asarray(X, np.float64) - mean) * inv
    a1 = x @ W1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0)
    z = h2 @ W3.T + b3
    z = z - z.max(axis=1, keepdims=True)
    lse = np.log(np.exp(z).sum(axis=1, keepdims=True))
    q = soft_labels(T, tau)
    n = len(X)
    loss = float(-(q * (z - lse)).sum() / n)
    dz = (np.exp(z - lse) - q) / n
    gW3, gb3 = dz.T @ h2, dz.sum(0)
    d2 = (dz @ W3) * (a2 > 0)
    gW2, gb2 = d2.T @ h1, d2.sum(0)
    d1 = (d2 @ W2) * (a1 > 0)
    gW1, gb1 = d1.T @ x, d1.sum(0)
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])


def ref_logits(model, X):
    W1, b1, W2, b2, W3, b3, mean, inv = unpack(model)
    x = (np.asarray(X, np.float64) - mean) * inv
    h1 = np.maximum(x @ W1.T + b1, 0)
    h2 = np.maximum(h1 @ W2.T + b2, 0)
    return h2 @ W3.T + b3


def random_model(rng):
    m = np.zeros(gs.MLP_MODEL_FLOATS, dtype=np.float32)
    m[:gs.MLP_NPARAM] = rng.normal(0, 0.3, gs.MLP_NPARAM)
    m[gs.MLP_NPARAM:gs.MLP_NPARAM + F] = rng.normal(0, 1, F)
    m[gs.MLP_NPARAM + F:] = rng.uniform(0.5, 2.0, F)
    return m


def random_data(rng, n):
    X = rng.normal(0, 2, (n, F)).astype(np.float32)
    T = rng.uniform(0.01, 2.0, (n, K)).astype(np.float32)
    T[rng.random((n, K)) < 0.1] = 0  # untimed variants
    return X, T


def test_training_gradient_matches_fp64(ctx):
    rng = np.random.default_rng(3)
    for n in (1, 37, 512):
        model = random_model(rng)
        X, T = random_data(rng, n)
        g, loss = ctx.mlp_grad(model, X, T, tau=0.1)
        rl, rg = ref_loss_grad(model, X, T, 0.1)
        assert abs(loss - rl) <= 1e-4 * max(1.0, abs(rl)), (n, loss, rl)
        err = np.linalg.norm(g - rg) / max(np.linalg.norm(rg), 1e-12)
        assert err <= 1e-4, (n, err)
        assert np.max(np.abs(g - rg)) <= 1e-4 * max(1.0, np.max(np.abs(rg)))


def test_warp_inference_matches_fp64_forward(ctx):
    rng = np.random.default_rng(5)
    model = random_model(rng)
    X, _ = random_data(rng, 2000)
    cls, prob = ctx.mlp_infer(model, X)
    z = ref_logits(model, X)
    top2 = np.sort(z, axis=1)[:, -2:]
    clear = (top2[:, 1] - top2[:, 0]) > 1e-4
    assert np.array_equal(cls[clear], z.argmax(axis=1)[clear])
    p = np.exp(z - z.max(axis=1, keepdims=True))
    p = p.max(axis=1) / p.sum(axis=1)
    assert np.allclose(prob, p, rtol=1e-4, atol=1e-6)


def test_training_learns_a_learnable_choice(ctx):
    rng = np.random.default_rng(11)
    n = 6000
    X = rng.normal(0, 1, (n, F)).astype(np.float32)
    P = rng.normal(0, 1, (F, K))
    best = (X @ P).argmax(axis=1)
    T = np.full((n, K), 2.0, dtype=np.float32)
    T[np.arange(n), best] = 1.0
    model, loss = ctx.mlp_train(X[:5000], T[:5000], epochs=600, lr=5e-3, tau=0.1, seed=1)
    assert loss[-1] < loss[0] * 0.5
    cls, _ = ctx.mlp_infer(model, X[5000:])
    assert np.mean(cls == best[5000:]) > 0.8


def test_label_levels_rmat(ctx):
    g = ctx.rmat(12, 16, seed=4, wmax=64, wseed=5)
    root = int(g.roots(3, 1)[0])
    for app in (gs.APP_BFS, gs.APP_SSSP, gs.APP_PR):
        X, T, R = g.label(app, root, max_levels=48, pr_iters=2)
        assert len(X) >= 2, app
        assert np.all(np.isfinite(X))
        assert (T > 0).mean() > 0.9, app
        assert np.all((R >= 0) & (R < gs.MLP_CLASSES)), app
    # labelling leaves the graph and the context as they were
    lv, _ = g.bfs(root)
    off, col, _ = g.download()
    assert np.array_equal(lv, oracle.bfs(oracle.Csr(off, col), root))


def test_results_exact_under_network_choices(ctx):
    """Whatever the network picks, results stay exact (a random network picks
    all sorts of variants)."""
    rng = np.random.default_rng(9)
    h = oracle.rmat(13, 16, seed=2)
    hw = oracle.add_weights(h, 5, 64)
    root = int(oracle.roots(h, 9, 1)[0])
    g = ctx.upload(hw.off, hw.col, hw.w)
    ref_bfs, ref_sssp = oracle.bfs(h, root), oracle.sssp_dijkstra(hw, root)
    for s in range(4):
        ctx.mlp_load(random_model(rng), 0.0)
        for captured in (False, True):
            lv, _ = g.bfs(root, gs.RunOpts(selector="mlp", captured=captured))
            assert np.array_equal(lv, ref_bfs), (s, captured)
        d, _ = g.sssp(root, gs.RunOpts(selector="mlp"))
        assert np.array_equal(d, ref_sssp), s
    ctx.mlp_load(None)


def test_committed_model_beats_rules_on_held_out_graphs(ctx):
    """Regret against the exhaustively timed best variant, summed over the
    levels of held-out graphs (seeds the corpus never used): the committed
    network loses less time than the rule-based selector."""
    model, _ = load_model()
    assert model is not None, "gswitch_b200/models/selector_mlp.json is missing"
    Xs, Ts, Rs = [], [], []
    specs = [ctx.rmat(16, 16, 0.6, 0.175, 0.175, seed=90001, wmax=64, wseed=2),
             ctx.rmat(17, 16, 0.5, 0.225, 0.225, seed=90002, wmax=64, wseed=2),
             ctx.er(1 << 16, 1 << 19, seed=90003, wmax=64, wseed=2),
             ctx.grid(256, 256, 100, seed=90004, wmax=64, wseed=2),
             ctx.powerlaw(1 << 16, 2.2, seed=90005, wmax=64, wseed=2)]
    for g in specs:
        root = int(g.roots(17, 1)[0])
        for app in (gs.APP_BFS, gs.APP_SSSP, gs.APP_PR):
            X, T, R = g.label(app, root, max_levels=48, pr_iters=2)
            Xs.append(X), Ts.append(T), Rs.append(R)
        g.close()
    X, T, R = np.concatenate(Xs), np.concatenate(Ts), np.concatenate(Rs)
    cls, _ = ctx.mlp_infer(model, X)
    rows = np.arange(len(T))
    both = (T[rows, cls] > 0) & (T[rows, np.clip(R, 0, gs.MLP_CLASSES - 1)] > 0) & (R >= 0)
    r_mlp, r_rules = regret(T[both], cls[both]), regret(T[both], R[both])
    assert r_mlp["chosen_ms"] < r_rules["chosen_ms"], (r_mlp, r_rules)
    # the selector's target: within 10% of the exhaustively timed best variant,
    # time-weighted over the held-out levels
    assert regret(T, cls)["time_weighted"] <= 0.10, regret(T, cls)


def test_committed_model_speeds_up_pagerank(ctx):
    """End to end: PageRank on a skewed RMAT graph runs faster with the
    network choosing the variant than with the rules (which pick a warp-mapped
    push that serialises on hubs), with the same result tolerance."""
    model, conf = load_model()
    assert model is not None
    ctx.mlp_load(model, conf)
    g = ctx.rmat(18, 16, seed=1)
    off, col, _ = g.download()
    h = oracle.Csr(off, col)
    times = {}
    for sel in ("rules", "mlp"):
        g.pagerank(iters=5, eps=0.0, opts=gs.RunOpts(selector=sel))
        pr, st = g.pagerank(iters=20, eps=0.0, opts=gs.RunOpts(selector=sel))
        l1, _ = _pr_l1(pr, h)
        assert l1 <= 1e-6, (sel, l1)
        times[sel] = st.ms
    ctx.mlp_load(None)
    assert times["mlp"] < times["rules"], times


def _biased_model(cls):
    """A network whose output is the constant class `cls`."""
    m = np.zeros(gs.MLP_MODEL_FLOATS, dtype=np.float32)
    m[gs.MLP_NPARAM - gs.MLP_CLASSES + cls] = 10.0  # b3[cls]
    m[gs.MLP_NPARAM + gs.MLP_FEATURES:] = 1.0
    return m


def test_sssp_exact_under_both_fusion_decisions(ctx):
    h = oracle.er(30000, 150000, seed=8)
    hw = oracle.add_weights(h, 9, 64)
    root = int(oracle.roots(h, 2, 1)[0])
    ref = oracle.sssp_dijkstra(hw, root)
    g = ctx.upload(hw.off, hw.col, hw.w)
    model, conf = load_model()
    ctx.mlp_load(model, conf)
    for cls in (0, 1):
        ctx.mlp_load_fusion(_biased_model(cls), 0.0)
        d, st = g.sssp(root, gs.RunOpts(selector="mlp"))
        assert np.array_equal(d, ref), cls
        assert ({t[3] for t in st.trace} == {"Fused"}) == (cls == 1)
    ctx.mlp_load_fusion(None)
    ctx.mlp_load(None)


def test_committed_fusion_model_not_slower_than_the_tree_on_fresh_graphs(ctx):
    """SSSP on graphs the fusion corpus never saw: on a graph where the
    learned fused/standalone decision and the reference tree pick different
    forms, the network's pick is faster; where they pick the same form the
    times differ only by noise (5% slack)."""
    from gswitch_b200.selector_train import load_fusion_model

    fm, fc = load_fusion_model()
    assert fm is not None, "gswitch_b200/models/fusion_mlp.json is missing"
    model, conf = load_model()
    ctx.mlp_load(model, conf)
    ctx.mlp_load_fusion(fm, fc)
    graphs = [ctx.er(1 << 19, 4 << 19, seed=91001, wmax=64, wseed=3),
              ctx.grid(2900, 2900, 100, seed=91002, wmax=1000, wseed=3),
              ctx.rmat(19, 16, 0.55, 0.2, 0.2, seed=91003, wmax=64, wseed=3)]
    out = []
    for g in graphs:
        root = int(g.roots(8, 1)[0])
        t, form = {}, {}
        for sel in ("mlp", "rules"):
            o = gs.RunOpts(selector=sel)
            g.sssp(root, o, out=False)
            runs = [g.sssp(root, o, out=False)[1] for _ in range(2)]
            t[sel] = min(st.ms for st in runs)
            form[sel] = runs[0].trace[0][3] if runs[0].trace else None  # fused or standalone from the start
        out.append((form["mlp"] == form["rules"], t["mlp"], t["rules"], form))
        g.close()
    ctx.mlp_load_fusion(None)
    ctx.mlp_load(None)
    for same, t_mlp, t_tree, form in out:
        if same:
            assert t_mlp <= 1.05 * t_tree, (t_mlp, t_tree, form)
        else:
            assert t_mlp < t_tree, (t_mlp, t_tree, form)
