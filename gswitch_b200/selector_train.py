"""Builds the learned selector: a seeded synthetic corpus, per-level labels
from timing every variant, training on the GPU with the library's own
kernels, and the regret of the network and of the rule-based selector
against the exhaustively timed best variant on held-out graphs.

Corpus (one seed per graph): RMAT with 2^14..2^20 vertices (log-uniform;
--big adds graphs with 2^21..2^23, --huge RMAT graphs with 2^24 for BFS and
PageRank),
edge factor 16, a in [0.45, 0.65], d = 0.05, b = c = (1 - a - d) / 2;
Erdos-Renyi G(n, m) with n in 2^14..2^20 and mean degree in [4, 32]; square
2D grids with 1% long-range edges, side 64..1024; power-law configuration
graphs with gamma in [1.8, 3.0].  Each graph is labelled for BFS, SSSP
(integer weights in [1, 64]) and PageRank.

    python -m gswitch_b200.selector_train --train 2000 --test 200 \\
        --out gswitch_b200/models/selector_mlp.json
    python -m gswitch_b200.selector_train fusion     # SSSP fused vs standalone
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import gswitch_b200 as gs  # noqa: E402

KINDS = ("rmat", "er", "grid", "powerlaw")
APPS = ((gs.APP_BFS, "bfs"), (gs.APP_SSSP, "sssp"), (gs.APP_PR, "pr"))


def corpus(count: int, seed: int, lg_min: int = 14, lg_max: int = 20):
    """`count` graph specifications drawn from one seed, with 2^lg_min ..
    2^lg_max vertices."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        kind = KINDS[i % len(KINDS)]
        gseed = int(rng.integers(1, 2**62))
        if kind == "rmat":
            a = float(rng.uniform(0.45, 0.65))
            bc = (1.0 - a - 0.05) / 2
            out.append({"kind": kind, "scale": int(rng.integers(lg_min, lg_max + 1)), "a": a, "b": bc, "c": bc,
                        "seed": gseed})
        elif kind == "er":
            n = int(2 ** rng.uniform(lg_min, lg_max))
            deg = float(rng.uniform(4, 32))
            out.append({"kind": kind, "n": n, "m_pairs": int(n * deg / 2), "seed": gseed})
        elif kind == "grid":
            side = int(2 ** rng.uniform(lg_min / 2 - 1, lg_max / 2))
            out.append({"kind": kind, "side": side, "seed": gseed})
        else:
            out.append({"kind": kind, "n": int(2 ** rng.uniform(lg_min, lg_max)), "gamma": float(rng.uniform(1.8, 3.0)),
                        "seed": gseed})
    return out


def build(ctx, spec, wmax=64):
    k = spec["kind"]
    if k == "rmat":
        return ctx.rmat(spec["scale"], 16, spec["a"], spec["b"], spec["c"], seed=spec["seed"], wmax=wmax,
                        wseed=spec["seed"] + 1)
    if k == "er":
        return ctx.er(spec["n"], spec["m_pairs"], seed=spec["seed"], wmax=wmax, wseed=spec["seed"] + 1)
    if k == "grid":
        return ctx.grid(spec["side"], spec["side"], 100, seed=spec["seed"], wmax=wmax, wseed=spec["seed"] + 1)
    return ctx.powerlaw(spec["n"], spec["gamma"], seed=spec["seed"], wmax=wmax, wseed=spec["seed"] + 1)


def label_corpus(ctx, specs, budget_s: float, log=None, apps=APPS):
    """Labels every graph (until the time budget runs out); returns rows
    X [r, 8], T [r, 20], R (rule class) [r], G (graph index) [r], A (app) [r]."""
    Xs, Ts, Rs, Gs, As = [], [], [], [], []
    t0 = time.time()
    done = 0
    for gi, spec in enumerate(specs):
        if time.time() - t0 > budget_s:
            break
        g = build(ctx, spec)
        root = int(g.roots(spec["seed"] % 1000 + 3, 1)[0])
        for app, _ in apps:
            X, T, R = g.label(app, root, max_levels=48, pr_iters=2)
            Xs.append(X)
            Ts.append(T)
            Rs.append(R)
            Gs.append(np.full(len(X), gi, dtype=np.int32))
            As.append(np.full(len(X), app, dtype=np.int32))
        g.close()
        done += 1
        if log and done % 50 == 0:
            log(f"labelled {done} graphs in {time.time() - t0:.0f} s")
    cat = lambda xs, shape, dt: np.concatenate(xs) if xs else np.zeros(shape, dt)
    return (cat(Xs, (0, 8), np.float32), cat(Ts, (0, 20), np.float32), cat(Rs, (0,), np.int32),
            cat(Gs, (0,), np.int32), cat(As, (0,), np.int32), done)


def regret(T, choice):
    """Time-weighted regret sum(t[choice]) / sum(t_best) - 1 over the rows
    whose choice was timed, and the mean per-level ratio minus 1."""
    tbest = np.where(T > 0, T, np.inf).min(axis=1)
    ok = (choice >= 0) & np.isfinite(tbest)
    tc = T[np.arange(len(T)), np.clip(choice, 0, 19)]
    ok &= tc > 0
    if not ok.any():
        return {"time_weighted": None, "per_level_mean": None, "rows": 0}
    return {"time_weighted": float(tc[ok].sum() / tbest[ok].sum() - 1.0),
            "per_level_mean": float(np.mean(tc[ok] / tbest[ok]) - 1.0), "rows": int(ok.sum()),
            "chosen_ms": float(tc[ok].sum()), "best_ms": float(tbest[ok].sum())}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--test", type=int, default=200)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--epochs", type=int, default=3000)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--tau", type=float, default=0.1)
    ap.add_argument("--budget-s", type=float, default=900.0, help="labelling time budget for the training corpus")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "models",
                                                  "selector_mlp.json"))
    ap.add_argument("--save-labels", default=None)
    ap.add_argument("--labels-in", default=None, help="start from labels saved by an earlier run")
    ap.add_argument("--big", type=int, default=0, help="extra graphs with 2^21..2^23 vertices")
    ap.add_argument("--big-test", type=int, default=0)
    ap.add_argument("--big-budget-s", type=float, default=600.0)
    ap.add_argument("--huge", type=int, default=0, help="extra RMAT graphs with 2^24 vertices (BFS, PageRank)")
    ap.add_argument("--huge-test", type=int, default=0)
    args = ap.parse_args(argv)
    log = lambda m: print(m, file=sys.stderr, flush=True)
    ctx = gs.Context(0)
    t0 = time.time()
    if args.labels_in:
        d = np.load(args.labels_in)
        Xtr, Ttr, Rtr, Gtr, Atr = d["Xtr"], d["Ttr"], d["Rtr"], d["Gtr"], d["Atr"]
        Xte, Tte, Rte, Gte, Ate = d["Xte"], d["Tte"], d["Rte"], d["Gte"], d["Ate"]
        ntr, nte = int(Gtr.max()) + 1 if len(Gtr) else 0, int(Gte.max()) + 1 if len(Gte) else 0
    else:
        Xtr, Ttr, Rtr, Gtr, Atr, ntr = label_corpus(ctx, corpus(args.train, args.seed), args.budget_s, log)
        Xte, Tte, Rte, Gte, Ate, nte = label_corpus(ctx, corpus(args.test, args.seed + 1), args.budget_s / 4, log)
    if args.big:
        parts = label_corpus(ctx, corpus(args.big, args.seed + 2, 21, 23), args.big_budget_s, log)
        Xtr, Ttr, Rtr, Atr = (np.concatenate([a, b]) for a, b in zip((Xtr, Ttr, Rtr, Atr), parts[:2] + parts[2:3] + parts[4:5]))
        Gtr = np.concatenate([Gtr, parts[3] + ntr])
        ntr += parts[5]
    if args.big_test:
        parts = label_corpus(ctx, corpus(args.big_test, args.seed + 3, 21, 23), args.big_budget_s / 4, log)
        Xte, Tte, Rte, Ate = (np.concatenate([a, b]) for a, b in zip((Xte, Tte, Rte, Ate), parts[:2] + parts[2:3] + parts[4:5]))
        Gte = np.concatenate([Gte, parts[3] + nte])
        nte += parts[5]
    for count, seed, test in ((args.huge, args.seed + 4, False), (args.huge_test, args.seed + 5, True)):
        if not count:
            continue
        rng = np.random.default_rng(seed)
        specs = []
        for _ in range(count):
            a = float(rng.uniform(0.5, 0.62))
            bc = (1.0 - a - 0.05) / 2
            specs.append({"kind": "rmat", "scale": 24, "a": a, "b": bc, "c": bc,
                          "seed": int(rng.integers(1000, 2**62))})
        parts = label_corpus(ctx, specs, args.big_budget_s, log, apps=((gs.APP_BFS, "bfs"), (gs.APP_PR, "pr")))
        if test:
            Xte, Tte, Rte, Ate = (np.concatenate([a, b]) for a, b in zip((Xte, Tte, Rte, Ate), parts[:3] + parts[4:5]))
            Gte = np.concatenate([Gte, parts[3] + nte])
            nte += parts[5]
        else:
            Xtr, Ttr, Rtr, Atr = (np.concatenate([a, b]) for a, b in zip((Xtr, Ttr, Rtr, Atr), parts[:3] + parts[4:5]))
            Gtr = np.concatenate([Gtr, parts[3] + ntr])
            ntr += parts[5]
    t_lab = time.time() - t0
    log(f"labels: train {len(Xtr)} rows / {ntr} graphs, test {len(Xte)} rows / {nte} graphs")
    if args.save_labels:
        np.savez_compressed(args.save_labels, Xtr=Xtr, Ttr=Ttr, Rtr=Rtr, Gtr=Gtr, Atr=Atr, Xte=Xte, Tte=Tte,
                            Rte=Rte, Gte=Gte, Ate=Ate)
    keep = (Ttr > 0).any(axis=1)
    t1 = time.time()
    model, loss = ctx.mlp_train(Xtr[keep], Ttr[keep], epochs=args.epochs, lr=args.lr, tau=args.tau, seed=args.seed)
    t_train = time.time() - t1
    cls, prob = ctx.mlp_infer(model, Xte)
    best = np.where(Tte > 0, Tte, np.inf).argmin(axis=1)
    report = {"train_graphs": ntr, "train_rows": int(keep.sum()), "test_graphs": nte, "test_rows": int(len(Xte)),
              "label_s": round(t_lab, 1), "train_s": round(t_train, 2), "epochs": args.epochs,
              "final_loss": float(loss[-1]), "test_accuracy": float(np.mean(cls == best)) if len(cls) else None,
              "regret_mlp": regret(Tte, cls), "regret_rules": regret(Tte, Rte),
              "per_app": {}}
    for app, name in APPS:
        m = Ate == app
        report["per_app"][name] = {"mlp": regret(Tte[m], cls[m]), "rules": regret(Tte[m], Rte[m])}
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    with open(args.out, "w") as f:
        json.dump({"format": "gswitch_b200 selector MLP 8-32-32-20 fp32", "model": [float(x) for x in model],
                   "min_conf": 0.0, "corpus_seed": args.seed, "report": report}, f)
    print(json.dumps(report))
    ctx.close()


# ---------------------------------------------------------------------------
# the fusion decision of SSSP (Mono pattern) runs
# ---------------------------------------------------------------------------
FUSION_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "models", "fusion_mlp.json")


def fusion_features(g):
    """The graph-level features of engine/mlp.cuh mlp_fusion_features (SSSP)."""
    a = g.attr()  # avg, std, range, max degree, Gini, entropy
    lg = lambda x: float(np.log2(1.0 + max(x, 0.0)))
    return np.array([lg(a[0]), lg(a[1]), lg(a[2]), a[4], a[5], lg(g.n), lg(g.m), 0.5], dtype=np.float32)


def fusion_corpus(count, seed):
    """Graphs for the fusion decision: the selector corpus shapes up to 2^22
    vertices, plus large grids (side up to 3,000)."""
    specs = corpus(count, seed, 14, 22)
    rng = np.random.default_rng(seed + 7)
    for s in specs:
        if s["kind"] == "grid" and rng.random() < 0.5:
            s["side"] = int(rng.uniform(1024, 3000))
    return specs


def label_fusion(ctx, specs, log=None, wmax_grid=1000):
    """Per graph: features, and SSSP device time with standalone (class 0) and
    fused (class 1) levels, the learned variant selector deciding the rest."""
    X, T, R = [], [], []
    for i, spec in enumerate(specs):
        g = build(ctx, spec, wmax=wmax_grid if spec["kind"] == "grid" else 64)
        root = int(g.roots(spec["seed"] % 1000 + 3, 1)[0])
        t = np.zeros(gs.MLP_CLASSES, dtype=np.float32)
        for k, fu in ((0, gs.STANDALONE), (1, gs.FUSED)):
            o = gs.RunOpts(selector="mlp", fusion=fu)
            g.sssp(root, o, out=False)
            t[k] = min(g.sssp(root, o, out=False)[1].ms for _ in range(2))
        _, st = g.sssp(root, gs.RunOpts(), out=False)  # the rule tree's decision
        X.append(fusion_features(g))
        T.append(t)
        R.append(1 if st.trace and st.trace[-1][3] == "Fused" else 0)
        g.close()
        if log and (i + 1) % 50 == 0:
            log(f"fusion labels: {i + 1} graphs")
    return np.array(X), np.array(T), np.array(R, dtype=np.int32)


def train_fusion(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=400)
    ap.add_argument("--test", type=int, default=80)
    ap.add_argument("--seed", type=int, default=3030)
    ap.add_argument("--epochs", type=int, default=2000)
    ap.add_argument("--out", default=FUSION_PATH)
    args = ap.parse_args(argv)
    log = lambda m: print(m, file=sys.stderr, flush=True)
    ctx = gs.Context(0)
    model, conf = load_model()
    ctx.mlp_load(model, conf)
    Xtr, Ttr, _ = label_fusion(ctx, fusion_corpus(args.train, args.seed), log)
    Xte, Tte, Rte = label_fusion(ctx, fusion_corpus(args.test, args.seed + 1), log)
    fmodel, loss = ctx.mlp_train(Xtr, Ttr, epochs=args.epochs, lr=3e-3, tau=0.05, seed=args.seed)
    cls, _ = ctx.mlp_infer(fmodel, Xte)
    cls = np.minimum(cls, 1)
    report = {"train_graphs": len(Xtr), "test_graphs": len(Xte), "final_loss": float(loss[-1]),
              "sssp_ms_test": {"mlp": float(Tte[np.arange(len(Tte)), cls].sum()),
                               "tree": float(Tte[np.arange(len(Tte)), Rte].sum()),
                               "always_standalone": float(Tte[:, 0].sum()),
                               "always_fused": float(Tte[:, 1].sum()),
                               "best": float(Tte[:, :2].min(axis=1).sum())}}
    with open(args.out, "w") as f:
        json.dump({"format": "gswitch_b200 fusion MLP 8-32-32-20 fp32 (classes 0 standalone, 1 fused)",
                   "model": [float(x) for x in fmodel], "min_conf": 0.0, "corpus_seed": args.seed,
                   "report": report}, f)
    print(json.dumps(report))
    ctx.close()


def load_fusion_model(path=None):
    path = path or FUSION_PATH
    if not os.path.exists(path):
        return None, 0.0
    d = json.load(open(path))
    return np.asarray(d["model"], dtype=np.float32), float(d.get("min_conf", 0.0))


def load_model(path=None):
    """The committed model as a float32 array, or None when absent."""
    path = path or os.path.join(os.path.dirname(os.path.abspath(__file__)), "models", "selector_mlp.json")
    if not os.path.exists(path):
        return None, 0.0
    d = json.load(open(path))
    return np.asarray(d["model"], dtype=np.float32), float(d.get("min_conf", 0.0))


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "fusion":
        train_fusion(sys.argv[2:])
    else:
        main()
