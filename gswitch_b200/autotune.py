"""Autotuner of the expand launches: for every variant (direction x format x
load balance, and the fused push forms) times the variant's expands under
grid caps of 1/4 .. 16x the kernel's resident grid and, where the variant has
them, under each of its shapes (STRICT: tiles of 512 / 1,024 / 2,048 slots;
thread-mapped push: 256 / 128 / 512 threads per CTA; thread-mapped pull:
candidates per thread 2 / 1 / 4 at each of those CTA sizes) on seeded
synthetic graphs, and keeps the fastest
(CUDA-event expand times summed over levels; BFS from three roots per graph).
The tables load with Context.tune_load() and Context.tune_load_shapes().

    python -m gswitch_b200.autotune --out gswitch_b200/models/tune.json
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import gswitch_b200 as gs  # noqa: E402

QUARTERS = (1, 2, 4, 8, 16, 32, 64)  # grid cap = resident grid x q / 4
STRICT_SHAPES = 3   # tile 1024 (default), 512, 2048
PUSH_TM_SHAPES = 3  # threads per CTA: 256 (default), 128, 512
PULL_TM_SHAPES = 9  # candidates per thread 2 (default), 1, 4 (shape % 3) at those CTA sizes (shape // 3)


def shapes_of(direction, lb):
    if lb == "STRICT":
        return STRICT_SHAPES
    if lb == "TM":
        return PULL_TM_SHAPES if direction == "Pull" else PUSH_TM_SHAPES
    return 1
VARIANTS = [(d, f, lb, False) for d in ("Push", "Pull") for f in ("Queue", "Bitmap")
            for lb in ("TM", "WM", "CM", "STRICT", "TWC")] + [("Push", "Queue", lb, True)
                                                              for lb in ("TM", "WM", "CM", "STRICT", "TWC")]
DEFAULT_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "models", "tune.json")


def expand_ms(g, roots, cfg):
    tot = 0.0
    for r in roots:
        _, st = g.bfs(int(r), gs.RunOpts.from_config(cfg, timing=True, persistent=False), out=False)
        tot += sum(st.level_ms)
    return tot


def tune(ctx, graphs, reps=2, log=None, only=None):
    """only: load-balance names to tune (None: all); the other entries stay 0."""
    table = np.zeros(gs.TUNE_ENTRIES, dtype=np.int32)
    shapes = np.zeros(gs.TUNE_ENTRIES, dtype=np.int32)
    report = {}
    for d, f, lb, fused in VARIANTS:
        if only and lb not in only:
            continue
        cfg = f"{d}-{f}-{lb}-{'Fused' if fused else 'Standalone'}"
        idx = gs.Context.tune_index(d, f, lb, fused)
        times = {}
        for sh in range(shapes_of(d, lb)):
            s = np.zeros(gs.TUNE_ENTRIES, dtype=np.int32)
            s[idx] = sh
            ctx.tune_load_shapes(s)
            for q in QUARTERS:
                t = np.zeros(gs.TUNE_ENTRIES, dtype=np.int32)
                t[idx] = q
                ctx.tune_load(t)
                tot = 0.0
                for g, roots in graphs:
                    expand_ms(g, roots, cfg)  # warm-up
                    tot += min(expand_ms(g, roots, cfg) for _ in range(reps))
                times[(sh, q)] = tot
        best = min(times, key=times.get)
        # keep the default (shape 0, the resident grid) unless another choice
        # is clearly faster
        if times[best] < 0.97 * times[(0, 4)]:
            shapes[idx], table[idx] = best[0], (0 if best[1] == 4 else best[1])
        report[cfg] = {"shape": int(shapes[idx]), "quarters": int(table[idx]) or 4,
                       "ms": {f"{k[0]}/{k[1]}": round(v, 4) for k, v in times.items()}}
        if log:
            log(f"{cfg}: shape {report[cfg]['shape']} quarters {report[cfg]['quarters']}")
    ctx.tune_load(None)
    ctx.tune_load_shapes(None)
    return table, shapes, report


def merge(old, table, shapes, report, only):
    """A re-tune of the load balances in `only` on top of an earlier table
    (the parsed json): the other variants keep their old entries."""
    table, shapes = table.copy(), shapes.copy()
    for d, f, lb, fused in VARIANTS:
        if lb in only:
            continue
        i = gs.Context.tune_index(d, f, lb, fused)
        table[i] = old["quarters"][i]
        shapes[i] = old.get("shapes", [0] * gs.TUNE_ENTRIES)[i]
    report = {**{k: v for k, v in old.get("report", {}).items() if k.split("-")[2] not in only}, **report}
    return table, shapes, report


def load_table(path=None):
    path = path or DEFAULT_PATH
    if not os.path.exists(path):
        return None
    return np.asarray(json.load(open(path))["quarters"], dtype=np.int32)


def load_shapes(path=None):
    """The tuned shapes (None when the table has none)."""
    path = path or DEFAULT_PATH
    if not os.path.exists(path):
        return None
    d = json.load(open(path))
    return np.asarray(d["shapes"], dtype=np.int32) if "shapes" in d else None


def load_into(ctx, path=None):
    """Loads both tables into a context (defaults where absent)."""
    ctx.tune_load(load_table(path))
    ctx.tune_load_shapes(load_shapes(path))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_PATH)
    ap.add_argument("--scale", type=int, default=20)
    ap.add_argument("--only", default=None,
                    help="comma-separated load balances to re-tune; the other entries are kept from --out")
    args = ap.parse_args(argv)
    only = set(args.only.split(",")) if args.only else None
    ctx = gs.Context(0)
    graphs = []
    for g in (ctx.rmat(args.scale, 16, seed=11), ctx.grid(1024, 1024, 100, seed=12),
              ctx.er(1 << args.scale, 8 << args.scale, seed=13)):
        graphs.append((g, g.roots(5, 3)))
    table, shapes, report = tune(ctx, graphs, log=lambda m: print(m, file=sys.stderr, flush=True), only=only)
    if only and os.path.exists(args.out):
        table, shapes, report = merge(json.load(open(args.out)), table, shapes, report, only)
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    with open(args.out, "w") as f:
        json.dump({"format": "gswitch_b200 expand grid caps, quarters of the resident grid, and shapes (STRICT "
                             "tile, thread-mapped CTA size and pull candidates per thread), "
                             "index ((pull*2+bitmap)*8+lb)*2+fused", "quarters": [int(x) for x in table],
                   "shapes": [int(x) for x in shapes],
                   "graphs": [f"rmat{args.scale}", "grid1024x1024_lr100", f"er2^{args.scale}"], "report": report}, f,
                  indent=0)
    print(json.dumps({k: [v.get("shape", 0), v.get("quarters")] for k, v in report.items()}))
    ctx.close()


if __name__ == "__main__":
    main()
