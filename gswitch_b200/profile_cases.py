"""Small fixed workloads for profiler captures (ncu -k ... python -m
gswitch_b200.profile_cases <case>):
  bfs   three BFS runs on RMAT scale 22 (ef 16, seed 1), learned selector
  bfs24 one BFS on RMAT scale 24 (ef 16, seed 1: the bench graph), learned
        selector
  sssp  SSSP on the 4096 x 4096 grid with 1% long-range edges (weights
        U[1, 1000]), Push-Queue-WM-Fused levels one launch each
  pr    two PageRank iterations on RMAT scale 22, Pull-Bitmap-STRICT then 2D
  mbfs  batched 256-source BFS on RMAT scale 20
"""
from __future__ import annotations

import os
import sys

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import gswitch_b200 as gs  # noqa: E402
from gswitch_b200.selector_train import load_model  # noqa: E402


def main(case: str) -> None:
    ctx = gs.Context(0)
    model, conf = load_model()
    if model is not None:
        ctx.mlp_load(model, conf)
    if case == "bfs":
        g = ctx.rmat(22, 16, seed=1)
        for r in g.roots(1000, 3):
            g.bfs(int(r), gs.RunOpts(selector="mlp"), out=False)
    elif case == "bfs24":
        g = ctx.rmat(24, 16, seed=1)
        g.bfs(int(g.roots(1000, 1)[0]), gs.RunOpts(selector="mlp"), out=False)
    elif case == "sssp":
        g = ctx.grid(4096, 4096, 100, seed=1, wmax=1000, wseed=5)
        o = gs.RunOpts.from_config("Push-Queue-WM-Fused")
        o.persistent = False
        g.sssp(int(g.roots(3, 1)[0]), o, out=False)
    elif case == "pr":
        g = ctx.rmat(22, 16, seed=1)
        g.pagerank(2, 0.85, 0.0, opts="Pull-Bitmap-STRICT", out=False)
        g.pagerank(2, 0.85, 0.0, opts="x-x-TWOD", out=False)
    elif case == "mbfs":
        g = ctx.rmat(20, 16, seed=1)
        g.mbfs(g.roots(77, 256), batched=True, out=False)
    else:
        raise SystemExit(f"unknown case {case!r} (bfs, bfs24, sssp, pr, mbfs)")
    print("ok", case)
    g.close()
    ctx.close()


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "bfs")
