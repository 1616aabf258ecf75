"""Headline benchmark: BFS GTEPS on an undirected RMAT graph (scale 24, edge
factor 16, a=.57 b=.19 c=.19, seed 1) on B200, with the selector switching
direction / frontier format / load balance per level.

One step = one BFS from a seeded non-isolated root (a different root per
step), graph resident in HBM.  GTEPS uses the Graph500 numerator (sum of the
degrees of reached vertices / 2).  Under torchrun every rank runs its own
replica with its own roots (weak scaling; the path has no exchange step).

Also reported:
  e2e          the same metric through the C ABI with host buffers: every
               step uploads the host CSR (pinned), runs BFS and reads the
               levels back;
  roofline     the dominant kernel's algorithmic bytes per launch over its
               average CUDA-event duration (the timed steps repeated with an
               event pair around every kernel), against the measured HBM copy
               bandwidth;
  apps         config C2's four applications on the same graph: the switched
               form (rule trees, learned selector, captured loop) against
               every fixed variant; the 256-source batched MBFS and the
               512-graph G(n, m) batch (config C4) batched vs unbatched;
  cpu_baseline the CPU oracle's restated reference BFS on the same graph,
               one core, bounded sample (rank 0, N=1).
`--impl reference` times the reference's own bfs_cpu (application/bfs.cu:
38-62, built from its sources into oracle/_ref) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GTEPS (BFS, RMAT scale 24 ef 16, switched selector)"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = None
        self.skip = 0

    def start(self):
        """Starts sampling every 20 ms and waits (up to 5 s) for the first
        sample, so that the timed region that follows is covered."""
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            t0 = time.time()
            while time.time() - t0 < 5.0 and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
            self.skip = sum(1 for _ in open(self.path))  # samples taken before the timed region
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = open(self.path).read().splitlines()
        # keep the samples of the timed region (the last pre-region one too,
        # when the region was shorter than the sampling period)
        lines = lines[max(0, self.skip - 1):]
        for line in lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def level_bytes(kind, n, A, U, D, E):
    """Algorithmic bytes of one expand (int32 levels, bitmap state probes), the
    per-unit figures of the path's roofline definition:
    push: work list + 16 B of row offsets per frontier vertex + 4 B column and
    2 bitmap probes per edge + 4 B level write per discovered vertex;
    pull: work list + 16 B offsets per candidate + 4 B column and one
    frontier-bit probe per scanned edge + 4 B write per discovered vertex."""
    direction, fmt = kind[0], kind[1]
    if direction == "Push":
        work = n / 8 if fmt == "Bitmap" else 4 * A
        return work + 16 * A + 4.25 * E + 4 * D
    work = n / 8 if fmt == "Bitmap" else 4 * U
    return work + 16 * U + 4.125 * E + 4 * D


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per vertex of
# one inspection launch, from an ncu capture of the third inspection of one
# BFS on the bench graph (135.47 MB + 4.42 MB over 16,777,216 vertices); the
# inspection streams every vertex once, so a launch's traffic scales with n
INSPECT_TRAFFIC_PER_VERTEX = (135.47e6 + 4.42e6) / 16777216
# DRAM bytes per launch of the thread-mapped pull expand on the bench graph
# (RMAT scale 24 ef 16 seed 1): the mean of the two launches of one BFS in the
# same capture (600.38 MB and 329.71 MB); per-launch traffic depends on the
# level, so this figure stands for the bench graph only
PULL_TM_TRAFFIC_RMAT24 = (600.38e6 + 329.71e6) / 2


def roofline_from(runs, n, peak_gbs, peak_kind):
    """runs: list of (timed RunStats, accounting RunStats, levels array)."""
    per = {}
    for timed, acc, lv in runs:
        cnt = np.bincount(lv[lv >= 0], minlength=len(timed.trace) + 2)
        unreached = int((lv < 0).sum())
        for i, t in enumerate(timed.trace):
            kind = t[:4]
            A = int(cnt[i]) if i < len(cnt) else 0
            D = int(cnt[i + 1]) if i + 1 < len(cnt) else 0
            U = int(cnt[i + 1:].sum()) + unreached
            E = acc.level_edges[i] if i < len(acc.level_edges) else 0
            key = "expand " + "-".join(kind)
            b = level_bytes(kind, n, A, U, D, max(E, 0))
            rec = per.setdefault(key, [0.0, 0.0, 0])
            rec[0] += timed.level_ms[i]
            rec[1] += b
            rec[2] += 1
            if timed.level_inspect_ms[i] > 0:
                rec = per.setdefault("inspect", [0.0, 0.0, 0])
                rec[0] += timed.level_inspect_ms[i]
                rec[1] += 8.0 * n + n / 4.0  # level + degree read, two bitmap words written
                rec[2] += 1
    shares = {k: round(v[0] / sum(x[0] for x in per.values()), 4) for k, v in per.items()}

    def line(name):
        ms, byt, launches = per[name]
        achieved = byt / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
        if name == "inspect":
            traffic = round(INSPECT_TRAFFIC_PER_VERTEX * n)
            note = "ncu DRAM bytes of one inspection on the bench graph, per vertex, times n"
        elif name == "expand Pull-Bitmap-TM-Standalone" and n == 1 << 24:
            traffic = round(PULL_TM_TRAFFIC_RMAT24)
            note = ("ncu DRAM bytes per launch on the bench graph (mean of one BFS's two pull levels); above the "
                    "algorithmic bytes because each candidate's first in-neighbour costs a 32-byte sector")
        else:
            traffic, note = None, "no per-launch ncu figure for this kernel's level mix"
        return {"bound": "hbm", "kernel": name, "achieved": round(achieved, 1), "peak": peak_gbs,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak_gbs, 4),
                "bytes_per_launch": round(byt / max(launches, 1)), "launches": launches,
                "avg_launch_ms": round(ms / max(launches, 1), 5), "traffic": traffic, "traffic_note": note}

    dom = max(per.items(), key=lambda kv: kv[1][0])[0]
    out = line(dom)
    out["time_shares"] = shares
    # the other kernels above a tenth of the time, same arithmetic
    out["others"] = [line(k) for k, v in sorted(per.items(), key=lambda kv: -kv[1][0])
                     if k != dom and shares[k] >= 0.1]
    return out


def run_opts(gs, selector, **kw):
    return gs.RunOpts(selector=selector, **kw)


def run_ours(args):
    import torch

    import gswitch_b200 as gs
    from gswitch_b200.selector_train import load_model

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist:
            dist.barrier()

    ctx = gs.Context(local)
    from gswitch_b200.autotune import load_into

    load_into(ctx, args.tune)  # autotuned expand grids and shapes (defaults when absent)
    selector = args.selector
    if selector == "mlp":
        from gswitch_b200.selector_train import load_fusion_model

        model, min_conf = load_model()
        if model is None:
            selector = "rules"
        else:
            ctx.mlp_load(model, min_conf)
            fmodel, fconf = load_fusion_model()
            if fmodel is not None:
                ctx.mlp_load_fusion(fmodel, fconf)
    sampler = ClockSampler(local)
    sampler.start()
    t0 = time.time()
    g = ctx.rmat(args.scale, args.ef, 0.57, 0.19, 0.19, seed=1)
    gen_s = time.time() - t0
    W, K = args.warmup, args.steps
    roots = g.roots(1000 + rank, W + K)
    for r in roots[:W]:
        g.bfs(int(r), run_opts(gs, selector), out=False)

    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    timed = []
    barrier()
    torch.cuda.synchronize()
    sampler.skip = sum(1 for _ in open(sampler.path)) if sampler.proc else 0
    e0.record(stream)
    edges = 0
    launches = 0
    for r in roots[W:W + K]:
        _, st = g.bfs(int(r), opts=run_opts(gs, selector), out=False)
        edges += st.edges
        launches += st.launches
        timed.append(st)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    barrier()
    ms_max, tot_edges = combine_ranks(dist, ms, edges, "cuda")
    value = tot_edges / (ms_max * 1e6)
    # end to end through the C ABI on every rank (replicas), combined the same way
    e2e_out = None
    if not args.no_e2e:
        e2e_ms, e2e_edges, e2e_steps, h2d, d2h = e2e(ctx, g, roots[W:W + min(K, 20)], gs, torch, selector)
        e2e_ms, e2e_edges = combine_ranks(dist, e2e_ms, e2e_edges, "cuda")
        e2e_out = {"value": round(e2e_edges / (e2e_ms * 1e6), 3), "unit": "GTEPS",
                   "ms_per_step": round(e2e_ms / e2e_steps, 3), "h2d_bytes_per_step": h2d,
                   "d2h_bytes_per_step": d2h, "per_step": "CSR upload from pinned memory + BFS + levels back"}
        r_ms, r_edges, r_steps, r_d2h = e2e_resident(ctx, g, roots[W:W + min(K, 20)], gs, torch, selector)
        r_ms, r_edges = combine_ranks(dist, r_ms, r_edges, "cuda")
        e2e_resident_out = {"value": round(r_edges / (r_ms * 1e6), 3), "unit": "GTEPS",
                            "ms_per_step": round(r_ms / r_steps, 3), "h2d_bytes_per_step": 4,
                            "d2h_bytes_per_step": r_d2h,
                            "per_step": "BFS from a root on the resident graph + levels back (the reference "
                                        "arm's unit of work: bfs_cpu per root on a CSR already in memory)"}

    out = None
    if rank == 0:
        # per-kernel pass: the same steps again with a CUDA event pair around
        # every inspection and expand (kept out of the timed region above,
        # whose value it would lower by the event records), plus an
        # accounting pass for the edges each expand touched
        runs = []
        for r in roots[W:W + K]:
            _, sti = g.bfs(int(r), opts=run_opts(gs, selector, timing=True), out=False)
            lv, acc = g.bfs(int(r), opts=run_opts(gs, selector, account=True))
            runs.append((sti, acc, lv))
        peak, kind = peaks()
        roof = roofline_from(runs, g.n, peak, kind)
        trace = [list(t[:4]) + [int(t[4])] for t in timed[0].trace]
        out = {
            "metric": METRIC, "value": round(value, 3), "unit": "GTEPS", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": round(ms_max / K, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int32", "data": "synthetic",
            "config": {"workload": f"bfs_rmat{args.scale}_ef{args.ef}", "scale": args.scale, "edge_factor": args.ef,
                       "rmat_abcd": [0.57, 0.19, 0.19, 0.05], "seed": 1, "n": g.n, "arcs": g.m,
                       "roots": "seeded non-isolated, one per step, per rank",
                       "l2": "inputs larger than L2 (CSR %.2f GB)" % ((8 * (g.n + 1) + 4 * g.m) / 1e9),
                       "parallelism": f"replicas x{world}",
                       "selector": "learned MLP (rules as fallback)" if selector == "mlp" else "rules (reference trees)",
                       "graph_build_s": round(gen_s, 2)},
            "roofline": roof, "gpu_launches": int(launches), "clocks": clocks,
            "levels_first_step": trace,
        }
        if world == 1 and not args.no_apps:
            out["apps"] = app_table(ctx, g, gs, args, roots[W:W + 3], selector)
        if e2e_out:
            out["e2e"] = e2e_out
            out["e2e_resident_graph"] = e2e_resident_out
        if world == 1 and not args.no_cpu:
            # the first two timed roots again, levels copied back, for the check
            check = {int(r): g.bfs(int(r), run_opts(gs, selector))[0] for r in roots[W:W + 2]}
            out["cpu_baseline"], out["parity"] = cpu_baseline(g, roots[W:], args.cpu_seconds, check)
    g.close()
    ctx.close()
    if dist:
        dist.destroy_process_group()
    if out:
        print(json.dumps(out))


FIXED = ["-".join((d, f, lb, "Standalone")) for d in ("Push", "Pull") for f in ("Queue", "Bitmap")
         for lb in ("TM", "WM", "CM", "STRICT", "TWC")] + [f"Push-Queue-{lb}-Fused" for lb in
                                                          ("TM", "WM", "CM", "STRICT", "TWC")]


def switch_headroom(g, app, root, pr_iters=2, ctx=None, model=None):
    """How much per-level switching can gain over one fixed variant: every
    standalone variant timed at each labelled level from the same state
    (gsw_label_levels: all levels up to 24, then every 8th; PageRank's
    iterations are alike, so two stand for all).  best_fixed = the smallest
    column total over the variants that ran at every level; per_level_best =
    the sum of each level's fastest; headroom = best_fixed / per_level_best
    bounds the speed-up any per-level choice among these variants can reach.
    With a model, the selectors' regret on the same levels: time of the
    chosen variants over the per-level best, minus one (the rules' class and
    the learned network's)."""
    X, T, R = g.label(app, root, max_levels=4096, pr_iters=pr_iters)
    if len(T) == 0:
        return None
    T = np.where(T > 0, T.astype(np.float64), np.inf)
    full = np.isfinite(T).all(axis=0)
    if not full.any():
        return None
    col_tot = T[:, full].sum(axis=0)
    best_fixed = float(col_tot.min())
    tbest = T.min(axis=1)
    per_level = float(tbest.sum())
    out = {"levels_labelled": int(len(T)), "best_fixed_ms": round(best_fixed, 4),
           "per_level_best_ms": round(per_level, 4), "headroom": round(best_fixed / per_level, 3)}

    def regret(choice):
        t = T[np.arange(len(T)), np.clip(choice, 0, T.shape[1] - 1)]
        ok = (choice >= 0) & np.isfinite(t)
        return round(float(t[ok].sum() / tbest[ok].sum() - 1.0), 4) if ok.any() else None

    out["regret_rules"] = regret(np.asarray(R))
    if ctx is not None and model is not None:
        cls, _ = ctx.mlp_infer(model, X)
        out["regret_mlp"] = regret(np.asarray(cls))
    return out


def app_table(ctx, g, gs, args, roots, selector):
    """The per-application table: BFS, SSSP, CC and PageRank on the same RMAT
    graph (SSSP on an int32-weighted copy, weights U[1, 64]): the switched
    form (rules, and the learned selector; host-driven and captured loop)
    against every fixed variant, GTEPS by each app's definition (BFS / SSSP:
    Graph500 edges of the reached component; CC: m/2; PageRank: m x
    iterations).  Plus the batched multi-source BFS (config C4's 256
    sources) against 256 sequential switched BFS runs."""
    gw = ctx.rmat(args.scale, args.ef, 0.57, 0.19, 0.19, seed=1, wmax=64, wseed=2)
    root = int(roots[0])
    from gswitch_b200.selector_train import load_model

    model, _ = load_model()
    pr_iters = 5

    def once(app, o):
        if app == "bfs":
            _, st = g.bfs(root, o, out=False)
        elif app == "sssp":
            _, st = gw.sssp(root, o, out=False)
        elif app == "pr":
            _, st = g.pagerank(pr_iters, 0.85, 0.0, opts=o, out=False)
        else:
            _, st = g.cc(o, out=False)
        return st.edges / (st.ms * 1e6) if st.ms > 0 else 0.0, st.ms

    def measure(app, o, reps):
        once(app, o)
        vals = sorted(once(app, o) for _ in range(reps))
        return vals[len(vals) // 2]

    table = {}
    for app in ("bfs", "sssp", "pr", "cc"):
        row = {"switched_rules": round(measure(app, gs.RunOpts(), 3)[0], 3)}
        if app != "cc":
            row["switched_mlp"] = round(measure(app, gs.RunOpts(selector="mlp"), 3)[0], 3)
        if app in ("bfs", "pr"):
            row["switched_mlp_captured"] = round(measure(app, gs.RunOpts(selector="mlp", captured=True), 3)[0], 3)
        fixed = {}
        if app == "cc":
            for cfg in ("x-Queue", "x-Bitmap"):
                fixed[cfg] = round(measure(app, gs.RunOpts.from_config(cfg), 1)[0], 3)
        else:
            for cfg in FIXED + (["x-x-TWOD"] if app == "pr" else []):
                if app == "pr" and cfg.endswith("Fused"):
                    continue
                fixed[cfg] = round(measure(app, gs.RunOpts.from_config(cfg), 1)[0], 3)
        best = max(fixed.items(), key=lambda kv: kv[1])
        if app != "cc":
            lab = {"bfs": gs.APP_BFS, "sssp": gs.APP_SSSP, "pr": gs.APP_PR}[app]
            row["switch_headroom_standalone"] = switch_headroom(gw if app == "sssp" else g, lab, root, ctx=ctx,
                                                                 model=model)
        sw = row.get("switched_mlp" if selector == "mlp" and app != "cc" else "switched_rules")
        row.update({"fixed": fixed, "best_fixed": {"variant": best[0], "gteps": best[1]},
                    "switched_vs_best_fixed": round(sw / best[1], 3) if best[1] > 0 else None})
        table[app] = row
    # hub sweeps of the tiered push (its CTA tier: lists of 256+ columns) with
    # 4-byte loads, int4 loads, or shared-memory chunks filled by TMA bulk
    # copies; GTEPS of the forced tiered variants on this graph
    hubs = {}
    for app in ("bfs", "sssp"):
        for cfg in ("Push-Queue-TWC-Standalone", "Push-Queue-TWC-Fused"):
            for name, hp in (("scalar", gs.HUB_SCALAR), ("vector", gs.HUB_VECTOR), ("staged_tma", gs.HUB_STAGED)):
                o = gs.RunOpts.from_config(cfg, hub_path=hp)
                hubs.setdefault(app, {}).setdefault(cfg, {})[name] = round(measure(app, o, 3)[0], 3)
    table["hub_paths"] = hubs
    table["definitions"] = {"bfs": "sum deg(reached)/2 / t", "sssp": "sum deg(reached)/2 / t", "cc": "m/2 / t",
                            "pr": f"m x {pr_iters} iterations / t", "unit": "GTEPS", "graph": "same RMAT as the headline"}
    gw.close()
    # batched multi-source BFS: 256 seeded sources in one bit-sliced run vs
    # 256 switched single-source runs
    if args.scale >= 22:
        gm = ctx.rmat(22, 16, 0.57, 0.19, 0.19, seed=1)
        src = gm.roots(77, 256)
        gm.mbfs(src, batched=True, out=False)
        _, stb = gm.mbfs(src, batched=True, out=False)
        _, sts = gm.mbfs(src, batched=False, opts=gs.RunOpts(selector=selector), out=False)
        table["mbfs_rmat22_256src"] = {"batched_gteps": round(stb.edges / (stb.ms * 1e6), 3),
                                       "sequential_switched_gteps": round(sts.edges / (sts.ms * 1e6), 3),
                                       "batched_vs_sequential": round(sts.ms / stb.ms, 3)}
        gm.close()
    table["er_batch_512"] = er_batch_entry(ctx, gs, selector)
    return table


def run_c3(args):
    import gswitch_b200 as gs
    from gswitch_b200.autotune import load_into
    from gswitch_b200.selector_train import load_model

    ctx = gs.Context(0)
    load_into(ctx, args.tune)
    selector = "rules"
    model, min_conf = load_model()
    if args.selector == "mlp" and model is not None:
        from gswitch_b200.selector_train import load_fusion_model

        ctx.mlp_load(model, min_conf)
        fmodel, fconf = load_fusion_model()
        if fmodel is not None:
            ctx.mlp_load_fusion(fmodel, fconf)
        selector = "mlp"
    print(json.dumps({"config": "C3", "selector": selector, "c3": c3_table(ctx, gs, selector)}))
    ctx.close()


def c3_table(ctx, gs, selector):
    """Config C3 (separate run, `--c3`): the 4096 x 4096 grid with 1%
    long-range edges (weights U[1, 1000]) for BFS, SSSP and BC, and RMAT
    scale 26 for BFS: the switched form against the fixed variants."""
    from gswitch_b200.selector_train import load_model

    model, _ = load_model()
    out = {}
    grid = ctx.grid(4096, 4096, 100, seed=1, wmax=1000, wseed=5)
    r26 = ctx.rmat(26, 16, 0.57, 0.19, 0.19, seed=1)

    def run(g, app, root, o):
        if app == "bfs":
            _, st = g.bfs(root, o, out=False)
        elif app == "sssp":
            _, st = g.sssp(root, o, out=False)
        else:
            _, _, st = g.bc(root, o, out=False)
        return st

    def measure(g, app, root, o):
        run(g, app, root, o)
        st = run(g, app, root, o)
        return {"ms": round(st.ms, 3), "gteps": round(st.edges / (st.ms * 1e6), 3), "levels": st.levels}

    for gname, g, apps in (("grid4096_lr100", grid, ("bfs", "sssp", "bc")), ("rmat26_ef16", r26, ("bfs",))):
        root = int(g.roots(1000, 1)[0])
        for app in apps:
            row = {"switched_rules": measure(g, app, root, gs.RunOpts()),
                   "switched_mlp": measure(g, app, root, gs.RunOpts(selector=selector))}
            fixed = {}
            for cfg in FIXED:
                fixed[cfg] = measure(g, app, root, gs.RunOpts.from_config(cfg))
            best = max(fixed.items(), key=lambda kv: kv[1]["gteps"])
            row.update({"fixed": {k: v["gteps"] for k, v in fixed.items()},
                        "best_fixed": {"variant": best[0], **best[1]},
                        "switched_vs_best_fixed": round(row["switched_mlp"]["gteps"] / best[1]["gteps"], 3)})
            if app in ("bfs", "sssp"):
                row["switch_headroom_standalone"] = switch_headroom(
                    g, gs.APP_BFS if app == "bfs" else gs.APP_SSSP, root, ctx=ctx, model=model)
            out[f"{app}_{gname}"] = row
    out["definitions"] = {"bfs/sssp/bc": "sum deg(reached)/2 / t (BC: both phases timed)", "unit": "GTEPS"}
    grid.close()
    r26.close()
    return out


def er_batch_entry(ctx, gs, selector):
    """Config C4's batch: 512 G(n, m) graphs, n log-uniform in [1e3, 2e5],
    mean degree uniform in [4, 32].  Batched: one BFS level loop over the
    disjoint union from one root per instance (and CC over the union);
    unbatched: each instance as its own graph, one BFS per graph."""
    gb, voff = ctx.er_batch(512, seed=7, nlo=1000, nhi=200000, dlo=4.0, dhi=32.0)
    off, col, _ = gb.download()
    parts, roots = [], []
    for i in range(512):
        a, b = int(voff[i]), int(voff[i + 1])
        o = off[a:b + 1] - off[a]
        c = col[off[a]:off[b]] - a
        h = ctx.upload(o, c)
        parts.append(h)
        roots.append(int(h.roots(11 + i, 1)[0]))
    groots = [int(voff[i]) + r for i, r in enumerate(roots)]
    o = gs.RunOpts(selector=selector)
    res = {"instances": 512, "vertices": int(gb.n), "arcs": int(gb.m)}
    for name, oo in (("batched", o), ("batched_captured", gs.RunOpts(selector=selector, captured=True))):
        gb.bfs_multi(groots, oo, out=False)
        _, st = gb.bfs_multi(groots, oo, out=False)
        res[f"bfs_{name}_ms"] = round(st.ms, 3)
        res[f"bfs_{name}_gteps"] = round(st.edges / (st.ms * 1e6), 3)
    tot_ms, tot_e = 0.0, 0
    for h, r in zip(parts, roots):
        _, st = h.bfs(r, o, out=False)
        tot_ms += st.ms
        tot_e += st.edges
    res["bfs_unbatched_ms"] = round(tot_ms, 3)
    res["bfs_unbatched_gteps"] = round(tot_e / (tot_ms * 1e6), 3)
    res["bfs_batched_vs_unbatched"] = round(tot_ms / res["bfs_batched_ms"], 2)
    gb.cc(out=False)
    _, st = gb.cc(out=False)
    cc_un = 0.0
    for h in parts:
        _, s2 = h.cc(out=False)
        cc_un += s2.ms
    res.update({"cc_batched_ms": round(st.ms, 3), "cc_unbatched_ms": round(cc_un, 3),
                "cc_batched_vs_unbatched": round(cc_un / st.ms, 2)})
    for h in parts:
        h.close()
    gb.close()
    return res


def combine_ranks(dist, ms, edges, device):
    """The job's time and work over replicas: the max of the ranks' device
    times and the sum of their traversed edges.  Every rank calls it, in the
    same order; without a process group it returns its arguments."""
    if not dist:
        return ms, edges
    import torch

    t = torch.tensor([float(ms)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e = torch.tensor([float(edges)], device=device, dtype=torch.float64)
    dist.all_reduce(e, op=dist.ReduceOp.SUM)
    return float(t.item()), int(e.item())


def e2e(ctx, g, roots, gs, torch, selector="rules"):
    """BFS through the C ABI with host buffers: upload (pinned CSR) + BFS +
    levels back to host, per step.  Returns (device ms, traversed edges,
    steps, host-to-device bytes per step, device-to-host bytes per step)."""
    off, col, _ = g.download()
    poff = torch.from_numpy(off).pin_memory().numpy()
    pcol = torch.from_numpy(col).pin_memory().numpy()
    plev = torch.empty(g.n, dtype=torch.int32).pin_memory().numpy()
    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    edges = 0
    torch.cuda.synchronize()
    e0.record(stream)
    for r in roots:
        h = ctx.upload(poff, pcol)
        st = h._run(gs.lib().gsw_bfs, gs.C.c_int32(int(r)), outs=[plev], opts=gs.RunOpts(selector=selector))
        edges += st.edges
        h.close()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return ms, edges, len(roots), int(poff.nbytes + pcol.nbytes), int(plev.nbytes)


def e2e_resident(ctx, g, roots, gs, torch, selector="rules"):
    """BFS queries on a graph already on the device, through the C ABI: per
    step the root goes in (a scalar argument) and the levels come back to a
    pinned host buffer, the work the reference arm times per root (its
    bfs_cpu on a CSR already in memory).  Returns (device ms, traversed edges,
    steps, device-to-host bytes per step)."""
    plev = torch.empty(g.n, dtype=torch.int32).pin_memory().numpy()
    stream = torch.cuda.ExternalStream(ctx.stream_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    edges = 0
    torch.cuda.synchronize()
    e0.record(stream)
    for r in roots:
        st = g._run(gs.lib().gsw_bfs, gs.C.c_int32(int(r)), outs=[plev], opts=gs.RunOpts(selector=selector))
        edges += st.edges
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), edges, len(roots), int(plev.nbytes)


def cpu_baseline(g, roots, budget_s, gpu_levels=None):
    """The oracle BFS (restated bfs_cpu) on the bench graph, one core, timed
    over about budget_s of runs from the given roots.  As the checker it also
    compares its levels with the GPU's for the roots in gpu_levels (the
    bench's first timed roots, run again through the same switched form with
    the levels copied back): returns (cpu_baseline entry, parity entry)."""
    import oracle

    off, col, _ = g.download()
    h = oracle.Csr(off, col)
    gpu_levels = gpu_levels or {}
    t_total, e_total, runs = 0.0, 0, 0
    checked, mismatches = [], 0
    for r in roots:
        t = time.perf_counter()
        lv = oracle.bfs(h, int(r))
        t_total += time.perf_counter() - t
        e_total += oracle.traversed_edges(h, lv)
        runs += 1
        if int(r) in gpu_levels:
            mismatches += int(np.count_nonzero(gpu_levels[int(r)] != lv))
            checked.append(int(r))
        if t_total >= budget_s and len(checked) == len(gpu_levels):
            break
    base = {"value": round(e_total / (t_total * 1e9), 5), "unit": "GTEPS", "cores": 1, "kind": "port",
            "sample": f"{runs} full BFS runs on the same graph (oracle restatement of application/bfs.cu:38-62), "
                      f"{t_total:.1f} s", "cpu": cpu_model(), "nproc": os.cpu_count()}
    parity = {"bfs_roots_checked": checked, "bfs_mismatches": mismatches, "vertices_per_root": int(h.n),
              "against": "oracle bfs (restated application/bfs.cu:38-62) on the downloaded bench graph"}
    return base, parity


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_bfs")
    W, K = args.warmup, args.steps
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_bfs was not built (reference tree absent at build time)"}))
        return
    import oracle

    t0 = time.time()
    h = oracle.rmat(args.scale, args.ef, seed=1)
    roots = oracle.roots(h, 1000, W + K)
    tmpdir = "/dev/shm" if os.path.isdir("/dev/shm") else tempfile.gettempdir()
    gp = os.path.join(tmpdir, f"gsw_ref_graph_{os.getpid()}.bin")
    rp = gp + ".roots"
    with open(gp, "wb") as f:
        np.array([h.n, h.m], dtype=np.int64).tofile(f)
        np.array([0, 0], dtype=np.int32).tofile(f)
        h.off.tofile(f)
        h.col.tofile(f)
    roots.astype(np.int32).tofile(rp)
    del h
    prep = time.time() - t0
    # all the host threads this process may use, each running the reference's
    # single-threaded bfs_cpu on its own root over the shared CSR
    threads = max(1, len(os.sched_getaffinity(0)))
    try:
        res = subprocess.run([exe, gp, "/dev/null", "--bench", rp, str(threads), str(W)], capture_output=True,
                             text=True, check=True)
    finally:
        for p in (gp, rp):
            if os.path.exists(p):
                os.unlink(p)
    if threads > 1:
        line = [x.split() for x in res.stdout.splitlines() if x.startswith("timed ")][0]
        ms, edges = float(line[2]), int(line[3])
    else:
        rows = [x.split() for x in res.stdout.splitlines() if len(x.split()) == 3]
        timed = rows[W:W + K]
        ms = sum(float(r[1]) for r in timed)
        edges = sum(int(r[2]) for r in timed)
    value = edges / (ms * 1e6)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 5), "unit": "GTEPS", "n_gpus": 1, "steps": K,
        "warmup": W, "ms_per_step": round(ms / max(K, 1), 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": f"bfs_rmat{args.scale}_ef{args.ef}", "scale": args.scale, "edge_factor": args.ef,
                   "seed": 1, "roots": "seeded non-isolated, one per step", "graph_prep_s": round(prep, 1)},
        "cpu_baseline": {"value": round(value, 5), "unit": "GTEPS", "cores": threads, "kind": "reference",
                         "sample": f"{K} reference bfs_cpu runs (application/bfs.cu:38-62 built from its sources), "
                                   f"{threads} at a time on {threads} threads sharing the CSR; wall time",
                         "cpu": cpu_model(), "nproc": os.cpu_count()},
        "e2e": {"value": round(value, 5), "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


PROFILE_CASES = {
    "bfs": "three BFS runs on RMAT scale 22 (ef 16, seed 1), learned selector",
    "bfs24": "one BFS on RMAT scale 24 (ef 16, seed 1: the bench graph), learned selector",
    "bfs24cap": "one BFS on the bench graph, learned selector, through the captured level loop",
    "sssp": "SSSP on the 4096 x 4096 grid with 1% long-range edges (weights U[1, 1000]), "
            "Push-Queue-WM-Fused levels one launch each",
    "pr": "two PageRank iterations on RMAT scale 22, Pull-Bitmap-STRICT then 2D",
    "mbfs": "batched 256-source BFS on RMAT scale 20",
    "twc24": "one BFS on RMAT scale 24 with the tiered push forced at every level (hub pieces swept one per "
             "CTA, staged in shared memory by TMA bulk copies)",
    "strict24": "one BFS on RMAT scale 24 with the edge-balanced (STRICT) push forced at every level",
    "cm24": "one BFS on RMAT scale 24 with the CTA-mapped (CM) push forced at every level",
    "bc20": "batched BC from 32 sources on RMAT scale 20 (one cooperative launch)",
}


def run_case(case: str) -> None:
    """Small fixed workloads for profiler captures (ncu -k <kernel> python
    bench.py --case <case>); they print no bench line."""
    import gswitch_b200 as gs
    from gswitch_b200.selector_train import load_model

    if case not in PROFILE_CASES:
        raise SystemExit(f"unknown case {case!r} ({', '.join(PROFILE_CASES)})")
    ctx = gs.Context(0)
    model, conf = load_model()
    if model is not None:
        ctx.mlp_load(model, conf)
    if case == "bfs":
        g = ctx.rmat(22, 16, seed=1)
        for r in g.roots(1000, 3):
            g.bfs(int(r), gs.RunOpts(selector="mlp"), out=False)
    elif case in ("bfs24", "bfs24cap"):
        g = ctx.rmat(24, 16, seed=1)
        g.bfs(int(g.roots(1000, 1)[0]), gs.RunOpts(selector="mlp", captured=case == "bfs24cap"), out=False)
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
    elif case in ("twc24", "strict24", "cm24"):
        g = ctx.rmat(24, 16, seed=1)
        cfg = {"twc24": "Push-Queue-TWC-Standalone", "strict24": "Push-Queue-STRICT-Standalone",
               "cm24": "Push-Queue-CM-Standalone"}[case]
        g.bfs(int(g.roots(1000, 1)[0]), gs.RunOpts.from_config(cfg), out=False)
    elif case == "bc20":
        g = ctx.rmat(20, 16, seed=1)
        g.bc_batch(g.roots(99, 32), out=False)
    print("ok", case)
    g.close()
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--ef", type=int, default=16)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--selector", default="mlp", choices=["mlp", "rules"])
    ap.add_argument("--no-apps", action="store_true")
    ap.add_argument("--c3", action="store_true", help="print config C3's switched-vs-fixed table instead")
    ap.add_argument("--tune", default=None, help="tuning table to load (default: the committed one)")
    ap.add_argument("--case", choices=sorted(PROFILE_CASES),
                    help="run one small fixed workload for a profiler capture instead of the bench")
    args = ap.parse_args()
    if args.case:
        return run_case(args.case)
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.c3:
        run_c3(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
