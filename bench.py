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
               average CUDA-event duration in the timed region, against the
               measured HBM copy bandwidth;
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

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
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
        for line in open(self.path):
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
    """Algorithmic bytes of one expand (int32 levels, bitmap state probes):
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
    dom = max(per.items(), key=lambda kv: kv[1][0])
    name, (ms, byt, launches) = dom
    achieved = byt / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
    shares = {k: round(v[0] / sum(x[0] for x in per.values()), 4) for k, v in per.items()}
    return {"bound": "hbm", "kernel": name, "achieved": round(achieved, 1), "peak": peak_gbs,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak_gbs, 4),
            "bytes_per_launch": round(byt / max(launches, 1)), "launches": launches,
            "avg_launch_ms": round(ms / max(launches, 1), 5), "traffic": None, "time_shares": shares}


def run_ours(args):
    import torch

    import gswitch_b200 as gs

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
    t0 = time.time()
    g = ctx.rmat(args.scale, args.ef, 0.57, 0.19, 0.19, seed=1)
    gen_s = time.time() - t0
    W, K = args.warmup, args.steps
    roots = g.roots(1000 + rank, W + K)
    for r in roots[:W]:
        g.bfs(int(r), out=False)

    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local)
    timed = []
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    e0.record(stream)
    edges = 0
    launches = 0
    for r in roots[W:W + K]:
        _, st = g.bfs(int(r), opts=gs.RunOpts(timing=True), out=False)
        edges += st.edges
        launches += st.launches
        timed.append(st)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    barrier()
    ms_max, tot_edges = ms, edges
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
        t = torch.tensor([edges], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        tot_edges = int(t.item())
    value = tot_edges / (ms_max * 1e6)

    out = None
    if rank == 0:
        # accounting pass (untimed): same roots, edges touched per expand
        runs = []
        for r, st in zip(roots[W:W + K], timed):
            lv, acc = g.bfs(int(r), opts=gs.RunOpts(account=True))
            runs.append((st, acc, lv))
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
                       "parallelism": f"replicas x{world}", "selector": "rules (reference trees)",
                       "graph_build_s": round(gen_s, 2)},
            "roofline": roof, "gpu_launches": int(launches), "clocks": clocks,
            "levels_first_step": trace,
        }
        if not args.no_e2e:
            out["e2e"] = e2e(ctx, g, roots[W:W + K], gs, torch)
        if world == 1 and not args.no_cpu:
            out["cpu_baseline"] = cpu_baseline(g, roots, args.cpu_seconds)
    g.close()
    ctx.close()
    if dist:
        dist.destroy_process_group()
    if out:
        print(json.dumps(out))


def e2e(ctx, g, roots, gs, torch):
    """BFS through the C ABI with host buffers: upload (pinned CSR) + BFS +
    levels back to host, per step."""
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
        st = h._run(gs.lib().gsw_bfs, gs.C.c_int32(int(r)), outs=[plev], opts=None)
        edges += st.edges
        h.close()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return {"value": round(edges / (ms * 1e6), 3), "unit": "GTEPS", "ms_per_step": round(ms / len(roots), 3),
            "h2d_bytes_per_step": int(poff.nbytes + pcol.nbytes), "d2h_bytes_per_step": int(plev.nbytes)}


def cpu_baseline(g, roots, budget_s):
    import oracle

    off, col, _ = g.download()
    h = oracle.Csr(off, col)
    t_total, e_total, runs = 0.0, 0, 0
    for r in roots:
        t = time.perf_counter()
        lv = oracle.bfs(h, int(r))
        t_total += time.perf_counter() - t
        e_total += oracle.traversed_edges(h, lv)
        runs += 1
        if t_total >= budget_s:
            break
    return {"value": round(e_total / (t_total * 1e9), 5), "unit": "GTEPS", "cores": 1, "kind": "port",
            "sample": f"{runs} full BFS runs on the same graph (oracle restatement of application/bfs.cu:38-62), "
                      f"{t_total:.1f} s", "cpu": cpu_model(), "nproc": os.cpu_count()}


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
    try:
        res = subprocess.run([exe, gp, "/dev/null", "--bench", rp], capture_output=True, text=True, check=True)
    finally:
        for p in (gp, rp):
            if os.path.exists(p):
                os.unlink(p)
    rows = [line.split() for line in res.stdout.splitlines() if len(line.split()) == 3]
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
        "cpu_baseline": {"value": round(value, 5), "unit": "GTEPS", "cores": 1, "kind": "reference",
                         "sample": f"{K} reference bfs_cpu runs (application/bfs.cu:38-62 built from its sources)",
                         "cpu": cpu_model(), "nproc": os.cpu_count()},
        "e2e": {"value": round(value, 5), "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--ef", type=int, default=16)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
