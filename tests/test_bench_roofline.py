"""bench.py's roofline arithmetic on synthetic level traces (CPU): the
dominant kernel is the one with the most event time, achieved = algorithmic
bytes / time, frac = achieved / peak, traffic comes from the ncu figures for
the kernels that have one, and every other kernel above a tenth of the time
gets its own line."""
import os
import sys
from types import SimpleNamespace

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _run(trace, level_ms, inspect_ms, level_edges):
    timed = SimpleNamespace(trace=trace, level_ms=level_ms, level_inspect_ms=inspect_ms)
    acc = SimpleNamespace(level_edges=level_edges)
    return timed, acc


def test_level_bytes_push_and_pull():
    n = 1 << 10
    # push, queue: 4 B work item + 16 B offsets per frontier vertex, 4.25 B per edge, 4 B per discovery
    assert bench.level_bytes(("Push", "Queue", "TM", "Standalone"), n, A=10, U=0, D=7, E=100) == 40 + 160 + 425 + 28
    # pull, bitmap: n/8 B of status words + 16 B per candidate + 4.125 B per scanned edge + 4 B per discovery
    assert bench.level_bytes(("Pull", "Bitmap", "TM", "Standalone"), n, A=0, U=50, D=20, E=80) == 128 + 800 + 330 + 80


def test_roofline_dominant_kernel_traffic_and_others():
    n = 1 << 24
    trace = [("Push", "Queue", "WM", "Standalone", 1), ("Pull", "Bitmap", "TM", "Standalone", n),
             ("Push", "Queue", "WM", "Fused", -1)]
    # levels: root at 0, 1000 at 1, the rest at 2, none unreached
    lv = np.full(n, 2, dtype=np.int32)
    lv[0] = 0
    lv[1:1001] = 1
    runs = [(*_run(trace, [0.01, 0.30, 0.02], [0.0, 0.04, 0.04], [16000, 900000, 10]), lv)]
    r = bench.roofline_from(runs, n, peak_gbs=6500.0, peak_kind="measured")
    assert r["kernel"] == "expand Pull-Bitmap-TM-Standalone"
    U = n - 1001  # candidates of the pull level: everything past level 1
    want = n / 8 + 16 * U + 4.125 * 900000 + 4 * U
    assert abs(r["bytes_per_launch"] - want) <= 1
    assert abs(r["achieved"] - want / 0.30e-3 / 1e9) < 0.1
    assert abs(r["frac"] - r["achieved"] / 6500.0) < 1e-4
    assert r["traffic"] == round(bench.PULL_TM_TRAFFIC_RMAT24)  # the bench graph's size
    assert abs(sum(r["time_shares"].values()) - 1) < 1e-3
    others = {o["kernel"]: o for o in r["others"]}
    assert set(others) == {"inspect"}  # 0.08 of 0.41 ms; the other expands are below a tenth
    ins = others["inspect"]
    assert ins["launches"] == 2 and ins["traffic"] == round(bench.INSPECT_TRAFFIC_PER_VERTEX * n)
    assert abs(ins["bytes_per_launch"] - (8 * n + n / 4)) <= 1


def test_roofline_traffic_is_null_off_the_bench_graph():
    n = 1 << 20
    trace = [("Pull", "Bitmap", "TM", "Standalone", n)]
    lv = np.zeros(n, dtype=np.int32)
    r = bench.roofline_from([(*_run(trace, [0.1], [0.0], [1000]), lv)], n, 6500.0, "measured")
    assert r["traffic"] is None and "no per-launch ncu figure" in r["traffic_note"]
