"""The reference's own application mains (application/*.cu), compiled
unchanged against gswitch_b200/compat/gswitch.h, run on this engine and
pass their own CPU validation (-V) on .mtx exports of the golden graphs, for
the selector's choices and for forced variants (-c)."""
import json
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "gswitch_b200", "compat", "_bin")
GRAPHS = ["rmat10", "grid24_lr", "er1500", "path10", "cycle9"]


def write_mtx(path, off, col):
    """Each undirected pair once, 1-based ids, no header."""
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern symmetric\n")
        for v in range(len(off) - 1):
            for u in col[off[v]:off[v + 1]]:
                if v < u:
                    f.write(f"{v + 1} {u + 1}\n")


@pytest.fixture(scope="module")
def mtx(tmp_path_factory):
    d = tmp_path_factory.mktemp("mtx")
    out = {}
    for name in GRAPHS:
        g = load_golden(name)
        p = str(d / f"{name}.mtx")
        write_mtx(p, g["off"], g["col"])
        out[name] = p
    return out


def run(app, path, *args):
    exe = os.path.join(BIN, app)
    if not os.path.exists(exe):
        pytest.fail(f"{exe} is not built (gswitch_b200/compat/build_apps.py)")
    r = subprocess.run([exe, path, "-V", "-r", "0", *args], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (app, r.returncode, r.stdout[-500:], r.stderr[-500:])
    return r.stdout


@pytest.mark.parametrize("name", GRAPHS)
@pytest.mark.parametrize("app,expect", [("bfs", ["passed"]), ("sssp", ["passed"]), ("cc", ["passed"]),
                                        ("pagerank", ["passed"]), ("gc", ["passed"]), ("mbfs", ["passed"]),
                                        ("bc", ["Forward passed"])])
def test_reference_app_passes_its_own_validation(mtx, name, app, expect):
    """BC: only the forward check.  The app's backward phase starts from the
    level its forward loop stopped at and never credits the root, so its own
    backward check fails on its own engine as well (reference bc built from
    its sources, same files, same roots: forward and backward both fail);
    this engine's BC runner (gsw_bc) is checked against the oracle in
    test_gpu_apps."""
    out = run(app, mtx[name])
    if app != "bc":
        assert "failed" not in out, (app, name, out[-400:])
    for e in expect:
        assert e in out, (app, name, out[-400:])


@pytest.mark.parametrize("cfg", ["Push-Queue-TM-Standalone", "Push-Queue-STRICT-Fused", "Pull-Bitmap-WM-Standalone",
                                 "Push-Bitmap-TWC-Standalone", "Pull-Queue-CM-Standalone"])
def test_reference_bfs_and_sssp_with_forced_variants(mtx, cfg):
    for app in ("bfs", "sssp"):
        out = run(app, mtx["rmat10"], "-c", cfg)
        assert "passed" in out and "failed" not in out, (app, cfg, out[-400:])


# feature records: the reference's bfs.cu with its training hook enabled
# (built by gswitch_b200/compat/build_apps.py as bfs_record) writes the
# layout of src/abstraction/features.cuh:86-104 / src/utils/json.cuh:34-48 to
# the -j file: one "{ ... }" block of keys "0".."22" per level, at most 100
BLOCK = re.compile(r'\{\n(?:"(\d+)": [^,\n]+,\n){22}"22": [^,\n]+\n\}\n')


def parse_records(text):
    """The blocks of a record file; values are what a C++ stream prints for
    a double, so "nan" / "inf" (a ratio of two zero times) map to JSON's."""
    blocks, pos = [], 0
    while pos < len(text):
        m = BLOCK.match(text, pos)
        assert m, text[pos:pos + 200]
        body = "{" + text[m.start() + 1:m.end() - 2].replace("\n", " ") + "}"
        body = re.sub(r": (-?)nan\b", ": NaN", body)
        body = re.sub(r": (-?)inf\b", r": \1Infinity", body)
        blocks.append(json.loads(body))
        pos = m.end()
    return blocks


def test_feature_records_from_reference_bfs(mtx, tmp_path):
    out = tmp_path / "rec.json"
    run("bfs_record", mtx["rmat10"], "-j", str(out))
    recs = parse_records(out.read_text())
    assert len(recs) >= 3
    g = load_golden("rmat10")
    n, nonisolated = len(g["off"]) - 1, int((np.diff(g["off"]) > 0).sum())
    for r in recs:
        assert sorted(r, key=int) == [str(i) for i in range(23)]
        # graph constants (vertex and edge counts as the app read the file)
        assert (r["0"], r["1"]) == (recs[0]["0"], recs[0]["1"])
        assert nonisolated <= r["0"] <= n


def test_feature_records_stop_at_100_per_run(tmp_path):
    n = 300  # a path: one level per vertex from vertex 0
    p = tmp_path / "path.mtx"
    with open(p, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern symmetric\n")
        for v in range(1, n):
            f.write(f"{v} {v + 1}\n")
    out = tmp_path / "rec.json"
    # standalone levels, one loop iteration (and one record) per level
    run("bfs_record", str(p), "-j", str(out), "-c", "Push-Queue-WM-Standalone")
    recs = parse_records(out.read_text())
    assert len(recs) == 100
    assert all(r["7"] == 1 for r in recs)  # one active vertex per level


def test_feature_records_through_the_c_abi(ctx, tmp_path):
    import gswitch_b200 as gs
    import oracle

    h = oracle.csr_from_pairs(150, np.arange(149), np.arange(1, 150))
    g = ctx.upload(h.off, h.col)
    out = tmp_path / "abi.json"
    ctx.record_features(str(out))
    try:
        lv, st = g.bfs(0, gs.RunOpts.from_config("Push-Queue-WM-Standalone"))
        recs = parse_records(out.read_text())
        assert len(recs) == min(st.levels, 100)
        assert all(r["0"] == 150 and r["7"] == 1 for r in recs)
        g.bfs(0, gs.RunOpts.from_config("Push-Queue-WM-Standalone"))  # a new run has its own 100
        assert len(parse_records(out.read_text())) == 2 * min(st.levels, 100)
    finally:
        ctx.record_features(None)
    g.close()
