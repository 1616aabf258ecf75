"""The reference's own application mains (application/*.cu), compiled
unchanged against gswitch_b200/compat/gswitch.h, run on this engine and
pass their own CPU validation (-V) on .mtx exports of the golden graphs, for
the selector's choices and for forced variants (-c)."""
import os
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
