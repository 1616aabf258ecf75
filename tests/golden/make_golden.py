"""Regenerates the golden fixtures in this folder.

Every expected output comes from the REFERENCE's own CPU validators, compiled
from its sources by ``oracle/ref/build_ref.sh`` into ``oracle/_ref/``
(``bfs_cpu`` application/bfs.cu:38-62, ``spfa`` sssp.cu:55-89, ``CC_CPU``
cc.cu:34-66, ``bc_cpu`` bc.cu:162-214, the PageRank and colouring
validations pagerank.cu:44-79 and gc.cu:45-74, ``graph_attr_t::fill``
src/utils/fileIO.cuh:35-67).  The script also asserts that the oracle
restatement reproduces each of them, so a fixture is never written from an
unpinned oracle.  Needs the reference tree (only present where it is
mounted): ``python tests/golden/make_golden.py``.
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")


def small_cases():
    """name -> (Csr, root, weight seed, weight max)"""
    o = oracle
    cases = {}
    n = 10
    cases["path10"] = (o.csr_from_pairs(n, np.arange(n - 1), np.arange(1, n)), 0)
    cases["star13"] = (o.csr_from_pairs(13, np.zeros(12), np.arange(1, 13)), 5)
    cases["cycle9"] = (o.csr_from_pairs(9, np.arange(9), (np.arange(9) + 1) % 9), 0)
    s = [0, 1, 2, 3, 6, 7, 8, 9, 6]
    d = [1, 2, 3, 4, 7, 8, 9, 6, 8]
    cases["twocomp_isolated"] = (o.csr_from_pairs(12, s, d), 6)
    s = [0, 0, 1, 1, 2, 2, 3, 3, 4, 5, 5, 0]
    d = [1, 1, 0, 1, 3, 3, 2, 4, 4, 0, 2, 5]  # duplicates, reversed dups, self-loops
    cases["dups_selfloops"] = (o.csr_from_pairs(6, s, d), 2)
    g = o.rmat(10, 16, seed=1)
    cases["rmat10"] = (g, 0)
    g = o.grid(24, 24, 100, seed=3)
    cases["grid24_lr"] = (g, int(o.roots(g, 3, 1)[0]))
    g = o.er(1500, 6000, seed=5)
    cases["er1500"] = (g, int(o.roots(g, 5, 1)[0]))
    return cases


def write_graph(path, g, root, w=None):
    with open(path, "wb") as f:
        np.array([g.n, g.m], dtype=np.int64).tofile(f)
        np.array([1 if w is not None else 0, root], dtype=np.int32).tofile(f)
        g.off.tofile(f)
        g.col.tofile(f)
        if w is not None:
            w.tofile(f)


def run(app, graph, out, extra=None):
    cmd = [os.path.join(REF, "ref_" + app), graph, out] + ([extra] if extra else [])
    return subprocess.run(cmd, check=True, capture_output=True, text=True).stdout


def greedy_colors(g):
    col = np.full(g.n, -1, dtype=np.int32)
    for v in range(g.n):
        used = {int(col[u]) for u in g.col[g.off[v]:g.off[v + 1]]}
        c = 0
        while c in used:
            c += 1
        col[v] = c
    return col


def main():
    subprocess.check_call([os.path.join(ROOT, "oracle", "ref", "build_ref.sh")],
                          stdout=subprocess.DEVNULL)
    oracle.build()
    tmp = tempfile.mkdtemp()
    for name, (g, root) in small_cases().items():
        wmax = 1000 if name.startswith("grid") else 64
        gw = oracle.add_weights(g, 11, wmax)
        gp, op = os.path.join(tmp, "g.bin"), os.path.join(tmp, "o.bin")
        ap = os.path.join(tmp, "a.bin")
        write_graph(gp, g, root)
        run("bfs", gp, op, ap)
        lvl = np.fromfile(op, dtype=np.int32)
        attr = np.fromfile(ap, dtype=np.float64)
        run("cc", gp, op)
        cc = np.fromfile(op, dtype=np.int32)
        run("bc", gp, op)
        bc = np.fromfile(op, dtype=np.int32).reshape(-1, 2)
        bc_nsp, bc_dep = bc[:, 0].copy(), bc[:, 1].copy().view(np.float32)
        write_graph(gp, gw, root, gw.w)
        run("sssp", gp, op)
        dist = np.fromfile(op, dtype=np.int32)

        # pin the oracle against every reference output
        assert np.array_equal(oracle.bfs(g, root), lvl), name
        assert np.array_equal(oracle.cc(g), cc), name
        nsp, dep = oracle.bc_f32(g, root)
        assert np.array_equal(nsp, bc_nsp) and np.array_equal(dep, bc_dep), name
        assert np.array_equal(oracle.sssp_spfa(gw, root), dist), name
        assert np.array_equal(oracle.sssp_dijkstra(gw, root), dist), name
        assert np.array_equal(oracle.degree_attr(g), attr), name

        # PageRank fix-point validation: a converged vector passes, a
        # perturbed one fails at the same vertex in both implementations
        write_graph(gp, g, root)
        pr = oracle.pagerank(g, 300, 0.85)
        od = g.degrees().astype(np.float64)
        pr_od = np.where(od > 0, pr / np.maximum(od, 1), pr).astype(np.float32)
        vp = os.path.join(tmp, "v.bin")
        verdicts = []
        for k, vec in enumerate([pr_od, pr_od * np.where(np.arange(g.n) == g.n // 2, 1.5, 1.0).astype(np.float32)]):
            vec.astype(np.float32).tofile(vp)
            out = run("pr", gp, op, vp)
            ref_ok = "passed" in out
            mine = oracle.pagerank_check(g, vec)
            assert ref_ok == (mine < 0), (name, k, out, mine)
            verdicts.append(int(ref_ok))
        # colouring validation
        gcv = []
        col = greedy_colors(g)
        bad = col.copy()
        for v in range(g.n):
            if g.off[v + 1] > g.off[v]:
                bad[v] = bad[g.col[g.off[v]]]
                break
        for vec in (col, bad):
            vec.tofile(vp)
            out = run("gc", gp, op, vp)
            ref_ok = "passed" in out
            assert ref_ok == (oracle.gc_check(g, vec) < 0), (name, out)
            gcv.append(int(ref_ok))

        np.savez_compressed(
            os.path.join(HERE, name + ".npz"), off=g.off, col=g.col, w=gw.w,
            root=np.int32(root), lvl=lvl, cc=cc, bc_nsp=bc_nsp, bc_dep=bc_dep,
            dist=dist, attr=attr, pr_vec=pr_od, pr_verdicts=np.array(verdicts),
            gc_colors=col, gc_bad=bad, gc_verdicts=np.array(gcv))
        print(f"{name}: n={g.n} m={g.m} root={root} pinned")


if __name__ == "__main__":
    main()
