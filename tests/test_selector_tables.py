"""The selector's decision-tree tables (converted from the reference's
trained trees by gswitch_b200/csrc/engine/gen_selector_trees.py) evaluate
exactly like the reference's generated if/else code.  The comparison
compiles the reference tree headers in place when the reference tree is
mounted; the table structure checks run everywhere."""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TABLES = os.path.join(ROOT, "gswitch_b200", "csrc", "engine", "selector_trees.h")
from gswitch_b200.compat import reference_tree

REF_MODEL = os.path.join(reference_tree(), "src", "model")
TREES = ["select_dir_idem", "select_dir_asso", "select_dir_asso_backup", "select_fmt", "select_fusion",
         "select_lb_idem", "select_lb_asso_forward", "select_lb_asso_forward_backup", "select_lb_asso_backward",
         "select_lb_asso_backward_backup", "select_stepping"]


def load_tables():
    txt = open(TABLES).read()
    out = {}
    for name in TREES:
        body = txt[txt.index(f"{name}_tree["):]
        body = body[body.index("{") + 1: body.index("};")]
        rows = re.findall(r"\{(-?\d+), ([-0-9.eE+]+), (-?\d+), (-?\d+)\}", body)
        out[name] = [(int(a), float(b), int(c), int(d)) for a, b, c, d in rows]
    return out


def eval_table(t, fv):
    i = 0
    while t[i][0] >= 0:
        i = t[i][2] if fv[t[i][0]] <= t[i][1] else t[i][3]
    return t[i][2]


def test_tables_are_well_formed():
    for name, t in load_tables().items():
        assert len(t) % 2 == 1, name  # full binary tree
        leaves = [r for r in t if r[0] < 0]
        assert len(leaves) == (len(t) + 1) // 2, name
        for f, thr, l, r in t:
            if f >= 0:
                assert 0 < l < len(t) and 0 < r < len(t)


@pytest.mark.skipif(not os.path.isdir(REF_MODEL), reason="reference tree not mounted")
def test_tables_match_reference_trees():
    tables = load_tables()
    rng = np.random.default_rng(7)
    nfeat = {k: 1 + max(r[0] for r in v) for k, v in tables.items()}
    nvec = 400
    tmp = tempfile.mkdtemp()
    src = os.path.join(tmp, "t.cpp")
    lines = ["#include <cstdio>", "#include <vector>"]
    lines += [f'#include "{REF_MODEL}/{n}.h"' for n in TREES]
    lines.append("int main(){ int n; double x; while (scanf(\"%d\", &n)==1) { std::vector<double> v;"
                 " for(int i=0;i<n;++i){scanf(\"%lf\",&x); v.push_back(x);} int t; scanf(\"%d\",&t); int r=-1;")
    for k, n in enumerate(TREES):
        lines.append(f"  if (t=={k}) r = {n}(v);")
    lines.append("  printf(\"%d\\n\", r);} }")
    open(src, "w").write("\n".join(lines))
    exe = os.path.join(tmp, "t")
    subprocess.check_call(["g++", "-O1", "-o", exe, src])
    inp, expect = [], []
    for k, name in enumerate(TREES):
        t = tables[name]
        thr = [r[1] for r in t if r[0] >= 0]
        for _ in range(nvec):
            fv = rng.choice(thr + [0.0, 1e9], size=nfeat[name]) * rng.choice([0.5, 1.0, 1.0, 2.0], size=nfeat[name])
            inp.append(f"{nfeat[name]} " + " ".join(repr(float(x)) for x in fv) + f" {k}")
            expect.append(eval_table(t, fv))
    out = subprocess.run([exe], input="\n".join(inp), capture_output=True, text=True, check=True).stdout.split()
    assert [int(x) for x in out] == expect
