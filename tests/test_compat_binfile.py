"""The drop-in header's binary CSR cache (host_graph_t::store_to_binfile /
load_from_binfile, the reference's src/utils/fileIO.cuh:334-387): the byte
layout is the reference's, and a stored graph loads back array for array.
Host code only: compiled with nvcc, run on the CPU."""
import os
import struct
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROG = r"""
#include "gswitch.h"
template <typename E>
static int check(const char *mtx, bool directed, bool weighted) {
  edgelist_t<E> el;
  el.read_mtx(mtx, directed, weighted, false);
  host_graph_t<CSR, E> a, b;
  a.build(el);
  a.store_to_binfile(mtx);
  b.load_from_binfile(mtx);
  auto same = [](const int *x, const int *y, int k) { return std::equal(x, x + k, y); };
  bool ok = a.nvertexs == b.nvertexs && a.nedges == b.nedges && a.directed == b.directed &&
            a.with_weight == b.with_weight && same(a.odegrees, b.odegrees, a.nvertexs) &&
            same(a.start_pos, b.start_pos, a.nvertexs + 1) && same(a.adj_list, b.adj_list, a.nedges);
  if constexpr (!std::is_same<E, Empty>::value)
    ok = ok && std::equal(a.edge_weights, a.edge_weights + a.nedges, b.edge_weights);
  if (directed)
    // the file keeps n start positions per side (rinse renumbers only the
    // forward side, as the reference's does, so the reverse end marker is not
    // part of what round-trips)
    ok = ok && same(a.r_odegrees, b.r_odegrees, a.nvertexs) && same(a.r_start_pos, b.r_start_pos, a.nvertexs) &&
         same(a.r_adj_list, b.r_adj_list, a.nedges);
  printf("%d %d %d\n", ok ? 1 : 0, a.nvertexs, a.nedges);
  return ok ? 0 : 1;
}
int main(int argc, char **argv) {
  const int mode = atoi(argv[2]);
  if (mode == 0) return check<Empty>(argv[1], false, false);
  if (mode == 1) return check<int>(argv[1], false, true);
  return check<Empty>(argv[1], true, false);
}
"""


@pytest.fixture(scope="module")
def prog():
    from gswitch_b200.compat.build_apps import FLAGS, NVCC

    d = tempfile.mkdtemp()
    src = os.path.join(d, "binfile.cu")
    open(src, "w").write(PROG)
    exe = os.path.join(d, "binfile")
    r = subprocess.run([NVCC, *FLAGS, "-o", exe, src], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return exe


def _mtx(d, name, weighted, seed):
    rng = np.random.default_rng(seed)
    src = rng.integers(1, 200, 1500)
    dst = rng.integers(1, 200, 1500)
    p = os.path.join(d, name)
    with open(p, "w") as f:
        f.write("% synthetic\n")
        for a, b in zip(src, dst):
            f.write(f"{a} {b} {int(rng.integers(1, 64))}\n" if weighted else f"{a} {b}\n")
    return p


@pytest.mark.parametrize("mode,weighted", [(0, False), (1, True), (2, False)])
def test_binfile_round_trip_and_layout(prog, mode, weighted):
    with tempfile.TemporaryDirectory() as d:
        mtx = _mtx(d, "g.mtx", weighted, 5 + mode)
        r = subprocess.run([prog, mtx, str(mode)], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        ok, n, m = map(int, r.stdout.split())
        assert ok == 1
        cache = os.path.join(d, ".csr_g.mtx")
        raw = open(cache, "rb").read()
        directed = mode == 2
        side = 4 * n + 4 * n + 4 * m + (4 * m if weighted else 0)
        assert len(raw) == 4 + 4 + 1 + 1 + side * (2 if directed else 1)
        assert struct.unpack("<iibb", raw[:10]) == (n, m, int(directed), int(weighted))
        # a second store leaves the existing cache untouched
        os.utime(cache, (1, 1))
        r = subprocess.run([prog, mtx, str(mode)], capture_output=True, text=True)
        assert r.returncode == 0 and os.path.getmtime(cache) == 1
