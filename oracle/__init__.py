"""CPU oracle (test infrastructure only).

ctypes binding of ``oracle/liboracle.so``: seeded graph generators, the
undirected CSR build, and restatements of the reference's CPU validators
(``application/bfs.cu:38-62``, ``sssp.cu:55-89``, ``cc.cu:34-66``,
``bc.cu:162-214``, ``pagerank.cu:44-79``, ``gc.cu:45-74``; degree statistics
``src/utils/fileIO.cuh:35-67``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the cpu_baseline leg of
``bench.py`` import this package, and only as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

I64P = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
I32P = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
U32P = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
F32P = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
F64P = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile liboracle.so (gcc) if it is missing or stale."""
    so = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "oracle.c")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return so


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    so = os.path.join(_HERE, "liboracle.so")
    if not os.path.exists(so):
        build()
    L = C.CDLL(so)
    i64, i32, u64, dbl = C.c_int64, C.c_int32, C.c_uint64, C.c_double
    L.or_sm64.restype = u64
    L.or_sm64.argtypes = [u64]
    L.or_rmat_edges.argtypes = [C.c_int, C.c_int, dbl, dbl, dbl, u64, U32P, U32P]
    L.or_grid_nedges.restype = i64
    L.or_grid_nedges.argtypes = [C.c_int, C.c_int, C.c_int]
    L.or_grid_edges.restype = i64
    L.or_grid_edges.argtypes = [C.c_int, C.c_int, C.c_int, u64, U32P, U32P]
    L.or_er_edges.argtypes = [i64, i64, u64, U32P, U32P]
    L.or_er_batch_params.argtypes = [u64, i64, i64, i64, dbl, dbl,
                                     C.POINTER(i64), C.POINTER(i64), C.POINTER(u64)]
    L.or_csr_build.restype = i64
    L.or_csr_build.argtypes = [i64, i64, U32P, U32P,
                               C.POINTER(C.POINTER(i64)), C.POINTER(C.POINTER(i32))]
    L.or_weights.argtypes = [u64, C.c_int, i64, I64P, I32P, I32P]
    L.or_roots.argtypes = [u64, i64, I64P, C.c_int, I32P]
    L.or_free.argtypes = [C.c_void_p]
    L.or_bfs.argtypes = [i64, I64P, I32P, i32, I32P]
    L.or_sssp_spfa.argtypes = [i64, I64P, I32P, I32P, i32, I32P]
    L.or_sssp_dijkstra.argtypes = [i64, I64P, I32P, I32P, i32, I32P]
    L.or_sssp_dial.restype = C.c_int
    L.or_sssp_dial.argtypes = [i64, I64P, I32P, I32P, i32, i32, I32P]
    L.or_cc.argtypes = [i64, I64P, I32P, I32P]
    L.or_cc_linear.argtypes = [i64, I64P, I32P, I32P]
    L.or_bc_f32.argtypes = [i64, I64P, I32P, i32, I32P, F32P]
    L.or_bc_f64.argtypes = [i64, I64P, I32P, i32, F64P, F64P, I32P]
    L.or_pagerank.argtypes = [i64, I64P, I32P, C.c_int, dbl, F64P]
    L.or_pagerank_check.restype = i64
    L.or_pagerank_check.argtypes = [i64, I64P, I32P, F32P, C.c_float, C.c_float]
    L.or_gc_check.restype = i64
    L.or_gc_check.argtypes = [i64, I64P, I32P, I32P]
    L.or_gc_levels.argtypes = [i64, I64P, I32P, I32P]
    L.or_mbfs.argtypes = [i64, I64P, I32P, C.c_int, I32P, I32P]
    L.or_degree_attr.argtypes = [i64, I64P, F64P]
    L.or_traversed_edges.restype = i64
    L.or_traversed_edges.argtypes = [i64, I64P, I32P]
    L.or_inspect_bfs.argtypes = [i64, I64P, I32P, i32, np.ctypeslib.ndpointer(np.uint64, flags="C")]
    _LIB = L
    return L


class Csr:
    """Host CSR: int64 offsets (n+1), int32 columns (m), optional int32 weights."""

    def __init__(self, off, col, w=None):
        self.off = np.ascontiguousarray(off, dtype=np.int64)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        self.w = None if w is None else np.ascontiguousarray(w, dtype=np.int32)

    @property
    def n(self) -> int:
        return len(self.off) - 1

    @property
    def m(self) -> int:
        return len(self.col)

    def degrees(self):
        return np.diff(self.off).astype(np.int32)


def csr_from_pairs(n, src, dst) -> Csr:
    L = lib()
    src = np.ascontiguousarray(src, dtype=np.uint32)
    dst = np.ascontiguousarray(dst, dtype=np.uint32)
    po, pc = C.POINTER(C.c_int64)(), C.POINTER(C.c_int32)()
    m = L.or_csr_build(n, len(src), src, dst, C.byref(po), C.byref(pc))
    off = np.ctypeslib.as_array(po, shape=(n + 1,)).copy()
    col = np.ctypeslib.as_array(pc, shape=(max(m, 1),))[:m].copy()
    L.or_free(C.cast(po, C.c_void_p))
    L.or_free(C.cast(pc, C.c_void_p))
    return Csr(off, col)


def add_weights(g: Csr, seed: int, wmax: int) -> Csr:
    w = np.empty(g.m, dtype=np.int32)
    lib().or_weights(seed, wmax, g.n, g.off, g.col, w)
    return Csr(g.off, g.col, w)


def rmat(scale, ef=16, a=0.57, b=0.19, c=0.19, seed=1) -> Csr:
    ne = ef << scale
    s = np.empty(ne, dtype=np.uint32)
    d = np.empty(ne, dtype=np.uint32)
    lib().or_rmat_edges(scale, ef, a, b, c, seed, s, d)
    return csr_from_pairs(1 << scale, s, d)


def grid(rows, cols, lr_div=100, seed=1) -> Csr:
    L = lib()
    ne = L.or_grid_nedges(rows, cols, lr_div)
    s = np.empty(ne, dtype=np.uint32)
    d = np.empty(ne, dtype=np.uint32)
    k = L.or_grid_edges(rows, cols, lr_div, seed, s, d)
    return csr_from_pairs(rows * cols, s[:k], d[:k])


def er(n, m, seed=1) -> Csr:
    s = np.empty(m, dtype=np.uint32)
    d = np.empty(m, dtype=np.uint32)
    lib().or_er_edges(n, m, seed, s, d)
    return csr_from_pairs(n, s, d)


def er_batch_params(seed, i, nlo=1000, nhi=200000, dlo=4.0, dhi=32.0):
    n, m, s = C.c_int64(), C.c_int64(), C.c_uint64()
    lib().or_er_batch_params(seed, i, nlo, nhi, dlo, dhi, C.byref(n), C.byref(m), C.byref(s))
    return n.value, m.value, s.value


def er_batch(seed, count, nlo=1000, nhi=200000, dlo=4.0, dhi=32.0):
    """The instances of a G(n, m) batch, each built on its own (the device
    builds them as one disjoint union)."""
    out = []
    for i in range(count):
        n, m, s = er_batch_params(seed, i, nlo, nhi, dlo, dhi)
        out.append(er(n, m, s))
    return out


def inspect_bfs(g: Csr, lvl, level):
    """The inspector's six counters for a BFS state (inspector.cuh:39-110)."""
    out = np.zeros(6, dtype=np.uint64)
    lib().or_inspect_bfs(g.n, g.off, np.ascontiguousarray(lvl, dtype=np.int32), level, out)
    return out


def roots(g: Csr, seed: int, count: int):
    r = np.empty(count, dtype=np.int32)
    lib().or_roots(seed, g.n, g.off, count, r)
    return r


def bfs(g: Csr, root: int):
    out = np.empty(g.n, dtype=np.int32)
    lib().or_bfs(g.n, g.off, g.col, root, out)
    return out


def sssp_spfa(g: Csr, root: int):
    out = np.empty(g.n, dtype=np.int32)
    lib().or_sssp_spfa(g.n, g.off, g.col, g.w, root, out)
    return out


def sssp_dijkstra(g: Csr, root: int):
    out = np.empty(g.n, dtype=np.int32)
    lib().or_sssp_dijkstra(g.n, g.off, g.col, g.w, root, out)
    return out


def sssp_dial(g: Csr, root: int, wmax: int):
    """Exact distances for integer weights in [1, wmax] (bucket queue)."""
    out = np.empty(g.n, dtype=np.int32)
    if lib().or_sssp_dial(g.n, g.off, g.col, g.w, root, wmax, out) != 0:
        raise ValueError("a weight lies outside [1, wmax]")
    return out


def cc_linear(g: Csr):
    """cc()'s labels in linear time, for graphs with large hubs."""
    out = np.empty(g.n, dtype=np.int32)
    lib().or_cc_linear(g.n, g.off, g.col, out)
    return out


def cc(g: Csr):
    out = np.empty(g.n, dtype=np.int32)
    lib().or_cc(g.n, g.off, g.col, out)
    return out


def bc_f32(g: Csr, root: int):
    nsp = np.empty(g.n, dtype=np.int32)
    dep = np.empty(g.n, dtype=np.float32)
    lib().or_bc_f32(g.n, g.off, g.col, root, nsp, dep)
    return nsp, dep


def bc_f64(g: Csr, root: int):
    nsp = np.empty(g.n, dtype=np.float64)
    dep = np.empty(g.n, dtype=np.float64)
    lvl = np.empty(g.n, dtype=np.int32)
    lib().or_bc_f64(g.n, g.off, g.col, root, nsp, dep, lvl)
    return nsp, dep, lvl


def pagerank(g: Csr, iters=20, damp=0.85):
    out = np.empty(g.n, dtype=np.float64)
    lib().or_pagerank(g.n, g.off, g.col, iters, damp, out)
    return out


def pagerank_check(g: Csr, pr_over_od, damp=0.85, eps=0.01) -> int:
    pr = np.ascontiguousarray(pr_over_od, dtype=np.float32)
    return int(lib().or_pagerank_check(g.n, g.off, g.col, pr, damp, eps))


def gc_check(g: Csr, color) -> int:
    col = np.ascontiguousarray(color, dtype=np.int32)
    return int(lib().or_gc_check(g.n, g.off, g.col, col))


def gc_levels(g: Csr):
    out = np.empty(g.n, dtype=np.int32)
    lib().or_gc_levels(g.n, g.off, g.col, out)
    return out


def mbfs(g: Csr, srcs):
    srcs = np.ascontiguousarray(srcs, dtype=np.int32)
    out = np.empty(len(srcs) * g.n, dtype=np.int32)
    lib().or_mbfs(g.n, g.off, g.col, len(srcs), srcs, out)
    return out.reshape(len(srcs), g.n)


def degree_attr(g: Csr):
    out = np.empty(6, dtype=np.float64)
    lib().or_degree_attr(g.n, g.off, out)
    return out


def traversed_edges(g: Csr, lvl) -> int:
    lv = np.ascontiguousarray(lvl, dtype=np.int32)
    return int(lib().or_traversed_edges(g.n, g.off, lv))
