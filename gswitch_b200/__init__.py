"""gswitch-b200: GSWITCH's level-loop graph engine for one NVIDIA B200.

Host-side mirror of the C ABI (include/gsw.h, libgsw.so).  It follows the
reference's operator/plugin vocabulary: an application runs the
inspect -> select -> filter -> expand level loop, and any subset of the
selector's choices can be forced with the reference's ``-c`` string
(``"Push-Queue-WM-Fused"``, ``x`` leaves a choice to the selector;
src/utils/cmdline.cuh:51-94).  Errors raise :class:`GswError` carrying the
C status code.  There is no CPU fallback: importing works anywhere, but every
call needs libgsw.so and a CUDA device.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgsw.so")

GSW_OK = 0
STATUS = {0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "CUDA", 4: "TIMEOUT", 5: "OVERFLOW",
          6: "UNSUPPORTED", 7: "NO_DEVICE"}
AUTO = -1
PUSH, PULL = 0, 1
QUEUE, BITMAP = 0, 1
LB = {"TM": 0, "WM": 1, "CM": 2, "STRICT": 3, "TWOD": 4, "TWC": 6}
LB_NAMES = {v: k for k, v in LB.items()}
FUSED, STANDALONE = 0, 1
MAX_TRACE = 4096

# exported symbols of libgsw.so, one per declaration in include/gsw.h
ABI_SYMBOLS = (
    "gsw_init", "gsw_destroy", "gsw_last_error_string", "gsw_version",
    "gsw_graph_upload", "gsw_graph_generate_rmat", "gsw_graph_generate_grid",
    "gsw_graph_generate_er", "gsw_graph_info", "gsw_graph_attr", "gsw_graph_download",
    "gsw_graph_destroy", "gsw_graph_roots", "gsw_ctx_stream", "gsw_ctx_record_features", "gsw_run_opts_default", "gsw_bfs", "gsw_sssp", "gsw_cc",
    "gsw_pagerank", "gsw_bc", "gsw_bc_batch", "gsw_gc", "gsw_mbfs", "gsw_bfs_strict_noalloc",
    "gsw_graph_generate_powerlaw", "gsw_label_levels", "gsw_mlp_train", "gsw_mlp_grad", "gsw_mlp_infer",
    "gsw_mlp_load", "gsw_graph_generate_er_batch", "gsw_bfs_multi", "gsw_bfs_inspect", "gsw_tune_load",
    "gsw_tune_save", "gsw_tune_load_shapes", "gsw_tune_save_shapes", "gsw_mlp_load_fusion", "gsw_pagerank_delta",
    "gsw_mlp_save", "gsw_select", "gsw_traversal_begin", "gsw_level_begin", "gsw_level_end",
    "gsw_traversal_end",
)
TUNE_ENTRIES = 64

# learned selector (include/gsw.h): 8 features -> 32 -> 32 -> 20 classes
MLP_FEATURES, MLP_CLASSES, MLP_NPARAM = 8, 20, 2004
MLP_MODEL_FLOATS = MLP_NPARAM + 2 * MLP_FEATURES
APP_BFS, APP_SSSP, APP_PR = 0, 1, 2
SELECT_RULES, SELECT_MLP = 0, 1


def mlp_class_name(k: int) -> str:
    """Class k of the learned selector as a ``Dir-Fmt-LB`` string."""
    return "-".join((("Push", "Pull")[k // 10], ("Queue", "Bitmap")[(k // 5) % 2],
                     ("TM", "WM", "CM", "STRICT", "TWC")[k % 5]))


class GswError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"gsw error {code} ({STATUS.get(code, '?')}): {msg}")
        self.code = code


class _Opts(C.Structure):
    _fields_ = [("direction", C.c_int), ("asfmt", C.c_int), ("lb", C.c_int), ("fusion", C.c_int),
                ("sorted_queue", C.c_int), ("max_iters", C.c_int), ("damping", C.c_float),
                ("eps", C.c_float), ("selector", C.c_int), ("verbose", C.c_int), ("timing", C.c_int),
                ("expand_grid", C.c_int), ("account", C.c_int), ("persistent", C.c_int), ("barrier_test", C.c_int),
                ("captured", C.c_int), ("hub_path", C.c_int),
                ("reserved", C.c_int * 3)]


class _Stats(C.Structure):
    _fields_ = [("ms", C.c_double), ("levels", C.c_int), ("edges", C.c_int64),
                ("device_error", C.c_uint), ("launches", C.c_int64), ("ntrace", C.c_int),
                ("level_cfg", C.c_int32 * MAX_TRACE), ("level_frontier", C.c_int64 * MAX_TRACE),
                ("level_ms", C.c_float * MAX_TRACE), ("level_inspect_ms", C.c_float * MAX_TRACE),
                ("level_edges", C.c_int64 * MAX_TRACE)]


_LIB = None


def lib():
    """Load libgsw.so; raise if it is missing (no fallback exists)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise GswError(7, f"{LIB_PATH} is not built; run gswitch_b200/build.py")
    L = C.CDLL(LIB_PATH)
    vp, i64, i32, u64 = C.c_void_p, C.c_int64, C.c_int32, C.c_uint64
    pvp = C.POINTER(C.c_void_p)
    L.gsw_init.argtypes = [C.c_int, pvp]
    L.gsw_destroy.argtypes = [vp]
    L.gsw_last_error_string.restype = C.c_char_p
    L.gsw_graph_upload.argtypes = [vp, i64, i64, vp, vp, vp, C.c_int, pvp]
    L.gsw_graph_generate_rmat.argtypes = [vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, u64,
                                          C.c_int, u64, pvp]
    L.gsw_graph_generate_grid.argtypes = [vp, C.c_int, C.c_int, C.c_int, u64, C.c_int, u64, pvp]
    L.gsw_graph_generate_er.argtypes = [vp, i64, i64, u64, C.c_int, u64, pvp]
    L.gsw_graph_info.argtypes = [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(C.c_int)]
    L.gsw_graph_attr.argtypes = [vp, vp]
    L.gsw_graph_download.argtypes = [vp, vp, vp, vp]
    L.gsw_graph_destroy.argtypes = [vp]
    L.gsw_graph_roots.argtypes = [vp, u64, C.c_int, vp]
    L.gsw_ctx_stream.argtypes = [vp, pvp]
    L.gsw_ctx_record_features.argtypes = [vp, C.c_char_p]
    L.gsw_run_opts_default.argtypes = [C.POINTER(_Opts)]
    L.gsw_run_opts_default.restype = None
    po, ps = C.POINTER(_Opts), C.POINTER(_Stats)
    L.gsw_bfs.argtypes = [vp, vp, i32, po, vp, ps]
    L.gsw_sssp.argtypes = [vp, vp, i32, po, vp, ps]
    L.gsw_cc.argtypes = [vp, vp, po, vp, ps]
    L.gsw_pagerank.argtypes = [vp, vp, po, vp, ps]
    L.gsw_pagerank_delta.argtypes = [vp, vp, po, vp, ps]
    L.gsw_bc.argtypes = [vp, vp, i32, po, vp, vp, ps]
    L.gsw_gc.argtypes = [vp, vp, po, vp, ps]
    L.gsw_mbfs.argtypes = [vp, vp, C.c_int, vp, C.c_int, po, vp, ps]
    L.gsw_bc_batch.argtypes = [vp, vp, C.c_int, vp, po, vp, vp, ps]
    L.gsw_bfs_strict_noalloc.argtypes = [i64, i64, vp, vp, i32, vp, vp]
    L.gsw_graph_generate_powerlaw.argtypes = [vp, i64, C.c_double, u64, C.c_int, u64, pvp]
    L.gsw_label_levels.argtypes = [vp, vp, C.c_int, i32, C.c_int, C.c_int, vp, vp, vp, C.POINTER(C.c_int)]
    L.gsw_mlp_train.argtypes = [vp, vp, vp, i64, C.c_int, C.c_float, C.c_float, u64, vp, vp]
    L.gsw_mlp_grad.argtypes = [vp, vp, vp, vp, i64, C.c_float, vp, vp]
    L.gsw_mlp_infer.argtypes = [vp, vp, vp, i64, vp, vp]
    L.gsw_mlp_load.argtypes = [vp, vp, C.c_float]
    L.gsw_graph_generate_er_batch.argtypes = [vp, C.c_int, u64, i64, i64, C.c_double, C.c_double, C.c_int, u64, vp,
                                              pvp]
    L.gsw_bfs_multi.argtypes = [vp, vp, C.c_int, vp, po, vp, ps]
    L.gsw_bfs_inspect.argtypes = [vp, vp, vp, i32, vp]
    L.gsw_tune_load.argtypes = [vp, vp]
    L.gsw_tune_load_shapes.argtypes = [vp, vp]
    L.gsw_mlp_save.argtypes = [vp, vp, vp]
    L.gsw_select.argtypes = [vp, vp, C.c_int, vp]
    L.gsw_traversal_begin.argtypes = [vp, vp, C.c_int, i32, vp, pvp]
    L.gsw_level_begin.argtypes = [vp, vp, C.POINTER(C.c_int)]
    L.gsw_level_end.argtypes = [vp, vp]
    L.gsw_traversal_end.argtypes = [vp, vp, vp]
    L.gsw_tune_save_shapes.argtypes = [vp, vp]
    L.gsw_mlp_load_fusion.argtypes = [vp, vp, C.c_float]
    L.gsw_tune_save.argtypes = [vp, vp]
    _LIB = L
    return L


def _check(code):
    if code != GSW_OK:
        raise GswError(code, lib().gsw_last_error_string().decode(errors="replace"))


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# how a CTA sweeps one hub's adjacency list (gsw_run_opts.hub_path)
HUB_SCALAR, HUB_VECTOR, HUB_STAGED = 0, 1, 2


class LevelStats(C.Structure):
    """gsw_level_stats: one level's inspection counters and the graph's degree
    statistics, the input of Context.select()."""
    _fields_ = [("nvertexs", C.c_int64), ("nedges", C.c_int64), ("attr", C.c_double * 6), ("active", C.c_int64),
                ("inactive", C.c_int64), ("push_workload", C.c_int64), ("pull_workload", C.c_int64),
                ("max_push", C.c_int64), ("max_pull", C.c_int64), ("pattern", C.c_int), ("fromall", C.c_int),
                ("toall", C.c_int), ("level", C.c_int), ("first_level", C.c_int), ("root_degree", C.c_int64)]


class LevelChoice(C.Structure):
    _fields_ = [("direction", C.c_int), ("asfmt", C.c_int), ("lb", C.c_int), ("done", C.c_int)]


class Traversal:
    """A BFS whose level loop the caller drives (gsw_traversal_* and
    gsw_level_*): level_begin() inspects the level and returns its
    LevelStats and whether the run is over; level_end(choice) runs that level
    as the standalone variant `choice` -- a LevelChoice or a (direction,
    format, LB) tuple of names as Context.select() returns; end() returns the
    levels and the run statistics and frees the state."""

    def __init__(self, graph, root, opts=None):
        self.graph = graph
        h = C.c_void_p()
        o = graph._opts(opts)
        _check(lib().gsw_traversal_begin(graph.ctx._h, graph._h, APP_BFS, C.c_int32(root), C.byref(o), C.byref(h)))
        self._h = h

    def level_begin(self):
        st = LevelStats()
        done = C.c_int(0)
        _check(lib().gsw_level_begin(self._h, C.byref(st), C.byref(done)))
        return st, bool(done.value)

    def level_end(self, choice):
        if not isinstance(choice, LevelChoice):
            d, a, b = choice
            choice = LevelChoice(PULL if d == "Pull" else PUSH, BITMAP if a == "Bitmap" else QUEUE, LB[b], 0)
        _check(lib().gsw_level_end(self._h, C.byref(choice)))

    def end(self, out=True):
        lv = np.empty(self.graph.n, dtype=np.int32) if out else None
        st = _Stats()
        h, self._h = self._h, None
        _check(lib().gsw_traversal_end(h, _ptr(lv), C.byref(st)))
        return lv, RunStats(st)


class RunOpts:
    """Forced choices and knobs of one run (None = selector decides)."""

    def __init__(self, direction=None, asfmt=None, lb=None, fusion=None, sorted_queue=True,
                 max_iters=0, damping=0.85, eps=0.01, verbose=False, timing=False, expand_grid=0,
                 account=False, persistent=None, barrier_test=False, captured=False, selector="rules",
                 hub_path=None):
        self.direction, self.asfmt, self.lb, self.fusion = direction, asfmt, lb, fusion
        self.sorted_queue, self.max_iters, self.damping, self.eps = sorted_queue, max_iters, damping, eps
        self.verbose, self.timing, self.expand_grid = verbose, timing, expand_grid
        self.account = account
        self.persistent = persistent
        self.barrier_test = barrier_test
        self.captured = captured
        self.selector = selector  # "rules" (decision trees) or "mlp" (loaded network, rules as fallback)
        self.hub_path = hub_path  # HUB_SCALAR / HUB_VECTOR / HUB_STAGED (None: by edge data)

    @classmethod
    def from_config(cls, cfg: str, **kw):
        """Parse the reference's ``-c Dir-Fmt-LB-Fusion`` string."""
        parts = (cfg.split("-") + ["x"] * 4)[:4] if cfg else ["x"] * 4
        o = cls(**kw)
        o.direction = {"Push": PUSH, "Pull": PULL}.get(parts[0])
        o.asfmt = {"Queue": QUEUE, "Bitmap": BITMAP}.get(parts[1])
        o.lb = LB.get(parts[2])
        o.fusion = {"Fused": FUSED, "Standalone": STANDALONE}.get(parts[3])
        return o

    def to_c(self) -> _Opts:
        o = _Opts()
        lib().gsw_run_opts_default(C.byref(o))
        f = lambda x: AUTO if x is None else int(x)
        o.direction, o.asfmt, o.lb, o.fusion = f(self.direction), f(self.asfmt), f(self.lb), f(self.fusion)
        o.sorted_queue = int(bool(self.sorted_queue))
        o.max_iters = int(self.max_iters)
        o.damping, o.eps = float(self.damping), float(self.eps)
        o.verbose, o.timing, o.expand_grid = int(self.verbose), int(self.timing), int(self.expand_grid)
        o.account = int(self.account)
        o.persistent = AUTO if self.persistent is None else int(bool(self.persistent))
        o.barrier_test = int(self.barrier_test)
        o.captured = int(bool(self.captured))
        o.selector = SELECT_MLP if self.selector == "mlp" else SELECT_RULES
        o.hub_path = AUTO if self.hub_path is None else int(self.hub_path)
        return o


class RunStats:
    def __init__(self, s: _Stats):
        self.ms = s.ms
        self.levels = s.levels
        self.edges = s.edges
        self.device_error = s.device_error
        self.launches = s.launches
        n = min(s.ntrace, MAX_TRACE)
        self.trace = [decode_cfg(s.level_cfg[i]) + (int(s.level_frontier[i]),) for i in range(n)]
        # levels whose expand was a persistent (grid-barrier) launch
        self.level_persistent = [bool(s.level_cfg[i] & 64) for i in range(n)]
        self.level_ms = [float(s.level_ms[i]) for i in range(n)]
        self.level_inspect_ms = [float(s.level_inspect_ms[i]) for i in range(n)]
        self.level_edges = [int(s.level_edges[i]) for i in range(n)]

    @property
    def gteps(self) -> float:
        return self.edges / (self.ms * 1e6) if self.ms > 0 else 0.0

    def variants(self):
        return {f"{d}-{f}-{lb}-{fu}" for d, f, lb, fu, _ in self.trace}


def decode_cfg(c: int):
    return ("Pull" if c & 1 else "Push", "Bitmap" if c & 2 else "Queue", LB_NAMES.get((c >> 2) & 7, "?"),
            "Fused" if c & 32 else "Standalone")


class Context:
    """One device and one stream (gsw_init / gsw_destroy)."""

    def __init__(self, device: int = 0):
        import weakref

        self._h = C.c_void_p()
        self._graphs = weakref.WeakSet()
        _check(lib().gsw_init(device, C.byref(self._h)))

    def close(self):
        # graphs belong to the context: release them first
        for g in list(self._graphs):
            g.close()
        if self._h:
            lib().gsw_destroy(self._h)
            self._h = C.c_void_p()

    @property
    def alive(self) -> bool:
        return bool(self._h)

    def stream_ptr(self) -> int:
        s = C.c_void_p()
        _check(lib().gsw_ctx_stream(self._h, C.byref(s)))
        return s.value or 0

    def record_features(self, path):
        """Append the reference's training records (feature_t::record) of
        every level of later runs to `path` (None: stop recording)."""
        _check(lib().gsw_ctx_record_features(self._h, path.encode() if path else None))

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload(self, off, col, w=None, directed=False) -> "Graph":
        off = np.ascontiguousarray(off, dtype=np.int64)
        col = np.ascontiguousarray(col, dtype=np.int32)
        w = None if w is None else np.ascontiguousarray(w, dtype=np.int32)
        h = C.c_void_p()
        _check(lib().gsw_graph_upload(self._h, len(off) - 1, len(col), _ptr(off), _ptr(col), _ptr(w),
                                      int(directed), C.byref(h)))
        return Graph(self, h)

    def rmat(self, scale, ef=16, a=0.57, b=0.19, c=0.19, seed=1, wmax=0, wseed=0) -> "Graph":
        h = C.c_void_p()
        _check(lib().gsw_graph_generate_rmat(self._h, scale, ef, a, b, c, seed, wmax, wseed, C.byref(h)))
        return Graph(self, h)

    def grid(self, rows, cols, lr_div=100, seed=1, wmax=0, wseed=0) -> "Graph":
        h = C.c_void_p()
        _check(lib().gsw_graph_generate_grid(self._h, rows, cols, lr_div, seed, wmax, wseed, C.byref(h)))
        return Graph(self, h)

    def er(self, n, m_pairs, seed=1, wmax=0, wseed=0) -> "Graph":
        h = C.c_void_p()
        _check(lib().gsw_graph_generate_er(self._h, n, m_pairs, seed, wmax, wseed, C.byref(h)))
        return Graph(self, h)

    def er_batch(self, count, seed=1, nlo=1000, nhi=200000, dlo=4.0, dhi=32.0, wmax=0, wseed=0):
        """`count` G(n, m) graphs as one disjoint union; returns (graph,
        vertex offsets [count + 1])."""
        h = C.c_void_p()
        voff = np.zeros(count + 1, dtype=np.int64)
        _check(lib().gsw_graph_generate_er_batch(self._h, count, seed, nlo, nhi, dlo, dhi, wmax, wseed, _ptr(voff),
                                                 C.byref(h)))
        return Graph(self, h), voff

    def powerlaw(self, n, gamma, seed=1, wmax=0, wseed=0) -> "Graph":
        h = C.c_void_p()
        _check(lib().gsw_graph_generate_powerlaw(self._h, n, float(gamma), seed, wmax, wseed, C.byref(h)))
        return Graph(self, h)

    # ---- learned selector
    def mlp_train(self, X, T, epochs=2000, lr=3e-3, tau=0.1, seed=1):
        """Train on features X [n, 8] and per-variant times T [n, 20]; returns
        (model [MLP_MODEL_FLOATS], per-epoch loss)."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        model = np.zeros(MLP_MODEL_FLOATS, dtype=np.float32)
        loss = np.zeros(epochs, dtype=np.float32)
        _check(lib().gsw_mlp_train(self._h, _ptr(X), _ptr(T), len(X), epochs, lr, tau, seed, _ptr(model),
                                   _ptr(loss)))
        return model, loss

    def mlp_grad(self, model, X, T, tau=0.1):
        model = np.ascontiguousarray(model, dtype=np.float32)
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        g = np.zeros(MLP_NPARAM, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        _check(lib().gsw_mlp_grad(self._h, _ptr(model), _ptr(X), _ptr(T), len(X), tau, _ptr(g), _ptr(loss)))
        return g, float(loss[0])

    def mlp_infer(self, model, X):
        model = np.ascontiguousarray(model, dtype=np.float32)
        X = np.ascontiguousarray(X, dtype=np.float32)
        cls = np.zeros(len(X), dtype=np.int32)
        prob = np.zeros(len(X), dtype=np.float32)
        _check(lib().gsw_mlp_infer(self._h, _ptr(model), _ptr(X), len(X), _ptr(cls), _ptr(prob)))
        return cls, prob

    @staticmethod
    def tune_index(direction, fmt, lb, fused=False):
        """Entry of (``"Push"|"Pull"``, ``"Queue"|"Bitmap"``, LB name, fused)."""
        return (((direction == "Pull") * 2 + (fmt == "Bitmap")) * 8 + LB[lb]) * 2 + int(bool(fused))

    def tune_load(self, quarters=None):
        """Expand grid caps in quarters of the resident grid (None: defaults)."""
        q = None if quarters is None else np.ascontiguousarray(quarters, dtype=np.int32)
        if q is not None and q.shape != (TUNE_ENTRIES,):
            raise ValueError(f"tune table has {TUNE_ENTRIES} entries")
        _check(lib().gsw_tune_load(self._h, _ptr(q)))

    def tune_save(self):
        q = np.zeros(TUNE_ENTRIES, dtype=np.int32)
        _check(lib().gsw_tune_save(self._h, _ptr(q)))
        return q

    def tune_load_shapes(self, shapes=None):
        """Tuned tile / candidates-per-thread shapes per variant (None: defaults)."""
        t = None if shapes is None else np.ascontiguousarray(shapes, dtype=np.int32)
        if t is not None and t.shape != (TUNE_ENTRIES,):
            raise ValueError(f"shape table has {TUNE_ENTRIES} entries")
        _check(lib().gsw_tune_load_shapes(self._h, _ptr(t)))

    def tune_save_shapes(self):
        t = np.zeros(TUNE_ENTRIES, dtype=np.int32)
        _check(lib().gsw_tune_save_shapes(self._h, _ptr(t)))
        return t

    def mlp_load_fusion(self, model=None, min_conf=0.0):
        m = None if model is None else np.ascontiguousarray(model, dtype=np.float32)
        _check(lib().gsw_mlp_load_fusion(self._h, _ptr(m), min_conf))

    def mlp_save(self):
        """The loaded model and its min_conf."""
        m = np.zeros(MLP_MODEL_FLOATS, dtype=np.float32)
        c = C.c_float(0.0)
        _check(lib().gsw_mlp_save(self._h, _ptr(m), C.byref(c)))
        return m, c.value

    def select(self, stats: "LevelStats", selector="rules"):
        """One level's standalone variant ("Push"|"Pull", "Queue"|"Bitmap", LB
        name) and whether the counters end the run (gsw_select)."""
        out = LevelChoice()
        _check(lib().gsw_select(self._h, C.byref(stats), SELECT_MLP if selector == "mlp" else SELECT_RULES,
                                C.byref(out)))
        return (("Pull" if out.direction == PULL else "Push"), ("Bitmap" if out.asfmt == BITMAP else "Queue"),
                LB_NAMES.get(out.lb, "?")), bool(out.done)

    def mlp_load(self, model=None, min_conf=0.0):
        m = None if model is None else np.ascontiguousarray(model, dtype=np.float32)
        _check(lib().gsw_mlp_load(self._h, _ptr(m), min_conf))


class Graph:
    """A device-resident graph (gsw_graph)."""

    def __init__(self, ctx: Context, h):
        self.ctx, self._h = ctx, h
        ctx._graphs.add(self)
        n, m, wt = C.c_int64(), C.c_int64(), C.c_int()
        _check(lib().gsw_graph_info(h, C.byref(n), C.byref(m), C.byref(wt)))
        self.n, self.m, self.weighted = n.value, m.value, bool(wt.value)

    def close(self):
        if self._h and self.ctx.alive:
            lib().gsw_graph_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def roots(self, seed, count):
        r = np.empty(count, dtype=np.int32)
        _check(lib().gsw_graph_roots(self._h, seed, count, _ptr(r)))
        return r

    def attr(self):
        out = np.empty(6, dtype=np.float64)
        _check(lib().gsw_graph_attr(self._h, _ptr(out)))
        return out

    def download(self):
        off = np.empty(self.n + 1, dtype=np.int64)
        col = np.empty(self.m, dtype=np.int32)
        w = np.empty(self.m, dtype=np.int32) if self.weighted else None
        _check(lib().gsw_graph_download(self._h, _ptr(off), _ptr(col), _ptr(w)))
        return off, col, w

    @staticmethod
    def _opts(opts):
        if opts is None:
            opts = RunOpts()
        elif isinstance(opts, str):
            opts = RunOpts.from_config(opts)
        return opts.to_c()

    def _run(self, fn, *args, outs, opts):
        st = _Stats()
        o = self._opts(opts)
        _check(fn(self.ctx._h, self._h, *args, C.byref(o), *[_ptr(x) for x in outs], C.byref(st)))
        return RunStats(st)

    def bfs(self, root, opts=None, out=True):
        lv = np.empty(self.n, dtype=np.int32) if out else None
        st = self._run(lib().gsw_bfs, C.c_int32(root), outs=[lv], opts=opts)
        return lv, st

    def traversal(self, root, opts=None):
        """A BFS level loop driven from Python (gsw_traversal_begin); see
        Traversal.  Nothing else may run on the context until it ends."""
        return Traversal(self, root, opts)

    def bfs_inspect(self, levels, level):
        """The inspector's six counters for a BFS state (gsw_bfs_inspect)."""
        lv = np.ascontiguousarray(levels, dtype=np.int32)
        out = np.zeros(6, dtype=np.uint64)
        _check(lib().gsw_bfs_inspect(self.ctx._h, self._h, _ptr(lv), level, _ptr(out)))
        return out

    def bfs_multi(self, roots, opts=None, out=True):
        """BFS from all `roots` at once (distance to the nearest root)."""
        roots = np.ascontiguousarray(roots, dtype=np.int32)
        lv = np.empty(self.n, dtype=np.int32) if out else None
        st = _Stats()
        o = self._opts(opts)
        _check(lib().gsw_bfs_multi(self.ctx._h, self._h, len(roots), _ptr(roots), C.byref(o), _ptr(lv),
                                   C.byref(st)))
        return lv, RunStats(st)

    def sssp(self, root, opts=None, out=True):
        d = np.empty(self.n, dtype=np.int32) if out else None
        st = self._run(lib().gsw_sssp, C.c_int32(root), outs=[d], opts=opts)
        return d, st

    def cc(self, opts=None, out=True):
        lab = np.empty(self.n, dtype=np.int32) if out else None
        st = self._run(lib().gsw_cc, outs=[lab], opts=opts)
        return lab, st

    def pagerank(self, iters=20, damping=0.85, eps=0.01, opts=None, out=True):
        if opts is None or isinstance(opts, str):
            opts = RunOpts.from_config(opts) if isinstance(opts, str) else RunOpts()
        opts.max_iters, opts.damping, opts.eps = iters, damping, eps
        pr = np.empty(self.n, dtype=np.float32) if out else None
        st = self._run(lib().gsw_pagerank, outs=[pr], opts=opts)
        return pr, st

    def pagerank_delta(self, eps=1e-4, damping=0.85, max_levels=0, opts=None, out=True):
        """Delta-PageRank (gsw_pagerank_delta): the values pr (not pr/od)."""
        if opts is None or isinstance(opts, str):
            opts = RunOpts.from_config(opts) if isinstance(opts, str) else RunOpts()
        opts.max_iters, opts.damping, opts.eps = max_levels, damping, eps
        pr = np.empty(self.n, dtype=np.float32) if out else None
        st = self._run(lib().gsw_pagerank_delta, outs=[pr], opts=opts)
        return pr, st

    def label(self, app, root=0, max_levels=64, pr_iters=3):
        """Per-level features [rows, 8], per-variant times in ms [rows, 20] and
        the rule-based selector's class per level [rows] (gsw_label_levels);
        app is APP_BFS, APP_SSSP or APP_PR."""
        X = np.zeros((max_levels, MLP_FEATURES), dtype=np.float32)
        T = np.zeros((max_levels, MLP_CLASSES), dtype=np.float32)
        R = np.zeros(max_levels, dtype=np.int32)
        rows = C.c_int(0)
        _check(lib().gsw_label_levels(self.ctx._h, self._h, app, root, max_levels, pr_iters, _ptr(X), _ptr(T),
                                      _ptr(R), C.byref(rows)))
        r = rows.value
        return X[:r], T[:r], R[:r]

    def bc(self, root, opts=None, out=True):
        nsp = np.empty(self.n, dtype=np.int32) if out else None
        dep = np.empty(self.n, dtype=np.float32) if out else None
        st = self._run(lib().gsw_bc, C.c_int32(root), outs=[nsp, dep], opts=opts)
        return nsp, dep, st

    def gc(self, opts=None, out=True):
        col = np.empty(self.n, dtype=np.int32) if out else None
        st = self._run(lib().gsw_gc, outs=[col], opts=opts)
        return col, st

    def bc_batch(self, roots, opts=None, out=True):
        """Path counts and dependencies from every root (rows of n, one per
        root), the sources advancing together in batches of 32."""
        roots = np.ascontiguousarray(roots, dtype=np.int32)
        nsp = np.empty((len(roots), self.n), dtype=np.int32) if out else None
        dep = np.empty((len(roots), self.n), dtype=np.float32) if out else None
        st = _Stats()
        o = self._opts(opts)
        _check(lib().gsw_bc_batch(self.ctx._h, self._h, len(roots), _ptr(roots), C.byref(o), _ptr(nsp), _ptr(dep),
                                  C.byref(st)))
        return nsp, dep, RunStats(st)

    def mbfs(self, roots, batched=True, opts=None, out=True):
        roots = np.ascontiguousarray(roots, dtype=np.int32)
        lv = np.empty((len(roots), self.n), dtype=np.int32) if out else None
        st = _Stats()
        o = self._opts(opts)
        _check(lib().gsw_mbfs(self.ctx._h, self._h, len(roots), _ptr(roots), int(batched), C.byref(o), _ptr(lv),
                              C.byref(st)))
        return lv, RunStats(st)
