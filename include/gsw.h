/*
 * gswitch-b200 C ABI (libgsw.so).
 *
 * The reference (PAA-NCIC/GSWITCH) is a header-only CUDA C++ template API with
 * no foreign-function interface; its callers are the application mains in
 * application/*.cu.  This ABI is the flat boundary underneath the
 * reference-compatible headers: plain pointers and sizes, status codes, no
 * C++ types.  Each declaration names the reference interface it replaces
 * (paths inside the PAA-NCIC/GSWITCH tree).
 *
 * Conventions
 *   - every call returns gsw_status (GSW_OK == 0); gsw_last_error_string()
 *     describes the first failure of the calling thread since its last
 *     successful call;
 *   - a context owns one CUDA stream on one device; a context is not
 *     thread-safe, distinct contexts may run concurrently;
 *   - host arrays passed in are copied; host arrays passed out are written
 *     in full before the call returns;
 *   - graphs are undirected unless `directed` is set; CSR row offsets are
 *     int64 (n + 1 entries), column ids int32, optional int32 arc weights.
 */
#ifndef GSW_H
#define GSW_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int gsw_status;
enum {
  GSW_OK = 0,
  GSW_ERR_INVALID_ARG = 1,
  GSW_ERR_OOM = 2,
  GSW_ERR_CUDA = 3,
  GSW_ERR_TIMEOUT = 4,
  GSW_ERR_OVERFLOW = 5,
  GSW_ERR_UNSUPPORTED = 6,
  GSW_ERR_NO_DEVICE = 7
};

typedef struct gsw_ctx gsw_ctx;
typedef struct gsw_graph gsw_graph;

/* Replaces parse_cmd's cudaSetDevice (src/utils/cmdline.cuh:164-232) and the
 * global stream helper (src/utils/utils.cuh:238-245). */
gsw_status gsw_init(int device, gsw_ctx **out);
gsw_status gsw_destroy(gsw_ctx *ctx);
/* Replaces the reference's exit()-on-error macros (src/utils/utils.cuh:61-87). */
const char *gsw_last_error_string(void);
/* ABI version, for loaders that check it. */
int gsw_version(void);

/* ---- graphs -------------------------------------------------------------
 * Replaces build_graph<VC|EC> / device_graph_t<CSR,E>::build
 * (src/data_structures/graph.cuh:149-215,268-280): upload a host CSR.  The
 * CSR is checked before any kernel indexes with it: row_off[0] = 0,
 * row_off[n] = m, offsets that never decrease and column indices in [0, n);
 * anything else is GSW_ERR_INVALID_ARG (the reference reads out of bounds). */
gsw_status gsw_graph_upload(gsw_ctx *ctx, int64_t n, int64_t m, const int64_t *row_off, const int32_t *col,
                            const int32_t *weights, int directed, gsw_graph **out);
/* Device-side generators (the reference reads .mtx files instead,
 * src/utils/fileIO.cuh:73-146): RMAT (Graph500 a/b/c, no noise), 2D grid with
 * long-range edges, G(n,m).  wmax > 0 adds symmetric weights in [1, wmax]
 * drawn from wseed. */
gsw_status gsw_graph_generate_rmat(gsw_ctx *ctx, int scale, int edge_factor, double a, double b, double c,
                                   uint64_t seed, int wmax, uint64_t wseed, gsw_graph **out);
gsw_status gsw_graph_generate_grid(gsw_ctx *ctx, int rows, int cols, int lr_div, uint64_t seed, int wmax,
                                   uint64_t wseed, gsw_graph **out);
gsw_status gsw_graph_generate_er(gsw_ctx *ctx, int64_t n, int64_t m_pairs, uint64_t seed, int wmax, uint64_t wseed,
                                 gsw_graph **out);
/* No counterpart in the reference.  A batch of `count` G(n, m) graphs as one
 * disjoint union (config C4): instance i has n_i log-uniform in [nlo, nhi],
 * mean degree uniform in [dlo, dhi] and m_i = floor(n_i * degree / 2) pairs,
 * drawn from its own seed exactly as gsw_graph_generate_er draws a single
 * graph; it owns vertices [vertex_offsets[i], vertex_offsets[i + 1])
 * (vertex_offsets: count + 1 entries, may be NULL). */
gsw_status gsw_graph_generate_er_batch(gsw_ctx *ctx, int count, uint64_t seed, int64_t nlo, int64_t nhi, double dlo,
                                       double dhi, int wmax, uint64_t wseed, int64_t *vertex_offsets,
                                       gsw_graph **out);
/* No counterpart in the reference (its corpus is downloaded graphs).
 * Undirected configuration-model graph for the selector corpus: vertex
 * degrees drawn from a power law P(d) ~ d^-gamma (d >= 1, capped at
 * sqrt(n * mean_degree)), stubs paired by a seeded shuffle, self-loops and
 * duplicate edges dropped. */
gsw_status gsw_graph_generate_powerlaw(gsw_ctx *ctx, int64_t n, double gamma, uint64_t seed, int wmax,
                                       uint64_t wseed, gsw_graph **out);
/* n, arcs, weighted flag */
gsw_status gsw_graph_info(const gsw_graph *g, int64_t *n, int64_t *m, int *weighted);
/* Degree statistics as graph_attr_t::fill (src/utils/fileIO.cuh:35-67):
 * out[0..5] = avg, std, range, max, Gini, Hoover-like "Her". */
gsw_status gsw_graph_attr(const gsw_graph *g, double *out6);
/* Copy the CSR back to host arrays (weights may be NULL). */
gsw_status gsw_graph_download(const gsw_graph *g, int64_t *row_off, int32_t *col, int32_t *weights);
/* A graph belongs to the context that made it: destroy it before the
 * context. */
gsw_status gsw_graph_destroy(gsw_graph *g);
/* `count` distinct seeded non-isolated vertices, the rule the reference's
 * random_root follows (src/utils/fileIO.cuh:389-397) with a counter-based
 * hash of (seed, draw) instead of random(). */
gsw_status gsw_graph_roots(const gsw_graph *g, uint64_t seed, int count, int32_t *roots);
/* The context's CUDA stream (cudaStream_t), for callers that time or order
 * work around the library's launches. */
gsw_status gsw_ctx_stream(gsw_ctx *ctx, void **stream);

/* Training records: replaces feature_t::record with cmd_opt.json
 * (src/abstraction/features.cuh:86-104, src/utils/json.cuh:34-48, the -j
 * option of src/utils/cmdline.cuh:208).  After this call every application
 * run on the context appends, after each expand (where the reference's
 * applications keep their training hook, application/bfs.cu:95), one block
 * {"0": fv[0], ..., "20": fv[20], "21": last filter ms, "22": last expand
 * ms} in the reference's layout to `path`, at most 100 blocks per run.
 * NULL or "" turns recording off. */
gsw_status gsw_ctx_record_features(gsw_ctx *ctx, const char *path);

/* ---- level-loop configuration --------------------------------------------
 * Replaces the -c Dir-Fmt-LB-Fusion override of src/utils/cmdline.cuh:51-94
 * (any field may be left to the selector with -1). */
enum { GSW_AUTO = -1 };
enum { GSW_PUSH = 0, GSW_PULL = 1 };
enum { GSW_QUEUE = 0, GSW_BITMAP = 1 };
enum { GSW_LB_TM = 0, GSW_LB_WM = 1, GSW_LB_CM = 2, GSW_LB_STRICT = 3, GSW_LB_TWOD = 4, GSW_LB_TWC = 6 };
enum { GSW_FUSED = 0, GSW_STANDALONE = 1 };
enum { GSW_SELECT_RULES = 0, GSW_SELECT_MLP = 1 };

typedef struct gsw_run_opts {
  int direction;     /* GSW_AUTO / GSW_PUSH / GSW_PULL */
  int asfmt;         /* GSW_AUTO / GSW_QUEUE / GSW_BITMAP */
  int lb;            /* GSW_AUTO / GSW_LB_* */
  int fusion;        /* GSW_AUTO / GSW_FUSED / GSW_STANDALONE */
  int sorted_queue;  /* 1: bitmap->queue in vertex order, 0: atomic append */
  int max_iters;     /* PageRank: iterations (0 = until the eps test passes) */
  float damping;     /* PageRank damping (0.85) */
  float eps;         /* PageRank per-vertex relative change threshold */
  int selector;      /* GSW_SELECT_RULES or GSW_SELECT_MLP */
  int verbose;       /* per-level trace on stdout */
  int timing;        /* per-level device times into gsw_run_stats (CUDA
                        events around each inspect / expand, resolved after
                        the run: no extra synchronisation) */
  int expand_grid;   /* >0: fixed expand grid (autotuner) */
  int account;       /* 1: count the edges each expand touches (with timing,
                        for roofline accounting; adds one atomic per thread) */
  int persistent;    /* fused levels in one grid-wide launch: GSW_AUTO (on),
                        0 off (one launch per level), 1 on */
  int barrier_test;  /* failure-path test only: in a grid-wide launch one
                        block leaves without reaching the level barrier, the
                        others' wait (bounded to 20 ms) expires and the call
                        returns GSW_ERR_TIMEOUT */
  int captured;      /* 1: run the whole level loop as one CUDA graph with
                        device-side selection and termination (BFS, SSSP, PR,
                        delta-PR, CC, GC; GSW_ERR_UNSUPPORTED for BC, MBFS and
                        batched BC, whose batched forms run every level in one
                        cooperative launch); 0: host-driven loop */
  int hub_path;      /* how a CTA sweeps one hub's adjacency list (the
                        thread/warp/CTA-tiered push's CTA tier): 0 four-byte
                        loads, 1 int4 loads of the 16-byte-aligned body,
                        2 shared-memory staging by 1-D TMA bulk copies;
                        GSW_AUTO: 2 without edge data, 1 with it */
  int reserved[3];
} gsw_run_opts;

void gsw_run_opts_default(gsw_run_opts *o);

#define GSW_MAX_TRACE 4096
typedef struct gsw_run_stats {
  double ms;               /* device time of the whole level loop */
  int levels;              /* expand steps executed */
  int64_t edges;           /* Graph500 traversed-edge count where defined */
  unsigned device_error;   /* DEV_ERR bits seen by kernels (0 = clean) */
  int64_t launches;        /* kernels launched by the run */
  int ntrace;              /* entries in the per-level trace below */
  /* per level: dir | fmt<<1 | lb<<2 | fused<<5 | persistent<<6; on a level
   * that ran inside a persistent launch, lb is the load balance the launched
   * kernel reported back */
  int32_t level_cfg[GSW_MAX_TRACE];
  int64_t level_frontier[GSW_MAX_TRACE];
  float level_ms[GSW_MAX_TRACE];         /* expand time, with opts.timing; captured
                                            loops: the whole iteration (decision,
                                            queue build, expand, next inspection),
                                            from device timestamps, always */
  float level_inspect_ms[GSW_MAX_TRACE]; /* inspection time, with opts.timing;
                                            captured loops: the device-side
                                            decision (k_dl_select) of the level */
  int64_t level_edges[GSW_MAX_TRACE];    /* edges touched, with opts.account */
} gsw_run_stats;

/* ---- applications ----------------------------------------------------------
 * Each runs the inspect -> select -> filter -> expand loop of the reference
 * application with the same operator semantics and returns the result to a
 * host array (NULL: leave it on the device).
 *   BFS  application/bfs.cu:16-102     levels (-1 unreached)
 *   SSSP application/sssp.cu:17-126    distances (INT32_MAX unreached)
 *   CC   application/cc.cu:15-289      component labels (min vertex id)
 *   PR   application/pagerank.cu:18-103 pr/out-degree (pr for sinks)
 *   BC   application/bc.cu:31-309      path counts and dependencies
 *   GC   application/gc.cu:15-99       colours
 *   MBFS application/mbfs.cu:16-246    levels per source (row-major)  */
gsw_status gsw_bfs(gsw_ctx *ctx, gsw_graph *g, int32_t root, const gsw_run_opts *o, int32_t *levels,
                   gsw_run_stats *st);
/* BFS from several roots at once: levels are distances to the nearest root.
 * Over a disjoint union of graphs with one root per part this runs every
 * part's BFS in one level loop (the batched form of config C4). */
gsw_status gsw_bfs_multi(gsw_ctx *ctx, gsw_graph *g, int nroots, const int32_t *roots, const gsw_run_opts *o,
                         int32_t *levels, gsw_run_stats *st);
/* Test hook: the six counters one inspection of the BFS state `levels` at
 * `level` produces (src/abstraction/inspector.cuh:39-110): active and
 * inactive vertices, their degree sums, and the reference's per-block sums
 * of per-thread maximum degrees (max over blocks, sum over blocks). */
gsw_status gsw_bfs_inspect(gsw_ctx *ctx, gsw_graph *g, const int32_t *levels, int32_t level, uint64_t *out6);
gsw_status gsw_sssp(gsw_ctx *ctx, gsw_graph *g, int32_t root, const gsw_run_opts *o, int32_t *dist,
                    gsw_run_stats *st);
gsw_status gsw_cc(gsw_ctx *ctx, gsw_graph *g, const gsw_run_opts *o, int32_t *labels, gsw_run_stats *st);
gsw_status gsw_pagerank(gsw_ctx *ctx, gsw_graph *g, const gsw_run_opts *o, float *pr_over_od, gsw_run_stats *st);
/* Delta-PageRank: no reference function corresponds (the reference's
 * docs/index.md:178 describes the algorithm; its code has none).  Same
 * fixed point as gsw_pagerank in the unnormalised form pr = (1-d) +
 * d * sum pr[u]/od[u]; a vertex sends only the change it accumulated, once
 * that change exceeds o->eps times its value (o->damping = d; o->max_iters
 * > 0 caps the levels).  pr receives the values themselves (not pr/od);
 * st->edges counts the out-edges of the vertices that sent. */
gsw_status gsw_pagerank_delta(gsw_ctx *ctx, gsw_graph *g, const gsw_run_opts *o, float *pr, gsw_run_stats *st);
gsw_status gsw_bc(gsw_ctx *ctx, gsw_graph *g, int32_t root, const gsw_run_opts *o, int32_t *nsp, float *dep,
                  gsw_run_stats *st);
gsw_status gsw_gc(gsw_ctx *ctx, gsw_graph *g, const gsw_run_opts *o, int32_t *colors, gsw_run_stats *st);
/* Multi-source BFS.  batched = 0 runs the single-source loop per source
 * (as application/mbfs.cu does); batched = 1 runs all sources together with
 * bit-sliced frontiers (64 sources per word) in one launch sequence. */
/* Betweenness centrality from many sources: no reference function
 * corresponds (application/bc.cu:246-309 runs one source); per source the
 * results are those of gsw_bc / bc_cpu (application/bc.cu:162-214): int32
 * path counts (wrapping like the reference's) and FP32 dependencies, rows of
 * n per source (nsrc x n, source-major).  Sources advance together in
 * batches of 32 (bit-sliced levels, then one forward and one backward pass
 * per level over all of a batch's sources), each batch in one cooperative
 * launch (o->persistent = 0: one launch per pass).  Undirected graphs only.
 * st->edges counts the forward traversals (Graph500 edges summed over the
 * sources). */
gsw_status gsw_bc_batch(gsw_ctx *ctx, gsw_graph *g, int nsrc, const int32_t *roots, const gsw_run_opts *o,
                        int32_t *nsp, float *dep, gsw_run_stats *st);
/* (gsw_mbfs with batched = 1 runs every level of a batch in one cooperative
 * launch; o->persistent = 0 launches per level.) */
gsw_status gsw_mbfs(gsw_ctx *ctx, gsw_graph *g, int nsrc, const int32_t *roots, int batched, const gsw_run_opts *o,
                    int32_t *levels, gsw_run_stats *st);

/* ---- learned selector -------------------------------------------------------
 * No counterpart in the reference, whose selector is decision trees
 * (src/abstraction/selector.cuh:22-303).  An FP32 MLP 8 -> 32 -> 32 -> 20
 * over per-level features; class k is the standalone variant
 * direction = k / 10 (push, pull), format = (k / 5) % 2 (queue, bitmap),
 * load balance = k % 5 (TM, WM, CM, STRICT, TWC).
 * A model is GSW_MLP_MODEL_FLOATS floats: the GSW_MLP_NPARAM parameters
 * (W1[32][8] b1[32] W2[32][32] b2[32] W3[20][32] b3[20]) followed by the
 * feature means (8) and inverse standard deviations (8). */
#define GSW_MLP_FEATURES 8
#define GSW_MLP_CLASSES 20
#define GSW_MLP_NPARAM 2004
#define GSW_MLP_MODEL_FLOATS (GSW_MLP_NPARAM + 2 * GSW_MLP_FEATURES)
enum { GSW_APP_BFS = 0, GSW_APP_SSSP = 1, GSW_APP_PR = 2 };

/* Labels for training: runs the application with standalone levels and, at
 * each labelled level (the first 24, then every 8th, at most max_levels; PR:
 * the first pr_iters iterations), times every one of the 20 variants from the
 * same snapshot of the level's state (filter + expand, CUDA events).
 * features: [max_levels][8]; times_ms: [max_levels][20] (0 = the variant
 * failed); rule_class: [max_levels] the class the rule-based selector chose
 * (may be NULL); *nlevels = rows written. */
gsw_status gsw_label_levels(gsw_ctx *ctx, gsw_graph *g, int app, int32_t root, int max_levels, int pr_iters,
                            float *features, float *times_ms, int32_t *rule_class, int *nlevels);
/* Trains a model on n samples with the project's forward/backward and Adam
 * kernels (full batch, soft labels q_k ~ exp(-(t_k / t_min - 1) / tau)).
 * loss: per-epoch mean loss (may be NULL). */
gsw_status gsw_mlp_train(gsw_ctx *ctx, const float *features, const float *times_ms, int64_t n, int epochs, float lr,
                         float tau, uint64_t seed, float *model_out, float *loss);
/* Loss and gradient (GSW_MLP_NPARAM floats) of a model on n samples. */
gsw_status gsw_mlp_grad(gsw_ctx *ctx, const float *model, const float *features, const float *times_ms, int64_t n,
                        float tau, float *grad, float *loss);
/* Warp-level inference: class and top probability per sample. */
gsw_status gsw_mlp_infer(gsw_ctx *ctx, const float *model, const float *features, int64_t n, int32_t *cls,
                         float *prob);
/* Loads (model != NULL) or unloads the model that runs with
 * opts.selector = GSW_SELECT_MLP; below min_conf top-class probability the
 * rules decide. */
gsw_status gsw_mlp_load(gsw_ctx *ctx, const float *model, float min_conf);
/* The loaded model (GSW_MLP_MODEL_FLOATS floats) and its min_conf;
 * GSW_ERR_INVALID_ARG when none is loaded. */
gsw_status gsw_mlp_save(gsw_ctx *ctx, float *model, float *min_conf);

/* ---- one level's decision, for callers that drive their own level loop ----
 * Replaces inspector_t::set_fets + selector_t::select of one level
 * (src/abstraction/inspector.cuh:206-241, selector.cuh:22-303): from the
 * graph's degree statistics (graph_attr_t::fill, src/utils/fileIO.cuh:35-67,
 * as gsw_graph_attr returns them) and the inspection's six counters of the
 * level, the features are built and flattened as the host loop builds them,
 * the reference's trees pick the standalone variant, and with
 * GSW_SELECT_MLP the loaded network may override them.  Fusion, the idle
 * count and the wall-clock rule depend on the run's history and stay with
 * the caller's loop (the choice is always standalone).  first_level = 1
 * uses the first level's known counters (one root: its degree) instead. */
typedef struct gsw_level_stats {
  int64_t nvertexs, nedges;
  double attr[6];              /* average degree, deviation, range, max degree, Gini, Hoover */
  int64_t active, inactive;    /* the six counters of the level's inspection */
  int64_t push_workload, pull_workload, max_push, max_pull;
  int pattern;                 /* 0 idempotent (BFS), 1 monotone (SSSP), 2 associative (PR, BC) */
  int fromall, toall;          /* the functor's from-all / to-all flags */
  int level, first_level;      /* level number; 1: the run's first level (root_degree holds its workload) */
  int64_t root_degree;
} gsw_level_stats;
typedef struct gsw_level_choice {
  int direction, asfmt, lb;    /* GSW_PUSH / GSW_PULL, GSW_QUEUE / GSW_BITMAP, GSW_LB_* */
  int done;                    /* 1: the counters end the run (no active vertex) */
} gsw_level_choice;
gsw_status gsw_select(gsw_ctx *ctx, const gsw_level_stats *in, int selector, gsw_level_choice *out);

/* ---- a level loop the caller drives --------------------------------------
 * Replaces the per-level calls of application/bfs.cu:78-102 (inspector.
 * inspect, selector.select, executor.filter, g.update_level, executor.expand,
 * as.finish) for a host framework that cannot instantiate the templates:
 *
 *   gsw_traversal_begin(ctx, g, GSW_APP_BFS, root, &o, &t);
 *   for (;;) {
 *     gsw_level_begin(t, &stats, &done);        inspection: the six counters
 *     if (done) break;
 *     gsw_select(ctx, &stats, GSW_SELECT_MLP, &choice);   or the caller's own
 *     gsw_level_end(t, &choice);                filter + one standalone expand
 *   }
 *   gsw_traversal_end(t, levels, &st);          levels back; frees t
 *
 * BFS only (app GSW_APP_BFS); every level is standalone and runs exactly the
 * given variant (TM / WM / CM / STRICT / TWC).  The state lives in the
 * context's buffers: nothing else may run on the context between begin and
 * end.  stats.first_level = 1 on the first level (not inspected: the root
 * and its degree).  gsw_level_end after the loop ended, or without a
 * gsw_level_begin for the level, is GSW_ERR_INVALID_ARG. */
typedef struct gsw_traversal gsw_traversal;
gsw_status gsw_traversal_begin(gsw_ctx *ctx, gsw_graph *g, int app, int32_t root, const gsw_run_opts *opts,
                               gsw_traversal **out);
gsw_status gsw_level_begin(gsw_traversal *t, gsw_level_stats *stats, int *done);
gsw_status gsw_level_end(gsw_traversal *t, const gsw_level_choice *choice);
gsw_status gsw_traversal_end(gsw_traversal *t, int32_t *values, gsw_run_stats *st);
/* The second network: whether a Mono-pattern run (SSSP) runs fused or
 * standalone levels, from graph features (avg, std and range of degree, Gini,
 * entropy, log n, log m, pattern); class 0 standalone, 1 fused.  Used with
 * opts.selector = GSW_SELECT_MLP; NULL unloads (the reference's tree decides). */
gsw_status gsw_mlp_load_fusion(gsw_ctx *ctx, const float *model, float min_conf);

/* ---- autotuned launch geometry ----------------------------------------------
 * No counterpart in the reference (its grids are fixed per kernel).  The
 * expand grid of every variant, as GSW_TUNE_ENTRIES int32 entries indexed
 * [pull][bitmap][load balance (GSW_LB_*)][fused]: the grid cap in quarters of
 * the kernel's resident grid (SMs x resident CTAs), 0 = the resident grid,
 * at most 64.  gswitch_b200/autotune.py measures and writes the table. */
#define GSW_TUNE_ENTRIES 64
gsw_status gsw_tune_load(gsw_ctx *ctx, const int32_t *quarters); /* NULL: defaults */
gsw_status gsw_tune_save(gsw_ctx *ctx, int32_t *quarters);
/* Tuned shapes, same indexing (0 = default everywhere): the STRICT variants'
 * tile (0: 1,024 slots, 1: 512, 2: 2,048; from-all pulls use at most 1,024);
 * the thread-mapped push's threads per CTA (0: 256, 1: 128, 2: 512); the
 * thread-mapped pull's candidates per thread (shape % 3 -- 0: 2, 1: 1, 2: 4)
 * and threads per CTA (shape / 3, as for the push), shapes 0..8; every other
 * variant takes 0 only.  The reference fixes these in THDNUM / SCRATH
 * (src/utils/common.cuh:12-24); NULL restores the defaults. */
gsw_status gsw_tune_load_shapes(gsw_ctx *ctx, const int32_t *shapes);
gsw_status gsw_tune_save_shapes(gsw_ctx *ctx, int32_t *shapes);

/* No counterpart in the reference.  BFS levels (-1 unreached) computed with
 * the edge-balanced push expand, for callers that cannot allocate device
 * memory: code inside a host framework whose memory pool already owns the
 * device memory, or latency-critical code that cannot take the device-wide
 * synchronisation of cudaMalloc / cudaFree.  The caller passes its own device
 * CSR (d_row_off: n + 1 int64, d_col: m int32) and its own device output
 * (d_levels: n int32); the call allocates nothing and keeps its working
 * memory in one fixed array of about 5 MiB per GPU, held until the process
 * exits.  Limits: n <= 2^18 vertices, m <= 2^28 arcs (GSW_ERR_UNSUPPORTED
 * beyond).  The first call on a device looks up that array's address; make
 * it before any stream capture.  Calls share the array: calls that overlap
 * on the GPU race and must be serialised by the caller.  stream may be NULL
 * (the legacy default stream). */
#define GSW_NOALLOC_MAX_VERTICES (1 << 18)
#define GSW_NOALLOC_MAX_ARCS (1 << 28)
gsw_status gsw_bfs_strict_noalloc(int64_t n, int64_t m, const int64_t *d_row_off, const int32_t *d_col, int32_t root,
                                  int32_t *d_levels, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* GSW_H */
