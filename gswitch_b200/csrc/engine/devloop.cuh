// Captured level loop: the whole inspect -> select -> filter -> expand loop of
// a vertex-centric run as ONE CUDA graph that runs to convergence without the
// host.  The reference drives every level from the host and synchronises
// four times per level (src/abstraction/inspector.cuh:39-110, selector.cuh:
// 22-76, executor.cuh:17-151, application/bfs.cu:104-153); here the host
// launches the graph once and reads the result.
//
//   WHILE (loop) {
//     k_dl_select            one CTA: consumes the last inspection's counters,
//                            runs the selector on the device (the same trees
//                            and arithmetic as the host loop), advances the
//                            level and the queue cursor and picks the bodies
//     SWITCH (filter) {...}  bitmap -> queue builders, one body per
//                            (sorted, target, input cursor), or visited reset
//     SWITCH (expand) {...}  one body per (direction, format, load balance,
//                            fusion) x queue cursor; each is the host loop's
//                            own launch sequence, captured once
//     IF (inspect) {...}     the next level's inspection (skipped on fused
//                            levels and when the expand found no input)
//   }
//
// The select kernel writes every conditional handle at every iteration (an
// out-of-range switch value runs no body): a body graph's handles keep their
// last value from one iteration to the next.  Kernels read the level through
// device_graph_t::dlevel and the queue cursor is baked per body, so no kernel
// parameter changes between levels.  Differences from the host loop: fused
// levels run one launch per level (never the cooperative multi-level kernel,
// whose early exit needs a host decision), and the wall-clock rule that
// returns a slow fused level to the standalone form (executor.cuh:128-131)
// does not apply.  With persistent launches on (the default), a fused
// push-queue body is the host loop's persistent launch: the multi-level
// cooperative kernel, then k_dl_persist_commit, which advances the level,
// the iteration count and the queue cursor by the levels it ran, halts the
// loop on an empty frontier, and otherwise returns it to inspected levels --
// that iteration's inspection always runs after such a body (it skips itself
// once the loop has halted).
#pragma once
#include <vector>

#include "mlp.cuh"

namespace gsw {

constexpr int DL_VARIANTS = 64;       // lb (3 bits) | bitmap << 3 | pull << 4 | fused << 5
constexpr int DL_FILTER_BODIES = 13;  // 12 builders (sorted x target x cursor) + visited reset
constexpr int DL_FILTER_CLEAR = 12;
constexpr int DL_MAX_TREE_NODES = 1344;  // all selector trees (1,323 nodes) fit shared memory

__host__ __device__ inline int dl_variant(Direction d, ASFmt a, LB lb, bool fused) {
  return ((int)lb & 7) | ((a == Bitmap) << 3) | ((d == Pull) << 4) | ((fused ? 1 : 0) << 5);
}
__host__ __device__ inline int dl_target_index(Status t) { return t == Active ? 0 : (t == Inactive ? 1 : 2); }
__host__ __device__ inline int dl_filter_body(bool sorted, Status target, int cursor) {
  return ((sorted ? 3 : 0) + dl_target_index(target)) * 2 + cursor;
}

enum dl_status_t { DL_RUNNING = 0, DL_DONE = 1, DL_LEVEL_CAP = 2, DL_NO_BODY = 3, DL_NOT_INSPECTED = 4 };

// Device state of one captured loop (lives in device memory; the host writes
// the initial image before each launch and reads it back afterwards).
struct dloop_t {
  feature_t fets;
  config_t conf;
  tree_set trees;               // device copies of the selector's trees
  const tree_node *tree_base;   // the one allocation `trees` points into
  int tree_nodes;
  const mlp_model *mlp;         // learned selector (null: the rules alone)
  level_counts raw;             // counters of the last inspection (frontier hints)
  int level;                    // the level kernels read
  int cursor;                   // Normal queue: input subqueue
  int halt;                     // set by an expand whose input is empty
  int inspected;                // the previous iteration ran the inspection
  int iter;                     // iterations (levels) so far
  int max_iters;                // > 0: stop at this iteration, after its inspection
  int iter_cap;                 // iterations before the loop gives up
  int sorted;                   // sorted bitmap -> queue builder
  int status;                   // dl_status_t
  int ntrace, trace_cap;
  int *trace_cfg;
  long long *trace_frontier;
  long long *trace_edges;
  // globaltimer (ns) at the start of each iteration's decision ([i]: level i
  // begins, level i-1 ends) and after it ([i]: the decision of level i took
  // trace_sel[i] - trace_t[i]); trace_cap + 1 entries each
  long long *trace_t, *trace_sel;
  unsigned long long *info;     // the inspector's statistics block
  unsigned long long *scanned;  // accounting counter (null: not counting)
  int *qsize;                   // the Normal queue's two size words
  long long nvertexs, nedges, as_size;
  long long launches;           // kernels the loop ran
  unsigned long long push_sum;  // push workload of the inspected levels that ran
  int variant_body[DL_VARIANTS];  // variant -> expand body (-1: none)
  int expand_kernels[2 * DL_VARIANTS];
  int filter_kernels[DL_FILTER_BODIES];
  int inspect_kernels;
  int n_expand_bodies;
  int persist_fused;            // fused push-queue bodies are persistent launches
  int pad_;
  cudaGraphConditionalHandle h_loop, h_filter, h_expand, h_inspect;
  // stepping window of Mono patterns (SSSP): the kernels read `win` through
  // vdata_t::dwin; when a level finds no input the probe body (the deferred
  // filter of fused runs, then k_exit into probe_flag) looks for values the
  // window kept out, and the next decision resets the window or stops
  window_t win;
  const tree_node *stepping;   // the stepping tree (device copy)
  int probe_flag;              // k_exit's flag: some value lies outside the window
  int window_on;               // the window is in use
  int probe_armed;             // the probe ran this iteration
  int probe_kernels;
  cudaGraphConditionalHandle h_probe;
};

__device__ inline void dl_stop(dloop_t &d, int status) {
  d.status = status;
  cudaGraphSetConditional(d.h_loop, 0);
  cudaGraphSetConditional(d.h_filter, DL_FILTER_BODIES);
  cudaGraphSetConditional(d.h_expand, 2 * DL_VARIANTS);
  cudaGraphSetConditional(d.h_inspect, 0);
}

// an iteration without filter or expand: only the inspection (after a window
// reset) or nothing but the probe (a level that inspected no active vertex)
__device__ inline void dl_skip_level(dloop_t &d, bool inspect) {
  cudaGraphSetConditional(d.h_filter, DL_FILTER_BODIES);
  cudaGraphSetConditional(d.h_expand, 2 * DL_VARIANTS);
  cudaGraphSetConditional(d.h_inspect, inspect ? 1 : 0);
  d.inspected = inspect ? 1 : 0;
  d.launches += 1 + (inspect ? d.inspect_kernels : 0);
}

// after the expand and the inspection: arm the window's exit probe when the
// level found no input (one thread)
__global__ void k_dl_gate(dloop_t *d) {
  const bool probe = d->status == DL_RUNNING && d->window_on && d->halt;
  cudaGraphSetConditional(d->h_probe, probe ? 1 : 0);
  d->probe_armed = probe ? 1 : 0;
  d->launches += 1 + (probe ? d->probe_kernels : 0);
}

// DL_GO: the level runs; DL_INSPECT_ONLY / DL_PROBE_ONLY: see dl_skip_level
enum { DL_STOPPED = 0, DL_GO = 1, DL_INSPECT_ONLY = 2, DL_PROBE_ONLY = 3 };

// One level's decisions: the host loop's inspect-finish-select sequence
// (gsw_capi.cu runners) on device state, by one thread.  Returns false when
// the loop stops here.
__device__ inline int dl_decide(dloop_t &d, const level_counts &c, unsigned long long scanned) {
  auto stop = [&](int status) {
    dl_stop(d, status);
    return (int)DL_STOPPED;
  };
  if (d.ntrace > 0 && d.ntrace <= d.trace_cap) d.trace_edges[d.ntrace - 1] = (long long)scanned;
  feature_t &fets = d.fets;
  config_t &conf = d.conf;
  if (d.halt) {  // the last expand found an empty input (or the inspection no active vertex)
    if (!(d.window_on && d.probe_armed)) return stop(DL_DONE);
    // the host loop's window_exit (executor.cuh): a vertex whose value the
    // window kept out restarts the loop on the next window
    d.probe_armed = 0;
    if (!d.probe_flag) return stop(DL_DONE);
    d.probe_flag = 0;
    d.win.reset();
    d.halt = 0;
    if (conf.conf_fusion) {
      conf.conf_fuse_inspect = false;
      conf.conf_switch_to_fusion = true;
    }
    if (d.iter >= d.iter_cap) return stop(DL_LEVEL_CAP);
    d.iter++;
    return DL_INSPECT_ONLY;
  }
  fets_level_init(fets, d.level, d.nvertexs, d.nedges);
  bool need = !conf.conf_fuse_inspect;
  bool done = false;
  if (need && conf.conf_first_round) {
    d.raw = fets_first(fets, d.nvertexs, d.nedges);
    need = false;
  }
  if (need) {
    if (!d.inspected) return stop(DL_NOT_INSPECTED);
    d.raw = c;
    done = fets_from_counts(fets, c, d.nvertexs, d.nedges);
  }
  fets.flatten();
  if (d.max_iters > 0 && d.iter == d.max_iters) return stop(DL_DONE);
  if (done && d.window_on) {  // nothing active in this window: probe before stopping
    d.halt = 1;
    return DL_PROBE_ONLY;
  }
  if (done) return stop(DL_DONE);
  if (d.iter >= d.iter_cap) return stop(DL_LEVEL_CAP);
  if (need) d.push_sum += (unsigned long long)c.push;
  selector_t sel;
  sel.trees = &d.trees;
  sel.decide(fets, conf);
  return DL_GO;
}

// the filter-update-trace part of the level, after the selector (and the
// network, when one is loaded) decided
__device__ inline void dl_commit(dloop_t &d) {
  auto stop = [&](int status) { dl_stop(d, status); };
  feature_t &fets = d.fets;
  config_t &conf = d.conf;
  // filter: queue build (or visited reset) from the pre-swap cursor, then swap
  int fbody = DL_FILTER_BODIES;  // none
  if (conf.conf_asfmt == Queue) {
    if (level_builds_queue(conf))
      fbody = dl_filter_body(d.sorted != 0, conf.conf_target, d.cursor);
    else if (!conf.conf_pruning)
      fbody = DL_FILTER_CLEAR;
    d.qsize[d.cursor] = 0;
    d.cursor ^= 1;
  }
  level_grid_bookkeeping(fets, conf);
  long long fr;
  if (conf.conf_asfmt == Bitmap) {
    fr = d.as_size;
  } else if (!conf.conf_fuse_inspect) {
    const Status t = conf.conf_target;
    fr = t == Active ? d.raw.active : (t == Inactive ? d.raw.inactive : d.raw.active + d.raw.inactive);
  } else {
    fr = -1;
  }
  if (fr < 0 || fr > d.as_size) fr = -1;
  d.level += 1;  // g.update_level()
  const int v = dl_variant(conf.conf_dir, conf.conf_asfmt, conf.conf_lb, conf.conf_fuse_inspect);
  const int vb = d.variant_body[v];
  if (vb < 0) return stop(DL_NO_BODY);
  const int ebody = vb * 2 + (conf.conf_asfmt == Queue ? d.cursor : 0);
  if (d.ntrace < d.trace_cap) {
    d.trace_cfg[d.ntrace] = (conf.conf_dir == Pull) | ((conf.conf_asfmt == Bitmap) << 1) | ((int)conf.conf_lb << 2) |
                            ((conf.conf_fuse_inspect ? 1 : 0) << 5);
    d.trace_frontier[d.ntrace] = fr;
    d.trace_edges[d.ntrace] = 0;
  }
  d.ntrace++;
  conf.conf_first_round = false;
  d.iter++;
  d.inspected = !conf.conf_fuse_inspect;
  if (conf.conf_fuse_inspect && d.persist_fused && conf.conf_dir == Push && conf.conf_asfmt == Queue) {
    // a persistent body: its inspection runs after it (see k_dl_persist_commit)
    d.inspected = 1;
    if (d.ntrace - 1 < d.trace_cap) d.trace_cfg[d.ntrace - 1] |= 1 << 6;
  }
  d.launches += 1 + (fbody < DL_FILTER_BODIES ? d.filter_kernels[fbody] : 0) + d.expand_kernels[ebody] +
                (d.inspected ? d.inspect_kernels : 0);
  cudaGraphSetConditional(d.h_filter, fbody);
  cudaGraphSetConditional(d.h_expand, ebody);
  cudaGraphSetConditional(d.h_inspect, d.inspected ? 1 : 0);
  // the window the next inspection and expand read (the host loop adjusts it
  // at the start of its next inspection, from the same features)
  if (d.window_on) d.win.adjust_with(fets, conf, d.stepping);
}

// After a persistent body (prep, the cooperative multi-level kernel): the
// launch ran L levels, the first of them the one this iteration committed;
// its last output sits in the queue slot out = cur ^ (L & 1), where the next
// level's swap expects it.  An empty frontier halts the loop; any other exit
// returns it to inspected (standalone) levels, as the host loop does after a
// frontier grew past its limit; a barrier timeout or a scan overflow (in the
// error word) halts it too.
__global__ void k_dl_persist_commit(dloop_t *d, as_counters_t *c, int cur) {
  const int L = c->plevels, reason = c->preason;
  if (L > 1) {
    d->level += L - 1;
    d->iter += L - 1;
  }
  d->cursor = (cur ^ (L & 1)) ^ 1;
  if (d->ntrace - 1 >= 0 && d->ntrace - 1 < d->trace_cap)
    d->trace_cfg[d->ntrace - 1] = (d->trace_cfg[d->ntrace - 1] & ~(7 << 2)) | ((c->plb & 7) << 2);
  d->conf.conf_fuse_inspect = false;
  if (reason == 0 || reason == 3 || reason == 4 || reason < 0) {
    d->halt = 1;
  } else {
    c->qsize[0] = 0;  // the next level builds its queue from the bitmaps
    c->qsize[1] = 0;
  }
}

// The decision thread works on a shared-memory copy of the loop state and of
// the trees (a tree walk is a chain of dependent loads; from shared memory it
// takes nanoseconds per node instead of an L2 round trip), and the block
// writes the state back at the end.
__global__ void __launch_bounds__(256) k_dl_select(dloop_t *d) {
  constexpr int WORDS = (int)(sizeof(dloop_t) / 8);
  static_assert(sizeof(dloop_t) % 8 == 0, "loop state is copied in 8-byte words");
  static_assert(sizeof(tree_node) % 8 == 0, "tree nodes are copied in 8-byte words");
  __shared__ __align__(16) unsigned long long s_state[WORDS];
  __shared__ __align__(16) unsigned long long s_tree[DL_MAX_TREE_NODES * sizeof(tree_node) / 8];
  __shared__ level_counts s_c;
  __shared__ unsigned long long s_scanned;
  __shared__ int s_go, s_mlp;
  __shared__ float s_x[MLP_IN];
  dloop_t &sd = *reinterpret_cast<dloop_t *>(s_state);
  const unsigned long long *src = reinterpret_cast<const unsigned long long *>(d);
  for (int i = threadIdx.x; i < WORDS; i += blockDim.x) s_state[i] = src[i];
  if (threadIdx.x == 0) {
    if (d->trace_t) d->trace_t[min(d->ntrace, d->trace_cap)] = (long long)globaltimer_ns();
    const unsigned long long *info = d->info;
    s_c.active = (int64_t)info[0];
    s_c.inactive = (int64_t)info[1];
    s_c.push = (int64_t)info[2];
    s_c.pull = (int64_t)info[3];
    s_c.max_push = (int64_t)info[4];
    s_c.max_pull = (int64_t)info[5];
    s_scanned = d->scanned ? *d->scanned : 0ull;
  }
  __syncthreads();
  // the trees (about 32 KB) in 16-byte loads, all of a thread's issued
  // before its stores: one L2 round trip instead of one per loop step
  const int tree_words = min(sd.tree_nodes, DL_MAX_TREE_NODES) * (int)(sizeof(tree_node) / 8);
  const unsigned long long *tsrc = reinterpret_cast<const unsigned long long *>(sd.tree_base);
  {
    constexpr int PER = (DL_MAX_TREE_NODES * (int)sizeof(tree_node) / 16 + 255) / 256;  // int4 per thread
    const int n4 = tree_words / 2;
    const int4 *s4 = reinterpret_cast<const int4 *>(tsrc);
    int4 *d4 = reinterpret_cast<int4 *>(s_tree);
    int4 r[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int i = threadIdx.x + k * 256;
      if (i < n4) r[k] = __ldg(s4 + i);
    }
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int i = threadIdx.x + k * 256;
      if (i < n4) d4[i] = r[k];
    }
    if (threadIdx.x == 0 && (tree_words & 1)) s_tree[tree_words - 1] = __ldg(tsrc + tree_words - 1);
  }
  // the counters start from zero for the next inspection
  for (int i = threadIdx.x; i < STAT_SLOTS; i += blockDim.x) sd.info[i] = 0;
  __syncthreads();
  if (threadIdx.x == 0) {
    if (sd.scanned) *sd.scanned = 0;
    const tree_set dev = sd.trees;
    const tree_node *base = sd.tree_base, *sh = reinterpret_cast<const tree_node *>(s_tree);
    sd.trees = tree_set{sh + (dev.dir_idem - base),        sh + (dev.dir_asso - base),
                        sh + (dev.dir_asso_backup - base), sh + (dev.fmt - base),
                        sh + (dev.fusion - base),          sh + (dev.lb_idem - base),
                        sh + (dev.lb_asso_forward - base), sh + (dev.lb_asso_backward - base),
                        sh + (dev.lb_asso_backward_backup - base)};
    const tree_node *dev_step = sd.stepping;
    if (dev_step) sd.stepping = sh + (dev_step - base);
    const int code = dl_decide(sd, s_c, s_scanned);
    if (code == DL_INSPECT_ONLY || code == DL_PROBE_ONLY) dl_skip_level(sd, code == DL_INSPECT_ONLY);
    s_go = code == DL_GO;
    sd.trees = dev;
    sd.stepping = dev_step;
    s_mlp = s_go && sd.mlp && mlp_applicable(*sd.mlp, sd.fets, sd.conf);
    if (s_mlp) mlp_features(sd.fets, s_x);
  }
  __syncthreads();
  // in-stream inference of the learned selector by warp 0
  if (s_mlp && threadIdx.x < 32) {
    float pt;
    const int k = mlp_predict_warp(*sd.mlp, s_x, &pt);
    if (threadIdx.x == 0 && pt >= sd.mlp->min_conf) mlp_apply(k, sd.conf);
  }
  __syncthreads();
  if (threadIdx.x == 0 && s_go) dl_commit(sd);
  if (threadIdx.x == 0 && sd.trace_sel && s_go && sd.ntrace - 1 < sd.trace_cap)
    sd.trace_sel[sd.ntrace - 1] = (long long)globaltimer_ns();
  __syncthreads();
  unsigned long long *dst = reinterpret_cast<unsigned long long *>(d);
  for (int i = threadIdx.x; i < WORDS; i += blockDim.x) dst[i] = s_state[i];
}

// ---------------------------------------------------------------------------
// graph construction
// ---------------------------------------------------------------------------

// adds a conditional node at the current capture position of `s`
inline bool dl_add_conditional(cudaStream_t s, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                               unsigned size, std::vector<cudaGraph_t> &bodies) {
  cudaStreamCaptureStatus st;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  if (GSW_CUDA(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd))) return false;
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = type;
  p.conditional.size = size;
  cudaGraphNode_t node;
  if (GSW_CUDA(cudaGraphAddNode(&node, g, deps, nd, &p))) return false;
  bodies.assign(p.conditional.phGraph_out, p.conditional.phGraph_out + size);
  return !GSW_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
}

inline int dl_count_nodes(cudaGraph_t g) {
  size_t n = 0;
  cudaGraphGetNodes(g, nullptr, &n);
  return (int)n;
}

// captures whatever `launch` issues on the context stream into `body`
template <typename L>
inline bool dl_capture(cudaGraph_t body, L &&launch) {
  if (GSW_CUDA(cudaStreamBeginCaptureToGraph(stream(), body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed)))
    return false;
  launch();
  cudaGraph_t out = nullptr;
  const bool good = !GSW_CUDA(cudaStreamEndCapture(stream(), &out));
  return good && ok();
}

// The persistent body of a fused push-queue variant: the host loop's
// persistent launch (executor_t::launch_persistent_lb) without its host
// side -- the results go to k_dl_persist_commit instead of the host.
template <int LB, typename G, typename F>
void dl_persistent_lb(executor_t &ex, active_set_t &as, G &g, F &f, config_t &conf, const feature_t &fets, dloop_t *d,
                      int cur) {
  auto kern = k_fused_persistent<LB, G, F>;
  const int grid = resident_grid(kern, EXPAND_THREADS);
  if (LB == STRICT && grid > as.workset.bsum_cap)
    return (void)set_error(GSW_ERR_OVERFLOW, "persistent strict: %s", "block sums");
  as_counters_t *c = as.dg_cnt;
  k_persist_prep<<<1, 1, 0, stream()>>>(c, cur);
  persist_state ps;
  ps.q[0] = as.queue.subqueue[cur].dg_queue;
  ps.q[1] = as.queue.subqueue[cur ^ 1].dg_queue;
  ps.cnt = c->pq;
  ps.cap = as.queue.subqueue[0].max_size;
  ps.grow_limit = fets.pattern == Idem ? (int)MAX((int64_t)4096, as.size / 64) : INT32_MAX;
  ps.max_levels = (int)MIN(as.size + 2, (int64_t)(1 << 24));
  ps.budget_ns = 2000000000ull;
  ps.leave_block = -1;
  ps.levels_done = &c->plevels;
  ps.exit_reason = &c->preason;
  ps.lb_out = &c->plb;
  ps.cur = cur;
  ps.level0 = &d->level;
  ps.sig = nullptr;
  ps.seq = 0;
  ps.eoff = as.workset.dg_eoff;
  ps.eoff_cap = as.size + 2;
  ps.bsum = as.workset.dg_bsum;
  ps.tile_lo = ex.dg_tile;
  ps.tile_cap = ex.tile_cap;
  void *args[] = {(void *)&as, (void *)&g, (void *)&f, (void *)&conf, (void *)&ps};
  if (GSW_CUDA(cudaLaunchCooperativeKernel((const void *)kern, grid, EXPAND_THREADS, args, 0, stream()))) return;
  k_dl_persist_commit<<<1, 1, 0, stream()>>>(d, c, cur);
  GSW_LAUNCHED();
}
template <typename E, typename F>
void dl_persistent_body(executor_t &ex, active_set_t &as, device_graph_t<CSR, E> &g, F &f, config_t &conf,
                        const feature_t &fets, dloop_t *d, int cur) {
  using G = device_graph_t<CSR, E>;
  switch (conf.conf_lb) {
    case TM: return dl_persistent_lb<TM, G, F>(ex, as, g, f, conf, fets, d, cur);
    case CM: return dl_persistent_lb<CM, G, F>(ex, as, g, f, conf, fets, d, cur);
    case STRICT: return dl_persistent_lb<STRICT, G, F>(ex, as, g, f, conf, fets, d, cur);
    case TWC: return dl_persistent_lb<TWC, G, F>(ex, as, g, f, conf, fets, d, cur);
    default: return dl_persistent_lb<WM, G, F>(ex, as, g, f, conf, fets, d, cur);
  }
}

// A built loop: the executable graph plus what the host needs to drive it.
struct dloop_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<unsigned long long> key;
  dloop_t image;  // handles and body tables; the per-run fields are filled at launch
  void destroy() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    key.clear();
  }
};

// Builds the captured loop of a CSR (vertex-centric) run.  `as`, `g`, `f`
// and `conf` are the run's own objects after init_conf; `d` is the device
// address of the loop state.  Every body is captured through the executor's
// ordinary launch code with the grid derived from resident occupancy.
template <typename E, typename F>
bool dl_build(dloop_graph &L, executor_t &ex, dloop_t *d, active_set_t as, device_graph_t<CSR, E> g, F f,
              config_t conf, const feature_t &fets, unsigned long long *info) {
  using G = device_graph_t<CSR, E>;
  L.destroy();
  g.dlevel = &d->level;
  f.data.dwin = &d->win;
  as.nt.dg_tag = &d->halt;
  as.nt.already = false;
  as.queue.traceback = false;
  const bool persist = conf.conf_persistent && as.queue.mode == Normal;
  conf.conf_persistent = false;
  const bool saved_timing = opts().timing;
  opts().timing = false;
  const long long launches0 = launch_count();
  const hints_t saved_hints = hints();
  hints().frontier = -1;
  hints().edges = -1;
  hints().max_deg = -1;  // a captured body sweeps whatever hubs its level lists
  ex.ensure_tiles(g.nedges + as.size + 1);
  dloop_t &im = L.image;
  im = dloop_t();
  im.persist_fused = persist ? 1 : 0;
  for (int &b : im.variant_body) b = -1;
  bool good = ok();
  // the variants this run can reach
  struct vdesc {
    Direction d;
    ASFmt a;
    LB lb;
    bool fused;
  };
  std::vector<vdesc> vs;
  const LB lbs[5] = {TM, WM, CM, STRICT, TWC};
  for (LB lb : lbs) {
    vs.push_back({Push, Queue, lb, false});
    vs.push_back({Push, Queue, lb, true});
    vs.push_back({Push, Bitmap, lb, false});
    vs.push_back({Pull, Queue, lb, false});
    vs.push_back({Pull, Bitmap, lb, false});
  }
  const bool twod_ok = fets.fromall && fets.toall && ex.twod.edge;
  if (twod_ok) vs.push_back({Push, Bitmap, TWOD, false});
  for (size_t i = 0; i < vs.size(); ++i) {
    const vdesc &v = vs[i];
    if (v.lb == TWOD) {
      for (Direction dd : {Push, Pull})
        for (ASFmt aa : {Queue, Bitmap}) im.variant_body[dl_variant(dd, aa, TWOD, false)] = (int)i;
    } else {
      im.variant_body[dl_variant(v.d, v.a, v.lb, v.fused)] = (int)i;
    }
  }
  im.n_expand_bodies = (int)vs.size();

  cudaGraph_t top = nullptr;
  good = good && !GSW_CUDA(cudaGraphCreate(&top, 0));
  L.graph = top;
  cudaGraphConditionalHandle hl = 0, hf = 0, he = 0, hi = 0, hp = 0;
  std::vector<cudaGraph_t> wbody, fbodies, ebodies, ibody, pbody;
  const bool window = conf.conf_window;
  if (good) good = !GSW_CUDA(cudaGraphConditionalHandleCreate(&hl, top, 1, cudaGraphCondAssignDefault));
  if (good) {
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = hl;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t wn;
    good = !GSW_CUDA(cudaGraphAddNode(&wn, top, nullptr, 0, &p));
    if (good) wbody.assign(p.conditional.phGraph_out, p.conditional.phGraph_out + 1);
  }
  const unsigned nexp = 2u * (unsigned)vs.size();
  if (good) {
    cudaGraph_t B = wbody[0];
    good = !GSW_CUDA(cudaGraphConditionalHandleCreate(&hf, B, DL_FILTER_BODIES, 0)) &&
           !GSW_CUDA(cudaGraphConditionalHandleCreate(&he, B, 2 * DL_VARIANTS, 0)) &&
           !GSW_CUDA(cudaGraphConditionalHandleCreate(&hi, B, 0, 0)) &&
           (!window || !GSW_CUDA(cudaGraphConditionalHandleCreate(&hp, B, 0, 0)));
    if (good)
      good = dl_capture(B, [&] {
        k_dl_select<<<1, 256, 0, stream()>>>(d);
        if (dl_add_conditional(stream(), hf, cudaGraphCondTypeSwitch, DL_FILTER_BODIES, fbodies) &&
            dl_add_conditional(stream(), he, cudaGraphCondTypeSwitch, nexp, ebodies) &&
            dl_add_conditional(stream(), hi, cudaGraphCondTypeIf, 1, ibody) && window) {
          k_dl_gate<<<1, 1, 0, stream()>>>(d);
          dl_add_conditional(stream(), hp, cudaGraphCondTypeIf, 1, pbody);
        }
      });
    good = good && fbodies.size() == DL_FILTER_BODIES && ebodies.size() == nexp && ibody.size() == 1 &&
           (!window || pbody.size() == 1);
  }
  // filter bodies
  for (int sorted = 0; good && sorted < 2; ++sorted)
    for (Status t : {Active, Inactive, All})
      for (int cur = 0; good && cur < 2; ++cur) {
        const int b = dl_filter_body(sorted != 0, t, cur);
        active_set_t a = as;
        a.fmt = Queue;
        a.queue.cursor = cur;
        good = dl_capture(fbodies[b], [&] { ex.build_queue(a, t, sorted != 0); });
        im.filter_kernels[b] = dl_count_nodes(fbodies[b]);
      }
  if (good) {
    good = dl_capture(fbodies[DL_FILTER_CLEAR],
                      [&] { fill_u32(as.bitmap.visited.dg_bits, 0, as.bitmap.visited.n_words); });
    im.filter_kernels[DL_FILTER_CLEAR] = dl_count_nodes(fbodies[DL_FILTER_CLEAR]);
  }
  // expand bodies
  for (size_t i = 0; good && i < vs.size(); ++i)
    for (int cur = 0; good && cur < 2; ++cur) {
      const vdesc &v = vs[i];
      config_t c = conf;
      c.conf_dir = v.d;
      c.conf_asfmt = v.a;
      c.conf_lb = v.lb;
      c.conf_fuse_inspect = v.fused;
      c.conf_fromall = fets.fromall;
      c.conf_toall = fets.toall;
      c.conf_centric = fets.centric;
      selector_t::set_target(c);
      active_set_t a = as;
      a.fmt = v.a;
      a.queue.cursor = cur;
      G gg = g;
      const int b = (int)i * 2 + cur;
      if (persist && v.fused && v.d == Push && v.a == Queue)
        good = dl_capture(ebodies[b], [&] { dl_persistent_body(ex, a, gg, f, c, fets, d, cur); });
      else
        good = dl_capture(ebodies[b], [&] { ex.launch_vc(a, gg, f, c); });
      im.expand_kernels[b] = dl_count_nodes(ebodies[b]);
    }
  // inspection body
  if (good) {
    good = dl_capture(ibody[0], [&] {
      launch_inspect_vc(as, g, f, info, &d->halt);
    });
    im.inspect_kernels = 1;
  }
  // window exit probe: the deferred filter of fused runs, then the probe
  // (window_delay_update and window_exit of the host loop)
  if (good && window) {
    good = dl_capture(pbody[0], [&] {
      if (conf.conf_fusion) window_delay_update(as, g, f);
      k_exit<<<resident_grid(k_exit<G, F>, 512), 512, 0, stream()>>>(g, f, &d->probe_flag);
    });
    im.probe_kernels = dl_count_nodes(pbody[0]);
  }
  if (good) good = !GSW_CUDA(cudaGraphInstantiate(&L.exec, top, 0));
  im.h_loop = hl;
  im.h_filter = hf;
  im.h_expand = he;
  im.h_inspect = hi;
  im.h_probe = hp;
  opts().timing = saved_timing;
  launch_count() = launches0;
  hints() = saved_hints;
  if (!good) {
    L.destroy();
    if (ok()) set_error(GSW_ERR_CUDA, "%s", "captured level loop: graph construction failed");
  }
  return good;
}

}  // namespace gsw
