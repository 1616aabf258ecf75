// Host side of the level loop: inspector_t, selector_t, executor_t,
// init_conf / reset_conf, active-set convergence and CC pointer jumping.
//
// The decision logic restates the reference (src/abstraction/inspector.cuh:
// 112-244, selector.cuh:20-304, executor.cuh:17-151, src/gswitch.h:19-108,
// data_structures/active_set.cuh:37-43, notification.cuh:233-254).  What
// changes is the host/device traffic: a standalone level costs one host
// synchronisation (the inspector's counters), not four.  The frontier size
// the kernels need is read on the device; grid sizes come from the counters
// the host already holds.  Fused levels synchronise once (convergence flag
// and next frontier size).  Explicit deviations:
//   * a forced fusion mode (`-c ...-Fused|Standalone`) holds for every level
//     (the reference lets trigger_fusion re-enable fusion for Idem patterns);
//   * a forced load balance also applies to fused levels (the reference's
//     fusion() always picks WM);
//   * the selector's label mapping quirk is kept: tree class 0 -> WM,
//     1 -> CM, anything else -> STRICT (selector.cuh:126-131, 209-214).
#pragma once
#include <chrono>
#include <unordered_map>

#include "k_persistent.cuh"
#include "k_twod.cuh"

namespace gsw {

inline int sm_count() {
  static thread_local int c = 0;
  if (!c) {
    int d = 0;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, d);
    if (c <= 0) c = 148;
  }
  return c;
}

// resident-grid size of a kernel (SMs x resident blocks per SM), cached
template <typename K>
inline int resident_grid(K kernel, int block, size_t smem = 0) {
  static thread_local std::unordered_map<const void *, int> cache;
  auto it = cache.find((const void *)kernel);
  if (it != cache.end()) return it->second;
  int per = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, block, smem) != cudaSuccess || per <= 0) per = 1;
  int gsz = per * sm_count();
  cache[(const void *)kernel] = gsz;
  return gsz;
}

inline int clamp_grid(int64_t want, int cap) {
  if (want < 1) want = 1;
  return (int)MIN(want, (int64_t)cap);
}

// the VC inspection on one wave of resident CTAs (no more CTAs than units)
template <typename G, typename F>
inline void launch_inspect_vc(const active_set_t &as, const G &g, const F &f, unsigned long long *info,
                              const int *skip_if = nullptr, unsigned long long *sig = nullptr,
                              unsigned long long seq = 0) {
  const int grid = clamp_grid(inspect_units(as.size), resident_grid(k_inspect_vc<G, F>, INSPECT_THREADS));
  k_inspect_vc<G, F><<<grid, INSPECT_THREADS, 0, stream()>>>(as, g, f, info, skip_if, sig, seq);
}

inline double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// per-run knobs of the engine (defaults reproduce the reference's behaviour)
struct engine_opts_t {
  bool verbose = false;
  bool timing = false;        // per-level CUDA-event timing into the stats
  int force_grid = 0;         // autotuner: fixed expand grid (0 = derive)
  bool barrier_leave_test = false;  // failure-path test of the level barrier
};
inline engine_opts_t &opts() {
  static thread_local engine_opts_t o;
  return o;
}

// sizes the host knows without a device round trip
struct hints_t {
  int64_t frontier = -1;     // entries in the expand's work list
  int64_t edges = -1;        // edges they touch
  bool persistent = false;   // the last expand ran as a persistent launch
  int persistent_lb = -1;    // the load balance that launch's kernel reported
  int64_t max_deg = -1;      // bound on the largest degree in the work list (-1: unknown)
};
inline hints_t &hints() {
  static thread_local hints_t h;
  return h;
}

// Event pairs recorded around kernels when per-level timing is on; they are
// resolved after the run, so timing adds no synchronisation.
struct event_pool {
  std::vector<cudaEvent_t> ev;
  size_t used = 0;
  int record() {
    if (used == ev.size()) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return -1;
      ev.push_back(e);
    }
    cudaEventRecord(ev[used], stream());
    return (int)used++;
  }
  float elapsed(int a, int b) const {
    float ms = 0;
    if (a < 0 || b < 0 || cudaEventElapsedTime(&ms, ev[a], ev[b]) != cudaSuccess) return 0;
    return ms;
  }
};
inline event_pool &timing_pool() {
  static thread_local event_pool p;
  return p;
}
// event indices of the last inspect and expand launches (-1 = none)
struct kernel_marks {
  int insp0 = -1, insp1 = -1, exp0 = -1, exp1 = -1;
};
inline kernel_marks &marks() {
  static thread_local kernel_marks m;
  return m;
}

// ===========================================================================
// Per-level decision arithmetic shared by the host loop and the in-stream
// (captured) loop, so both take the same decisions from the same counters.
// ===========================================================================
struct level_counts {  // statistics block [0..5] of one inspection
  int64_t active, inactive, push, pull, max_push, max_pull;
};

// inspector_t::init_fets (inspector.cuh:115-130)
__host__ __device__ inline void fets_level_init(feature_t &fets, int level, int64_t nvertexs, int64_t edges) {
  fets.level = level;
  fets.active_vertex = 0;
  fets.active_vertex_ratio = 0;
  fets.unactive_vertex = (double)nvertexs;
  fets.unactive_vertex_ratio = 1;
  fets.growing_rate = fets.push_workload;
  fets.push_workload = 0;
  fets.pull_workload = (double)edges;
  fets.push_workload_ratio = 0;
  fets.pull_workload_ratio = 1;
  fets.cur_avg_deg_active = 0;
  fets.cur_avg_deg_unactive = fets.avg_deg;
}

// inspector_t::set_first_fets (inspector.cuh:180-204): the first level is
// known without inspecting (one root, or every vertex)
__host__ __device__ inline level_counts fets_first(feature_t &fets, int64_t nvertexs, int64_t nedges) {
  if (fets.use_root < 0) {
    fets.active_vertex = (double)nvertexs;
    fets.unactive_vertex = 0;
    fets.push_workload = (double)nedges;
    fets.pull_workload = 0;
  } else {
    fets.active_vertex = fets.first_active;
    fets.unactive_vertex = (double)nvertexs - fets.first_active;
    fets.push_workload = fets.first_workload;
    fets.pull_workload = nedges - fets.first_workload;
  }
  fets.active_vertex_ratio = fets.active_vertex / nvertexs;
  fets.unactive_vertex_ratio = fets.unactive_vertex / nvertexs;
  fets.push_workload_ratio = fets.push_workload / nedges;
  fets.pull_workload_ratio = fets.pull_workload / nedges;
  fets.cur_avg_deg_active = DIV(fets.push_workload, fets.active_vertex);
  fets.cur_avg_deg_unactive = DIV(fets.pull_workload, fets.unactive_vertex);
  fets.cur_max_deg_active = fets.push_workload;
  fets.cur_max_deg_unactive = fets.avg_deg;
  level_counts c;
  c.active = (int64_t)fets.active_vertex;
  c.inactive = (int64_t)fets.unactive_vertex;
  c.push = (int64_t)fets.push_workload;
  c.pull = (int64_t)fets.pull_workload;
  c.max_push = c.max_pull = 0;
  return c;
}

// inspector_t::set_fets (inspector.cuh:206-241); returns true when the loop
// is done (no active vertex, or an Idem pattern with nothing left to reach)
__host__ __device__ inline bool fets_from_counts(feature_t &fets, const level_counts &c, int64_t nvertexs,
                                                 int64_t nedges) {
  fets.active_vertex = (double)c.active;
  fets.unactive_vertex = (double)c.inactive;
  fets.active_vertex_ratio = (double)c.active / nvertexs;
  fets.unactive_vertex_ratio = (double)c.inactive / nvertexs;
  bool done = fets.active_vertex <= 0;
  if (fets.pattern == Idem && fets.unactive_vertex <= 0) done = true;
  fets.growing_rate = (0.0 + c.push) / fets.growing_rate;
  fets.push_workload = (double)c.push;
  fets.pull_workload = (double)c.pull;
  fets.push_workload_ratio = (double)c.push / nedges;
  fets.pull_workload_ratio = (double)c.pull / nedges;
  fets.cur_avg_deg_active = DIV(fets.push_workload, fets.active_vertex);
  fets.cur_avg_deg_unactive = DIV(fets.pull_workload, fets.unactive_vertex);
  fets.cur_max_deg_active = (double)c.max_push;
  fets.cur_max_deg_unactive = (double)c.max_pull;
  return done;
}

// executor_t::filter (executor.cuh:21-29): does a Queue level rebuild its
// queue from the bitmaps?
__host__ __device__ inline bool level_builds_queue(config_t &conf) {
  bool tofilter = !conf.conf_fuse_inspect;
  if (conf.conf_switch_to_fusion) {
    tofilter = true;
    conf.conf_switch_to_fusion = false;
  }
  if (conf.conf_first_round) tofilter = true;
  return tofilter;
}

// grid bookkeeping of executor_t::filter (executor.cuh:30-52): idle levels
// feed trigger_fusion, tiny STRICT levels fall back to CM
__host__ __device__ inline void level_grid_bookkeeping(const feature_t &fets, config_t &conf) {
  conf.thdnum = THDNUM_EXPAND;
  if (conf.conf_fuse_inspect) {
    conf.ctanum = 32;
  } else {
    const double workloads = conf.conf_dir == Push ? fets.push_workload : fets.pull_workload;
    conf.ctanum = (int)MIN((double)CTANUM_EXPAND, workloads / conf.thdnum / 2 + 1);
    conf.conf_idle = conf.ctanum < 4 ? conf.conf_idle + 1 : 0;
    if (conf.ctanum < 5 && conf.conf_lb == STRICT && !conf.force.has_lb) conf.conf_lb = CM;
  }
}

// ===========================================================================
// inspector_t
// ===========================================================================
struct inspector_t {
  template <typename E, typename F>
  void inspect(active_set_t &as, device_graph_t<CSR, E> g, F &f, stat_t &stat, feature_t &fets, config_t &conf) {
    stat.last_filter_time = now_ms();
    f.data.window.adjust(fets, conf);
    bool need_inspect = !conf.conf_fuse_inspect;
    init_fets(stat, fets, g.nvertexs, g.nedges);
    if (need_inspect && conf.conf_first_round) {
      set_first_fets(fets, g.nvertexs, g.nedges);
      need_inspect = false;
    }
    marks().insp0 = marks().insp1 = -1;
    if (need_inspect) {
      if (opts().timing) marks().insp0 = timing_pool().record();
      const unsigned long long seq = stat.arm();
      launch_inspect_vc(as, g, f, stat.dg_runtime_info, nullptr, seq ? stat.d_sig : nullptr, seq);
      GSW_LAUNCHED();
      if (opts().timing) marks().insp1 = timing_pool().record();
      set_fets(as, stat, fets, conf, g.nvertexs, g.nedges, seq);
    }
    fets.flatten();
  }

  template <typename E, typename F>
  void inspect(active_set_t &as, device_graph_t<COO, E> g, F &f, stat_t &stat, feature_t &fets, config_t &conf) {
    stat.last_filter_time = now_ms();
    init_fets(stat, fets, g.nvertexs, g.nedges);
    if (conf.conf_first_round) {
      conf.conf_first_round = false;
      fets.active_vertex = (double)g.nedges;
      fets.active_vertex_ratio = 1;
      raw_frontier = g.nedges;
      return;
    }
    marks().insp0 = marks().insp1 = -1;
    if (opts().timing) marks().insp0 = timing_pool().record();
    k_inspect_ec<<<EC_INSPECT_CTAS, EC_INSPECT_THREADS, 0, stream()>>>(as, g, f, stat.dg_runtime_info);
    GSW_LAUNCHED();
    if (opts().timing) marks().insp1 = timing_pool().record();
    set_fets(as, stat, fets, conf, g.nvertexs, g.nedges);
    fets.flatten();
  }

  void init_fets(stat_t &stat, feature_t &fets, int64_t nvertexs, int64_t edges) {
    fets_level_init(fets, stat.level, nvertexs, edges);
  }

  void set_first_fets(feature_t &fets, int64_t nvertexs, int64_t nedges) {
    keep(fets_first(fets, nvertexs, nedges));
  }

  // seq != 0: the inspection reports through the mapped block (and left the
  // device counters zeroed); otherwise copy them back and clear them
  void set_fets(active_set_t &as, stat_t &stat, feature_t &fets, const config_t &conf, int64_t nvertexs,
                int64_t nedges, unsigned long long seq = 0) {
    if (!(seq && stat.await(seq))) {
      stat.collect(6);  // the one synchronisation of a standalone level
      stat.clean();
    }
    const level_counts c = {stat.active_num(),    stat.unactive_num(),   stat.push_workload(),
                            stat.pull_workload(), stat.max_deg_active(), stat.max_deg_unactive()};
    keep(c);
    if (fets_from_counts(fets, c, nvertexs, nedges)) {
      if (conf.conf_qmode == Cached) as.queue.swap();
      as.halt_host();
    }
  }
  void keep(const level_counts &c) {
    raw_frontier = c.active;
    raw_inactive = c.inactive;
    raw_push = c.push;
    raw_pull = c.pull;
    // the push max counter sums per-thread maxima, so it bounds the largest
    // active degree from above; the first level has only its workload
    raw_max_push = c.max_push > 0 ? c.max_push : c.push;
  }

  // raw counters of the last inspection (before cross() folding)
  int64_t raw_frontier = 0, raw_inactive = 0, raw_push = 0, raw_pull = 0, raw_max_push = 0;
};

// ===========================================================================
// selector_t
// ===========================================================================
__host__ __device__ inline LB lb_from_class(int l) { return l == 0 ? WM : (l == 1 ? CM : STRICT); }

struct selector_t {
  // null: the host tables; the in-stream selector points this at a copy of
  // the trees on the device
  const tree_set *trees = nullptr;
  __host__ __device__ const tree_set &T() const {
#ifdef __CUDA_ARCH__
    return *trees;
#else
    return trees ? *trees : host_tree_set();
#endif
  }

  void select(stat_t &stats, feature_t &fets, config_t &conf) { select_based_on_model(stats, fets, conf); }

  __host__ __device__ void trigger_fusion(const feature_t &fets, config_t &conf) {
    if (conf.force.has_fusion) return;
    if (!conf.conf_fuse_inspect) {
      const double potential = fets.push_workload_ratio + fets.pull_workload_ratio;
      if (potential < 0.001) {
        conf.conf_fuse_inspect = true;
        conf.conf_switch_to_fusion = true;
      }
      if (fets.growing_rate > 2) conf.conf_idle = 0;
      if (conf.conf_idle >= 3) {
        conf.conf_fuse_inspect = true;
        conf.conf_switch_to_fusion = true;
        conf.conf_idle = 0;
      }
    }
  }

  __host__ __device__ void fusion(const feature_t &fets, config_t &conf) {
    conf.conf_dir = Push;
    conf.conf_asfmt = Queue;
    conf.conf_cm = Interleave;
    conf.conf_lb = conf.force.has_lb && conf.force.lb != TWOD ? conf.force.lb : WM;
    conf.conf_fuse_inspect = true;
    conf.conf_centric = fets.centric;
    conf.conf_fromall = fets.fromall;
    conf.conf_toall = fets.toall;
    set_target(conf);
  }

  __host__ __device__ static void set_target(config_t &conf) {
    if (conf.conf_dir == Push)
      conf.conf_target = conf.conf_fromall ? All : Active;
    else
      conf.conf_target = (conf.conf_toall && conf.conf_dir == Pull) ? All : Inactive;
  }

  __host__ __device__ static void dir_ratios(const feature_t &fets, double *v) {
    const double *fv = fets.fv;
    v[0] = fv[8] / (fv[7] + 0.1);
    v[1] = fv[10] / (fv[9] + 0.1);
    v[2] = fv[16] / (fv[15] + 0.1);
    v[3] = fv[18] / (fv[17] + 0.1);
    v[4] = fv[9] / (fv[15] + 0.1);
    v[5] = fv[10] / (fv[16] + 0.1);
    v[6] = fv[9] / (fv[17] + 0.1);
    v[7] = fv[10] / (fv[18] + 0.1);
  }

  __host__ __device__ void select_idem(feature_t &fets, config_t &conf) {
    double v[16];
    dir_ratios(fets, v);
    conf.conf_dir = eval_tree(T().dir_idem, v) == 1 ? Pull : Push;
    if (fets.push_workload_ratio * 5 < fets.pull_workload_ratio) conf.conf_dir = Push;
    if (conf.force.has_direction) conf.conf_dir = conf.force.d;
    if (conf.conf_dir == Pull) {
      conf.conf_asfmt = fets.fv[12] < 0.01 ? Queue : Bitmap;
    } else {
      v[0] = fets.fv[11];
      conf.conf_asfmt = eval_tree(T().fmt, v) ? Bitmap : Queue;
    }
    if (conf.force.has_asfmt) conf.conf_asfmt = conf.force.asf;
    if (conf.conf_dir == Pull) {
      conf.conf_lb = TM;
    } else {
      int k = 0;
      for (int i = 0; i < 7; ++i) v[k++] = fets.fv[i];
      for (int i = 7; i < 18; i += 2) v[k++] = fets.fv[i];
      conf.conf_lb = lb_from_class(eval_tree(T().lb_idem, v));
    }
    if (conf.force.has_lb) conf.conf_lb = conf.force.lb;
  }

  __host__ __device__ void select_ASSO(feature_t &fets, config_t &conf) {
    double v[24];
    dir_ratios(fets, v);
    conf.conf_dir = eval_tree(T().dir_asso, v) == 1 ? Pull : Push;
    if (conf.force.has_direction) conf.conf_dir = conf.force.d;
    if (conf.conf_fromall && conf.conf_toall) {
      for (int i = 0; i < 7; ++i) v[i] = fets.fv[i];
      conf.conf_dir = eval_tree(T().dir_asso_backup, v) ? Pull : Push;
      if (conf.force.has_direction) conf.conf_dir = conf.force.d;
    }
    v[0] = conf.conf_dir == Push ? fets.fv[11] : fets.fv[12];
    conf.conf_asfmt = eval_tree(T().fmt, v) ? Bitmap : Queue;
    if (fets.fromall && fets.toall && !conf.conf_fixed) conf.conf_asfmt = Bitmap;
    if (conf.force.has_asfmt) conf.conf_asfmt = conf.force.asf;
    int k = 0;
    for (int i = 0; i < 7; ++i) v[k++] = fets.fv[i];
    int l;
    const bool all2all = conf.conf_fromall && conf.conf_toall && !conf.conf_fixed;
    if (conf.conf_dir == Pull) {
      if (all2all) {
        l = eval_tree(T().lb_asso_backward_backup, v);
      } else {
        for (int i = 8; i <= 18; i += 2) v[k++] = fets.fv[i];
        l = eval_tree(T().lb_asso_backward, v);
      }
    } else {
      if (all2all) {
        l = eval_tree(T().lb_asso_backward_backup, v);
      } else {
        for (int i = 7; i < 18; i += 2) v[k++] = fets.fv[i];
        l = eval_tree(T().lb_asso_forward, v);
      }
    }
    conf.conf_lb = lb_from_class(l);
    if (conf.force.has_lb) conf.conf_lb = conf.force.lb;
  }

  __host__ __device__ void select_Mono(feature_t &fets, config_t &conf) {
    conf.conf_dir = conf.force.has_direction ? conf.force.d : Push;
    conf.conf_asfmt = conf.force.has_asfmt ? conf.force.asf : Queue;
    double v[16];
    int k = 0;
    for (int i = 0; i < 7; ++i) v[k++] = fets.fv[i];
    for (int i = 7; i < 18; i += 2) v[k++] = fets.fv[i];
    conf.conf_lb = lb_from_class(eval_tree(T().lb_asso_forward, v));
    if (conf.force.has_lb) conf.conf_lb = conf.force.lb;
  }

  void select_based_on_model(stat_t &, feature_t &fets, config_t &conf) { decide(fets, conf); }

  // selector_t::select_based_on_model (selector.cuh:22-76)
  __host__ __device__ void decide(feature_t &fets, config_t &conf) {
    if (fets.centric == EC) {
      conf.conf_target = Active;
      conf.conf_asfmt = fets.active_vertex_ratio > 0.8 ? Bitmap : Queue;
      if (conf.force.has_asfmt) conf.conf_asfmt = conf.force.asf;
      conf.conf_fuse_inspect = false;
      return;
    }
    if (conf.conf_toall && conf.conf_fromall && !conf.conf_fixed) {
      conf.conf_inherit = true;
      return;
    }
    conf.conf_centric = fets.centric;
    conf.conf_fromall = fets.fromall;
    conf.conf_toall = fets.toall;
    if (fets.pattern == Idem)
      trigger_fusion(fets, conf);
    else
      conf.conf_fuse_inspect = conf.conf_fusion;
    if (conf.conf_fuse_inspect) {
      fusion(fets, conf);
      return;
    }
    if (fets.pattern == Idem)
      select_idem(fets, conf);
    else if (fets.pattern == ASSO)
      select_ASSO(fets, conf);
    else
      select_Mono(fets, conf);
    set_target(conf);
  }
};

// ===========================================================================
// tuned shapes
// ===========================================================================
constexpr int STRICT_TILE_MIN = 512;
constexpr int STRICT_SHAPES = 3;   // tile 1024 (default), 512, 2048
constexpr int PUSH_TM_SHAPES = 3;  // threads per CTA: 256 (default), 128, 512
constexpr int PULL_TM_SHAPES = 9;  // candidates per thread 2 (default), 1, 4, times those CTA sizes
inline int strict_tile_of(int shape) { return shape == 1 ? 512 : (shape == 2 ? 2048 : STRICT_TILE); }
inline int pull_tm_k_of(int shape) { return shape % 3 == 1 ? 1 : (shape % 3 == 2 ? 4 : 2); }
// thread-mapped variants: threads per CTA (push: of the shape, pull: of shape / 3)
inline int tm_threads_of(int cta_shape) { return cta_shape == 1 ? 128 : (cta_shape == 2 ? 512 : EXPAND_THREADS); }
// shapes a variant may take (1: none but the default)
inline int shape_count(bool pull, int lb) {
  if (lb == STRICT) return STRICT_SHAPES;
  if (lb == TM) return pull ? PULL_TM_SHAPES : PUSH_TM_SHAPES;
  return 1;
}

// ===========================================================================
// executor_t
// ===========================================================================
struct executor_t {
  int *dg_tile = nullptr;  // STRICT tile owners
  hub_piece_t *dg_hubs = nullptr;  // tiered push: hub pieces of the level
  int64_t hub_cap = 0;
  // Autotuned expand grids: for (pull, bitmap, load balance, fused) the grid
  // cap in quarters of the kernel's resident grid (0: the resident grid).
  struct tune_t {
    int quarters[2][2][8][2] = {};
    // tuned shape per variant (0: the default): STRICT variants pick the tile
    // (strict_tile_of), the thread-mapped pull its candidates per thread
    // (pull_tm_k_of); other variants have no shape
    int shapes[2][2][8][2] = {};
  } tune;
  twod_layout twod;                 // 2D-partition layout of the current graph
  int64_t persistent_levels = 0;    // levels run inside persistent launches
  int64_t persistent_launches = 0;  // persistent launches
  bool last_persistent = false;     // the last expand was a persistent launch
  // zero-copy report of persistent launches (mapped pinned, 3 words; see
  // persist_state::sig) and the tag of the last one
  unsigned long long *h_psig = nullptr, *d_psig = nullptr;
  unsigned long long psig_seq = 0;
  Computation pattern = Idem;       // pattern of the run being expanded
  int64_t tile_cap = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  inspector_t *insp = nullptr;  // source of the host-known frontier sizes

  void destroy() {
    cudaFree(dg_tile);
    dg_tile = nullptr;
    tile_cap = 0;
    cudaFree(dg_hubs);
    dg_hubs = nullptr;
    hub_cap = 0;
    if (h_psig) cudaFreeHost(h_psig);
    h_psig = d_psig = nullptr;
    for (auto &e : ev)
      if (e) {
        cudaEventDestroy(e);
        e = nullptr;
      }
  }

  // bitmap -> queue (src/kernel_libs/filter.cuh:197-252)
  void build_queue(active_set_t &as, Status target, bool sorted) {
    const int64_t nwords = (as.size + 31) >> 5;
    if (nwords == 0) {  // an empty set (an edge-centric run without edges): an empty queue
      GSW_CUDA(cudaMemsetAsync(as.queue.output_size_ptr(), 0, sizeof(int), stream()));
      return;
    }
    if (sorted) {
      const int64_t nb = (nwords + FILTER_WORDS - 1) / FILTER_WORDS;
      if (nb + 1 > as.workset.bsum_cap) return (void)set_error(GSW_ERR_OVERFLOW, "filter: %s", "block sums");
      k_filter_count<<<(unsigned)nb, FILTER_WORDS, 0, stream()>>>(as, target, as.workset.dg_bsum);
      k_scan_single_block<<<1, 1024, 0, stream()>>>(as.workset.dg_bsum, nb);
      k_filter_write<<<(unsigned)nb, FILTER_WORDS, 0, stream()>>>(as, target, as.workset.dg_bsum, nb);
    } else {
      // the append builder starts from an empty output whatever ran before
      GSW_CUDA(cudaMemsetAsync(as.queue.output_size_ptr(), 0, sizeof(int), stream()));
      const int grid = clamp_grid((nwords + 255) / 256, resident_grid(k_filter_unsorted, 256));
      k_filter_unsorted<<<grid, 256, 0, stream()>>>(as, target);
    }
    GSW_LAUNCHED();
  }

  template <typename G, typename F>
  void filter(active_set_t &as, G &g, F &f, stat_t &stat, feature_t &fets, config_t &conf) {
    const double s = stat.last_filter_time;
    as.set_fmt(conf.conf_asfmt);
    if (conf.conf_asfmt == Queue) {
      if (level_builds_queue(conf)) {
        if (!(as.queue.mode == Cached && as.queue.traceback)) build_queue(as, conf.conf_target, conf.conf_sorted_queue);
      } else if (!conf.conf_pruning) {
        fill_u32(as.bitmap.visited.dg_bits, 0, as.bitmap.visited.n_words);
      }
      as.queue.swap();
    }
    // grid bookkeeping of the reference (executor.cuh:30-52): idle levels
    // feed trigger_fusion, tiny STRICT levels fall back to CM
    level_grid_bookkeeping(fets, conf);
    set_hints(as, fets, conf);
    if (conf.conf_centric == VC && conf.conf_fuse_inspect && !conf.conf_first_round && conf.conf_compensation &&
        as.fmt == Queue)
      compensation(as, g, f);
    const double e = now_ms();
    stat.level = g.level;
    stat.last_filter_time = e - s;
    stat.avg_filter_time = (stat.avg_filter_time * g.level + stat.last_filter_time) / (g.level + 1);
    fets.last_filter_time = stat.last_filter_time;
    fets.avg_filter_time = stat.avg_filter_time;
  }

  void set_hints(active_set_t &as, const feature_t &fets, const config_t &conf) {
    hints_t &h = hints();
    if (as.fmt == Bitmap) {
      h.frontier = as.size;
    } else if (!conf.conf_fuse_inspect && insp) {
      const Status t = conf.conf_target;
      h.frontier = t == Active ? insp->raw_frontier : (t == Inactive ? insp->raw_inactive : insp->raw_frontier + insp->raw_inactive);
      if (conf.conf_qmode == Cached && as.queue.traceback) h.frontier = as.size;
    } else {
      h.frontier = -1;  // fused: the device knows; use resident grids
    }
    if (!conf.conf_fuse_inspect && insp)
      h.edges = conf.conf_dir == Push ? insp->raw_push + (conf.conf_target == All ? insp->raw_pull : 0)
                                      : insp->raw_pull + (conf.conf_target == All ? insp->raw_push : 0);
    else
      h.edges = -1;
    if (h.frontier < 0 || h.frontier > as.size) h.frontier = -1;
    h.max_deg = (!conf.conf_fuse_inspect && insp && conf.conf_dir == Push && conf.conf_target == Active &&
                 as.fmt == Queue)
                    ? insp->raw_max_push
                    : -1;
  }

  // deferred filter updates of fused levels (kernel_fusion.cuh:54-109)
  template <typename E, typename F>
  void compensation(active_set_t &as, device_graph_t<CSR, E> &g, F &f) {
    using G = device_graph_t<CSR, E>;
    const int grid = resident_grid(k_compensation<G, F>, 512);
    k_compensation<G, F><<<grid, 512, 0, stream()>>>(as, g, f);
    GSW_LAUNCHED();
  }
  template <typename E, typename F>
  void compensation(active_set_t &, device_graph_t<COO, E> &, F &) {}

  // The hub list of a per-launch push whose hubs start at min_deg columns,
  // or none when the inspection bounds the frontier's degrees below that
  template <typename E>
  hub_list_t hub_list_for(active_set_t &as, const device_graph_t<CSR, E> &g, int min_deg) {
    const int64_t md = hints().max_deg;
    if (md >= 0 && md < min_deg) return hub_list_t();
    ensure_hubs(g.nedges);
    if (!ok() || !dg_hubs) return hub_list_t();
    return hub_list_t{dg_hubs, &as.dg_cnt->hub_pieces, &as.dg_cnt->hub_done, hub_cap};
  }

  // room for every hub piece a level can list: at most one piece per
  // EXPAND_THREADS arcs plus one per TWC_HUB_PIECE arcs
  void ensure_hubs(int64_t arcs) {
    const int64_t need = arcs / EXPAND_THREADS + arcs / TWC_HUB_PIECE + 2;
    if (need <= hub_cap) return;
    cudaFree(dg_hubs);
    dg_hubs = nullptr;
    if (GSW_CUDA(cudaMalloc((void **)&dg_hubs, sizeof(hub_piece_t) * need))) return;
    hub_cap = need;
  }

  // the table is sized for the smallest tile any shape uses
  void ensure_tiles(int64_t slots_cap) {
    const int64_t need = slots_cap / STRICT_TILE_MIN + 2;
    if (need <= tile_cap) return;
    cudaFree(dg_tile);
    dg_tile = nullptr;
    if (GSW_CUDA(cudaMalloc((void **)&dg_tile, sizeof(int) * need))) return;
    tile_cap = need;
  }

  template <bool PULL, int T, typename G>
  void strict_prepare(active_set_t &as, G &g, Status want) {
    const int64_t items = hints().frontier >= 0 ? hints().frontier : (as.fmt == Queue ? as.size + 1 : as.size);
    const int64_t nb = items / STRICT_ITEMS + 1;
    ensure_tiles(g.nedges + as.size + 1);
    if (!ok()) return;
    if (nb + 1 > as.workset.bsum_cap) return (void)set_error(GSW_ERR_OVERFLOW, "strict: %s", "block sums");
    if (nb == 1 && hints().frontier >= 0) {
      // a frontier known to fit one scan block: one launch, no block sums
      k_strict_scan<PULL, T><<<1, 256, 0, stream()>>>(as, g, want, nullptr, 1, dg_tile, tile_cap);
    } else if (hints().frontier < 0) {
      // a frontier only the device knows (fused levels, captured loops): a
      // fixed grid over its own number of scan blocks, not the capacity's
      const int grid = (int)MIN(nb, (int64_t)sm_count() * 8);
      k_strict_count<PULL><<<grid, 256, 0, stream()>>>(as, g, want, as.workset.dg_bsum);
      k_strict_bsum_scan<<<1, 1024, 0, stream()>>>(as, as.workset.dg_bsum);
      k_strict_scan<PULL, T><<<grid, 256, 0, stream()>>>(as, g, want, as.workset.dg_bsum, -1, dg_tile, tile_cap);
    } else {
      k_strict_count<PULL><<<(unsigned)nb, 256, 0, stream()>>>(as, g, want, as.workset.dg_bsum);
      k_scan_single_block<<<1, 1024, 0, stream()>>>(as.workset.dg_bsum, nb);
      k_strict_scan<PULL, T><<<(unsigned)nb, 256, 0, stream()>>>(as, g, want, as.workset.dg_bsum, nb, dg_tile,
                                                                tile_cap);
    }
    GSW_LAUNCHED();
  }

  template <typename E, typename F>
  void launch_vc(active_set_t &as, device_graph_t<CSR, E> &g, F &f, config_t &conf) {
    using G = device_graph_t<CSR, E>;
    const bool fused = conf.conf_fuse_inspect;
    const int64_t fr = hints().frontier;
    const int64_t ed = hints().edges;
    const int B = EXPAND_THREADS;
    const int fg = opts().force_grid;
    // autotuned grid of this variant: quarters of the resident grid
    const int tq = tune.quarters[conf.conf_dir == Pull][as.fmt == Bitmap][(int)conf.conf_lb & 7][fused ? 1 : 0];
    const int shape = tune.shapes[conf.conf_dir == Pull][as.fmt == Bitmap][(int)conf.conf_lb & 7][fused ? 1 : 0];
    auto grid_for = [&](auto kern, int64_t want) {
      const int res = resident_grid(kern, B);
      if (fg > 0) return fg;
      const int cap = tq > 0 ? (int)MAX((int64_t)1, (int64_t)res * tq / 4) : res;
      return want < 0 ? cap : clamp_grid(want, cap);
    };
    // the same for a kernel launched with bt threads per CTA
    auto grid_for_bt = [&](auto kern, int64_t want, int bt) {
      const int res = resident_grid(kern, bt);
      if (fg > 0) return fg;
      const int cap = tq > 0 ? (int)MAX((int64_t)1, (int64_t)res * tq / 4) : res;
      return want < 0 ? cap : clamp_grid(want, cap);
    };
#define GSW_GO(kern, want, ...)                                   \
  do {                                                            \
    auto _k = kern;                                               \
    _k<<<grid_for(_k, want), B, 0, stream()>>>(__VA_ARGS__);      \
  } while (0)
// the hub pieces a per-launch push listed, one per CTA
#define GSW_HUBS(hl)                                                          \
  do {                                                                        \
    if ((hl).piece) {                                                         \
      if (fused) GSW_GO((k_push_twc_hubs<true, G, F>), -1, as, g, f, conf, hl);  \
      else GSW_GO((k_push_twc_hubs<false, G, F>), -1, as, g, f, conf, hl);       \
    }                                                                         \
  } while (0)
    if (conf.conf_lb == TWOD) {
      launch_twod(g, f, conf);
      return;
    }
    if (conf.conf_dir == Push && fused && conf.conf_persistent && as.queue.mode == Normal) {
      launch_persistent(as, g, f, conf);
      return;
    }
    if (conf.conf_dir == Push) {
      switch (conf.conf_lb) {
        case TM:
        {
          // thread-mapped: the tuned CTA size (BT threads)
          auto go = [&](auto bt) {
            constexpr int BT = decltype(bt)::value;
            auto k = fused ? k_push_tm<true, BT, G, F> : k_push_tm<false, BT, G, F>;
            k<<<grid_for_bt(k, fr < 0 ? -1 : fr / BT + 1, BT), BT, 0, stream()>>>(as, g, f, conf);
          };
          switch (tm_threads_of(shape)) {
            case 128: go(std::integral_constant<int, 128>{}); break;
            case 512: go(std::integral_constant<int, 512>{}); break;
            default: go(std::integral_constant<int, EXPAND_THREADS>{}); break;
          }
        }
          break;
        case CM:
          {
            const hub_list_t hl = hub_list_for(as, g, CM_HUB_MIN);
            if (!ok()) return;
            if (fused) GSW_GO((k_push_cm<true, G, F>), fr < 0 ? -1 : fr / B + 1, as, g, f, conf, hl);
            else GSW_GO((k_push_cm<false, G, F>), fr < 0 ? -1 : fr / B + 1, as, g, f, conf, hl);
            GSW_HUBS(hl);
          }
          break;
        case TWC: {
          // tiles, then the hub pieces they listed (one piece per CTA)
          const hub_list_t hl = hub_list_for(as, g, B);
          if (!ok()) return;
          if (fused) GSW_GO((k_push_twc<true, G, F>), fr < 0 ? -1 : fr / B + 1, as, g, f, conf, hl);
          else GSW_GO((k_push_twc<false, G, F>), fr < 0 ? -1 : fr / B + 1, as, g, f, conf, hl);
          GSW_HUBS(hl);
          break;
        }
        case STRICT: {
          auto go = [&](auto tile) {
            constexpr int T = decltype(tile)::value;
            strict_prepare<false, T>(as, g, conf.want());
            if (!ok()) return;
            const int64_t want = (ed < 0 || fr < 0) ? -1 : (ed + fr) / T + 1;
            if (fused) GSW_GO((k_push_strict<true, T, G, F>), want, as, g, f, conf, dg_tile);
            else GSW_GO((k_push_strict<false, T, G, F>), want, as, g, f, conf, dg_tile);
          };
          switch (strict_tile_of(shape)) {
            case 512: go(std::integral_constant<int, 512>{}); break;
            case 2048: go(std::integral_constant<int, 2048>{}); break;
            default: go(std::integral_constant<int, STRICT_TILE>{}); break;
          }
          if (!ok()) return;
          break;
        }
        case WM:
        default:
          {
            const hub_list_t hl = hub_list_for(as, g, WM_HUB_MIN);
            if (!ok()) return;
            if (fused) GSW_GO((k_push_wm<true, G, F>), fr < 0 ? -1 : fr / B + 1, as, g, f, conf, hl);
            else GSW_GO((k_push_wm<false, G, F>), fr < 0 ? -1 : fr / B + 1, as, g, f, conf, hl);
            GSW_HUBS(hl);
          }
          break;
      }
    } else {
      switch (conf.conf_lb) {
        case WM: GSW_GO((k_pull_wm<G, F>), fr < 0 ? -1 : fr / B + 1, as, g, f, conf); break;
        case CM: GSW_GO((k_pull_cm<G, F>), fr < 0 ? -1 : fr / B + 1, as, g, f, conf); break;
        case TWC: GSW_GO((k_pull_twc<G, F>), fr < 0 ? -1 : fr / B + 1, as, g, f, conf); break;
        case STRICT: {
          // from-all pulls stage a per-vertex sum too: their tiles stop at
          // 1,024 slots (48 KB of static shared memory)
          const bool all = sizeof(typename F::wa_t) <= 4 && conf.conf_fromall;
          auto go = [&](auto tile) {
            constexpr int T = decltype(tile)::value;
            strict_prepare<true, T>(as, g, conf.want());
            if (!ok()) return;
            const int64_t want = (ed < 0 || fr < 0) ? -1 : (ed + fr) / T + 1;
            if constexpr (sizeof(typename F::wa_t) <= 4 && T <= 1024) {
              if (all) {
                GSW_GO((k_pull_strict_all<T, G, F>), want, as, g, f, conf, dg_tile);
                return;
              }
            }
            GSW_GO((k_pull_strict<T, G, F>), want, as, g, f, conf, dg_tile);
          };
          const int t = strict_tile_of(shape);
          if (t == 512)
            go(std::integral_constant<int, 512>{});
          else if (t == 2048 && !all)
            go(std::integral_constant<int, 2048>{});
          else
            go(std::integral_constant<int, STRICT_TILE>{});
          if (!ok()) return;
          break;
        }
        case TM:
        default: {
          // K candidates per thread and BT threads per CTA, as tuned
          auto go = [&](auto kc, auto bt) {
            constexpr int K = decltype(kc)::value, BT = decltype(bt)::value;
            auto kern = k_pull_tm<K, BT, G, F>;
            kern<<<grid_for_bt(kern, fr < 0 ? -1 : fr / BT + 1, BT), BT, 0, stream()>>>(as, g, f, conf);
          };
          auto with_k = [&](auto bt) {
            switch (pull_tm_k_of(shape)) {
              case 1: go(std::integral_constant<int, 1>{}, bt); break;
              case 4: go(std::integral_constant<int, 4>{}, bt); break;
              default: go(std::integral_constant<int, 2>{}, bt); break;
            }
          };
          switch (tm_threads_of(shape / 3)) {
            case 128: with_k(std::integral_constant<int, 128>{}); break;
            case 512: with_k(std::integral_constant<int, 512>{}); break;
            default: with_k(std::integral_constant<int, EXPAND_THREADS>{}); break;
          }
          break;
        }
      }
    }
#undef GSW_HUBS
#undef GSW_GO
    GSW_LAUNCHED();
  }

  // Consecutive fused levels in one cooperative launch (k_persistent.cuh).
  // Afterwards the host state looks as if the levels had run one by one:
  // g.level is advanced, the last output queue sits where the next swap
  // expects it, an empty frontier halts the loop, and a frontier that grew
  // past the limit returns the loop to the inspected (standalone) form so the
  // selector can pick direction and format again.
  template <typename E, typename F>
  void launch_persistent(active_set_t &as, device_graph_t<CSR, E> &g, F &f, config_t &conf) {
    switch (conf.conf_lb) {
      case TM: return launch_persistent_lb<TM>(as, g, f, conf);
      case CM: return launch_persistent_lb<CM>(as, g, f, conf);
      case STRICT: return launch_persistent_lb<STRICT>(as, g, f, conf);
      case TWC: return launch_persistent_lb<TWC>(as, g, f, conf);
      default: return launch_persistent_lb<WM>(as, g, f, conf);
    }
  }

  template <int LB, typename E, typename F>
  void launch_persistent_lb(active_set_t &as, device_graph_t<CSR, E> &g, F &f, config_t &conf) {
    using G = device_graph_t<CSR, E>;
    auto kern = k_fused_persistent<LB, G, F>;
    const int grid = resident_grid(kern, EXPAND_THREADS);
    if (LB == STRICT) {
      ensure_tiles(g.nedges + as.size + 1);
      if (!ok()) return;
      if (grid > as.workset.bsum_cap) return (void)set_error(GSW_ERR_OVERFLOW, "persistent strict: %s", "block sums");
    }
    as_counters_t *c = as.dg_cnt;
    const int cur = as.queue.cursor;
    k_persist_prep<<<1, 1, 0, stream()>>>(c, cur);
    persist_state ps;
    ps.q[0] = as.queue.subqueue[cur].dg_queue;
    ps.q[1] = as.queue.subqueue[cur ^ 1].dg_queue;
    ps.cnt = c->pq;
    ps.cap = as.queue.subqueue[0].max_size;
    // only Idem patterns leave fused mode when the frontier grows (the
    // selector keeps Mono / ASSO patterns fused level after level)
    ps.grow_limit = pattern == Idem ? (int)MAX((int64_t)4096, as.size / 64) : INT32_MAX;
    ps.max_levels = (int)MIN(as.size + 2, (int64_t)(1 << 24));  // a BFS-like frontier runs at most n levels
    ps.budget_ns = opts().barrier_leave_test ? 20000000ull : 2000000000ull;  // per barrier wait
    ps.leave_block = opts().barrier_leave_test ? 0 : -1;
    ps.levels_done = &c->plevels;
    ps.exit_reason = &c->preason;
    ps.lb_out = &c->plb;
    ps.cur = cur;
    ps.level0 = nullptr;
    if (!h_psig) {
      // without the mapped block the launch reports through a copy-back
      if (cudaHostAlloc((void **)&h_psig, 4 * sizeof(unsigned long long), cudaHostAllocMapped) == cudaSuccess) {
        memset(h_psig, 0, 4 * sizeof(unsigned long long));
        if (cudaHostGetDevicePointer((void **)&d_psig, h_psig, 0) != cudaSuccess) {
          cudaGetLastError();
          cudaFreeHost(h_psig);
          h_psig = d_psig = nullptr;
        }
      } else {
        cudaGetLastError();
        h_psig = nullptr;
      }
    }
    const unsigned long long seq = d_psig ? (++psig_seq % 0xffffffull) + 1 : 0;
    ps.sig = seq ? d_psig : nullptr;
    ps.seq = seq;
    ps.eoff = as.workset.dg_eoff;
    ps.eoff_cap = as.size + 2;
    ps.bsum = as.workset.dg_bsum;
    ps.tile_lo = dg_tile;
    ps.tile_cap = tile_cap;
    void *args[] = {(void *)&as, (void *)&g, (void *)&f, (void *)&conf, (void *)&ps};
    if (GSW_CUDA(cudaLaunchCooperativeKernel((const void *)kern, grid, EXPAND_THREADS, args, 0, stream()))) return;
    GSW_LAUNCHED();
    int res[3] = {0, -1, -1};
    if (!(seq && await_persist(seq, res))) {
      GSW_CUDA(cudaMemcpyAsync(res, &c->plevels, sizeof(res), cudaMemcpyDeviceToHost, stream()));
      GSW_CUDA(cudaStreamSynchronize(stream()));
    }
    const int L = res[0], reason = res[1];
    hints().persistent_lb = res[2];
    persistent_levels += L;
    persistent_launches++;
    last_persistent = true;
    if (reason == 4) {
      set_error(GSW_ERR_OVERFLOW, "%s", "persistent STRICT levels: frontier exceeds the scan buffer");
      return;
    }
    if (reason == 3 || reason < 0) {
      set_error(GSW_ERR_TIMEOUT, "%s", "persistent fused levels: grid barrier timed out");
      return;
    }
    if (L > 0) g.level += L - 1;
    // the kernel published its last output (q[L & 1]) in the output slot
    as.queue.cursor = (cur ^ (L & 1)) ^ 1;
    if (reason == 0) as.halt_host();
    if (reason == 1) {
      // back to inspected levels: the queue is rebuilt from the bitmaps
      conf.conf_fuse_inspect = false;
      as.queue.clean_size(0);
      as.queue.clean_size(1);
    }
  }

  // Waits for the persistent launch tagged `seq` to report {levels, reason,
  // LB} through the mapped block.  Every 256 polls the stream is queried, so
  // a launch that ended without reporting (a block left early) ends the wait:
  // false then, and the caller copies the device words back.
  bool await_persist(unsigned long long seq, int res[3]) {
    volatile unsigned long long *h = h_psig;
    auto arrived = [&] { return (h[0] >> 40) == seq && (h[1] >> 40) == seq && (h[2] >> 40) == seq; };
    for (unsigned spin = 1;; ++spin) {
      if (arrived()) break;
      if ((spin & 255) == 0) {
        const cudaError_t q = cudaStreamQuery(stream());
        if (q != cudaErrorNotReady) {
          if (arrived()) break;
          if (q != cudaSuccess) GSW_CUDA(q);
          return false;
        }
      }
    }
    const unsigned long long m = (1ull << 40) - 1;
    res[0] = (int)(h[0] & m);
    res[1] = (int)(h[1] & m) - 1;
    res[2] = (int)(h[2] & m);
    return true;
  }

  // 2D-partition expand (k_twod.cuh): all sources to all destinations, so
  // only for from-all / to-all patterns, unweighted, 4-byte messages
  template <typename E, typename F>
  void launch_twod(device_graph_t<CSR, E> &g, F &f, config_t &conf) {
    using G = device_graph_t<CSR, E>;
    using WA = typename F::wa_t;
    if constexpr (sizeof(WA) <= 4 && std::is_same<E, Empty>::value) {
      if (!conf.conf_fromall || !conf.conf_toall) {
        set_error(GSW_ERR_UNSUPPORTED, "%s", "2D-partition expand needs a from-all/to-all pattern");
        return;
      }
      if (!twod.edge) {
        set_error(GSW_ERR_UNSUPPORTED, "%s", "2D-partition layout not built for this graph");
        return;
      }
      const int grid = (int)MAX((int64_t)1, MIN(twod.nitems, (int64_t)resident_grid(k_twod<G, F>, TWOD_THREADS)));
      k_twod<G, F><<<grid, TWOD_THREADS, 0, stream()>>>(g, f, twod);
      GSW_LAUNCHED();
    } else {
      set_error(GSW_ERR_UNSUPPORTED, "%s", "2D-partition expand needs unweighted edges and 4-byte vertex data");
    }
  }

  template <typename E, typename F>
  void launch_ec(active_set_t &as, device_graph_t<COO, E> &g, F &f) {
    const int grid = resident_grid(k_expand_ec<device_graph_t<COO, E>, F>, 512);
    k_expand_ec<<<grid, 512, 0, stream()>>>(as, g, f);
    GSW_LAUNCHED();
  }

  template <typename E, typename F>
  void dispatch(active_set_t &as, device_graph_t<CSR, E> &g, F &f, config_t &conf) {
    launch_vc(as, g, f, conf);
  }
  template <typename E, typename F>
  void dispatch(active_set_t &as, device_graph_t<COO, E> &g, F &f, config_t &) {
    launch_ec(as, g, f);
  }

  template <typename G, typename F>
  void expand(active_set_t &as, G &g, F &f, stat_t &stat, feature_t &fets, config_t &conf) {
    const double s = now_ms();
    // fused levels read the convergence flag right after the expand
    const bool sync_needed = conf.conf_fuse_inspect || opts().verbose;
    if (sync_needed && !ev[0])
      for (auto &e : ev) cudaEventCreate(&e);
    if (conf.conf_count_edges) GSW_CUDA(cudaMemsetAsync(&as.dg_cnt->scanned, 0, sizeof(unsigned long long), stream()));
    if (sync_needed) cudaEventRecord(ev[0], stream());
    marks().exp0 = opts().timing ? timing_pool().record() : -1;
    last_persistent = false;
    pattern = fets.pattern;
    dispatch(as, g, f, conf);
    hints().persistent = last_persistent;
    marks().exp1 = opts().timing ? timing_pool().record() : -1;
    double e = s;
    if (sync_needed) {
      cudaEventRecord(ev[1], stream());
      GSW_CUDA(cudaStreamSynchronize(stream()));
      float ms = 0;
      cudaEventElapsedTime(&ms, ev[0], ev[1]);
      e = s + ms;
    }
    stat.last_scanned = 0;
    if (conf.conf_count_edges) {
      unsigned long long c = 0;
      GSW_CUDA(cudaMemcpyAsync(&c, &as.dg_cnt->scanned, sizeof(c), cudaMemcpyDeviceToHost, stream()));
      GSW_CUDA(cudaStreamSynchronize(stream()));
      stat.last_scanned = (int64_t)c;
    }
    stat.last_time = stat.last_filter_time + e - s;
    const int lv = g.level > 0 ? g.level : 1;
    stat.avg_time = (stat.avg_time * (lv - 1) + stat.last_time) / lv;
    stat.last_expand_time = e - s;
    stat.avg_expand_time = (stat.avg_expand_time * (lv - 1) + stat.last_expand_time) / lv;
    fets.last_expand_time = stat.last_expand_time;
    // a fused level that is far slower than average goes back to the
    // standalone form (executor.cuh:128-131)
    if (fets.pattern == Idem && fets.avg_expand_time > 0 && fets.last_expand_time > 5 * fets.avg_expand_time &&
        !conf.force.has_fusion && !last_persistent) {
      conf.conf_fuse_inspect = false;
      as.queue.swap();
    }
    fets.avg_expand_time = stat.avg_expand_time;
    fets.last_time = stat.last_time;
    fets.avg_time = stat.avg_time;
    if (opts().verbose) {
      stat.show_hints();
      conf.show_hints();
      printf("\n");
    }
    conf.conf_first_round = false;
  }

};

// ===========================================================================
// convergence (active_set.cuh:37-43, notification.cuh:233-254)
// ===========================================================================
template <typename E, typename F>
bool window_exit(active_set_t &as, device_graph_t<CSR, E> &g, F &f, config_t &conf) {
  if (!conf.conf_window) return true;
  GSW_CUDA(cudaMemsetAsync(&as.dg_cnt->cnt, 0, sizeof(int), stream()));
  k_exit<<<resident_grid(k_exit<device_graph_t<CSR, E>, F>, 512), 512, 0, stream()>>>(g, f, &as.dg_cnt->cnt);
  int c = 0;
  GSW_CUDA(cudaMemcpyAsync(&c, &as.dg_cnt->cnt, sizeof(int), cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  if (c) {
    as.nt.reset();
    f.data.window.reset();
    if (conf.conf_fusion) {
      conf.conf_fuse_inspect = false;
      conf.conf_switch_to_fusion = true;
    }
    return false;
  }
  return true;
}
template <typename E, typename F>
bool window_exit(active_set_t &, device_graph_t<COO, E> &, F &, config_t &) {
  return true;
}

template <typename E, typename F>
void window_delay_update(active_set_t &as, device_graph_t<CSR, E> &g, F &f) {
  k_filter_all<<<resident_grid(k_filter_all<device_graph_t<CSR, E>, F>, 512), 512, 0, stream()>>>(g, f, as.size);
  GSW_LAUNCHED();
}
template <typename E, typename F>
void window_delay_update(active_set_t &, device_graph_t<COO, E> &, F &) {}

template <typename G, typename F>
bool finish(active_set_t &as, G &g, F &f, config_t &conf) {
  if (!ok()) return true;  // an error ends the loop; the caller reports it
  const bool converged = as.is_converged();
  if (conf.conf_window && conf.conf_fusion && converged) window_delay_update(as, g, f);
  return converged && window_exit(as, g, f, conf);
}

template <typename G, typename F, typename C>
bool active_set_t::finish(G &g, F &f, C &conf) {
  return gsw::finish(*this, g, f, conf);
}

// ===========================================================================
// init_conf / reset_conf (src/gswitch.h:19-108)
// ===========================================================================
template <typename E>
int64_t root_degree(const device_graph_t<CSR, E> &g, int root) {
  int d = 0;
  GSW_CUDA(cudaMemcpyAsync(&d, g.dg_odegree + root, sizeof(int), cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  return d;
}
template <typename E>
int64_t root_degree(const device_graph_t<COO, E> &, int) {
  return 0;
}

template <typename G, typename F>
void init_conf_impl(stat_t &stats, feature_t &fets, config_t &conf, G &dg, F &f, double mean_weight,
                    double avg_deg_attr, bool reset_only, int64_t known_root_degree = -1) {
  if (reset_only)
    conf.reset();
  else
    stats.build();
  fets.architecture_features();
  conf.conf_inherit = false;
  if (fets.use_root >= 0)
    fets.first_workload =
        (double)(known_root_degree >= 0 ? known_root_degree : root_degree(dg, fets.use_root));
  if (fets.centric == VC) {
    fets.flatten();
    double v[5];
    for (int i = 2; i < 7; ++i) v[i - 2] = fets.fv[i];
    conf.conf_fuse_inspect = eval_tree(select_fusion_tree, v) != 0;
    if (conf.force.has_fusion) conf.conf_fuse_inspect = conf.force.fusion == Fused;
    // from-all/to-all patterns update vertex state only in the inspector's
    // filter pass, so a fused level (which skips it) cannot advance them:
    // they stay standalone even when fusion is forced
    if (fets.toall && fets.fromall) conf.conf_fuse_inspect = false;
    if (conf.conf_fuse_inspect) conf.conf_fusion = true;
    if (!conf.conf_fuse_inspect) conf.conf_qmode = Normal;
  }
  if (conf.conf_window) {
    f.data.window.enable = true;
    f.data.window.set_init_winsize(DIV(8 * mean_weight * 32, avg_deg_attr));
  }
}

// CC root compression after each hooking level (intrinsics.cuh:351-362)
template <typename F>
void p_jump(F &f, int64_t nvertexs, active_set_t &as) {
  const int grid = resident_grid(k_pointer_jump, 512);
  k_pointer_jump<<<grid, 512, 0, stream()>>>((int *)f.data.dg_wa, nvertexs, &as.dg_cnt->err);
  GSW_LAUNCHED();
}

}  // namespace gsw
