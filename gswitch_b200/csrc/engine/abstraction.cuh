// Operator-facing state: vdata_t / Functor, the SSSP window, and the
// feature / statistics / configuration records of the level loop.
//
// Names, fields and meanings follow the reference (src/data_structures/
// functor.cuh:12-98, window.cuh:44-123, src/abstraction/features.cuh:13-84,
// statistics.cuh:11-30, config.cuh:9-122) so functors and level loops
// written against it compile unchanged.  Differences: the Functor base has no
// virtual methods (user functors are concrete template arguments, so calls
// bind statically and the object stays a plain kernel argument); statistics
// counters are 64-bit (frontier workloads exceed 2^31 on scale-26 graphs);
// a forced-variant override (the reference's `-c Dir-Fmt-LB-Fusion`) lives
// in config_t so one process can run several forced configurations.
#pragma once
#include <sstream>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "frontier.cuh"
#include "graph.cuh"
#include "selector_trees.h"

namespace gsw {

__host__ __device__ inline int eval_tree(const tree_node *t, const double *fv) {
  int i = 0;
  for (int guard = 0; guard < 4096 && t[i].feat >= 0; ++guard)
    i = fv[t[i].feat] <= t[i].thr ? t[i].left : t[i].right;
  return t[i].left;
}
inline int eval_tree(const tree_node *t, const std::vector<double> &fv) { return eval_tree(t, fv.data()); }

// The selector's trees: the host tables of selector_trees.h, or their copy in
// device memory for the in-stream selector of the captured level loop.
struct tree_set {
  const tree_node *dir_idem, *dir_asso, *dir_asso_backup, *fmt, *fusion, *lb_idem, *lb_asso_forward,
      *lb_asso_backward, *lb_asso_backward_backup;
};
inline const tree_set &host_tree_set() {
  static const tree_set t = {select_dir_idem_tree, select_dir_asso_tree, select_dir_asso_backup_tree,
                             select_fmt_tree,      select_fusion_tree,   select_lb_idem_tree,
                             select_lb_asso_forward_tree, select_lb_asso_backward_tree,
                             select_lb_asso_backward_backup_tree};
  return t;
}

// Products in decision arithmetic are rounded on their own (never fused into
// a multiply-add), so the device selector reproduces the host's doubles bit
// for bit.
__host__ __device__ __forceinline__ double mul_unfused(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}

}  // namespace gsw

// ---------------------------------------------------------------------------
// SSSP stepping window (src/data_structures/window.cuh:44-123): vertices are
// admitted while their value lies in [th, th + wsz); the size shrinks,
// inflates or resets per level from a two-feature tree.
// ---------------------------------------------------------------------------
struct window_t {
  double th = 0, wsz_lim = 0, wsz = 0;
  double shrink_rate = 0.3;
  double inflat_rate = 0.1;
  double reset_rate = 1;
  int win_bot = 3328;
  int win_top = 33679;
  bool enable = false;

  __host__ __device__ bool too_large(double size) const { return size > 5 * 33679; }
  __host__ __device__ bool ok(int size) const { return size <= win_top && size > win_bot; }
  void set_lim(int bot, int top) {
    win_bot = bot;
    win_top = top;
  }
  template <typename FT, typename CT>
  void adjust(const FT &fets, const CT &conf) {
    adjust_with(fets, conf, gsw::select_stepping_tree);
  }
  // the same step on the device, with a device copy of the stepping tree
  template <typename FT, typename CT>
  __host__ __device__ void adjust_with(const FT &fets, const CT &conf, const gsw::tree_node *stepping) {
    if (conf.conf_fusion) {
      wsz = wsz_lim;
      return;
    }
    double v1[2];
    v1[0] = fets.active_vertex;
    v1[1] = v1[0] * fets.cur_avg_deg_active;
    int l = gsw::eval_tree(stepping, v1);
    if (enable) {
      if (l == 1) {
        shrink();
        if (too_large(v1[1])) shrink();
      } else if (l == 0) {
        inflat();
      }
    }
  }
  void set_init_winsize(double lim) {
    th = 0;
    wsz_lim = lim;
    wsz = lim;
  }
  __host__ __device__ void shrink() { wsz = wsz * shrink_rate; }
  __host__ __device__ void inflat() {
    wsz = wsz / inflat_rate;
    if (wsz > wsz_lim) wsz = wsz_lim;
  }
  __host__ __device__ __forceinline__ bool in(float x) const {
    if (!enable) return true;
    return x < th + wsz && x >= th;
  }
  __host__ __device__ __forceinline__ bool less(float x) const { return x < th; }
  __host__ __device__ __forceinline__ bool greater(float x) const { return x >= th + wsz; }
  __host__ __device__ void reset() {
    th = th + wsz;
    wsz = wsz_lim * reset_rate;
  }
};

// ---------------------------------------------------------------------------
// Per-vertex data: WA (read/write) and RA (read-only) arrays plus host
// mirrors (functor.cuh:12-66).
// ---------------------------------------------------------------------------
template <typename WA, typename RA>
struct vdata_t {
  WA zero;
  RA *dg_ra = nullptr;
  WA *dg_wa = nullptr;
  RA *h_ra = nullptr;
  WA *h_wa = nullptr;
  int64_t size = 0;
  WA *sb = nullptr;  // 2D-partition partial-contribution buffer
  int64_t sb_size = 0;
  window_t window;
  // captured level loops keep the window in device memory (the loop moves
  // it between levels); null: the by-value member above
  const window_t *dwin = nullptr;
  __host__ __device__ __forceinline__ const window_t &win() const {
#ifdef __CUDA_ARCH__
    if (dwin) return *dwin;
#endif
    return window;
  }

  void build(int64_t n) {
    size = n;
    if (!std::is_same<Empty, WA>::value) {
      GSW_CUDA(cudaMalloc((void **)&dg_wa, sizeof(WA) * (n + 1)));
      h_wa = (WA *)malloc(sizeof(WA) * (n + 1));
    }
    if (!std::is_same<Empty, RA>::value) {
      GSW_CUDA(cudaMalloc((void **)&dg_ra, sizeof(RA) * (n + 1)));
      h_ra = (RA *)malloc(sizeof(RA) * (n + 1));
    }
  }
  void destroy() {
    cudaFree(dg_wa);
    cudaFree(dg_ra);
    cudaFree(sb);
    free(h_wa);
    free(h_ra);
    dg_wa = nullptr;
    dg_ra = nullptr;
    sb = nullptr;
    h_wa = nullptr;
    h_ra = nullptr;
  }
  template <typename X>
  void init_wa(X init) {
    for (int64_t i = 0; i < size; ++i) h_wa[i] = init((int)i);
    GSW_CUDA(cudaMemcpyAsync(dg_wa, h_wa, sizeof(WA) * size, cudaMemcpyHostToDevice, gsw::stream()));
    GSW_CUDA(cudaStreamSynchronize(gsw::stream()));
  }
  template <typename X>
  void init_ra(X init) {
    for (int64_t i = 0; i < size; ++i) h_ra[i] = init((int)i);
    GSW_CUDA(cudaMemcpyAsync(dg_ra, h_ra, sizeof(RA) * size, cudaMemcpyHostToDevice, gsw::stream()));
    GSW_CUDA(cudaStreamSynchronize(gsw::stream()));
  }
  void set_zero(WA z) { zero = z; }
  void sync_wa() {
    GSW_CUDA(cudaMemcpyAsync(h_wa, dg_wa, sizeof(WA) * size, cudaMemcpyDeviceToHost, gsw::stream()));
    GSW_CUDA(cudaStreamSynchronize(gsw::stream()));
  }
  void sync_ra() {
    GSW_CUDA(cudaMemcpyAsync(h_ra, dg_ra, sizeof(RA) * size, cudaMemcpyDeviceToHost, gsw::stream()));
    GSW_CUDA(cudaStreamSynchronize(gsw::stream()));
  }
  __device__ __forceinline__ WA *fetch_wa(int v) const { return dg_wa + v; }
  __device__ __forceinline__ RA *fetch_ra(int v) const { return dg_ra + v; }
};

template <Centric C, typename WA, typename RA, typename E>
struct Functor {};

template <typename WA, typename RA, typename E>
struct Functor<EC, WA, RA, E> {
  typedef WA wa_t;
  typedef RA ra_t;
  typedef E e_t;
  using G = device_graph_t<COO, E>;
  vdata_t<WA, RA> data;
  __device__ __forceinline__ WA *wa_of(int v) const { return data.fetch_wa(v); }
  __device__ __forceinline__ RA *ra_of(int v) const { return data.fetch_ra(v); }
  __device__ Status filter(int, int, E *) { return Inactive; }
  __device__ void update(int, int, E *) {}
};

template <typename WA, typename RA, typename E>
struct Functor<VC, WA, RA, E> {
  typedef WA wa_t;
  typedef RA ra_t;
  typedef E e_t;
  using G = device_graph_t<CSR, E>;
  vdata_t<WA, RA> data;
  __device__ __forceinline__ WA *wa_of(int v) const { return data.fetch_wa(v); }
  __device__ __forceinline__ RA *ra_of(int v) const { return data.fetch_ra(v); }
  __device__ Status filter(int, G) { return Inactive; }
  __device__ WA emit(int v, E *, G) { return *data.fetch_wa(v); }
  __device__ bool cond(int, WA, G) { return false; }
  __device__ bool comp(WA *, WA, G) { return true; }
  __device__ bool compAtomic(WA *, WA, G) { return true; }
  __device__ bool exit(int, G) { return false; }
};

template <Centric C = VC, LB S = WM, Direction D = Push>
struct ExpandProxy {};

// ---------------------------------------------------------------------------
// Forced-variant override (the `-c Push-Queue-CM-Fused` flag of
// src/utils/cmdline.cuh:51-94): any subset of the four choices.
// ---------------------------------------------------------------------------
struct ins_t {
  Direction d = Push;
  ASFmt asf = Queue;
  LB lb = WM;
  Fusion fusion = Standalone;
  bool has_direction = false;
  bool has_asfmt = false;
  bool has_lb = false;
  bool has_fusion = false;
};

// ---------------------------------------------------------------------------
// config_t (src/abstraction/config.cuh:9-122)
// ---------------------------------------------------------------------------
struct config_t {
  Direction conf_dir = Push;
  Status conf_target = Active;
  CullMode conf_cm = Interleave;
  ASFmt conf_asfmt = Queue;
  LB conf_lb = WM;
  Centric conf_centric = VC;
  QueueMode conf_qmode = Normal;

  bool conf_fromall = false;
  bool conf_toall = false;
  bool conf_fixed = false;
  bool conf_inherit = false;
  bool conf_2d_partition = false;

  bool conf_first_round = true;
  bool conf_switch_to_fusion = false;
  bool conf_switch_to_standalone = false;
  bool conf_pruning = false;
  bool conf_once = false;
  bool conf_ignore_u_state = false;
  bool conf_fuse_inspect = false;
  bool conf_lite = false;
  bool conf_window = false;
  bool conf_compensation = false;
  bool conf_super_fusion = false;
  bool conf_fusion = false;
  int conf_idle = 0;
  int ctanum = CTANUM_EXPAND;
  int thdnum = THDNUM_EXPAND;

  // engine extensions
  bool conf_sorted_queue = true;   // bitmap->queue in vertex order
  bool conf_persistent = false;    // run fused levels in one grid-wide launch
  int conf_hub_path = -1;          // how CTA-wide hub sweeps read columns
                                   // (HUB_SCALAR / HUB_VECTOR / HUB_STAGED;
                                   // -1: by the graph's edge data)
  bool conf_count_edges = false;   // accounting pass: expands count edges
  ins_t force;                     // forced choices (empty = selector decides)

  void reset() {
    conf_first_round = true;
    conf_switch_to_fusion = false;
    conf_switch_to_standalone = false;
    conf_fuse_inspect = false;
    conf_idle = 0;
  }
  __host__ __device__ __forceinline__ bool ignore_u_state() const { return conf_ignore_u_state; }
  __host__ __device__ __forceinline__ Status want() const { return conf_target; }
  __host__ __device__ __forceinline__ bool pruning() const { return conf_pruning; }
  __host__ __device__ __forceinline__ bool fuse_inspect() const { return conf_fuse_inspect; }

  const char *lb_name() const {
    switch (conf_lb) {
      case TM: return "TM";
      case WM: return "WM";
      case CM: return "CM";
      case STRICT: return "STRICT";
      case TWOD: return "2D-partition";
      case ELB: return "ELB";
      case TWC: return "TWC";
    }
    return "Unknown";
  }
  void show_hints() const {
    printf("[%s|%s|%s|%s] ", conf_dir == Push ? "Push" : "Pull", conf_asfmt == Queue ? "Queue" : "Bitmap",
           lb_name(), conf_fuse_inspect ? "Fused" : "Standalone");
  }
};

// ---------------------------------------------------------------------------
// stat_t (src/abstraction/statistics.cuh:11-30): device counters reduced by
// the inspector plus per-level timing history.
//   [0] active vertices  [1] inactive vertices  [2] push workload
//   [3] pull workload    [4] max push degree    [5] max pull degree
// The last two keep the reference's definition (inspector.cuh:101-109): each
// block of the 256x512 inspection grid sums its threads' maxima, then the
// push figure takes the maximum over blocks and the pull figure the sum.
// ---------------------------------------------------------------------------
struct stat_t {
  unsigned long long *dg_runtime_info = nullptr;
  unsigned long long *h_runtime_info = nullptr;
  // Zero-copy report of a VC inspection (mapped pinned, 8 words): the
  // kernel's last CTA writes the six counters to [0..5], each word holding
  // the value in its low 40 bits and the launch's tag (1 .. 2^24-1) in the
  // top 24, and clears the device counters for the next launch; the host
  // polls the tags instead of copying and synchronising.
  unsigned long long *h_sig = nullptr, *d_sig = nullptr;
  unsigned long long sig_seq = 0;
  int size = 0;
  double last_time = 0, avg_time = 0;
  double last_filter_time = 0, last_expand_time = 0;
  double avg_filter_time = 0, avg_expand_time = 0;
  int level = 0;
  int64_t last_scanned = 0;  // edges the last expand touched (accounting)

  void build(int _size = gsw::STAT_SLOTS) {
    if (dg_runtime_info) return;
    size = _size;
    // the inspection's merge scratch follows the counters; only the
    // counters are cleared per level
    const size_t bytes = (size + gsw::STAT_SCRATCH) * sizeof(unsigned long long);
    GSW_CUDA(cudaMalloc((void **)&dg_runtime_info, bytes));
    GSW_CUDA(cudaMemsetAsync(dg_runtime_info, 0, bytes, gsw::stream()));
    GSW_CUDA(cudaMallocHost((void **)&h_runtime_info, size * sizeof(unsigned long long)));
    memset(h_runtime_info, 0, size * sizeof(unsigned long long));
    if (GSW_CUDA(cudaHostAlloc((void **)&h_sig, 8 * sizeof(unsigned long long), cudaHostAllocMapped)) == 0) {
      memset(h_sig, 0, 8 * sizeof(unsigned long long));
      if (GSW_CUDA(cudaHostGetDevicePointer((void **)&d_sig, h_sig, 0))) d_sig = nullptr;
    }
  }
  void destroy() {
    cudaFree(dg_runtime_info);
    cudaFreeHost(h_runtime_info);
    if (h_sig) cudaFreeHost(h_sig);
    dg_runtime_info = nullptr;
    h_runtime_info = nullptr;
    h_sig = d_sig = nullptr;
  }
  // tag for the next signalled inspection (0: no report block)
  unsigned long long arm() { return d_sig ? (++sig_seq % 0xffffffull) + 1 : 0; }
  // Waits for the report tagged `tag` and takes its counters.  Every 256
  // polls the stream is queried, so the wait ends when the stream runs dry;
  // false then (or on an error), and the caller reads the device block.
  bool await(unsigned long long tag) {
    volatile unsigned long long *h = h_sig;
    auto arrived = [&] {
      for (int i = 0; i < 6; ++i)
        if ((h[i] >> 40) != tag) return false;
      return true;
    };
    for (unsigned spin = 1;; ++spin) {
      if (arrived()) break;
      if ((spin & 255) == 0) {
        const cudaError_t q = cudaStreamQuery(gsw::stream());
        if (q != cudaErrorNotReady) {
          if (arrived()) break;
          if (q != cudaSuccess) GSW_CUDA(q);
          return false;
        }
      }
    }
    for (int i = 0; i < 6; ++i) h_runtime_info[i] = h[i] & ((1ull << 40) - 1);
    return true;
  }
  void reset() {}
  void collect(int num) {
    GSW_CUDA(cudaMemcpyAsync(h_runtime_info, dg_runtime_info, num * sizeof(unsigned long long),
                             cudaMemcpyDeviceToHost, gsw::stream()));
    GSW_CUDA(cudaStreamSynchronize(gsw::stream()));
  }
  void clean() {
    GSW_CUDA(cudaMemsetAsync(dg_runtime_info, 0, sizeof(unsigned long long) * size, gsw::stream()));
  }
  int64_t active_num() const { return (int64_t)h_runtime_info[0]; }
  int64_t unactive_num() const { return (int64_t)h_runtime_info[1]; }
  int64_t push_workload() const { return (int64_t)h_runtime_info[2]; }
  int64_t pull_workload() const { return (int64_t)h_runtime_info[3]; }
  int64_t max_deg_active() const { return (int64_t)h_runtime_info[4]; }
  int64_t max_deg_unactive() const { return (int64_t)h_runtime_info[5]; }
  void show_hints() const { printf("Iteration %d: (Filter %.3f ms) (Expand %.3f ms) ", level, last_filter_time, last_expand_time); }
};

// ---------------------------------------------------------------------------
// feature_t (src/abstraction/features.cuh:13-84): the 21-entry feature
// vector the selector reads, with the from-all / to-all folding of cross().
// ---------------------------------------------------------------------------
struct feature_t {
  Centric centric = VC;
  Computation pattern = Idem;
  int use_root = -1;
  double first_active = 1;  // vertices active at the first level when it starts from roots (multi-root runs)
  bool fromall = false;
  bool toall = false;

  int64_t nvertexs = 0;
  int64_t nedges = 0;
  double avg_deg = 0, std_deg = 0, max_deg = 0, range = 0, GI = 0, Her = 0;
  double avg_edata = 0;

  double active_vertex = 0, unactive_vertex = 0;
  double active_vertex_ratio = 0, unactive_vertex_ratio = 0;
  double push_workload = 0, pull_workload = 0;
  double push_workload_ratio = 0, pull_workload_ratio = 0;
  double cur_max_deg_active = 0, cur_avg_deg_active = 0;
  double cur_max_deg_unactive = 0, cur_avg_deg_unactive = 0;

  int level = 0;
  double last_time = 0, avg_time = 0;
  double last_filter_time = 0, last_expand_time = 0;
  double avg_filter_time = 0, avg_expand_time = 0;
  double growing_rate = 0;
  double first_workload = 0;

  double cap = 0;
  int thread_lim = 0, register_lim = 0, sm_num = 0;

  double fv[21] = {0};
  const char *record_path = nullptr;  // sink of record() (nullptr: none)
  int records = 0;                    // record() blocks written so far

  void reset() {}

  __host__ __device__ void flatten() {
    fv[0] = (double)nvertexs;
    fv[1] = (double)nedges;
    fv[2] = avg_deg;
    fv[3] = std_deg;
    fv[4] = range;
    fv[5] = GI;
    fv[6] = Her;
    fv[7] = active_vertex;
    fv[8] = unactive_vertex;
    fv[9] = push_workload;
    fv[10] = pull_workload;
    fv[11] = active_vertex_ratio;
    fv[12] = unactive_vertex_ratio;
    fv[13] = push_workload_ratio;
    fv[14] = pull_workload_ratio;
    fv[15] = cur_avg_deg_active;
    fv[16] = cur_avg_deg_unactive;
    fv[17] = cur_max_deg_active;
    fv[18] = cur_max_deg_unactive;
    fv[19] = DIV(last_filter_time, avg_filter_time);
    fv[20] = DIV(last_expand_time, avg_expand_time);
    cross();
  }

  // from-all patterns see every vertex as a source, to-all patterns every
  // vertex as a target: fold the other side's workload in (features.cuh:46-84)
  __host__ __device__ void cross() {
    const double av = active_vertex, uv = unactive_vertex;
    const double mixed = (av + uv == 0) ? 0
                                        : ((gsw::mul_unfused(cur_avg_deg_active, av) +
                                            gsw::mul_unfused(cur_avg_deg_unactive, uv)) /
                                           (av + uv));
    if (fromall) {
      fv[7] += unactive_vertex;
      fv[9] += pull_workload;
      fv[11] += unactive_vertex_ratio;
      fv[13] += pull_workload_ratio;
      fv[15] += mixed;
      fv[17] = MAX(cur_max_deg_unactive, cur_max_deg_active);
    }
    if (toall) {
      fv[8] += active_vertex;
      fv[10] += push_workload;
      fv[12] += active_vertex_ratio;
      fv[14] += push_workload_ratio;
      fv[16] += mixed;
      fv[18] = MAX(cur_max_deg_active, cur_max_deg_unactive);
    }
    active_vertex = fv[7];
    unactive_vertex = fv[8];
    push_workload = fv[9];
    pull_workload = fv[10];
    active_vertex_ratio = fv[11];
    unactive_vertex_ratio = fv[12];
    push_workload_ratio = fv[13];
    pull_workload_ratio = fv[14];
    cur_avg_deg_active = fv[15];
    cur_avg_deg_unactive = fv[16];
    cur_max_deg_active = fv[17];
    cur_max_deg_unactive = fv[18];
  }

  // The training record of src/abstraction/features.cuh:86-104 with the
  // writer of src/utils/json.cuh:34-48: the 21 flattened features and the
  // last filter / expand times as keys "0".."22", values in the stream's
  // default format (6 significant digits), one "{ ... }" block per call
  // appended to record_path; a feature object writes at most 100 blocks.
  void record() {
    flatten();
    if (!record_path) return;
    if (++records > 100) return;
    std::ostringstream o;
    o << "{\n";
    for (int i = 0; i < 23; ++i) {
      if (i > 0) o << ",\n";
      o << "\"" << i << "\": " << (i < 21 ? fv[i] : i == 21 ? last_filter_time : last_expand_time);
    }
    o << "\n}\n";
    FILE *f = fopen(record_path, "a");
    if (!f) return;
    fputs(o.str().c_str(), f);
    fclose(f);
  }

  void architecture_features(int device = -1) {
    if (device < 0) cudaGetDevice(&device);
    static thread_local int cached_dev = -1;
    static thread_local cudaDeviceProp prop;
    if (cached_dev != device) {
      if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return;
      cached_dev = device;
    }
    cap = prop.minor;
    while (cap > 1) cap /= 10;
    cap += prop.major;
    register_lim = prop.regsPerBlock / 512;
    thread_lim = prop.maxThreadsPerBlock;
    sm_num = prop.multiProcessorCount;
  }
};
