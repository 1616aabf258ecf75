// Expand kernels: every load-balance variant, push and pull, standalone and
// fused (the expand enqueues the next frontier itself).
//
// Per-edge semantics are the reference's (src/kernel_libs/expand_VC_TM.cuh,
// expand_VC_WM.cuh, expand_VC_CM.cuh, expand_VC_STRICT.cuh):
//   push/standalone  prune (mark visited) -> target must be Inactive unless
//                    to-all -> compAtomic(wa[u], emit(v))
//   push/fused       emit(v) -> cond(u) unless to-all -> compAtomic ->
//                    exactly-once enqueue through the visited bitmap
//   pull             for a candidate v, combine emit(u) of active (or all,
//                    when from-all) in-neighbours u with comp, stop at the
//                    first hit when the pattern allows pruning.
// The work decompositions are this engine's:
//   TM      one thread per frontier vertex;
//   WM      one warp per 32 frontier vertices, degrees scanned with warp
//           shuffles, 32 edges per round, owner found by a 5-step search;
//   CM      one CTA per 256 frontier vertices, block scan, 256 edges/round;
//   STRICT  exact edge balance: a (degree+1) scan over the frontier whose
//           epilogue also records, for every tile of STRICT_TILE slots, the
//           frontier index owning the tile's first slot (this replaces the
//           reference's moderngpu scan + sorted search); every CTA stages a
//           tile's owners in shared memory;
//   TWC     thread/warp/CTA tiers by degree inside one kernel: CTA-wide
//           sweeps for degree >= 256, warp sweeps for degree >= 32, and a
//           CTA-scan mapping for the rest (the intent recorded in
//           src/kernel_libs/expand_VC_TWC.cuh:11-63).
// Loops that enqueue run with warp-uniform trip counts so a warp can stage its
// appends in shared memory and reserve queue space once per STAGE_SLOTS.
#pragma once
#include "k_inspect_filter.cuh"

namespace gsw {

constexpr int EXPAND_THREADS = 256;
constexpr int STRICT_TILE = 1024;   // default slots per STRICT tile (4 per thread); the
                                    // autotuner may pick 512 or 2048 per variant
constexpr int STRICT_ITEMS = 1024;  // frontier entries per STRICT scan block

// ---- per-edge operations ---------------------------------------------------
template <typename G, typename F>
__device__ __forceinline__ void push_edge_std(active_set_t &as, const G &g, F &f, const config_t &conf, int v,
                                              int u, int64_t ei) {
  bool tp = true;
  if (conf.conf_pruning) tp = as.bitmap.mark_duplicate_lite(u);
  if (tp && !conf.conf_toall) tp = as.bitmap.is_inactive(u);
  if (tp) {
    auto vd = f.emit(v, g.fetch_edata(ei), g);
    f.compAtomic(f.wa_of(u), vd, g);
  }
}

template <typename G, typename F>
__device__ __forceinline__ bool push_edge_fused(active_set_t &as, const G &g, F &f, const config_t &conf, int v,
                                                int u, int64_t ei) {
  auto vd = f.emit(v, g.fetch_edata(ei), g);
  bool tp = true;
  if (!conf.conf_toall) tp = f.cond(u, vd, g);
  if (tp) tp = f.compAtomic(f.wa_of(u), vd, g);
  if (tp) tp = as.bitmap.mark_duplicate_atomic(u);
  return tp;
}

// Fused levels append the vertices they activate to the output queue.  A warp
// stages its appends in shared memory and reserves queue space once per
// STAGE_SLOTS entries (and once when it is done), not once per 32-edge round:
// on a large fused level every warp of the grid would otherwise hit the one
// queue counter each round, and those same-address atomics serialise at the
// L2 (4M-vertex SSSP levels ran at 9 G edges/s instead of 30+).  The order of
// a level's queue is unspecified either way.
constexpr int STAGE_SLOTS = 128;

struct warp_stage_t {
  int *buf;       // this warp's STAGE_SLOTS slots in shared memory
  int n = 0;      // staged entries, warp-uniform
  int *out;       // nullptr: appends are dropped (Cached replay)
  int *cnt;
  int64_t cap;
  unsigned *err;

  __device__ __forceinline__ warp_stage_t(int *smem, int *o, int *c, int64_t cp, unsigned *e)
      : buf(smem), out(o), cnt(c), cap(cp), err(e) {}
  __device__ __forceinline__ warp_stage_t(int *smem, const active_set_t &as)
      : buf(smem),
        out(as.queue.mode == Cached && as.queue.traceback ? nullptr : as.queue.output_base()),
        cnt(as.queue.output_size()),
        cap(as.queue.output_cap()),
        err(as.queue.dg_err) {}

  // every lane of the warp calls it
  __device__ __forceinline__ void flush() {
    if (n == 0) return;
    __syncwarp();
    int base = 0;
    if (lane_id() == 0) {
      base = atomicAdd(cnt, n);
      if ((int64_t)base + n > cap) {
        atomicOr(err, DEV_ERR_QUEUE_OVERFLOW);
        base = -1;
      }
    }
    base = __shfl_sync(FULL, base, 0);
    if (base >= 0)
      for (int i = lane_id(); i < n; i += 32) out[base + i] = buf[i];
    n = 0;
    __syncwarp();
  }
  // every lane of the warp calls it; lanes with tp append u
  __device__ __forceinline__ void push(bool tp, int u) {
    const unsigned m = __ballot_sync(FULL, tp && out != nullptr);
    if (!m) return;
    const int c = __popc(m);
    if (n + c > STAGE_SLOTS) flush();
    if (tp) buf[n + __popc(m & ((1u << lane_id()) - 1u))] = u;
    n += c;
  }
};

template <typename G>
__device__ __forceinline__ void vertex_range(const G &g, bool pull, int v, int64_t &st, int &deg) {
  if (v < 0) {
    st = 0;
    deg = 0;
    return;
  }
  const int64_t *off = pull ? g.dgr_row_off : g.dg_row_off;
  st = __ldg(off + v);
  deg = (int)(__ldg(off + v + 1) - st);
}

// accounting pass only: one atomic per thread at kernel exit
__device__ __forceinline__ void account(const active_set_t &as, const config_t &conf, unsigned long long c) {
  if (conf.conf_count_edges && c) atomicAdd(&as.dg_cnt->scanned, c);
}

// Where a push body reads its work list.  Per-launch kernels read the active
// set (queue or bitmap, read-only path).  Levels inside a persistent launch
// read the queue array the previous level wrote, with plain loads (the
// read-only path may hold lines of an array written during the same launch),
// and apply the deferred filter update of each vertex they fetch (what the
// compensation launch does between per-launch fused levels).
struct as_src_t {
  const active_set_t *as;
  Status want;
  __device__ __forceinline__ int operator()(int64_t i) const { return as->fetch(i, want); }
  template <typename G, typename F>
  __device__ __forceinline__ void visit(int, const G &, F &) const {}
};
struct level_src_t {
  const int *q;
  bool compensate;
  __device__ __forceinline__ int operator()(int64_t i) const { return q[i]; }
  template <typename G, typename F>
  __device__ __forceinline__ void visit(int v, const G &g, F &f) const {
    if (compensate && v >= 0) f.filter(v, g);
  }
};

#define GSW_HALT_IF_EMPTY(n)                                     \
  if ((n) == 0) {                                                \
    if (blockIdx.x == 0 && threadIdx.x == 0) as.halt_device();   \
    return;                                                      \
  }

// ===========================================================================
// TM
// ===========================================================================
// fused TM level over src[0..n): warp-uniform trip counts, so the warp
// stages its appends together
template <typename G, typename F, typename Src>
__device__ __forceinline__ void push_tm_fused_body(active_set_t &as, const G &g, F &f, const config_t &conf,
                                                   const Src &src, int64_t n, warp_stage_t &stage) {
  const int64_t STRIDE = (int64_t)blockDim.x * gridDim.x;
  unsigned long long cnt = 0;
  for (int64_t w0 = (threadIdx.x & ~31u) + (int64_t)blockIdx.x * blockDim.x; w0 < n; w0 += STRIDE) {
    const int64_t idx = w0 + lane_id();
    const int v = idx < n ? src(idx) : -1;
    src.visit(v, g, f);
    int64_t st;
    int deg;
    vertex_range(g, false, v, st, deg);
    cnt += deg;
    const int rounds = (int)__reduce_max_sync(FULL, (unsigned)deg);
    for (int k = 0; k < rounds; ++k) {
      bool tp = false;
      int u = -1;
      if (k < deg) {
        u = __ldg(g.dg_adj_list + st + k);
        tp = push_edge_fused(as, g, f, conf, v, u, st + k);
      }
      stage.push(tp, u);
    }
  }
  account(as, conf, cnt);
}

// BT: threads per CTA (a tuned shape: 128, 256 or 512)
template <bool FUSED, int BT, typename G, typename F>
__global__ void __launch_bounds__(BT) k_push_tm(active_set_t as, G g, F f, config_t conf) {
  const int64_t n = as.get_size();
  GSW_HALT_IF_EMPTY(n);
  const Status want = conf.want();
  const int64_t STRIDE = (int64_t)blockDim.x * gridDim.x;
  unsigned long long cnt = 0;
  if constexpr (FUSED) {
    __shared__ int s_stage[BT / 32][STAGE_SLOTS];
    warp_stage_t stage(s_stage[warp_id()], as);
    push_tm_fused_body(as, g, f, conf, as_src_t{&as, want}, n, stage);
    stage.flush();
  } else {
    for (int64_t idx = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; idx < n; idx += STRIDE) {
      const int v = as.fetch(idx, want);
      if (v < 0) continue;
      int64_t st;
      int deg;
      vertex_range(g, false, v, st, deg);
      cnt += deg;
      for (int k = 0; k < deg; ++k) push_edge_std(as, g, f, conf, v, __ldg(g.dg_adj_list + st + k), st + k);
    }
  }
  account(as, conf, cnt);
}

// Thread per candidate, K candidates per thread (2 by default; the autotuner
// may pick 1 or 4): the dependent chain of a candidate (status bit -> offsets
// -> first in-neighbour -> its frontier bit) is issued for all K before any
// is resolved.  Most candidates of a large pull level stop at the first
// neighbour; the rest walk their lists one edge at a time, and a warp waits
// for its longest walk, so more candidates per thread cost more in
// divergence than they gain in overlap (RMAT s24 pull levels: 105 us at 1,
// 93 at 2, 103 at 4, 135 at 8).  Measured and not kept (section 3 of the
// design notes has the numbers): fetching four neighbours per walk step, a
// warp-cooperative walk of the unresolved candidates, a first-in-neighbour
// side array (less DRAM traffic, no faster), skipping vertices without
// in-edges by a bitmap, and capping thread walks at 8 edges with 8-lane
// groups finishing the rest (40 registers, 75% occupancy, slower).  BT:
// threads per CTA (a tuned shape together with K: 128, 256 or 512).
template <int K, int BT, typename G, typename F>
__global__ void __launch_bounds__(BT) k_pull_tm(active_set_t as, G g, F f, config_t conf) {
  using WA = typename F::wa_t;
  const int64_t n = as.get_size();
  GSW_HALT_IF_EMPTY(n);
  const Status want = conf.want();
  const int64_t STRIDE = (int64_t)blockDim.x * gridDim.x;
  unsigned long long cnt = 0;
  for (int64_t base = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; base < n; base += K * STRIDE) {
    int v[K], deg[K], u0[K];
    int64_t st[K];
    bool a0[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int64_t idx = base + k * STRIDE;
      v[k] = idx < n ? as.fetch(idx, want) : -1;
    }
#pragma unroll
    for (int k = 0; k < K; ++k) vertex_range(g, true, v[k], st[k], deg[k]);
#pragma unroll
    for (int k = 0; k < K; ++k) u0[k] = deg[k] > 0 ? __ldg(g.dgr_adj_list + st[k]) : 0;
#pragma unroll
    for (int k = 0; k < K; ++k) a0[k] = deg[k] > 0 && (conf.conf_fromall || as.bitmap.is_active(u0[k]));
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (v[k] < 0 || deg[k] == 0) continue;
      WA acc;
      bool have = false;
      int e = 1;
      if (a0[k]) {
        acc = f.emit(u0[k], g.fetch_edata_r(st[k]), g);
        have = true;
      }
      if (!(have && conf.conf_pruning)) {
        for (; e < deg[k]; ++e) {
          const int u = __ldg(g.dgr_adj_list + st[k] + e);
          if (conf.conf_fromall || as.bitmap.is_active(u)) {
            WA x = f.emit(u, g.fetch_edata_r(st[k] + e), g);
            if (have)
              f.comp(&acc, x, g);
            else {
              acc = x;
              have = true;
            }
            if (conf.conf_pruning) {
              ++e;
              break;
            }
          }
        }
      }
      cnt += e;
      if (have) f.comp(f.wa_of(v[k]), acc, g);
    }
  }
  account(as, conf, cnt);
}

// ===========================================================================
// Hub lists of per-launch pushes
// ===========================================================================
// A push whose grid is sized by frontier vertices runs a level whose frontier
// is a few hubs on a few CTAs, and a tile (warp or CTA) that holds a hub
// sweeps all of its columns alone.  Per-launch tiered (TWC), warp-mapped (WM)
// and CTA-mapped (CM) pushes therefore cut each vertex of at least their hub
// degree into pieces of at most TWC_HUB_PIECE columns, append them to a hub
// list, and a second kernel (k_push_twc_hubs) sweeps one piece per CTA over
// the resident grid.  Persistent launches keep the in-tile sweep (the list
// would need one more grid barrier per level), and so does a hub that finds
// the list full (a fused queue may hold a vertex more than once).  The hub
// kernel's last CTA to read the count sets it back to 0 for the next level,
// so no memset node sits in captured loops.
constexpr int TWC_HUB_PIECE = 8192;
constexpr int WM_HUB_MIN = 1024;  // WM: a warp would take 32+ rounds alone
constexpr int CM_HUB_MIN = 4096;  // CM: a CTA would take 16+ rounds alone
struct hub_piece_t {
  int v;
  int len;
  int64_t st;
};
struct hub_list_t {
  hub_piece_t *piece = nullptr;  // null: sweep hubs in their tile
  int *count = nullptr;
  unsigned *done = nullptr;
  int64_t cap = 0;
};
// Lists v's columns as hub pieces when a list is given and deg >= min_deg;
// true when they were listed (the caller then drops them).  A hub that does
// not fit whole writes empty pieces into its slots below the cap and stays
// with its tile.
__device__ __forceinline__ bool defer_hub(active_set_t &as, const config_t &conf, const hub_list_t &hubs, int v,
                                          int64_t st, int deg, int min_deg) {
  if (!hubs.piece || deg < min_deg) return false;
  const int np = (deg + TWC_HUB_PIECE - 1) / TWC_HUB_PIECE;
  const int at = atomicAdd(hubs.count, np);
  const bool fits = (int64_t)at + np <= hubs.cap;
  for (int k = 0; k < np && (int64_t)at + k < hubs.cap; ++k)
    hubs.piece[at + k] = fits ? hub_piece_t{v, MIN(TWC_HUB_PIECE, deg - k * TWC_HUB_PIECE),
                                            st + (int64_t)k * TWC_HUB_PIECE}
                              : hub_piece_t{v, 0, 0};
  if (fits) account(as, conf, (unsigned long long)deg);
  return fits;
}

// ===========================================================================
// WM: warp per 32 frontier vertices
// ===========================================================================
template <bool FUSED, typename G, typename F, typename Src>
__device__ __forceinline__ void push_wm_body(active_set_t &as, const G &g, F &f, const config_t &conf, const Src &src,
                                             int64_t n, warp_stage_t &stage, hub_list_t hubs = hub_list_t()) {
  constexpr int W = EXPAND_THREADS / 32;
  __shared__ int s_scan[W][32];
  __shared__ int s_v[W][32];
  __shared__ int64_t s_st[W][32];
  const int lane = lane_id(), w = warp_id();
  const int64_t nwarps = (int64_t)gridDim.x * W;
  for (int64_t tile = (int64_t)blockIdx.x * W + w; tile * 32 < n; tile += nwarps) {
    const int64_t idx = tile * 32 + lane;
    const int v = idx < n ? src(idx) : -1;
    src.visit(v, g, f);
    int64_t st;
    int deg;
    vertex_range(g, false, v, st, deg);
    if (defer_hub(as, conf, hubs, v, st, deg, WM_HUB_MIN)) deg = 0;
    const int incl = warp_inclusive_sum(deg);
    const int total = __shfl_sync(FULL, incl, 31);
    if (lane == 0) account(as, conf, (unsigned long long)total);
    s_scan[w][lane] = incl - deg;
    s_v[w][lane] = v;
    s_st[w][lane] = st;
    __syncwarp();
    for (int base = 0; base < total; base += 32) {
      const int i = base + lane;
      bool tp = false;
      int u = -1;
      if (i < total) {
        const int id = upper_bound(s_scan[w], 32, i) - 1;
        const int64_t ei = s_st[w][id] + (i - s_scan[w][id]);
        u = __ldg(g.dg_adj_list + ei);
        if (FUSED)
          tp = push_edge_fused(as, g, f, conf, s_v[w][id], u, ei);
        else
          push_edge_std(as, g, f, conf, s_v[w][id], u, ei);
      }
      if (FUSED) stage.push(tp, u);
    }
    __syncwarp();
  }
}

template <bool FUSED, typename G, typename F>
__global__ void __launch_bounds__(EXPAND_THREADS) k_push_wm(active_set_t as, G g, F f, config_t conf,
                                                            hub_list_t hubs) {
  __shared__ int s_stage[FUSED ? EXPAND_THREADS / 32 : 1][FUSED ? STAGE_SLOTS : 1];
  const int64_t n = as.get_size();
  GSW_HALT_IF_EMPTY(n);
  warp_stage_t stage(s_stage[FUSED ? warp_id() : 0], as);
  push_wm_body<FUSED>(as, g, f, conf, as_src_t{&as, conf.want()}, n, stage, hubs);
  if (FUSED) stage.flush();
}

template <typename G, typename F>
__global__ void __launch_bounds__(EXPAND_THREADS) k_pull_wm(active_set_t as, G g, F f, config_t conf) {
  using WA = typename F::wa_t;
  constexpr int W = EXPAND_THREADS / 32;
  __shared__ int s_scan[W][33];
  __shared__ int s_v[W][32];
  __shared__ int64_t s_st[W][32];
  const int64_t n = as.get_size();
  GSW_HALT_IF_EMPTY(n);
  const Status want = conf.want();
  const int lane = lane_id(), w = warp_id();
  const int64_t nwarps = (int64_t)gridDim.x * W;
  for (int64_t tile = (int64_t)blockIdx.x * W + w; tile * 32 < n; tile += nwarps) {
    const int64_t idx = tile * 32 + lane;
    const int v = idx < n ? as.fetch(idx, want) : -1;
    int64_t st;
    int deg;
    vertex_range(g, true, v, st, deg);
    const int incl = warp_inclusive_sum(deg);
    const int total = __shfl_sync(FULL, incl, 31);
    if (lane == 0) account(as, conf, (unsigned long long)total);
    s_scan[w][lane] = incl - deg;
    if (lane == 31) s_scan[w][32] = total;
    s_v[w][lane] = v;
    s_st[w][lane] = st;
    __syncwarp();
    for (int base = 0; base < total; base += 32) {
      const int i = base + lane;
      int id = 31;
      bool vote = false;
      WA val;
      memset(&val, 0, sizeof(WA));
      if (i < total) {
        id = upper_bound(s_scan[w], 32, i) - 1;
        const int64_t ei = s_st[w][id] + (i - s_scan[w][id]);
        const int u = __ldg(g.dgr_adj_list + ei);
        if (conf.conf_fromall || as.bitmap.is_active(u)) {
          vote = true;
          val = f.emit(u, g.fetch_edata_r(ei), g);
        }
      } else {
        id = 32 + lane;  // past-the-end lanes form their own segments
      }
      // segmented reduction toward the first lane of each owner's run
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int oid = __shfl_down_sync(FULL, id, d);
        const bool ovote = __shfl_down_sync(FULL, vote, d);
        const WA oval = shfl_down_any(val, d);
        if (lane + d < 32 && oid == id && ovote) {
          if (vote)
            f.comp(&val, oval, g);
          else
            val = oval;
          vote = true;
        }
      }
      const int pid = __shfl_up_sync(FULL, id, 1);
      const bool head = (lane == 0) || (pid != id);
      if (i < total && head && vote) f.comp(f.wa_of(s_v[w][id]), val, g);
    }
    __syncwarp();
  }
}

// ===========================================================================
// CM: CTA per 256 frontier vertices
// ===========================================================================
template <bool FUSED, typename G, typename F, typename Src>
__device__ __forceinline__ void push_cm_body(active_set_t &as, const G &g, F &f, const config_t &conf, const Src &src,
                                             int64_t n, warp_stage_t &stage, hub_list_t hubs = hub_list_t()) {
  constexpr int B = EXPAND_THREADS;
  __shared__ int s_scan[B];
  __shared__ int s_v[B];
  __shared__ int64_t s_st[B];
  __shared__ int s_tmp[33];
  for (int64_t tile = blockIdx.x; tile * B < n; tile += gridDim.x) {
    const int64_t idx = tile * B + threadIdx.x;
    const int v = idx < n ? src(idx) : -1;
    src.visit(v, g, f);
    int64_t st;
    int deg;
    vertex_range(g, false, v, st, deg);
    if (defer_hub(as, conf, hubs, v, st, deg, CM_HUB_MIN)) deg = 0;
    int total;
    const int ex = block_exclusive_scan(deg, s_tmp, &total);
    if (threadIdx.x == 0) account(as, conf, (unsigned long long)total);
    s_scan[threadIdx.x] = ex;
    s_v[threadIdx.x] = v;
    s_st[threadIdx.x] = st;
    __syncthreads();
    for (int base = 0; base < total; base += B) {
      const int i = base + threadIdx.x;
      bool tp = false;
      int u = -1;
      if (i < total) {
        const int id = upper_bound(s_scan, B, i) - 1;
        const int64_t ei = s_st[id] + (i - s_scan[id]);
        u = __ldg(g.dg_adj_list + ei);
        if (FUSED)
          tp = push_edge_fused(as, g, f, conf, s_v[id], u, ei);
        else
          push_edge_std(as, g, f, conf, s_v[id], u, ei);
      }
      if (FUSED) stage.push(tp, u);
    }
    __syncthreads();
  }
}

template <bool FUSED, typename G, typename F>
__global__ void __launch_bounds__(EXPAND_THREADS) k_push_cm(active_set_t as, G g, F f, config_t conf,
                                                            hub_list_t hubs) {
  __shared__ int s_stage[FUSED ? EXPAND_THREADS / 32 : 1][FUSED ? STAGE_SLOTS : 1];
  const int64_t n = as.get_size();
  GSW_HALT_IF_EMPTY(n);
  warp_stage_t stage(s_stage[FUSED ? warp_id() : 0], as);
  push_cm_body<FUSED>(as, g, f, conf, as_src_t{&as, conf.want()}, n, stage, hubs);
  if (FUSED) stage.flush();
}

template <typename G, typename F>
__global__ void __launch_bounds__(EXPAND_THREADS) k_pull_cm(active_set_t as, G g, F f, config_t conf) {
  constexpr int B = EXPAND_THREADS;
  __shared__ int s_scan[B];
  __shared__ int s_v[B];
  __shared__ int64_t s_st[B];
  __shared__ int s_tmp[33];
  const int64_t n = as.get_size();
  GSW_HALT_IF_EMPTY(n);
  const Status want = conf.want();
  for (int64_t tile = blockIdx.x; tile * B < n; tile += gridDim.x) {
    const int64_t idx = tile * B + threadIdx.x;
    const int v = idx < n ? as.fetch(idx, want) : -1;
    int64_t st;
    int deg;
    vertex_range(g, true, v, st, deg);
    int total;
    const int ex = block_exclusive_scan(deg, s_tmp, &total);
    if (threadIdx.x == 0) account(as, conf, (unsigned long long)total);
    s_scan[threadIdx.x] = ex;
    s_v[threadIdx.x] = v;
    s_st[threadIdx.x] = st;
    __syncthreads();
    for (int base = 0; base < total; base += B) {
      const int i = base + threadIdx.x;
      if (i < total) {
        const int id = upper_bound(s_scan, B, i) - 1;
        const int64_t ei = s_st[id] + (i - s_scan[id]);
        const int u = __ldg(g.dgr_adj_list + ei);
        if (conf.conf_fromall || as.bitmap.is_active(u)) {
          auto vd = f.emit(u, g.fetch_edata_r(ei), g);
          f.compAtomic(f.wa_of(s_v[id]), vd, g);
        }
      }
    }
    __syncthreads();
  }
}

// ===========================================================================
// STRICT: exact edge balance
// ===========================================================================
template <bool PULL, typename G>
__device__ __forceinline__ int64_t strict_slots_of(const G &g, int v) {
  if (v < 0) return 1;
  const int64_t *off = PULL ? g.dgr_row_off : g.dg_row_off;
  return __ldg(off + v + 1) - __ldg(off + v) + 1;
}
template <bool PULL, typename G>
__device__ __forceinline__ int64_t strict_slots(const active_set_t &as, const G &g, int64_t idx, Status want) {
  return strict_slots_of<PULL>(g, as.fetch(idx, want));
}

// Epilogue of the STRICT scan for 4 consecutive frontier entries base..base+3
// (d[k] slots each, the first starting at slot `off`): eoff[idx] gets the
// entry's first slot, tile_lo[t] the entry owning slot t*STRICT_TILE.  Every
// lane of the warp calls it.
template <int T = STRICT_TILE>
__device__ __forceinline__ void strict_scan_epilogue(const active_set_t &as, int64_t base, int64_t n,
                                                     const int64_t (&d)[4], int64_t off, int64_t *eoff, int *tile_lo,
                                                     int64_t tile_cap) {
  auto own = [&](int64_t t, int item) {
    if (t < tile_cap)
      tile_lo[t] = item;
    else
      as.raise(DEV_ERR_SCRATCH_OVERFLOW);
  };
  const int lane = lane_id();
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int64_t idx = base + k;
    const bool valid = idx < n;
    if (valid) eoff[idx] = off;
    // tiles whose first slot falls in [off, off + d): ta <= t < tb
    const int64_t ta = (off + T - 1) / T;
    const int64_t tb = valid ? (off + d[k] + T - 1) / T : ta;
    // a hub owns many tiles, and a sorted frontier puts the hubs side by
    // side: long runs are written by the whole warp, 32 tiles a step
    const bool many = tb - ta > 2;
    if (!many)
      for (int64_t t = ta; t < tb; ++t) own(t, (int)idx);
    for (unsigned pend = __ballot_sync(FULL, many); pend; pend &= pend - 1) {
      const int src = __ffs(pend) - 1;
      const int64_t a = __shfl_sync(FULL, ta, src), b = __shfl_sync(FULL, tb, src);
      const int item = __shfl_sync(FULL, (int)idx, src);
      for (int64_t t = a + lane; t < b; t += 32) own(t, item);
    }
    off += d[k];
  }
}

template <bool PULL, typename G>
__global__ void __launch_bounds__(256) k_strict_count(active_set_t as, G g, Status want, int64_t *bsum) {
  __shared__ int64_t s_red[32];
  const int64_t n = as.get_size();
  // scan blocks blk = blockIdx.x, + gridDim.x, ... of the frontier's n / STRICT_ITEMS + 1
  // (a launch of that many CTAs takes one each; a captured body, which cannot
  // know n, launches a fixed grid)
  // (every CTA of the launch writes its first sum, zero past the frontier, so
  // a host-sized scan of the sums never reads a stale one)
  const int64_t nb = MAX(n / STRICT_ITEMS + 1, (int64_t)gridDim.x);
  for (int64_t blk = blockIdx.x; blk < nb; blk += gridDim.x) {
    const int64_t b0 = blk * STRICT_ITEMS;
    int64_t s = 0;
    for (int k = threadIdx.x; k < STRICT_ITEMS; k += blockDim.x) {
      const int64_t idx = b0 + k;
      if (idx < n) s += strict_slots<PULL>(as, g, idx, want);
    }
    s = block_reduce(s, s_red);
    if (threadIdx.x == 0) bsum[blk] = s;
  }
}

// eoff[idx] = exclusive scan of (degree+1); tile_lo[t] = frontier index that
// owns slot t*STRICT_TILE.  Each thread scans 4 consecutive entries.
template <bool PULL, int T, typename G>
__device__ __forceinline__ void strict_scan_block(active_set_t &as, const G &g, Status want, const int64_t *bsum,
                                                  int64_t nblocks, int *tile_lo, int64_t tile_cap, int64_t blk,
                                                  int64_t n, int64_t *s);
// the block sums of a frontier whose size only the device knows
__global__ void __launch_bounds__(1024) k_strict_bsum_scan(active_set_t as, int64_t *bsum) {
  scan_single_block_body(bsum, as.get_size() / STRICT_ITEMS + 1);
}
template <bool PULL, int T, typename G>
__global__ void __launch_bounds__(256) k_strict_scan(active_set_t as, G g, Status want, const int64_t *bsum,
                                                     int64_t nblocks, int *tile_lo, int64_t tile_cap) {
  __shared__ int64_t s[33];
  const int64_t n = as.get_size();
  // scan blocks as in k_strict_count; nblocks < 0: the frontier's own count
  const int64_t nb = bsum ? (nblocks >= 0 ? nblocks : n / STRICT_ITEMS + 1) : 1;
  for (int64_t blk = blockIdx.x; blk < nb; blk += gridDim.x) {
    strict_scan_block<PULL, T>(as, g, want, bsum, nb, tile_lo, tile_cap, blk, n, s);
    __syncthreads();  // s is reused by the next block
  }
}
template <bool PULL, int T, typename G>
__device__ __forceinline__ void strict_scan_block(active_set_t &as, const G &g, Status want, const int64_t *bsum,
                                                  int64_t nblocks, int *tile_lo, int64_t tile_cap, int64_t blk,
                                                  int64_t n, int64_t *s) {
  const int64_t base = blk * STRICT_ITEMS + threadIdx.x * 4;
  int64_t d[4], loc = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    d[k] = (base + k < n) ? strict_slots<PULL>(as, g, base + k, want) : 0;
    loc += d[k];
  }
  int64_t incl = warp_inclusive_sum(loc);
  __syncthreads();
  if (lane_id() == 31) s[warp_id()] = incl;
  __syncthreads();
  if (warp_id() == 0) {
    int64_t y = lane_id() < (int)(blockDim.x >> 5) ? s[lane_id()] : 0;
    int64_t yi = warp_inclusive_sum(y);
    if (lane_id() < (int)(blockDim.x >> 5)) s[lane_id()] = yi - y;
    if (lane_id() == 31) s[32] = yi;  // the block's total
  }
  __syncthreads();
  // bsum == nullptr: the whole frontier is this one block (no block sums)
  const int64_t off = (bsum ? bsum[blk] : 0) + s[warp_id()] + incl - loc;
  int64_t *eoff = as.workset.dg_eoff;
  strict_scan_epilogue<T>(as, base, n, d, off, eoff, tile_lo, tile_cap);
  if (blk == 0 && threadIdx.x == 0) {
    const int64_t total = bsum ? bsum[nblocks] : s[32];
    eoff[n] = total;
    as.dg_cnt->total_edges = (unsigned long long)total;
  }
}

// STRICT push over the tiles of a scanned frontier src[0..n) (eoff: the
// (degree+1) scan, tile_lo: tile owners)
template <bool FUSED, int T, typename G, typename F, typename Src>
__device__ __forceinline__ void push_strict_body(active_set_t &as, const G &g, F &f, const config_t &conf,
                                                 const Src &src, int64_t n, const int64_t *eoff, const int *tile_lo,
                                                 warp_stage_t &stage) {
  __shared__ int s_v[T + 2];
  __shared__ int64_t s_sc[T + 2];
  __shared__ int64_t s_st[T + 2];
  const int64_t total = eoff[n];
  const int64_t ntiles = (total + T - 1) / T;
  if (blockIdx.x == 0 && threadIdx.x == 0) account(as, conf, (unsigned long long)(total - n));
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t lo = tile_lo[t];
    const int64_t hi = (t + 1 < ntiles) ? tile_lo[t + 1] : n - 1;
    const int cnt = (int)(hi - lo + 1);
    for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
      const int v = src(lo + j);
      s_v[j] = v;
      s_sc[j] = eoff[lo + j];
      s_st[j] = v >= 0 ? __ldg(g.dg_row_off + v) : 0;
    }
    if (threadIdx.x == 0) s_sc[cnt] = eoff[hi + 1];
    __syncthreads();
    const int64_t t0 = t * T;
    const int64_t t1 = MIN(total, t0 + T);
#pragma unroll
    for (int k = 0; k < T / EXPAND_THREADS; ++k) {
      const int64_t s = t0 + k * EXPAND_THREADS + threadIdx.x;
      bool tp = false;
      int u = -1;
      if (s < t1) {
        const int j = upper_bound(s_sc, cnt, s) - 1;
        const int64_t local = s - s_sc[j];
        if (local < s_sc[j + 1] - s_sc[j] - 1) {
          const int64_t ei = s_st[j] + local;
          u = __ldg(g.dg_adj_list + ei);
          if (FUSED)
            tp = push_edge_fused(as, g, f, conf, s_v[j], u, ei);
          else
            push_edge_std(as, g, f, conf, s_v[j], u, ei);
        }
      }
      if (FUSED) stage.push(tp, u);
    }
    __syncthreads();
  }
}

template <bool FUSED, int T, typename G, typename F>
__global__ void __launch_bounds__(EXPAND_THREADS) k_push_strict(active_set_t as, G g, F f, config_t conf,
                                                                const int *tile_lo) {
  __shared__ int s_stage[FUSED ? EXPAND_THREADS / 32 : 1][FUSED ? STAGE_SLOTS : 1];
  const int64_t n = as.get_size();
  GSW_HALT_IF_EMPTY(n);
  warp_stage_t stage(s_stage[FUSED ? warp_id() : 0], as);
  push_strict_body<FUSED, T>(as, g, f, conf, as_src_t{&as, conf.want()}, n, as.workset.dg_eoff, tile_lo, stage);
  if (FUSED) stage.flush();
}

// Pull: each thread walks 4 consecutive slots and folds runs of the same
// candidate before one compAtomic (the "stride mode" of expand_VC_STRICT.cuh:
// 453-510).
// Edge-balanced pull.  A tile's slots are read warp-contiguously (slot
// t*T + k*B + lane + 32*warp at pass k, so the in-edge loads coalesce), the
// messages of each warp pass are combined per destination by a segmented
// shuffle scan, and only the last lane of each run writes: with a plain
// comp() when the run holds every in-edge of its vertex, with compAtomic()
// when the vertex's edges continue in another pass or tile.  A hub therefore
// costs one atomic per 32 edges instead of one per thread.
template <int T, typename G, typename F>
__global__ void __launch_bounds__(EXPAND_THREADS) k_pull_strict(active_set_t as, G g, F f, config_t conf,
                                                                const int *tile_lo) {
  using WA = typename F::wa_t;
  constexpr int B = EXPAND_THREADS;
  constexpr int PER = T / B;
  __shared__ int s_v[T + 2];
  __shared__ int64_t s_sc[T + 2];
  __shared__ int64_t s_st[T + 2];
  const int64_t n = as.get_size();
  GSW_HALT_IF_EMPTY(n);
  const Status want = conf.want();
  const int64_t *eoff = as.workset.dg_eoff;
  const int64_t total = eoff[n];
  const int64_t ntiles = (total + T - 1) / T;
  const int lane = lane_id();
  if (blockIdx.x == 0 && threadIdx.x == 0) account(as, conf, (unsigned long long)(total - n));
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t lo = tile_lo[t];
    const int64_t hi = (t + 1 < ntiles) ? tile_lo[t + 1] : n - 1;
    const int cnt = (int)(hi - lo + 1);
    for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
      const int v = as.fetch(lo + j, want);
      s_v[j] = v;
      s_sc[j] = eoff[lo + j];
      s_st[j] = v >= 0 ? __ldg(g.dgr_row_off + v) : 0;
    }
    if (threadIdx.x == 0) s_sc[cnt] = eoff[hi + 1];
    __syncthreads();
    const int64_t t1 = MIN(total, t * T + T);
    for (int k = 0; k < PER; ++k) {
      const int64_t wbase = t * T + (int64_t)k * B + (threadIdx.x & ~31);
      if (wbase >= t1) break;  // warp-uniform
      const int64_t s = wbase + lane;
      int j = -1;
      bool have = false;
      WA x = f.data.zero;
      if (s < t1) {
        j = upper_bound(s_sc, cnt, s) - 1;
        const int64_t local = s - s_sc[j];
        if (local < s_sc[j + 1] - s_sc[j] - 1) {
          const int64_t ei = s_st[j] + local;
          const int u = __ldg(g.dgr_adj_list + ei);
          if (conf.conf_fromall || as.bitmap.is_active(u)) {
            x = f.emit(u, g.fetch_edata_r(ei), g);
            have = true;
          }
        }
      }
      // segmented inclusive scan over runs of equal j (j is non-decreasing
      // across the lanes)
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const WA ox = shfl_up_any(x, d);
        const int oj = __shfl_up_sync(FULL, j, d);
        const bool oh = __shfl_up_sync(FULL, have ? 1 : 0, d) != 0;
        if (lane >= d && oj == j && oh) {
          if (have) {
            f.comp(&x, ox, g);
          } else {
            x = ox;
            have = true;
          }
        }
      }
      const int nj = __shfl_down_sync(FULL, j, 1);
      const bool tail = lane == 31 || nj != j;
      if (tail && have && j >= 0) {
        const int64_t first = s_sc[j];
        const int64_t last = s_sc[j + 1] - 2;  // the vertex's last edge slot
        if (first >= wbase && last <= wbase + 31)
          f.comp(f.wa_of(s_v[j]), x, g);
        else
          f.compAtomic(f.wa_of(s_v[j]), x, g);
      }
    }
    __syncthreads();
  }
}

// Edge-balanced pull for from-all patterns (every in-edge carries a message,
// e.g. PageRank): each warp reads 128 consecutive slots of the tile as four
// windows of 32.  The owner of a slot comes from a bitmap of the vertex
// boundaries that fall inside the window (every vertex holds at least one
// slot, so boundaries are distinct), not from a per-lane search; messages of
// a run are combined by a segmented shuffle scan whose run heads come from
// the same bitmap (f.data.zero fills the slots without a message), the run
// tails meet in shared memory, and every vertex
// of the tile is written once: comp() when all its slots lie in the tile,
// compAtomic() otherwise.
template <int T, typename G, typename F>
__global__ void __launch_bounds__(EXPAND_THREADS) k_pull_strict_all(active_set_t as, G g, F f, config_t conf,
                                                                    const int *tile_lo) {
  using WA = typename F::wa_t;
  constexpr int WSLOTS = T / (EXPAND_THREADS / 32);  // slots per warp
  __shared__ int s_v[T + 2];
  __shared__ int64_t s_sc[T + 2];
  __shared__ int64_t s_st[T + 2];
  __shared__ WA s_acc[T + 2];
  const int64_t n = as.get_size();
  GSW_HALT_IF_EMPTY(n);
  const Status want = conf.want();
  const int64_t *eoff = as.workset.dg_eoff;
  const int64_t total = eoff[n];
  const int64_t ntiles = (total + T - 1) / T;
  const int lane = lane_id(), w = warp_id();
  if (blockIdx.x == 0 && threadIdx.x == 0) account(as, conf, (unsigned long long)(total - n));
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t lo = tile_lo[t];
    const int64_t hi = (t + 1 < ntiles) ? tile_lo[t + 1] : n - 1;
    const int cnt = (int)(hi - lo + 1);
    for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
      const int v = as.fetch(lo + j, want);
      s_v[j] = v;
      s_sc[j] = eoff[lo + j];
      s_st[j] = v >= 0 ? __ldg(g.dgr_row_off + v) : 0;
      s_acc[j] = f.data.zero;
    }
    if (threadIdx.x == 0) s_sc[cnt] = eoff[hi + 1];
    __syncthreads();
    const int64_t t1 = MIN(total, t * T + T);
    const int64_t wbeg = t * T + (int64_t)w * WSLOTS;
    if (wbeg < t1) {
      int j0 = upper_bound(s_sc, cnt, wbeg) - 1;  // owner of the warp's first slot
      for (int64_t wb = wbeg; wb < MIN(t1, wbeg + WSLOTS); wb += 32) {
        const int64_t s = wb + lane;
        // boundaries (first slots of the next vertices) inside this window
        const int bj = j0 + 1 + lane;
        const int64_t bpos = bj <= cnt ? s_sc[bj] : INT64_MAX;
        const unsigned bm = __reduce_or_sync(FULL, bpos <= wb + 31 ? 1u << (int)(bpos - wb) : 0u);
        const unsigned upto = bm & (0xffffffffu >> (31 - lane));  // boundaries at or before this lane
        const int j = j0 + __popc(upto);
        const int head = upto ? 31 - __clz(upto) : 0;  // first lane of this lane's run
        WA x = f.data.zero;
        if (s < t1) {
          const int64_t local = s - s_sc[j];
          if (local < s_sc[j + 1] - s_sc[j] - 1) {
            const int64_t ei = s_st[j] + local;
            const int u = __ldg(g.dgr_adj_list + ei);
            x = f.emit(u, g.fetch_edata_r(ei), g);
          }
        }
        // segmented inclusive scan: runs start at the boundary lanes
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const WA ox = shfl_up_any(x, d);
          if (lane - d >= head) f.comp(&x, ox, g);
        }
        // a run ends at lane 31, before the next boundary, or at the tile's
        // last slot (the lanes past it hold the identity)
        const bool tail = lane == 31 || ((bm >> (lane + 1)) & 1u) || s + 1 == t1;
        if (tail && s < t1) f.compAtomic(&s_acc[j], x, g);
        j0 = __shfl_sync(FULL, j, 31);
        if (j0 + 1 <= cnt && s_sc[j0 + 1] <= wb + 32) ++j0;  // a vertex starting right after the window
      }
    }
    __syncthreads();
    for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
      const int v = s_v[j];
      const int64_t first = s_sc[j], deg = s_sc[j + 1] - s_sc[j] - 1;
      if (v < 0 || deg <= 0) continue;
      if (first >= t * T && first + deg <= t * T + T)
        f.comp(f.wa_of(v), s_acc[j], g);
      else
        f.compAtomic(f.wa_of(v), s_acc[j], g);
    }
    __syncthreads();
  }
}

// ===========================================================================
// Hub runs: the edges [a, a + len) of one vertex swept by the whole CTA
// ===========================================================================
// How a CTA reads a hub's columns (config_t::conf_hub_path):
//   HUB_SCALAR  4-byte read-only loads, one column per thread per round;
//   HUB_VECTOR  the 16-byte-aligned body of the run with int4 loads, four
//               consecutive columns per thread per round;
//   HUB_STAGED  the aligned body moves to shared memory in HUB_CHUNK-column
//               chunks by 1-D TMA bulk copies into two buffers (chunk c+2 is
//               issued into a buffer as soon as chunk c has been consumed, so
//               the next chunk is in flight while the CTA works on one).
// The ragged head and tail of a run (fewer than 4 columns each) are read
// with plain loads.  `edge(valid, u, ei)` runs for every thread in every
// round (warp-uniform trip counts, so fused levels can stage their appends
// per warp).  The staged form returns false, in every thread, if a copy did
// not complete in time; the caller then leaves the kernel.
enum { HUB_SCALAR = 0, HUB_VECTOR = 1, HUB_STAGED = 2 };
constexpr int HUB_CHUNK = 2048;  // columns per staged chunk (8 KB)

struct hub_stage_t {
  int (*buf)[HUB_CHUNK];     // [2][HUB_CHUNK] in shared memory, 16-byte aligned
  unsigned long long *bar;   // [2] mbarriers, initialised with count 1
  unsigned ph[2] = {0, 0};   // phase parity each buffer waits for next
};

template <int B, typename EDGE>
__device__ __forceinline__ bool hub_run(const int *col, int64_t a, int64_t len, int path, hub_stage_t &hs,
                                        unsigned *err, EDGE &&edge) {
  const int t = threadIdx.x;
  const int64_t e = a + len;
  const int64_t ba = (a + 3) & ~int64_t(3), bb = e & ~int64_t(3);
  if (path == HUB_SCALAR || bb - ba < 4 * B) {
    for (int64_t base = a; base < e; base += B) {
      const int64_t k = base + t;
      edge(k < e, k < e ? __ldg(col + k) : -1, k);
    }
    return true;
  }
  {  // ragged ends: head [a, ba) on threads 0.., tail [bb, e) after them
    const int nh = (int)(ba - a), nt = (int)(e - bb);
    const int64_t k = t < nh ? a + t : bb + (t - nh);
    const bool valid = t < nh + nt;
    edge(valid, valid ? __ldg(col + k) : -1, k);
  }
  if (path == HUB_VECTOR) {
    const int4 *c4 = reinterpret_cast<const int4 *>(col + ba);
    const int64_t n4 = (bb - ba) >> 2;
    for (int64_t r = t; r - t < n4; r += B) {
      const bool valid = r < n4;
      int4 q = make_int4(-1, -1, -1, -1);
      if (valid) q = __ldg(c4 + r);
      const int64_t k = ba + 4 * r;
      edge(valid, q.x, k);
      edge(valid, q.y, k + 1);
      edge(valid, q.z, k + 2);
      edge(valid, q.w, k + 3);
    }
    return true;
  }
  // staged: chunks [ba + c*HUB_CHUNK, ...) of the body
  const int64_t body = bb - ba;
  const int nch = (int)((body + HUB_CHUNK - 1) / HUB_CHUNK);
  auto issue = [&](int c) {
    const int64_t c0 = ba + (int64_t)c * HUB_CHUNK;
    const unsigned bytes = (unsigned)(4 * MIN((int64_t)HUB_CHUNK, bb - c0));
    fence_proxy_async_smem();
    mbar_expect_tx(&hs.bar[c & 1], bytes);
    bulk_copy_g2s(hs.buf[c & 1], col + c0, bytes, &hs.bar[c & 1]);
  };
  __syncthreads();  // the buffers' previous contents are consumed
  if (t == 0) {
    issue(0);
    if (nch > 1) issue(1);
  }
  bool okk = true;
  for (int c = 0; c < nch; ++c) {
    const int b = c & 1;
    const bool arrived = mbar_wait(&hs.bar[b], hs.ph[b], err);
    hs.ph[b] ^= 1u;
    okk = __syncthreads_and(arrived) != 0;
    if (!okk) {
      // let a copy still in flight land before the CTA leaves
      if (t == 0 && c + 1 < nch) mbar_wait(&hs.bar[b ^ 1], hs.ph[b ^ 1], err);
      return false;
    }
    const int64_t c0 = ba + (int64_t)c * HUB_CHUNK;
    const int cn = (int)MIN((int64_t)HUB_CHUNK, bb - c0);
    for (int base = 0; base < cn; base += B) {
      const int k = base + t;
      edge(k < cn, k < cn ? hs.buf[b][k] : -1, c0 + k);
    }
    __syncthreads();  // chunk c consumed: its buffer takes chunk c+2
    if (t == 0 && c + 2 < nch) issue(c + 2);
  }
  return true;
}

// ===========================================================================
// TWC: thread / warp / CTA tiers by degree
// ===========================================================================
// Per-launch tiered pushes list their hubs (deg >= EXPAND_THREADS) for the
// hub kernel instead of sweeping them in the tile that found them (see
// hub_list_t above).
template <bool FUSED, typename G, typename F, typename Src>
__device__ __forceinline__ void push_twc_body(active_set_t &as, const G &g, F &f, const config_t &conf, const Src &src,
                                              int64_t n, warp_stage_t &stage, hub_list_t hubs = hub_list_t()) {
  constexpr int B = EXPAND_THREADS;
  __shared__ int s_owner;
  __shared__ int s_cv;
  __shared__ int s_cdeg;
  __shared__ int64_t s_cst;
  __shared__ int s_scan[B];
  __shared__ int s_v[B];
  __shared__ int64_t s_st[B];
  __shared__ int s_tmp[33];
  __shared__ __align__(16) int s_hub[2][HUB_CHUNK];
  __shared__ __align__(8) unsigned long long s_bar[2];
  const int lane = lane_id();
  // measured on RMAT scale 24 (forced tiered push, whole runs): staging in
  // shared memory is fastest without edge data (BFS 7.3 -> 11.5 GTEPS), int4
  // loads with it (SSSP 6.1 -> 10.7); the edge data stays in global memory
  const int hub_path = conf.conf_hub_path >= 0 ? conf.conf_hub_path
                                               : (std::is_same<typename G::edge_t, Empty>::value ? HUB_STAGED
                                                                                                 : HUB_VECTOR);
  hub_stage_t hs{s_hub, s_bar};
  if (threadIdx.x == 0) {
    s_owner = -1;
    if (hub_path == HUB_STAGED) {
      mbar_init(&s_bar[0], 1);
      mbar_init(&s_bar[1], 1);
      fence_mbar_init();
    }
  }
  __syncthreads();
  for (int64_t tile = blockIdx.x; tile * B < n; tile += gridDim.x) {
    const int64_t idx = tile * B + threadIdx.x;
    const int v = idx < n ? src(idx) : -1;
    src.visit(v, g, f);
    int64_t st;
    int deg;
    vertex_range(g, false, v, st, deg);
    if (defer_hub(as, conf, hubs, v, st, deg, B)) deg = 0;  // hub: swept by the hub kernel
    // CTA tier
    for (;;) {
      if (deg >= B) s_owner = threadIdx.x;
      __syncthreads();
      const int owner = s_owner;
      __syncthreads();  // every thread has read the owner before it is cleared
      if (owner < 0) break;
      if ((int)threadIdx.x == owner) {
        s_cv = v;
        s_cst = st;
        s_cdeg = deg;
        deg = 0;
        s_owner = -1;
      }
      __syncthreads();
      const int cv = s_cv, cdeg = s_cdeg;
      const int64_t cst = s_cst;
      if (threadIdx.x == 0) account(as, conf, (unsigned long long)cdeg);
      const bool okk = hub_run<B>(g.dg_adj_list, cst, cdeg, hub_path, hs, &as.dg_cnt->err,
                                  [&](bool valid, int u, int64_t ei) {
                                    bool tp = false;
                                    if (valid) {
                                      if (FUSED)
                                        tp = push_edge_fused(as, g, f, conf, cv, u, ei);
                                      else
                                        push_edge_std(as, g, f, conf, cv, u, ei);
                                    }
                                    if (FUSED) stage.push(tp, u);
                                  });
      if (!okk) return;  // a staging copy timed out (recorded in the error word)
      __syncthreads();
    }
    // warp tier
    for (;;) {
      const unsigned m = __ballot_sync(FULL, deg >= 32);
      if (!m) break;
      const int leader = __ffs(m) - 1;
      const int wv = __shfl_sync(FULL, v, leader);
      const int wdeg = __shfl_sync(FULL, deg, leader);
      const int64_t wst = __shfl_sync(FULL, st, leader);
      if (lane == leader) {
        deg = 0;
        account(as, conf, (unsigned long long)wdeg);
      }
      for (int base = 0; base < wdeg; base += 32) {
        const int k = base + lane;
        bool tp = false;
        int u = -1;
        if (k < wdeg) {
          u = __ldg(g.dg_adj_list + wst + k);
          if (FUSED)
            tp = push_edge_fused(as, g, f, conf, wv, u, wst + k);
          else
            push_edge_std(as, g, f, conf, wv, u, wst + k);
        }
        if (FUSED) stage.push(tp, u);
      }
    }
    // thread tier: remaining small lists mapped through a CTA scan
    int total;
    const int ex = block_exclusive_scan(deg, s_tmp, &total);
    if (threadIdx.x == 0) account(as, conf, (unsigned long long)total);
    s_scan[threadIdx.x] = ex;
    s_v[threadIdx.x] = v;
    s_st[threadIdx.x] = st;
    __syncthreads();
    for (int base = 0; base < total; base += B) {
      const int i = base + threadIdx.x;
      bool tp = false;
      int u = -1;
      if (i < total) {
        const int id = upper_bound(s_scan, B, i) - 1;
        const int64_t ei = s_st[id] + (i - s_scan[id]);
        u = __ldg(g.dg_adj_list + ei);
        if (FUSED)
          tp = push_edge_fused(as, g, f, conf, s_v[id], u, ei);
        else
          push_edge_std(as, g, f, conf, s_v[id], u, ei);
      }
      if (FUSED) stage.push(tp, u);
    }
    __syncthreads();
  }
  // the barriers may be initialised again by the next call (persistent
  // launches run this body once per level); every copy has landed
  if (hub_path == HUB_STAGED && threadIdx.x == 0) {
    mbar_inval(&s_bar[0]);
    mbar_inval(&s_bar[1]);
  }
}

template <bool FUSED, typename G, typename F>
__global__ void __launch_bounds__(EXPAND_THREADS) k_push_twc(active_set_t as, G g, F f, config_t conf,
                                                             hub_list_t hubs) {
  __shared__ int s_stage[FUSED ? EXPAND_THREADS / 32 : 1][FUSED ? STAGE_SLOTS : 1];
  const int64_t n = as.get_size();
  GSW_HALT_IF_EMPTY(n);
  warp_stage_t stage(s_stage[FUSED ? warp_id() : 0], as);
  push_twc_body<FUSED>(as, g, f, conf, as_src_t{&as, conf.want()}, n, stage, hubs);
  if (FUSED) stage.flush();
}

// the hub pieces the tiered push listed: one piece per CTA at a time
template <bool FUSED, typename G, typename F>
__global__ void __launch_bounds__(EXPAND_THREADS) k_push_twc_hubs(active_set_t as, G g, F f, config_t conf,
                                                                  hub_list_t hubs) {
  constexpr int B = EXPAND_THREADS;
  __shared__ int s_stage[FUSED ? B / 32 : 1][FUSED ? STAGE_SLOTS : 1];
  __shared__ __align__(16) int s_hub[2][HUB_CHUNK];
  __shared__ __align__(8) unsigned long long s_bar[2];
  __shared__ int s_np;
  if (threadIdx.x == 0) {
    s_np = (int)MIN((int64_t)*(volatile int *)hubs.count, hubs.cap);
    __threadfence();
    if (atomicAdd(hubs.done, 1u) == gridDim.x - 1) {  // every CTA has read the count
      *hubs.count = 0;
      *hubs.done = 0;
    }
  }
  __syncthreads();
  const int np = s_np;
  if ((int)blockIdx.x >= np) return;  // no piece for this CTA (uniform)
  const int hub_path = conf.conf_hub_path >= 0 ? conf.conf_hub_path
                                               : (std::is_same<typename G::edge_t, Empty>::value ? HUB_STAGED
                                                                                                 : HUB_VECTOR);
  warp_stage_t stage(s_stage[FUSED ? warp_id() : 0], as);
  hub_stage_t hs{s_hub, s_bar};
  if (threadIdx.x == 0 && hub_path == HUB_STAGED) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  bool okk = true;
  for (int p = blockIdx.x; okk && p < np; p += gridDim.x) {
    const hub_piece_t pc = hubs.piece[p];
    okk = hub_run<B>(g.dg_adj_list, pc.st, pc.len, hub_path, hs, &as.dg_cnt->err, [&](bool valid, int u, int64_t ei) {
      bool tp = false;
      if (valid) {
        if (FUSED)
          tp = push_edge_fused(as, g, f, conf, pc.v, u, ei);
        else
          push_edge_std(as, g, f, conf, pc.v, u, ei);
      }
      if (FUSED) stage.push(tp, u);
    });
    __syncthreads();
  }
  if (!okk) return;  // a staging copy timed out (recorded in the error word)
  if (hub_path == HUB_STAGED && threadIdx.x == 0) {
    mbar_inval(&s_bar[0]);
    mbar_inval(&s_bar[1]);
  }
  if (FUSED) stage.flush();
}

// TWC pull: candidates with large in-degree are swept by the whole CTA or a
// warp with a cooperative reduction (and a ballot-driven early exit when the
// pattern allows pruning); the rest by one thread each.
template <typename G, typename F>
__global__ void __launch_bounds__(EXPAND_THREADS) k_pull_twc(active_set_t as, G g, F f, config_t conf) {
  using WA = typename F::wa_t;
  constexpr int B = EXPAND_THREADS;
  constexpr int NW = B / 32;
  __shared__ int s_owner;
  __shared__ int s_cv;
  __shared__ int s_cdeg;
  __shared__ int64_t s_cst;
  __shared__ int s_stop;
  __shared__ WA s_part[NW];
  __shared__ int s_have[NW];
  const int64_t n = as.get_size();
  GSW_HALT_IF_EMPTY(n);
  const Status want = conf.want();
  const int lane = lane_id(), w = warp_id();
  if (threadIdx.x == 0) s_owner = -1;
  __syncthreads();
  for (int64_t tile = blockIdx.x; tile * B < n; tile += gridDim.x) {
    const int64_t idx = tile * B + threadIdx.x;
    const int v = idx < n ? as.fetch(idx, want) : -1;
    int64_t st;
    int deg;
    vertex_range(g, true, v, st, deg);
    // CTA tier
    for (;;) {
      if (deg >= B) s_owner = threadIdx.x;
      __syncthreads();
      const int owner = s_owner;
      __syncthreads();  // every thread has read the owner before it is cleared
      if (owner < 0) break;
      if ((int)threadIdx.x == owner) {
        s_cv = v;
        s_cst = st;
        s_cdeg = deg;
        deg = 0;
        s_owner = -1;
        s_stop = 0;
      }
      __syncthreads();
      const int cv = s_cv, cdeg = s_cdeg;
      const int64_t cst = s_cst;
      if (threadIdx.x == 0) account(as, conf, (unsigned long long)cdeg);
      WA acc;
      bool have = false;
      for (int base = 0; base < cdeg; base += B) {
        const int k = base + threadIdx.x;
        if (k < cdeg) {
          const int u = __ldg(g.dgr_adj_list + cst + k);
          if (conf.conf_fromall || as.bitmap.is_active(u)) {
            WA x = f.emit(u, g.fetch_edata_r(cst + k), g);
            if (have)
              f.comp(&acc, x, g);
            else {
              acc = x;
              have = true;
            }
          }
        }
        if (conf.conf_pruning) {
          if (__syncthreads_or(have)) break;
        }
      }
      // warp-level fold of the per-thread partials, then across warps
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) {
        const WA o = shfl_down_any(acc, d);
        const bool oh = __shfl_down_sync(FULL, have, d);
        if (oh) {
          if (have)
            f.comp(&acc, o, g);
          else {
            acc = o;
            have = true;
          }
        }
      }
      if (lane == 0) {
        s_part[w] = acc;
        s_have[w] = have;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        WA tot;
        bool th = false;
        for (int k = 0; k < NW; ++k)
          if (s_have[k]) {
            if (th)
              f.comp(&tot, s_part[k], g);
            else {
              tot = s_part[k];
              th = true;
            }
          }
        if (th) f.comp(f.wa_of(cv), tot, g);
      }
      __syncthreads();
    }
    // warp tier
    for (;;) {
      const unsigned m = __ballot_sync(FULL, deg >= 32);
      if (!m) break;
      const int leader = __ffs(m) - 1;
      const int wv = __shfl_sync(FULL, v, leader);
      const int wdeg = __shfl_sync(FULL, deg, leader);
      const int64_t wst = __shfl_sync(FULL, st, leader);
      if (lane == leader) {
        deg = 0;
        account(as, conf, (unsigned long long)wdeg);
      }
      WA acc;
      bool have = false;
      for (int base = 0; base < wdeg; base += 32) {
        const int k = base + lane;
        if (k < wdeg) {
          const int u = __ldg(g.dgr_adj_list + wst + k);
          if (conf.conf_fromall || as.bitmap.is_active(u)) {
            WA x = f.emit(u, g.fetch_edata_r(wst + k), g);
            if (have)
              f.comp(&acc, x, g);
            else {
              acc = x;
              have = true;
            }
          }
        }
        if (conf.conf_pruning && __any_sync(FULL, have)) break;
      }
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) {
        const WA o = shfl_down_any(acc, d);
        const bool oh = __shfl_down_sync(FULL, have, d);
        if (oh) {
          if (have)
            f.comp(&acc, o, g);
          else {
            acc = o;
            have = true;
          }
        }
      }
      if (lane == 0 && have) f.comp(f.wa_of(wv), acc, g);
    }
    // thread tier
    account(as, conf, (unsigned long long)deg);
    if (deg > 0) {
      WA acc;
      bool have = false;
      for (int k = 0; k < deg; ++k) {
        const int u = __ldg(g.dgr_adj_list + st + k);
        if (conf.conf_fromall || as.bitmap.is_active(u)) {
          WA x = f.emit(u, g.fetch_edata_r(st + k), g);
          if (have)
            f.comp(&acc, x, g);
          else {
            acc = x;
            have = true;
          }
          if (conf.conf_pruning) break;
        }
      }
      if (have) f.comp(f.wa_of(v), acc, g);
    }
    __syncthreads();
  }
}

// ===========================================================================
// edge-centric, pointer jumping, exit probe, compensation
// ===========================================================================
template <typename G, typename F>
__global__ void __launch_bounds__(512) k_expand_ec(active_set_t as, G g, F f) {
  const int64_t n = as.get_size();
  const int64_t STRIDE = (int64_t)blockDim.x * gridDim.x;
  for (int64_t idx = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; idx < n; idx += STRIDE) {
    const int e = as.fetch(idx, Active);
    if (e < 0) continue;
    const packed_t vv = g.dg_coo[e];
    f.update((int)(vv >> 32), (int)(vv & 0xffffffffll), (typename G::edge_t *)nullptr);
  }
}

// Every vertex is re-pointed at the root of its chain (the fixed point the
// reference's repeated single jumps reach, src/utils/intrinsics.cuh:328-362);
// chains only shorten while this runs, and the walk is bounded by n steps.
__global__ void __launch_bounds__(512) k_pointer_jump(int *wa, int64_t n, unsigned *err) {
  const int64_t STRIDE = (int64_t)blockDim.x * gridDim.x;
  for (int64_t v = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; v < n; v += STRIDE) {
    int r = wa[v];
    int64_t guard = 0;
    for (;;) {
      const int p = ((volatile int *)wa)[r];
      if (p == r) break;
      r = p;
      if (++guard > n) {
        atomicOr(err, DEV_ERR_BAD_VERTEX);
        break;
      }
    }
    wa[v] = r;
  }
}

template <typename G, typename F>
__global__ void __launch_bounds__(512) k_exit(G g, F f, int *cnt) {
  const int64_t STRIDE = (int64_t)blockDim.x * gridDim.x;
  for (int64_t v = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; v < g.nvertexs; v += STRIDE)
    if (f.exit((int)v, g)) {
      *cnt = 1;
      return;
    }
}

template <typename G, typename F>
__global__ void __launch_bounds__(512) k_filter_all(G g, F f, int64_t n) {
  const int64_t STRIDE = (int64_t)blockDim.x * gridDim.x;
  for (int64_t v = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; v < n; v += STRIDE) f.filter((int)v, g);
}

template <typename G, typename F>
__global__ void __launch_bounds__(512) k_compensation(active_set_t as, G g, F f) {
  const int64_t n = as.get_queue_size_hard();
  const int64_t STRIDE = (int64_t)blockDim.x * gridDim.x;
  for (int64_t idx = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; idx < n; idx += STRIDE)
    f.filter(as.fetch_queue(idx), g);
}

}  // namespace gsw
