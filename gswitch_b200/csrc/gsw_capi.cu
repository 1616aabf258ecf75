// libgsw.so: the C ABI declared in include/gsw.h.
//
// Owns contexts (device + stream + reusable workspaces), device graphs
// (int64 row offsets, int32 columns, int32 degrees, optional weights, lazily
// built edge list for edge-centric operators) and the level loops of the
// seven applications, written the way the reference's application mains
// drive inspector / selector / executor (file:line per runner).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <unordered_map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gsw.h"
#include "apps.cuh"
#include "engine/devloop.cuh"
#include "engine/mlp.cuh"
#include "graphgen.cuh"
#include "bc_batch.cuh"
#include "mbfs.cuh"

using namespace gsw;

// ---------------------------------------------------------------------------
// context and graph objects
// ---------------------------------------------------------------------------
struct gsw_graph {
  gsw_ctx *ctx = nullptr;
  int64_t n = 0, m = 0;
  bool directed = false, weighted = false;
  int64_t *off = nullptr;
  int *col = nullptr, *odeg = nullptr, *w = nullptr;
  int64_t *roff = nullptr;
  int *rcol = nullptr, *rdeg = nullptr, *rw = nullptr;
  packed_t *coo = nullptr;
  int64_t ncoo = -1;
  double attr[6] = {0, 0, 0, 0, 0, 0};
  double mean_weight = 0;
  std::vector<int> hdeg;  // host copy of the out-degrees (root features, roots)
  struct twod_store {
    uint64_t *edge = nullptr;
    int64_t *tile_off = nullptr, *heavy_off = nullptr, *heavy_beg = nullptr, *heavy_end = nullptr;
    int *heavy_src = nullptr;
    int *item_tile = nullptr, *tile_items = nullptr;
    int64_t *item_beg = nullptr, *item_end = nullptr;
    twod_layout L;
  } *twod = nullptr;  // 2D-partition layout, built on first use

  template <typename E>
  device_graph_t<CSR, E> view() const {
    device_graph_t<CSR, E> g;
    g.dg_row_off = off;
    g.dg_adj_list = col;
    g.dg_odegree = odeg;
    g.dg_edgedata = (E *)w;
    g.dgr_row_off = directed ? roff : off;
    g.dgr_adj_list = directed ? rcol : col;
    g.dgr_odegree = directed ? rdeg : odeg;
    g.dgr_edgedata = (E *)(directed ? rw : w);
    g.nvertexs = (int)n;
    g.nedges = m;
    g.level = 0;
    g.directed = directed;
    return g;
  }
};

struct gsw_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t upload_stream = nullptr;  // graph uploads: the column copy
  cudaEvent_t up0 = nullptr, up1 = nullptr;
  executor_t executor;
  std::map<std::pair<int64_t, int>, active_set_t> as_cache;
  std::map<std::string, std::pair<void *, size_t>> bufs;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  stat_t stats;  // inspector counters, reused by every run of the context
  tree_node *dtrees = nullptr;  // the selector's trees in device memory
  int ntree_nodes = 0;
  tree_set dts{};
  const tree_node *dstepping = nullptr;  // the window's stepping tree, in dtrees
  std::map<int, dloop_graph> dl;  // captured level loops, one per application
  mlp_model mlp{};                // learned selector (valid = 0: none loaded)
  mlp_model mlp_fusion{};         // learned fusion decision of Mono-pattern runs
  mlp_model *dmlp = nullptr;      // its device copy (captured loops)
  std::string record_path;        // per-level feature records (empty: off)

  // Device blocks of destroyed graphs, kept for the next graph of a fitting
  // size: a graph uploaded per call otherwise pays a fresh cudaMalloc and
  // cudaFree's device-wide synchronisation every time (about 10 ms for a
  // 2.2 GB CSR).  Blocks go back to the pool on graph destroy (stream order
  // on the context's one stream keeps a reused block from being overwritten
  // while a kernel still reads it); the pool keeps at most GRAPH_POOL_CAP
  // bytes, gives back all of it when any of the context's allocations fails,
  // and is freed with the context.
  static constexpr size_t GRAPH_POOL_CAP = (size_t)8 << 30;
  std::multimap<size_t, void *> graph_pool;     // free blocks by size
  std::unordered_map<void *, size_t> graph_blocks;  // every pool-managed block
  size_t graph_pool_bytes = 0;
  void graph_pool_trim() {
    for (auto &kv : graph_pool) {
      graph_blocks.erase(kv.second);
      cudaFree(kv.second);
    }
    graph_pool.clear();
    graph_pool_bytes = 0;
  }
  void *graph_alloc(size_t bytes) {
    bytes = bytes ? bytes : 1;
    auto it = graph_pool.lower_bound(bytes);
    if (it != graph_pool.end() && it->first <= bytes + bytes / 4) {  // at most a quarter unused
      void *p = it->second;
      graph_pool_bytes -= it->first;
      graph_pool.erase(it);
      return p;
    }
    void *p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      cudaGetLastError();
      graph_pool_trim();
      if (GSW_CUDA(cudaMalloc(&p, bytes))) return nullptr;
    }
    graph_blocks[p] = bytes;
    return p;
  }
  void graph_free(void *p) {
    if (!p) return;
    auto it = graph_blocks.find(p);
    if (it == graph_blocks.end() || graph_pool_bytes + it->second > GRAPH_POOL_CAP) {
      if (it != graph_blocks.end()) graph_blocks.erase(it);
      cudaFree(p);
      return;
    }
    graph_pool.emplace(it->second, p);
    graph_pool_bytes += it->second;
  }

  void *buf(const std::string &name, size_t bytes) {
    auto it = bufs.find(name);
    if (it != bufs.end() && it->second.second >= bytes) return it->second.first;
    if (it != bufs.end()) {
      cudaFree(it->second.first);
      bufs.erase(it);
    }
    void *p = nullptr;
    if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) {
      cudaGetLastError();
      graph_pool_trim();
      if (GSW_CUDA(cudaMalloc(&p, bytes ? bytes : 1))) return nullptr;
    }
    bufs[name] = {p, bytes};
    return p;
  }
  active_set_t *aset(int64_t size, QueueMode qm) {
    auto key = std::make_pair(size, (int)qm);
    auto it = as_cache.find(key);
    if (it != as_cache.end()) return &it->second;
    active_set_t as;
    if (as.build(size, qm)) {
      as.destroy();
      if (graph_pool_bytes == 0) return nullptr;
      // give the cached graph blocks back and try once more
      clear_error();
      graph_pool_trim();
      as = active_set_t();
      if (as.build(size, qm)) {
        as.destroy();
        return nullptr;
      }
    }
    return &(as_cache[key] = as);
  }
};

namespace gsw {
// text of the calling thread's last failed ABI call (also set by the
// allocation-free entry point in gsw_noalloc.cu)
thread_local std::string g_last_error;
}  // namespace gsw

namespace {

// where the level loops of the current call write feature records (nullptr:
// nowhere); set from the context on every entry
inline const char *&record_sink() {
  static thread_local const char *p = nullptr;
  return p;
}

struct entry_guard {  // binds the context's device and stream for one call
  explicit entry_guard(gsw_ctx *ctx) {
    clear_error();
    record_sink() = nullptr;
    if (ctx) {
      cudaSetDevice(ctx->device);
      stream() = ctx->stream;
      if (!ctx->record_path.empty()) record_sink() = ctx->record_path.c_str();
    }
  }
  gsw_status finish() {
    if (!ok()) g_last_error = err().msg;
    return err().code;
  }
};

gsw_status fail(int code, const char *msg) {
  set_error(code, "%s", msg);
  g_last_error = msg;
  return code;
}

int grid_for(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256 + 1, (int64_t)sm_count() * 8); }

// Degree statistics of graph_attr_t::fill (src/utils/fileIO.cuh:35-67) from a
// device histogram of the degrees: the integer sums (average, deviation,
// range, maximum) come out exactly as the reference's ascending double sums;
// the Gini and Hoover-like terms are summed per run of equal degrees in
// closed form (equal to the per-vertex sums up to rounding).
__global__ void k_deg_max(const int *odeg, int64_t n, int *out) {
  int m = 0;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
    m = odeg[v] > m ? odeg[v] : m;
  m = warp_max(m);
  if (lane_id() == 0) atomicMax(out, m);
}
constexpr int HIST_SMEM = 2048;
__global__ void __launch_bounds__(256) k_deg_hist(const int *odeg, int64_t n, unsigned long long *hist) {
  __shared__ unsigned s_h[HIST_SMEM];
  for (int i = threadIdx.x; i < HIST_SMEM; i += blockDim.x) s_h[i] = 0;
  __syncthreads();
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int d = odeg[v];
    if (d < HIST_SMEM)
      atomicAdd(&s_h[d], 1u);
    else
      atomicAdd(hist + d, 1ull);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < HIST_SMEM; i += blockDim.x)
    if (s_h[i]) atomicAdd(hist + i, (unsigned long long)s_h[i]);
}

void compute_attr(gsw_graph *g) {
  if (g->n < 2) return;
  int *dmax = (int *)g->ctx->buf("attr_max", sizeof(int));
  if (!dmax) return;
  GSW_CUDA(cudaMemsetAsync(dmax, 0, sizeof(int), stream()));
  k_deg_max<<<grid_for(g->n), 256, 0, stream()>>>(g->odeg, g->n, dmax);
  int mx = 0;
  GSW_CUDA(cudaMemcpyAsync(&mx, dmax, sizeof(int), cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  const size_t bins = (size_t)MAX(mx + 1, HIST_SMEM);
  unsigned long long *dh = (unsigned long long *)g->ctx->buf("attr_hist", sizeof(unsigned long long) * bins);
  if (!dh || !ok()) return;
  GSW_CUDA(cudaMemsetAsync(dh, 0, sizeof(unsigned long long) * bins, stream()));
  k_deg_hist<<<grid_for(g->n), 256, 0, stream()>>>(g->odeg, g->n, dh);
  std::vector<unsigned long long> hist(bins);
  GSW_CUDA(cudaMemcpyAsync(hist.data(), dh, sizeof(unsigned long long) * bins, cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  if (!ok()) return;
  const double nv = (double)g->n;
  double avg = 0, sd = 0;
  int mn = -1;
  for (int d = 0; d <= mx; ++d) {
    if (!hist[d]) continue;
    if (mn < 0) mn = d;
    avg += (double)hist[d] * d;  // integer-valued: exact in any order
    sd += (double)hist[d] * ((double)d * d);
  }
  const double sum = avg;
  sd = std::sqrt((sd - avg * avg / nv) / (nv - 1));
  avg /= nv;
  double gi = 0, her = 0, i0 = 0;
  const double lsum = std::log(sum);
  for (int d = 0; d <= mx; ++d) {
    const double c = (double)hist[d];
    if (c == 0) continue;
    // sum over positions i0+1 .. i0+c of (n - i + 0.5) * d / n / sum
    gi += (c * (nv + 0.5) - (c * i0 + c * (c + 1) / 2)) * d / nv / sum;
    if (d != 0) her += c * d * (lsum - std::log((double)d)) / sum;
    i0 += c;
  }
  gi = 1 - 2 * gi;
  her = her / std::log(nv);
  g->attr[0] = avg;
  g->attr[1] = sd;
  g->attr[2] = (double)(mx - (mn < 0 ? 0 : mn));
  g->attr[3] = mx;
  g->attr[4] = gi;
  g->attr[5] = her;
}

// host copy of the degrees, fetched once when a caller needs it
const std::vector<int> &host_degrees(gsw_graph *g) {
  if ((int64_t)g->hdeg.size() != g->n) {
    g->hdeg.resize(g->n);
    GSW_CUDA(cudaMemcpyAsync(g->hdeg.data(), g->odeg, sizeof(int) * g->n, cudaMemcpyDeviceToHost, stream()));
    GSW_CUDA(cudaStreamSynchronize(stream()));
  }
  return g->hdeg;
}

__global__ void k_sum_weights(const int *w, int64_t m, unsigned long long *out) {
  unsigned long long s = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) s += w[i];
  s = warp_sum(s);
  if (lane_id() == 0 && s) atomicAdd(out, s);
}

void finalize_graph(gsw_graph *g) {
  int64_t *off = g->off;
  if (!g->odeg) {
    if (!(g->odeg = (int *)g->ctx->graph_alloc(sizeof(int) * (g->n + 1)))) return;
    k_deg_to_i32<<<grid_for(g->n), 256, 0, stream()>>>(off, g->n, g->odeg);
    GSW_LAUNCHED();
  }
  if (g->weighted) {
    unsigned long long *d = (unsigned long long *)g->ctx->buf("wsum", 8);
    if (!d) return;
    GSW_CUDA(cudaMemsetAsync(d, 0, 8, stream()));
    k_sum_weights<<<grid_for(g->m), 256, 0, stream()>>>(g->w, g->m, d);
    unsigned long long s = 0;
    GSW_CUDA(cudaMemcpyAsync(&s, d, 8, cudaMemcpyDeviceToHost, stream()));
    GSW_CUDA(cudaStreamSynchronize(stream()));
    g->mean_weight = g->m ? (double)s / (double)g->m : 0;
  }
  compute_attr(g);
}

// CSR from device keys (both directions of every pair, self-loops = ~0)
int csr_from_keys(gsw_graph *g, uint64_t *keys, int64_t nkeys) {
  void *tmp = nullptr;
  size_t tmpb = 0;
  uint64_t *sorted = nullptr;
  int *flag = nullptr;
  int64_t *pos = nullptr;
  if (GSW_CUDA(cudaMalloc((void **)&sorted, sizeof(uint64_t) * (nkeys + 1)))) return err().code;
  cub::DeviceRadixSort::SortKeys(nullptr, tmpb, keys, sorted, nkeys, 0, 64, stream());
  if (GSW_CUDA(cudaMalloc(&tmp, tmpb))) return err().code;
  GSW_CUDA(cub::DeviceRadixSort::SortKeys(tmp, tmpb, keys, sorted, nkeys, 0, 64, stream()));
  cudaFree(tmp);
  tmp = nullptr;
  // unique: flags -> positions (reuse `keys` as the compacted output)
  if (GSW_CUDA(cudaMalloc((void **)&flag, sizeof(int) * (nkeys + 1)))) return err().code;
  if (GSW_CUDA(cudaMalloc((void **)&pos, sizeof(int64_t) * (nkeys + 1)))) return err().code;
  k_unique_flags<<<grid_for(nkeys), 256, 0, stream()>>>(sorted, nkeys, flag);
  int *num = (int *)g->ctx->buf("nsel", 8);
  tmpb = 0;
  cub::DeviceSelect::Flagged(nullptr, tmpb, sorted, flag, keys, num, nkeys, stream());
  if (GSW_CUDA(cudaMalloc(&tmp, tmpb))) return err().code;
  GSW_CUDA(cub::DeviceSelect::Flagged(tmp, tmpb, sorted, flag, keys, num, nkeys, stream()));
  int m = 0;
  GSW_CUDA(cudaMemcpyAsync(&m, num, sizeof(int), cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  cudaFree(tmp);
  cudaFree(sorted);
  cudaFree(flag);
  cudaFree(pos);
  g->m = m;
  if (!(g->col = (int *)g->ctx->graph_alloc(sizeof(int) * ((size_t)m + 1)))) return err().code;
  if (!(g->off = (int64_t *)g->ctx->graph_alloc(sizeof(int64_t) * (g->n + 1)))) return err().code;
  unsigned long long *deg = (unsigned long long *)g->off;  // count into off[1..n]
  GSW_CUDA(cudaMemsetAsync(g->off, 0, sizeof(int64_t) * (g->n + 1), stream()));
  k_split_keys<<<grid_for(m), 256, 0, stream()>>>(keys, m, g->col, deg + 1);
  tmpb = 0;
  cub::DeviceScan::InclusiveSum(nullptr, tmpb, g->off + 1, g->off + 1, g->n, stream());
  if (GSW_CUDA(cudaMalloc(&tmp, tmpb))) return err().code;
  GSW_CUDA(cub::DeviceScan::InclusiveSum(tmp, tmpb, g->off + 1, g->off + 1, g->n, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  cudaFree(tmp);
  return err().code;
}

int64_t root_deg(const gsw_graph *g, int64_t root) {
  if (root < 0 || root >= g->n) return -1;
  if ((int64_t)g->hdeg.size() == g->n) return g->hdeg[root];
  int d = 0;  // one value instead of the whole table
  GSW_CUDA(cudaMemcpyAsync(&d, g->odeg + root, sizeof(int), cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  return d;
}

gsw_graph *new_graph(gsw_ctx *ctx, int64_t n) {
  gsw_graph *g = new gsw_graph();
  g->ctx = ctx;
  g->n = n;
  return g;
}

void free_graph(gsw_graph *g) {
  if (!g) return;
  for (void *p : {(void *)g->off, (void *)g->col, (void *)g->odeg, (void *)g->w, (void *)g->roff, (void *)g->rcol,
                  (void *)g->rdeg, (void *)g->rw})
    g->ctx->graph_free(p);
  cudaFree(g->coo);
  if (g->twod) {
    cudaFree(g->twod->edge);
    cudaFree(g->twod->tile_off);
    cudaFree(g->twod->heavy_off);
    cudaFree(g->twod->heavy_beg);
    cudaFree(g->twod->heavy_end);
    cudaFree(g->twod->heavy_src);
    cudaFree(g->twod->item_tile);
    cudaFree(g->twod->tile_items);
    cudaFree(g->twod->item_beg);
    cudaFree(g->twod->item_end);
    delete g->twod;
  }
  delete g;
}

int add_weights(gsw_graph *g, int wmax, uint64_t wseed) {
  if (wmax <= 0) return GSW_OK;
  if (!(g->w = (int *)g->ctx->graph_alloc(sizeof(int) * ((size_t)g->m + 1)))) return err().code;
  k_weights<<<grid_for(g->n), 256, 0, stream()>>>(g->off, g->col, g->n, stream_key(wseed, ST_W), wmax, g->w);
  g->weighted = true;
  return GSW_LAUNCHED();
}

gsw_status finish_generate(gsw_ctx *ctx, gsw_graph *g, uint64_t *keys, int64_t nkeys, int wmax, uint64_t wseed,
                           gsw_graph **out, entry_guard &eg) {
  if (csr_from_keys(g, keys, nkeys) == GSW_OK) add_weights(g, wmax, wseed);
  cudaFree(keys);
  if (ok()) finalize_graph(g);
  if (!ok()) {
    free_graph(g);
    return eg.finish();
  }
  *out = g;
  return GSW_OK;
}

// ---- COO (edge list) for edge-centric operators ---------------------------
__global__ void k_coo_count(const int64_t *off, const int *col, int64_t n, bool all, int64_t *cnt) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    int64_t c = 0;
    for (int64_t e = off[v]; e < off[v + 1]; ++e) c += all || col[e] > v;
    cnt[v] = c;
  }
}
__global__ void k_coo_write(const int64_t *off, const int *col, int64_t n, bool all, const int64_t *pos,
                            packed_t *coo) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    int64_t p = pos[v];
    for (int64_t e = off[v]; e < off[v + 1]; ++e)
      if (all || col[e] > v) coo[p++] = ((packed_t)v << 32) | (uint32_t)col[e];
  }
}

int ensure_coo(gsw_graph *g) {
  if (g->coo) return GSW_OK;
  int64_t *cnt = (int64_t *)g->ctx->buf("coo_cnt", sizeof(int64_t) * (g->n + 1));
  if (!cnt) return err().code;
  const bool all = g->directed;
  k_coo_count<<<grid_for(g->n), 256, 0, stream()>>>(g->off, g->col, g->n, all, cnt);
  GSW_CUDA(cudaMemsetAsync(cnt + g->n, 0, sizeof(int64_t), stream()));
  void *tmp = nullptr;
  size_t tmpb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmpb, cnt, cnt, g->n + 1, stream());
  if (GSW_CUDA(cudaMalloc(&tmp, tmpb))) return err().code;
  GSW_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmpb, cnt, cnt, g->n + 1, stream()));
  int64_t total = 0;
  GSW_CUDA(cudaMemcpyAsync(&total, cnt + g->n, sizeof(int64_t), cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  cudaFree(tmp);
  if (GSW_CUDA(cudaMalloc((void **)&g->coo, sizeof(packed_t) * (total + 1)))) return err().code;
  k_coo_write<<<grid_for(g->n), 256, 0, stream()>>>(g->off, g->col, g->n, all, cnt, g->coo);
  g->ncoo = total;
  return GSW_LAUNCHED();
}

// ---- 2D-partition layout (k_twod.cuh) ---------------------------------------
__global__ void k_twod_count(const int64_t *off, const int *col, int64_t n, int64_t ntiles, int *cnt) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = (v >> TWOD_TILE_BITS) * ntiles;
    for (int64_t e = off[v]; e < off[v + 1]; ++e) atomicAdd(cnt + row + (col[e] >> TWOD_TILE_BITS), 1);
  }
}
__global__ void k_twod_keys(const int64_t *off, const int *col, int64_t n, int64_t ntiles, const int *cnt,
                            uint64_t *keys) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t dt = (uint64_t)v >> TWOD_TILE_BITS, dl = (uint64_t)v & (TWOD_TILE - 1);
    for (int64_t e = off[v]; e < off[v + 1]; ++e) {
      const uint64_t u = (uint64_t)col[e];
      const uint64_t st = u >> TWOD_TILE_BITS;
      const uint64_t light = cnt[dt * ntiles + st] < TWOD_HEAVY ? 1 : 0;
      keys[e] = twod_key(dt, light, st, dl, u & (TWOD_TILE - 1));
    }
  }
}

// in-edges of every destination, keyed and sorted; heavy block table on the
// host from the per-pair counts
int ensure_twod(gsw_graph *g) {
  if (g->twod) return GSW_OK;
  const int64_t n = g->n, m = g->m;
  const int64_t ntiles = (n + TWOD_TILE - 1) / TWOD_TILE;
  if (ntiles >= (1 << 19)) return set_error(GSW_ERR_UNSUPPORTED, "%s", "2D partition: too many tiles");
  const int64_t *roff = g->directed ? g->roff : g->off;
  const int *rcol = g->directed ? g->rcol : g->col;
  int *cnt = nullptr;
  uint64_t *keys = nullptr, *sorted = nullptr;
  void *tmp = nullptr;
  size_t tmpb = 0;
  auto cleanup = [&]() {
    cudaFree(cnt);
    cudaFree(keys);
    cudaFree(tmp);
  };
  if (GSW_CUDA(cudaMalloc((void **)&cnt, sizeof(int) * ntiles * ntiles))) return cleanup(), err().code;
  GSW_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * ntiles * ntiles, stream()));
  k_twod_count<<<grid_for(n), 256, 0, stream()>>>(roff, rcol, n, ntiles, cnt);
  if (GSW_CUDA(cudaMalloc((void **)&keys, sizeof(uint64_t) * (m + 1)))) return cleanup(), err().code;
  if (GSW_CUDA(cudaMalloc((void **)&sorted, sizeof(uint64_t) * (m + 1)))) return cleanup(), err().code;
  k_twod_keys<<<grid_for(n), 256, 0, stream()>>>(roff, rcol, n, ntiles, cnt, keys);
  cub::DeviceRadixSort::SortKeys(nullptr, tmpb, keys, sorted, m, 0, 64, stream());
  if (GSW_CUDA(cudaMalloc(&tmp, tmpb))) return cudaFree(sorted), cleanup(), err().code;
  GSW_CUDA(cub::DeviceRadixSort::SortKeys(tmp, tmpb, keys, sorted, m, 0, 64, stream()));
  std::vector<int> hc((size_t)(ntiles * ntiles));
  GSW_CUDA(cudaMemcpyAsync(hc.data(), cnt, sizeof(int) * hc.size(), cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  cleanup();
  if (!ok()) {
    cudaFree(sorted);
    return err().code;
  }
  std::vector<int64_t> tile_off(ntiles + 1, 0), heavy_off(ntiles + 1, 0), hbeg, hend;
  std::vector<int> hsrc;
  for (int64_t dt = 0; dt < ntiles; ++dt) {
    int64_t pos = tile_off[dt];
    heavy_off[dt] = (int64_t)hsrc.size();
    int64_t tot = 0;
    for (int64_t st = 0; st < ntiles; ++st) {
      const int c = hc[dt * ntiles + st];
      tot += c;
      if (c >= TWOD_HEAVY) {
        hsrc.push_back((int)st);
        hbeg.push_back(pos);
        hend.push_back(pos + c);
        pos += c;
      }
    }
    tile_off[dt + 1] = tile_off[dt] + tot;
  }
  heavy_off[ntiles] = (int64_t)hsrc.size();
  // work items: each tile's edges cut into near-equal pieces of at most
  // TWOD_ITEM_EDGES
  std::vector<int> it_tile, tile_items(ntiles);
  std::vector<int64_t> it_beg, it_end;
  for (int64_t dt = 0; dt < ntiles; ++dt) {
    const int64_t a = tile_off[dt], e = tile_off[dt + 1] - a;
    if (e == 0) continue;
    const int64_t k = (e + TWOD_ITEM_EDGES - 1) / TWOD_ITEM_EDGES;
    tile_items[dt] = (int)k;
    for (int64_t i = 0; i < k; ++i) {
      it_tile.push_back((int)dt);
      it_beg.push_back(a + e * i / k);
      it_end.push_back(a + e * (i + 1) / k);
    }
  }
  auto *t = new gsw_graph::twod_store();
  t->edge = sorted;
  auto up = [&](void **dst, const void *src, size_t bytes) {
    if (GSW_CUDA(cudaMalloc(dst, bytes ? bytes : 8))) return;
    if (bytes) GSW_CUDA(cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, stream()));
  };
  up((void **)&t->tile_off, tile_off.data(), sizeof(int64_t) * tile_off.size());
  up((void **)&t->heavy_off, heavy_off.data(), sizeof(int64_t) * heavy_off.size());
  up((void **)&t->heavy_beg, hbeg.data(), sizeof(int64_t) * hbeg.size());
  up((void **)&t->heavy_end, hend.data(), sizeof(int64_t) * hend.size());
  up((void **)&t->heavy_src, hsrc.data(), sizeof(int) * hsrc.size());
  up((void **)&t->item_tile, it_tile.data(), sizeof(int) * it_tile.size());
  up((void **)&t->tile_items, tile_items.data(), sizeof(int) * tile_items.size());
  up((void **)&t->item_beg, it_beg.data(), sizeof(int64_t) * it_beg.size());
  up((void **)&t->item_end, it_end.data(), sizeof(int64_t) * it_end.size());
  GSW_CUDA(cudaStreamSynchronize(stream()));
  t->L.edge = t->edge;
  t->L.tile_off = t->tile_off;
  t->L.heavy_off = t->heavy_off;
  t->L.heavy_beg = t->heavy_beg;
  t->L.heavy_end = t->heavy_end;
  t->L.heavy_src = t->heavy_src;
  t->L.ntiles = ntiles;
  t->L.nheavy = (int64_t)hsrc.size();
  t->L.m = m;
  t->L.item_tile = t->item_tile;
  t->L.item_beg = t->item_beg;
  t->L.item_end = t->item_end;
  t->L.tile_items = t->tile_items;
  t->L.nitems = (int64_t)it_tile.size();
  g->twod = t;
  return err().code;
}

// ---------------------------------------------------------------------------
// run helpers
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_fill(T *p, T v, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = v;
}
template <typename T>
__global__ void k_fill_root(T *p, T v, T rootv, int64_t root, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = i == root ? rootv : v;
}
template <typename T>
void fill(T *p, T v, int64_t n) {
  k_fill<T><<<grid_for(n), 256, 0, stream()>>>(p, v, n);
}
template <typename T>
void fill_root(T *p, T v, T rootv, int64_t root, int64_t n) {
  k_fill_root<T><<<grid_for(n), 256, 0, stream()>>>(p, v, rootv, root, n);
}

__global__ void k_set_roots(int *wa, const int *roots, int nroots, int v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nroots) wa[roots[i]] = v;
}
// the roots are Active (and not Inactive) in the first inspection's bitmaps
__global__ void k_mark_roots(uint32_t *active, uint32_t *inactive, const int *roots, int nroots) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nroots) {
    const int r = roots[i];
    atomicOr(active + (r >> 5), 1u << (r & 31));
    atomicOr(inactive + (r >> 5), 1u << (r & 31));
  }
}

// Graph500 numerator: sum of degrees of reached vertices, halved
__global__ void k_reached_edges(const int *lvl_or_dist, int stride_ints, int unreached, const int *odeg, int64_t n,
                                unsigned long long *out) {
  unsigned long long s = 0;
  const int64_t T = (int64_t)gridDim.x * blockDim.x;
  const int64_t gt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (stride_ints == 1) {  // four vertices per 16-byte load
    const int64_t n4 = n / 4;
    for (int64_t q = gt; q < n4; q += T) {
      const int4 x = __ldg((const int4 *)lvl_or_dist + q);
      const int4 d = __ldg((const int4 *)odeg + q);
      s += (x.x != unreached && x.x >= 0) ? d.x : 0;
      s += (x.y != unreached && x.y >= 0) ? d.y : 0;
      s += (x.z != unreached && x.z >= 0) ? d.z : 0;
      s += (x.w != unreached && x.w >= 0) ? d.w : 0;
    }
    for (int64_t v = 4 * n4 + gt; v < n; v += T) {
      const int x = lvl_or_dist[v];
      if (x != unreached && x >= 0) s += odeg[v];
    }
  } else {
    for (int64_t v = gt; v < n; v += T) {
      const int x = lvl_or_dist[v * stride_ints];
      if (x != unreached && x >= 0) s += odeg[v];
    }
  }
  s = warp_sum(s);
  if (lane_id() == 0 && s) atomicAdd(out, s);
}

int64_t reached_edges(gsw_ctx *ctx, gsw_graph *g, const int *vals, int stride, int unreached) {
  unsigned long long *d = (unsigned long long *)ctx->buf("redges", 8);
  if (!d) return 0;
  GSW_CUDA(cudaMemsetAsync(d, 0, 8, stream()));
  k_reached_edges<<<grid_for(g->n), 256, 0, stream()>>>(vals, stride, unreached, g->odeg, g->n, d);
  unsigned long long s = 0;
  GSW_CUDA(cudaMemcpyAsync(&s, d, 8, cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  return (int64_t)(s / 2);
}

void apply_opts(const gsw_run_opts *o, config_t &conf) {
  conf.conf_persistent = true;
  opts().barrier_leave_test = false;
  if (!o) return;
  if (o->direction >= 0) {
    conf.force.has_direction = true;
    conf.force.d = o->direction == GSW_PULL ? Pull : Push;
  }
  if (o->asfmt >= 0) {
    conf.force.has_asfmt = true;
    conf.force.asf = o->asfmt == GSW_BITMAP ? Bitmap : Queue;
  }
  if (o->lb >= 0) {
    conf.force.has_lb = true;
    conf.force.lb = (LB)o->lb;
  }
  if (o->fusion >= 0) {
    conf.force.has_fusion = true;
    conf.force.fusion = o->fusion == GSW_FUSED ? Fused : Standalone;
  }
  conf.conf_sorted_queue = o->sorted_queue != 0;
  conf.conf_count_edges = o->account != 0;
  conf.conf_persistent = o->persistent != 0;
  conf.conf_hub_path = (o->hub_path >= 0 && o->hub_path <= 2) ? o->hub_path : -1;
  opts().barrier_leave_test = o->barrier_test != 0;
  opts().verbose = o->verbose != 0;
  opts().timing = o->timing != 0;
  opts().force_grid = o->expand_grid;
}

void set_graph_features(feature_t &fets, const gsw_graph *g) {
  fets.nvertexs = g->n;
  fets.nedges = g->m;
  fets.avg_deg = g->attr[0];
  fets.std_deg = g->attr[1];
  fets.range = g->attr[2];
  fets.max_deg = g->attr[3];
  fets.GI = g->attr[4];
  fets.Her = g->attr[5];
  fets.avg_edata = g->mean_weight;
}

struct loop_trace {
  gsw_run_stats *st;
  int64_t cap = 0;
  int64_t count = 0;
  int last = -1;
  std::vector<kernel_marks> pending;  // per traced level, resolved in finish()
  void level(const config_t &conf, int64_t frontier) {
    if (cap > 0 && ++count > cap) set_error(GSW_ERR_TIMEOUT, "%s", "level loop did not converge within the level cap");
    last = -1;
    if (!st) return;
    if (st->ntrace < GSW_MAX_TRACE) {
      last = st->ntrace;
      st->level_cfg[last] = (conf.conf_dir == Pull) | ((conf.conf_asfmt == Bitmap) << 1) |
                            ((int)conf.conf_lb << 2) | ((conf.conf_fuse_inspect ? 1 : 0) << 5);
      st->level_frontier[last] = frontier;
      st->level_ms[last] = 0;
      st->level_edges[last] = -1;
      st->ntrace++;
    }
    st->levels++;
  }
  // after the expand: the feature record where the reference's applications
  // keep their (commented-out) training hook (application/bfs.cu:95), the
  // edge count now, kernel times once the run is over
  void done(const stat_t &stats, feature_t &fets) {
    if (record_sink()) {
      fets.record_path = record_sink();
      fets.record();
    }
    if (!st || last < 0) return;
    // a persistent launch reports the load balance its kernel ran
    if (hints().persistent)
      st->level_cfg[last] = (st->level_cfg[last] & ~(7 << 2)) | ((hints().persistent_lb & 7) << 2) | (1 << 6);
    st->level_edges[last] = stats.last_scanned;
    st->level_inspect_ms[last] = 0;
    if (opts().timing) {
      if ((int)pending.size() <= last) pending.resize(last + 1);
      pending[last] = marks();
    }
  }
  // after the final synchronisation of the run
  void resolve() {
    if (!st || !opts().timing) return;
    const event_pool &p = timing_pool();
    for (int i = 0; i < (int)pending.size() && i < st->ntrace; ++i) {
      st->level_ms[i] = p.elapsed(pending[i].exp0, pending[i].exp1);
      st->level_inspect_ms[i] = p.elapsed(pending[i].insp0, pending[i].insp1);
    }
    timing_pool().used = 0;
  }
};

struct timer {
  gsw_ctx *ctx;
  explicit timer(gsw_ctx *c) : ctx(c) {
    if (!ctx->e0) {
      cudaEventCreate(&ctx->e0);
      cudaEventCreate(&ctx->e1);
    }
    cudaEventRecord(ctx->e0, stream());
  }
  double stop() {
    cudaEventRecord(ctx->e1, stream());
    cudaEventSynchronize(ctx->e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->e0, ctx->e1);
    return ms;
  }
};

void begin_stats(gsw_run_stats *st) {
  if (!st) return;
  st->ms = 0;
  st->levels = 0;
  st->edges = 0;
  st->device_error = 0;
  st->ntrace = 0;
  st->launches = 0;
  launch_count() = 0;
  timing_pool().used = 0;
}

// levels of persistent launches count one each in the loop; report real levels
void add_persistent_levels(gsw_run_stats *st, executor_t &ex, int64_t lv0, int64_t ln0) {
  if (st) st->levels += (int)((ex.persistent_levels - lv0) - (ex.persistent_launches - ln0));
}

unsigned end_checks(active_set_t *as, gsw_run_stats *st) {
  const unsigned e = as->read_error();
  if (st) {
    st->device_error = e;
    st->launches = launch_count();
  }
  if (e & DEV_ERR_QUEUE_OVERFLOW) set_error(GSW_ERR_OVERFLOW, "%s", "frontier queue overflow");
  if (e & DEV_ERR_SCRATCH_OVERFLOW) set_error(GSW_ERR_OVERFLOW, "%s", "STRICT tile table overflow");
  if (e & DEV_ERR_BARRIER_TIMEOUT) set_error(GSW_ERR_TIMEOUT, "%s", "grid barrier timed out");
  if (e & DEV_ERR_STAGE_TIMEOUT) set_error(GSW_ERR_TIMEOUT, "%s", "shared-memory staging copy did not complete");
  if (e & DEV_ERR_BAD_VERTEX) set_error(GSW_ERR_CUDA, "%s", "pointer chain longer than n");
  GSW_CUDA(cudaMemsetAsync(&as->dg_cnt->err, 0, sizeof(unsigned), stream()));
  return e;
}

// level cap of every loop: far above any legitimate run, it turns a loop
// that cannot converge into an error instead of a hang
inline int level_cap(int64_t n) { return (int)std::min<int64_t>(std::max<int64_t>(4 * n, 100000), 1 << 30); }
#define MAX_LEVELS level_cap(gr->n)

// ---------------------------------------------------------------------------
// captured level loop (engine/devloop.cuh)
// ---------------------------------------------------------------------------
enum { DL_APP_BFS = 0, DL_APP_PR = 1, DL_APP_CC = 2, DL_APP_SSSP = 3, DL_APP_GC = 4, DL_APP_PRD = 5 };

const tree_set *device_trees(gsw_ctx *ctx) {
  if (ctx->dtrees) return &ctx->dts;
  // the selector's nine trees, then the stepping tree of the window
  const tree_node *h[10] = {select_dir_idem_tree,        select_dir_asso_tree,         select_dir_asso_backup_tree,
                            select_fmt_tree,             select_fusion_tree,           select_lb_idem_tree,
                            select_lb_asso_forward_tree, select_lb_asso_backward_tree, select_lb_asso_backward_backup_tree,
                            select_stepping_tree};
  const int sz[10] = {select_dir_idem_tree_size,        select_dir_asso_tree_size,
                      select_dir_asso_backup_tree_size, select_fmt_tree_size,
                      select_fusion_tree_size,          select_lb_idem_tree_size,
                      select_lb_asso_forward_tree_size, select_lb_asso_backward_tree_size,
                      select_lb_asso_backward_backup_tree_size, select_stepping_tree_size};
  int total = 0;
  for (int x : sz) total += x;
  if (total > DL_MAX_TREE_NODES) return fail(GSW_ERR_UNSUPPORTED, "selector trees exceed the in-stream copy"), nullptr;
  std::vector<tree_node> all;
  all.reserve(total);
  for (int i = 0; i < 10; ++i) all.insert(all.end(), h[i], h[i] + sz[i]);
  if (GSW_CUDA(cudaMalloc((void **)&ctx->dtrees, sizeof(tree_node) * total))) return nullptr;
  if (GSW_CUDA(cudaMemcpy(ctx->dtrees, all.data(), sizeof(tree_node) * total, cudaMemcpyHostToDevice))) return nullptr;
  ctx->ntree_nodes = total;
  const tree_node *p[9];
  int off = 0;
  for (int i = 0; i < 9; ++i) {
    p[i] = ctx->dtrees + off;
    off += sz[i];
  }
  ctx->dts = tree_set{p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8]};
  ctx->dstepping = ctx->dtrees + off;
  return &ctx->dts;
}

// the values a captured loop bakes into its kernels: a cached graph is
// reused only when all of them are unchanged
struct dl_key {
  std::vector<unsigned long long> v;
  template <typename T>
  dl_key &operator<<(const T &x) {
    static_assert(sizeof(T) <= 8, "key fields are scalars");
    unsigned long long w = 0;
    memcpy(&w, &x, sizeof(T));
    v.push_back(w);
    return *this;
  }
};

// One prepared run of a captured loop: built (or found in the context's
// cache) before the timed region, launched inside it, collected after it.
struct dl_run {
  gsw_ctx *ctx = nullptr;
  dloop_graph *L = nullptr;
  dloop_t *d = nullptr;
  int *trace_cfg = nullptr;
  long long *trace_frontier = nullptr, *trace_edges = nullptr, *trace_t = nullptr, *trace_sel = nullptr;
  dloop_t image;
  unsigned long long push_sum = 0;  // after dl_collect: the loop's push workload
};

template <typename E, typename F>
bool dl_prepare(dl_run &R, gsw_ctx *ctx, int app, dl_key key, active_set_t &as, device_graph_t<CSR, E> g, F &f,
                const config_t &conf, const feature_t &fets, int max_iters, int iter_cap, int selector) {
  if (conf.conf_qmode != Normal || conf.conf_compensation || fets.centric != VC)
    return fail(GSW_ERR_UNSUPPORTED, "captured level loop: needs a Normal queue without compensation"), false;
  const tree_set *trees = device_trees(ctx);
  R.ctx = ctx;
  R.d = (dloop_t *)ctx->buf("dl_state", sizeof(dloop_t));
  R.trace_cfg = (int *)ctx->buf("dl_trace_cfg", sizeof(int) * GSW_MAX_TRACE);
  R.trace_frontier = (long long *)ctx->buf("dl_trace_frontier", sizeof(long long) * GSW_MAX_TRACE);
  R.trace_edges = (long long *)ctx->buf("dl_trace_edges", sizeof(long long) * GSW_MAX_TRACE);
  R.trace_t = (long long *)ctx->buf("dl_trace_t", sizeof(long long) * (GSW_MAX_TRACE + 1));
  R.trace_sel = (long long *)ctx->buf("dl_trace_sel", sizeof(long long) * (GSW_MAX_TRACE + 1));
  if (!trees || !R.d || !R.trace_cfg || !R.trace_frontier || !R.trace_edges || !R.trace_t || !R.trace_sel)
    return false;
  executor_t &ex = ctx->executor;
  ex.ensure_tiles(g.nedges + as.size + 1);
  if (!ok()) return false;
  key << app << R.d << g.dg_row_off << g.dg_adj_list << g.dg_odegree << g.dg_edgedata << g.dgr_row_off
      << g.dgr_adj_list << g.dgr_odegree << g.dgr_edgedata << g.nvertexs << g.nedges << g.directed;
  key << as.size << as.bitmap.visited.dg_bits << as.bitmap.active.dg_bits << as.bitmap.inactive.dg_bits
      << as.queue.subqueue[0].dg_queue << as.queue.subqueue[1].dg_queue << as.queue.subqueue[0].max_size
      << as.dg_cnt << as.workset.dg_eoff << as.workset.dg_bsum << as.workset.bsum_cap;
  key << conf.conf_pruning << conf.conf_count_edges << conf.conf_sorted_queue << fets.fromall << fets.toall
      << ex.dg_tile << ex.tile_cap << ex.twod.edge << opts().force_grid << ctx->stats.dg_runtime_info;
  key << conf.conf_window << conf.conf_fusion << f.data.dg_ra << conf.conf_persistent;
  for (int q : ex.tune.quarters[0][0][0]) key << q;  // first row: cheap change detector
  {
    const int *flat = &ex.tune.quarters[0][0][0][0];
    const int *shp = &ex.tune.shapes[0][0][0][0];
    unsigned long long h = 1469598103934665603ull;  // FNV-1a over both tables
    for (size_t i = 0; i < sizeof(ex.tune.quarters) / sizeof(int); ++i) h = (h ^ (unsigned)flat[i]) * 1099511628211ull;
    for (size_t i = 0; i < sizeof(ex.tune.shapes) / sizeof(int); ++i) h = (h ^ (unsigned)shp[i]) * 1099511628211ull;
    key << h;
  }
  dloop_graph &L = ctx->dl[app];
  R.L = &L;
  if (L.key != key.v || !L.exec) {
    if (!dl_build(L, ex, R.d, as, g, f, conf, fets, ctx->stats.dg_runtime_info)) return false;
    L.key = key.v;
  }
  dloop_t &im = R.image;
  im = L.image;
  im.fets = fets;
  im.conf = conf;
  im.trees = *trees;
  im.tree_base = ctx->dtrees;
  im.tree_nodes = ctx->ntree_nodes;
  im.mlp = (selector == GSW_SELECT_MLP && ctx->mlp.valid) ? ctx->dmlp : nullptr;
  im.raw = level_counts{0, 0, 0, 0, 0, 0};
  im.level = g.level;
  im.cursor = as.queue.cursor;
  im.halt = 0;
  im.inspected = 0;
  im.iter = 0;
  im.max_iters = max_iters;
  im.iter_cap = iter_cap;
  im.sorted = conf.conf_sorted_queue ? 1 : 0;
  im.status = DL_RUNNING;
  im.ntrace = 0;
  im.trace_cap = GSW_MAX_TRACE;
  im.trace_cfg = R.trace_cfg;
  im.trace_frontier = R.trace_frontier;
  im.trace_edges = R.trace_edges;
  im.trace_t = R.trace_t;
  im.trace_sel = R.trace_sel;
  im.info = ctx->stats.dg_runtime_info;
  im.scanned = conf.conf_count_edges ? &as.dg_cnt->scanned : nullptr;
  im.qsize = as.dg_cnt->qsize;
  im.nvertexs = g.nvertexs;
  im.nedges = g.nedges;
  im.as_size = as.size;
  im.launches = 0;
  im.push_sum = 0;
  im.win = f.data.window;
  im.window_on = conf.conf_window ? 1 : 0;
  im.stepping = ctx->dstepping;
  im.probe_flag = 0;
  im.probe_armed = 0;
  return ok();
}

// inside the timed region: state image in, one graph launch
void dl_launch(dl_run &R) {
  if (GSW_CUDA(cudaMemcpyAsync(R.d, &R.image, sizeof(dloop_t), cudaMemcpyHostToDevice, stream()))) return;
  if (R.image.scanned) GSW_CUDA(cudaMemsetAsync(R.image.scanned, 0, sizeof(unsigned long long), stream()));
  GSW_CUDA(cudaGraphLaunch(R.L->exec, stream()));
}

// after the timed region: state and trace back into the run statistics
void dl_collect(dl_run &R, gsw_run_stats *st) {
  dloop_t out;
  if (GSW_CUDA(cudaMemcpyAsync(&out, R.d, sizeof(dloop_t), cudaMemcpyDeviceToHost, stream()))) return;
  if (GSW_CUDA(cudaStreamSynchronize(stream()))) return;
  launch_count() += out.launches;
  R.push_sum = out.push_sum;
  if (out.status == DL_LEVEL_CAP) set_error(GSW_ERR_TIMEOUT, "%s", "level loop did not converge within the level cap");
  if (out.status == DL_NO_BODY) set_error(GSW_ERR_UNSUPPORTED, "%s", "captured level loop: variant has no body");
  if (out.status == DL_NOT_INSPECTED) set_error(GSW_ERR_CUDA, "%s", "captured level loop: inspection missing");
  if (out.status == DL_RUNNING) set_error(GSW_ERR_CUDA, "%s", "captured level loop did not finish");
  if (!st) return;
  st->levels = out.iter;
  const int nt = std::min(out.ntrace, (int)GSW_MAX_TRACE);
  st->ntrace = nt;
  if (nt > 0) {
    std::vector<int> cfg(nt);
    std::vector<long long> fr(nt), ed(nt), t0(nt + 1), ts(nt);
    GSW_CUDA(cudaMemcpyAsync(cfg.data(), R.trace_cfg, sizeof(int) * nt, cudaMemcpyDeviceToHost, stream()));
    GSW_CUDA(cudaMemcpyAsync(fr.data(), R.trace_frontier, sizeof(long long) * nt, cudaMemcpyDeviceToHost, stream()));
    GSW_CUDA(cudaMemcpyAsync(ed.data(), R.trace_edges, sizeof(long long) * nt, cudaMemcpyDeviceToHost, stream()));
    // iteration i: from its decision's start to the next one's (the final
    // decision, which stops the loop, writes t0[nt])
    const int nts = out.ntrace <= out.trace_cap && nt == out.ntrace ? nt + 1 : nt;
    GSW_CUDA(cudaMemcpyAsync(t0.data(), R.trace_t, sizeof(long long) * nts, cudaMemcpyDeviceToHost, stream()));
    GSW_CUDA(cudaMemcpyAsync(ts.data(), R.trace_sel, sizeof(long long) * nt, cudaMemcpyDeviceToHost, stream()));
    GSW_CUDA(cudaStreamSynchronize(stream()));
    for (int i = 0; i < nt; ++i) {
      st->level_cfg[i] = cfg[i];
      st->level_frontier[i] = fr[i];
      st->level_edges[i] = ed[i];
      st->level_ms[i] = i + 1 < nts ? (float)((t0[i + 1] - t0[i]) * 1e-6) : 0.f;
      st->level_inspect_ms[i] = (float)((ts[i] - t0[i]) * 1e-6);
    }
  }
}

// ---------------------------------------------------------------------------
// learned selector in the host-driven loop (engine/mlp.cuh)
// ---------------------------------------------------------------------------
bool mlp_override(const mlp_model &m, const feature_t &fets, config_t &conf) {
  if (!mlp_applicable(m, fets, conf)) return false;
  float x[MLP_IN], pt = 0;
  mlp_features(fets, x);
  const int k = mlp_predict_host(m, x, &pt);
  if (pt < m.min_conf) return false;
  mlp_apply(k, conf);
  return true;
}

// Mono-pattern runs (SSSP) keep one fusion mode for the whole run (the
// reference's select_fusion tree, src/model/select_fusion.h); with the
// learned selector a second network over graph features takes that
// decision.  Forced fusion wins.
void mlp_fusion_override(gsw_ctx *ctx, const gsw_run_opts *o, const feature_t &fets, config_t &conf) {
  const mlp_model &m = ctx->mlp_fusion;
  if (!o || o->selector != GSW_SELECT_MLP || !m.valid || conf.force.has_fusion || fets.centric != VC ||
      fets.pattern != Mono)
    return;
  float x[MLP_IN], pt = 0;
  mlp_fusion_features(fets, x);
  const int k = mlp_predict_host(m, x, &pt);
  if (pt < m.min_conf || k > 1) return;
  conf.conf_fuse_inspect = conf.conf_fusion = (k == 1);
  if (!conf.conf_fuse_inspect) conf.conf_qmode = Normal;
}

void select_level(gsw_ctx *ctx, const gsw_run_opts *o, selector_t &sel, stat_t &stats, feature_t &fets,
                  config_t &conf) {
  sel.select(stats, fets, conf);
  if (o && o->selector == GSW_SELECT_MLP) mlp_override(ctx->mlp, fets, conf);
}

// ---------------------------------------------------------------------------
// per-level labels for the learned selector
// ---------------------------------------------------------------------------
struct label_sink {
  int max_levels = 0, rows = 0, level = 0, every = 8, first = 24, level_limit = 1 << 30;
  float *X = nullptr, *T = nullptr;
  int32_t *R = nullptr;
};
thread_local label_sink *g_label = nullptr;

// Times every variant for this level from one snapshot of the state the
// expand touches (vertex data, the visited bits and the counters block), then
// puts everything back so the run continues exactly as without labelling.
template <typename G, typename F>
void label_level(gsw_ctx *ctx, active_set_t &as, G &g, F &f, stat_t &stats, feature_t &fets, config_t &conf) {
  label_sink *L = g_label;
  if (!L || !ok()) return;
  const int lv = L->level++;
  if (L->rows >= L->max_levels || lv >= L->level_limit || !(lv < L->first || lv % L->every == 0)) return;
  using WA = typename F::wa_t;
  using RA = typename F::ra_t;
  const int64_t n = as.size;
  const size_t wab = std::is_same<WA, Empty>::value ? 0 : sizeof(WA) * n;
  const size_t rab = std::is_same<RA, Empty>::value ? 0 : sizeof(RA) * n;
  const size_t vb = sizeof(uint32_t) * as.bitmap.visited.n_words;
  char *snap = (char *)ctx->buf("label_snap", wab + rab + vb + sizeof(as_counters_t) + 64);
  if (!snap) return;
  char *s_wa = snap, *s_ra = s_wa + wab, *s_vis = s_ra + rab, *s_cnt = s_vis + vb;
  auto copy_state = [&](bool save) {
    auto cp = [&](void *dev, char *keep, size_t bytes) {
      if (bytes)
        GSW_CUDA(cudaMemcpyAsync(save ? (void *)keep : dev, save ? dev : (void *)keep, bytes, cudaMemcpyDeviceToDevice,
                                 stream()));
    };
    cp(f.data.dg_wa, s_wa, wab);
    cp(f.data.dg_ra, s_ra, rab);
    cp(as.bitmap.visited.dg_bits, s_vis, vb);
    cp(as.dg_cnt, s_cnt, sizeof(as_counters_t));
  };
  // a level the inspection already halted (loops that test convergence after
  // the expand) expands nothing: no label, and the halt must survive
  if (*as.nt.h_tag) return;
  copy_state(true);
  const active_set_t as0 = as;
  const config_t conf0 = conf;
  const feature_t fets0 = fets;
  const int level0 = g.level;
  const double lt = stats.last_time, at = stats.avg_time, lf = stats.last_filter_time, le = stats.last_expand_time,
               af = stats.avg_filter_time, ae = stats.avg_expand_time;
  const int slevel = stats.level;
  executor_t &ex = ctx->executor;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float *X = L->X + (size_t)L->rows * MLP_IN, *T = L->T + (size_t)L->rows * MLP_K;
  mlp_features(fets, X);
  if (L->R) L->R[L->rows] = conf.conf_fuse_inspect ? -1 : mlp_class(conf.conf_dir, conf.conf_asfmt, conf.conf_lb);
  for (int k = 0; k < MLP_K; ++k) {
    Direction d;
    ASFmt a;
    LB lb;
    mlp_variant(k, d, a, lb);
    conf.conf_dir = d;
    conf.conf_asfmt = a;
    conf.conf_lb = lb;
    conf.conf_fuse_inspect = false;
    selector_t::set_target(conf);
    conf.force.has_lb = true;  // no small-level STRICT -> CM fallback while timing STRICT
    conf.force.lb = lb;
    cudaEventRecord(e0, stream());
    ex.filter(as, g, f, stats, fets, conf);
    g.update_level();
    ex.expand(as, g, f, stats, fets, conf);
    cudaEventRecord(e1, stream());
    float ms = 0;
    const bool good = ok() && cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
    const unsigned derr = as.read_error();
    T[k] = (good && !derr) ? (ms > 0 ? ms : 1e-4f) : 0.f;
    clear_error();
    GSW_CUDA(cudaStreamSynchronize(stream()));
    // back to the snapshot
    as = as0;
    conf = conf0;
    fets = fets0;
    g.level = level0;
    stats.last_time = lt, stats.avg_time = at, stats.last_filter_time = lf, stats.last_expand_time = le;
    stats.avg_filter_time = af, stats.avg_expand_time = ae, stats.level = slevel;
    copy_state(false);
    as.nt.reset();  // a trial's empty expand may have raised the halt flag
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  GSW_CUDA(cudaStreamSynchronize(stream()));
  L->rows++;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int gsw_version(void) { return 1; }

const char *gsw_last_error_string(void) { return g_last_error.c_str(); }

void gsw_run_opts_default(gsw_run_opts *o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->direction = o->asfmt = o->lb = o->fusion = GSW_AUTO;
  o->sorted_queue = 1;
  o->max_iters = 0;
  o->damping = 0.85f;
  o->eps = 0.01f;
  o->selector = GSW_SELECT_RULES;
  o->persistent = GSW_AUTO;
  o->hub_path = GSW_AUTO;
}

gsw_status gsw_init(int device, gsw_ctx **out) {
  entry_guard eg(nullptr);
  if (!out) return fail(GSW_ERR_INVALID_ARG, "gsw_init: out is NULL");
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return fail(GSW_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= count) return fail(GSW_ERR_INVALID_ARG, "gsw_init: device out of range");
  if (GSW_CUDA(cudaSetDevice(device))) return eg.finish();
  gsw_ctx *c = new gsw_ctx();
  c->device = device;
  if (GSW_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking))) {
    delete c;
    return eg.finish();
  }
  *out = c;
  return GSW_OK;
}

gsw_status gsw_destroy(gsw_ctx *ctx) {
  if (!ctx) return GSW_OK;
  entry_guard eg(ctx);
  cudaStreamSynchronize(ctx->stream);
  for (auto &kv : ctx->as_cache) kv.second.destroy();
  for (auto &kv : ctx->bufs) cudaFree(kv.second.first);
  ctx->graph_pool_trim();
  for (auto &kv : ctx->dl) kv.second.destroy();
  cudaFree(ctx->dtrees);
  cudaFree(ctx->dmlp);
  ctx->executor.destroy();
  ctx->stats.destroy();
  if (ctx->e0) cudaEventDestroy(ctx->e0);
  if (ctx->e1) cudaEventDestroy(ctx->e1);
  if (ctx->up0) cudaEventDestroy(ctx->up0);
  if (ctx->up1) cudaEventDestroy(ctx->up1);
  if (ctx->upload_stream) {
    cudaStreamSynchronize(ctx->upload_stream);
    cudaStreamDestroy(ctx->upload_stream);
  }
  cudaStreamDestroy(ctx->stream);
  stream() = 0;
  delete ctx;
  return GSW_OK;
}

// Checks of a caller's CSR before any kernel indexes with it: offsets that
// never decrease (bit 1), column indices in [0, n) (bit 2).
__global__ void k_check_offsets(const int64_t *off, int64_t n, int *bad) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
    if (off[v + 1] < off[v]) atomicOr(bad, 1);
}
__global__ void k_check_cols(const int *col, int64_t m, int64_t n, int *bad) {
  bool b = false;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x)
    b |= (unsigned)col[e] >= (unsigned long long)n;
  if (__any_sync(0xffffffffu, b) && (threadIdx.x & 31) == 0) atomicOr(bad, 2);
}

gsw_status gsw_graph_upload(gsw_ctx *ctx, int64_t n, int64_t m, const int64_t *row_off, const int32_t *col,
                            const int32_t *weights, int directed, gsw_graph **out) {
  entry_guard eg(ctx);
  if (!ctx || !out || n <= 0 || m < 0 || !row_off || (m > 0 && !col))
    return fail(GSW_ERR_INVALID_ARG, "gsw_graph_upload: bad arguments");
  if (n >= (int64_t)INT32_MAX) return fail(GSW_ERR_UNSUPPORTED, "gsw_graph_upload: n must fit int32");
  if (row_off[0] != 0 || row_off[n] != m) return fail(GSW_ERR_INVALID_ARG, "gsw_graph_upload: row_off[0] != 0 or row_off[n] != m");
  gsw_graph *g = new_graph(ctx, n);
  g->m = m;
  g->directed = directed != 0;
  g->weighted = weights != nullptr;
  auto up = [&](void **dst, const void *src, size_t bytes, cudaStream_t s) {
    if (!(*dst = ctx->graph_alloc(bytes))) return false;
    if (bytes && GSW_CUDA(cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, s))) return false;
    return true;
  };
  // The columns (and weights) copy on a second stream while the degrees and
  // the degree statistics come from the offsets on the context's stream.  The
  // second stream first waits for everything queued before the upload, so a
  // pooled block reused here is not overwritten while an earlier kernel still
  // reads it, and the context's stream waits for the copy before returning.
  if (!ctx->upload_stream) {
    if (GSW_CUDA(cudaStreamCreateWithFlags(&ctx->upload_stream, cudaStreamNonBlocking)) ||
        GSW_CUDA(cudaEventCreateWithFlags(&ctx->up0, cudaEventDisableTiming)) ||
        GSW_CUDA(cudaEventCreateWithFlags(&ctx->up1, cudaEventDisableTiming))) {
      free_graph(g);
      return eg.finish();
    }
  }
  cudaStream_t s2 = ctx->upload_stream;
  int *bad = (int *)ctx->buf("csr_check", sizeof(int));
  int hbad = 0, host_bad = 0;
  if (bad) GSW_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), stream()));
  GSW_CUDA(cudaEventRecord(ctx->up0, stream()));
  GSW_CUDA(cudaStreamWaitEvent(s2, ctx->up0, 0));
  bool okk = up((void **)&g->off, row_off, sizeof(int64_t) * (n + 1), stream()) &&
             (g->col = (int *)ctx->graph_alloc(sizeof(int) * m)) != nullptr;
  // the columns in chunks, each checked on the copy stream while the next
  // one crosses the link (the reverse CSR of a directed graph is built, and
  // its columns checked, on the host)
  constexpr int64_t COL_CHUNK = (int64_t)1 << 26;
  for (int64_t c0 = 0; okk && c0 < m; c0 += COL_CHUNK) {
    const int64_t cn = std::min(COL_CHUNK, m - c0);
    okk = !GSW_CUDA(cudaMemcpyAsync(g->col + c0, col + c0, sizeof(int) * cn, cudaMemcpyHostToDevice, s2));
    if (okk && bad && !g->directed) k_check_cols<<<grid_for(cn), 256, 0, s2>>>(g->col + c0, cn, n, bad);
  }
  if (okk && weights) okk = up((void **)&g->w, weights, sizeof(int) * m, s2);
  GSW_CUDA(cudaEventRecord(ctx->up1, s2));
  // the weights' mean and the reverse CSR need the copy first
  if (weights || g->directed) GSW_CUDA(cudaStreamWaitEvent(stream(), ctx->up1, 0));
  // the offsets are checked before anything derives degrees from them
  if (okk && bad) {
    k_check_offsets<<<grid_for(n), 256, 0, stream()>>>(g->off, n, bad);
    GSW_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, stream()));
    GSW_CUDA(cudaStreamSynchronize(stream()));
    if (hbad & 1) okk = false;
  }
  if (okk && g->directed) {
    // reverse CSR on the host (counting sort by destination)
    for (int64_t e = 0; e < m && okk; ++e) okk = col[e] >= 0 && col[e] < n;
    if (!okk) host_bad = 2;
  }
  if (okk && g->directed) {
    std::vector<int64_t> roff(n + 1, 0);
    for (int64_t e = 0; e < m; ++e) roff[(size_t)col[e] + 1]++;
    for (int64_t v = 0; v < n; ++v) roff[v + 1] += roff[v];
    std::vector<int> rcol(m), rw(weights ? m : 0);
    std::vector<int64_t> fillp(roff.begin(), roff.end() - 1);
    for (int64_t v = 0; v < n; ++v)
      for (int64_t e = row_off[v]; e < row_off[v + 1]; ++e) {
        const int64_t p = fillp[col[e]]++;
        rcol[p] = (int)v;
        if (weights) rw[p] = weights[e];
      }
    okk = up((void **)&g->roff, roff.data(), sizeof(int64_t) * (n + 1), stream()) &&
          up((void **)&g->rcol, rcol.data(), sizeof(int) * m, stream());
    if (okk && weights) okk = up((void **)&g->rw, rw.data(), sizeof(int) * m, stream());
    if (okk) {
      okk = (g->rdeg = (int *)ctx->graph_alloc(sizeof(int) * (n + 1))) != nullptr;
      if (okk) k_deg_to_i32<<<grid_for(n), 256, 0, stream()>>>(g->roff, n, g->rdeg);
    }
    GSW_CUDA(cudaStreamSynchronize(stream()));
  }
  if (okk) finalize_graph(g);
  GSW_CUDA(cudaStreamWaitEvent(stream(), ctx->up1, 0));
  if (bad) GSW_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  hbad |= host_bad;
  if (ok() && hbad) {
    free_graph(g);
    return fail(GSW_ERR_INVALID_ARG, (hbad & 1) ? "gsw_graph_upload: row offsets decrease at some vertex"
                                                : "gsw_graph_upload: a column index is outside [0, n)");
  }
  if (!ok()) {
    free_graph(g);
    return eg.finish();
  }
  *out = g;
  return GSW_OK;
}

gsw_status gsw_graph_generate_rmat(gsw_ctx *ctx, int scale, int edge_factor, double a, double b, double c,
                                   uint64_t seed, int wmax, uint64_t wseed, gsw_graph **out) {
  entry_guard eg(ctx);
  if (!ctx || !out || scale < 1 || scale > 30 || edge_factor < 1)
    return fail(GSW_ERR_INVALID_ARG, "gsw_graph_generate_rmat: bad arguments");
  const int64_t npairs = (int64_t)edge_factor << scale;
  if (2 * npairs >= (int64_t)INT32_MAX * 2) return fail(GSW_ERR_UNSUPPORTED, "rmat: too many arcs");
  gsw_graph *g = new_graph(ctx, (int64_t)1 << scale);
  uint64_t *keys = nullptr;
  if (GSW_CUDA(cudaMalloc((void **)&keys, sizeof(uint64_t) * (2 * npairs + 1)))) {
    free_graph(g);
    return eg.finish();
  }
  k_rmat_keys<<<grid_for(npairs), 256, 0, stream()>>>(make_rmat(scale, a, b, c, seed), npairs, keys);
  return finish_generate(ctx, g, keys, 2 * npairs, wmax, wseed, out, eg);
}

gsw_status gsw_graph_generate_grid(gsw_ctx *ctx, int rows, int cols, int lr_div, uint64_t seed, int wmax,
                                   uint64_t wseed, gsw_graph **out) {
  entry_guard eg(ctx);
  if (!ctx || !out || rows < 1 || cols < 2) return fail(GSW_ERR_INVALID_ARG, "gsw_graph_generate_grid: bad arguments");
  const int64_t nl = (int64_t)rows * (cols - 1) + (int64_t)(rows - 1) * cols;
  const int64_t nlr = lr_div > 0 ? nl / lr_div : 0;
  gsw_graph *g = new_graph(ctx, (int64_t)rows * cols);
  uint64_t *keys = nullptr;
  if (GSW_CUDA(cudaMalloc((void **)&keys, sizeof(uint64_t) * (2 * (nl + nlr) + 1)))) {
    free_graph(g);
    return eg.finish();
  }
  k_grid_keys<<<grid_for(nl + nlr), 256, 0, stream()>>>(rows, cols, nl, nlr, stream_key(seed, ST_GRID), keys);
  return finish_generate(ctx, g, keys, 2 * (nl + nlr), wmax, wseed, out, eg);
}

gsw_status gsw_graph_generate_er(gsw_ctx *ctx, int64_t n, int64_t m_pairs, uint64_t seed, int wmax, uint64_t wseed,
                                 gsw_graph **out) {
  entry_guard eg(ctx);
  if (!ctx || !out || n < 2 || m_pairs < 0) return fail(GSW_ERR_INVALID_ARG, "gsw_graph_generate_er: bad arguments");
  gsw_graph *g = new_graph(ctx, n);
  uint64_t *keys = nullptr;
  if (GSW_CUDA(cudaMalloc((void **)&keys, sizeof(uint64_t) * (2 * m_pairs + 1)))) {
    free_graph(g);
    return eg.finish();
  }
  k_er_keys<<<grid_for(m_pairs), 256, 0, stream()>>>(n, m_pairs, stream_key(seed, ST_ER), keys);
  return finish_generate(ctx, g, keys, 2 * m_pairs, wmax, wseed, out, eg);
}

gsw_status gsw_graph_generate_er_batch(gsw_ctx *ctx, int count, uint64_t seed, int64_t nlo, int64_t nhi, double dlo,
                                       double dhi, int wmax, uint64_t wseed, int64_t *vertex_offsets,
                                       gsw_graph **out) {
  entry_guard eg(ctx);
  if (!ctx || !out || count <= 0 || nlo < 2 || nhi < nlo || !(dlo > 0) || dhi < dlo)
    return fail(GSW_ERR_INVALID_ARG, "gsw_graph_generate_er_batch: bad arguments");
  // instance parameters: n log-uniform in [nlo, nhi], mean degree uniform
  // in [dlo, dhi], m = floor(n * degree / 2) pairs, its own seed
  std::vector<int64_t> voff(count + 1, 0), poff(count + 1, 0);
  std::vector<uint64_t> ikey(count);
  const uint64_t key = stream_key(seed, ST_ERB);
  auto unit = [](uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); };
  for (int i = 0; i < count; ++i) {
    const double u1 = unit(sm64(key + 3 * (uint64_t)i)), u2 = unit(sm64(key + 3 * (uint64_t)i + 1));
    int64_t n = (int64_t)std::llround(std::exp(std::log((double)nlo) + u1 * (std::log((double)nhi) - std::log((double)nlo))));
    n = std::min(std::max(n, nlo), nhi);
    const double deg = dlo + u2 * (dhi - dlo);
    voff[i + 1] = voff[i] + n;
    poff[i + 1] = poff[i] + (int64_t)std::floor((double)n * deg / 2.0);
    ikey[i] = stream_key(sm64(key + 3 * (uint64_t)i + 2), ST_ER);
  }
  const int64_t N = voff[count], P = poff[count];
  if (N >= (int64_t)INT32_MAX) return fail(GSW_ERR_UNSUPPORTED, "gsw_graph_generate_er_batch: union exceeds int32 ids");
  int64_t *dv = nullptr, *dp = nullptr;
  uint64_t *dk = nullptr, *keys = nullptr;
  auto cleanup = [&]() {
    cudaFree(dv);
    cudaFree(dp);
    cudaFree(dk);
  };
  if (GSW_CUDA(cudaMalloc((void **)&dv, sizeof(int64_t) * (count + 1))) ||
      GSW_CUDA(cudaMalloc((void **)&dp, sizeof(int64_t) * (count + 1))) ||
      GSW_CUDA(cudaMalloc((void **)&dk, sizeof(uint64_t) * count)) ||
      GSW_CUDA(cudaMalloc((void **)&keys, sizeof(uint64_t) * (2 * P + 1))))
    return cleanup(), cudaFree(keys), eg.finish();
  GSW_CUDA(cudaMemcpyAsync(dv, voff.data(), sizeof(int64_t) * (count + 1), cudaMemcpyHostToDevice, stream()));
  GSW_CUDA(cudaMemcpyAsync(dp, poff.data(), sizeof(int64_t) * (count + 1), cudaMemcpyHostToDevice, stream()));
  GSW_CUDA(cudaMemcpyAsync(dk, ikey.data(), sizeof(uint64_t) * count, cudaMemcpyHostToDevice, stream()));
  k_er_batch_keys<<<grid_for(P), 256, 0, stream()>>>(count, dv, dp, dk, keys);
  GSW_CUDA(cudaStreamSynchronize(stream()));
  cleanup();
  if (!ok()) return cudaFree(keys), eg.finish();
  if (vertex_offsets) memcpy(vertex_offsets, voff.data(), sizeof(int64_t) * (count + 1));
  gsw_graph *g = new_graph(ctx, N);
  return finish_generate(ctx, g, keys, 2 * P, wmax, wseed, out, eg);
}

gsw_status gsw_graph_generate_powerlaw(gsw_ctx *ctx, int64_t n, double gamma, uint64_t seed, int wmax,
                                       uint64_t wseed, gsw_graph **out) {
  entry_guard eg(ctx);
  if (!ctx || !out || n < 2 || !(gamma > 1.0) || n >= (int64_t)INT32_MAX)
    return fail(GSW_ERR_INVALID_ARG, "gsw_graph_generate_powerlaw: bad arguments");
  const int64_t cap = std::max<int64_t>(2, (int64_t)std::sqrt((double)n) * 4);
  int64_t *deg = nullptr, *off = nullptr;
  uint64_t *skey = nullptr, *skey2 = nullptr, *keys = nullptr;
  int *sval = nullptr, *sval2 = nullptr;
  void *tmp = nullptr;
  auto cleanup = [&]() {
    cudaFree(deg);
    cudaFree(off);
    cudaFree(skey);
    cudaFree(skey2);
    cudaFree(sval);
    cudaFree(sval2);
    cudaFree(tmp);
  };
  if (GSW_CUDA(cudaMalloc((void **)&deg, sizeof(int64_t) * (n + 1))) ||
      GSW_CUDA(cudaMalloc((void **)&off, sizeof(int64_t) * (n + 1))))
    return cleanup(), eg.finish();
  GSW_CUDA(cudaMemsetAsync(deg + n, 0, sizeof(int64_t), stream()));
  k_pl_degrees<<<grid_for(n), 256, 0, stream()>>>(n, gamma, cap, stream_key(seed, ST_PL), deg);
  size_t tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, deg, off, n + 1, stream());
  if (GSW_CUDA(cudaMalloc(&tmp, tb))) return cleanup(), eg.finish();
  GSW_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, deg, off, n + 1, stream()));
  int64_t S = 0;
  GSW_CUDA(cudaMemcpyAsync(&S, off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  cudaFree(tmp);
  tmp = nullptr;
  if (!ok()) return cleanup(), eg.finish();
  const int64_t npairs = S / 2;
  if (GSW_CUDA(cudaMalloc((void **)&skey, sizeof(uint64_t) * (S + 1))) ||
      GSW_CUDA(cudaMalloc((void **)&skey2, sizeof(uint64_t) * (S + 1))) ||
      GSW_CUDA(cudaMalloc((void **)&sval, sizeof(int) * (S + 1))) ||
      GSW_CUDA(cudaMalloc((void **)&sval2, sizeof(int) * (S + 1))))
    return cleanup(), eg.finish();
  k_pl_stubs<<<grid_for(n), 256, 0, stream()>>>(n, off, stream_key(seed, ST_PL + 100), skey, sval);
  tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, skey, skey2, sval, sval2, S, 0, 64, stream());
  if (GSW_CUDA(cudaMalloc(&tmp, tb))) return cleanup(), eg.finish();
  GSW_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, skey, skey2, sval, sval2, S, 0, 64, stream()));
  if (GSW_CUDA(cudaMalloc((void **)&keys, sizeof(uint64_t) * (2 * npairs + 1)))) return cleanup(), eg.finish();
  k_pl_pairs<<<grid_for(npairs), 256, 0, stream()>>>(sval2, npairs, keys);
  GSW_CUDA(cudaStreamSynchronize(stream()));
  cleanup();
  if (!ok()) {
    cudaFree(keys);
    return eg.finish();
  }
  gsw_graph *g = new_graph(ctx, n);
  return finish_generate(ctx, g, keys, 2 * npairs, wmax, wseed, out, eg);
}

gsw_status gsw_graph_info(const gsw_graph *g, int64_t *n, int64_t *m, int *weighted) {
  if (!g) return fail(GSW_ERR_INVALID_ARG, "gsw_graph_info: NULL graph");
  if (n) *n = g->n;
  if (m) *m = g->m;
  if (weighted) *weighted = g->weighted;
  return GSW_OK;
}

gsw_status gsw_graph_attr(const gsw_graph *g, double *out6) {
  if (!g || !out6) return fail(GSW_ERR_INVALID_ARG, "gsw_graph_attr: NULL argument");
  memcpy(out6, g->attr, sizeof(g->attr));
  return GSW_OK;
}

gsw_status gsw_graph_download(const gsw_graph *g, int64_t *row_off, int32_t *col, int32_t *weights) {
  if (!g) return fail(GSW_ERR_INVALID_ARG, "gsw_graph_download: NULL graph");
  entry_guard eg(g->ctx);
  if (row_off) GSW_CUDA(cudaMemcpyAsync(row_off, g->off, sizeof(int64_t) * (g->n + 1), cudaMemcpyDeviceToHost, stream()));
  if (col) GSW_CUDA(cudaMemcpyAsync(col, g->col, sizeof(int) * g->m, cudaMemcpyDeviceToHost, stream()));
  if (weights && g->w) GSW_CUDA(cudaMemcpyAsync(weights, g->w, sizeof(int) * g->m, cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  return eg.finish();
}

gsw_status gsw_graph_destroy(gsw_graph *g) {
  if (!g) return GSW_OK;
  entry_guard eg(g->ctx);
  cudaStreamSynchronize(stream());
  free_graph(g);
  return eg.finish();
}

gsw_status gsw_graph_roots(const gsw_graph *g, uint64_t seed, int count, int32_t *roots) {
  if (!g || !roots || count < 0) return fail(GSW_ERR_INVALID_ARG, "gsw_graph_roots: bad arguments");
  entry_guard eg(g->ctx);
  const std::vector<int> &deg = host_degrees(const_cast<gsw_graph *>(g));
  if (!ok()) return eg.finish();
  const uint64_t key = stream_key(seed, ST_ROOT);
  int got = 0;
  uint64_t j = 0;
  const uint64_t budget = 64ull * (uint64_t)g->n + 4096;
  while (got < count && j < budget) {
    const int v = (int)(sm64(key + j) % (uint64_t)g->n);
    ++j;
    if (deg[v] == 0) continue;
    bool dup = false;
    for (int q = 0; q < got; ++q) dup |= roots[q] == v;
    if (!dup) roots[got++] = v;
  }
  for (int64_t v = 0; got < count && v < g->n; ++v) {
    if (deg[v] == 0) continue;
    bool dup = false;
    for (int q = 0; q < got; ++q) dup |= roots[q] == (int)v;
    if (!dup) roots[got++] = (int)v;
  }
  while (got < count) roots[got++] = -1;
  return eg.finish();
}

gsw_status gsw_ctx_record_features(gsw_ctx *ctx, const char *path) {
  if (!ctx) return fail(GSW_ERR_INVALID_ARG, "gsw_ctx_record_features: bad arguments");
  ctx->record_path = path ? path : "";
  return GSW_OK;
}

gsw_status gsw_ctx_stream(gsw_ctx *ctx, void **s) {
  if (!ctx || !s) return fail(GSW_ERR_INVALID_ARG, "gsw_ctx_stream: bad arguments");
  *s = (void *)ctx->stream;
  return GSW_OK;
}

// ---------------------------------------------------------------------------
// BFS: application/bfs.cu:78-102 (loop) and :104-130 (set-up)
// ---------------------------------------------------------------------------
// BFS from one root, or from several at once (levels = distance to the
// nearest root; over a disjoint union of graphs with one root per part this
// is one BFS per part, all in the same level loop)
gsw_status bfs_run(gsw_ctx *ctx, gsw_graph *gr, const int32_t *roots, int nroots, const gsw_run_opts *o,
                   int32_t *levels, gsw_run_stats *st, entry_guard &eg) {
  const int32_t root = roots[0];
  begin_stats(st);
  auto g = gr->view<Empty>();
  app::BFS f;
  f.data.size = gr->n;
  f.data.dg_wa = (int *)ctx->buf("wa", sizeof(int) * (gr->n + 1));
  if (!f.data.dg_wa) return eg.finish();
  int64_t root_degree_sum = 0;
  if (nroots == 1) {
    fill_root<int>(f.data.dg_wa, -1, 0, root, gr->n);
    root_degree_sum = root_deg(gr, root);
  } else {
    int *droots = (int *)ctx->buf("bfs_roots", sizeof(int) * nroots);
    if (!droots) return eg.finish();
    GSW_CUDA(cudaMemcpyAsync(droots, roots, sizeof(int) * nroots, cudaMemcpyHostToDevice, stream()));
    fill<int>(f.data.dg_wa, -1, gr->n);
    k_set_roots<<<(nroots + 255) / 256, 256, 0, stream()>>>(f.data.dg_wa, droots, nroots, 0);
    host_degrees(gr);
    for (int i = 0; i < nroots; ++i) root_degree_sum += gr->hdeg[roots[i]];
  }
  feature_t fets;
  config_t conf;
  stat_t &stats = ctx->stats;
  stats.clean();
  inspector_t inspector;
  selector_t selector;
  executor_t &executor = ctx->executor;
  executor.insp = &inspector;
  executor.twod = twod_layout();
  const int64_t plv0 = executor.persistent_levels, pln0 = executor.persistent_launches;
  fets.centric = VC;
  fets.pattern = Idem;
  fets.fromall = false;
  fets.toall = false;
  conf.conf_pruning = true;
  apply_opts(o, conf);
  set_graph_features(fets, gr);
  fets.use_root = root;
  fets.first_active = nroots;
  init_conf_impl(stats, fets, conf, g, f, gr->mean_weight, gr->attr[0], false, root_degree_sum);
  active_set_t *asp = ctx->aset(gr->n, conf.conf_qmode);
  if (!asp) return eg.finish();
  active_set_t &as = *asp;
  as.reset();
  if (nroots == 1) {
    as.init(root);
  } else {
    as.init(ALL_INACTIVE);
    int *droots = (int *)ctx->buf("bfs_roots", sizeof(int) * nroots);
    k_mark_roots<<<(nroots + 255) / 256, 256, 0, stream()>>>(as.bitmap.active.dg_bits, as.bitmap.inactive.dg_bits,
                                                           droots, nroots);
  }
  loop_trace tr{st, MAX_LEVELS};
  const bool captured = o && o->captured;
  dl_run R;
  if (captured && !dl_prepare(R, ctx, DL_APP_BFS, dl_key() << f.data.dg_wa, as, g, f, conf, fets, 0, MAX_LEVELS,
                              o->selector))
    return eg.finish();
  timer tm(ctx);
  if (captured) dl_launch(R);
  for (int level = 0; !captured && ok(); level++) {
    inspector.inspect(as, g, f, stats, fets, conf);
    if (finish(as, g, f, conf)) break;
    select_level(ctx, o, selector, stats, fets, conf);
    if (g_label) label_level(ctx, as, g, f, stats, fets, conf);
    executor.filter(as, g, f, stats, fets, conf);
    g.update_level();
    tr.level(conf, hints().frontier);
    executor.expand(as, g, f, stats, fets, conf);
    tr.done(stats, fets);
    if (finish(as, g, f, conf)) break;
  }
  const double ms = tm.stop();
  if (captured) dl_collect(R, st);
  tr.resolve();
  end_checks(&as, st);
  add_persistent_levels(st, executor, plv0, pln0);
  if (st) {
    st->ms = ms;
    st->edges = reached_edges(ctx, gr, f.data.dg_wa, 1, -1);
  }
  if (levels && ok())
    GSW_CUDA(cudaMemcpyAsync(levels, f.data.dg_wa, sizeof(int) * gr->n, cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  return eg.finish();
}

gsw_status gsw_bfs(gsw_ctx *ctx, gsw_graph *gr, int32_t root, const gsw_run_opts *o, int32_t *levels,
                   gsw_run_stats *st) {
  entry_guard eg(ctx);
  if (!ctx || !gr || root < 0 || root >= gr->n) return fail(GSW_ERR_INVALID_ARG, "gsw_bfs: bad arguments");
  return bfs_run(ctx, gr, &root, 1, o, levels, st, eg);
}

gsw_status gsw_bfs_inspect(gsw_ctx *ctx, gsw_graph *gr, const int32_t *levels, int32_t level, uint64_t *out6) {
  entry_guard eg(ctx);
  if (!ctx || !gr || !levels || !out6) return fail(GSW_ERR_INVALID_ARG, "gsw_bfs_inspect: bad arguments");
  auto g = gr->view<Empty>();
  g.level = level;
  app::BFS f;
  f.data.size = gr->n;
  f.data.dg_wa = (int *)ctx->buf("wa", sizeof(int) * (gr->n + 1));
  if (!f.data.dg_wa) return eg.finish();
  GSW_CUDA(cudaMemcpyAsync(f.data.dg_wa, levels, sizeof(int) * gr->n, cudaMemcpyHostToDevice, stream()));
  active_set_t *asp = ctx->aset(gr->n, Normal);
  if (!asp) return eg.finish();
  stat_t &stats = ctx->stats;
  stats.build();
  stats.clean();
  launch_inspect_vc(*asp, g, f, stats.dg_runtime_info);
  GSW_LAUNCHED();
  stats.collect(6);
  stats.clean();
  for (int i = 0; i < 6; ++i) out6[i] = stats.h_runtime_info[i];
  return eg.finish();
}

gsw_status gsw_bfs_multi(gsw_ctx *ctx, gsw_graph *gr, int nroots, const int32_t *roots, const gsw_run_opts *o,
                         int32_t *levels, gsw_run_stats *st) {
  entry_guard eg(ctx);
  if (!ctx || !gr || nroots <= 0 || !roots) return fail(GSW_ERR_INVALID_ARG, "gsw_bfs_multi: bad arguments");
  for (int i = 0; i < nroots; ++i)
    if (roots[i] < 0 || roots[i] >= gr->n) return fail(GSW_ERR_INVALID_ARG, "gsw_bfs_multi: root out of range");
  return bfs_run(ctx, gr, roots, nroots, o, levels, st, eg);
}

// ---------------------------------------------------------------------------
// A BFS level loop that the caller drives (the reference's per-level calls
// from application/bfs.cu:78-102: inspector.inspect, selector.select,
// executor.filter, g.update_level, executor.expand, as.finish), one level per
// gsw_level_begin / gsw_level_end pair.  The state lives in the context's
// buffers, so nothing else may run on the context between begin and end.
// ---------------------------------------------------------------------------
}  // extern "C"
struct gsw_traversal {
  gsw_ctx *ctx = nullptr;
  gsw_graph *gr = nullptr;
  device_graph_t<CSR, Empty> g;
  app::BFS f;
  feature_t fets;
  config_t conf;
  inspector_t inspector;
  active_set_t *as = nullptr;
  gsw_run_stats st;
  loop_trace tr{nullptr, 0};
  int64_t root_degree = 0;
  int64_t plv0 = 0, pln0 = 0;
  double ms = 0;
  int first = 1;      // the next level is the run's first (not inspected)
  int done = 0;       // the loop is over
  int inspected = 0;  // gsw_level_begin ran for the current level
};
extern "C" {

gsw_status gsw_traversal_begin(gsw_ctx *ctx, gsw_graph *gr, int app, int32_t root, const gsw_run_opts *o,
                               gsw_traversal **out) {
  entry_guard eg(ctx);
  if (!ctx || !gr || !out || app != GSW_APP_BFS || root < 0 || root >= gr->n)
    return fail(GSW_ERR_INVALID_ARG, "gsw_traversal_begin: bad arguments (BFS from a vertex of the graph)");
  if (o && o->captured) return fail(GSW_ERR_UNSUPPORTED, "gsw_traversal_begin: the caller drives the loop");
  *out = nullptr;
  auto *t = new gsw_traversal();
  t->ctx = ctx;
  t->gr = gr;
  begin_stats(&t->st);
  t->g = gr->view<Empty>();
  t->f.data.size = gr->n;
  t->f.data.dg_wa = (int *)ctx->buf("wa", sizeof(int) * (gr->n + 1));
  if (!t->f.data.dg_wa) return delete t, eg.finish();
  fill_root<int>(t->f.data.dg_wa, -1, 0, root, gr->n);
  t->root_degree = root_deg(gr, root);
  ctx->stats.clean();
  executor_t &executor = ctx->executor;
  executor.insp = &t->inspector;
  executor.twod = twod_layout();
  t->plv0 = executor.persistent_levels;
  t->pln0 = executor.persistent_launches;
  feature_t &fets = t->fets;
  config_t &conf = t->conf;
  fets.centric = VC;
  fets.pattern = Idem;
  fets.fromall = false;
  fets.toall = false;
  conf.conf_pruning = true;
  apply_opts(o, conf);
  // standalone levels of the caller's variants: no fusion, no persistent launch
  conf.force.has_fusion = true;
  conf.force.fusion = Standalone;
  conf.conf_persistent = false;
  set_graph_features(fets, gr);
  fets.use_root = root;
  fets.first_active = 1;
  init_conf_impl(ctx->stats, fets, conf, t->g, t->f, gr->mean_weight, gr->attr[0], false, t->root_degree);
  t->as = ctx->aset(gr->n, conf.conf_qmode);
  if (!t->as) return delete t, eg.finish();
  t->as->reset();
  t->as->init(root);
  t->tr = loop_trace{&t->st, level_cap(gr->n)};
  if (!ok()) return delete t, eg.finish();
  *out = t;
  return eg.finish();
}

gsw_status gsw_level_begin(gsw_traversal *t, gsw_level_stats *out, int *done) {
  if (!t || !out || !done) return fail(GSW_ERR_INVALID_ARG, "gsw_level_begin: bad arguments");
  entry_guard eg(t->ctx);
  gsw_graph *gr = t->gr;
  memset(out, 0, sizeof(*out));
  out->nvertexs = gr->n;
  out->nedges = gr->m;
  for (int i = 0; i < 6; ++i) out->attr[i] = gr->attr[i];
  out->pattern = 0;
  out->level = t->g.level;
  if (t->done) {
    *done = 1;
    return eg.finish();
  }
  timer tm(t->ctx);
  stat_t &stats = t->ctx->stats;
  t->inspector.inspect(*t->as, t->g, t->f, stats, t->fets, t->conf);
  t->done = finish(*t->as, t->g, t->f, t->conf) ? 1 : 0;
  t->ms += tm.stop();
  if (t->first) {
    out->first_level = 1;
    out->active = 1;
    out->inactive = gr->n - 1;
    out->root_degree = t->root_degree;
    out->push_workload = t->root_degree;
    out->pull_workload = gr->m - t->root_degree;
  } else {
    out->active = (int64_t)stats.active_num();
    out->inactive = (int64_t)stats.unactive_num();
    out->push_workload = (int64_t)stats.push_workload();
    out->pull_workload = (int64_t)stats.pull_workload();
    out->max_push = (int64_t)stats.max_deg_active();
    out->max_pull = (int64_t)stats.max_deg_unactive();
  }
  t->inspected = 1;
  *done = t->done;
  return eg.finish();
}

gsw_status gsw_level_end(gsw_traversal *t, const gsw_level_choice *choice) {
  if (!t || !choice) return fail(GSW_ERR_INVALID_ARG, "gsw_level_end: bad arguments");
  entry_guard eg(t->ctx);
  if (t->done) return fail(GSW_ERR_INVALID_ARG, "gsw_level_end: the traversal is over");
  if (!t->inspected) return fail(GSW_ERR_INVALID_ARG, "gsw_level_end: call gsw_level_begin first");
  if ((choice->direction != GSW_PUSH && choice->direction != GSW_PULL) ||
      (choice->asfmt != GSW_QUEUE && choice->asfmt != GSW_BITMAP) ||
      !(choice->lb == GSW_LB_TM || choice->lb == GSW_LB_WM || choice->lb == GSW_LB_CM ||
        choice->lb == GSW_LB_STRICT || choice->lb == GSW_LB_TWC))
    return fail(GSW_ERR_INVALID_ARG, "gsw_level_end: bad choice (push/pull, queue/bitmap, TM/WM/CM/STRICT/TWC)");
  config_t &conf = t->conf;
  const auto force0 = conf.force;
  conf.conf_dir = choice->direction == GSW_PULL ? Pull : Push;
  conf.conf_asfmt = choice->asfmt == GSW_BITMAP ? Bitmap : Queue;
  conf.conf_lb = (LB)choice->lb;
  conf.conf_fuse_inspect = false;
  conf.conf_centric = VC;
  conf.conf_fromall = false;
  conf.conf_toall = false;
  selector_t::set_target(conf);
  conf.force.has_lb = true;  // the level runs the caller's load balance as given
  conf.force.lb = conf.conf_lb;
  executor_t &executor = t->ctx->executor;
  executor.insp = &t->inspector;
  stat_t &stats = t->ctx->stats;
  timer tm(t->ctx);
  executor.filter(*t->as, t->g, t->f, stats, t->fets, conf);
  t->g.update_level();
  t->tr.level(conf, hints().frontier);
  executor.expand(*t->as, t->g, t->f, stats, t->fets, conf);
  t->tr.done(stats, t->fets);
  t->done = finish(*t->as, t->g, t->f, conf) ? 1 : 0;
  t->ms += tm.stop();
  conf.force = force0;
  t->first = 0;
  t->inspected = 0;
  return eg.finish();
}

gsw_status gsw_traversal_end(gsw_traversal *t, int32_t *values, gsw_run_stats *st) {
  if (!t) return fail(GSW_ERR_INVALID_ARG, "gsw_traversal_end: NULL traversal");
  entry_guard eg(t->ctx);
  gsw_graph *gr = t->gr;
  t->tr.resolve();
  end_checks(t->as, &t->st);
  add_persistent_levels(&t->st, t->ctx->executor, t->plv0, t->pln0);
  t->st.ms = t->ms;
  t->st.edges = reached_edges(t->ctx, gr, t->f.data.dg_wa, 1, -1);
  if (values && ok())
    GSW_CUDA(cudaMemcpyAsync(values, t->f.data.dg_wa, sizeof(int) * gr->n, cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  if (st) *st = t->st;
  t->ctx->executor.insp = nullptr;
  delete t;
  return eg.finish();
}

// ---------------------------------------------------------------------------
// SSSP: application/sssp.cu:106-126 (loop) and :128-160 (set-up)
// ---------------------------------------------------------------------------
gsw_status gsw_sssp(gsw_ctx *ctx, gsw_graph *gr, int32_t root, const gsw_run_opts *o, int32_t *dist,
                    gsw_run_stats *st) {
  entry_guard eg(ctx);
  if (!ctx || !gr || root < 0 || root >= gr->n) return fail(GSW_ERR_INVALID_ARG, "gsw_sssp: bad arguments");
  if (!gr->weighted) return fail(GSW_ERR_INVALID_ARG, "gsw_sssp: graph has no weights");
  begin_stats(st);
  auto g = gr->view<int>();
  app::SSSP f;
  f.data.size = gr->n;
  f.data.dg_wa = (int *)ctx->buf("wa", sizeof(int) * (gr->n + 1));
  f.data.dg_ra = (int *)ctx->buf("ra", sizeof(int) * (gr->n + 1));
  if (!f.data.dg_wa || !f.data.dg_ra) return eg.finish();
  fill_root<int>(f.data.dg_wa, INT_MAX, 0, root, gr->n);
  fill_root<int>(f.data.dg_ra, INT_MAX, 0, root, gr->n);
  feature_t fets;
  config_t conf;
  stat_t &stats = ctx->stats;
  stats.clean();
  inspector_t inspector;
  selector_t selector;
  executor_t &executor = ctx->executor;
  executor.insp = &inspector;
  executor.twod = twod_layout();
  const int64_t plv0 = executor.persistent_levels, pln0 = executor.persistent_launches;
  fets.centric = VC;
  fets.pattern = Mono;
  fets.fromall = false;
  fets.toall = true;
  conf.conf_window = true;
  apply_opts(o, conf);
  set_graph_features(fets, gr);
  fets.use_root = root;
  init_conf_impl(stats, fets, conf, g, f, gr->mean_weight, gr->attr[0], false, root_deg(gr, root));
  mlp_fusion_override(ctx, o, fets, conf);
  active_set_t *asp = ctx->aset(gr->n, conf.conf_qmode);
  if (!asp) return eg.finish();
  active_set_t &as = *asp;
  as.reset();
  as.init(root);
  loop_trace tr{st, MAX_LEVELS};
  const bool captured = o && o->captured;
  dl_run R;
  if (captured && !dl_prepare(R, ctx, DL_APP_SSSP, dl_key() << f.data.dg_wa, as, g, f, conf, fets, 0, MAX_LEVELS,
                              o->selector))
    return eg.finish();
  timer tm(ctx);
  if (captured) dl_launch(R);
  for (int level = 0; !captured && ok(); level++) {
    inspector.inspect(as, g, f, stats, fets, conf);
    select_level(ctx, o, selector, stats, fets, conf);
    if (g_label) label_level(ctx, as, g, f, stats, fets, conf);
    executor.filter(as, g, f, stats, fets, conf);
    g.update_level();
    tr.level(conf, hints().frontier);
    executor.expand(as, g, f, stats, fets, conf);
    tr.done(stats, fets);
    if (finish(as, g, f, conf)) break;
  }
  const double ms = tm.stop();
  if (captured) dl_collect(R, st);
  tr.resolve();
  end_checks(&as, st);
  add_persistent_levels(st, executor, plv0, pln0);
  if (st) {
    st->ms = ms;
    st->edges = reached_edges(ctx, gr, f.data.dg_wa, 1, INT_MAX);
  }
  if (dist && ok()) GSW_CUDA(cudaMemcpyAsync(dist, f.data.dg_wa, sizeof(int) * gr->n, cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  return eg.finish();
}

// ---------------------------------------------------------------------------
// CC: application/cc.cu:263-289 (loop) and :291-311 (set-up)
// ---------------------------------------------------------------------------
__global__ void k_iota(int *p, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = (int)i;
}

// Captured CC: the edge-centric loop of application/cc.cu:82-108 as one CUDA
// graph.  WHILE { inspection of the active edges (k_inspect_ec); one thread
// reads the active count and stops, or picks the format the host loop picks
// (queue below 80% active, else bitmap: selector.cuh:22-76 for EC);
// SWITCH { queue: bitmap -> queue, hooking, pointer jumping | bitmap:
// hooking, pointer jumping } }.  The first iteration's inspection finds every
// edge active (labels start as vertex ids and no edge is a self-loop), which
// is what the host loop assumes for its first level without inspecting; the
// format rule is the host loop's (active edges over the vertex count, the
// bitmap at the first level).
struct cc_loop_t {
  unsigned long long *info;  // the inspection's active-edge counter
  long long nedges, nvertexs;
  int iter, iter_cap, status;  // status: dl_status_t
  int ntrace, trace_cap;
  int *trace_cfg;
  long long *trace_frontier;
  long long launches, per_queue, per_bitmap, per_inspect;
  cudaGraphConditionalHandle h_loop, h_body;
};

__global__ void k_cc_select(cc_loop_t *d) {
  cc_loop_t &s = *d;
  const unsigned long long a = *s.info;
  *s.info = 0;  // the next inspection counts from zero
  s.launches += s.per_inspect + 1;
  if (a == 0 || s.iter >= s.iter_cap) {
    s.status = a == 0 ? DL_DONE : DL_LEVEL_CAP;
    cudaGraphSetConditional(s.h_loop, 0);
    cudaGraphSetConditional(s.h_body, 2);  // no body
    return;
  }
  // the host loop's rule: active edges over the vertex count (the reference's
  // active_vertex_ratio of an edge-centric run), 1 at the first level
  const double ratio = s.iter == 0 ? 1.0 : (double)a / (double)s.nvertexs;
  const bool bitmap = ratio > 0.8;
  cudaGraphSetConditional(s.h_body, bitmap ? 1 : 0);
  s.launches += bitmap ? s.per_bitmap : s.per_queue;
  if (s.ntrace < s.trace_cap) {
    s.trace_cfg[s.ntrace] = (bitmap ? 1 : 0) << 1;
    s.trace_frontier[s.ntrace] = (long long)a;
  }
  s.ntrace++;
  s.iter++;
}

static bool cc_captured_run(gsw_ctx *ctx, device_graph_t<COO, Empty> g, app::CC f, active_set_t as, int iter_cap,
                            gsw_run_stats *st, double *ms_out) {
  executor_t &ex = ctx->executor;
  cc_loop_t *d = (cc_loop_t *)ctx->buf("cc_loop", sizeof(cc_loop_t));
  int *tcfg = (int *)ctx->buf("cc_trace_cfg", sizeof(int) * GSW_MAX_TRACE);
  long long *tfr = (long long *)ctx->buf("cc_trace_fr", sizeof(long long) * GSW_MAX_TRACE);
  unsigned long long *info = ctx->stats.dg_runtime_info;
  if (!d || !tcfg || !tfr || !info) return false;
  dl_key key;
  key << DL_APP_CC << d << g.dg_coo << g.nedges << g.nvertexs << f.data.dg_wa << as.size << as.bitmap.active.dg_bits
      << as.queue.subqueue[0].dg_queue << as.queue.subqueue[1].dg_queue << as.dg_cnt << as.workset.dg_bsum << info;
  dloop_graph &L = ctx->dl[DL_APP_CC];
  cc_loop_t im{};
  if (L.key != key.v || !L.exec) {
    L.destroy();
    cudaGraph_t top = nullptr;
    bool good = !GSW_CUDA(cudaGraphCreate(&top, 0));
    L.graph = top;
    cudaGraphConditionalHandle hl = 0, hb = 0;
    std::vector<cudaGraph_t> wbody, bodies;
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
    // queue form: the inspection's bitmap -> queue (into subqueue 1), then
    // the expand reads subqueue 1; bitmap form: the expand reads the bitmap
    active_set_t aq = as, ae = as, ab = as;
    aq.fmt = Queue;
    aq.queue.cursor = 0;
    ae.fmt = Queue;
    ae.queue.cursor = 1;
    ab.fmt = Bitmap;
    const long long launches0 = launch_count();
    if (good) {
      cudaGraph_t B = wbody[0];
      good = !GSW_CUDA(cudaGraphConditionalHandleCreate(&hb, B, 2, 0));
      if (good)
        good = dl_capture(B, [&] {
          k_inspect_ec<<<EC_INSPECT_CTAS, EC_INSPECT_THREADS, 0, stream()>>>(as, g, f, info);
          k_cc_select<<<1, 1, 0, stream()>>>(d);
          dl_add_conditional(stream(), hb, cudaGraphCondTypeSwitch, 2, bodies);
        });
      good = good && bodies.size() == 2;
    }
    if (good)
      good = dl_capture(bodies[0], [&] {
        ex.build_queue(aq, Active, true);
        ex.launch_ec(ae, g, f);
        p_jump(f, g.nvertexs, as);
      });
    if (good) {
      im.per_queue = dl_count_nodes(bodies[0]);
      good = dl_capture(bodies[1], [&] {
        ex.launch_ec(ab, g, f);
        p_jump(f, g.nvertexs, as);
      });
      im.per_bitmap = dl_count_nodes(bodies[1]);
    }
    launch_count() = launches0;
    if (good) good = !GSW_CUDA(cudaGraphInstantiate(&L.exec, top, 0));
    if (!good) {
      L.destroy();
      if (ok()) set_error(GSW_ERR_CUDA, "%s", "captured CC loop: graph construction failed");
      return false;
    }
    im.h_loop = hl;
    im.h_body = hb;
    L.image.h_loop = hl;
    L.image.h_expand = hb;
    L.image.expand_kernels[0] = (int)im.per_queue;
    L.image.expand_kernels[1] = (int)im.per_bitmap;
    L.key = key.v;
  } else {
    im.h_loop = L.image.h_loop;
    im.h_body = L.image.h_expand;
    im.per_queue = L.image.expand_kernels[0];
    im.per_bitmap = L.image.expand_kernels[1];
  }
  im.info = info;
  im.nedges = g.nedges;
  im.nvertexs = g.nvertexs;
  im.iter_cap = iter_cap;
  im.status = DL_RUNNING;
  im.trace_cap = GSW_MAX_TRACE;
  im.trace_cfg = tcfg;
  im.trace_frontier = tfr;
  im.per_inspect = 1;
  GSW_CUDA(cudaMemsetAsync(info, 0, sizeof(unsigned long long), stream()));
  timer tm(ctx);
  GSW_CUDA(cudaMemcpyAsync(d, &im, sizeof(im), cudaMemcpyHostToDevice, stream()));
  GSW_CUDA(cudaGraphLaunch(L.exec, stream()));
  *ms_out = tm.stop();
  cc_loop_t out;
  if (GSW_CUDA(cudaMemcpyAsync(&out, d, sizeof(out), cudaMemcpyDeviceToHost, stream()))) return false;
  if (GSW_CUDA(cudaStreamSynchronize(stream()))) return false;
  launch_count() += out.launches;
  if (out.status == DL_LEVEL_CAP) set_error(GSW_ERR_TIMEOUT, "%s", "level loop did not converge within the level cap");
  else if (out.status != DL_DONE) set_error(GSW_ERR_CUDA, "%s", "captured CC loop did not finish");
  if (st) {
    st->levels = out.iter;
    const int nt = std::min(out.ntrace, (int)GSW_MAX_TRACE);
    st->ntrace = nt;
    std::vector<int> cfg(nt);
    std::vector<long long> fr(nt);
    if (nt > 0) {
      GSW_CUDA(cudaMemcpyAsync(cfg.data(), tcfg, sizeof(int) * nt, cudaMemcpyDeviceToHost, stream()));
      GSW_CUDA(cudaMemcpyAsync(fr.data(), tfr, sizeof(long long) * nt, cudaMemcpyDeviceToHost, stream()));
      GSW_CUDA(cudaStreamSynchronize(stream()));
    }
    for (int i = 0; i < nt; ++i) {
      st->level_cfg[i] = cfg[i];
      st->level_frontier[i] = fr[i];
      st->level_ms[i] = st->level_inspect_ms[i] = 0;
      st->level_edges[i] = -1;
    }
  }
  return ok();
}

gsw_status gsw_cc(gsw_ctx *ctx, gsw_graph *gr, const gsw_run_opts *o, int32_t *labels, gsw_run_stats *st) {
  entry_guard eg(ctx);
  if (!ctx || !gr) return fail(GSW_ERR_INVALID_ARG, "gsw_cc: bad arguments");
  begin_stats(st);
  if (ensure_coo(gr)) return eg.finish();
  device_graph_t<COO, Empty> g;
  g.dg_coo = gr->coo;
  g.dg_edgedata = nullptr;
  g.nvertexs = (int)gr->n;
  g.nedges = gr->ncoo;
  g.level = 0;
  app::CC f;
  f.data.size = gr->n;
  f.data.dg_wa = (int *)ctx->buf("wa", sizeof(int) * (gr->n + 1));
  if (!f.data.dg_wa) return eg.finish();
  k_iota<<<grid_for(gr->n), 256, 0, stream()>>>(f.data.dg_wa, gr->n);
  feature_t fets;
  config_t conf;
  stat_t &stats = ctx->stats;
  stats.clean();
  inspector_t inspector;
  selector_t selector;
  executor_t &executor = ctx->executor;
  executor.insp = &inspector;
  executor.twod = twod_layout();
  const int64_t plv0 = executor.persistent_levels, pln0 = executor.persistent_launches;
  fets.centric = EC;
  fets.pattern = ASSO;
  apply_opts(o, conf);
  set_graph_features(fets, gr);
  init_conf_impl(stats, fets, conf, g, f, 0.0, gr->attr[0], false);
  active_set_t *asp = ctx->aset(std::max<int64_t>(gr->ncoo, 1), conf.conf_qmode);
  if (!asp) return eg.finish();
  active_set_t &as = *asp;
  as.reset();
  as.init(ALL_ACTIVE);
  if (o && o->captured) {
    double ms = 0;
    if (gr->ncoo > 0) cc_captured_run(ctx, g, f, as, MAX_LEVELS, st, &ms);
    end_checks(&as, st);
    if (st) {
      st->ms = ms;
      st->edges = gr->ncoo;
    }
    if (labels && ok())
      GSW_CUDA(cudaMemcpyAsync(labels, f.data.dg_wa, sizeof(int) * gr->n, cudaMemcpyDeviceToHost, stream()));
    GSW_CUDA(cudaStreamSynchronize(stream()));
    return eg.finish();
  }
  loop_trace tr{st, MAX_LEVELS};
  timer tm(ctx);
  for (int level = 0; ok() && gr->ncoo > 0; level++) {
    inspector.inspect(as, g, f, stats, fets, conf);
    if (finish(as, g, f, conf)) break;
    selector.select(stats, fets, conf);
    executor.filter(as, g, f, stats, fets, conf);
    g.update_level();
    tr.level(conf, hints().frontier);
    executor.expand(as, g, f, stats, fets, conf);
    tr.done(stats, fets);
    p_jump(f, gr->n, as);
    if (finish(as, g, f, conf)) break;
  }
  const double ms = tm.stop();
  tr.resolve();
  end_checks(&as, st);
  add_persistent_levels(st, executor, plv0, pln0);
  if (st) {
    st->ms = ms;
    st->edges = gr->ncoo;
  }
  if (labels && ok())
    GSW_CUDA(cudaMemcpyAsync(labels, f.data.dg_wa, sizeof(int) * gr->n, cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  return eg.finish();
}

// ---------------------------------------------------------------------------
// PageRank: application/pagerank.cu:81-103 (loop) and :105-131 (set-up).
// max_iters > 0 stops after exactly that many Jacobi steps (the filter of
// inspection k computes pr_k); eps keeps the reference's convergence test.
// ---------------------------------------------------------------------------
__global__ void k_pr_init(const int *odeg, int64_t n, float damp, float *ra) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
    ra[v] = odeg[v] ? (1 - damp) / odeg[v] : (1 - damp);
}

gsw_status gsw_pagerank(gsw_ctx *ctx, gsw_graph *gr, const gsw_run_opts *o, float *pr_over_od, gsw_run_stats *st) {
  entry_guard eg(ctx);
  if (!ctx || !gr) return fail(GSW_ERR_INVALID_ARG, "gsw_pagerank: bad arguments");
  begin_stats(st);
  gsw_run_opts def;
  gsw_run_opts_default(&def);
  const gsw_run_opts *op = o ? o : &def;
  auto g = gr->view<Empty>();
  app::PR f;
  f.damp = op->damping;
  f.eps = op->eps;
  f.data.size = gr->n;
  f.data.dg_wa = (float *)ctx->buf("wa", sizeof(float) * (gr->n + 1));
  f.data.dg_ra = (float *)ctx->buf("ra", sizeof(float) * (gr->n + 1));
  if (!f.data.dg_wa || !f.data.dg_ra) return eg.finish();
  fill<float>(f.data.dg_wa, 0.0f, gr->n);
  k_pr_init<<<grid_for(gr->n), 256, 0, stream()>>>(gr->odeg, gr->n, f.damp, f.data.dg_ra);
  f.data.zero = 0.0f;
  feature_t fets;
  config_t conf;
  stat_t &stats = ctx->stats;
  stats.clean();
  inspector_t inspector;
  selector_t selector;
  executor_t &executor = ctx->executor;
  executor.insp = &inspector;
  executor.twod = twod_layout();
  const int64_t plv0 = executor.persistent_levels, pln0 = executor.persistent_launches;
  fets.centric = VC;
  fets.pattern = ASSO;
  fets.fromall = true;
  fets.toall = true;
  apply_opts(op, conf);
  if (conf.force.has_lb && conf.force.lb == TWOD) {
    if (ensure_twod(gr)) return eg.finish();
    executor.twod = gr->twod->L;
  }
  set_graph_features(fets, gr);
  init_conf_impl(stats, fets, conf, g, f, 0.0, gr->attr[0], false);
  active_set_t *asp = ctx->aset(gr->n, conf.conf_qmode);
  if (!asp) return eg.finish();
  active_set_t &as = *asp;
  as.reset();
  as.init(ALL_ACTIVE);
  loop_trace tr{st, MAX_LEVELS};
  const bool captured = op->captured != 0;
  dl_run R;
  if (captured && !dl_prepare(R, ctx, DL_APP_PR,
                              dl_key() << f.data.dg_wa << f.data.dg_ra << f.damp << f.eps << f.data.zero, as, g, f,
                              conf, fets, op->max_iters, MAX_LEVELS, op->selector))
    return eg.finish();
  timer tm(ctx);
  int steps = 0;
  if (captured) dl_launch(R);
  for (int level = 0; !captured && ok(); level++) {
    inspector.inspect(as, g, f, stats, fets, conf);
    if (op->max_iters > 0 && level == op->max_iters) break;
    if (finish(as, g, f, conf)) break;
    select_level(ctx, op, selector, stats, fets, conf);
    if (g_label) label_level(ctx, as, g, f, stats, fets, conf);
    executor.filter(as, g, f, stats, fets, conf);
    g.update_level();
    tr.level(conf, hints().frontier);
    executor.expand(as, g, f, stats, fets, conf);
    tr.done(stats, fets);
    steps++;
    if (finish(as, g, f, conf)) break;
  }
  const double ms = tm.stop();
  if (captured) {
    gsw_run_stats tmp;
    dl_collect(R, st ? st : &tmp);
    steps = st ? st->levels : tmp.levels;
  }
  tr.resolve();
  end_checks(&as, st);
  add_persistent_levels(st, executor, plv0, pln0);
  if (st) {
    st->ms = ms;
    st->edges = gr->m * (int64_t)steps;
  }
  if (pr_over_od && ok())
    GSW_CUDA(cudaMemcpyAsync(pr_over_od, f.data.dg_ra, sizeof(float) * gr->n, cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  return eg.finish();
}

// ---------------------------------------------------------------------------
// Delta-PageRank (docs/index.md:178 of the reference describes it; its code
// has none): the PageRank level loop above with the PRDelta functor.  Level 0
// has every vertex send (1-d) worth of value; afterwards only vertices whose
// accumulated change passed the threshold send.  The loop ends when no
// vertex is active (or after max_iters levels when that is positive).
// edges = out-edges of the vertices that sent, summed over levels.
// ---------------------------------------------------------------------------
__global__ void k_prd_init(const int *odeg, int64_t n, float damp, float *pr, float *ra, float *wa) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    pr[v] = 1 - damp;
    ra[v] = odeg[v] ? damp * (1 - damp) / odeg[v] : 0.0f;
    wa[v] = 0.0f;
  }
}

gsw_status gsw_pagerank_delta(gsw_ctx *ctx, gsw_graph *gr, const gsw_run_opts *o, float *pr, gsw_run_stats *st) {
  entry_guard eg(ctx);
  if (!ctx || !gr) return fail(GSW_ERR_INVALID_ARG, "gsw_pagerank_delta: bad arguments");
  begin_stats(st);
  gsw_run_opts def;
  gsw_run_opts_default(&def);
  const gsw_run_opts *op = o ? o : &def;
  if (op->eps <= 0 || op->damping <= 0 || op->damping >= 1)
    return fail(GSW_ERR_INVALID_ARG, "gsw_pagerank_delta: need eps > 0 and 0 < damping < 1");
  auto g = gr->view<Empty>();
  app::PRDelta f;
  f.damp = op->damping;
  f.eps = op->eps;
  f.data.size = gr->n;
  f.data.dg_wa = (float *)ctx->buf("wa", sizeof(float) * (gr->n + 1));
  f.data.dg_ra = (float *)ctx->buf("ra", sizeof(float) * (gr->n + 1));
  f.pr = (float *)ctx->buf("prd", sizeof(float) * (gr->n + 1));
  if (!f.data.dg_wa || !f.data.dg_ra || !f.pr) return eg.finish();
  k_prd_init<<<grid_for(gr->n), 256, 0, stream()>>>(gr->odeg, gr->n, f.damp, f.pr, f.data.dg_ra, f.data.dg_wa);
  f.data.zero = 0.0f;
  feature_t fets;
  config_t conf;
  stat_t &stats = ctx->stats;
  stats.clean();
  inspector_t inspector;
  selector_t selector;
  executor_t &executor = ctx->executor;
  executor.insp = &inspector;
  executor.twod = twod_layout();
  const int64_t plv0 = executor.persistent_levels, pln0 = executor.persistent_launches;
  fets.centric = VC;
  fets.pattern = ASSO;
  fets.fromall = false;
  fets.toall = true;
  apply_opts(op, conf);
  // Standalone levels only: a fused level enqueues the targets whose update
  // reports success, but here a vertex becomes active only once everything a
  // level sent it has been summed, which the inspection's filter pass sees
  if (conf.force.has_fusion && conf.force.fusion == Fused)
    return fail(GSW_ERR_UNSUPPORTED, "gsw_pagerank_delta: standalone levels only");
  conf.force.has_fusion = true;
  conf.force.fusion = Standalone;
  set_graph_features(fets, gr);
  init_conf_impl(stats, fets, conf, g, f, 0.0, gr->attr[0], false);
  active_set_t *asp = ctx->aset(gr->n, conf.conf_qmode);
  if (!asp) return eg.finish();
  active_set_t &as = *asp;
  as.reset();
  as.init(ALL_ACTIVE);
  loop_trace tr{st, MAX_LEVELS};
  const int cap = op->max_iters > 0 ? op->max_iters : MAX_LEVELS;
  int64_t work = 0;
  // captured: the loop stops at `cap` iterations after that iteration's
  // inspection, as here, and sums the push workload of the levels it ran
  const bool captured = op->captured != 0;
  dl_run R;
  if (captured && !dl_prepare(R, ctx, DL_APP_PRD, dl_key() << f.data.dg_wa << f.pr << f.damp << f.eps, as, g, f,
                              conf, fets, cap, cap + 1, op->selector))
    return eg.finish();
  timer tm(ctx);
  if (captured) dl_launch(R);
  for (int level = 0; !captured && ok(); level++) {
    const bool inspected = level > 0 && !conf.conf_fuse_inspect;
    inspector.inspect(as, g, f, stats, fets, conf);
    if (level == cap) break;
    if (finish(as, g, f, conf)) break;
    work += level == 0 ? gr->m : (inspected ? stats.push_workload() : 0);
    select_level(ctx, op, selector, stats, fets, conf);
    executor.filter(as, g, f, stats, fets, conf);
    g.update_level();
    tr.level(conf, hints().frontier);
    executor.expand(as, g, f, stats, fets, conf);
    tr.done(stats, fets);
  }
  const double ms = tm.stop();
  if (captured) {
    dl_collect(R, st);
    work = gr->m + (int64_t)R.push_sum;  // the first level sends along every arc
  }
  tr.resolve();
  end_checks(&as, st);
  add_persistent_levels(st, executor, plv0, pln0);
  if (st) {
    st->ms = ms;
    st->edges = work;
  }
  if (pr && ok()) GSW_CUDA(cudaMemcpyAsync(pr, f.pr, sizeof(float) * gr->n, cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  return eg.finish();
}

// ---------------------------------------------------------------------------
// BC: application/bc.cu:246-309 (both phases) and :391-431 (set-up).  The
// cached queue that replays the forward levels backwards is kept for every
// start (the reference drops to a Normal queue when its fusion tree picks the
// standalone form, which leaves the deepest level's dependencies unpushed).
// ---------------------------------------------------------------------------
__global__ void k_bc_init(app::fwdata_t *wa, int64_t n, int64_t root) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    wa[i] = i == root ? app::fwdata_t{0, 1} : app::fwdata_t{-100, 0};
}
__global__ void k_bc_handoff(const app::fwdata_t *fw, int64_t n, int *lvl, app::bwdata_t *bw) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    lvl[i] = fw[i].level;
    bw[i] = app::bwdata_t{fw[i].nsp, 0.0f};
  }
}
__global__ void k_bc_split(const app::bwdata_t *bw, int64_t n, int *nsp, float *dep) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    nsp[i] = bw[i].nsp;
    dep[i] = bw[i].dep;
  }
}

__global__ void k_max_int(const int *a, int64_t n, int *out) {
  int m = INT_MIN;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    m = a[i] > m ? a[i] : m;
  m = warp_max(m);
  if (lane_id() == 0) atomicMax(out, m);
}

int max_level(gsw_ctx *ctx, const int *a, int64_t n) {
  int *d = (int *)ctx->buf("maxlvl", sizeof(int));
  if (!d) return 0;
  const int init = INT_MIN;
  GSW_CUDA(cudaMemcpyAsync(d, &init, sizeof(int), cudaMemcpyHostToDevice, stream()));
  k_max_int<<<grid_for(n), 256, 0, stream()>>>(a, n, d);
  int r = 0;
  GSW_CUDA(cudaMemcpyAsync(&r, d, sizeof(int), cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  return r;
}

gsw_status gsw_bc(gsw_ctx *ctx, gsw_graph *gr, int32_t root, const gsw_run_opts *o, int32_t *nsp, float *dep,
                  gsw_run_stats *st) {
  entry_guard eg(ctx);
  if (!ctx || !gr || root < 0 || root >= gr->n) return fail(GSW_ERR_INVALID_ARG, "gsw_bc: bad arguments");
  if (o && o->captured) return fail(GSW_ERR_UNSUPPORTED, "gsw_bc: no captured level loop");
  begin_stats(st);
  auto g = gr->view<Empty>();
  app::BCForward f;
  app::BCBackward h;
  f.data.size = h.data.size = gr->n;
  f.data.dg_wa = (app::fwdata_t *)ctx->buf("wa", sizeof(app::fwdata_t) * (gr->n + 1));
  h.data.dg_wa = (app::bwdata_t *)ctx->buf("wa2", sizeof(app::bwdata_t) * (gr->n + 1));
  h.data.dg_ra = (int *)ctx->buf("ra", sizeof(int) * (gr->n + 1));
  if (!f.data.dg_wa || !h.data.dg_wa || !h.data.dg_ra) return eg.finish();
  k_bc_init<<<grid_for(gr->n), 256, 0, stream()>>>(f.data.dg_wa, gr->n, root);
  feature_t fets;
  config_t conf;
  stat_t &stats = ctx->stats;
  stats.clean();
  inspector_t inspector;
  selector_t selector;
  executor_t &executor = ctx->executor;
  executor.insp = &inspector;
  executor.twod = twod_layout();
  const int64_t plv0 = executor.persistent_levels, pln0 = executor.persistent_launches;
  fets.centric = VC;
  fets.pattern = ASSO;
  fets.fromall = false;
  fets.toall = false;
  conf.conf_fuse_inspect = false;
  conf.conf_qmode = Cached;
  apply_opts(o, conf);
  set_graph_features(fets, gr);
  fets.use_root = root;
  init_conf_impl(stats, fets, conf, g, f, 0.0, gr->attr[0], false, root_deg(gr, root));
  // The backward sweep replays the forward frontiers from the cached queue
  // only when every forward level enqueued its frontier, i.e. when the levels
  // run fused (always Push + Queue).  Otherwise each backward level inspects
  // the forward levels instead, which holds for every direction and format.
  const bool replay = conf.conf_fusion;
  conf.conf_qmode = replay ? Cached : Normal;
  active_set_t *asp = ctx->aset(gr->n, conf.conf_qmode);
  if (!asp) return eg.finish();
  active_set_t &as = *asp;
  as.reset();
  as.init(root);
  loop_trace tr{st, MAX_LEVELS};
  timer tm(ctx);
  for (int level = 0; ok(); level++) {
    inspector.inspect(as, g, f, stats, fets, conf);
    if (finish(as, g, f, conf)) break;
    selector.select(stats, fets, conf);
    executor.filter(as, g, f, stats, fets, conf);
    g.update_level();
    tr.level(conf, hints().frontier);
    executor.expand(as, g, f, stats, fets, conf);
    tr.done(stats, fets);
    if (finish(as, g, f, conf)) break;
  }
  const int64_t fwd_edges = st ? reached_edges(ctx, gr, (const int *)f.data.dg_wa, 2, -100) : 0;
  // hand-off (bc.cu:391-395); the sweep starts at the deepest forward level
  k_bc_handoff<<<grid_for(gr->n), 256, 0, stream()>>>(f.data.dg_wa, gr->n, h.data.dg_ra, h.data.dg_wa);
  const int lmax = max_level(ctx, h.data.dg_ra, gr->n);
  as.reset(replay);
  conf.reset();
  stats.reset();
  conf.conf_compensation = true;
  g.level = lmax;
  if (!replay) conf.conf_first_round = false;  // inspect the deepest level too
  as.init(ALL_INACTIVE);
  for (int level = 0; ok(); level++) {
    inspector.inspect(as, g, h, stats, fets, conf);
    if (finish(as, g, h, conf)) break;
    selector.select(stats, fets, conf);
    executor.filter(as, g, h, stats, fets, conf);
    g.update_level(-1);
    tr.level(conf, hints().frontier);
    executor.expand(as, g, h, stats, fets, conf);
    tr.done(stats, fets);
    if (finish(as, g, h, conf)) break;
  }
  const double ms = tm.stop();
  tr.resolve();
  end_checks(&as, st);
  add_persistent_levels(st, executor, plv0, pln0);
  if (st) {
    st->ms = ms;
    st->edges = fwd_edges;
  }
  if ((nsp || dep) && ok()) {
    int *dn = (int *)ctx->buf("bc_nsp", sizeof(int) * (gr->n + 1));
    float *dd = (float *)ctx->buf("bc_dep", sizeof(float) * (gr->n + 1));
    if (dn && dd) {
      k_bc_split<<<grid_for(gr->n), 256, 0, stream()>>>(h.data.dg_wa, gr->n, dn, dd);
      if (nsp) GSW_CUDA(cudaMemcpyAsync(nsp, dn, sizeof(int) * gr->n, cudaMemcpyDeviceToHost, stream()));
      if (dep) GSW_CUDA(cudaMemcpyAsync(dep, dd, sizeof(float) * gr->n, cudaMemcpyDeviceToHost, stream()));
    }
  }
  GSW_CUDA(cudaStreamSynchronize(stream()));
  return eg.finish();
}

// ---------------------------------------------------------------------------
// GC: application/gc.cu:76-99 (loop) and :101-122 (set-up)
// ---------------------------------------------------------------------------
gsw_status gsw_gc(gsw_ctx *ctx, gsw_graph *gr, const gsw_run_opts *o, int32_t *colors, gsw_run_stats *st) {
  entry_guard eg(ctx);
  if (!ctx || !gr) return fail(GSW_ERR_INVALID_ARG, "gsw_gc: bad arguments");
  begin_stats(st);
  auto g = gr->view<Empty>();
  app::GC f;
  f.data.size = gr->n;
  f.data.dg_wa = (int *)ctx->buf("wa", sizeof(int) * (gr->n + 1));
  f.data.dg_ra = (int *)ctx->buf("ra", sizeof(int) * (gr->n + 1));
  if (!f.data.dg_wa || !f.data.dg_ra) return eg.finish();
  fill<int>(f.data.dg_wa, -1, gr->n);
  fill<int>(f.data.dg_ra, -1, gr->n);
  f.data.set_zero(-1);  // identity of the max the colouring accumulates
  feature_t fets;
  config_t conf;
  stat_t &stats = ctx->stats;
  stats.clean();
  inspector_t inspector;
  selector_t selector;
  executor_t &executor = ctx->executor;
  executor.insp = &inspector;
  executor.twod = twod_layout();
  const int64_t plv0 = executor.persistent_levels, pln0 = executor.persistent_launches;
  fets.centric = VC;
  fets.pattern = ASSO;
  fets.fromall = true;
  fets.toall = true;
  conf.conf_fixed = true;
  apply_opts(o, conf);
  if (conf.force.has_lb && conf.force.lb == TWOD) {
    if (ensure_twod(gr)) return eg.finish();
    executor.twod = gr->twod->L;
  }
  set_graph_features(fets, gr);
  init_conf_impl(stats, fets, conf, g, f, 0.0, gr->attr[0], false);
  active_set_t *asp = ctx->aset(gr->n, conf.conf_qmode);
  if (!asp) return eg.finish();
  active_set_t &as = *asp;
  as.reset();
  as.init(ALL_ACTIVE);
  loop_trace tr{st, MAX_LEVELS};
  // captured: the rule trees decide on the device, as selector.select does here
  const bool captured = o && o->captured;
  dl_run R;
  if (captured && !dl_prepare(R, ctx, DL_APP_GC, dl_key() << f.data.dg_wa, as, g, f, conf, fets, 0, MAX_LEVELS,
                              GSW_SELECT_RULES))
    return eg.finish();
  timer tm(ctx);
  if (captured) dl_launch(R);
  for (int level = 0; !captured && ok(); level++) {
    inspector.inspect(as, g, f, stats, fets, conf);
    if (finish(as, g, f, conf)) break;
    selector.select(stats, fets, conf);
    executor.filter(as, g, f, stats, fets, conf);
    g.update_level();
    tr.level(conf, hints().frontier);
    executor.expand(as, g, f, stats, fets, conf);
    tr.done(stats, fets);
    if (finish(as, g, f, conf)) break;
  }
  const double ms = tm.stop();
  if (captured) dl_collect(R, st);
  tr.resolve();
  end_checks(&as, st);
  add_persistent_levels(st, executor, plv0, pln0);
  if (st) {
    st->ms = ms;
    st->edges = gr->m / 2;
  }
  if (colors && ok())
    GSW_CUDA(cudaMemcpyAsync(colors, f.data.dg_ra, sizeof(int) * gr->n, cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  return eg.finish();
}

// ---------------------------------------------------------------------------
// MBFS: application/mbfs.cu:222-297 runs the single-source loop per source;
// the batched form runs 64 sources per bit-sliced word (mbfs.cuh).
// ---------------------------------------------------------------------------
gsw_status gsw_mbfs(gsw_ctx *ctx, gsw_graph *gr, int nsrc, const int32_t *roots, int batched, const gsw_run_opts *o,
                    int32_t *levels, gsw_run_stats *st) {
  entry_guard eg(ctx);
  if (!ctx || !gr || nsrc <= 0 || !roots) return fail(GSW_ERR_INVALID_ARG, "gsw_mbfs: bad arguments");
  if (o && o->captured) return fail(GSW_ERR_UNSUPPORTED, "gsw_mbfs: no captured level loop");
  for (int s = 0; s < nsrc; ++s)
    if (roots[s] < 0 || roots[s] >= gr->n) return fail(GSW_ERR_INVALID_ARG, "gsw_mbfs: root out of range");
  if (!batched) {
    double tot = 0;
    int64_t edges = 0;
    int lv = 0;
    gsw_run_stats one;
    for (int s = 0; s < nsrc; ++s) {
      gsw_status r = gsw_bfs(ctx, gr, roots[s], o, levels ? levels + (int64_t)s * gr->n : nullptr, &one);
      if (r) return r;
      tot += one.ms;
      edges += one.edges;
      lv += one.levels;
    }
    if (st) {
      begin_stats(st);
      st->ms = tot;
      st->edges = edges;
      st->levels = lv;
    }
    return GSW_OK;
  }
  begin_stats(st);
  // every level in one cooperative launch unless the options turn persistent
  // launches off
  const bool persistent = !o || o->persistent != 0;
  mbfs_result r = run_mbfs_batched(
      gr->view<Empty>(), nsrc, roots, [&](const char *name, size_t bytes) { return ctx->buf(name, bytes); }, levels,
      persistent);
  if (st && ok()) {
    st->ms = r.ms;
    st->levels = r.levels;
    st->edges = r.edges;
  }
  return eg.finish();
}

// ---------------------------------------------------------------------------
// batched BC (bc_batch.cuh): the sources in batches of BCB_SOURCES
// ---------------------------------------------------------------------------
gsw_status gsw_bc_batch(gsw_ctx *ctx, gsw_graph *gr, int nsrc, const int32_t *roots, const gsw_run_opts *o,
                        int32_t *nsp, float *dep, gsw_run_stats *st) {
  entry_guard eg(ctx);
  if (!ctx || !gr || nsrc <= 0 || !roots) return fail(GSW_ERR_INVALID_ARG, "gsw_bc_batch: bad arguments");
  if (o && o->captured) return fail(GSW_ERR_UNSUPPORTED, "gsw_bc_batch: no captured level loop");
  if (gr->directed) return fail(GSW_ERR_UNSUPPORTED, "gsw_bc_batch: undirected graphs only");
  for (int s = 0; s < nsrc; ++s)
    if (roots[s] < 0 || roots[s] >= gr->n) return fail(GSW_ERR_INVALID_ARG, "gsw_bc_batch: root out of range");
  begin_stats(st);
  double ms = 0;
  int64_t edges = 0;
  int levels = 0;
  auto buf = [&](const char *name, size_t bytes) { return ctx->buf(name, bytes); };
  for (int s0 = 0; s0 < nsrc && ok(); s0 += BCB_SOURCES) {
    const int k = std::min(BCB_SOURCES, nsrc - s0);
    const size_t row = (size_t)gr->n;
    bcb_result r = bc_batch_run(gr->view<Empty>(), k, roots + s0, buf, nsp ? nsp + row * s0 : nullptr,
                                dep ? dep + row * s0 : nullptr, !o || o->persistent != 0);
    ms += r.ms;
    edges += r.edges;
    levels = std::max(levels, r.levels);
  }
  if (st && ok()) {
    st->ms = ms;
    st->edges = edges;
    st->levels = levels;
    st->launches = launch_count();
  }
  return eg.finish();
}

// ---------------------------------------------------------------------------
// learned selector: labels, training, inference, loading (engine/mlp.cuh)
// ---------------------------------------------------------------------------
gsw_status gsw_label_levels(gsw_ctx *ctx, gsw_graph *gr, int app, int32_t root, int max_levels, int pr_iters,
                            float *features, float *times_ms, int32_t *rule_class, int *nlevels) {
  if (!ctx || !gr || max_levels <= 0 || !features || !times_ms || app < 0 || app > 2)
    return fail(GSW_ERR_INVALID_ARG, "gsw_label_levels: bad arguments");
  label_sink L;
  L.max_levels = max_levels;
  L.X = features;
  L.T = times_ms;
  L.R = rule_class;
  if (app == GSW_APP_PR) {
    L.first = pr_iters > 0 ? pr_iters : 3;
    L.level_limit = L.first;
  }
  gsw_run_opts o;
  gsw_run_opts_default(&o);
  o.fusion = GSW_STANDALONE;
  o.persistent = 0;
  g_label = &L;
  gsw_status r;
  if (app == GSW_APP_BFS) {
    r = gsw_bfs(ctx, gr, root, &o, nullptr, nullptr);
  } else if (app == GSW_APP_SSSP) {
    r = gsw_sssp(ctx, gr, root, &o, nullptr, nullptr);
  } else {
    o.max_iters = L.first;
    o.eps = 0.0f;
    r = gsw_pagerank(ctx, gr, &o, nullptr, nullptr);
  }
  g_label = nullptr;
  if (nlevels) *nlevels = L.rows;
  return r;
}

namespace {
// model floats (parameters, means, inverse deviations) -> device mlp_model
mlp_model model_from_floats(const float *m, float min_conf) {
  mlp_model h;
  memcpy(h.p, m, sizeof(float) * MLP_NPARAM);
  memcpy(h.mean, m + MLP_NPARAM, sizeof(float) * MLP_IN);
  memcpy(h.inv_std, m + MLP_NPARAM + MLP_IN, sizeof(float) * MLP_IN);
  h.min_conf = min_conf;
  h.valid = 1;
  return h;
}
}  // namespace

gsw_status gsw_mlp_grad(gsw_ctx *ctx, const float *model, const float *X, const float *T, int64_t n, float tau,
                        float *grad, float *loss) {
  entry_guard eg(ctx);
  if (!ctx || !model || !X || !T || n <= 0 || !grad || !(tau > 0)) return fail(GSW_ERR_INVALID_ARG, "gsw_mlp_grad: bad arguments");
  float *d = (float *)ctx->buf("mlp_work", sizeof(float) * (MLP_NPARAM * 2 + 2 * MLP_IN + 8));
  float *dX = (float *)ctx->buf("mlp_X", sizeof(float) * n * MLP_IN);
  float *dT = (float *)ctx->buf("mlp_T", sizeof(float) * n * MLP_K);
  float *dQ = (float *)ctx->buf("mlp_Q", sizeof(float) * n * MLP_K);
  if (!d || !dX || !dT || !dQ) return eg.finish();
  float *dP = d, *dG = d + MLP_NPARAM, *dmean = dG + MLP_NPARAM, *dinv = dmean + MLP_IN, *dloss = dinv + MLP_IN;
  GSW_CUDA(cudaMemcpyAsync(dP, model, sizeof(float) * (MLP_NPARAM), cudaMemcpyHostToDevice, stream()));
  GSW_CUDA(cudaMemcpyAsync(dmean, model + MLP_NPARAM, sizeof(float) * 2 * MLP_IN, cudaMemcpyHostToDevice, stream()));
  GSW_CUDA(cudaMemcpyAsync(dX, X, sizeof(float) * n * MLP_IN, cudaMemcpyHostToDevice, stream()));
  GSW_CUDA(cudaMemcpyAsync(dT, T, sizeof(float) * n * MLP_K, cudaMemcpyHostToDevice, stream()));
  GSW_CUDA(cudaMemsetAsync(dG, 0, sizeof(float) * MLP_NPARAM, stream()));
  GSW_CUDA(cudaMemsetAsync(dloss, 0, sizeof(float), stream()));
  k_mlp_soft_labels<<<grid_for(n), 256, 0, stream()>>>(dT, n, tau, dQ);
  const int gb = (int)std::min<int64_t>((n + MLP_TRAIN_THREADS - 1) / MLP_TRAIN_THREADS, 2 * sm_count());
  k_mlp_grad<<<gb, MLP_TRAIN_THREADS, 0, stream()>>>(dP, dmean, dinv, dX, dQ, n, dG, dloss);
  GSW_LAUNCHED();
  GSW_CUDA(cudaMemcpyAsync(grad, dG, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost, stream()));
  if (loss) GSW_CUDA(cudaMemcpyAsync(loss, dloss, sizeof(float), cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  return eg.finish();
}

gsw_status gsw_mlp_train(gsw_ctx *ctx, const float *X, const float *T, int64_t n, int epochs, float lr, float tau,
                         uint64_t seed, float *model_out, float *loss_out) {
  entry_guard eg(ctx);
  if (!ctx || !X || !T || n <= 0 || epochs <= 0 || !model_out || !(lr > 0) || !(tau > 0))
    return fail(GSW_ERR_INVALID_ARG, "gsw_mlp_train: bad arguments");
  // feature normalisation of this corpus (host, FP64)
  std::vector<float> model(MLP_NPARAM + 2 * MLP_IN, 0.f);
  for (int j = 0; j < MLP_IN; ++j) {
    double s = 0, s2 = 0;
    for (int64_t i = 0; i < n; ++i) {
      s += X[i * MLP_IN + j];
      s2 += (double)X[i * MLP_IN + j] * X[i * MLP_IN + j];
    }
    const double mu = s / n, var = std::max(s2 / n - mu * mu, 0.0);
    model[MLP_NPARAM + j] = (float)mu;
    model[MLP_NPARAM + MLP_IN + j] = (float)(1.0 / std::sqrt(var + 1e-6));
  }
  // He-uniform initial weights from the seed, zero biases
  auto init = [&](int off, int fan_out, int fan_in) {
    const double r = std::sqrt(6.0 / fan_in);
    for (int i = 0; i < fan_out * fan_in; ++i) {
      const double u = (double)(sm64(stream_key(seed, 11) + (uint64_t)(off + i)) >> 11) * (1.0 / 9007199254740992.0);
      model[off + i] = (float)((2 * u - 1) * r);
    }
  };
  init(MLP_W1, MLP_H, MLP_IN);
  init(MLP_W2, MLP_H, MLP_H);
  init(MLP_W3, MLP_K, MLP_H);
  float *d = (float *)ctx->buf("mlp_work", sizeof(float) * (MLP_NPARAM * 4 + 2 * MLP_IN + 8));
  float *dX = (float *)ctx->buf("mlp_X", sizeof(float) * n * MLP_IN);
  float *dT = (float *)ctx->buf("mlp_T", sizeof(float) * n * MLP_K);
  float *dQ = (float *)ctx->buf("mlp_Q", sizeof(float) * n * MLP_K);
  float *dL = (float *)ctx->buf("mlp_L", sizeof(float) * epochs);
  if (!d || !dX || !dT || !dQ || !dL) return eg.finish();
  float *dP = d, *dG = d + MLP_NPARAM, *dM1 = dG + MLP_NPARAM, *dM2 = dM1 + MLP_NPARAM, *dmean = dM2 + MLP_NPARAM,
        *dinv = dmean + MLP_IN;
  GSW_CUDA(cudaMemcpyAsync(dP, model.data(), sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice, stream()));
  GSW_CUDA(cudaMemcpyAsync(dmean, model.data() + MLP_NPARAM, sizeof(float) * 2 * MLP_IN, cudaMemcpyHostToDevice,
                           stream()));
  GSW_CUDA(cudaMemcpyAsync(dX, X, sizeof(float) * n * MLP_IN, cudaMemcpyHostToDevice, stream()));
  GSW_CUDA(cudaMemcpyAsync(dT, T, sizeof(float) * n * MLP_K, cudaMemcpyHostToDevice, stream()));
  GSW_CUDA(cudaMemsetAsync(dM1, 0, sizeof(float) * 2 * MLP_NPARAM, stream()));
  GSW_CUDA(cudaMemsetAsync(dL, 0, sizeof(float) * epochs, stream()));
  k_mlp_soft_labels<<<grid_for(n), 256, 0, stream()>>>(dT, n, tau, dQ);
  const int gb = (int)std::min<int64_t>((n + MLP_TRAIN_THREADS - 1) / MLP_TRAIN_THREADS, 2 * sm_count());
  for (int e = 0; e < epochs && ok(); ++e) {
    GSW_CUDA(cudaMemsetAsync(dG, 0, sizeof(float) * MLP_NPARAM, stream()));
    k_mlp_grad<<<gb, MLP_TRAIN_THREADS, 0, stream()>>>(dP, dmean, dinv, dX, dQ, n, dG, dL + e);
    k_mlp_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, stream()>>>(dP, dG, dM1, dM2, e + 1, lr, 1e-5f);
    GSW_LAUNCHED();
  }
  GSW_CUDA(cudaMemcpyAsync(model.data(), dP, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost, stream()));
  if (loss_out) GSW_CUDA(cudaMemcpyAsync(loss_out, dL, sizeof(float) * epochs, cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  if (ok()) memcpy(model_out, model.data(), sizeof(float) * model.size());
  return eg.finish();
}

gsw_status gsw_mlp_infer(gsw_ctx *ctx, const float *model, const float *X, int64_t n, int32_t *cls, float *prob) {
  entry_guard eg(ctx);
  if (!ctx || !model || !X || n <= 0 || !cls) return fail(GSW_ERR_INVALID_ARG, "gsw_mlp_infer: bad arguments");
  const mlp_model h = model_from_floats(model, 0.f);
  mlp_model *dm = (mlp_model *)ctx->buf("mlp_model_tmp", sizeof(mlp_model));
  float *dX = (float *)ctx->buf("mlp_X", sizeof(float) * n * MLP_IN);
  int *dc = (int *)ctx->buf("mlp_cls", sizeof(int) * n);
  float *dp = (float *)ctx->buf("mlp_prob", sizeof(float) * n);
  if (!dm || !dX || !dc || !dp) return eg.finish();
  GSW_CUDA(cudaMemcpyAsync(dm, &h, sizeof(h), cudaMemcpyHostToDevice, stream()));
  GSW_CUDA(cudaMemcpyAsync(dX, X, sizeof(float) * n * MLP_IN, cudaMemcpyHostToDevice, stream()));
  k_mlp_infer<<<(unsigned)((n * 32 + 255) / 256), 256, 0, stream()>>>(dm, dX, n, dc, dp);
  GSW_LAUNCHED();
  GSW_CUDA(cudaMemcpyAsync(cls, dc, sizeof(int) * n, cudaMemcpyDeviceToHost, stream()));
  if (prob) GSW_CUDA(cudaMemcpyAsync(prob, dp, sizeof(float) * n, cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  return eg.finish();
}

gsw_status gsw_tune_load(gsw_ctx *ctx, const int32_t *quarters) {
  entry_guard eg(ctx);
  if (!ctx) return fail(GSW_ERR_INVALID_ARG, "gsw_tune_load: NULL context");
  auto &q = ctx->executor.tune.quarters;
  int *flat = &q[0][0][0][0];
  const int count = (int)(sizeof(q) / sizeof(int));
  for (int i = 0; i < count; ++i) {
    const int v = quarters ? quarters[i] : 0;
    if (v < 0 || v > 64) return fail(GSW_ERR_INVALID_ARG, "gsw_tune_load: entries are 0..64 quarters");
    flat[i] = v;
  }
  return GSW_OK;
}

gsw_status gsw_tune_load_shapes(gsw_ctx *ctx, const int32_t *shapes) {
  entry_guard eg(ctx);
  if (!ctx) return fail(GSW_ERR_INVALID_ARG, "gsw_tune_load_shapes: NULL context");
  auto &t = ctx->executor.tune.shapes;
  for (int pull = 0; pull < 2; ++pull)
    for (int bm = 0; bm < 2; ++bm)
      for (int lb = 0; lb < 8; ++lb)
        for (int fu = 0; fu < 2; ++fu) {
          const int i = ((pull * 2 + bm) * 8 + lb) * 2 + fu;
          const int v = shapes ? shapes[i] : 0;
          if (v < 0 || v >= shape_count(pull != 0, lb))
            return fail(GSW_ERR_INVALID_ARG, "gsw_tune_load_shapes: shape out of range for its variant");
        }
  for (int i = 0; i < (int)(sizeof(t) / sizeof(int)); ++i) (&t[0][0][0][0])[i] = shapes ? shapes[i] : 0;
  return GSW_OK;
}

gsw_status gsw_tune_save_shapes(gsw_ctx *ctx, int32_t *shapes) {
  if (!ctx || !shapes) return fail(GSW_ERR_INVALID_ARG, "gsw_tune_save_shapes: bad arguments");
  memcpy(shapes, &ctx->executor.tune.shapes[0][0][0][0], sizeof(ctx->executor.tune.shapes));
  return GSW_OK;
}

gsw_status gsw_tune_save(gsw_ctx *ctx, int32_t *quarters) {
  if (!ctx || !quarters) return fail(GSW_ERR_INVALID_ARG, "gsw_tune_save: bad arguments");
  const auto &q = ctx->executor.tune.quarters;
  memcpy(quarters, &q[0][0][0][0], sizeof(q));
  return GSW_OK;
}

gsw_status gsw_mlp_load_fusion(gsw_ctx *ctx, const float *model, float min_conf) {
  entry_guard eg(ctx);
  if (!ctx) return fail(GSW_ERR_INVALID_ARG, "gsw_mlp_load_fusion: NULL context");
  if (!model)
    ctx->mlp_fusion.valid = 0;
  else
    ctx->mlp_fusion = model_from_floats(model, min_conf);
  return GSW_OK;
}

gsw_status gsw_mlp_save(gsw_ctx *ctx, float *model, float *min_conf) {
  entry_guard eg(ctx);
  if (!ctx || !model) return fail(GSW_ERR_INVALID_ARG, "gsw_mlp_save: bad arguments");
  if (!ctx->mlp.valid) return fail(GSW_ERR_INVALID_ARG, "gsw_mlp_save: no model loaded");
  memcpy(model, &ctx->mlp, sizeof(float) * GSW_MLP_MODEL_FLOATS);
  if (min_conf) *min_conf = ctx->mlp.min_conf;
  return GSW_OK;
}

gsw_status gsw_select(gsw_ctx *ctx, const gsw_level_stats *in, int sel_kind, gsw_level_choice *out) {
  entry_guard eg(ctx);
  if (!ctx || !in || !out || in->nvertexs <= 0 || in->pattern < 0 || in->pattern > 2)
    return fail(GSW_ERR_INVALID_ARG, "gsw_select: bad arguments");
  feature_t fets;
  config_t conf;
  fets.centric = VC;
  fets.pattern = in->pattern == 0 ? Idem : (in->pattern == 1 ? Mono : ASSO);
  fets.fromall = in->fromall != 0;
  fets.toall = in->toall != 0;
  fets.nvertexs = in->nvertexs;
  fets.nedges = in->nedges;
  fets.avg_deg = in->attr[0];
  fets.std_deg = in->attr[1];
  fets.range = in->attr[2];
  fets.max_deg = in->attr[3];
  fets.GI = in->attr[4];
  fets.Her = in->attr[5];
  fets.architecture_features();
  conf.conf_pruning = fets.pattern == Idem;
  conf.conf_fromall = fets.fromall;
  conf.conf_toall = fets.toall;
  conf.conf_fusion = false;
  conf.conf_fuse_inspect = false;
  conf.force.has_fusion = true;  // fusion stays with the caller's loop
  conf.force.fusion = Standalone;
  fets_level_init(fets, in->level, in->nvertexs, in->nedges);
  bool done = false;
  if (in->first_level) {
    fets.use_root = 0;
    fets.first_active = (double)std::max<int64_t>(in->active, 1);
    fets.first_workload = (double)in->root_degree;
    fets_first(fets, in->nvertexs, in->nedges);
  } else {
    const level_counts c = {in->active, in->inactive, in->push_workload, in->pull_workload, in->max_push, in->max_pull};
    done = fets_from_counts(fets, c, in->nvertexs, in->nedges);
  }
  fets.flatten();
  out->done = done ? 1 : 0;
  // the host loop's order: the trees, the network, then the filter step's
  // grid bookkeeping (a tiny STRICT level goes to CM)
  selector_t selector;
  selector.decide(fets, conf);
  if (sel_kind == GSW_SELECT_MLP && ctx->mlp.valid) mlp_override(ctx->mlp, fets, conf);
  level_grid_bookkeeping(fets, conf);
  out->direction = conf.conf_dir == Pull ? GSW_PULL : GSW_PUSH;
  out->asfmt = conf.conf_asfmt == Bitmap ? GSW_BITMAP : GSW_QUEUE;
  out->lb = (int)conf.conf_lb;
  return eg.finish();
}

gsw_status gsw_mlp_load(gsw_ctx *ctx, const float *model, float min_conf) {
  entry_guard eg(ctx);
  if (!ctx) return fail(GSW_ERR_INVALID_ARG, "gsw_mlp_load: NULL context");
  if (!model) {
    ctx->mlp.valid = 0;
  } else {
    ctx->mlp = model_from_floats(model, min_conf);
  }
  if (!ctx->dmlp && GSW_CUDA(cudaMalloc((void **)&ctx->dmlp, sizeof(mlp_model)))) return eg.finish();
  GSW_CUDA(cudaMemcpyAsync(ctx->dmlp, &ctx->mlp, sizeof(mlp_model), cudaMemcpyHostToDevice, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  return eg.finish();
}

}  // extern "C"
