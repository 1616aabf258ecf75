// Batched multi-source BFS with bit-sliced frontiers.
//
// The reference's MBFS re-runs the single-source loop per source
// (application/mbfs.cu:222-297).  Here all sources advance together: bit s
// of word g stands for source 64*g + s, and each vertex keeps W = ceil(k/64)
// words of `seen`, `frontier` and `next` stored vertex-major, so one 32-byte
// sector carries every source's state of a vertex (256 sources).  Levels are
// level-synchronous and identical to per-source BFS.
//   push : a warp per adjacency chunk (at most 1024 edges of one vertex) ORs
//          (frontier & ~seen[u]) into next[u]
//   pull : a warp per chunk of a vertex with unseen bits ORs the
//          neighbours' frontier words and stops once every unseen bit is
//          covered
//   update: next & ~seen becomes the new frontier, levels are written for
//          the new bits (vertex-major, so one vertex's writes share its row
//          of nsrc entries; one tiled transpose gives the source-major
//          result at the end), and the counters that pick the next direction
//          (frontier edges vs. unexplored edges, Beamer's alpha = 14) are
//          reduced.
#pragma once
#include <vector>

#include <cub/cub.cuh>

#include "engine/executor.cuh"

namespace gsw {

constexpr int MBFS_MAXW = 8;  // up to 512 sources per batch

struct mbfs_result {
  double ms = 0;
  int levels = 0;
  int64_t edges = 0;
};

struct mbfs_counters {
  unsigned long long active_v;    // vertices with new bits
  unsigned long long active_e;    // their degree sum
  unsigned long long unseen_e;    // degree sum of vertices with unseen bits
  unsigned long long reached_e;   // sum over vertices of deg * popcount(seen)
};

// Adjacency lists cut into pieces of at most MBFS_CHUNK edges, so a hub's
// edges spread over many warps instead of serialising one.
constexpr int64_t MBFS_CHUNK = 1024;

__global__ void k_mbfs_chunk_count(const int64_t *off, int64_t n, int64_t *cnt) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int64_t d = off[v + 1] - off[v];
    cnt[v] = d == 0 ? 0 : (d + MBFS_CHUNK - 1) / MBFS_CHUNK;
  }
}
__global__ void k_mbfs_chunk_fill(const int64_t *off, int64_t n, const int64_t *coff, int *cv, int64_t *cbeg) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
    for (int64_t i = coff[v], b = off[v]; i < coff[v + 1]; ++i, b += MBFS_CHUNK) {
      cv[i] = (int)v;
      cbeg[i] = b;
    }
}

// Frontier words are rewritten every level; inside a persistent launch they
// must be read with plain loads (RO = false), per-level launches may use the
// read-only path.
template <bool RO>
__device__ __forceinline__ uint64_t mbfs_ld(const uint64_t *p) {
  if constexpr (RO)
    return __ldg(p);
  else
    return *(volatile const uint64_t *)p;
}

// push, warp per chunk: the chunk's vertex's frontier bits go to every
// neighbour that has not seen them
template <int W, bool RO>
__device__ __forceinline__ void mbfs_push_body(const device_graph_t<CSR, Empty> &g, const int *cv, const int64_t *cbeg,
                                               int64_t nchunks, const uint64_t *frontier, const uint64_t *seen,
                                               uint64_t *next) {
  const int lane = lane_id();
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t c = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp_id(); c < nchunks; c += nwarps) {
    const int v = cv[c];
    uint64_t f[W];
    bool any = false;
#pragma unroll
    for (int k = 0; k < W; ++k) {
      f[k] = mbfs_ld<RO>(frontier + (int64_t)v * W + k);
      any |= f[k] != 0;
    }
    if (!any) continue;
    const int64_t b = cbeg[c], e = MIN(b + MBFS_CHUNK, __ldg(g.dg_row_off + v + 1));
    for (int64_t i = b + lane; i < e; i += 32) {
      const int u = __ldg(g.dg_adj_list + i);
#pragma unroll
      for (int k = 0; k < W; ++k) {
        const uint64_t m = f[k] & ~seen[(int64_t)u * W + k];
        if (m) atomicOr((unsigned long long *)(next + (int64_t)u * W + k), (unsigned long long)m);
      }
    }
  }
}
template <int W>
__global__ void __launch_bounds__(256) k_mbfs_push_chunks(device_graph_t<CSR, Empty> g, const int *cv,
                                                           const int64_t *cbeg, int64_t nchunks,
                                                           const uint64_t *frontier, const uint64_t *seen,
                                                           uint64_t *next) {
  mbfs_push_body<W, true>(g, cv, cbeg, nchunks, frontier, seen, next);
}

// pull, warp per chunk: OR of the in-neighbours' frontier words over the
// chunk, cut short once every bit the vertex still needs is covered; a vertex
// with several chunks combines them with atomicOr
template <int W, bool RO>
__device__ __forceinline__ void mbfs_pull_body(const device_graph_t<CSR, Empty> &g, const int *cv, const int64_t *cbeg,
                                               int64_t nchunks, const uint64_t *frontier, const uint64_t *seen,
                                               uint64_t *next, const uint64_t *valid) {
  const int lane = lane_id();
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t c = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp_id(); c < nchunks; c += nwarps) {
    const int v = cv[c];
    uint64_t need[W], acc[W];
    bool any = false;
#pragma unroll
    for (int k = 0; k < W; ++k) {
      need[k] = valid[k] & ~seen[(int64_t)v * W + k];
      acc[k] = 0;
      any |= need[k] != 0;
    }
    if (!any) continue;
    const int64_t st = __ldg(g.dgr_row_off + v), en = __ldg(g.dgr_row_off + v + 1);
    const int64_t b = cbeg[c], e = MIN(b + MBFS_CHUNK, en);
    for (int64_t base = b; base < e; base += 32) {
      const int64_t i = base + lane;
      if (i < e) {
        const int u = __ldg(g.dgr_adj_list + i);
#pragma unroll
        for (int k = 0; k < W; ++k) acc[k] |= mbfs_ld<RO>(frontier + (int64_t)u * W + k);
      }
      // every 32 edges: stop when the warp's bits cover what v needs
      bool covered = true;
#pragma unroll
      for (int k = 0; k < W; ++k) {
        const unsigned lo = __reduce_or_sync(FULL, (unsigned)acc[k]);
        const unsigned hi = __reduce_or_sync(FULL, (unsigned)(acc[k] >> 32));
        covered &= ((((uint64_t)hi << 32) | lo) & need[k]) == need[k];
      }
      if (covered) break;
    }
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const unsigned lo = __reduce_or_sync(FULL, (unsigned)acc[k]);
      const unsigned hi = __reduce_or_sync(FULL, (unsigned)(acc[k] >> 32));
      acc[k] = (((uint64_t)hi << 32) | lo) & need[k];
    }
    if (lane < W) {
      uint64_t mine = 0;
#pragma unroll
      for (int k = 0; k < W; ++k)
        if (k == lane) mine = acc[k];
      uint64_t *dst = next + (int64_t)v * W + lane;
      if (e - b == en - st)
        *dst = mine;  // the only chunk of v
      else if (mine)
        atomicOr((unsigned long long *)dst, (unsigned long long)mine);
    }
  }
}
template <int W>
__global__ void __launch_bounds__(256) k_mbfs_pull_chunks(device_graph_t<CSR, Empty> g, const int *cv,
                                                           const int64_t *cbeg, int64_t nchunks,
                                                           const uint64_t *frontier, const uint64_t *seen,
                                                           uint64_t *next, const uint64_t *valid) {
  mbfs_pull_body<W, true>(g, cv, cbeg, nchunks, frontier, seen, next, valid);
}

template <int W>
__device__ __forceinline__ void mbfs_update_body(const device_graph_t<CSR, Empty> &g, uint64_t *frontier,
                                                 uint64_t *seen, uint64_t *next, int *levels, int nsrc, int level,
                                                 const uint64_t *valid, mbfs_counters *cnt) {
  __shared__ unsigned long long s_red[32];
  const int64_t n = g.nvertexs;
  const int64_t STRIDE = (int64_t)blockDim.x * gridDim.x;
  unsigned long long av = 0, ae = 0, ue = 0;
  for (int64_t v = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; v < n; v += STRIDE) {
    const int deg = __ldg(g.dg_odegree + v);
    bool nb_any = false, unseen = false;
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const uint64_t s = seen[v * W + k];
      const uint64_t nb = next[v * W + k] & ~s;
      next[v * W + k] = 0;
      frontier[v * W + k] = nb;
      if (nb) {
        nb_any = true;
        seen[v * W + k] = s | nb;
        uint64_t b = nb;
        while (b) {
          const int bit = __ffsll((long long)b) - 1;
          b &= b - 1;
          const int src = k * 64 + bit;
          if (src < nsrc) levels[v * nsrc + src] = level;  // vertex-major while running
        }
      }
      unseen |= (valid[k] & ~(s | nb)) != 0;
    }
    if (nb_any) {
      av++;
      ae += deg;
    }
    if (unseen) ue += deg;
  }
  unsigned long long r = block_reduce(av, s_red);
  if (threadIdx.x == 0 && r) atomicAdd(&cnt->active_v, r);
  r = block_reduce(ae, s_red);
  if (threadIdx.x == 0 && r) atomicAdd(&cnt->active_e, r);
  r = block_reduce(ue, s_red);
  if (threadIdx.x == 0 && r) atomicAdd(&cnt->unseen_e, r);
}
template <int W>
__global__ void __launch_bounds__(256) k_mbfs_update(device_graph_t<CSR, Empty> g, uint64_t *frontier, uint64_t *seen,
                                                      uint64_t *next, int *levels, int nsrc, int level,
                                                      const uint64_t *valid, mbfs_counters *cnt) {
  mbfs_update_body<W>(g, frontier, seen, next, levels, nsrc, level, valid, cnt);
}

// ---- batched BC passes over the vertex-major levels of a <= 32-source batch
// (bc_batch.cuh drives them; lane s of a warp is source s) ----------------
constexpr int BCB_SOURCES = 32;  // sources per batch: one per lane

// forward pass of level L (L >= 1): nsp[v] = sum of nsp[u] over the
// in-neighbours one level closer, per source (undirected graphs: the chunk
// list covers the adjacency lists, which are the in-lists as well)
__device__ __forceinline__ void bcb_forward_body(const device_graph_t<CSR, Empty> &g, const int *cv, const int64_t *cbeg,
                                                 int64_t nchunks, const int *lvl, int nsrc, int L, int *nsp) {
  const int lane = lane_id();
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t c = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp_id(); c < nchunks; c += nwarps) {
    const int v = cv[c];
    const bool mine = lane < nsrc && lvl[(int64_t)v * nsrc + lane] == L;
    if (!__any_sync(FULL, mine)) continue;
    const int64_t st = __ldg(g.dg_row_off + v), en = __ldg(g.dg_row_off + v + 1);
    const int64_t b = cbeg[c], e = MIN(b + MBFS_CHUNK, en);
    int acc = 0;
    for (int64_t base = b; base < e; base += 32) {
      const int cnt = (int)MIN((int64_t)32, e - base);
      const int u_l = lane < cnt ? __ldg(g.dg_adj_list + base + lane) : 0;
      for (int j = 0; j < cnt; ++j) {
        const int u = __shfl_sync(FULL, u_l, j);
        const bool parent = mine && lvl[(int64_t)u * nsrc + lane] == L - 1;
        if (parent) acc += nsp[(int64_t)u * nsrc + lane];  // int32, wraps like the reference
      }
    }
    if (mine) {
      int *dst = nsp + (int64_t)v * nsrc + lane;
      if (e - b == en - st)
        *dst = acc;  // the vertex's only chunk
      else
        atomicAdd(dst, acc);
    }
  }
}

// backward pass of level L: sum[v] = sum over children w of (1 + dep[w]) /
// nsp[w], with dep[w] = nsp[w] * sum[w] from the pass of level L+1
__device__ __forceinline__ void bcb_backward_body(const device_graph_t<CSR, Empty> &g, const int *cv,
                                                  const int64_t *cbeg, int64_t nchunks, const int *lvl, int nsrc, int L,
                                                  const int *nsp, float *sum) {
  const int lane = lane_id();
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t c = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp_id(); c < nchunks; c += nwarps) {
    const int v = cv[c];
    const bool mine = lane < nsrc && lvl[(int64_t)v * nsrc + lane] == L;
    if (!__any_sync(FULL, mine)) continue;
    const int64_t st = __ldg(g.dg_row_off + v), en = __ldg(g.dg_row_off + v + 1);
    const int64_t b = cbeg[c], e = MIN(b + MBFS_CHUNK, en);
    float acc = 0.0f;
    for (int64_t base = b; base < e; base += 32) {
      const int cnt = (int)MIN((int64_t)32, e - base);
      const int w_l = lane < cnt ? __ldg(g.dg_adj_list + base + lane) : 0;
      for (int j = 0; j < cnt; ++j) {
        const int w = __shfl_sync(FULL, w_l, j);
        const int64_t r = (int64_t)w * nsrc + lane;
        if (mine && lvl[r] == L + 1) {
          const float nw = (float)nsp[r];
          acc += (1.0f + nw * sum[r]) / nw;
        }
      }
    }
    if (mine) {
      float *dst = sum + (int64_t)v * nsrc + lane;
      if (e - b == en - st)
        *dst = acc;
      else
        atomicAdd(dst, acc);
    }
  }
}

// dep = nsp * sum, in place over the sums
__device__ __forceinline__ void bcb_finish_body(const int *nsp, float *sum, int64_t cells) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cells; i += (int64_t)gridDim.x * blockDim.x)
    sum[i] = (float)nsp[i] * sum[i];
}

__global__ void __launch_bounds__(256) k_bcb_forward(device_graph_t<CSR, Empty> g, const int *cv, const int64_t *cbeg,
                                                     int64_t nchunks, const int *lvl, int nsrc, int L, int *nsp) {
  bcb_forward_body(g, cv, cbeg, nchunks, lvl, nsrc, L, nsp);
}
__global__ void __launch_bounds__(256) k_bcb_backward(device_graph_t<CSR, Empty> g, const int *cv, const int64_t *cbeg,
                                                      int64_t nchunks, const int *lvl, int nsrc, int L, const int *nsp,
                                                      float *sum) {
  bcb_backward_body(g, cv, cbeg, nchunks, lvl, nsrc, L, nsp, sum);
}
__global__ void k_bcb_finish(const int *nsp, float *sum, int64_t cells) { bcb_finish_body(nsp, sum, cells); }
// roots: nsp = 1 for their own source
__global__ void k_bcb_seed(const int *roots, int nsrc, int *nsp) {
  const int s = threadIdx.x;
  if (s < nsrc) nsp[(int64_t)roots[s] * nsrc + s] = 1;
}

// ---- every level in one cooperative launch ----------------------------------
// The per-level loop above needs the host after every level (the counters
// decide the next direction).  The persistent form keeps the whole grid
// resident: push or pull, a grid barrier, the update (counters into the
// level's slot of two), a grid barrier, and every block reads the same
// counters to stop or to pick the next direction (Beamer's test, alpha = 14).
// With BC, the same launch continues with the forward passes (levels 1 ..
// depth-1) and the backward passes (depth-2 .. 0), a barrier after each, and
// the final dep = nsp * sum.  Barrier waits are bounded (budget_ns each);
// after a timeout every block leaves and status says so.
struct mbfs_persist_t {
  unsigned *bar;             // [0] arrivals, [1] generation, [2] error word
  mbfs_counters *cnt;        // [2], by level parity, zero at launch
  int *out;                  // [0] levels (the one that found nothing), [1] status (0 ok, 1 barrier timeout)
  unsigned long long budget_ns;
  int max_levels;
};

template <int W, bool BC>
__global__ void __launch_bounds__(256) k_mbfs_persistent(device_graph_t<CSR, Empty> g, const int *cv,
                                                          const int64_t *cbeg, int64_t nchunks, uint64_t *frontier,
                                                          uint64_t *seen, uint64_t *next, int *levels, int nsrc,
                                                          const uint64_t *valid, mbfs_persist_t P, int *nsp,
                                                          float *sum) {
  unsigned gen = 0;
  auto barrier = [&]() { return grid_barrier(P.bar, P.bar + 1, P.bar + 2, gen, P.budget_ns); };
  bool push = true, okk = true;
  int level = 1;
  for (; level <= P.max_levels; ++level) {
    if (push)
      mbfs_push_body<W, false>(g, cv, cbeg, nchunks, frontier, seen, next);
    else
      mbfs_pull_body<W, false>(g, cv, cbeg, nchunks, frontier, seen, next, valid);
    if (!(okk = barrier())) break;
    // the slot of the next level was last read before the barrier above
    if (blockIdx.x == 0 && threadIdx.x == 0) P.cnt[(level + 1) & 1] = mbfs_counters{0, 0, 0, 0};
    mbfs_update_body<W>(g, frontier, seen, next, levels, nsrc, level, valid, &P.cnt[level & 1]);
    if (!(okk = barrier())) break;
    const volatile mbfs_counters *c = &P.cnt[level & 1];
    if (c->active_v == 0) break;
    push = c->active_e * 14 < c->unseen_e;
  }
  if constexpr (BC) {
    const int depth = level;
    for (int L = 1; okk && L < depth; ++L) {
      bcb_forward_body(g, cv, cbeg, nchunks, levels, nsrc, L, nsp);
      okk = barrier();
    }
    for (int L = depth - 2; okk && L >= 0; --L) {
      bcb_backward_body(g, cv, cbeg, nchunks, levels, nsrc, L, nsp, sum);
      okk = barrier();
    }
    if (okk) bcb_finish_body(nsp, sum, (int64_t)g.nvertexs * nsrc);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    P.out[0] = level;
    P.out[1] = okk ? 0 : 1;
  }
}

template <int W>
__global__ void k_mbfs_seed(uint64_t *frontier, uint64_t *seen, const int *roots, int nsrc, int *levels, int64_t n) {
  for (int s = threadIdx.x + blockIdx.x * blockDim.x; s < nsrc; s += blockDim.x * gridDim.x) {
    const int64_t r = roots[s];
    atomicOr((unsigned long long *)(frontier + r * W + (s >> 6)), 1ull << (s & 63));
    atomicOr((unsigned long long *)(seen + r * W + (s >> 6)), 1ull << (s & 63));
    levels[r * nsrc + s] = 0;
  }
}

template <int W>
__global__ void __launch_bounds__(256) k_mbfs_reached(device_graph_t<CSR, Empty> g, const uint64_t *seen,
                                                       mbfs_counters *cnt) {
  __shared__ unsigned long long s_red[32];
  unsigned long long s = 0;
  for (int64_t v = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; v < g.nvertexs; v += (int64_t)blockDim.x * gridDim.x) {
    int pc = 0;
#pragma unroll
    for (int k = 0; k < W; ++k) pc += __popcll(seen[v * W + k]);
    s += (unsigned long long)pc * __ldg(g.dg_odegree + v);
  }
  s = block_reduce(s, s_red);
  if (threadIdx.x == 0 && s) atomicAdd(&cnt->reached_e, s);
}

// vertex-major [n][nsrc] -> source-major [nsrc][n] through 32 x 32 tiles
__global__ void __launch_bounds__(256) k_mbfs_transpose(const int *vm, int64_t n, int nsrc, int *sm) {
  __shared__ int tile[32][33];
  const int64_t vt = (n + 31) / 32, st = (nsrc + 31) / 32;
  for (int64_t t = blockIdx.x; t < vt * st; t += gridDim.x) {
    const int64_t v0 = (t / st) * 32;
    const int s0 = (int)(t % st) * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      const int64_t v = v0 + r;
      const int s = s0 + threadIdx.x;
      tile[r][threadIdx.x] = (v < n && s < nsrc) ? vm[v * nsrc + s] : 0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      const int s = s0 + r;
      const int64_t v = v0 + threadIdx.x;
      if (v < n && s < nsrc) sm[(int64_t)s * n + v] = tile[threadIdx.x][r];
    }
    __syncthreads();
  }
}

inline int grid_for_n(int64_t n) { return (int)MIN((n + 255) / 256 + 1, (int64_t)sm_count() * 16); }

template <typename T>
__global__ void k_mbfs_fill(T *p, T v, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = v;
}

// transpose = false leaves the levels vertex-major in the "mb_levels_vm"
// buffer (row v holds nsrc levels) for a caller that keeps working on them.
// persistent = true runs every level in one cooperative launch; with
// bc_nsp / bc_sum (W = 1, at most BCB_SOURCES sources) that launch also runs
// the batched BC passes into them.
template <int W, typename Buf>
mbfs_result mbfs_impl(device_graph_t<CSR, Empty> g, int nsrc, const int32_t *roots_host, Buf buf, int32_t *levels_host,
                      bool transpose = true, bool persistent = false, int *bc_nsp = nullptr, float *bc_sum = nullptr) {
  mbfs_result res;
  const int64_t n = g.nvertexs;
  const int grid = sm_count() * 8;
  uint64_t *frontier = (uint64_t *)buf("mb_front", sizeof(uint64_t) * n * W);
  uint64_t *seen = (uint64_t *)buf("mb_seen", sizeof(uint64_t) * n * W);
  uint64_t *next = (uint64_t *)buf("mb_next", sizeof(uint64_t) * n * W);
  int *levels = (int *)buf("mb_levels_vm", sizeof(int) * (size_t)n * nsrc);  // vertex-major, while running
  int *levels_sm = (int *)buf("mb_levels", sizeof(int) * (size_t)n * nsrc);   // source-major result
  int *roots = (int *)buf("mb_roots", sizeof(int) * nsrc);
  uint64_t *valid = (uint64_t *)buf("mb_valid", sizeof(uint64_t) * W);
  mbfs_counters *cnt = (mbfs_counters *)buf("mb_cnt", sizeof(mbfs_counters));
  mbfs_counters *hcnt = nullptr;
  if (!frontier || !seen || !next || !levels || !levels_sm || !roots || !valid || !cnt) return res;
  // the chunk list of the adjacency lists (the graph is undirected, so it
  // serves pushes and pulls alike)
  int64_t *ccnt = (int64_t *)buf("mb_ccnt", sizeof(int64_t) * (n + 1));
  int64_t *coff = (int64_t *)buf("mb_coff", sizeof(int64_t) * (n + 1));
  if (!ccnt || !coff) return res;
  GSW_CUDA(cudaMemsetAsync(ccnt + n, 0, sizeof(int64_t), stream()));
  k_mbfs_chunk_count<<<grid_for_n(n), 256, 0, stream()>>>(g.dg_row_off, n, ccnt);
  size_t tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, ccnt, coff, n + 1, stream());
  void *tmp = buf("mb_scan_tmp", tb);
  if (!tmp) return res;
  GSW_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, ccnt, coff, n + 1, stream()));
  int64_t nchunks = 0;
  GSW_CUDA(cudaMemcpyAsync(&nchunks, coff + n, sizeof(int64_t), cudaMemcpyDeviceToHost, stream()));
  GSW_CUDA(cudaStreamSynchronize(stream()));
  int *cv = (int *)buf("mb_cv", sizeof(int) * (nchunks + 1));
  int64_t *cbeg = (int64_t *)buf("mb_cbeg", sizeof(int64_t) * (nchunks + 1));
  if (!cv || !cbeg) return res;
  k_mbfs_chunk_fill<<<grid_for_n(n), 256, 0, stream()>>>(g.dg_row_off, n, coff, cv, cbeg);
  if (GSW_CUDA(cudaMallocHost((void **)&hcnt, sizeof(mbfs_counters)))) return res;
  uint64_t hv[W];
  for (int k = 0; k < W; ++k) {
    const int lo = k * 64;
    const int c = nsrc - lo >= 64 ? 64 : (nsrc - lo > 0 ? nsrc - lo : 0);
    hv[k] = c == 64 ? ~0ull : ((1ull << c) - 1);
  }
  cudaStream_t s = stream();
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  GSW_CUDA(cudaMemcpyAsync(valid, hv, sizeof(hv), cudaMemcpyHostToDevice, s));
  GSW_CUDA(cudaMemcpyAsync(roots, roots_host, sizeof(int) * nsrc, cudaMemcpyHostToDevice, s));
  GSW_CUDA(cudaMemsetAsync(frontier, 0, sizeof(uint64_t) * n * W, s));
  GSW_CUDA(cudaMemsetAsync(seen, 0, sizeof(uint64_t) * n * W, s));
  GSW_CUDA(cudaMemsetAsync(next, 0, sizeof(uint64_t) * n * W, s));
  k_mbfs_fill<int><<<grid, 256, 0, s>>>(levels, -1, n * (int64_t)nsrc);
  const bool bc = bc_nsp && bc_sum;
  if (bc) {
    GSW_CUDA(cudaMemsetAsync(bc_nsp, 0, sizeof(int) * (size_t)n * nsrc, s));
    GSW_CUDA(cudaMemsetAsync(bc_sum, 0, sizeof(float) * (size_t)n * nsrc, s));
  }
  cudaEventRecord(e0, s);
  k_mbfs_seed<W><<<1, 256, 0, s>>>(frontier, seen, roots, nsrc, levels, n);
  if (bc) k_bcb_seed<<<1, BCB_SOURCES, 0, s>>>(roots, nsrc, bc_nsp);
  if (persistent) {
    unsigned *bar = (unsigned *)buf("mb_bar", sizeof(unsigned) * 4);
    mbfs_counters *pc = (mbfs_counters *)buf("mb_pcnt", sizeof(mbfs_counters) * 2);
    int *pout = (int *)buf("mb_pout", sizeof(int) * 2);
    if (bar && pc && pout) {
      GSW_CUDA(cudaMemsetAsync(bar, 0, sizeof(unsigned) * 4, s));
      GSW_CUDA(cudaMemsetAsync(pc, 0, sizeof(mbfs_counters) * 2, s));
      mbfs_persist_t P{bar, pc, pout, 2000000000ull, (int)MIN(n + 1, (int64_t)INT32_MAX - 1)};
      auto kern = bc ? k_mbfs_persistent<W, true> : k_mbfs_persistent<W, false>;
      const int pgrid = resident_grid(kern, 256);
      void *args[] = {(void *)&g,    (void *)&cv,     (void *)&cbeg,   (void *)&nchunks, (void *)&frontier,
                      (void *)&seen, (void *)&next,   (void *)&levels, (void *)&nsrc,    (void *)&valid,
                      (void *)&P,    (void *)&bc_nsp, (void *)&bc_sum};
      if (!GSW_CUDA(cudaLaunchCooperativeKernel((const void *)kern, pgrid, 256, args, 0, s))) {
        GSW_LAUNCHED();
        int out[2] = {0, 1};
        GSW_CUDA(cudaMemcpyAsync(out, pout, sizeof(out), cudaMemcpyDeviceToHost, s));
        GSW_CUDA(cudaStreamSynchronize(s));
        res.levels = out[0];
        if (out[1] != 0) set_error(GSW_ERR_TIMEOUT, "%s", "batched BFS: grid barrier timed out");
      }
    }
  }
  // the first level pushes from the sources
  bool push = true;
  for (int level = 1; !persistent && level <= n + 1 && ok(); ++level) {
    if (push)
      k_mbfs_push_chunks<W><<<grid, 256, 0, s>>>(g, cv, cbeg, nchunks, frontier, seen, next);
    else
      k_mbfs_pull_chunks<W><<<grid, 256, 0, s>>>(g, cv, cbeg, nchunks, frontier, seen, next, valid);
    GSW_CUDA(cudaMemsetAsync(cnt, 0, sizeof(mbfs_counters), s));
    k_mbfs_update<W><<<grid, 256, 0, s>>>(g, frontier, seen, next, levels, nsrc, level, valid, cnt);
    GSW_CUDA(cudaMemcpyAsync(hcnt, cnt, sizeof(mbfs_counters), cudaMemcpyDeviceToHost, s));
    GSW_CUDA(cudaStreamSynchronize(s));
    res.levels = level;
    if (hcnt->active_v == 0) break;
    // Beamer's direction test with alpha = 14
    push = hcnt->active_e * 14 < hcnt->unseen_e;
  }
  if (transpose) k_mbfs_transpose<<<sm_count() * 8, dim3(32, 8), 0, s>>>(levels, n, nsrc, levels_sm);
  cudaEventRecord(e1, s);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  res.ms = ms;
  GSW_CUDA(cudaMemsetAsync(cnt, 0, sizeof(mbfs_counters), s));
  k_mbfs_reached<W><<<grid, 256, 0, s>>>(g, seen, cnt);
  GSW_CUDA(cudaMemcpyAsync(hcnt, cnt, sizeof(mbfs_counters), cudaMemcpyDeviceToHost, s));
  GSW_CUDA(cudaStreamSynchronize(s));
  res.edges = (int64_t)(hcnt->reached_e / 2);
  if (levels_host && transpose && ok())
    GSW_CUDA(cudaMemcpyAsync(levels_host, levels_sm, sizeof(int) * (size_t)n * nsrc, cudaMemcpyDeviceToHost, s));
  GSW_CUDA(cudaStreamSynchronize(s));
  cudaFreeHost(hcnt);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return res;
}

template <typename Buf>
mbfs_result run_mbfs_batched(device_graph_t<CSR, Empty> g, int nsrc, const int32_t *roots, Buf buf,
                             int32_t *levels_host, bool persistent) {
  const int w = (nsrc + 63) / 64;
  if (w <= 1) return mbfs_impl<1>(g, nsrc, roots, buf, levels_host, true, persistent);
  if (w <= 2) return mbfs_impl<2>(g, nsrc, roots, buf, levels_host, true, persistent);
  if (w <= 4) return mbfs_impl<4>(g, nsrc, roots, buf, levels_host, true, persistent);
  if (w <= 8) return mbfs_impl<8>(g, nsrc, roots, buf, levels_host, true, persistent);
  set_error(GSW_ERR_UNSUPPORTED, "%s", "mbfs: at most 512 sources per batch");
  return mbfs_result();
}

}  // namespace gsw
