// gsw_bfs_strict_noalloc: breadth-first search with the edge-balanced
// (STRICT) push expand, for callers that cannot allocate device memory.
//
// Who needs it: code embedded in a host framework whose memory pool already
// owns the device memory (a cudaMalloc there fails or fragments that pool),
// and latency-critical callers that cannot afford the device-wide
// synchronisation cudaMalloc / cudaFree imply.  Such a caller passes its own
// device CSR and its own output array; everything else this search needs
// (two frontier queues, the degree scan, the tile table, counters) lives in
// one file-scope __device__ array below, so the call allocates nothing.
//
// Limits: n <= GSW_NOALLOC_MAX_VERTICES (2^18), arcs <= GSW_NOALLOC_MAX_ARCS
// (2^28); the array takes about 5 MiB of every GPU that loads the library,
// until the process exits.
//
// Set-up: the first call on a device looks up the array's device address
// (cudaGetSymbolAddress, with that device current) and keeps it for later
// calls on that device; make that first call before any stream capture.
// Every call reuses the same array and the array keeps the previous call's
// contents: the counters are cleared at the start of each call.  Calls that
// overlap on the GPU (other streams, other host threads) race on the array;
// callers must serialise them.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/gsw.h"
#include "engine/common.cuh"

namespace gsw {
extern thread_local std::string g_last_error;  // defined in gsw_capi.cu
}

namespace {

constexpr int64_t NA_MAX_VERTICES = int64_t(1) << 18;
constexpr int64_t NA_MAX_ARCS = int64_t(1) << 28;
constexpr int NA_THREADS = 256;
constexpr int NA_TILE = 1024;   // slots per expand tile (4 per thread)
constexpr int NA_ITEMS = 1024;  // frontier entries per scan block
constexpr int64_t NA_MAX_BLOCKS = NA_MAX_VERTICES / NA_ITEMS + 2;
constexpr int64_t NA_MAX_TILES = (NA_MAX_ARCS + NA_MAX_VERTICES) / NA_TILE + 2;

struct na_scratch {
  int queue[2][NA_MAX_VERTICES];
  long long eoff[NA_MAX_VERTICES + 1];   // exclusive scan of (degree + 1)
  long long bsum[NA_MAX_BLOCKS + 1];     // per-block partial sums
  int tile_lo[NA_MAX_TILES];             // frontier index owning each tile's first slot
  int qsize[2];
  unsigned err;
};

// One array per device for the whole process.
static __device__ __align__(256) na_scratch g_na_scratch;

std::mutex g_na_mu;
na_scratch *g_na_ptr[64] = {};

// device address of the array for `dev`, looked up once with `dev` current
int na_address(int dev, na_scratch **out) {
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (dev < 0 || dev >= 64) return gsw::set_error(GSW_ERR_UNSUPPORTED, "%s", "gsw_bfs_strict_noalloc: device id >= 64");
  if (!g_na_ptr[dev]) {
    na_scratch *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void **)&p, g_na_scratch);
    if (e != cudaSuccess || !p) return GSW_CUDA(e == cudaSuccess ? cudaErrorInvalidSymbol : e);
    g_na_ptr[dev] = p;
  }
  *out = g_na_ptr[dev];
  return GSW_OK;
}

__global__ void k_na_init(na_scratch *S, int *levels, int64_t n, int root) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
    levels[v] = v == root ? 0 : -1;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    S->queue[0][0] = root;
    S->qsize[0] = 1;
    S->qsize[1] = 0;
    S->err = 0;
  }
}

__device__ __forceinline__ long long na_slots(const int64_t *off, int v) {
  return __ldg(off + v + 1) - __ldg(off + v) + 1;
}

__global__ void __launch_bounds__(NA_THREADS) k_na_count(na_scratch *S, int c, const int64_t *off) {
  __shared__ long long s_red[32];
  const int64_t F = S->qsize[c];
  const int64_t b0 = (int64_t)blockIdx.x * NA_ITEMS;
  long long s = 0;
  for (int k = threadIdx.x; k < NA_ITEMS; k += blockDim.x)
    if (b0 + k < F) s += na_slots(off, S->queue[c][b0 + k]);
  s = gsw::block_reduce(s, s_red);
  if (threadIdx.x == 0) S->bsum[blockIdx.x] = s;
}

__global__ void __launch_bounds__(1024) k_na_scan_blocks(na_scratch *S, int64_t len) {
  __shared__ long long s[33];
  long long carry = 0;
  for (int64_t base = 0; base < len; base += blockDim.x) {
    const int64_t i = base + threadIdx.x;
    const long long x = i < len ? S->bsum[i] : 0;
    const long long incl = gsw::warp_inclusive_sum(x);
    __syncthreads();
    if (gsw::lane_id() == 31) s[gsw::warp_id()] = incl;
    __syncthreads();
    if (gsw::warp_id() == 0) {
      const int nw = blockDim.x >> 5;
      const long long y = gsw::lane_id() < nw ? s[gsw::lane_id()] : 0;
      const long long yi = gsw::warp_inclusive_sum(y);
      if (gsw::lane_id() < nw) s[gsw::lane_id()] = yi - y;
      if (gsw::lane_id() == 31) s[32] = yi;
    }
    __syncthreads();
    if (i < len) S->bsum[i] = carry + s[gsw::warp_id()] + incl - x;
    carry += s[32];
    __syncthreads();
  }
  if (threadIdx.x == 0) S->bsum[len] = carry;
}

// eoff and the tile owners; 4 consecutive entries per thread
__global__ void __launch_bounds__(NA_THREADS) k_na_scan(na_scratch *S, int c, const int64_t *off, int64_t nblocks) {
  __shared__ long long s[33];
  const int64_t F = S->qsize[c];
  const int64_t base = (int64_t)blockIdx.x * NA_ITEMS + threadIdx.x * 4;
  long long d[4], loc = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    d[k] = base + k < F ? na_slots(off, S->queue[c][base + k]) : 0;
    loc += d[k];
  }
  const long long incl = gsw::warp_inclusive_sum(loc);
  __syncthreads();
  if (gsw::lane_id() == 31) s[gsw::warp_id()] = incl;
  __syncthreads();
  if (gsw::warp_id() == 0) {
    const int nw = blockDim.x >> 5;
    const long long y = gsw::lane_id() < nw ? s[gsw::lane_id()] : 0;
    const long long yi = gsw::warp_inclusive_sum(y);
    if (gsw::lane_id() < nw) s[gsw::lane_id()] = yi - y;
  }
  __syncthreads();
  long long o = S->bsum[blockIdx.x] + s[gsw::warp_id()] + incl - loc;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int64_t idx = base + k;
    if (idx < F) {
      S->eoff[idx] = o;
      for (long long t = (o + NA_TILE - 1) / NA_TILE; t * NA_TILE < o + d[k]; ++t) {
        if (t < NA_MAX_TILES)
          S->tile_lo[t] = (int)idx;
        else
          atomicOr(&S->err, gsw::DEV_ERR_SCRATCH_OVERFLOW);
      }
    }
    o += d[k];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) S->eoff[F] = S->bsum[nblocks];
}

// One BFS level: every edge of the frontier in queue[c], edge-balanced by
// tiles; an unvisited neighbour is claimed once (compare-and-swap on its
// level) and appended to queue[c ^ 1] with one atomic per warp.
__global__ void __launch_bounds__(NA_THREADS) k_na_expand(na_scratch *S, int c, const int64_t *off, const int *col,
                                                           int *levels, int level, int64_t n) {
  __shared__ long long s_sc[NA_TILE + 2];
  __shared__ long long s_st[NA_TILE + 2];
  const int64_t F = S->qsize[c];
  if (F == 0) return;
  const long long total = S->eoff[F];
  int64_t ntiles = (total + NA_TILE - 1) / NA_TILE;
  if (ntiles > NA_MAX_TILES - 1) {  // only an inconsistent CSR gets here
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&S->err, gsw::DEV_ERR_SCRATCH_OVERFLOW);
    ntiles = NA_MAX_TILES - 1;
  }
  int *out = S->queue[c ^ 1];
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t lo = S->tile_lo[t];
    const int64_t hi = (t + 1 < ntiles) ? S->tile_lo[t + 1] : F - 1;
    const int cnt = (int)(hi - lo + 1);
    if (cnt < 1 || cnt > NA_TILE + 1 || lo < 0 || hi >= F) {  // block-uniform
      if (threadIdx.x == 0) atomicOr(&S->err, gsw::DEV_ERR_SCRATCH_OVERFLOW);
      continue;
    }
    for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
      const int v = S->queue[c][lo + j];
      s_sc[j] = S->eoff[lo + j];
      s_st[j] = __ldg(off + v);
    }
    if (threadIdx.x == 0) s_sc[cnt] = S->eoff[hi + 1];
    __syncthreads();
    const long long t0 = t * NA_TILE;
    const long long t1 = t0 + NA_TILE < total ? t0 + NA_TILE : total;
#pragma unroll
    for (int k = 0; k < NA_TILE / NA_THREADS; ++k) {
      const long long sl = t0 + k * NA_THREADS + threadIdx.x;
      bool claim = false;
      int u = -1;
      if (sl < t1) {
        const int j = gsw::upper_bound(s_sc, cnt, sl) - 1;
        const long long local = sl - s_sc[j];
        if (local < s_sc[j + 1] - s_sc[j] - 1) {
          u = __ldg(col + s_st[j] + local);
          if ((unsigned long long)u < (unsigned long long)n)
            claim = levels[u] == -1 && atomicCAS(levels + u, -1, level) == -1;
          else
            atomicOr(&S->err, gsw::DEV_ERR_BAD_VERTEX);
        }
      }
      const unsigned m = __ballot_sync(gsw::FULL, claim);
      if (m) {
        const int leader = __ffs(m) - 1;
        int pos = 0;
        if (gsw::lane_id() == leader) pos = atomicAdd(&S->qsize[c ^ 1], __popc(m));
        pos = __shfl_sync(gsw::FULL, pos, leader);
        const int mine = pos + __popc(m & ((1u << gsw::lane_id()) - 1u));
        if (claim) {
          if (mine < NA_MAX_VERTICES)
            out[mine] = u;
          else
            atomicOr(&S->err, gsw::DEV_ERR_QUEUE_OVERFLOW);
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace

static gsw_status na_run(int64_t n, int64_t m, const int64_t *d_row_off, const int32_t *d_col, int32_t root,
                         int32_t *d_levels, void *stream_handle);

extern "C" gsw_status gsw_bfs_strict_noalloc(int64_t n, int64_t m, const int64_t *d_row_off, const int32_t *d_col,
                                             int32_t root, int32_t *d_levels, void *stream_handle) {
  gsw::clear_error();
  const gsw_status r = na_run(n, m, d_row_off, d_col, root, d_levels, stream_handle);
  if (r != GSW_OK) gsw::g_last_error = gsw::err().msg;
  return r;
}

static gsw_status na_run(int64_t n, int64_t m, const int64_t *d_row_off, const int32_t *d_col, int32_t root,
                         int32_t *d_levels, void *stream_handle) {
  if (n <= 0 || m < 0 || !d_row_off || (m > 0 && !d_col) || !d_levels || root < 0 || root >= n)
    return gsw::set_error(GSW_ERR_INVALID_ARG, "%s", "gsw_bfs_strict_noalloc: bad arguments");
  if (n > NA_MAX_VERTICES)
    return gsw::set_error(GSW_ERR_UNSUPPORTED, "%s",
                          "gsw_bfs_strict_noalloc: more vertices than the fixed scratch holds (max 2^18)");
  if (m > NA_MAX_ARCS)
    return gsw::set_error(GSW_ERR_UNSUPPORTED, "%s",
                          "gsw_bfs_strict_noalloc: more arcs than the fixed scratch holds (max 2^28)");
  int dev = 0;
  if (GSW_CUDA(cudaGetDevice(&dev))) return gsw::err().code;
  na_scratch *S = nullptr;
  if (na_address(dev, &S)) return gsw::err().code;
  cudaStream_t st = (cudaStream_t)stream_handle;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (sms <= 0) sms = 148;
  const int grid_v = (int)((n + 255) / 256 < 4 * sms ? (n + 255) / 256 : 4 * sms);
  k_na_init<<<grid_v, 256, 0, st>>>(S, d_levels, n, root);
  int c = 0;
  int frontier = 1;
  for (int level = 1; frontier > 0 && level <= n; ++level) {
    const int64_t nb = frontier / NA_ITEMS + 1;
    k_na_count<<<(unsigned)nb, NA_THREADS, 0, st>>>(S, c, d_row_off);
    k_na_scan_blocks<<<1, 1024, 0, st>>>(S, nb);
    k_na_scan<<<(unsigned)nb, NA_THREADS, 0, st>>>(S, c, d_row_off, nb);
    k_na_expand<<<4 * sms, NA_THREADS, 0, st>>>(S, c, d_row_off, d_col, d_levels, level, n);
    if (GSW_CUDA(cudaGetLastError())) return gsw::err().code;
    // the finished frontier's counter starts the level after next at zero
    if (GSW_CUDA(cudaMemsetAsync(&S->qsize[c], 0, sizeof(int), st))) return gsw::err().code;
    if (GSW_CUDA(cudaMemcpyAsync(&frontier, &S->qsize[c ^ 1], sizeof(int), cudaMemcpyDeviceToHost, st)))
      return gsw::err().code;
    if (GSW_CUDA(cudaStreamSynchronize(st))) return gsw::err().code;
    c ^= 1;
  }
  unsigned e = 0;
  if (GSW_CUDA(cudaMemcpyAsync(&e, &S->err, sizeof(unsigned), cudaMemcpyDeviceToHost, st))) return gsw::err().code;
  if (GSW_CUDA(cudaStreamSynchronize(st))) return gsw::err().code;
  // a column index outside [0, n) is the caller's CSR at fault, not a
  // capacity problem: the kernel skipped that arc and flagged it
  if (e & gsw::DEV_ERR_BAD_VERTEX)
    return gsw::set_error(GSW_ERR_INVALID_ARG, "%s", "gsw_bfs_strict_noalloc: column index out of range");
  if (e) return gsw::set_error(GSW_ERR_OVERFLOW, "%s", "gsw_bfs_strict_noalloc: scratch bound exceeded");
  return GSW_OK;
}
