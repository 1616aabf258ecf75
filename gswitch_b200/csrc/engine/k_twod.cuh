// 2D-partition (TWOD) expand for patterns where every vertex sends to every
// neighbour (from-all / to-all, e.g. PageRank): wa[v] (+)= emit(u) over all
// in-edges (u -> v).
//
// The reference tiles the adjacency matrix into 3072-vertex panels, keeps
// "heavy" chunks (more than 24,576 edges) apart, stages source values in
// shared memory, writes partial contributions to a stream buffer and reduces
// them per destination panel in a second phase (src/utils/2d_partition.cuh:
// 13-299, src/kernel_libs/expand_VC_TWOD.cuh:12-124).  Here a CTA takes one
// work item - up to TWOD_ITEM_EDGES consecutive edges of one destination tile
// of TILE vertices - and accumulates directly in shared memory, so there is
// no second phase and no stream buffer; a tile split over several items
// (a tile holding hubs) flushes with compAtomic, any other tile with comp:
//   heavy blocks - (destination tile, source tile) pairs with at least
//                  HEAVY edges: the CTA first stages emit() of the whole
//                  source tile in shared memory, then every edge of the block
//                  reads its message from there;
//   light edges  - everything else: the message comes from emit() on the
//                  source vertex (an L2 gather).
// Each edge is one 64-bit word: destination tile | light flag | source tile |
// destination offset | source offset, sorted, so a tile's heavy blocks come
// first, grouped by source tile.  The runtime builds the layout once per
// graph on the device (counts per tile pair, key build, radix sort) and keeps
// it with the graph.
#pragma once
#include "k_expand.cuh"

namespace gsw {

constexpr int TWOD_TILE_BITS = 12;
constexpr int TWOD_TILE = 1 << TWOD_TILE_BITS;  // vertices per tile
constexpr int TWOD_HEAVY = TWOD_TILE;           // edges that make a block heavy
constexpr int TWOD_THREADS = 512;
constexpr int64_t TWOD_ITEM_EDGES = 32768;     // edges per work item

struct twod_layout {
  const uint64_t *edge = nullptr;   // sorted edge words
  const int64_t *tile_off = nullptr;  // per destination tile: first edge, ntiles + 1
  const int64_t *heavy_off = nullptr; // per destination tile: first heavy block, ntiles + 1
  const int64_t *heavy_beg = nullptr; // heavy block i: [heavy_beg[i], heavy_end[i]) of edge[]
  const int64_t *heavy_end = nullptr;
  const int *heavy_src = nullptr;     // heavy block i: its source tile
  int64_t ntiles = 0;
  int64_t nheavy = 0;
  int64_t m = 0;
  // work items: at most TWOD_ITEM_EDGES consecutive edges of one destination
  // tile, so a tile that receives a large share of the edges (the hubs of a
  // skewed graph) is spread over many CTAs
  const int *item_tile = nullptr;
  const int64_t *item_beg = nullptr, *item_end = nullptr;
  const int *tile_items = nullptr;  // items per destination tile (>1: flush atomically)
  int64_t nitems = 0;
};

__host__ __device__ __forceinline__ uint64_t twod_key(uint64_t dt, uint64_t light, uint64_t st, uint64_t dl,
                                                      uint64_t sl) {
  return (dt << 44) | (light << 43) | (st << 24) | (dl << TWOD_TILE_BITS) | sl;
}
__device__ __forceinline__ int twod_src(uint64_t k) {
  return (int)(((k >> 24) & 0x7FFFFull) << TWOD_TILE_BITS | (k & (TWOD_TILE - 1)));
}
__device__ __forceinline__ int twod_dl(uint64_t k) { return (int)((k >> TWOD_TILE_BITS) & (TWOD_TILE - 1)); }
__device__ __forceinline__ int twod_sl(uint64_t k) { return (int)(k & (TWOD_TILE - 1)); }

template <typename G, typename F>
__global__ void __launch_bounds__(TWOD_THREADS) k_twod(G g, F f, twod_layout L) {
  using WA = typename F::wa_t;
  __shared__ WA s_acc[TWOD_TILE];
  __shared__ WA s_src[TWOD_TILE];
  __shared__ bool s_have[TWOD_TILE];
  const int64_t n = g.nvertexs;
  for (int64_t it = blockIdx.x; it < L.nitems; it += gridDim.x) {
    const int64_t dt = L.item_tile[it];
    const int64_t a = L.item_beg[it], b = L.item_end[it];
    const int64_t base_v = dt << TWOD_TILE_BITS;
    for (int i = threadIdx.x; i < TWOD_TILE; i += blockDim.x) {
      s_acc[i] = f.data.zero;
      s_have[i] = false;
    }
    __syncthreads();
    // heavy blocks overlapping [a, b): stage the source tile, then read the
    // messages from shared memory
    const int64_t h0 = L.heavy_off[dt], h1 = L.heavy_off[dt + 1];
    const int64_t light_beg = MAX(a, h1 > h0 ? L.heavy_end[h1 - 1] : L.tile_off[dt]);
    for (int64_t hb = h0; hb < h1; ++hb) {
      const int64_t hbeg = L.heavy_beg[hb], hend = L.heavy_end[hb];
      if (hend <= a) continue;
      if (hbeg >= b) break;
      const int64_t sbase = (int64_t)L.heavy_src[hb] << TWOD_TILE_BITS;
      for (int i = threadIdx.x; i < TWOD_TILE; i += blockDim.x)
        if (sbase + i < n) s_src[i] = f.emit((int)(sbase + i), g.fetch_edata_r(0), g);
      __syncthreads();
      for (int64_t e = MAX(a, hbeg) + threadIdx.x; e < MIN(b, hend); e += blockDim.x) {
        const uint64_t k = __ldg((const unsigned long long *)L.edge + e);
        const int dl = twod_dl(k);
        f.compAtomic(&s_acc[dl], s_src[twod_sl(k)], g);
        s_have[dl] = true;
      }
      __syncthreads();
    }
    // light edges: message straight from the source vertex
    for (int64_t e = light_beg + threadIdx.x; e < b; e += blockDim.x) {
      const uint64_t k = __ldg((const unsigned long long *)L.edge + e);
      const int dl = twod_dl(k);
      f.compAtomic(&s_acc[dl], f.emit(twod_src(k), g.fetch_edata_r(0), g), g);
      s_have[dl] = true;
    }
    __syncthreads();
    const bool shared_tile = L.tile_items[dt] > 1;
    for (int i = threadIdx.x; i < TWOD_TILE; i += blockDim.x)
      if (base_v + i < n && s_have[i]) {
        if (shared_tile)
          f.compAtomic(f.wa_of((int)(base_v + i)), s_acc[i], g);
        else
          f.comp(f.wa_of((int)(base_v + i)), s_acc[i], g);
      }
    __syncthreads();
  }
}

}  // namespace gsw
