// Device-side synthetic graph construction.
//
// Generators draw from a counter-based hash (SplitMix64 finaliser keyed by
// seed, stream and element index) with integer thresholds, so every element
// is reproducible in isolation and the device output is bit-identical to a
// host generator using the same definition:
//   RMAT  : ef * 2^scale pairs; level l picks a quadrant with 32 random bits
//           against thresholds a, a+b, a+b+c and fixes bit (scale-1-l) of
//           (src, dst) - Graph500 Kronecker, no noise, no permutation;
//   grid  : rows x cols 4-neighbour lattice plus (lattice edges / lr_div)
//           uniform long-range pairs;
//   G(n,m): m uniform pairs;
//   power law (configuration model): vertex degrees from P(d) ~ d^-gamma by
//           inversion, stubs shuffled by sorting on hashed keys and paired.
// The undirected CSR build drops self-loops, adds both directions, sorts by
// (src, dst), removes duplicates and derives int64 row offsets - the clean
// form the reference's rinse() produces (src/utils/fileIO.cuh:399-443) except
// that isolated vertices keep their ids.  Sorting and the offset scan use CUB
// from the CUDA toolkit: construction is not on the measured path.
#pragma once
#include <cub/cub.cuh>

#include "engine/common.cuh"

namespace gsw {

__host__ __device__ __forceinline__ uint64_t sm64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__host__ __device__ __forceinline__ uint64_t stream_key(uint64_t seed, uint64_t stream) {
  return sm64(seed ^ sm64(stream));
}
enum gen_stream : uint64_t { ST_RMAT = 1, ST_W = 2, ST_GRID = 3, ST_ER = 4, ST_ERB = 5, ST_PL = 6, ST_ROOT = 7 };

struct rmat_params {
  int scale;
  uint32_t ta, tab, tabc;
  uint64_t key;
};

inline rmat_params make_rmat(int scale, double a, double b, double c, uint64_t seed) {
  rmat_params p;
  p.scale = scale;
  p.ta = (uint32_t)(a * 4294967296.0);
  p.tab = (uint32_t)((a + b) * 4294967296.0);
  p.tabc = (uint32_t)((a + b + c) * 4294967296.0);
  p.key = stream_key(seed, ST_RMAT);
  return p;
}

__device__ __forceinline__ void rmat_pair(const rmat_params &p, uint64_t i, uint32_t &s, uint32_t &d) {
  const uint64_t base = sm64(p.key + i);
  s = 0;
  d = 0;
  uint64_t h = 0;
  for (int l = 0; l < p.scale; ++l) {
    uint32_t r;
    if ((l & 1) == 0) {
      h = sm64(base + (uint64_t)(l >> 1));
      r = (uint32_t)h;
    } else {
      r = (uint32_t)(h >> 32);
    }
    const uint32_t bit = 1u << (p.scale - 1 - l);
    if (r < p.ta) {
    } else if (r < p.tab) {
      d |= bit;
    } else if (r < p.tabc) {
      s |= bit;
    } else {
      s |= bit;
      d |= bit;
    }
  }
}

// both arc directions of pair i (self-loops become the sentinel ~0)
__global__ void k_rmat_keys(rmat_params p, int64_t npairs, uint64_t *keys) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npairs; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t s, d;
    rmat_pair(p, (uint64_t)i, s, d);
    const bool loop = s == d;
    keys[2 * i] = loop ? ~0ull : (((uint64_t)s << 32) | d);
    keys[2 * i + 1] = loop ? ~0ull : (((uint64_t)d << 32) | s);
  }
}

__global__ void k_grid_keys(int rows, int cols, int64_t nlattice, int64_t nlr, uint64_t key, uint64_t *keys) {
  const int64_t total = nlattice + nlr;
  const int64_t hcount = (int64_t)rows * (cols - 1);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t s, d;
    if (i < hcount) {  // horizontal edges (r, c)-(r, c+1)
      const int64_t r = i / (cols - 1), c = i % (cols - 1);
      s = (uint64_t)(r * cols + c);
      d = s + 1;
    } else if (i < nlattice) {  // vertical edges (r, c)-(r+1, c)
      const int64_t j = i - hcount;
      s = (uint64_t)j;
      d = s + (uint64_t)cols;
    } else {
      const uint64_t j = (uint64_t)(i - nlattice);
      const uint64_t n = (uint64_t)rows * (uint64_t)cols;
      s = sm64(key + 2 * j) % n;
      d = sm64(key + 2 * j + 1) % n;
    }
    const bool loop = s == d;
    keys[2 * i] = loop ? ~0ull : ((s << 32) | d);
    keys[2 * i + 1] = loop ? ~0ull : ((d << 32) | s);
  }
}

__global__ void k_er_keys(int64_t n, int64_t m, uint64_t key, uint64_t *keys) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t s = sm64(key + 2 * (uint64_t)i) % (uint64_t)n;
    const uint64_t d = sm64(key + 2 * (uint64_t)i + 1) % (uint64_t)n;
    const bool loop = s == d;
    keys[2 * i] = loop ? ~0ull : ((s << 32) | d);
    keys[2 * i + 1] = loop ? ~0ull : ((d << 32) | s);
  }
}

// power-law degree of v: floor((1 - u)^(-1 / (gamma - 1))), at least 1, at
// most cap, with u uniform in [0, 1) from the vertex's hash
__global__ void k_pl_degrees(int64_t n, double gamma, int64_t cap, uint64_t key, int64_t *deg) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const double u = (double)(sm64(key + (uint64_t)v) >> 11) * (1.0 / 9007199254740992.0);
    double d = floor(pow(1.0 - u, -1.0 / (gamma - 1.0)));
    if (!(d >= 1.0)) d = 1.0;
    deg[v] = (int64_t)(d > (double)cap ? (double)cap : d);
  }
}

// stub i of vertex v (at off[v] + j) gets a random sort key; value = v
__global__ void k_pl_stubs(int64_t n, const int64_t *off, uint64_t key, uint64_t *skey, int *sval) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
    for (int64_t i = off[v]; i < off[v + 1]; ++i) {
      skey[i] = sm64(key + (uint64_t)i);
      sval[i] = (int)v;
    }
}

// consecutive shuffled stubs form an edge (both directions; loops dropped)
__global__ void k_pl_pairs(const int *sval, int64_t npairs, uint64_t *keys) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npairs; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t s = (uint64_t)sval[2 * i], d = (uint64_t)sval[2 * i + 1];
    const bool loop = s == d;
    keys[2 * i] = loop ? ~0ull : ((s << 32) | d);
    keys[2 * i + 1] = loop ? ~0ull : ((d << 32) | s);
  }
}

// A batch of G(n_i, m_i) instances as one disjoint union: instance i owns
// vertices [voff[i], voff[i+1]) and pairs [poff[i], poff[i+1]); its pairs are
// drawn exactly as k_er_keys draws a standalone instance with key ikey[i],
// then shifted by voff[i].
__global__ void k_er_batch_keys(int count, const int64_t *voff, const int64_t *poff, const uint64_t *ikey,
                                uint64_t *keys) {
  const int64_t total = poff[count];
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total; p += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = count;  // instance: last i with poff[i] <= p
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (poff[mid] <= p) lo = mid; else hi = mid;
    }
    const int64_t j = p - poff[lo];
    const uint64_t n = (uint64_t)(voff[lo + 1] - voff[lo]), base = (uint64_t)voff[lo];
    const uint64_t s = sm64(ikey[lo] + 2 * (uint64_t)j) % n + base;
    const uint64_t d = sm64(ikey[lo] + 2 * (uint64_t)j + 1) % n + base;
    const bool loop = s == d;
    keys[2 * p] = loop ? ~0ull : ((s << 32) | d);
    keys[2 * p + 1] = loop ? ~0ull : ((d << 32) | s);
  }
}

// after sorting: keep the first of each run of equal keys, drop sentinels
__global__ void k_unique_flags(const uint64_t *keys, int64_t len, int *flag) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
    flag[i] = keys[i] != ~0ull && (i == 0 || keys[i] != keys[i - 1]);
}

__global__ void k_split_keys(const uint64_t *keys, int64_t m, int *col, unsigned long long *deg) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    col[i] = (int)(k & 0xffffffffu);
    atomicAdd(deg + (k >> 32), 1ull);
  }
}

__global__ void k_deg_to_i32(const int64_t *off, int64_t n, int *odeg) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
    odeg[v] = (int)(off[v + 1] - off[v]);
}

// symmetric per-edge weights 1 + H(min, max) % wmax
__global__ void k_weights(const int64_t *off, const int *col, int64_t n, uint64_t key, int wmax, int *w) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
    for (int64_t e = off[v]; e < off[v + 1]; ++e) {
      const uint64_t u = (uint64_t)col[e];
      const uint64_t lo = (uint64_t)v < u ? (uint64_t)v : u;
      const uint64_t hi = (uint64_t)v < u ? u : (uint64_t)v;
      w[e] = 1 + (int)(sm64(key + ((lo << 32) | hi)) % (uint64_t)wmax);
    }
}

}  // namespace gsw
