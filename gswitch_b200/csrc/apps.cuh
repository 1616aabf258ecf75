// The seven applications as operators of the engine.
//
// Each functor restates the operator semantics of the reference application
// (file:line per struct); the level loops live in gsw_capi.cu.
#pragma once
#include <climits>

#include "engine/executor.cuh"

namespace gsw {
namespace app {

using GE = device_graph_t<CSR, Empty>;
using GW = device_graph_t<CSR, int>;

// application/bfs.cu:16-36 - level == current level: frontier; -1: not yet
// reached; a message carries the new level.
struct BFS : Functor<VC, int, Empty, Empty> {
  __device__ __forceinline__ Status filter(int v, GE g) {
    const int l = *wa_of(v);
    return l == g.get_level() ? Active : (l < 0 ? Inactive : Fixed);
  }
  __device__ __forceinline__ int emit(int, Empty *, GE g) { return g.get_level(); }
  __device__ __forceinline__ bool cond(int v, int, GE) { return *wa_of(v) == -1; }
  __device__ __forceinline__ bool comp(int *v, int nv, GE) {
    *v = nv;
    return true;
  }
  __device__ __forceinline__ bool compAtomic(int *v, int nv, GE) {
    *v = nv;
    return true;
  }
};

// application/sssp.cu:17-53 - wa = tentative distance, ra = distance at the
// last activation; activation is gated by the stepping window.
struct SSSP : Functor<VC, int, int, int> {
  __device__ __forceinline__ Status filter(int v, GW) {
    int *nd = wa_of(v);
    int *od = ra_of(v);
    if (*nd == *od) return Inactive;
    if (data.win().in((float)*nd)) {
      *od = *nd;
      return Active;
    }
    return Inactive;
  }
  __device__ __forceinline__ int emit(int v, int *w, GW) { return *wa_of(v) + *w; }
  __device__ __forceinline__ bool comp(int *d, int nv, GW) {
    if (*d > nv) {
      *d = nv;
      return data.win().in((float)nv);
    }
    return false;
  }
  __device__ __forceinline__ bool compAtomic(int *v, int nv, GW) {
    const int old = atomicMin(v, nv);
    return old > nv ? data.win().in((float)nv) : false;
  }
  __device__ __forceinline__ bool cond(int v, int msg, GW) { return *wa_of(v) > msg; }
  __device__ __forceinline__ bool exit(int v, GW) { return *wa_of(v) != *ra_of(v); }
};

// application/cc.cu:15-32 - edge-centric hooking of the larger root under
// the smaller one.
struct CC : Functor<EC, int, Empty, Empty> {
  __device__ __forceinline__ Status filter(int v, int u, Empty *) {
    return *wa_of(v) == *wa_of(u) ? Fixed : Active;
  }
  __device__ __forceinline__ void update(int v, int u, Empty *) {
    int *rv = wa_of(*wa_of(v));
    int *ru = wa_of(*wa_of(u));
    const int a = *rv, b = *ru;
    if (a < b)
      atomicMin(ru, a);
    else if (a > b)
      atomicMin(rv, b);
  }
};

// application/pagerank.cu:18-42 - wa accumulates sum(pr/od) of in-neighbours,
// ra holds pr/od (pr for sinks); the filter folds one Jacobi step.
struct PR : Functor<VC, float, float, Empty> {
  float damp = 0.85f;
  float eps = 0.01f;
  __device__ __forceinline__ Status filter(int v, GE g) {
    float *cache = wa_of(v);
    float *pr = ra_of(v);
    const int od = g.get_out_degree(v);
    float newpr = (*cache * damp + 1 - damp);
    if (od) newpr /= od;
    const float err = (newpr - *pr) / (*pr);
    *cache = 0;
    *pr = newpr;
    if (err > -eps && err < eps) return Inactive;
    return Active;
  }
  __device__ __forceinline__ float emit(int v, Empty *, GE) { return *ra_of(v); }
  __device__ __forceinline__ bool comp(float *v, float nv, GE) {
    *v += nv;
    return true;
  }
  __device__ __forceinline__ bool compAtomic(float *v, float nv, GE) {
    atomicAdd(v, nv);
    return true;
  }
};

// Delta-PageRank (the variant described at docs/index.md:178; the reference
// ships no code for it): wa = change accumulated from in-neighbours since the
// vertex last sent, ra = the message it sends to each out-neighbour, pr =
// the PageRank value (the reference's unnormalised form, pr = (1-d) +
// d * sum pr[u]/od[u]).  A vertex whose accumulated change exceeds eps times
// its value adds the change to its value and becomes active; an active
// vertex sends d * change / od to every out-neighbour, which accumulate it.
// Every change is positive, so pr rises monotonically to within
// eps / (1 - d) (normalised L1) of the fixed point.  Activation depends on a
// whole level's accumulated change, which only the inspection's filter pass
// sees, so this functor runs standalone levels only.
struct PRDelta : Functor<VC, float, float, Empty> {
  float damp = 0.85f;
  float eps = 0.01f;
  float *pr = nullptr;
  __device__ __forceinline__ Status filter(int v, GE g) {
    float *acc = wa_of(v);
    const float a = *acc;
    if (!(a > eps * pr[v])) return Inactive;
    *acc = 0;
    pr[v] += a;
    const int od = g.get_out_degree(v);
    *ra_of(v) = od ? damp * a / od : 0.0f;
    return Active;
  }
  __device__ __forceinline__ float emit(int v, Empty *, GE) { return *ra_of(v); }
  __device__ __forceinline__ bool comp(float *v, float nv, GE) {
    *v += nv;
    return true;
  }
  __device__ __forceinline__ bool compAtomic(float *v, float nv, GE) {
    atomicAdd(v, nv);
    return true;
  }
};

// application/bc.cu:175-243 - forward: (level, path count); backward:
// (path count, dependency) with the forward level as read-only data.
struct fwdata_t {
  int level;
  int nsp;
};
struct bwdata_t {
  int nsp;
  float dep;
};

struct BCForward : Functor<VC, fwdata_t, Empty, Empty> {
  __device__ __forceinline__ Status filter(int v, GE g) {
    const fwdata_t *d = wa_of(v);
    if (d->level == g.get_level()) return Active;
    return d->level < 0 ? Inactive : Fixed;
  }
  __device__ __forceinline__ fwdata_t emit(int v, Empty *, GE) {
    fwdata_t d = *wa_of(v);
    d.level++;
    return d;
  }
  __device__ __forceinline__ bool cond(int v, fwdata_t, GE g) {
    return wa_of(v)->level < 0 || wa_of(v)->level == g.get_level();
  }
  __device__ __forceinline__ bool comp(fwdata_t *v, fwdata_t u, GE) {
    v->level = u.level;
    v->nsp += u.nsp;
    return true;
  }
  __device__ __forceinline__ bool compAtomic(fwdata_t *v, fwdata_t u, GE) {
    v->level = u.level;
    atomicAdd(&v->nsp, u.nsp);
    return true;
  }
};

struct BCBackward : Functor<VC, bwdata_t, int, Empty> {
  __device__ __forceinline__ Status filter(int v, GE g) {
    const int l = *ra_of(v);
    if (l == g.get_level()) {
      bwdata_t *d = wa_of(v);
      d->dep = d->nsp * d->dep;
      return Active;
    }
    return l < g.get_level() ? Inactive : Fixed;
  }
  __device__ __forceinline__ bwdata_t emit(int v, Empty *, GE) {
    bwdata_t d = *wa_of(v);
    d.dep = (d.dep + 1) / d.nsp;
    return d;
  }
  __device__ __forceinline__ bool cond(int v, bwdata_t, GE g) { return *ra_of(v) == g.get_level(); }
  __device__ __forceinline__ bool comp(bwdata_t *v, bwdata_t nv, GE) {
    v->dep += nv.dep;
    return true;
  }
  __device__ __forceinline__ bool compAtomic(bwdata_t *v, bwdata_t nv, GE) {
    atomicAdd(&v->dep, nv.dep);
    return true;
  }
};

// application/gc.cu:15-43 - a vertex whose id exceeds every uncoloured
// neighbour's id takes the current level as its colour.
struct GC : Functor<VC, int, int, Empty> {
  __device__ __forceinline__ Status filter(int v, GE g) {
    int *color = ra_of(v);
    int *maxid = wa_of(v);
    if (*color != -1) return Fixed;
    if (*maxid < v) {
      *color = g.get_level();
      return Fixed;
    }
    *maxid = -1;
    return Active;
  }
  __device__ __forceinline__ int emit(int v, Empty *, GE) {
    const int color = *ra_of(v);
    return color == -1 ? v : -1;
  }
  __device__ __forceinline__ bool cond(int v, int, GE) { return *ra_of(v) == -1; }
  __device__ __forceinline__ bool comp(int *v, int m, GE) {
    if (*v < m) *v = m;
    return true;
  }
  __device__ __forceinline__ bool compAtomic(int *v, int m, GE) {
    atomicMax(v, m);
    return true;
  }
};

}  // namespace app
}  // namespace gsw
