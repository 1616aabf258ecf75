// Learned variant selector: a small FP32 multilayer perceptron
//   8 features -> 32 (ReLU) -> 32 (ReLU) -> 20 variant logits
// over the inspector's per-level statistics.  It has no counterpart in the
// reference, whose selector is a set of trained decision trees
// (src/abstraction/selector.cuh:22-303, src/model/select_*.h); those stay as
// the rule-based selector and as the fallback when no model is loaded or the
// network is not confident.
//
// The 20 classes are the standalone variants {Push, Pull} x {Queue, Bitmap}
// x {TM, WM, CM, STRICT, TWC}; fusion stays with the rules (trigger_fusion /
// select_fusion), which decide whether a level is inspected at all.
//
// Everything here is hand-written: host inference (the host-driven loop), a
// warp-level device inference (one lane per hidden unit; the captured loop
// runs it in-stream), and the training forward/backward and Adam kernels.
#pragma once
#include <cmath>

#include "executor.cuh"

namespace gsw {

constexpr int MLP_IN = 8;
constexpr int MLP_H = 32;
constexpr int MLP_K = 20;
constexpr int MLP_LBS = 5;
// parameter block: W1[H][IN] b1[H] W2[H][H] b2[H] W3[K][H] b3[K]
constexpr int MLP_W1 = 0;
constexpr int MLP_B1 = MLP_W1 + MLP_H * MLP_IN;
constexpr int MLP_W2 = MLP_B1 + MLP_H;
constexpr int MLP_B2 = MLP_W2 + MLP_H * MLP_H;
constexpr int MLP_W3 = MLP_B2 + MLP_H;
constexpr int MLP_B3 = MLP_W3 + MLP_K * MLP_H;
constexpr int MLP_NPARAM = MLP_B3 + MLP_K;  // 2004

// a loaded model: parameters plus the feature normalisation of its corpus
struct mlp_model {
  float p[MLP_NPARAM];
  float mean[MLP_IN], inv_std[MLP_IN];
  float min_conf;  // below this top-class probability the rules decide
  int valid;
};

__host__ __device__ inline LB mlp_lb(int i) {
  return i == 0 ? TM : i == 1 ? WM : i == 2 ? CM : i == 3 ? STRICT : TWC;
}
__host__ __device__ inline int mlp_lb_index(LB lb) {
  return lb == TM ? 0 : lb == WM ? 1 : lb == CM ? 2 : lb == STRICT ? 3 : lb == TWC ? 4 : -1;
}
// class k <-> (direction, format, load balance)
__host__ __device__ inline int mlp_class(Direction d, ASFmt a, LB lb) {
  const int l = mlp_lb_index(lb);
  return l < 0 ? -1 : ((d == Pull) * 2 + (a == Bitmap)) * MLP_LBS + l;
}
__host__ __device__ inline void mlp_variant(int k, Direction &d, ASFmt &a, LB &lb) {
  d = (k / MLP_LBS) >= 2 ? Pull : Push;
  a = ((k / MLP_LBS) & 1) ? Bitmap : Queue;
  lb = mlp_lb(k % MLP_LBS);
}

__host__ __device__ inline float mlp_log2p1(double x) { return (float)log2(1.0 + (x > 0 ? x : 0.0)); }

// The 8 features, from the flattened (and cross-folded) feature vector the
// rules see: frontier vertices and edges, unvisited edges and fraction,
// frontier degree skew, graph degree and skew, and the update pattern.
__host__ __device__ inline void mlp_features(const feature_t &f, float *x) {
  const double *fv = f.fv;
  x[0] = mlp_log2p1(fv[7]);   // frontier vertices
  x[1] = mlp_log2p1(fv[9]);   // frontier (push) edges
  x[2] = mlp_log2p1(fv[10]);  // unvisited (pull) edges
  x[3] = (float)fv[12];       // unvisited fraction
  x[4] = mlp_log2p1(fv[17]);  // largest frontier degree
  x[5] = mlp_log2p1(fv[2]);   // mean degree
  x[6] = mlp_log2p1(fv[2] > 0 ? fv[3] / fv[2] : 0.0);  // degree skew (std / mean)
  x[7] = f.pattern == Idem ? 0.f : (f.pattern == Mono ? 0.5f : 1.f);
}

// The rules decide first (fusion, and a from-all/to-all pattern keeping its
// first choice); the network re-decides direction, format and load balance
// of an inspected standalone level of a vertex-centric run.  Forced choices
// always win.
__host__ __device__ inline bool mlp_applicable(const mlp_model &m, const feature_t &fets, const config_t &conf) {
  return m.valid && fets.centric == VC && !conf.conf_fuse_inspect && !conf.conf_inherit && conf.conf_lb != TWOD;
}
__host__ __device__ inline void mlp_apply(int k, config_t &conf) {
  Direction d;
  ASFmt a;
  LB lb;
  mlp_variant(k, d, a, lb);
  conf.conf_dir = conf.force.has_direction ? conf.force.d : d;
  conf.conf_asfmt = conf.force.has_asfmt ? conf.force.asf : a;
  conf.conf_lb = conf.force.has_lb ? conf.force.lb : lb;
  selector_t::set_target(conf);
}

// Graph-level features for the fusion decision of a run (the quantities the
// reference's select_fusion tree reads, log-scaled, plus size and pattern).
// Class 0 = standalone levels, class 1 = fused levels.
__host__ __device__ inline void mlp_fusion_features(const feature_t &f, float *x) {
  x[0] = mlp_log2p1(f.avg_deg);
  x[1] = mlp_log2p1(f.std_deg);
  x[2] = mlp_log2p1(f.range);
  x[3] = (float)f.GI;
  x[4] = (float)f.Her;
  x[5] = mlp_log2p1((double)f.nvertexs);
  x[6] = mlp_log2p1((double)f.nedges);
  x[7] = f.pattern == Idem ? 0.f : (f.pattern == Mono ? 0.5f : 1.f);
}

// forward pass on the host (the device warp version below computes the same
// sums in the same order)
inline int mlp_predict_host(const mlp_model &m, const float *xin, float *prob_top) {
  float x[MLP_IN], h1[MLP_H], h2[MLP_H], z[MLP_K];
  for (int i = 0; i < MLP_IN; ++i) x[i] = (xin[i] - m.mean[i]) * m.inv_std[i];
  for (int o = 0; o < MLP_H; ++o) {
    float a = m.p[MLP_B1 + o];
    for (int i = 0; i < MLP_IN; ++i) a += m.p[MLP_W1 + o * MLP_IN + i] * x[i];
    h1[o] = a > 0 ? a : 0;
  }
  for (int o = 0; o < MLP_H; ++o) {
    float a = m.p[MLP_B2 + o];
    for (int i = 0; i < MLP_H; ++i) a += m.p[MLP_W2 + o * MLP_H + i] * h1[i];
    h2[o] = a > 0 ? a : 0;
  }
  int best = 0;
  for (int k = 0; k < MLP_K; ++k) {
    float a = m.p[MLP_B3 + k];
    for (int i = 0; i < MLP_H; ++i) a += m.p[MLP_W3 + k * MLP_H + i] * h2[i];
    z[k] = a;
    if (z[k] > z[best]) best = k;
  }
  if (prob_top) {
    double s = 0;
    for (int k = 0; k < MLP_K; ++k) s += std::exp((double)z[k] - z[best]);
    *prob_top = (float)(1.0 / s);
  }
  return best;
}

// ---------------------------------------------------------------------------
// device inference: one warp, lane o holds hidden unit o (and logit o for
// o < K); the layers exchange activations by shuffles.  Products and sums are
// rounded one by one (no fused multiply-add), in the host's order, so the
// device and the host pick the same class from the same features.
// ---------------------------------------------------------------------------
__device__ inline int mlp_predict_warp(const mlp_model &m, const float *xin, float *prob_top) {
  const int lane = threadIdx.x & 31;
  float x[MLP_IN];
#pragma unroll
  for (int i = 0; i < MLP_IN; ++i) x[i] = __fmul_rn(__fsub_rn(xin[i], m.mean[i]), m.inv_std[i]);
  float a = m.p[MLP_B1 + lane];
#pragma unroll
  for (int i = 0; i < MLP_IN; ++i) a = __fadd_rn(a, __fmul_rn(m.p[MLP_W1 + lane * MLP_IN + i], x[i]));
  const float h1 = a > 0 ? a : 0;
  a = m.p[MLP_B2 + lane];
#pragma unroll
  for (int i = 0; i < MLP_H; ++i)
    a = __fadd_rn(a, __fmul_rn(m.p[MLP_W2 + lane * MLP_H + i], __shfl_sync(FULL, h1, i)));
  const float h2 = a > 0 ? a : 0;
  float z = -INFINITY;
  const int k = lane < MLP_K ? lane : MLP_K - 1;
  a = m.p[MLP_B3 + k];
#pragma unroll
  for (int i = 0; i < MLP_H; ++i)
    a = __fadd_rn(a, __fmul_rn(m.p[MLP_W3 + k * MLP_H + i], __shfl_sync(FULL, h2, i)));
  if (lane < MLP_K) z = a;
  // argmax, lowest class on ties (the host's strict '>' scan)
  float bz = z;
  int bk = lane;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    const float oz = __shfl_xor_sync(FULL, bz, d);
    const int ok = __shfl_xor_sync(FULL, bk, d);
    if (oz > bz || (oz == bz && ok < bk)) {
      bz = oz;
      bk = ok;
    }
  }
  if (prob_top) {
    double e = lane < MLP_K ? exp((double)z - bz) : 0.0;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) e += __shfl_xor_sync(FULL, e, d);
    *prob_top = (float)(1.0 / e);
  }
  return bk;
}

// one warp per sample
__global__ void k_mlp_infer(const mlp_model *m, const float *X, int64_t n, int *cls, float *prob) {
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= n) return;  // warp-uniform
  float pt;
  const int c = mlp_predict_warp(*m, X + w * MLP_IN, &pt);
  if ((threadIdx.x & 31) == 0) {
    cls[w] = c;
    if (prob) prob[w] = pt;
  }
}

// ---------------------------------------------------------------------------
// training.  Loss per sample: cross entropy against soft labels that favour
// fast variants, q_k ~ exp(-(t_k / t_min - 1) / tau) over the timed variants
// (q_k = 0 for a variant without a time).  One thread per sample runs the
// forward and backward pass; gradients meet in shared memory, then in the
// global gradient block.
// ---------------------------------------------------------------------------
__global__ void k_mlp_soft_labels(const float *T, int64_t n, float tau, float *Q) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float *t = T + i * MLP_K;
    float tmin = INFINITY;
    for (int k = 0; k < MLP_K; ++k)
      if (t[k] > 0 && t[k] < tmin) tmin = t[k];
    double s = 0;
    double q[MLP_K];
    for (int k = 0; k < MLP_K; ++k) {
      q[k] = (t[k] > 0 && tmin < INFINITY) ? exp(-((double)t[k] / tmin - 1.0) / tau) : 0.0;
      s += q[k];
    }
    for (int k = 0; k < MLP_K; ++k) Q[i * MLP_K + k] = s > 0 ? (float)(q[k] / s) : 0.f;
  }
}

// normalised inputs of sample i
__device__ __forceinline__ void mlp_norm_x(const float *X, int64_t i, const float *mean, const float *inv_std,
                                           float *x) {
#pragma unroll
  for (int j = 0; j < MLP_IN; ++j) x[j] = (X[i * MLP_IN + j] - mean[j]) * inv_std[j];
}

constexpr int MLP_TRAIN_THREADS = 128;

// grad += d(mean loss)/d(params) over samples [0, n); *loss += mean loss
__global__ void __launch_bounds__(MLP_TRAIN_THREADS) k_mlp_grad(const float *P, const float *mean,
                                                               const float *inv_std, const float *X,
                                                               const float *Q, int64_t n, float *grad,
                                                               float *loss) {
  __shared__ float s_g[MLP_NPARAM];
  __shared__ float s_loss;
  for (int i = threadIdx.x; i < MLP_NPARAM; i += blockDim.x) s_g[i] = 0;
  if (threadIdx.x == 0) s_loss = 0;
  __syncthreads();
  const float inv_n = 1.0f / (float)n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float x[MLP_IN], h1[MLP_H], h2[MLP_H], z[MLP_K];
    mlp_norm_x(X, i, mean, inv_std, x);
    for (int o = 0; o < MLP_H; ++o) {
      float a = P[MLP_B1 + o];
      for (int j = 0; j < MLP_IN; ++j) a += P[MLP_W1 + o * MLP_IN + j] * x[j];
      h1[o] = a > 0 ? a : 0;
    }
    for (int o = 0; o < MLP_H; ++o) {
      float a = P[MLP_B2 + o];
      for (int j = 0; j < MLP_H; ++j) a += P[MLP_W2 + o * MLP_H + j] * h1[j];
      h2[o] = a > 0 ? a : 0;
    }
    float zmax = -INFINITY;
    for (int k = 0; k < MLP_K; ++k) {
      float a = P[MLP_B3 + k];
      for (int j = 0; j < MLP_H; ++j) a += P[MLP_W3 + k * MLP_H + j] * h2[j];
      z[k] = a;
      zmax = fmaxf(zmax, a);
    }
    float se = 0;
    for (int k = 0; k < MLP_K; ++k) se += __expf(z[k] - zmax);
    const float lse = zmax + __logf(se);
    float l = 0;
    // dz = (softmax - q) / n, kept in z
    for (int k = 0; k < MLP_K; ++k) {
      const float q = Q[i * MLP_K + k];
      l -= q * (z[k] - lse);
      z[k] = (__expf(z[k] - lse) - q) * inv_n;
    }
    atomicAdd(&s_loss, l * inv_n);
    float d2[MLP_H];
    for (int j = 0; j < MLP_H; ++j) d2[j] = 0;
    for (int k = 0; k < MLP_K; ++k) {
      atomicAdd(&s_g[MLP_B3 + k], z[k]);
      for (int j = 0; j < MLP_H; ++j) {
        atomicAdd(&s_g[MLP_W3 + k * MLP_H + j], z[k] * h2[j]);
        d2[j] += P[MLP_W3 + k * MLP_H + j] * z[k];
      }
    }
    float d1[MLP_H];
    for (int j = 0; j < MLP_H; ++j) d1[j] = 0;
    for (int o = 0; o < MLP_H; ++o) {
      const float g = h2[o] > 0 ? d2[o] : 0.f;
      if (g == 0.f) continue;
      atomicAdd(&s_g[MLP_B2 + o], g);
      for (int j = 0; j < MLP_H; ++j) {
        atomicAdd(&s_g[MLP_W2 + o * MLP_H + j], g * h1[j]);
        d1[j] += P[MLP_W2 + o * MLP_H + j] * g;
      }
    }
    for (int o = 0; o < MLP_H; ++o) {
      const float g = h1[o] > 0 ? d1[o] : 0.f;
      if (g == 0.f) continue;
      atomicAdd(&s_g[MLP_B1 + o], g);
      for (int j = 0; j < MLP_IN; ++j) atomicAdd(&s_g[MLP_W1 + o * MLP_IN + j], g * x[j]);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < MLP_NPARAM; i += blockDim.x)
    if (s_g[i] != 0.f) atomicAdd(grad + i, s_g[i]);
  if (threadIdx.x == 0) atomicAdd(loss, s_loss);
}

// Adam step (beta1 0.9, beta2 0.999), step number t >= 1
__global__ void k_mlp_adam(float *P, const float *grad, float *m1, float *m2, int t, float lr, float wd) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= MLP_NPARAM) return;
  const float g = grad[i] + wd * P[i];
  m1[i] = 0.9f * m1[i] + 0.1f * g;
  m2[i] = 0.999f * m2[i] + 0.001f * g * g;
  const float mh = m1[i] / (1.f - powf(0.9f, (float)t));
  const float vh = m2[i] / (1.f - powf(0.999f, (float)t));
  P[i] -= lr * mh / (sqrtf(vh) + 1e-8f);
}

}  // namespace gsw
