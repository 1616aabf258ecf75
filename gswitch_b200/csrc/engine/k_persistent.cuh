// Persistent fused expand: one cooperative launch runs consecutive fused
// levels (expand + enqueue of the next frontier) with a grid-wide barrier
// between levels, instead of one launch and one host round trip per level.
// This is the grid-wide form of the reference's single-CTA __super_fusion
// (src/kernel_libs/kernel_fusion.cuh:111-183, disabled there) and of its
// fused WM expand (src/kernel_libs/expand_VC_WM.cuh:126-232).
//
// Queues ping-pong by level parity; the three size counters rotate by level
// modulo 3, so the counter the next level appends to was last read one full
// barrier earlier and can be cleared without a second barrier.  The launch
// returns to the host when the frontier empties, when it grows past
// `grow_limit` vertices (the selector then reconsiders direction and
// format), after `max_levels` levels, or when a barrier wait exceeds its time
// budget (the error word gets DEV_ERR_BARRIER_TIMEOUT and every block
// returns).
#pragma once
#include "k_expand.cuh"

namespace gsw {

struct persist_state {
  int *q[2];            // queue buffers (q[0] holds the first level's input)
  int *cnt;             // 3 size counters
  int64_t cap;          // queue capacity
  int grow_limit;       // stop when a new frontier exceeds this
  int max_levels;
  unsigned long long budget_ns;  // per barrier wait
  int *levels_done;     // out: levels executed
  int *exit_reason;     // out: 0 empty, 1 growth, 2 level cap, 3 error
  int leave_block;      // test hook: this block leaves before the first
                        // barrier so the others' bounded wait expires (-1: none)
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Sense-free generation barrier over all blocks of a cooperative launch.
// Returns false (in every thread) after a timeout or a recorded error.
__device__ __forceinline__ bool grid_barrier(as_counters_t *c, unsigned &gen, unsigned long long budget_ns) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned target = gen + 1;
    __threadfence();
    const unsigned arrived = atomicAdd(&c->bar_count, 1u) + 1;
    bool okk = true;
    if (arrived == gridDim.x) {
      atomicExch(&c->bar_count, 0u);
      __threadfence();
      atomicExch(&c->bar_gen, target);
    } else {
      const unsigned long long t0 = globaltimer_ns();
      while (ld_acquire_u32(&c->bar_gen) != target) {
        if (ld_acquire_u32(&c->err) & DEV_ERR_BARRIER_TIMEOUT) {
          okk = false;
          break;
        }
        if (globaltimer_ns() - t0 > budget_ns) {
          atomicOr(&c->err, DEV_ERR_BARRIER_TIMEOUT);
          okk = false;
          break;
        }
        __nanosleep(100);
      }
    }
    __threadfence();
    gen = target;
    s_ok = okk;
  }
  __syncthreads();
  // every thread acquires at device scope, so its plain loads of vertex
  // state written by other SMs in the previous level see the new values
  __threadfence();
  return s_ok != 0;
}

// one fused WM level over in[0..n) appending to out / *out_cnt
template <typename G, typename F>
__device__ __forceinline__ void persist_wm_level(active_set_t &as, const G &g, F &f, const config_t &conf,
                                                 const int *in, int64_t n, int *out, int *out_cnt, int64_t cap) {
  constexpr int W = EXPAND_THREADS / 32;
  __shared__ int s_scan[W][32];
  __shared__ int s_v[W][32];
  __shared__ int64_t s_st[W][32];
  __shared__ int s_stage[W][STAGE_SLOTS];
  const int lane = lane_id(), w = warp_id();
  warp_stage_t stage(s_stage[w], out, out_cnt, cap, &as.dg_cnt->err);
  const int64_t nwarps = (int64_t)gridDim.x * W;
  for (int64_t tile = (int64_t)blockIdx.x * W + w; tile * 32 < n; tile += nwarps) {
    const int64_t idx = tile * 32 + lane;
    const int v = idx < n ? in[idx] : -1;
    if (conf.conf_compensation && v >= 0) f.filter(v, g);
    int64_t st;
    int deg;
    vertex_range(g, false, v, st, deg);
    const int incl = warp_inclusive_sum(deg);
    const int total = __shfl_sync(FULL, incl, 31);
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
        tp = push_edge_fused(as, g, f, conf, s_v[w][id], u, ei);
      }
      stage.push(tp, u);
    }
    __syncwarp();
  }
  stage.flush();
}

template <typename G, typename F>
__global__ void __launch_bounds__(EXPAND_THREADS) k_fused_persistent(active_set_t as, G g, F f, config_t conf,
                                                                     persist_state ps) {
  as_counters_t *c = as.dg_cnt;
  unsigned gen = 0;
  int L = 0;
  int reason = 2;
  for (; L < ps.max_levels; ++L) {
    const int n = ((volatile int *)ps.cnt)[L % 3];
    if (n == 0) {
      reason = 0;
      break;
    }
    if (L > 0 && n > ps.grow_limit) {
      reason = 1;
      break;
    }
    // the counter level L+1 appends to is free since the barrier before L
    if (blockIdx.x == 0 && threadIdx.x == 0) ps.cnt[(L + 2) % 3] = 0;
    if (L > 0) g.update_level();
    persist_wm_level(as, g, f, conf, ps.q[L & 1], n, ps.q[(L + 1) & 1], ps.cnt + (L + 1) % 3, ps.cap);
    if ((int)blockIdx.x == ps.leave_block) return;  // never arrives: exercises the timeout path
    if (!grid_barrier(c, gen, ps.budget_ns)) {
      reason = 3;
      break;
    }
    if (!conf.conf_pruning) {
      // patterns that may revisit a vertex: clear the visited bits of the new
      // frontier before the next level marks again
      const int m = ((volatile int *)ps.cnt)[(L + 1) % 3];
      const int *nq = ps.q[(L + 1) & 1];
      for (int64_t i = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; i < m && i < ps.cap;
           i += (int64_t)gridDim.x * blockDim.x) {
        const int u = nq[i];
        atomicAnd(as.bitmap.visited.dg_bits + (u >> 5), ~(1u << (u & 31)));
      }
      if (!grid_barrier(c, gen, ps.budget_ns)) {
        reason = 3;
        ++L;
        break;
      }
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *ps.levels_done = L;
    *ps.exit_reason = reason;
  }
}

// seeds the rotating counters from the Normal queue's current input size
__global__ void k_persist_prep(as_counters_t *c, int cursor) {
  c->pq[0] = c->qsize[cursor];
  c->pq[1] = 0;
  c->pq[2] = 0;
  c->plevels = 0;
  c->preason = -1;
  c->bar_count = 0;
  c->bar_gen = 0;
}

// publishes the persistent launch's last output as the Normal queue's output
__global__ void k_persist_finish(as_counters_t *c, int out_idx, int cursor, int slot) {
  c->qsize[out_idx] = c->pq[slot];
  c->qsize[cursor] = 0;
}

}  // namespace gsw
