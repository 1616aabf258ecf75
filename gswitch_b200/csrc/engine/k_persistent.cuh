// Persistent fused expand: one cooperative launch runs consecutive fused
// levels (expand + enqueue of the next frontier) with a grid-wide barrier
// between levels, instead of one launch and one host round trip per level.
// This is the grid-wide form of the reference's single-CTA __super_fusion
// (src/kernel_libs/kernel_fusion.cuh:111-183, disabled there) and of its
// fused expands, one per load balance: TM (src/kernel_libs/expand_VC_TM.cuh:
// 67-108), WM (expand_VC_WM.cuh:126-232), CM (expand_VC_CM.cuh:12-130) and
// STRICT (expand_VC_STRICT.cuh:59-168), plus this engine's TWC.  Each level
// runs the same body as the per-launch fused kernel of its load balance
// (k_expand.cuh), reading the queue the previous level wrote.
//
// Queues ping-pong by level parity; the three size counters rotate by level
// modulo 3, so the counter the next level appends to was last read one full
// barrier earlier and can be cleared without a second barrier.  STRICT levels
// scan the frontier's degrees inside the launch (two more barriers per
// level).  The launch returns to the host when the frontier empties, when it
// grows past `grow_limit` vertices (the selector then reconsiders direction
// and format), after `max_levels` levels, or when a barrier wait exceeds its
// time budget (the error word gets DEV_ERR_BARRIER_TIMEOUT and every block
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
  int *exit_reason;     // out: 0 empty, 1 growth, 2 level cap, 3 barrier
                        // timeout, 4 STRICT scan capacity exceeded
  int *lb_out;          // out: the kernel's load balance (LB value)
  int cur;              // the Normal queue's input cursor at the launch
  const int *level0;    // captured loops: the first level's number, read at
                        // the start (null: the graph view's own level)
  // zero-copy report (mapped pinned, 3 words: levels, reason + 1, LB), each
  // word tagged with `seq` in its top 24 bits; null: the host copies back
  unsigned long long *sig;
  unsigned long long seq;
  int leave_block;      // test hook: this block leaves before the first
                        // barrier so the others' bounded wait expires (-1: none)
  // STRICT levels: (degree+1) scan of the frontier, per-block chunk sums and
  // the owner of every STRICT_TILE-slot tile
  int64_t *eoff;
  int64_t eoff_cap;
  int64_t *bsum;
  int *tile_lo;
  int64_t tile_cap;
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Sense-free generation barrier over all blocks of a cooperative launch, on
// an arrival counter, a generation word and an error word in global memory.
// Returns false (in every thread) after a timeout or a recorded timeout.
__device__ __forceinline__ bool grid_barrier(unsigned *count, unsigned *genw, unsigned *err, unsigned &gen,
                                             unsigned long long budget_ns) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned target = gen + 1;
    __threadfence();
    const unsigned arrived = atomicAdd(count, 1u) + 1;
    bool okk = true;
    if (arrived == gridDim.x) {
      atomicExch(count, 0u);
      __threadfence();
      atomicExch(genw, target);
    } else {
      const unsigned long long t0 = globaltimer_ns();
      while (ld_acquire_u32(genw) != target) {
        if (ld_acquire_u32(err) & DEV_ERR_BARRIER_TIMEOUT) {
          okk = false;
          break;
        }
        if (globaltimer_ns() - t0 > budget_ns) {
          atomicOr(err, DEV_ERR_BARRIER_TIMEOUT);
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
__device__ __forceinline__ bool grid_barrier(as_counters_t *c, unsigned &gen, unsigned long long budget_ns) {
  return grid_barrier(&c->bar_count, &c->bar_gen, &c->err, gen, budget_ns);
}

// Grid-wide (degree+1) scan of a STRICT level's frontier src[0..n): block b
// owns the contiguous chunk [n*b/G, n*(b+1)/G).  The first pass sums each
// chunk (and applies the deferred filter updates, once per vertex); after a
// barrier every block adds up the chunk sums before its own and scans its
// chunk, four entries per thread, writing eoff and the tile owners with the
// per-launch scan's epilogue; a second barrier publishes them.
template <typename G, typename F>
__device__ bool persist_strict_scan(active_set_t &as, const G &g, F &f, const level_src_t &src, int64_t n,
                                    const persist_state &ps, unsigned &gen) {
  __shared__ int64_t s_red[32];
  __shared__ int64_t s_w[33];
  const int64_t nb = gridDim.x;
  const int64_t c0 = n * blockIdx.x / nb, c1 = n * (blockIdx.x + 1) / nb;
  int64_t s = 0;
  for (int64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
    const int v = src(i);
    src.visit(v, g, f);
    s += strict_slots_of<false>(g, v);
  }
  s = block_reduce(s, s_red);
  if (threadIdx.x == 0) ps.bsum[blockIdx.x] = s;
  if (!grid_barrier(as.dg_cnt, gen, ps.budget_ns)) return false;
  int64_t pre = 0, tot = 0;
  for (int64_t b = threadIdx.x; b < nb; b += blockDim.x) {
    const int64_t x = ((volatile int64_t *)ps.bsum)[b];
    tot += x;
    if (b < (int64_t)blockIdx.x) pre += x;
  }
  pre = block_reduce(pre, s_red);
  tot = block_reduce(tot, s_red);
  const int64_t per = (int64_t)blockDim.x * 4;
  for (int64_t p0 = c0; p0 < c1; p0 += per) {
    const int64_t base = p0 + threadIdx.x * 4;
    int64_t d[4], loc = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      d[k] = base + k < c1 ? strict_slots_of<false>(g, src(base + k)) : 0;
      loc += d[k];
    }
    const int64_t incl = warp_inclusive_sum(loc);
    __syncthreads();
    if (lane_id() == 31) s_w[warp_id()] = incl;
    __syncthreads();
    if (warp_id() == 0) {
      const int nw = (int)(blockDim.x >> 5);
      const int64_t y = lane_id() < nw ? s_w[lane_id()] : 0;
      const int64_t yi = warp_inclusive_sum(y);
      if (lane_id() < nw) s_w[lane_id()] = yi - y;
      if (lane_id() == 31) s_w[32] = yi;
    }
    __syncthreads();
    strict_scan_epilogue<STRICT_TILE>(as, base, c1, d, pre + s_w[warp_id()] + incl - loc, ps.eoff, ps.tile_lo,
                                      ps.tile_cap);
    pre += s_w[32];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) ps.eoff[n] = tot;
  return grid_barrier(as.dg_cnt, gen, ps.budget_ns);
}

template <int LB, typename G, typename F>
__global__ void __launch_bounds__(EXPAND_THREADS) k_fused_persistent(active_set_t as, G g, F f, config_t conf,
                                                                     persist_state ps) {
  __shared__ int s_stage[EXPAND_THREADS / 32][STAGE_SLOTS];
  as_counters_t *c = as.dg_cnt;
  unsigned gen = 0;
  int L = 0;
  int reason = 2;
  if (ps.level0) {  // the levels advance in this launch's own copy
    g.level = *(volatile const int *)ps.level0;
    g.dlevel = nullptr;
  }
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
    if (LB == STRICT && (int64_t)n + 1 >= ps.eoff_cap) {
      if (blockIdx.x == 0 && threadIdx.x == 0) as.raise(DEV_ERR_SCRATCH_OVERFLOW);
      reason = 4;
      break;
    }
    // the counter level L+1 appends to is free since the barrier before L
    if (blockIdx.x == 0 && threadIdx.x == 0) ps.cnt[(L + 2) % 3] = 0;
    if (L > 0) g.update_level();
    const level_src_t src{ps.q[L & 1], conf.conf_compensation};
    warp_stage_t stage(s_stage[warp_id()], ps.q[(L + 1) & 1], ps.cnt + (L + 1) % 3, ps.cap, &c->err);
    if constexpr (LB == TM) {
      push_tm_fused_body(as, g, f, conf, src, n, stage);
    } else if constexpr (LB == CM) {
      push_cm_body<true>(as, g, f, conf, src, n, stage);
    } else if constexpr (LB == TWC) {
      push_twc_body<true>(as, g, f, conf, src, n, stage);
    } else if constexpr (LB == STRICT) {
      if (!persist_strict_scan(as, g, f, src, n, ps, gen)) {
        reason = 3;
        break;
      }
      push_strict_body<true, STRICT_TILE>(as, g, f, conf, level_src_t{ps.q[L & 1], false}, n, ps.eoff, ps.tile_lo,
                                          stage);
    } else {
      push_wm_body<true>(as, g, f, conf, src, n, stage);
    }
    stage.flush();
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
    *ps.lb_out = LB;
    // the last output (q[L & 1], size pq[L % 3]) becomes the Normal queue's
    // output slot, where the next level's swap expects it; the host sets
    // its cursor to out ^ 1
    const int out = ps.cur ^ (L & 1);
    c->qsize[out] = ((volatile int *)c->pq)[L % 3];
    c->qsize[out ^ 1] = 0;
    if (ps.sig) {
      volatile unsigned long long *h = ps.sig;
      const unsigned long long t = ps.seq << 40;
      h[0] = t | (unsigned)L;
      h[1] = t | (unsigned)(reason + 1);
      h[2] = t | (unsigned)LB;
    }
  }
}

// seeds the rotating counters from the Normal queue's current input size
__global__ void k_persist_prep(as_counters_t *c, int cursor) {
  c->pq[0] = c->qsize[cursor];
  c->pq[1] = 0;
  c->pq[2] = 0;
  c->plevels = 0;
  c->preason = -1;
  c->plb = -1;
  c->bar_count = 0;
  c->bar_gen = 0;
}

}  // namespace gsw
