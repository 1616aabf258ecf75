// Inspector and frontier builders.
//
// inspect: one pass of f.filter over every vertex (VC) or active edge (EC)
// that writes the status bitmaps with one ballot per warp and reduces the
// six level counters (src/abstraction/inspector.cuh:10-110 defines the
// statuses and counters).  The VC pass keeps the reference's 256 x 512
// grid-stride decomposition on purpose: the two max-degree counters are
// defined by it (per-thread maxima summed per block, then max / sum over
// blocks) and the selector's decision trees were trained on those values.
//
// filter: status bitmaps -> compact queue of Active, Inactive or "unfixed"
// (Active or Inactive) vertices (src/kernel_libs/filter.cuh:30-112).  The
// unsorted builder reserves one slot range per warp with a single atomic;
// the sorted builder emits vertices in id order (block counts, one scan,
// block-offset write), which keeps the following expand's CSR reads ordered.
#pragma once
#include "abstraction.cuh"

namespace gsw {

// The statistics block: [0..5] the counters above, [6] blocks finished,
// [8..8+256) and [264..264+256) the per-virtual-block sums of the two
// max-degree counters.
constexpr int INSPECT_VTHREADS = 256 * 512;  // the reference's grid, one virtual thread each
constexpr int INSPECT_VBLOCK = 512;          // virtual threads per virtual block
constexpr int INSPECT_VPB = 128;             // virtual threads per physical block
constexpr int INSPECT_HALVES = 2;            // physical threads per virtual thread
constexpr int INSPECT_THREADS = INSPECT_VPB * INSPECT_HALVES;
constexpr int INSPECT_CTAS = INSPECT_VTHREADS / INSPECT_VPB;
constexpr int INSPECT_UNROLL = 4;
static_assert(STAT_SLOTS == 8 + 2 * (INSPECT_VTHREADS / INSPECT_VBLOCK), "statistics block layout");
constexpr int EC_INSPECT_CTAS = 256;
constexpr int EC_INSPECT_THREADS = 512;

// Virtual thread t (0 <= t < 131072) visits vertices t, t + 131072, ...
// exactly as thread t of the reference's 256 x 512 grid-stride launch, so the
// max-degree counters are the reference's.  Two physical threads share one
// virtual thread (even / odd steps of its sequence) and merge their maxima
// in shared memory; a physical block holds 128 virtual threads (a quarter
// virtual block), each thread keeps four vertices in flight, vertex counts
// are taken per warp from the ballots, and the last block to finish folds the
// per-virtual-block sums (max over blocks for push, sum for pull).
template <typename G, typename F>
__global__ void __launch_bounds__(INSPECT_THREADS, 7) k_inspect_vc(active_set_t as, G g, F f,
                                                                 unsigned long long *info,
                                                                 const int *skip_if = nullptr) {
  // captured loops: a level whose expand found an empty input ends the loop
  // before this inspection (the host loop stops there too)
  if (skip_if && *(volatile const int *)skip_if) return;
  __shared__ unsigned long long s_red[32];
  __shared__ unsigned s_mp[INSPECT_VPB], s_ml[INSPECT_VPB];
  __shared__ bool s_last;
  const int S = INSPECT_VTHREADS;
  const int half = threadIdx.x / INSPECT_VPB;
  const int vt_local = threadIdx.x % INSPECT_VPB;
  const int t = blockIdx.x * INSPECT_VPB + vt_local;
  const int lane = lane_id();
  const int n = (int)as.size;
  unsigned active_num = 0, inactive_num = 0;  // per warp, kept by lane 0
  unsigned long long push_wl = 0, pull_wl = 0;
  unsigned max_push = 0, max_pull = 0;
  const long long step = (long long)INSPECT_HALVES * S;
  for (long long base = t + (long long)half * S; base - lane < n; base += INSPECT_UNROLL * step) {
    Status st[INSPECT_UNROLL];
    int od[INSPECT_UNROLL];
#pragma unroll
    for (int k = 0; k < INSPECT_UNROLL; ++k) {
      const long long idx = base + k * step;
      od[k] = idx < n ? __ldg(g.dg_odegree + idx) : 0;
    }
#pragma unroll
    for (int k = 0; k < INSPECT_UNROLL; ++k) {
      const long long idx = base + k * step;
      st[k] = idx < n ? f.filter((int)idx, g) : Inactive;
    }
#pragma unroll
    for (int k = 0; k < INSPECT_UNROLL; ++k) {
      const long long idx = base + k * step;
      const long long wbase = idx - lane;
      if (wbase >= n) break;  // warp-uniform
      const bool valid = idx < n;
      const bool tag_active = valid && st[k] == Active;
      const bool tag_inactive = valid && st[k] != Inactive;  // 0 only for Inactive
      const unsigned aw = __ballot_sync(FULL, tag_active);
      const unsigned iw = __ballot_sync(FULL, tag_inactive);
      if (lane == 0) {
        as.bitmap.active.dg_bits[wbase >> 5] = aw;
        as.bitmap.inactive.dg_bits[wbase >> 5] = iw;
        const long long rem = n - wbase;
        const unsigned nvalid = rem >= 32 ? 32u : (unsigned)rem;
        active_num += __popc(aw);
        inactive_num += nvalid - __popc(iw);
      }
      const unsigned oa = tag_active ? (unsigned)od[k] : 0u;
      const unsigned oi = (valid && !tag_inactive) ? (unsigned)od[k] : 0u;
      push_wl += oa;
      pull_wl += oi;
      max_push = max_push > oa ? max_push : oa;
      max_pull = max_pull > oi ? max_pull : oi;
    }
  }
  // merge the two halves of every virtual thread
  if (half == 1) {
    s_mp[vt_local] = max_push;
    s_ml[vt_local] = max_pull;
  }
  __syncthreads();
  unsigned long long vmp = 0, vml = 0;
  if (half == 0) {
    vmp = MAX(max_push, s_mp[vt_local]);
    vml = MAX(max_pull, s_ml[vt_local]);
  }
  unsigned long long r;
  r = block_reduce((unsigned long long)active_num, s_red);
  if (threadIdx.x == 0 && r) atomicAdd(info + 0, r);
  r = block_reduce((unsigned long long)inactive_num, s_red);
  if (threadIdx.x == 0 && r) atomicAdd(info + 1, r);
  r = block_reduce(push_wl, s_red);
  if (threadIdx.x == 0 && r) atomicAdd(info + 2, r);
  r = block_reduce(pull_wl, s_red);
  if (threadIdx.x == 0 && r) atomicAdd(info + 3, r);
  const int vb = t / INSPECT_VBLOCK;
  const int NVB = INSPECT_VTHREADS / INSPECT_VBLOCK;
  r = block_reduce(vmp, s_red);
  if (threadIdx.x == 0 && r) atomicAdd(info + 8 + vb, r);
  r = block_reduce(vml, s_red);
  if (threadIdx.x == 0 && r) atomicAdd(info + 8 + NVB + vb, r);
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(info + 6, 1ull) == (unsigned long long)gridDim.x - 1;
  }
  __syncthreads();
  if (s_last) {  // last block: fold the virtual-block sums
    __threadfence();
    unsigned long long mp = 0, sp = 0;
    for (int i = threadIdx.x; i < NVB; i += blockDim.x) {
      const unsigned long long a = ((volatile unsigned long long *)info)[8 + i];
      mp = MAX(mp, a);
      sp += ((volatile unsigned long long *)info)[8 + NVB + i];
    }
    mp = block_reduce<unsigned long long, true>(mp, s_red);
    sp = block_reduce(sp, s_red);
    if (threadIdx.x == 0) {
      info[4] = mp;
      info[5] = sp;
    }
  }
}

// EC: the active set ranges over edges (inspector.cuh:10-37).  An edge stays
// active while it was active and f.filter still reports Active.
template <typename G, typename F>
__global__ void __launch_bounds__(EC_INSPECT_THREADS) k_inspect_ec(active_set_t as, G g, F f,
                                                                 unsigned long long *info) {
  __shared__ unsigned long long s_red[32];
  const int64_t STRIDE = (int64_t)blockDim.x * gridDim.x;
  const int64_t gtid = threadIdx.x + (int64_t)blockIdx.x * blockDim.x;
  const int lane = lane_id();
  const int64_t n = as.size;
  unsigned long long active_num = 0;
  for (int64_t idx = gtid; idx - lane < n; idx += STRIDE) {
    const bool valid = idx < n;
    const bool prev = valid && as.bitmap.is_active((int)idx);
    bool next = false;
    if (prev) {
      packed_t vv = g.dg_coo[idx];
      next = f.filter((int)(vv >> 32), (int)(vv & 0xffffffffll), (typename G::edge_t *)nullptr) == Active;
    }
    const unsigned aw = __ballot_sync(FULL, next);
    if (lane == 0) as.bitmap.active.dg_bits[idx >> 5] = aw;
    if (prev && next) active_num++;
  }
  unsigned long long r = block_reduce(active_num, s_red);
  if (threadIdx.x == 0 && r) atomicAdd(info + 0, r);
}

// ---- bitmap -> queue ----------------------------------------------------

// status word -> bits of the wanted vertices, with the padding past n masked
__device__ __forceinline__ uint32_t wanted_bits(const active_set_t &as, int64_t word, Status want) {
  const uint32_t a = as.bitmap.active.dg_bits[word];
  const uint32_t i = as.bitmap.inactive.dg_bits[word];
  uint32_t b = want == Active ? a : (want == Inactive ? ~i : (a | ~i));
  const int64_t base = word << 5;
  if (base + 32 > as.size) {
    const int64_t valid = as.size - base;
    b = valid <= 0 ? 0u : (b & (valid >= 32 ? 0xffffffffu : ((1u << valid) - 1u)));
  }
  return b;
}

__device__ __forceinline__ void write_bits(int *out, int64_t pos, uint32_t bits, int64_t base_vertex) {
  while (bits) {
    const int b = __ffs(bits) - 1;
    bits &= bits - 1;
    out[pos++] = (int)(base_vertex + b);
  }
}

// unsorted: one atomic reservation per warp
__global__ void __launch_bounds__(256) k_filter_unsorted(active_set_t as, Status want) {
  const int64_t nwords = (as.size + 31) >> 5;
  const int64_t STRIDE = (int64_t)blockDim.x * gridDim.x;
  int *out = as.queue.output_base();
  for (int64_t w = threadIdx.x + (int64_t)blockIdx.x * blockDim.x; w - lane_id() < nwords; w += STRIDE) {
    const uint32_t bits = w < nwords ? wanted_bits(as, w, want) : 0u;
    const int c = __popc(bits);
    const int incl = warp_inclusive_sum(c);
    const int tot = __shfl_sync(FULL, incl, 31);
    int64_t base = 0;
    if (lane_id() == 31 && tot) base = as.queue.reserve(tot);
    base = __shfl_sync(FULL, base, 31);
    if (base >= 0 && bits) write_bits(out, base + incl - c, bits, w << 5);
  }
}

constexpr int FILTER_WORDS = 256;  // words per block of the sorted builder

__global__ void __launch_bounds__(FILTER_WORDS) k_filter_count(active_set_t as, Status want, int64_t *bsum) {
  __shared__ int64_t s_red[32];
  const int64_t nwords = (as.size + 31) >> 5;
  const int64_t w = (int64_t)blockIdx.x * FILTER_WORDS + threadIdx.x;
  int64_t c = w < nwords ? __popc(wanted_bits(as, w, want)) : 0;
  c = block_reduce(c, s_red);
  if (threadIdx.x == 0) bsum[blockIdx.x] = c;
}

// In-place exclusive scan of a[0..len) by one block; a[len] receives the total.
__global__ void __launch_bounds__(1024) k_scan_single_block(int64_t *a, int64_t len) {
  __shared__ int64_t s[33];
  int64_t carry = 0;
  for (int64_t base = 0; base < len; base += blockDim.x) {
    const int64_t i = base + threadIdx.x;
    int64_t x = i < len ? a[i] : 0;
    int64_t incl = warp_inclusive_sum(x);
    __syncthreads();
    if (lane_id() == 31) s[warp_id()] = incl;
    __syncthreads();
    if (warp_id() == 0) {
      const int nw = blockDim.x >> 5;
      int64_t y = lane_id() < nw ? s[lane_id()] : 0;
      int64_t yi = warp_inclusive_sum(y);
      if (lane_id() < nw) s[lane_id()] = yi - y;
      if (lane_id() == 31) s[32] = yi;
    }
    __syncthreads();
    if (i < len) a[i] = carry + s[warp_id()] + incl - x;
    carry += s[32];
    __syncthreads();
  }
  if (threadIdx.x == 0) a[len] = carry;
}

__global__ void __launch_bounds__(FILTER_WORDS) k_filter_write(active_set_t as, Status want, const int64_t *bsum,
                                                               int64_t nblocks) {
  __shared__ int s_scan[33];
  const int64_t nwords = (as.size + 31) >> 5;
  const int64_t w = (int64_t)blockIdx.x * FILTER_WORDS + threadIdx.x;
  const uint32_t bits = w < nwords ? wanted_bits(as, w, want) : 0u;
  int tot;
  const int ex = block_exclusive_scan(__popc(bits), s_scan, &tot);
  const int64_t pos = bsum[blockIdx.x] + ex;
  const int64_t total = bsum[nblocks];
  int *out = as.queue.output_base();
  if (total > as.queue.output_cap()) {
    if (threadIdx.x == 0 && blockIdx.x == 0) as.raise(DEV_ERR_QUEUE_OVERFLOW);
    return;
  }
  if (bits) write_bits(out, pos, bits, w << 5);
  if (blockIdx.x == 0 && threadIdx.x == 0) *as.queue.output_size() = (int)total;
}

}  // namespace gsw
