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
// max-degree counters.  Behind it (never cleared by the host) the inspection
// keeps its merge scratch: per-virtual-thread maxima for push and pull and a
// per-virtual-block count of finished steps, all zero between launches.
constexpr int INSPECT_VTHREADS = 256 * 512;  // the reference's grid, one virtual thread each
constexpr int INSPECT_VBLOCK = 512;          // virtual threads per virtual block
constexpr int INSPECT_NVB = INSPECT_VTHREADS / INSPECT_VBLOCK;
constexpr int INSPECT_SPAN = 4;              // consecutive vertices a physical thread takes per step
constexpr int INSPECT_OWNERS = INSPECT_VBLOCK / INSPECT_SPAN;  // 128 threads cover one virtual block
#ifndef GSW_INSPECT_PARTS
#define GSW_INSPECT_PARTS 2
#endif
constexpr int INSPECT_PARTS = GSW_INSPECT_PARTS;  // thread groups of a CTA taking alternate steps
constexpr int INSPECT_THREADS = INSPECT_OWNERS * INSPECT_PARTS;
constexpr int INSPECT_SCRATCH_U32 = 2 * INSPECT_VTHREADS + INSPECT_NVB;
constexpr int INSPECT_SCRATCH_U64 = (INSPECT_SCRATCH_U32 + 1) / 2;
#ifndef GSW_INSPECT_UNROLL
#define GSW_INSPECT_UNROLL 2
#endif
#ifndef GSW_INSPECT_MINBLOCKS
#define GSW_INSPECT_MINBLOCKS 4
#endif
constexpr int INSPECT_UNROLL = GSW_INSPECT_UNROLL;
static_assert(STAT_SLOTS == 8 + 2 * INSPECT_NVB, "statistics block layout");
static_assert(STAT_SCRATCH == INSPECT_SCRATCH_U64, "inspection scratch layout");
constexpr int INSPECT_REPORT_BITS = 40;  // value bits of a zero-copy report word
constexpr unsigned long long INSPECT_REPORT_MASK = (1ull << INSPECT_REPORT_BITS) - 1;
constexpr int EC_INSPECT_CTAS = 256;
constexpr int EC_INSPECT_THREADS = 512;

// steps of the reference's grid-stride loop: virtual thread t visits
// t + k * 131072 for k < inspect_steps(n)
__host__ __device__ __forceinline__ unsigned inspect_steps(int64_t n) {
  const int64_t k = (n + INSPECT_VTHREADS - 1) / INSPECT_VTHREADS;
  return k > 0 ? (unsigned)k : 1u;
}
// work units (virtual block, step): 512 consecutive vertices each
__host__ __device__ __forceinline__ int64_t inspect_units(int64_t n) { return (int64_t)INSPECT_NVB * inspect_steps(n); }

// Virtual thread t (0 <= t < 131072) visits vertices t, t + 131072, ...
// exactly as thread t of the reference's 256 x 512 grid-stride launch, so the
// max-degree counters are the reference's.  The work is cut into units
// (virtual block b, step k) = vertices b*512 + k*131072 + [0, 512); CTA c of
// the (resident-sized) grid takes units [c*U/G, (c+1)*U/G) in b-major order,
// so every SM gets the same share whatever the graph size.  Inside a unit,
// owner thread q reads vertices 4q .. 4q+3 (virtual threads 4q .. 4q+3 of b;
// a warp covers 128 consecutive vertices: four bitmap words, built with
// shuffles) and the CTA's two thread groups take alternate steps.  At the end
// of each run of units of one virtual block (a segment) the CTA folds its
// per-virtual-thread maxima into the global scratch with atomicMax and adds
// the segment's step count to the block's counter; the CTA that completes a
// virtual block sums its 512 maxima, clears the scratch and folds the sum
// into the push (max over blocks) and pull (sum over blocks) counters; the
// last CTA to finish only reports.  All vertex arithmetic is 32-bit (vertex
// ids are below 2^31), and units that lie wholly below n take a path without
// per-vertex bounds checks.
template <typename G, typename F>
__global__ void __launch_bounds__(INSPECT_THREADS, GSW_INSPECT_MINBLOCKS)
    k_inspect_vc(active_set_t as, G g, F f, unsigned long long *info, const int *skip_if = nullptr,
                 unsigned long long *sig = nullptr, unsigned long long seq = 0) {
  // captured loops: a level whose expand found an empty input ends the loop
  // before this inspection (the host loop stops there too)
  if (skip_if && *(volatile const int *)skip_if) return;
  __shared__ unsigned long long s_red[32];
  __shared__ unsigned s_mp[INSPECT_OWNERS][INSPECT_SPAN], s_ml[INSPECT_OWNERS][INSPECT_SPAN];
  __shared__ int s_fold;
  __shared__ bool s_last;
  unsigned *vmax = reinterpret_cast<unsigned *>(info + STAT_SLOTS);  // [2][INSPECT_VTHREADS]
  unsigned *vdone = vmax + 2 * INSPECT_VTHREADS;                      // [INSPECT_NVB]
  constexpr unsigned S = INSPECT_VTHREADS;
  const unsigned n = (unsigned)as.size;
  const unsigned K = inspect_steps(as.size);
  const unsigned long long U = (unsigned long long)INSPECT_NVB * K;
  const unsigned long long lo = U * blockIdx.x / gridDim.x, hi = U * (blockIdx.x + 1) / gridDim.x;
  const unsigned part = threadIdx.x / INSPECT_OWNERS;
  const unsigned q = threadIdx.x % INSPECT_OWNERS;
  const unsigned lane = lane_id();
  unsigned active_num = 0, inactive_num = 0;
  unsigned long long push_wl = 0, pull_wl = 0;

  for (unsigned long long u = lo; u < hi;) {
    const unsigned b = (unsigned)(u / K);
    const unsigned k0 = (unsigned)(u % K);
    const unsigned k1 = (unsigned)MIN((unsigned long long)K, k0 + (hi - u));  // segment: steps [k0, k1) of b
    const unsigned vq = b * INSPECT_VBLOCK + INSPECT_SPAN * q;  // this thread's first vertex of step 0
    unsigned mp[INSPECT_SPAN] = {0, 0, 0, 0}, ml[INSPECT_SPAN] = {0, 0, 0, 0};

    // UNROLL steps k, k + PARTS, ...; FULLU: all of them exist and lie below n
    auto steps = [&](auto full_tag, unsigned k) {
      constexpr bool FULLU = decltype(full_tag)::value;
      int od[INSPECT_UNROLL][INSPECT_SPAN];
      Status st[INSPECT_UNROLL][INSPECT_SPAN];
#pragma unroll
      for (int j = 0; j < INSPECT_UNROLL; ++j) {
        const unsigned kj = k + j * INSPECT_PARTS;
        const unsigned v = vq + kj * S;  // a multiple of 4: 16-byte aligned
        if (FULLU || (kj < k1 && v + 3 < n)) {
          const int4 d4 = __ldg(reinterpret_cast<const int4 *>(g.dg_odegree + v));
          od[j][0] = d4.x, od[j][1] = d4.y, od[j][2] = d4.z, od[j][3] = d4.w;
        } else {
#pragma unroll
          for (int i = 0; i < INSPECT_SPAN; ++i) od[j][i] = (kj < k1 && v + i < n) ? __ldg(g.dg_odegree + v + i) : 0;
        }
      }
#pragma unroll
      for (int j = 0; j < INSPECT_UNROLL; ++j) {
        const unsigned kj = k + j * INSPECT_PARTS;
        const unsigned v = vq + kj * S;
#pragma unroll
        for (int i = 0; i < INSPECT_SPAN; ++i)
          st[j][i] = (FULLU || (kj < k1 && v + i < n)) ? f.filter((int)(v + i), g) : Inactive;
      }
#pragma unroll
      for (int j = 0; j < INSPECT_UNROLL; ++j) {
        const unsigned kj = k + j * INSPECT_PARTS;
        const unsigned v0 = vq + kj * S;
        if (!FULLU && (kj >= k1 || v0 - INSPECT_SPAN * lane >= n)) break;  // warp-uniform
        unsigned na = 0, ni = 0, oa[INSPECT_SPAN], oi[INSPECT_SPAN];
#pragma unroll
        for (int i = 0; i < INSPECT_SPAN; ++i) {
          const bool tag_active = st[j][i] == Active;
          const bool tag_inactive = st[j][i] != Inactive;  // 0 only for Inactive
          na |= (unsigned)tag_active << i;
          ni |= (unsigned)tag_inactive << i;
          oa[i] = tag_active ? (unsigned)od[j][i] : 0u;
          oi[i] = tag_inactive ? 0u : (unsigned)od[j][i];
          mp[i] = max(mp[i], oa[i]);
          ml[i] = max(ml[i], oi[i]);
        }
        // degrees are below 2^31, so a pair sums without overflow in 32 bits
        push_wl += (unsigned long long)(oa[0] + oa[1]) + (oa[2] + oa[3]);
        pull_wl += (unsigned long long)(oi[0] + oi[1]) + (oi[2] + oi[3]);
        active_num += __popc(na);
        // out-of-range vertices have status Inactive and degree 0, so only
        // the count of valid vertices needs the bound
        unsigned nvalid = INSPECT_SPAN;
        if (!FULLU && v0 + INSPECT_SPAN > n) nvalid = v0 < n ? n - v0 : 0u;
        inactive_num += nvalid - (unsigned)__popc(ni & ((1u << nvalid) - 1u));
        // lanes 8j .. 8j+7 hold the 32 vertices of bitmap word j of the warp
        unsigned wa = na << (4 * (lane & 7)), wi = ni << (4 * (lane & 7));
#pragma unroll
        for (int d = 1; d < 8; d <<= 1) {
          wa |= __shfl_xor_sync(FULL, wa, d);
          wi |= __shfl_xor_sync(FULL, wi, d);
        }
        if ((lane & 7) == 0 && (FULLU || v0 < n)) {
          as.bitmap.active.dg_bits[v0 >> 5] = wa;
          as.bitmap.inactive.dg_bits[v0 >> 5] = wi;
        }
      }
    };
    for (unsigned k = k0 + part; k < k1; k += INSPECT_PARTS * INSPECT_UNROLL) {
      const unsigned klast = k + (INSPECT_UNROLL - 1) * INSPECT_PARTS;
      // the last step's unit ends at or below n: every vertex is valid
      if (klast < k1 && b * INSPECT_VBLOCK + klast * S + INSPECT_VBLOCK <= n)
        steps(std::true_type{}, k);
      else
        steps(std::false_type{}, k);
    }

    // fold the segment: the other groups hand their maxima to group 0,
    // which publishes
    for (unsigned h = 1; h < INSPECT_PARTS; ++h) {
      if (part == h)
#pragma unroll
        for (int i = 0; i < INSPECT_SPAN; ++i)
          s_mp[q][i] = h == 1 ? mp[i] : max(s_mp[q][i], mp[i]), s_ml[q][i] = h == 1 ? ml[i] : max(s_ml[q][i], ml[i]);
      __syncthreads();
    }
    if (part == 0) {
      unsigned *vp = vmax + b * INSPECT_VBLOCK + INSPECT_SPAN * q;
#pragma unroll
      for (int i = 0; i < INSPECT_SPAN; ++i) {
        const unsigned a = INSPECT_PARTS > 1 ? max(mp[i], s_mp[q][i]) : mp[i];
        const unsigned c = INSPECT_PARTS > 1 ? max(ml[i], s_ml[q][i]) : ml[i];
        if (a) atomicMax(vp + i, a);
        if (c) atomicMax(vp + INSPECT_VTHREADS + i, c);
      }
    }
    __syncthreads();  // every maximum is issued before the count, and s_mp is free
    if (threadIdx.x == 0) {
      __threadfence();
      s_fold = atomicAdd(vdone + b, k1 - k0) + (k1 - k0) == K;
    }
    __syncthreads();
    if (s_fold) {  // this CTA completed virtual block b
      __threadfence();
      unsigned long long sp = 0, sl = 0;
      for (int t = threadIdx.x; t < INSPECT_VBLOCK; t += blockDim.x) {
        sp += atomicExch(vmax + b * INSPECT_VBLOCK + t, 0u);
        sl += atomicExch(vmax + INSPECT_VTHREADS + b * INSPECT_VBLOCK + t, 0u);
      }
      sp = block_reduce(sp, s_red);
      sl = block_reduce(sl, s_red);
      if (threadIdx.x == 0) {
        info[8 + b] = sp;
        info[8 + INSPECT_NVB + b] = sl;
        // fold into the two counters now (max over blocks for push, sum for
        // pull: order-free on integers), so the last CTA has nothing left
        if (sp) atomicMax(info + 4, sp);
        if (sl) atomicAdd(info + 5, sl);
        vdone[b] = 0;
      }
    }
    u += k1 - k0;
  }

  // the four counters in one block reduction
  {
    unsigned long long c4[4] = {active_num, inactive_num, push_wl, pull_wl};
    __shared__ unsigned long long s_c4[INSPECT_THREADS / 32][4];
#pragma unroll
    for (int i = 0; i < 4; ++i) c4[i] = warp_sum(c4[i]);
    if (lane == 0)
#pragma unroll
      for (int i = 0; i < 4; ++i) s_c4[warp_id()][i] = c4[i];
    __syncthreads();
    if (threadIdx.x < 4) {
      unsigned long long t = 0;
      for (int w = 0; w < INSPECT_THREADS / 32; ++w) t += s_c4[w][threadIdx.x];
      if (t) atomicAdd(info + threadIdx.x, t);
      __threadfence();
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(info + 6, 1ull) == (unsigned long long)gridDim.x - 1;
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {  // last block: every counter is final
    __threadfence();
    if (sig) {
      // Report to the mapped host block and leave zeroed counters behind.
      // Every counter is below 2^40 (each is bounded by the arc count), so
      // each report word carries the launch's tag in its top 24 bits and the
      // host takes the report once all six carry it: no write ordering, so
      // no system-scope fence.
      volatile unsigned long long *vi = info;
      unsigned long long w[6];
#pragma unroll
      for (int i = 0; i < 6; ++i) w[i] = (vi[i] & INSPECT_REPORT_MASK) | (seq << INSPECT_REPORT_BITS);
#pragma unroll
      for (int i = 0; i < 7; ++i) vi[i] = 0;
#pragma unroll
      for (int i = 0; i < 6; ++i) ((volatile unsigned long long *)sig)[i] = w[i];
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
__device__ __forceinline__ void scan_single_block_body(int64_t *a, int64_t len) {
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
__global__ void __launch_bounds__(1024) k_scan_single_block(int64_t *a, int64_t len) { scan_single_block_body(a, len); }

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
