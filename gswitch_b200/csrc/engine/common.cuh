// GSWITCH-on-B200 engine: shared vocabulary, error state and warp/block
// primitives.
//
// The enums, the ALL_ACTIVE/ALL_INACTIVE roots and the Empty edge type are
// the reference's operator-API vocabulary (src/utils/common.cuh:6-37,
// src/utils/utils.cuh:247-249) and keep their names and values so user
// functors written against the reference compile unchanged.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <cstring>
#include <type_traits>

#include "../../../include/gsw.h"

#define ALL_ACTIVE -1
#define ALL_INACTIVE -2

enum Status { Inactive = 0, Active = 1, All = 2, Fixed = 3 };
enum GraphFmt { CSR, COO };
enum Centric { EC, VC };
enum Computation { Idem, Mono, ASSO };
enum QueueMode { Normal, Cached };
enum Direction { Push, Pull };
enum ASFmt { Queue, Bitmap };
enum LB { TM, WM, CM, STRICT, TWOD, ELB, TWC };
enum Fusion { Fused, Standalone };
enum CullMode { Interleave, Stride };

// Launch-shape constants of the reference API (src/utils/common.cuh:12-24).
// The engine's own kernels size their grids from the SM count instead; these
// remain for code that names them.
const int CTANUM = 256;
const int THDNUM = 512;
const int CTANUM_EXPAND = 256;
const int THDNUM_EXPAND = 512;
const int BSZ = THDNUM_EXPAND * 6;      // 2D-partition tile (vertices)
const int THRESHOLD = 6144 * 4;         // 2D-partition heavy-tile edge count

struct Empty {
  char placeholder;
};

typedef int64_t packed_t;

#ifndef MIN
#define MIN(a, b) ((a) < (b) ? (a) : (b))
#endif
#ifndef MAX
#define MAX(a, b) ((a) > (b) ? (a) : (b))
#endif
#define DIV(a, b) ((b) == 0 ? 0 : ((a + .0) / (b)))

namespace gsw {

// status codes are the C ABI's (GSW_OK, GSW_ERR_*), include/gsw.h

// slots of the inspector's statistics block (six counters, a completion
// counter, a spare, and 2 x 256 per-virtual-block partial sums)
constexpr int STAT_SLOTS = 8 + 2 * 256;
// behind it, in u64 words: the VC inspection's merge scratch (two u32 maxima
// per virtual thread of the 256 x 512 grid, one u32 step counter per virtual
// block), zeroed once at allocation and left zeroed by every inspection
constexpr int STAT_SCRATCH = (2 * 256 * 512 + 256 + 1) / 2;

// Device error word bits, written by kernels and read by the host.
enum device_error_bits : unsigned {
  DEV_ERR_QUEUE_OVERFLOW = 1u,
  DEV_ERR_BARRIER_TIMEOUT = 2u,
  DEV_ERR_BAD_VERTEX = 4u,
  DEV_ERR_SCRATCH_OVERFLOW = 8u,
  DEV_ERR_STAGE_TIMEOUT = 16u,  // a shared-memory staging copy did not complete
};

// Sticky host-side error (first error wins until cleared), one per thread.
struct error_state {
  int code = GSW_OK;
  char msg[512] = {0};
};
inline error_state &err() {
  static thread_local error_state e;
  return e;
}
inline int set_error(int code, const char *fmt, const char *a = "", int line = 0) {
  error_state &e = err();
  if (e.code == GSW_OK) {
    e.code = code;
    snprintf(e.msg, sizeof(e.msg), fmt, a, line);
  }
  return code;
}
inline void clear_error() {
  err().code = GSW_OK;
  err().msg[0] = 0;
}
inline bool ok() { return err().code == GSW_OK; }

inline int cuda_check(cudaError_t e, const char *file, int line) {
  if (e == cudaSuccess) return GSW_OK;
  char buf[256];
  snprintf(buf, sizeof(buf), "%s: %%s:%%d", cudaGetErrorString(e));
  return set_error(e == cudaErrorMemoryAllocation ? GSW_ERR_OOM : GSW_ERR_CUDA, buf, file, line);
}
#define GSW_CUDA(x) ::gsw::cuda_check((x), __FILE__, __LINE__)
// kernels launched by the engine on this thread (reported per run)
inline long long &launch_count() {
  static thread_local long long c = 0;
  return c;
}
#define GSW_LAUNCHED() (++::gsw::launch_count(), ::gsw::cuda_check(cudaGetLastError(), __FILE__, __LINE__))

// ---- device primitives --------------------------------------------------
static constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ int warp_id() { return threadIdx.x >> 5; }

template <typename T>
__device__ __forceinline__ T warp_inclusive_sum(T x) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    T y = __shfl_up_sync(FULL, x, d);
    if (lane_id() >= d) x += y;
  }
  return x;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T x) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) x += __shfl_xor_sync(FULL, x, d);
  return x;
}

template <typename T>
__device__ __forceinline__ T warp_max(T x) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    T y = __shfl_xor_sync(FULL, x, d);
    x = x > y ? x : y;
  }
  return x;
}

// Block-wide reduction; every thread of the block must call it.
// smem needs 32 slots of T.
template <typename T, bool IS_MAX = false>
__device__ __forceinline__ T block_reduce(T x, T *smem) {
  x = IS_MAX ? warp_max(x) : warp_sum(x);
  __syncthreads();
  if (lane_id() == 0) smem[warp_id()] = x;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  T r = threadIdx.x < nw ? smem[threadIdx.x] : T(0);
  if (warp_id() == 0) r = IS_MAX ? warp_max(r) : warp_sum(r);
  if (threadIdx.x == 0) smem[0] = r;
  __syncthreads();
  r = smem[0];
  __syncthreads();
  return r;
}

// Block-wide exclusive scan of ints; returns the block total in *total.
// smem needs 33 ints.  Every thread of the block must call it.
__device__ __forceinline__ int block_exclusive_scan(int x, int *smem, int *total) {
  int incl = warp_inclusive_sum(x);
  __syncthreads();
  if (lane_id() == 31) smem[warp_id()] = incl;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  if (warp_id() == 0) {
    int s = lane_id() < nw ? smem[lane_id()] : 0;
    int si = warp_inclusive_sum(s);
    if (lane_id() < nw) smem[lane_id()] = si - s;
    if (lane_id() == 31) smem[32] = si;
  }
  __syncthreads();
  int r = smem[warp_id()] + incl - x;
  *total = smem[32];
  __syncthreads();
  return r;
}

// Number of entries of the ascending array a[0..n) that are <= key, i.e. the
// index of the segment that owns `key` plus one (src/utils/intrinsics.cuh:
// 78-91 computes the same bound).
template <typename T>
__device__ __forceinline__ int upper_bound(const T *a, int n, T key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] <= key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}
template <typename T>
__device__ __forceinline__ int64_t upper_bound64(const T *a, int64_t n, T key) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (a[mid] <= key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// 4-byte-packed shuffle of an arbitrary value type (the reference's
// __exshfl_down, src/utils/intrinsics.cuh:293-302).
template <typename T>
__device__ __forceinline__ T shfl_up_any(T v, int delta) {
  static_assert(sizeof(T) % 4 == 0 || sizeof(T) < 4, "4-byte packed type");
  if (sizeof(T) < 4) {
    int x = 0;
    memcpy(&x, &v, sizeof(T));
    x = __shfl_up_sync(FULL, x, delta);
    memcpy(&v, &x, sizeof(T));
    return v;
  }
  int x[sizeof(T) / 4 > 0 ? sizeof(T) / 4 : 1];
  memcpy(x, &v, sizeof(T));
#pragma unroll
  for (int i = 0; i < (int)(sizeof(T) / 4); ++i) x[i] = __shfl_up_sync(FULL, x[i], delta);
  memcpy(&v, x, sizeof(T));
  return v;
}
template <typename T>
__device__ __forceinline__ T shfl_down_any(T v, int delta) {
  static_assert(sizeof(T) % 4 == 0 || sizeof(T) < 4, "4-byte packed type");
  if (sizeof(T) < 4) {
    int x = 0;
    memcpy(&x, &v, sizeof(T));
    x = __shfl_down_sync(FULL, x, delta);
    memcpy(&v, &x, sizeof(T));
    return v;
  }
  int x[sizeof(T) / 4 > 0 ? sizeof(T) / 4 : 1];
  memcpy(x, &v, sizeof(T));
#pragma unroll
  for (int i = 0; i < (int)(sizeof(T) / 4); ++i) x[i] = __shfl_down_sync(FULL, x[i], delta);
  memcpy(&v, x, sizeof(T));
  return v;
}

template <typename T>
__device__ __forceinline__ bool equals_any(const T &a, const T &b) {
  return memcmp(&a, &b, sizeof(T)) == 0;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ---- 1-D TMA bulk copies global -> shared (cp.async.bulk, no multicast) ----
// Used to stage runs of a hub's adjacency list in shared memory.  The source
// is always this GPU's own memory (the graph's column array); source and
// destination are 16-byte aligned and the size is a multiple of 16 bytes
// (callers copy the aligned body of a run and read its ragged ends with
// plain loads).  Completion is tracked by a CTA-local mbarrier: one thread
// arms it with the byte count and issues the copy; every thread waits on the
// barrier's phase parity.
__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
// makes barrier initialisation visible to the async proxy (bulk copies)
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_inval(unsigned long long *bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  unsigned long long state;
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 %0, [%1], %2;"
               : "=l"(state)
               : "r"(smem_addr(bar)), "r"(bytes)
               : "memory");
  asm volatile("" ::"l"(state));  // the arrival token is not needed
}
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned long long *bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Bounded wait for a phase: false (and DEV_ERR_STAGE_TIMEOUT in *err) after
// about `budget_ns`; a copy from valid device memory completes long before.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, unsigned *err,
                                          uint64_t budget_ns = 200000000ull) {
  if (mbar_test(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  while (!mbar_test(bar, parity)) {
    if (globaltimer_ns() - t0 > budget_ns) {
      atomicOr(err, DEV_ERR_STAGE_TIMEOUT);
      return false;
    }
  }
  return true;
}
// orders this thread's earlier generic-proxy accesses of shared memory before
// a following async-proxy (bulk copy) write to it
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

}  // namespace gsw

// float atomicMin used by user functors (src/utils/intrinsics.cuh:304-313
// offers the same overload): CAS loop on the bit pattern.
__device__ __forceinline__ float atomicMin(float *address, float val) {
  int *ai = (int *)address;
  int old = *ai, assumed;
  do {
    assumed = old;
    float cur = __int_as_float(assumed);
    if (!(val < cur)) break;
    old = atomicCAS(ai, assumed, __float_as_int(val));
  } while (assumed != old);
  return __int_as_float(old);
}
