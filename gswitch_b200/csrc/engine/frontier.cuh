// Frontier ("active set") storage: status bitmaps, ping-pong / cached
// queues, the edge-balanced work set and the convergence flag.
//
// Semantics follow the reference's active set (src/data_structures/
// active_set.cuh:14-130, queue.cuh:86-226, bitmap.cuh:7-164,
// notification.cuh:34-94, workset.cuh:8-44); the storage is this engine's:
//   - bitmaps are 32-bit words written one word per warp by a ballot
//     (reference: byte-granular); `active` bit = status Active, `inactive`
//     bit = status != Inactive (0 only for Inactive vertices), `visited` for
//     de-duplication;
//   - queue sizes, the device error word and the grid-barrier words live in
//     one device "counters" block so a captured or persistent level loop
//     never needs the host;
//   - the STRICT work set holds int64 edge offsets (frontiers beyond 2^31
//     edges on scale-26 graphs).
#pragma once
#include "common.cuh"

namespace gsw {

// One stream per thread of control; the C ABI sets it per context.
inline cudaStream_t &stream() {
  static thread_local cudaStream_t s = 0;
  return s;
}

static __global__ void k_fill_u32(uint32_t *p, uint32_t v, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

inline int fill_u32(uint32_t *p, uint32_t v, int64_t n) {
  if (n <= 0) return GSW_OK;
  int grid = (int)MIN((n + 255) / 256, (int64_t)2048);
  k_fill_u32<<<grid, 256, 0, stream()>>>(p, v, n);
  return GSW_LAUNCHED();
}

// device counters shared by every kernel of one active set
struct as_counters_t {
  int qsize[2];          // Normal-mode subqueue sizes
  unsigned err;          // DEV_ERR_* bits
  unsigned bar_count;    // grid barrier arrivals
  unsigned bar_gen;      // grid barrier generation
  int dlevel;            // device-side level for loops run on the device
  int halt;              // device-side convergence flag
  int cnt;               // __exit / probe counter
  unsigned long long total_edges;  // STRICT: edges in the current frontier
  unsigned long long scanned;      // accounting: edges an expand touched
  int pq[3];                       // persistent fused levels: rotating sizes
  int plevels;                     // persistent fused levels: levels done
  int preason;                     // persistent fused levels: exit reason
  int plb;                         // persistent fused levels: the load
                                   // balance the launched kernel ran
  int hub_pieces;                  // tiered push: pieces in the hub list
  unsigned hub_done;               // tiered push: hub-kernel CTAs that read it
};

struct bits_t {
  uint32_t *dg_bits = nullptr;
  int64_t n_words = 0;

  __device__ __forceinline__ uint32_t load_word(int v) const { return dg_bits[v >> 5]; }
  __device__ __forceinline__ bool test(int v) const { return (dg_bits[v >> 5] >> (v & 31)) & 1u; }
  // reference bits_t::query: true when the bit of v is 0
  __device__ __forceinline__ bool query(int v) const { return !test(v); }
  // Marks v and reports whether it was unmarked.  Races between threads may
  // let several of them see "unmarked"; callers treat it as a hint
  // (bitmap.cuh:87-99 has the same contract).
  __device__ __forceinline__ bool query_and_mark(int v) {
    const uint32_t m = 1u << (v & 31);
    if (dg_bits[v >> 5] & m) return false;
    atomicOr(dg_bits + (v >> 5), m);
    return true;
  }
  // exactly-once marking
  __device__ __forceinline__ bool query_and_mark_atomic(int v) {
    const uint32_t m = 1u << (v & 31);
    return !(atomicOr(dg_bits + (v >> 5), m) & m);
  }
  __device__ __forceinline__ void store_word(int v, uint32_t w) { dg_bits[v >> 5] = w; }
};

struct bitmap_t {
  bits_t visited, active, inactive;

  __device__ __forceinline__ bool is_active(int v) const { return active.test(v); }
  __device__ __forceinline__ bool is_inactive(int v) const { return !inactive.test(v); }
  __device__ __forceinline__ bool is_valid(int v) const { return is_active(v) || is_inactive(v); }
  __device__ __forceinline__ bool mark_duplicate_lite(int v) { return visited.query_and_mark(v); }
  __device__ __forceinline__ bool mark_duplicate_atomic(int v) { return visited.query_and_mark_atomic(v); }
};

struct subqueue_t {
  int *dg_queue = nullptr;
  int *dg_qsize = nullptr;  // Normal mode: into the counters block
  int64_t max_size = 0;

  __device__ __forceinline__ int get_qsize() const { return *(volatile int *)dg_qsize; }
  __device__ __forceinline__ int fetch(int64_t idx) const { return __ldg(dg_queue + idx); }
};

// Normal mode: subqueue[cursor] is the input, subqueue[cursor^1] the output.
// Cached mode (replay of every level, used by BC's backward sweep):
// subqueue[0] keeps all levels back to back, subqueue[1] keeps the sizes.
struct queue_t {
  subqueue_t subqueue[2];
  bool traceback = false;
  int cursor = 0;
  int64_t offset_in = 0, offset_out = 0;
  QueueMode mode = Normal;
  unsigned *dg_err = nullptr;

  // ---- Normal
  __device__ __forceinline__ int get_qsize_Normal() const { return subqueue[cursor].get_qsize(); }
  __device__ __forceinline__ int fetch_Normal(int64_t idx) const { return subqueue[cursor].fetch(idx); }
  __device__ __forceinline__ int *output_base_Normal() const { return subqueue[cursor ^ 1].dg_queue; }
  __device__ __forceinline__ int *output_size_Normal() const { return subqueue[cursor ^ 1].dg_qsize; }
  __device__ __forceinline__ int64_t output_cap_Normal() const { return subqueue[cursor ^ 1].max_size; }
  // ---- Cached
  __device__ __forceinline__ int get_qsize_Cached() const { return ((volatile int *)subqueue[1].dg_queue)[cursor]; }
  __device__ __forceinline__ int fetch_Cached(int64_t idx) const { return __ldg(subqueue[0].dg_queue + offset_in + idx); }
  __device__ __forceinline__ int *output_base_Cached() const { return subqueue[0].dg_queue + offset_out; }
  __device__ __forceinline__ int *output_size_Cached() const { return subqueue[1].dg_queue + cursor + 1; }
  __device__ __forceinline__ int64_t output_cap_Cached() const { return subqueue[0].max_size - offset_out; }

  __device__ __forceinline__ int *output_base() const { return mode == Normal ? output_base_Normal() : output_base_Cached(); }
  __device__ __forceinline__ int *output_size() const { return mode == Normal ? output_size_Normal() : output_size_Cached(); }
  __device__ __forceinline__ int64_t output_cap() const { return mode == Normal ? output_cap_Normal() : output_cap_Cached(); }

  // append one element; an overflow is recorded, never written out of bounds
  __device__ __forceinline__ void push(int ele) {
    if (mode == Cached && traceback) return;
    int idx = atomicAdd(output_size(), 1);
    if (idx < output_cap())
      output_base()[idx] = ele;
    else
      atomicOr(dg_err, DEV_ERR_QUEUE_OVERFLOW);
  }
  // reserve cnt consecutive slots (warp-aggregated enqueue); returns -1 on
  // overflow after recording it
  __device__ __forceinline__ int64_t reserve(int cnt) {
    if (mode == Cached && traceback) return -1;
    int idx = atomicAdd(output_size(), cnt);
    if ((int64_t)idx + cnt > output_cap()) {
      atomicOr(dg_err, DEV_ERR_QUEUE_OVERFLOW);
      return -1;
    }
    return idx;
  }

  // ---- host side
  int get_qsize_host() const {
    int r = 0;
    if (mode == Normal)
      GSW_CUDA(cudaMemcpyAsync(&r, subqueue[cursor].dg_qsize, sizeof(int), cudaMemcpyDeviceToHost, stream()));
    else
      GSW_CUDA(cudaMemcpyAsync(&r, subqueue[1].dg_queue + cursor, sizeof(int), cudaMemcpyDeviceToHost, stream()));
    GSW_CUDA(cudaStreamSynchronize(stream()));
    return r;
  }
  void clean_size(int which) { GSW_CUDA(cudaMemsetAsync(subqueue[which].dg_qsize, 0, sizeof(int), stream())); }
  // device address of the size the next builder appends to
  int *output_size_ptr() const {
    return mode == Normal ? subqueue[cursor ^ 1].dg_qsize : subqueue[1].dg_queue + cursor + 1;
  }
  void reset(bool _traceback = false) {
    if (mode == Normal) {
      clean_size(0);
      clean_size(1);
    }
    reset_host(_traceback);
  }
  // reset() without clearing the Normal-mode sizes (active_set_t::reset
  // clears them in its own kernel)
  void reset_host(bool _traceback) {
    traceback = _traceback;
    if (!traceback) {
      cursor = 0;
      offset_in = offset_out = 0;
      if (mode == Cached)
        GSW_CUDA(cudaMemsetAsync(subqueue[1].dg_queue, 0, sizeof(int) * subqueue[1].max_size, stream()));
    }
  }
  // queue.cuh:113-127: Normal flips the ping-pong pair; Cached walks the
  // per-level segments forward (or backward while tracing back).
  void swap() {
    if (mode == Normal) {
      clean_size(cursor);
      cursor ^= 1;
    } else if (traceback) {
      if (cursor > 0) {
        cursor--;
        offset_in -= get_qsize_host();
      }
    } else {
      // one size slot per level; a chain of n vertices has n levels
      if (cursor + 2 >= subqueue[1].max_size) {
        set_error(GSW_ERR_OVERFLOW, "%s", "cached queue: more levels than size slots");
        return;
      }
      cursor++;
      offset_in = offset_out;
      offset_out += get_qsize_host();
    }
  }
};

struct workset_t {
  int64_t *dg_eoff = nullptr;  // exclusive scan of frontier degrees, size+1
  int64_t *dg_bsum = nullptr;  // per-block partial sums of the scan
  int64_t cap = 0;
  int64_t bsum_cap = 0;
};

struct notification_t {
  volatile int *h_tag = nullptr;  // mapped pinned: written by device or host
  int *dg_tag = nullptr;
  bool already = false;

  __device__ __forceinline__ void notify_device() {
    if (!already) *(volatile int *)dg_tag = 1;
  }
  void notify_host() {
    *h_tag = 1;
    already = true;
  }
  bool is_converged() const { return *h_tag != 0; }
  void reset() {
    *h_tag = 0;
    already = false;
  }
};

struct active_set_t {
  ASFmt fmt = Queue;
  int64_t size = 0;
  int64_t size_cached = 0;
  bitmap_t bitmap;
  queue_t queue;
  workset_t workset;
  notification_t nt;
  as_counters_t *dg_cnt = nullptr;

  // ---- device
  __device__ __forceinline__ int64_t get_bitmap_size() const { return size; }
  __device__ __forceinline__ int64_t get_queue_size_hard() const {
    return queue.mode == Normal ? queue.get_qsize_Normal() : queue.get_qsize_Cached();
  }
  __device__ __forceinline__ int64_t get_size() const { return fmt == Queue ? get_queue_size_hard() : size; }
  __device__ __forceinline__ int fetch_queue(int64_t idx) const {
    return queue.mode == Normal ? queue.fetch_Normal(idx) : queue.fetch_Cached(idx);
  }
  __device__ __forceinline__ int fetch_bitmap(int64_t idx, Status wanted) const {
    const int v = (int)idx;
    if (wanted == All && (bitmap.is_active(v) || bitmap.is_inactive(v))) return v;
    if (wanted == Active && bitmap.is_active(v)) return v;
    if (wanted == Inactive && bitmap.is_inactive(v)) return v;
    return -1;
  }
  __device__ __forceinline__ int fetch(int64_t idx, Status wanted) const {
    return fmt == Queue ? fetch_queue(idx) : fetch_bitmap(idx, wanted);
  }
  __device__ __forceinline__ void halt_device() { nt.notify_device(); }
  __device__ __forceinline__ void raise(unsigned bits) const { atomicOr(&dg_cnt->err, bits); }

  // ---- host
  // the reference's as.finish(g, f, conf) (active_set.cuh:37-43): true when
  // the level loop is over; defined beside the engine's finish() in
  // executor.cuh
  template <typename G, typename F, typename C>
  bool finish(G &g, F &f, C &conf);
  int build(int64_t _size, QueueMode qmode);
  void destroy();
  void reset(bool traceback = false);
  void init(int64_t root = ALL_ACTIVE);
  void set_fmt(ASFmt f) { fmt = f; }
  void halt_host() { nt.notify_host(); }
  bool is_converged() const { return nt.is_converged(); }
  int64_t get_size_host() {
    size_cached = fmt == Queue ? queue.get_qsize_host() : size;
    return size_cached;
  }
  int64_t get_size_host_cached() const { return size_cached; }
  unsigned read_error() const {
    unsigned e = 0;
    GSW_CUDA(cudaMemcpyAsync(&e, &dg_cnt->err, sizeof(unsigned), cudaMemcpyDeviceToHost, stream()));
    GSW_CUDA(cudaStreamSynchronize(stream()));
    return e;
  }
};

inline int active_set_t::build(int64_t _size, QueueMode qmode) {
  size = _size;
  const int64_t words = (size + 31) / 32 + 1;
  auto alloc = [&](void **p, size_t bytes) { return GSW_CUDA(cudaMalloc(p, bytes)); };
  if (alloc((void **)&dg_cnt, sizeof(as_counters_t))) return err().code;
  GSW_CUDA(cudaMemsetAsync(dg_cnt, 0, sizeof(as_counters_t), stream()));
  bits_t *bs[3] = {&bitmap.visited, &bitmap.active, &bitmap.inactive};
  for (bits_t *b : bs) {
    b->n_words = words;
    if (alloc((void **)&b->dg_bits, sizeof(uint32_t) * words)) return err().code;
    GSW_CUDA(cudaMemsetAsync(b->dg_bits, 0, sizeof(uint32_t) * words, stream()));
  }
  queue.mode = qmode;
  queue.dg_err = &dg_cnt->err;
  // Cached mode keeps the per-level sizes in subqueue[1]: levels <= n, plus
  // the empty level that ends the loop, plus headroom
  for (int i = 0; i < 2; ++i) {
    queue.subqueue[i].max_size = size + 8;
    if (alloc((void **)&queue.subqueue[i].dg_queue, sizeof(int) * (size + 8))) return err().code;
    queue.subqueue[i].dg_qsize = &dg_cnt->qsize[i];
  }
  if (qmode == Cached)
    GSW_CUDA(cudaMemsetAsync(queue.subqueue[1].dg_queue, 0, sizeof(int) * (size + 8), stream()));
  workset.cap = size + 1;
  if (alloc((void **)&workset.dg_eoff, sizeof(int64_t) * (size + 2))) return err().code;
  workset.bsum_cap = (size + 1) / 1024 + 4096;
  if (alloc((void **)&workset.dg_bsum, sizeof(int64_t) * workset.bsum_cap)) return err().code;
  int *h = nullptr;
  if (GSW_CUDA(cudaHostAlloc((void **)&h, sizeof(int), cudaHostAllocMapped))) return err().code;
  nt.h_tag = h;
  if (GSW_CUDA(cudaHostGetDevicePointer((void **)&nt.dg_tag, h, 0))) return err().code;
  nt.reset();
  return err().code;
}

inline void active_set_t::destroy() {
  cudaFree(dg_cnt);
  cudaFree(bitmap.visited.dg_bits);
  cudaFree(bitmap.active.dg_bits);
  cudaFree(bitmap.inactive.dg_bits);
  cudaFree(queue.subqueue[0].dg_queue);
  cudaFree(queue.subqueue[1].dg_queue);
  cudaFree(workset.dg_eoff);
  cudaFree(workset.dg_bsum);
  if (nt.h_tag) cudaFreeHost((void *)nt.h_tag);
  *this = active_set_t();
}

// the device part of active_set_t::reset in one launch: the three bitmaps,
// the halt flag and (Normal mode) both queue sizes
static __global__ void k_as_reset(uint32_t *visited, uint32_t *active, uint32_t *inactive, int64_t words,
                                  as_counters_t *c, bool clear_sizes) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < words; i += (int64_t)gridDim.x * blockDim.x) {
    visited[i] = 0;
    active[i] = 0;
    inactive[i] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    c->halt = 0;
    if (clear_sizes) c->qsize[0] = c->qsize[1] = 0;
  }
}

// bitmap_t::init in one launch (see active_set_t::init)
static __global__ void k_as_init(uint32_t *active, uint32_t *inactive, int64_t words, int64_t root) {
  const uint32_t fill = root == ALL_ACTIVE ? 0xffffffffu : 0u;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < words; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t v = (root >= 0 && i == (root >> 5)) ? 1u << (root & 31) : fill;
    active[i] = v;
    inactive[i] = v;
  }
}

inline int bitmap_grid(int64_t words) { return (int)MAX((int64_t)1, MIN((words + 255) / 256, (int64_t)2048)); }

inline void active_set_t::reset(bool traceback) {
  queue.reset_host(traceback);
  const int64_t w = bitmap.visited.n_words;
  k_as_reset<<<bitmap_grid(w), 256, 0, stream()>>>(bitmap.visited.dg_bits, bitmap.active.dg_bits,
                                                   bitmap.inactive.dg_bits, w, dg_cnt, queue.mode == Normal);
  GSW_LAUNCHED();
  nt.reset();
}

// bitmap_t::init (bitmap.cuh:133-144): ALL_ACTIVE -> every vertex Active,
// root >= 0 -> only the root Active, the rest Inactive; ALL_INACTIVE -> all
// Inactive.  The queue is built from the bitmaps by the first filter.
inline void active_set_t::init(int64_t root) {
  const int64_t w = bitmap.active.n_words;
  k_as_init<<<bitmap_grid(w), 256, 0, stream()>>>(bitmap.active.dg_bits, bitmap.inactive.dg_bits, w, root);
  GSW_LAUNCHED();
}

inline active_set_t build_active_set(int64_t size, QueueMode qmode) {
  active_set_t as;
  as.build(size, qmode);
  return as;
}

}  // namespace gsw
