// Device graph views handed to kernels and to user functors by value.
//
// Operator-API names follow the reference (src/data_structures/graph.cuh:
// 114-277: device_graph_t<CSR|COO,E>, get_level, get_out_degree,
// get_in_degree, get_in_start_pos, fetch_edata, update_level, reset_level).
// The layout is this engine's own: int64 row offsets (n+1) so graphs beyond
// 2^31 arcs fit, int32 column ids, an int32 out-degree array for the O(1)
// degree queries user functors make, and optional per-arc edge data.  The
// reverse (in-edge) arrays alias the forward ones for undirected graphs.
#pragma once
#include "common.cuh"

template <GraphFmt fmt, typename E>
struct device_graph_t {};

template <typename E>
struct device_graph_t<CSR, E> {
  typedef E edge_t;

  const int64_t *dg_row_off;  // n+1
  const int *dg_adj_list;     // m
  const int *dg_odegree;      // n
  E *dg_edgedata;             // m (null for Empty)
  const int64_t *dgr_row_off;
  const int *dgr_adj_list;
  const int *dgr_odegree;
  E *dgr_edgedata;

  int nvertexs;
  int64_t nedges;
  int level;
  bool directed;
  // captured level loops keep the level in device memory (the loop advances
  // it between levels); null: the by-value member above
  const int *dlevel = nullptr;

  __host__ __device__ __forceinline__ int get_level() const {
#ifdef __CUDA_ARCH__
    if (dlevel) return *dlevel;
#endif
    return level;
  }
  __device__ __forceinline__ int get_out_degree(const int v) const { return __ldg(dg_odegree + v); }
  __device__ __forceinline__ int get_in_degree(const int v) const { return __ldg(dgr_odegree + v); }
  __device__ __forceinline__ int64_t get_out_start_pos(const int v) const { return __ldg(dg_row_off + v); }
  __device__ __forceinline__ int64_t get_in_start_pos(const int v) const { return __ldg(dgr_row_off + v); }
  __device__ __forceinline__ E *fetch_edata(const int64_t eid) const {
    return std::is_same<E, Empty>::value ? (E *)nullptr : dg_edgedata + eid;
  }
  __device__ __forceinline__ E *fetch_edata_r(const int64_t eid) const {
    return std::is_same<E, Empty>::value ? (E *)nullptr : dgr_edgedata + eid;
  }
  // The level is a by-value member: the host advances it between launches
  // and kernels that loop over levels on the device advance their own copy.
  __host__ __device__ __forceinline__ void update_level(int inc = 1) { level += inc; }
  __host__ __device__ __forceinline__ void reset_level(int = 1) { level = 0; }
};

// Edge-centric view: one packed (v << 32 | u) word per edge.
template <typename E>
struct device_graph_t<COO, E> {
  typedef E edge_t;
  const packed_t *dg_coo;
  E *dg_edgedata;
  int nvertexs;
  int64_t nedges;
  int level;
  const int *dlevel = nullptr;  // as in the CSR view

  __host__ __device__ __forceinline__ int get_level() const {
#ifdef __CUDA_ARCH__
    if (dlevel) return *dlevel;
#endif
    return level;
  }
  __host__ __device__ __forceinline__ void update_level(int inc = 1) { level += inc; }
  __host__ __device__ __forceinline__ void reset_level(int = 1) { level = 0; }
  __device__ __forceinline__ E *fetch_edata(const int64_t eid) const {
    return std::is_same<E, Empty>::value ? (E *)nullptr : dg_edgedata + eid;
  }
};
