// Batched betweenness centrality: many sources' Brandes passes together.
//
// The reference runs BC from one source, forward and backward through its
// level loop (application/bc.cu:97-160 with bc_cpu, bc.cu:162-214, as the
// validator).  Here up to BCB_SOURCES sources share every launch:
//   levels   the bit-sliced multi-source BFS (mbfs.cuh) gives each vertex's
//            level per source, vertex-major: row v holds the batch's levels;
//   forward  for each level L, a warp per adjacency chunk (at most 1024 edges
//            of one vertex, so a hub spreads over many warps) of a vertex
//            that some source reached at L: lane s sums the path counts of
//            the in-neighbours at level L-1 for source s
//            (nsp[v] += nsp[u] where level_s(u) + 1 == level_s(v));
//   backward for each level L from the deepest down, the same chunks sum
//            (1 + dep[w]) / nsp[w] over the neighbours one level further for
//            source s, and dep[v] = nsp[v] * that sum
//            (bc_cpu's "dep[v] *= nsp[v]" once v's children are in);
//   output   path counts and dependencies transposed to source-major rows.
// By default all of it (every BFS level, every forward and backward pass)
// runs in one cooperative launch with a grid barrier between steps
// (k_mbfs_persistent); with persistent launches off, one launch per step.
// Path counts are int32 and wrap like the reference's; dependencies are
// FP32.  The columns of a chunk are read 32 at a time, one per lane, and
// handed out by shuffles, so each edge costs one coalesced 128-byte row of
// the neighbour's levels (and a row of its counts when it qualifies).
#pragma once
#include "mbfs.cuh"

namespace gsw {

struct bcb_result {
  double ms = 0;
  int64_t edges = 0;
  int levels = 0;
};

// one batch of at most BCB_SOURCES sources; nsp / dep receive source-major
// rows (nsrc x n) on the host.  persistent: levels, forward and backward
// passes in one cooperative launch; otherwise one launch per pass.
template <typename Buf>
bcb_result bc_batch_run(device_graph_t<CSR, Empty> g, int nsrc, const int32_t *roots_host, Buf buf, int32_t *nsp_host,
                        float *dep_host, bool persistent) {
  bcb_result res;
  const int64_t n = g.nvertexs;
  const int64_t cells = n * (int64_t)nsrc;
  cudaStream_t s = stream();
  int *nsp = (int *)buf("bcb_nsp", sizeof(int) * (size_t)cells);
  float *sum = (float *)buf("bcb_sum", sizeof(float) * (size_t)cells);
  if (!nsp || !sum) return res;
  mbfs_result mb = persistent ? mbfs_impl<1>(g, nsrc, roots_host, buf, nullptr, false, true, nsp, sum)
                              : mbfs_impl<1>(g, nsrc, roots_host, buf, nullptr, false, false, nsp, sum);
  if (!ok()) return res;
  int *lvl = (int *)buf("mb_levels_vm", sizeof(int) * (size_t)cells);
  int *tr = (int *)buf("mb_levels", sizeof(int) * (size_t)cells);  // transposed rows
  // the chunk list mbfs_impl built for this graph
  int64_t *coff = (int64_t *)buf("mb_coff", sizeof(int64_t) * (n + 1));
  if (!lvl || !tr || !coff) return res;
  int64_t nchunks = 0;
  GSW_CUDA(cudaMemcpyAsync(&nchunks, coff + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  GSW_CUDA(cudaStreamSynchronize(s));
  int *cv = (int *)buf("mb_cv", sizeof(int) * (nchunks + 1));
  int64_t *cbeg = (int64_t *)buf("mb_cbeg", sizeof(int64_t) * (nchunks + 1));
  if (!cv || !cbeg) return res;
  const int depth = mb.levels;  // levels 0 .. depth-1 carry vertices
  float ms = 0;
  const int grid = sm_count() * 8;
  if (!persistent) {
    // mbfs_impl seeded nsp and cleared sum; one launch per pass
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    for (int L = 1; L < depth && ok(); ++L)
      k_bcb_forward<<<grid, 256, 0, s>>>(g, cv, cbeg, nchunks, lvl, nsrc, L, nsp);
    for (int L = depth - 2; L >= 0 && ok(); --L)
      k_bcb_backward<<<grid, 256, 0, s>>>(g, cv, cbeg, nchunks, lvl, nsrc, L, nsp, sum);
    k_bcb_finish<<<grid, 256, 0, s>>>(nsp, sum, cells);
    cudaEventRecord(e1, s);
    GSW_LAUNCHED();
    GSW_CUDA(cudaEventSynchronize(e1));
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  if (nsp_host) {
    k_mbfs_transpose<<<grid, dim3(32, 8), 0, s>>>(nsp, n, nsrc, tr);
    GSW_CUDA(cudaMemcpyAsync(nsp_host, tr, sizeof(int) * (size_t)cells, cudaMemcpyDeviceToHost, s));
  }
  if (dep_host) {
    // the transpose moves 4-byte words: float rows go through it bit for bit
    k_mbfs_transpose<<<grid, dim3(32, 8), 0, s>>>((const int *)sum, n, nsrc, tr);
    GSW_CUDA(cudaMemcpyAsync(dep_host, tr, sizeof(float) * (size_t)cells, cudaMemcpyDeviceToHost, s));
  }
  GSW_CUDA(cudaStreamSynchronize(s));
  res.ms = mb.ms + ms;
  res.edges = mb.edges;
  res.levels = depth;
  return res;
}

}  // namespace gsw
