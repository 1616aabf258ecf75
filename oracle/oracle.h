/*
 * CPU oracle for the GSWITCH level-loop hot path.  TEST INFRASTRUCTURE ONLY.
 *
 * Only the test-suite, the smoke check and the bench's cpu_baseline leg may
 * load this library; it is the checker, never the thing shipped or measured.
 *
 * Contents
 *   - seeded synthetic graph generators (RMAT, 2D grid + long-range, G(n,m),
 *     ER batch, seeded roots) and the undirected CSR build (drop self-loops,
 *     symmetrise, sort, dedup), restated independently of the product's
 *     device generator so the two can be compared bit for bit;
 *   - restatements of the reference's CPU validators (file:line cited per
 *     function, paths relative to the PAA-NCIC/GSWITCH tree);
 *   - FP64 extensions the reference does not have (BC in FP64, PageRank as a
 *     fixed-iteration Jacobi), and the degree statistics behind the
 *     selector's graph features.
 *
 * Parity pin: the BFS / SSSP / CC / BC validators are checked against the
 * reference's own functions compiled from its sources (oracle/ref) and
 * against the golden vectors under tests/golden produced by them.
 */
#ifndef GSW_ORACLE_H
#define GSW_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- hashing / generators -------------------------------------------- */
uint64_t or_sm64(uint64_t x);
uint64_t or_stream_key(uint64_t seed, uint64_t stream);

/* RMAT edge list: ef * 2^scale directed pairs (self-loops included; the CSR
 * build drops them). src/dst must hold ef<<scale entries. */
void or_rmat_edges(int scale, int ef, double a, double b, double c,
                   uint64_t seed, uint32_t *src, uint32_t *dst);
/* rows x cols 4-neighbour grid plus (grid edges / lr_div) long-range pairs.
 * Returns the number of pairs written (caller sizes with or_grid_nedges). */
int64_t or_grid_nedges(int rows, int cols, int lr_div);
int64_t or_grid_edges(int rows, int cols, int lr_div, uint64_t seed,
                      uint32_t *src, uint32_t *dst);
/* G(n, m) with replacement: m uniform pairs. */
void or_er_edges(int64_t n, int64_t m, uint64_t seed, uint32_t *src,
                 uint32_t *dst);
/* parameters of instance i of the ER batch: n in logU[nlo,nhi], mean degree
 * U[dlo,dhi], m = floor(n*deg/2), instance seed. */
void or_er_batch_params(uint64_t seed, int64_t i, int64_t nlo, int64_t nhi,
                        double dlo, double dhi, int64_t *n, int64_t *m,
                        uint64_t *iseed);

/* Undirected CSR from a pair list: drops self-loops, adds both directions,
 * sorts each adjacency, removes duplicates.  *off (n+1 int64) and *col
 * (m int32) are malloc'd; returns m (arcs). */
int64_t or_csr_build(int64_t n, int64_t npairs, const uint32_t *src,
                     const uint32_t *dst, int64_t **off, int32_t **col);
/* symmetric weights 1 + H(seed, min(u,v), max(u,v)) % wmax, one per arc */
void or_weights(uint64_t seed, int wmax, int64_t n, const int64_t *off,
                const int32_t *col, int32_t *w);
/* k-th seeded non-isolated root (draws skip isolated vertices and repeats
 * of earlier roots); writes count roots. */
void or_roots(uint64_t seed, int64_t n, const int64_t *off, int count,
              int32_t *roots);
void or_free(void *p);

/* ---- validators -------------------------------------------------------- */
void or_bfs(int64_t n, const int64_t *off, const int32_t *col, int32_t root,
            int32_t *lvl);
void or_sssp_spfa(int64_t n, const int64_t *off, const int32_t *col,
                  const int32_t *w, int32_t root, int32_t *dist);
void or_sssp_dijkstra(int64_t n, const int64_t *off, const int32_t *col,
                      const int32_t *w, int32_t root, int32_t *dist);
/* Dial's bucket queue for integer weights in [1, wmax]; -1 if a weight is
 * outside that range. */
int or_sssp_dial(int64_t n, const int64_t *off, const int32_t *col,
                 const int32_t *w, int32_t root, int32_t wmax, int32_t *dis);
void or_cc(int64_t n, const int64_t *off, const int32_t *col, int32_t *label);
/* CC_CPU's labels in linear time (the seed is marked when its component
 * starts instead of re-entering the queue from each neighbour). */
void or_cc_linear(int64_t n, const int64_t *off, const int32_t *col, int32_t *id);
void or_bc_f32(int64_t n, const int64_t *off, const int32_t *col, int32_t root,
               int32_t *nsp, float *dep);
void or_bc_f64(int64_t n, const int64_t *off, const int32_t *col, int32_t root,
               double *nsp, double *dep, int32_t *lvl);
void or_pagerank(int64_t n, const int64_t *off, const int32_t *col, int iters,
                 double damp, double *pr);
int64_t or_pagerank_check(int64_t n, const int64_t *off, const int32_t *col,
                          const float *pr_over_od, float damp, float eps);
int64_t or_gc_check(int64_t n, const int64_t *off, const int32_t *col,
                    const int32_t *color);
void or_gc_levels(int64_t n, const int64_t *off, const int32_t *col, int32_t *color);
void or_mbfs(int64_t n, const int64_t *off, const int32_t *col, int nsrc,
             const int32_t *roots, int32_t *lvl /* nsrc*n */);
/* degree statistics as graph_attr_t::fill: out[0..5] = avg, std, range,
 * max, GI, Her */
void or_degree_attr(int64_t n, const int64_t *off, double *out);
/* Graph500 traversed-edge count: (sum of degrees of reached vertices)/2 */
int64_t or_traversed_edges(int64_t n, const int64_t *off, const int32_t *lvl);

void or_inspect_bfs(int64_t n, const int64_t *off, const int32_t *lvl, int32_t level, uint64_t *out);
#ifdef __cplusplus
}
#endif
#endif
