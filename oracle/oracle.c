/*
 * CPU oracle for the GSWITCH level-loop hot path.  TEST INFRASTRUCTURE ONLY:
 * loaded by tests/, the smoke check and bench.py's cpu_baseline leg as the
 * checker; never linked into the product.
 *
 * Reference citations are paths inside the PAA-NCIC/GSWITCH tree.
 */
#include "oracle.h"

#include <limits.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ------------------------------------------------------------------------ */
/* minimal parallel-for over [0, n) in chunks (pthreads; the generators and  */
/* the CSR build use it, the validators stay sequential like the reference)  */
/* ------------------------------------------------------------------------ */
typedef void (*range_fn)(int64_t lo, int64_t hi, void *arg);
typedef struct {
  range_fn fn;
  void *arg;
  int64_t n, chunk;
  int64_t next;
} pfor_t;

static void *pfor_worker(void *p) {
  pfor_t *w = (pfor_t *)p;
  for (;;) {
    int64_t lo = __atomic_fetch_add(&w->next, w->chunk, __ATOMIC_RELAXED);
    if (lo >= w->n) break;
    int64_t hi = lo + w->chunk < w->n ? lo + w->chunk : w->n;
    w->fn(lo, hi, w->arg);
  }
  return NULL;
}

static void parallel_for(int64_t n, int64_t chunk, range_fn fn, void *arg) {
  long nt = sysconf(_SC_NPROCESSORS_ONLN);
  if (nt < 1) nt = 1;
  if (nt > 256) nt = 256;
  if (n <= chunk || nt == 1) {
    fn(0, n, arg);
    return;
  }
  pfor_t w = {fn, arg, n, chunk, 0};
  pthread_t th[256];
  long started = 0;
  for (long t = 1; t < nt; ++t)
    if (pthread_create(&th[started], NULL, pfor_worker, &w) == 0) ++started;
  pfor_worker(&w);
  for (long t = 0; t < started; ++t) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------------------ */
/* counter-based hashing (SplitMix64 finaliser, Steele/Lea/Flood 2014)        */
/* ------------------------------------------------------------------------ */
uint64_t or_sm64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

uint64_t or_stream_key(uint64_t seed, uint64_t stream) {
  return or_sm64(seed ^ or_sm64(stream));
}

enum { ST_RMAT = 1, ST_W = 2, ST_GRID = 3, ST_ER = 4, ST_ERB = 5, ST_ROOT = 7 };

void or_free(void *p) { free(p); }

typedef struct {
  int scale;
  uint64_t key;
  uint32_t ta, tab, tabc;
  uint32_t *src, *dst;
} rmat_job;

static void rmat_range(int64_t lo, int64_t hi, void *p) {
  const rmat_job *j = (const rmat_job *)p;
  for (int64_t i = lo; i < hi; ++i) {
    uint64_t base = or_sm64(j->key + (uint64_t)i);
    uint32_t s = 0, d = 0;
    uint64_t h = 0;
    for (int l = 0; l < j->scale; ++l) {
      uint32_t r;
      if ((l & 1) == 0) {
        h = or_sm64(base + (uint64_t)(l >> 1));
        r = (uint32_t)h;
      } else {
        r = (uint32_t)(h >> 32);
      }
      const uint32_t bit = 1u << (j->scale - 1 - l);
      if (r < j->ta) {
      } else if (r < j->tab) {
        d |= bit;
      } else if (r < j->tabc) {
        s |= bit;
      } else {
        s |= bit;
        d |= bit;
      }
    }
    j->src[i] = s;
    j->dst[i] = d;
  }
}

/* Graph500-style recursive quadrant choice, no noise, no permutation.
 * Level l fixes bit (scale-1-l) of (src, dst); 32 random bits per level,
 * compared against integer thresholds so every platform picks the same
 * quadrant. */
void or_rmat_edges(int scale, int ef, double a, double b, double c,
                   uint64_t seed, uint32_t *src, uint32_t *dst) {
  rmat_job j;
  j.scale = scale;
  j.key = or_stream_key(seed, ST_RMAT);
  j.ta = (uint32_t)(a * 4294967296.0);
  j.tab = (uint32_t)((a + b) * 4294967296.0);
  j.tabc = (uint32_t)((a + b + c) * 4294967296.0);
  j.src = src;
  j.dst = dst;
  parallel_for((int64_t)ef << scale, 1 << 16, rmat_range, &j);
}

int64_t or_grid_nedges(int rows, int cols, int lr_div) {
  int64_t eg = (int64_t)rows * (cols - 1) + (int64_t)(rows - 1) * cols;
  return eg + (lr_div > 0 ? eg / lr_div : 0);
}

int64_t or_grid_edges(int rows, int cols, int lr_div, uint64_t seed,
                      uint32_t *src, uint32_t *dst) {
  int64_t k = 0;
  for (int r = 0; r < rows; ++r)
    for (int c = 0; c < cols; ++c) {
      uint32_t v = (uint32_t)r * (uint32_t)cols + (uint32_t)c;
      if (c + 1 < cols) {
        src[k] = v;
        dst[k] = v + 1;
        ++k;
      }
      if (r + 1 < rows) {
        src[k] = v;
        dst[k] = v + (uint32_t)cols;
        ++k;
      }
    }
  const int64_t eg = k;
  const int64_t nlr = lr_div > 0 ? eg / lr_div : 0;
  const uint64_t key = or_stream_key(seed, ST_GRID);
  const uint64_t n = (uint64_t)rows * (uint64_t)cols;
  for (int64_t j = 0; j < nlr; ++j) {
    src[k] = (uint32_t)(or_sm64(key + 2 * (uint64_t)j) % n);
    dst[k] = (uint32_t)(or_sm64(key + 2 * (uint64_t)j + 1) % n);
    ++k;
  }
  return k;
}

void or_er_edges(int64_t n, int64_t m, uint64_t seed, uint32_t *src,
                 uint32_t *dst) {
  const uint64_t key = or_stream_key(seed, ST_ER);
  for (int64_t j = 0; j < m; ++j) {
    src[j] = (uint32_t)(or_sm64(key + 2 * (uint64_t)j) % (uint64_t)n);
    dst[j] = (uint32_t)(or_sm64(key + 2 * (uint64_t)j + 1) % (uint64_t)n);
  }
}

static double unit53(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

void or_er_batch_params(uint64_t seed, int64_t i, int64_t nlo, int64_t nhi,
                        double dlo, double dhi, int64_t *n, int64_t *m,
                        uint64_t *iseed) {
  const uint64_t key = or_stream_key(seed, ST_ERB);
  double u1 = unit53(or_sm64(key + 3 * (uint64_t)i));
  double u2 = unit53(or_sm64(key + 3 * (uint64_t)i + 1));
  double ln = log((double)nlo) + u1 * (log((double)nhi) - log((double)nlo));
  int64_t nn = (int64_t)llround(exp(ln));
  if (nn < nlo) nn = nlo;
  if (nn > nhi) nn = nhi;
  double deg = dlo + u2 * (dhi - dlo);
  *n = nn;
  *m = (int64_t)floor((double)nn * deg / 2.0);
  *iseed = or_sm64(key + 3 * (uint64_t)i + 2);
}

static int cmp_i32(const void *a, const void *b) {
  int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
  return (x > y) - (x < y);
}

typedef struct {
  const uint32_t *src, *dst;
  int64_t *cnt, *cur, *uniq, *off;
  int32_t *tmp, *col;
} csr_job;

static void csr_count(int64_t lo, int64_t hi, void *p) {
  csr_job *j = (csr_job *)p;
  for (int64_t i = lo; i < hi; ++i) {
    if (j->src[i] == j->dst[i]) continue;
    __atomic_fetch_add(&j->cnt[j->src[i] + 1], 1, __ATOMIC_RELAXED);
    __atomic_fetch_add(&j->cnt[j->dst[i] + 1], 1, __ATOMIC_RELAXED);
  }
}
static void csr_scatter(int64_t lo, int64_t hi, void *p) {
  csr_job *j = (csr_job *)p;
  for (int64_t i = lo; i < hi; ++i) {
    if (j->src[i] == j->dst[i]) continue;
    j->tmp[__atomic_fetch_add(&j->cur[j->src[i]], 1, __ATOMIC_RELAXED)] = (int32_t)j->dst[i];
    j->tmp[__atomic_fetch_add(&j->cur[j->dst[i]], 1, __ATOMIC_RELAXED)] = (int32_t)j->src[i];
  }
}
static void csr_sort(int64_t lo, int64_t hi, void *p) {
  csr_job *j = (csr_job *)p;
  for (int64_t v = lo; v < hi; ++v) {
    int32_t *a = j->tmp + j->cnt[v];
    const int64_t len = j->cnt[v + 1] - j->cnt[v];
    if (len > 1) qsort(a, (size_t)len, sizeof(int32_t), cmp_i32);
    int64_t u = 0;
    for (int64_t k = 0; k < len; ++k)
      if (k == 0 || a[k] != a[k - 1]) a[u++] = a[k];
    j->uniq[v] = u;
  }
}
static void csr_compact(int64_t lo, int64_t hi, void *p) {
  csr_job *j = (csr_job *)p;
  for (int64_t v = lo; v < hi; ++v)
    memcpy(j->col + j->off[v], j->tmp + j->cnt[v], sizeof(int32_t) * (size_t)j->uniq[v]);
}

/* Counting build, parallel over pairs and vertices, deterministic: scatter
 * both directions of every non-loop pair, sort and de-duplicate each
 * adjacency, compact. */
int64_t or_csr_build(int64_t n, int64_t npairs, const uint32_t *src,
                     const uint32_t *dst, int64_t **off_out,
                     int32_t **col_out) {
  csr_job j;
  j.src = src;
  j.dst = dst;
  j.cnt = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
  parallel_for(npairs, 1 << 16, csr_count, &j);
  for (int64_t v = 0; v < n; ++v) j.cnt[v + 1] += j.cnt[v];
  const int64_t k = j.cnt[n];
  j.tmp = (int32_t *)malloc(sizeof(int32_t) * (size_t)(k + 1));
  j.cur = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n + 1));
  memcpy(j.cur, j.cnt, sizeof(int64_t) * (size_t)(n + 1));
  parallel_for(npairs, 1 << 16, csr_scatter, &j);
  j.uniq = j.cur; /* reused */
  parallel_for(n, 1024, csr_sort, &j);
  j.off = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n + 1));
  j.off[0] = 0;
  for (int64_t v = 0; v < n; ++v) j.off[v + 1] = j.off[v] + j.uniq[v];
  const int64_t m = j.off[n];
  j.col = (int32_t *)malloc(sizeof(int32_t) * (size_t)(m + 1));
  parallel_for(n, 1024, csr_compact, &j);
  free(j.tmp);
  free(j.cur);
  free(j.cnt);
  *off_out = j.off;
  *col_out = j.col;
  return m;
}

void or_weights(uint64_t seed, int wmax, int64_t n, const int64_t *off,
                const int32_t *col, int32_t *w) {
  const uint64_t key = or_stream_key(seed, ST_W);
  for (int64_t v = 0; v < n; ++v)
    for (int64_t e = off[v]; e < off[v + 1]; ++e) {
      uint64_t u = (uint64_t)col[e];
      uint64_t lo = (uint64_t)v < u ? (uint64_t)v : u;
      uint64_t hi = (uint64_t)v < u ? u : (uint64_t)v;
      w[e] = 1 + (int32_t)(or_sm64(key + ((lo << 32) | hi)) % (uint64_t)wmax);
    }
}

void or_roots(uint64_t seed, int64_t n, const int64_t *off, int count,
              int32_t *roots) {
  const uint64_t key = or_stream_key(seed, ST_ROOT);
  int got = 0;
  uint64_t j = 0;
  const uint64_t budget = 64ull * (uint64_t)n + 4096;
  while (got < count && j < budget) {
    int32_t v = (int32_t)(or_sm64(key + j) % (uint64_t)n);
    ++j;
    if (off[v + 1] == off[v]) continue;
    int dup = 0;
    for (int q = 0; q < got; ++q) dup |= roots[q] == v;
    if (!dup) roots[got++] = v;
  }
  for (int64_t v = 0; got < count && v < n; ++v) { /* tiny graphs */
    if (off[v + 1] == off[v]) continue;
    int dup = 0;
    for (int q = 0; q < got; ++q) dup |= roots[q] == (int32_t)v;
    if (!dup) roots[got++] = (int32_t)v;
  }
  while (got < count) roots[got++] = -1;
}

/* ------------------------------------------------------------------------ */
/* validators                                                                 */
/* ------------------------------------------------------------------------ */

/* bfs_cpu: application/bfs.cu:38-62 (FIFO queue, first discovery wins). */
void or_bfs(int64_t n, const int64_t *off, const int32_t *col, int32_t root,
            int32_t *lvl) {
  int32_t *q = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
  for (int64_t i = 0; i < n; ++i) lvl[i] = -1;
  int64_t head = 0, tail = 0;
  lvl[root] = 0;
  q[tail++] = root;
  while (head < tail) {
    int32_t v = q[head++];
    for (int64_t j = off[v]; j < off[v + 1]; ++j) {
      int32_t u = col[j];
      if (lvl[u] == -1) {
        lvl[u] = lvl[v] + 1;
        q[tail++] = u;
      }
    }
  }
  free(q);
}

/* spfa: application/sssp.cu:55-89 (FIFO label-correcting, in-queue flags,
 * INT_MAX for unreached). */
void or_sssp_spfa(int64_t n, const int64_t *off, const int32_t *col,
                  const int32_t *w, int32_t root, int32_t *dis) {
  /* circular FIFO: at most n vertices are queued at once (in-queue flag) */
  int32_t *q = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
  char *inq = (char *)calloc((size_t)n, 1);
  for (int64_t i = 0; i < n; ++i) dis[i] = INT_MAX;
  int64_t head = 0, cnt = 0, cap = n + 1;
  dis[root] = 0;
  inq[root] = 1;
  q[0] = root;
  cnt = 1;
  while (cnt > 0) {
    int32_t v = q[head];
    head = (head + 1) % cap;
    --cnt;
    inq[v] = 0;
    for (int64_t j = off[v]; j < off[v + 1]; ++j) {
      int32_t u = col[j];
      int32_t nd = dis[v] + w[j];
      if (dis[u] > nd) {
        dis[u] = nd;
        if (!inq[u]) {
          q[(head + cnt) % cap] = u;
          ++cnt;
          inq[u] = 1;
        }
      }
    }
  }
  free(q);
  free(inq);
}

/* Dijkstra with a binary heap (lazy deletion); cross-check for SPFA. */
typedef struct {
  int32_t d;
  int32_t v;
} hnode;
static void hpush(hnode *h, int64_t *sz, hnode x) {
  int64_t i = (*sz)++;
  while (i > 0) {
    int64_t p = (i - 1) >> 1;
    if (h[p].d <= x.d) break;
    h[i] = h[p];
    i = p;
  }
  h[i] = x;
}
static hnode hpop(hnode *h, int64_t *sz) {
  hnode top = h[0], x = h[--(*sz)];
  int64_t i = 0;
  for (;;) {
    int64_t l = 2 * i + 1, r = l + 1, s = i;
    int32_t sd = x.d;
    if (l < *sz && h[l].d < sd) { s = l; sd = h[l].d; }
    if (r < *sz && h[r].d < sd) { s = r; }
    if (s == i) break;
    h[i] = h[s];
    i = s;
  }
  h[i] = x;
  return top;
}
void or_sssp_dijkstra(int64_t n, const int64_t *off, const int32_t *col,
                      const int32_t *w, int32_t root, int32_t *dis) {
  hnode *h = (hnode *)malloc(sizeof(hnode) * (size_t)(off[n] + 2));
  int64_t sz = 0;
  for (int64_t i = 0; i < n; ++i) dis[i] = INT_MAX;
  dis[root] = 0;
  hnode s0 = {0, root};
  hpush(h, &sz, s0);
  while (sz > 0) {
    hnode t = hpop(h, &sz);
    if (t.d != dis[t.v]) continue;
    for (int64_t j = off[t.v]; j < off[t.v + 1]; ++j) {
      int32_t u = col[j];
      int32_t nd = t.d + w[j];
      if (nd < dis[u]) {
        dis[u] = nd;
        hnode x = {nd, u};
        hpush(h, &sz, x);
      }
    }
  }
  free(h);
}

/* Dial's bucket-queue shortest paths (R. B. Dial, CACM 12(11), 1969) for
 * integer weights in [1, wmax]: wmax+1 circular buckets of vertex lists, a
 * vertex settled when its bucket comes round with its label unchanged.  Same
 * distances as spfa / Dijkstra (unique for positive weights) at O(m + n + D)
 * cost, for the large graphs the heap version takes minutes on.  Returns -1
 * when a weight lies outside [1, wmax] (nothing computed), else 0. */
int or_sssp_dial(int64_t n, const int64_t *off, const int32_t *col,
                 const int32_t *w, int32_t root, int32_t wmax, int32_t *dis) {
  const int64_t m = off[n];
  for (int64_t j = 0; j < m; ++j)
    if (w[j] < 1 || w[j] > wmax) return -1;
  const int64_t nb = (int64_t)wmax + 1;
  /* bucket lists as singly linked entries (vertex, next) in a pool that grows
   * by one entry per successful relaxation */
  int64_t cap = n + 16, used = 0;
  int32_t *ev = (int32_t *)malloc(sizeof(int32_t) * (size_t)cap);
  int64_t *en = (int64_t *)malloc(sizeof(int64_t) * (size_t)cap);
  int64_t *head = (int64_t *)malloc(sizeof(int64_t) * (size_t)nb);
  for (int64_t b = 0; b < nb; ++b) head[b] = -1;
  for (int64_t i = 0; i < n; ++i) dis[i] = INT_MAX;
  dis[root] = 0;
  ev[0] = root;
  en[0] = -1;
  head[0] = 0;
  used = 1;
  int64_t pending = 1;
  for (int64_t d = 0; pending > 0; ++d) {
    const int64_t b = d % nb;
    int64_t e = head[b];
    head[b] = -1;
    while (e >= 0) {
      const int32_t v = ev[e];
      const int64_t next = en[e];
      --pending;
      if (dis[v] == d) {
        for (int64_t j = off[v]; j < off[v + 1]; ++j) {
          const int32_t u = col[j];
          const int64_t nd = d + w[j];
          if (nd < dis[u]) {
            dis[u] = (int32_t)nd;
            if (used == cap) {
              cap *= 2;
              ev = (int32_t *)realloc(ev, sizeof(int32_t) * (size_t)cap);
              en = (int64_t *)realloc(en, sizeof(int64_t) * (size_t)cap);
            }
            ev[used] = u;
            en[used] = head[nd % nb];
            head[nd % nb] = used++;
            ++pending;
          }
        }
      }
      e = next;
    }
  }
  free(ev);
  free(en);
  free(head);
  return 0;
}

/* CC_CPU: application/cc.cu:34-66 - components seeded in increasing id
 * order, so every label is the minimum vertex id of its component. */
void or_cc(int64_t n, const int64_t *off, const int32_t *col, int32_t *id) {
  int32_t *q = (int32_t *)malloc(sizeof(int32_t) * (size_t)(off[n] + n + 1));
  for (int64_t i = 0; i < n; ++i) id[i] = (int32_t)i;
  for (int64_t i = 0; i < n; ++i) {
    if (id[i] != i) continue;
    int32_t c = id[i];
    int64_t head = 0, tail = 0;
    q[tail++] = (int32_t)i;
    while (head < tail) {
      int32_t v = q[head++];
      for (int64_t j = off[v]; j < off[v + 1]; ++j) {
        int32_t u = col[j];
        if (id[u] == u) {
          id[u] = c;
          q[tail++] = u;
        }
      }
    }
  }
  free(q);
}

/* The labels of CC_CPU in linear time.  CC_CPU tests "id[u] == u" for
 * "not yet labelled", which also holds for the component's seed, so the seed
 * re-enters the queue once per neighbour and a hub of degree d costs d^2
 * edge visits (hours at RMAT scale 24).  Here the seed is marked when its
 * component starts; every other step is CC_CPU's, so the labels (the
 * smallest vertex id of each component) are the same. */
void or_cc_linear(int64_t n, const int64_t *off, const int32_t *col, int32_t *id) {
  int32_t *q = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
  char *seen = (char *)calloc((size_t)n, 1);
  for (int64_t i = 0; i < n; ++i) id[i] = (int32_t)i;
  for (int64_t i = 0; i < n; ++i) {
    if (seen[i]) continue;
    seen[i] = 1;
    int64_t head = 0, tail = 0;
    q[tail++] = (int32_t)i;
    while (head < tail) {
      int32_t v = q[head++];
      for (int64_t j = off[v]; j < off[v + 1]; ++j) {
        int32_t u = col[j];
        if (!seen[u]) {
          seen[u] = 1;
          id[u] = (int32_t)i;
          q[tail++] = u;
        }
      }
    }
  }
  free(q);
  free(seen);
}

/* bc_cpu: application/bc.cu:162-214, single source, int32 path counts and
 * FP32 dependencies exactly as the reference types them. */
void or_bc_f32(int64_t n, const int64_t *off, const int32_t *col, int32_t root,
               int32_t *nsp, float *dep) {
  int32_t *vis = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  int32_t *order = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
  for (int64_t i = 0; i < n; ++i) { nsp[i] = 0; vis[i] = -1; dep[i] = 0; }
  nsp[root] = 1;
  vis[root] = 1;
  int64_t head = 0, tail = 0;
  order[tail++] = root;
  while (head < tail) { /* forward: order[] doubles as queue and stack */
    int32_t v = order[head++];
    for (int64_t j = off[v]; j < off[v + 1]; ++j) {
      int32_t u = col[j];
      if (vis[u] == -1) { order[tail++] = u; vis[u] = vis[v] + 1; }
      /* int32 wrap-around as the reference's int counter, without UB */
      if (vis[u] == vis[v] + 1) nsp[u] = (int32_t)((uint32_t)nsp[u] + (uint32_t)nsp[v]);
    }
  }
  for (int64_t k = tail - 1; k >= 0; --k) { /* backward: pop in reverse */
    int32_t v = order[k];
    dep[v] *= nsp[v];
    for (int64_t j = off[v]; j < off[v + 1]; ++j) {
      int32_t u = col[j];
      if (vis[u] + 1 == vis[v]) {
        float tmp = (1 + dep[v]) / nsp[v];
        dep[u] += tmp;
      }
    }
  }
  free(vis);
  free(order);
}

/* The same Brandes recurrence in FP64 with FP64 path counts (no overflow). */
void or_bc_f64(int64_t n, const int64_t *off, const int32_t *col, int32_t root,
               double *nsp, double *dep, int32_t *lvl) {
  int32_t *order = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
  for (int64_t i = 0; i < n; ++i) { nsp[i] = 0; lvl[i] = -1; dep[i] = 0; }
  nsp[root] = 1;
  lvl[root] = 0;
  int64_t head = 0, tail = 0;
  order[tail++] = root;
  while (head < tail) {
    int32_t v = order[head++];
    for (int64_t j = off[v]; j < off[v + 1]; ++j) {
      int32_t u = col[j];
      if (lvl[u] == -1) { order[tail++] = u; lvl[u] = lvl[v] + 1; }
      if (lvl[u] == lvl[v] + 1) nsp[u] += nsp[v];
    }
  }
  for (int64_t k = tail - 1; k >= 0; --k) {
    int32_t v = order[k];
    dep[v] *= nsp[v];
    for (int64_t j = off[v]; j < off[v + 1]; ++j) {
      int32_t u = col[j];
      if (lvl[u] + 1 == lvl[v]) dep[u] += (1.0 + dep[v]) / nsp[v];
    }
  }
  free(order);
}

/* PageRank in the reference's unnormalised form (application/pagerank.cu:
 * 19-32,120-125): pr_0 = 1-d; pr_{k+1}(v) = (1-d) + d * sum_{u in N(v)}
 * pr_k(u)/od(u).  FP64 Jacobi for exactly iters steps; returns pr_iters. */
typedef struct {
  const int64_t *off;
  const int32_t *col;
  double damp;
  double *pr, *contrib;
} pr_job;
static void pr_contrib_range(int64_t lo, int64_t hi, void *p) {
  const pr_job *j = (const pr_job *)p;
  for (int64_t v = lo; v < hi; ++v) {
    int64_t od = j->off[v + 1] - j->off[v];
    j->contrib[v] = od ? j->pr[v] / (double)od : j->pr[v];
  }
}
static void pr_gather_range(int64_t lo, int64_t hi, void *p) {
  const pr_job *j = (const pr_job *)p;
  for (int64_t v = lo; v < hi; ++v) {
    double s = 0;
    for (int64_t e = j->off[v]; e < j->off[v + 1]; ++e) s += j->contrib[j->col[e]];
    j->pr[v] = (1.0 - j->damp) + j->damp * s;
  }
}
/* Each vertex's sum runs over its own list in list order whichever thread
 * takes it, so the result does not depend on the thread count. */
void or_pagerank(int64_t n, const int64_t *off, const int32_t *col, int iters,
                 double damp, double *pr) {
  double *contrib = (double *)malloc(sizeof(double) * (size_t)n);
  for (int64_t v = 0; v < n; ++v) pr[v] = 1.0 - damp;
  pr_job j = {off, col, damp, pr, contrib};
  for (int it = 0; it < iters; ++it) {
    parallel_for(n, 1 << 14, pr_contrib_range, &j);
    parallel_for(n, 1 << 12, pr_gather_range, &j);
  }
  free(contrib);
}

/* validation(): application/pagerank.cu:44-79, the fix-point residual test
 * in FP32 on the device's pr/od output.  Returns the first failing vertex or
 * -1 when every vertex passes. */
int64_t or_pagerank_check(int64_t n, const int64_t *off, const int32_t *col,
                          const float *pr_over_od, float damp, float eps) {
  float *pr = (float *)malloc(sizeof(float) * (size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    int64_t od = off[i + 1] - off[i];
    pr[i] = od ? pr_over_od[i] * (float)od : pr_over_od[i];
  }
  int64_t bad = -1;
  for (int64_t i = 0; i < n && bad < 0; ++i) {
    float sum = 0;
    for (int64_t j = off[i]; j < off[i + 1]; ++j) {
      int32_t u = col[j];
      sum += pr[u] / (float)(off[u + 1] - off[u]);
    }
    sum = sum * damp + 1 - damp;
    float diff = (sum - pr[i]) / sum;
    if (!(fabsf(diff) < eps)) bad = i;
  }
  free(pr);
  return bad;
}

/* validation(): application/gc.cu:45-74 - no edge joins two equal colours
 * and no vertex with an edge stays uncoloured (-1).  Returns the first
 * failing vertex or -1. */
int64_t or_gc_check(int64_t n, const int64_t *off, const int32_t *col,
                    const int32_t *color) {
  for (int64_t i = 0; i < n; ++i) {
    int32_t vc = color[i];
    for (int64_t j = off[i]; j < off[i + 1]; ++j) {
      int32_t uc = color[col[j]];
      if (uc == vc && uc != -1) return i;
      if (uc == -1 || vc == -1) return i;
    }
  }
  return -1;
}

/* The colouring application/gc.cu:15-43 computes when its functor runs in the
 * level loop: in the first expand every vertex sends its id to every
 * neighbour; at level L an uncoloured vertex whose id exceeds the largest
 * id it received takes colour L, the others clear their maximum and send
 * their id again.  Deterministic, so GPU colours compare bit for bit. */
void or_gc_levels(int64_t n, const int64_t *off, const int32_t *col, int32_t *color) {
  int32_t *maxid = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  char *active = (char *)malloc((size_t)n);
  for (int64_t v = 0; v < n; ++v) { color[v] = -1; maxid[v] = -1; }
  for (int64_t v = 0; v < n; ++v)
    for (int64_t j = off[v]; j < off[v + 1]; ++j)
      if ((int32_t)v > maxid[col[j]]) maxid[col[j]] = (int32_t)v;
  for (int32_t level = 1;; ++level) {
    int any = 0;
    for (int64_t v = 0; v < n; ++v) {
      active[v] = 0;
      if (color[v] != -1) continue;
      if (maxid[v] < v) {
        color[v] = level;
      } else {
        maxid[v] = -1;
        active[v] = 1;
        any = 1;
      }
    }
    if (!any) break;
    for (int64_t v = 0; v < n; ++v)
      if (active[v])
        for (int64_t j = off[v]; j < off[v + 1]; ++j)
          if ((int32_t)v > maxid[col[j]]) maxid[col[j]] = (int32_t)v;
  }
  free(maxid);
  free(active);
}

void or_mbfs(int64_t n, const int64_t *off, const int32_t *col, int nsrc,
             const int32_t *roots, int32_t *lvl) {
  for (int s = 0; s < nsrc; ++s) or_bfs(n, off, col, roots[s], lvl + (int64_t)s * n);
}

static int cmp_double(const void *a, const void *b) {
  double x = *(const double *)a, y = *(const double *)b;
  return (x > y) - (x < y);
}

/* graph_attr_t::fill: src/utils/fileIO.cuh:35-67, same summation order
 * (ascending degrees) so the doubles agree bit for bit. */
void or_degree_attr(int64_t n, const int64_t *off, double *out) {
  double *t = (double *)malloc(sizeof(double) * (size_t)n);
  for (int64_t i = 0; i < n; ++i) t[i] = (double)(off[i + 1] - off[i]);
  qsort(t, (size_t)n, sizeof(double), cmp_double);
  double avg = 0, sd = 0, gi = 0, her = 0, sum = 0;
  for (int64_t i = 0; i < n; ++i) { avg += t[i]; sd += t[i] * t[i]; }
  sd = sqrt((sd - avg * avg / n) / (n - 1));
  avg /= n;
  double range = t[n - 1] - t[0];
  double mx = t[n - 1];
  for (int64_t i = 1; i <= n; ++i) sum += t[i - 1];
  for (int64_t i = 1; i <= n; ++i) {
    double du = t[i - 1];
    gi += (n - i + 0.5) * du / n / sum;
    if (du != 0) her += du * (log(sum) - log(du)) / sum;
  }
  gi = 1 - 2 * gi;
  her = her / log((double)n);
  out[0] = avg; out[1] = sd; out[2] = range; out[3] = mx; out[4] = gi; out[5] = her;
  free(t);
}

int64_t or_traversed_edges(int64_t n, const int64_t *off, const int32_t *lvl) {
  int64_t s = 0;
  for (int64_t v = 0; v < n; ++v)
    if (lvl[v] >= 0) s += off[v + 1] - off[v];
  return s / 2;
}

/* The six counters of one vertex-centric inspection of a BFS state
 * (src/abstraction/inspector.cuh:39-110): thread t of the 256 x 512 launch
 * visits vertices t, t + 131072, ...; Active = level, Inactive = unreached;
 * [0] active vertices, [1] inactive vertices, [2] their out-degree sum,
 * [3] the inactive out-degree sum, [4] max over blocks of the sum of the
 * threads' largest active degree, [5] sum over blocks of the sum of the
 * threads' largest inactive degree.  Sums are 64-bit here (int32 in the
 * reference). */
void or_inspect_bfs(int64_t n, const int64_t *off, const int32_t *lvl, int32_t level, uint64_t *out) {
  const int64_t S = 256 * 512;
  uint64_t c[4] = {0, 0, 0, 0}, bmax = 0, bsum_l = 0;
  for (int64_t b = 0; b < 256; ++b) {
    uint64_t sp = 0, sl = 0;
    for (int64_t t = b * 512; t < (b + 1) * 512; ++t) {
      uint64_t mp = 0, ml = 0;
      for (int64_t v = t; v < n; v += S) {
        const uint64_t od = (uint64_t)(off[v + 1] - off[v]);
        if (lvl[v] == level) {
          c[0]++;
          c[2] += od;
          if (od > mp) mp = od;
        } else if (lvl[v] < 0) {
          c[1]++;
          c[3] += od;
          if (od > ml) ml = od;
        }
      }
      sp += mp;
      sl += ml;
    }
    if (sp > bmax) bmax = sp;
    bsum_l += sl;
  }
  out[0] = c[0];
  out[1] = c[1];
  out[2] = c[2];
  out[3] = c[3];
  out[4] = bmax;
  out[5] = bsum_l;
}
