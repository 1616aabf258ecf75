// Test-infrastructure driver: runs the REFERENCE's own CPU validator for one
// application on a graph file, to pin the oracle restatement.
//
// The reference application source is #included in place from the reference
// tree (the include path is given by oracle/ref/build_ref.sh); nothing of it
// is copied here.  Its main() is renamed by -Dmain=gsw_ref_app_main and this
// file supplies its own entry point.  The binaries go to oracle/_ref/ only.
//
// Graph file (little endian): int64 n, int64 m, int32 has_w, int32 root,
// int64 off[n+1], int32 col[m], int32 w[m] if has_w.  The arcs are fed to the
// reference's edgelist_t/host_graph_t as a directed list in CSR order with
// quiet=true, so its host CSR is exactly the file's CSR (no rinse/renumber).
#include <atomic>
#include <chrono>
#include <cstdint>
#include <string>
#include <thread>
#include <cstdio>
#include <cstdlib>
#include <vector>

#if defined(GSW_REF_BFS)
#include "application/bfs.cu"
#elif defined(GSW_REF_SSSP)
#include "application/sssp.cu"
#elif defined(GSW_REF_CC)
#include "application/cc.cu"
#elif defined(GSW_REF_BC)
#include "application/bc.cu"
#elif defined(GSW_REF_PR)
#include "application/pagerank.cu"
#elif defined(GSW_REF_GC)
#include "application/gc.cu"
#else
#error "define one GSW_REF_<APP>"
#endif
#undef main

struct gsw_file_graph {
  int64_t n = 0, m = 0;
  int32_t has_w = 0, root = 0;
  std::vector<int64_t> off;
  std::vector<int32_t> col, w;
};

static bool gsw_read_graph(const char *path, gsw_file_graph &g) {
  FILE *f = fopen(path, "rb");
  if (!f) return false;
  bool ok = fread(&g.n, 8, 1, f) == 1 && fread(&g.m, 8, 1, f) == 1 &&
            fread(&g.has_w, 4, 1, f) == 1 && fread(&g.root, 4, 1, f) == 1;
  if (ok) {
    g.off.resize(g.n + 1);
    g.col.resize(g.m);
    ok = fread(g.off.data(), 8, g.n + 1, f) == (size_t)(g.n + 1) &&
         fread(g.col.data(), 4, g.m, f) == (size_t)g.m;
    if (ok && g.has_w) {
      g.w.resize(g.m);
      ok = fread(g.w.data(), 4, g.m, f) == (size_t)g.m;
    }
  }
  fclose(f);
  return ok;
}

template <typename E> static void gsw_push_w(std::vector<E> &v, int32_t w) {
  v.push_back((E)w);
}
template <> void gsw_push_w<Empty>(std::vector<Empty> &, int32_t) {}

template <typename E>
static edgelist_t<E> gsw_to_edgelist(const gsw_file_graph &g) {
  edgelist_t<E> el;
  el.directed = true;
  el.with_weight = g.has_w != 0;
  el.vmin = 0;
  el.vmax = (int)g.n - 1;
  el.nvertexs = (int)g.n;
  el.nedges = (int)g.m;
  el.vvector.reserve(2 * g.m);
  for (int64_t v = 0; v < g.n; ++v)
    for (int64_t e = g.off[v]; e < g.off[v + 1]; ++e) {
      el.vvector.push_back((int)v);
      el.vvector.push_back(g.col[e]);
      if (g.has_w) gsw_push_w<E>(el.evector, g.w[e]);
    }
  return el;
}

template <typename T>
static void gsw_write(const char *path, const T *p, size_t cnt) {
  FILE *f = fopen(path, "wb");
  if (!f) exit(3);
  fwrite(p, sizeof(T), cnt, f);
  fclose(f);
}

int main(int argc, char **argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s graph.bin out.bin [values.bin]\n", argv[0]);
    return 2;
  }
  gsw_file_graph fg;
  if (!gsw_read_graph(argv[1], fg)) {
    fprintf(stderr, "cannot read %s\n", argv[1]);
    return 2;
  }
#if defined(GSW_REF_BFS)
  edgelist_t<Empty> el = gsw_to_edgelist<Empty>(fg);
  host_graph_t<CSR, Empty> hg;
  hg.build(el, true);
  if (argc > 4 && std::string(argv[3]) == "--bench") {
    // timed mode: the reference's bfs_cpu from every root in argv[4]
    // (int32 list); one line per root: root, milliseconds, traversed edges
    std::vector<int> roots;
    FILE *rf = fopen(argv[4], "rb");
    int r;
    while (rf && fread(&r, 4, 1, rf) == 1) roots.push_back(r);
    if (rf) fclose(rf);
    const int threads = argc > 5 ? atoi(argv[5]) : 1;
    const size_t warm = argc > 6 ? (size_t)atoi(argv[6]) : 0;
    if (threads > 1) {
      // throughput mode: `threads` workers share the read-only CSR and each
      // runs the reference's bfs_cpu on the next unclaimed root (bfs_cpu
      // allocates its own state per call); the first `warm` roots run
      // untimed, then one line: timed roots, wall milliseconds, edges
      auto run_set = [&](size_t b, size_t e) {
        std::atomic<size_t> next(b);
        std::atomic<long long> edges(0);
        std::vector<std::thread> ts;
        for (int t = 0; t < threads; ++t)
          ts.emplace_back([&] {
            for (size_t i; (i = next++) < e;) {
              int *lv = bfs_cpu(hg, roots[i]);
              long long te = 0;
              for (int64_t v = 0; v < fg.n; ++v)
                if (lv[v] >= 0) te += fg.off[v + 1] - fg.off[v];
              edges += te / 2;
              free(lv);
            }
          });
        for (auto &t : ts) t.join();
        return edges.load();
      };
      run_set(0, std::min(warm, roots.size()));
      auto t0 = std::chrono::steady_clock::now();
      const long long te = run_set(std::min(warm, roots.size()), roots.size());
      auto t1 = std::chrono::steady_clock::now();
      printf("timed %zu %.6f %lld\n", roots.size() - std::min(warm, roots.size()),
             std::chrono::duration<double, std::milli>(t1 - t0).count(), te);
      return 0;
    }
    for (int root : roots) {
      auto t0 = std::chrono::steady_clock::now();
      int *lv = bfs_cpu(hg, root);
      auto t1 = std::chrono::steady_clock::now();
      long long te = 0;
      for (int64_t v = 0; v < fg.n; ++v)
        if (lv[v] >= 0) te += fg.off[v + 1] - fg.off[v];
      printf("%d %.6f %lld\n", root, std::chrono::duration<double, std::milli>(t1 - t0).count(), te / 2);
      fflush(stdout);
      free(lv);
    }
    return 0;
  }
  int *lvl = bfs_cpu(hg, fg.root);
  gsw_write(argv[2], lvl, fg.n);
  // graph statistics the selector features are built from
  double attr[6] = {hg.attr.avg_deg, hg.attr.std_deg, hg.attr.range,
                    hg.attr.max_deg, hg.attr.GI,      hg.attr.Her};
  if (argc > 3) gsw_write(argv[3], attr, 6);
#elif defined(GSW_REF_SSSP)
  edgelist_t<int> el = gsw_to_edgelist<int>(fg);
  host_graph_t<CSR, int> hg;
  hg.build(el, true);
  int *dis = spfa(hg, fg.root);
  gsw_write(argv[2], dis, fg.n);
#elif defined(GSW_REF_CC)
  edgelist_t<Empty> el = gsw_to_edgelist<Empty>(fg);
  int *id = CC_CPU(el);
  gsw_write(argv[2], id, fg.n);
#elif defined(GSW_REF_BC)
  edgelist_t<Empty> el = gsw_to_edgelist<Empty>(fg);
  host_graph_t<CSR, Empty> hg;
  hg.build(el, true);
  bwdata_t *r = bc_cpu(hg, fg.root);
  gsw_write(argv[2], r, fg.n);
#elif defined(GSW_REF_PR)
  // argv[3]: float pr/od per vertex; the reference's fix-point validation
  // prints passed/failed; the verdict byte (1 = passed) goes to argv[2].
  edgelist_t<Empty> el = gsw_to_edgelist<Empty>(fg);
  host_graph_t<CSR, Empty> hg;
  hg.build(el, true);
  std::vector<float> pr(fg.n);
  FILE *f = argc > 3 ? fopen(argv[3], "rb") : nullptr;
  if (!f || fread(pr.data(), 4, fg.n, f) != (size_t)fg.n) return 2;
  fclose(f);
  fflush(stdout);
  validation(hg, pr.data());
#elif defined(GSW_REF_GC)
  edgelist_t<Empty> el = gsw_to_edgelist<Empty>(fg);
  host_graph_t<CSR, Empty> hg;
  hg.build(el, true);
  std::vector<int> color(fg.n);
  FILE *f = argc > 3 ? fopen(argv[3], "rb") : nullptr;
  if (!f || fread(color.data(), 4, fg.n, f) != (size_t)fg.n) return 2;
  fclose(f);
  validation(hg, color.data(), (int)fg.n);
#endif
  return 0;
}
