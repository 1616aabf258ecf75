// Source-level drop-in for the reference's public header (src/gswitch.h of
// PAA-NCIC/GSWITCH): the seven application mains (application/bfs.cu, cc.cu,
// sssp.cu, pagerank.cu, bc.cu, gc.cu, mbfs.cu) compile against this header
// unchanged (nvcc -I gswitch_b200/compat) and run on this engine: their
// functors are inlined into this engine's sm_100a kernels, and their level
// loops call this engine's inspector / selector / executor.
//
// What the header supplies beyond the engine: the command line of
// src/utils/cmdline.cuh, the helpers of src/utils/utils.cuh, the .mtx
// edge-list reader and the host CSR of src/utils/fileIO.cuh (same id shift,
// self-loop removal, duplicate removal and isolated-vertex compaction, so a
// file gives the same graph and the same vertex ids as in the reference),
// build_graph / graph_t (src/data_structures/graph.cuh:176-280), and
// init_conf / reset_conf / build_active_set / p_jump with the reference's
// signatures.  Forced variants come from `-c Dir-Fmt-LB-Fusion` as in the
// reference.
#pragma once
#include <getopt.h>
#include <sys/stat.h>
#include <sys/time.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "../csrc/engine/executor.cuh"

using namespace gsw;

// ---------------------------------------------------------------------------
// src/utils/cmdline.cuh:27-232
// ---------------------------------------------------------------------------
struct cmd_t {
  int src = -1;
  std::string configs = "";
  std::string path = "";
  std::string json = "";
  bool verbose = false;
  bool validation = false;
  bool with_header = false;
  bool with_weight = false;
  bool directed = false;
  int device = 0;
  ins_t ins;

  // "Dir-Fmt-LB-Fusion", any field "x" (or missing) left to the selector
  void prase_configs(const std::string &input) {
    std::vector<std::string> c;
    std::istringstream iss(input);
    std::string t;
    while (std::getline(iss, t, '-')) c.push_back(t);
    while (c.size() < 4) c.push_back("x");
    ins = ins_t();
    if (c[0] == "Push" || c[0] == "Pull") {
      ins.has_direction = true;
      ins.d = c[0] == "Push" ? Push : Pull;
    }
    if (c[1] == "Queue" || c[1] == "Bitmap") {
      ins.has_asfmt = true;
      ins.asf = c[1] == "Queue" ? Queue : Bitmap;
    }
    const char *lbs[] = {"TM", "WM", "CM", "STRICT", "TWOD", "ELB", "TWC"};
    for (int i = 0; i < 7; ++i)
      if (c[2] == lbs[i]) {
        ins.has_lb = true;
        ins.lb = (LB)i;
      }
    if (c[3] == "Fused" || c[3] == "Standalone") {
      ins.has_fusion = true;
      ins.fusion = c[3] == "Fused" ? Fused : Standalone;
    }
  }
};
inline cmd_t cmd_opt;

#define LOG(...) \
  if (cmd_opt.verbose) fprintf(stdout, __VA_ARGS__);

inline void gsw_compat_help(const std::string &exec) {
  std::cout << "./" << exec << " <graph_path> [options]\n"
            << "  -r, --src=<int>        root vertex (default: random non-isolated)\n"
            << "  -v, --verbose          per-level trace\n"
            << "  -V, --validation       CPU reference validation\n"
            << "  -H, --with-header      the file has a size line\n"
            << "  -W, --with-weight      the file has edge weights\n"
            << "  -d, --directed         the graph is directed\n"
            << "  -c, --configs=Push-Queue-CM-Fused   force choices (x = selector)\n"
            << "  -D, --device=<int>     GPU\n"
            << "  -j, --json=<string>    append feature_t::record() blocks to this file\n";
}

inline void parse_cmd(int argc, char *argv[], std::string exec = "test") {
  if (argc < 2) {
    gsw_compat_help(exec);
    exit(0);
  }
  cmd_opt.path = argv[1];
  struct stat sb;
  if (stat(cmd_opt.path.c_str(), &sb) != 0) {
    std::cout << " file \"" << cmd_opt.path << "\" does not exist." << std::endl;
    exit(0);
  }
  const struct option longopts[] = {
      {"src", required_argument, 0, 'r'},     {"verbose", no_argument, 0, 'v'},
      {"validation", no_argument, 0, 'V'},    {"with-header", no_argument, 0, 'H'},
      {"with-weight", no_argument, 0, 'W'},   {"directed", no_argument, 0, 'd'},
      {"configs", required_argument, 0, 'c'}, {"json", required_argument, 0, 'j'},
      {"device", required_argument, 0, 'D'},  {0, 0, 0, 0},
  };
  int idx, opt;
  optind = 1;
  while ((opt = getopt_long(argc - 1, &argv[1], "r:vVHWdc:j:D:", longopts, &idx)) != -1) {
    switch (opt) {
      case 'r': cmd_opt.src = atoi(optarg); break;
      case 'v': cmd_opt.verbose = true; break;
      case 'V': cmd_opt.validation = true; break;
      case 'H': cmd_opt.with_header = true; break;
      case 'W': cmd_opt.with_weight = true; break;
      case 'd': cmd_opt.directed = true; break;
      case 'c': cmd_opt.configs = optarg; break;
      case 'j': cmd_opt.json = optarg; break;
      case 'D': cmd_opt.device = atoi(optarg); break;
      default: gsw_compat_help(exec); exit(0);
    }
  }
  cmd_opt.prase_configs(cmd_opt.configs);
  opts().verbose = cmd_opt.verbose;
  cudaSetDevice(cmd_opt.device);
}

// ---------------------------------------------------------------------------
// src/utils/utils.cuh
// ---------------------------------------------------------------------------
inline double wtime() {
  timeval tv;
  gettimeofday(&tv, nullptr);
  return tv.tv_sec + tv.tv_usec * 1e-6;
}
inline double mwtime() { return 1000 * wtime(); }

// validation tolerance of the BC and PageRank checks (utils.cuh:186-193):
// relative 1e-2 above magnitude 1, absolute below; NaN / inf accepted
inline bool isAcceptable(float a, float b) {
  if (std::isnan(a) || std::isinf(a)) return true;
  if (std::fabs(a) > 1) return std::fabs(b / a - 1) < 1e-2;
  return std::fabs(b - a) < 1e-2;
}

// ---------------------------------------------------------------------------
// src/utils/fileIO.cuh:30-67 degree statistics (the graph features the
// selector trees read)
// ---------------------------------------------------------------------------
struct graph_attr_t {
  double avg_deg = 0, std_deg = 0, max_deg = 0, range = 0, GI = 0, Her = 0;
  void fill(const int *deg, int nv) {
    std::vector<double> t(deg, deg + nv);
    std::sort(t.begin(), t.end());
    avg_deg = std_deg = GI = Her = 0;
    for (double x : t) {
      avg_deg += x;
      std_deg += x * x;
    }
    std_deg = std::sqrt((std_deg - avg_deg * avg_deg / nv) / (nv - 1));
    avg_deg /= nv;
    range = t[nv - 1] - t[0];
    max_deg = t[nv - 1];
    double sum = 0;
    for (int i = 1; i <= nv; ++i) sum += t[i - 1];
    for (int i = 1; i <= nv; ++i) {
      const double du = t[i - 1];
      GI += (nv - i + 0.5) * du / nv / sum;
      if (du != 0) Her += du * (std::log(sum) - std::log(du)) / sum;
    }
    GI = 1 - 2 * GI;
    Her = Her / std::log((double)nv);
  }
};

// ---------------------------------------------------------------------------
// src/utils/fileIO.cuh:69-206 edge list: .mtx text, comment lines skipped,
// optional size line, "v0 v1 [w]" per line, self-loops dropped, ids later
// shifted by the smallest id seen
// ---------------------------------------------------------------------------
template <typename E>
struct edgelist_t {
  std::vector<int> vvector;
  std::vector<E> evector;
  int vmin = 0, vmax = -1;
  int nvertexs = 0;
  int nedges = 0;
  bool directed = false;
  bool with_weight = false;
  double mean_weight = 0;

  void read_mtx(std::string path, bool directed_ = false, bool with_weight_ = false, bool with_header = false) {
    directed = directed_;
    with_weight = with_weight_;
    std::ifstream fin(path);
    if (!fin.is_open()) {
      fprintf(stderr, "can not open file %s\n", path.c_str());
      exit(1);
    }
    while (true) {
      const int c = fin.peek();
      if (c == EOF || (c >= '0' && c <= '9')) break;
      fin.ignore(std::numeric_limits<std::streamsize>::max(), fin.widen('\n'));
    }
    if (with_header) {
      fin >> nvertexs >> nvertexs >> nedges;
      fin.ignore(std::numeric_limits<std::streamsize>::max(), fin.widen('\n'));
    }
    vvector.clear();
    evector.clear();
    vmin = std::numeric_limits<int>::max();
    vmax = -1;
    double tot = 0;
    while (fin.good()) {
      int v0, v1;
      fin >> v0 >> v1;
      if (fin.eof()) break;
      vmin = std::min(vmin, std::min(v0, v1));
      vmax = std::max(vmax, std::max(v0, v1));
      E w{};
      if (with_weight)
        read_weight(fin, w);
      else
        fin.ignore(std::numeric_limits<std::streamsize>::max(), fin.widen('\n'));
      if (fin.eof()) break;
      if (v0 == v1) continue;
      vvector.push_back(v0);
      vvector.push_back(v1);
      if (with_weight) {
        evector.push_back(w);
        tot += weight_value(w);
      }
    }
    nvertexs = vmax - vmin + 1;
    nedges = (int)(vvector.size() >> 1);
    if (nvertexs <= 0 || nedges == 0) exit(1);
    if (with_weight) mean_weight = tot / evector.size();
  }

  // weights 1..lim from the C library's rand() (rand_weight of the reference)
  void gen_weight(int lim) {
    if (with_weight) return;
    with_weight = true;
    evector.clear();
    double tot = 0;
    for (int i = 0; i < nedges; ++i) {
      E w = make_weight(rand() % lim + 1);
      tot += weight_value(w);
      evector.push_back(w);
    }
    mean_weight = tot / nedges;
  }

 private:
  template <typename T>
  static void read_weight(std::istream &in, T &w) {
    in >> w;
  }
  static void read_weight(std::istream &in, Empty &) {
    double skip;
    in >> skip;
  }
  template <typename T>
  static double weight_value(const T &w) {
    return (double)w;
  }
  static double weight_value(const Empty &) { return 0; }
  static E make_weight(int x) {
    if constexpr (std::is_same<E, Empty>::value)
      return E{};
    else
      return (E)x;
  }
};

// ---------------------------------------------------------------------------
// src/utils/fileIO.cuh:206-450 host CSR: both directions of every listed
// pair for undirected graphs; unweighted graphs are "rinsed" (neighbour
// lists sorted, duplicates removed, isolated vertices removed and the rest
// renumbered in order)
// ---------------------------------------------------------------------------
template <GraphFmt Fmt, typename E>
class host_graph_t {};

template <typename E>
class host_graph_t<CSR, E> {
 public:
  E *edge_weights = nullptr;
  int *adj_list = nullptr;
  int *start_pos = nullptr;
  int *odegrees = nullptr;
  E *r_edge_weights = nullptr;
  int *r_adj_list = nullptr;
  int *r_start_pos = nullptr;
  int *r_odegrees = nullptr;
  int nvertexs = 0;
  int nedges = 0;
  bool directed = false;
  bool with_weight = false;
  graph_attr_t attr;

  void build(edgelist_t<E> el, bool quiet = false) {
    directed = el.directed;
    with_weight = !std::is_same<Empty, E>::value;
    const int vmin = el.vmin;
    nvertexs = el.vmax - el.vmin + 1;
    nedges = (int)(el.vvector.size() >> 1);
    if (!directed) nedges <<= 1;
    odegrees = (int *)calloc(nvertexs, sizeof(int));
    start_pos = (int *)malloc(sizeof(int) * (nvertexs + 1));
    adj_list = (int *)malloc(sizeof(int) * std::max(nedges, 1));
    if (with_weight) edge_weights = (E *)malloc(sizeof(E) * std::max(nedges, 1));
    if (directed) {
      r_odegrees = (int *)calloc(nvertexs, sizeof(int));
      r_start_pos = (int *)malloc(sizeof(int) * (nvertexs + 1));
      r_adj_list = (int *)malloc(sizeof(int) * std::max(nedges, 1));
      if (with_weight) r_edge_weights = (E *)malloc(sizeof(E) * std::max(nedges, 1));
    }
    for (size_t i = 0; i < el.vvector.size(); i += 2) {
      odegrees[el.vvector[i] - vmin]++;
      if (!directed)
        odegrees[el.vvector[i + 1] - vmin]++;
      else
        r_odegrees[el.vvector[i + 1] - vmin]++;
    }
    prefix(start_pos, odegrees);
    if (directed) prefix(r_start_pos, r_odegrees);
    for (size_t i = 0; i < (el.vvector.size() >> 1); ++i) {
      const int v0 = el.vvector[2 * i] - vmin, v1 = el.vvector[2 * i + 1] - vmin;
      put(adj_list, edge_weights, start_pos, odegrees, v0, v1, el, i);
      if (!directed)
        put(adj_list, edge_weights, start_pos, odegrees, v1, v0, el, i);
      else
        put(r_adj_list, r_edge_weights, r_start_pos, r_odegrees, v1, v0, el, i);
    }
    if (!quiet && !with_weight) rinse();
    attr.fill(odegrees, nvertexs);
  }

  // Binary CSR cache (src/utils/fileIO.cuh:334-387): "<dir>/.csr_<file>"
  // holds int nvertexs, int nedges, bool directed, bool with_weight, then
  // odegrees[n], start_pos[n], adj_list[m] (+ edge_weights[m]) and, for
  // directed graphs, the same four arrays of the reverse graph -- the
  // reference's byte layout, so either side reads the other's cache.  An
  // existing cache is left as it is; loading a missing one exits(1), both as
  // the reference does.  A path without a directory resolves to ".".
  static std::string binfile_path(const std::string &fname) {
    const size_t k = fname.find_last_of('/');
    const std::string dir = k == std::string::npos ? "." : fname.substr(0, k);
    const std::string base = k == std::string::npos ? fname : fname.substr(k + 1);
    return dir + "/.csr_" + base;
  }
  void store_to_binfile(std::string fname) {
    const std::string fpath = binfile_path(fname);
    if (FILE *chk = fopen(fpath.c_str(), "rb")) {
      fclose(chk);
      return;
    }
    std::ofstream fout(fpath, std::ios::binary);
    fout.write((const char *)&nvertexs, sizeof(nvertexs));
    fout.write((const char *)&nedges, sizeof(nvertexs));
    fout.write((const char *)&directed, sizeof(directed));
    fout.write((const char *)&with_weight, sizeof(with_weight));
    write_side(fout, odegrees, start_pos, adj_list, edge_weights);
    if (directed) write_side(fout, r_odegrees, r_start_pos, r_adj_list, r_edge_weights);
  }
  void load_from_binfile(std::string fname) {
    const std::string fpath = binfile_path(fname);
    std::ifstream fin(fpath, std::ios::binary);
    if (!fin) exit(1);
    fin.read((char *)&nvertexs, sizeof(nvertexs));
    fin.read((char *)&nedges, sizeof(nvertexs));
    fin.read((char *)&directed, sizeof(directed));
    fin.read((char *)&with_weight, sizeof(with_weight));
    read_side(fin, odegrees, start_pos, adj_list, edge_weights);
    if (directed) read_side(fin, r_odegrees, r_start_pos, r_adj_list, r_edge_weights);
    attr.fill(odegrees, nvertexs);
  }

  // a random vertex with out-edges (C library random(), as the reference)
  int random_root() {
    while (true) {
      const int r = (int)(random() % nvertexs);
      if (odegrees[r]) return r;
    }
  }

 private:
  void write_side(std::ofstream &out, const int *deg, const int *sp, const int *adj, const E *w) const {
    out.write((const char *)deg, sizeof(int) * nvertexs);
    out.write((const char *)sp, sizeof(int) * nvertexs);
    out.write((const char *)adj, sizeof(int) * nedges);
    if (with_weight) out.write((const char *)w, sizeof(E) * nedges);
  }
  void read_side(std::ifstream &in, int *&deg, int *&sp, int *&adj, E *&w) {
    free(deg), free(sp), free(adj), free(w);
    deg = (int *)malloc(sizeof(int) * std::max(nvertexs, 1));
    sp = (int *)malloc(sizeof(int) * (nvertexs + 1));
    adj = (int *)malloc(sizeof(int) * std::max(nedges, 1));
    w = with_weight ? (E *)malloc(sizeof(E) * std::max(nedges, 1)) : nullptr;
    in.read((char *)deg, sizeof(int) * nvertexs);
    in.read((char *)sp, sizeof(int) * nvertexs);
    in.read((char *)adj, sizeof(int) * nedges);
    if (with_weight) in.read((char *)w, sizeof(E) * nedges);
    sp[nvertexs] = nedges;
  }
  void prefix(int *sp, int *deg) {
    sp[0] = 0;
    for (int i = 1; i <= nvertexs; ++i) sp[i] = sp[i - 1] + deg[i - 1];
    for (int i = 0; i < nvertexs; ++i) deg[i] = 0;
  }
  static void put(int *adj, E *w, const int *sp, int *deg, int v, int u, const edgelist_t<E> &el, size_t i) {
    adj[sp[v] + deg[v]] = u;
    if constexpr (!std::is_same<E, Empty>::value) {
      if (w) w[sp[v] + deg[v]] = el.evector[i];
    }
    deg[v]++;
  }
  void rinse() {
    int t = 0;
    for (int v = 0; v < nvertexs; ++v) {
      const int s = start_pos[v], e = start_pos[v + 1];
      start_pos[v] = t;
      std::sort(adj_list + s, adj_list + e);
      for (int j = s; j < e; ++j)
        if (j == s || adj_list[j] != adj_list[j - 1]) adj_list[t++] = adj_list[j];
      odegrees[v] = t - start_pos[v];
    }
    start_pos[nvertexs] = t;
    nedges = t;
    std::vector<int> rename(nvertexs, -1);
    int top = 0;
    for (int v = 0; v < nvertexs; ++v)
      if (odegrees[v]) rename[v] = top++;
    int k = 0;
    for (int v = 0; v < nvertexs; ++v) {
      if (!odegrees[v]) continue;
      const int s = start_pos[v], d = odegrees[v];
      start_pos[k] = s;
      odegrees[k] = d;
      for (int j = s; j < s + d; ++j) adj_list[j] = rename[adj_list[j]];
      ++k;
    }
    nvertexs = top;
    start_pos[nvertexs] = nedges;
  }
};

// edge-centric host form: one packed (v << 32 | u) word per listed pair
template <typename E>
class host_graph_t<COO, E> {
 public:
  E *edge_weights = nullptr;
  packed_t *edge_list = nullptr;
  int nvertexs = 0;
  int nedges = 0;
  bool directed = false;
  bool with_weight = false;
  graph_attr_t attr;

  void build(edgelist_t<E> el, bool = false) {
    directed = el.directed;
    with_weight = el.with_weight;
    nvertexs = el.vmax - el.vmin + 1;
    nedges = (int)(el.vvector.size() >> 1);
    edge_list = (packed_t *)malloc(sizeof(packed_t) * std::max(nedges, 1));
    if constexpr (!std::is_same<E, Empty>::value) {
      if (with_weight) edge_weights = (E *)malloc(sizeof(E) * std::max(nedges, 1));
    }
    for (int i = 0; i < nedges; ++i) {
      const int v0 = el.vvector[2 * i] - el.vmin, v1 = el.vvector[2 * i + 1] - el.vmin;
      edge_list[i] = ((int64_t)v0) << 32 | v1;
      if constexpr (!std::is_same<E, Empty>::value) {
        if (with_weight) edge_weights[i] = el.evector[i];
      }
    }
  }
};

// ---------------------------------------------------------------------------
// src/data_structures/graph.cuh:176-280 graph bundle and build_graph
// ---------------------------------------------------------------------------
namespace gsw_compat {
template <typename T>
T *to_device(const T *h, size_t count) {
  T *d = nullptr;
  if (cudaMalloc((void **)&d, sizeof(T) * (count ? count : 1)) != cudaSuccess) {
    fprintf(stderr, "gswitch: device allocation of %zu bytes failed\n", sizeof(T) * count);
    exit(1);
  }
  if (count) cudaMemcpy(d, h, sizeof(T) * count, cudaMemcpyHostToDevice);
  return d;
}
// int32 start positions + degrees -> int64 row offsets (n + 1)
inline std::vector<int64_t> offsets(const int *start_pos, int n, int nedges) {
  std::vector<int64_t> off(n + 1);
  for (int i = 0; i < n; ++i) off[i] = start_pos[i];
  off[n] = nedges;
  return off;
}
template <typename E>
device_graph_t<CSR, E> upload(const host_graph_t<CSR, E> &hg) {
  device_graph_t<CSR, E> g;
  const auto off = offsets(hg.start_pos, hg.nvertexs, hg.nedges);
  g.dg_row_off = to_device(off.data(), off.size());
  g.dg_adj_list = to_device(hg.adj_list, (size_t)hg.nedges);
  g.dg_odegree = to_device(hg.odegrees, (size_t)hg.nvertexs);
  g.dg_edgedata = std::is_same<E, Empty>::value ? nullptr : to_device(hg.edge_weights, (size_t)hg.nedges);
  if (hg.directed) {
    const auto roff = offsets(hg.r_start_pos, hg.nvertexs, hg.nedges);
    g.dgr_row_off = to_device(roff.data(), roff.size());
    g.dgr_adj_list = to_device(hg.r_adj_list, (size_t)hg.nedges);
    g.dgr_odegree = to_device(hg.r_odegrees, (size_t)hg.nvertexs);
    g.dgr_edgedata = std::is_same<E, Empty>::value ? nullptr : to_device(hg.r_edge_weights, (size_t)hg.nedges);
  } else {
    g.dgr_row_off = g.dg_row_off;
    g.dgr_adj_list = g.dg_adj_list;
    g.dgr_odegree = g.dg_odegree;
    g.dgr_edgedata = g.dg_edgedata;
  }
  g.nvertexs = hg.nvertexs;
  g.nedges = hg.nedges;
  g.level = 0;
  g.directed = hg.directed;
  return g;
}
template <typename E>
device_graph_t<COO, E> upload(const host_graph_t<COO, E> &hg) {
  device_graph_t<COO, E> g;
  g.dg_coo = to_device(hg.edge_list, (size_t)hg.nedges);
  g.dg_edgedata = (std::is_same<E, Empty>::value || !hg.edge_weights) ? nullptr
                                                                      : to_device(hg.edge_weights, (size_t)hg.nedges);
  g.nvertexs = hg.nvertexs;
  g.nedges = hg.nedges;
  g.level = 0;
  return g;
}
template <GraphFmt Fmt, typename E>
void set_features(feature_t &fets, const edgelist_t<E> &el, const host_graph_t<Fmt, E> &hg) {
  fets.avg_deg = hg.attr.avg_deg;
  fets.std_deg = hg.attr.std_deg;
  fets.range = hg.attr.range;
  fets.max_deg = hg.attr.max_deg;
  fets.GI = hg.attr.GI;
  fets.Her = hg.attr.Her;
  fets.nvertexs = el.nvertexs;
  fets.nedges = el.nedges;
  fets.avg_edata = el.mean_weight;
}
}  // namespace gsw_compat

template <GraphFmt Fmt, typename E>
struct graph_t {
  edgelist_t<E> el;
  host_graph_t<Fmt, E> hg;
  device_graph_t<Fmt, E> dg;
};

template <Centric C, typename E>
struct gsw_graph_fmt {
  static constexpr GraphFmt value = C == VC ? CSR : COO;
};

template <Centric C, typename E = Empty>
graph_t<gsw_graph_fmt<C, E>::value, E> build_graph(edgelist_t<E> el, feature_t &fets) {
  graph_t<gsw_graph_fmt<C, E>::value, E> g;
  g.el = el;
  g.hg.build(g.el);
  if (C == EC) {  // the vertex features come from the CSR form of the same list
    host_graph_t<CSR, E> h;
    h.build(g.el, true);
    g.hg.attr = h.attr;
  }
  g.dg = gsw_compat::upload(g.hg);
  gsw_compat::set_features(fets, g.el, g.hg);
  // fets.record() appends to the -j file (features.cuh:96-104 reads
  // cmd_opt.json the same way); no -j, no records
  fets.record_path = cmd_opt.json.empty() ? nullptr : cmd_opt.json.c_str();
  return g;
}

template <Centric C, typename E = Empty>
graph_t<gsw_graph_fmt<C, E>::value, E> build_graph(std::string path, feature_t &fets, bool with_header = false,
                                                   bool with_weight = false, bool directed = false) {
  edgelist_t<E> el;
  el.read_mtx(path, directed, with_weight, with_header);
  return build_graph<C, E>(el, fets);
}

// ---------------------------------------------------------------------------
// src/gswitch.h:19-108 and the engine calls with the reference's signatures
// ---------------------------------------------------------------------------
inline active_set_t build_active_set(int64_t size, const config_t &conf) {
  return gsw::build_active_set(size, conf.conf_qmode);
}

template <typename G, typename F>
void init_conf(stat_t &stats, feature_t &fets, config_t &conf, G &g, F &f) {
  conf.force = cmd_opt.ins;
  init_conf_impl(stats, fets, conf, g.dg, f, g.el.mean_weight, g.hg.attr.avg_deg, false);
}

template <typename G, typename F>
void reset_conf(stat_t &stats, feature_t &fets, config_t &conf, G &g, F &f) {
  conf.force = cmd_opt.ins;
  init_conf_impl(stats, fets, conf, g.dg, f, g.el.mean_weight, g.hg.attr.avg_deg, true);
}

// CC root compression after a hooking level (src/utils/intrinsics.cuh:
// 328-362); the flag buffers of the reference's signature are not needed
template <typename F>
void p_jump(F &f, int nvertexs, int *, int *) {
  static unsigned *err = nullptr;
  if (!err) cudaMalloc((void **)&err, sizeof(unsigned));
  k_pointer_jump<<<resident_grid(k_pointer_jump, 512), 512, 0, stream()>>>((int *)f.data.dg_wa, nvertexs, err);
}
