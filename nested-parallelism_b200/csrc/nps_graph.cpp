// Host-side graph construction for the SSSP library: seeded generators, the
// CSR builder and the DIMACS9 / DIMACS10 / SNAP ("SLNDC") front-ends.
//
// CSR convention.  The reference builds CSR from per-vertex std::list
// adjacency lists by popping from the back (common/global.cpp:211-225), so every
// row holds its edges in REVERSE insertion order and vertexArray[n] = m.  The
// builder here keeps that convention, so a graph written with
// nps_write_dimacs9() and read back by the reference's readInputDIMACS9() +
// convertCSR() yields the same arrays.
//
// Random numbers.  Generators use a counter-based stream: every edge (or
// undirected pair) owns a key derived from (seed, index) with splitmix64
// (Steele, Lea, Flood 2014), and successive draws hash key + k * golden-ratio.
// Output is therefore independent of the thread count.
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <list>
#include <string>
#include <vector>

#include <omp.h>

#include "nps.h"
#include "nps_internal.h"

namespace {

inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

struct Stream {
  uint64_t key;
  uint64_t k = 0;
  Stream(uint64_t seed, uint64_t salt, uint64_t index)
      : key(splitmix64(splitmix64(seed ^ salt) ^ (index * 0xD6E8FEB86659FD93ull))) {}
  uint64_t next() { return splitmix64(key + (k++) * 0x9E3779B97F4A7C15ull); }
  // uniform integer in [0, n) by multiply-high of the top 32 bits
  uint32_t below(uint32_t n) { return (uint32_t)(((next() >> 32) * (uint64_t)n) >> 32); }
  double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

constexpr uint64_t kSaltUniform = 0x756E69666F726D31ull;  // "uniform1"
constexpr uint64_t kSaltRmat = 0x726D617431323334ull;
constexpr uint64_t kSaltGridDrop = 0x6772696464726F70ull;
constexpr uint64_t kSaltGridW = 0x677269647765696Full;

bool alloc_graph(nps_graph* g, int32_t n, int64_t m) {
  g->n = n;
  g->m = m;
  g->source = 0;
  g->row_ptr = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n + 1));
  g->col = (int32_t*)malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(m, 1));
  g->w = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)std::max<int64_t>(m, 1));
  if (!g->row_ptr || !g->col || !g->w) {
    free(g->row_ptr);
    free(g->col);
    free(g->w);
    g->row_ptr = g->col = nullptr;
    g->w = nullptr;
    return false;
  }
  return true;
}

// Highest out-degree vertex, lowest id on ties.
int32_t max_degree_vertex(const nps_graph* g) {
  int32_t best = 0, bestd = -1;
  for (int32_t v = 0; v < g->n; ++v) {
    int32_t d = g->row_ptr[v + 1] - g->row_ptr[v];
    if (d > bestd) {
      bestd = d;
      best = v;
    }
  }
  return best;
}

}  // namespace

// ---------------------------------------------------------------------------
// CSR builder: stable bucket of edges by source with per-thread histograms,
// optional (src,dst) dedupe keeping the earliest edge, rows reversed.
nps_status nps_build_csr(int32_t n, int64_t m, const int32_t* src, const int32_t* dst,
                         const uint32_t* w, bool dedupe, bool drop_self, nps_graph* out) {
  if (n <= 0 || m < 0 || m >= (int64_t)INT32_MAX) return nps_fail(NPS_ERR_INVALID_ARG, "csr: bad n/m");
  const int T = std::max(1, std::min(omp_get_max_threads(), 64));
  const int64_t per = (m + T - 1) / T;
  // per-thread counts: count[t*(n) + v]; use 32-bit counts
  std::vector<int32_t> cnt((size_t)T * n, 0);
  std::atomic<bool> bad{false};
#pragma omp parallel num_threads(T)
  {
    int t = omp_get_thread_num();
    int64_t lo = std::min(m, t * per), hi = std::min(m, lo + per);
    int32_t* c = cnt.data() + (size_t)t * n;
    for (int64_t e = lo; e < hi; ++e) {
      int32_t s = src[e], d = dst[e];
      if ((uint32_t)s >= (uint32_t)n || (uint32_t)d >= (uint32_t)n) {
        bad = true;
        continue;
      }
      if (drop_self && s == d) continue;
      c[s]++;
    }
  }
  if (bad) return nps_fail(NPS_ERR_FORMAT, "csr: vertex id out of range");
  // offsets: row-major over (v, t)
  std::vector<int64_t> rowstart((size_t)n + 1);
  {
    int64_t acc = 0;
    for (int32_t v = 0; v < n; ++v) {
      rowstart[v] = acc;
      for (int t = 0; t < T; ++t) {
        int32_t c = cnt[(size_t)t * n + v];
        cnt[(size_t)t * n + v] = (int32_t)(acc - rowstart[v]);  // offset within the row
        acc += c;
      }
    }
    rowstart[n] = acc;
  }
  const int64_t mk = rowstart[n];
  std::vector<int64_t> order((size_t)std::max<int64_t>(mk, 1));  // edge ids bucketed by src, ascending id
#pragma omp parallel num_threads(T)
  {
    int t = omp_get_thread_num();
    int64_t lo = std::min(m, t * per), hi = std::min(m, lo + per);
    int32_t* c = cnt.data() + (size_t)t * n;
    for (int64_t e = lo; e < hi; ++e) {
      int32_t s = src[e], d = dst[e];
      if (drop_self && s == d) continue;
      order[rowstart[s] + c[s]++] = e;
    }
  }
  cnt.clear();
  cnt.shrink_to_fit();
  // per-row dedupe -> kept count
  std::vector<int32_t> keep((size_t)n, 0);
  if (dedupe) {
#pragma omp parallel num_threads(T)
    {
      std::vector<std::pair<int32_t, int64_t>> tmp;
#pragma omp for schedule(dynamic, 256)
      for (int32_t v = 0; v < n; ++v) {
        int64_t a = rowstart[v], b = rowstart[v + 1];
        if (b - a <= 1) {
          keep[v] = (int32_t)(b - a);
          continue;
        }
        tmp.clear();
        for (int64_t i = a; i < b; ++i) tmp.emplace_back(dst[order[i]], order[i]);
        std::sort(tmp.begin(), tmp.end());
        int64_t k = 0;
        for (size_t i = 0; i < tmp.size(); ++i)
          if (i == 0 || tmp[i].first != tmp[i - 1].first) tmp[k++] = tmp[i];
        // kept edge ids back in ascending (insertion) order
        std::vector<int64_t> ids((size_t)k);
        for (int64_t i = 0; i < k; ++i) ids[i] = tmp[i].second;
        std::sort(ids.begin(), ids.end());
        for (int64_t i = 0; i < k; ++i) order[a + i] = ids[i];
        keep[v] = (int32_t)k;
      }
    }
  } else {
    for (int32_t v = 0; v < n; ++v) keep[v] = (int32_t)(rowstart[v + 1] - rowstart[v]);
  }
  int64_t mout = 0;
  for (int32_t v = 0; v < n; ++v) mout += keep[v];
  if (!alloc_graph(out, n, mout)) return nps_fail(NPS_ERR_OOM, "csr: host allocation failed");
  {
    int64_t acc = 0;
    for (int32_t v = 0; v < n; ++v) {
      out->row_ptr[v] = (int32_t)acc;
      acc += keep[v];
    }
    out->row_ptr[n] = (int32_t)acc;
  }
#pragma omp parallel for num_threads(T) schedule(dynamic, 1024)
  for (int32_t v = 0; v < n; ++v) {
    int64_t a = rowstart[v];
    int32_t k = keep[v];
    int32_t o = out->row_ptr[v];
    for (int32_t i = 0; i < k; ++i) {  // reverse insertion order
      int64_t e = order[a + (k - 1 - i)];
      out->col[o + i] = dst[e];
      out->w[o + i] = w[e];
    }
  }
  return NPS_OK;
}

extern "C" nps_status nps_csr_from_edges(int32_t n, int64_t m, const int32_t* src,
                                         const int32_t* dst, const uint32_t* w, int32_t dedupe,
                                         int32_t drop_self_loops, nps_graph* out) {
  if (!out || (m > 0 && (!src || !dst || !w))) return nps_fail(NPS_ERR_INVALID_ARG, "csr: null pointer");
  memset(out, 0, sizeof(*out));
  return nps_build_csr(n, m, src, dst, w, dedupe != 0, drop_self_loops != 0, out);
}

extern "C" void nps_graph_free(nps_graph* g) {
  if (!g) return;
  free(g->row_ptr);
  free(g->col);
  free(g->w);
  g->row_ptr = nullptr;
  g->col = nullptr;
  g->w = nullptr;
  g->n = 0;
  g->m = 0;
}

extern "C" uint64_t nps_fnv1a_u32(const uint32_t* a, int64_t n) {
  uint64_t h = 1469598103934665603ull;
  for (int64_t i = 0; i < n; ++i) h = (h ^ (uint64_t)a[i]) * 1099511628211ull;
  return h;
}

// ---------------------------------------------------------------------------
// Generators

extern "C" nps_status nps_gen_uniform(int32_t n, int64_t m, uint32_t wmax, uint64_t seed,
                                      nps_graph* out) {
  if (!out || n < 2 || m < 0 || m >= (int64_t)INT32_MAX || wmax == 0)
    return nps_fail(NPS_ERR_INVALID_ARG, "gen_uniform: need n>=2, 0<=m<2^31, wmax>=1");
  memset(out, 0, sizeof(*out));
  std::vector<int32_t> s((size_t)m), d((size_t)m);
  std::vector<uint32_t> w((size_t)m);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < m; ++e) {
    Stream r(seed, kSaltUniform, (uint64_t)e);
    uint32_t u, v;
    do {  // self-loops are rejected and the pair redrawn
      u = r.below((uint32_t)n);
      v = r.below((uint32_t)n);
    } while (u == v);
    s[e] = (int32_t)u;
    d[e] = (int32_t)v;
    w[e] = 1 + r.below(wmax);
  }
  nps_status st = nps_build_csr(n, m, s.data(), d.data(), w.data(), false, false, out);
  if (st == NPS_OK) out->source = 0;
  return st;
}

extern "C" nps_status nps_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b,
                                   double c, uint32_t wmax, uint64_t seed, nps_graph* out) {
  if (!out || scale < 1 || scale > 30 || edge_factor < 1 || wmax == 0 || a < 0 || b < 0 || c < 0 ||
      a + b + c > 1.0 + 1e-12)
    return nps_fail(NPS_ERR_INVALID_ARG, "gen_rmat: bad parameters");
  const int64_t n = (int64_t)1 << scale;
  const int64_t m = n * edge_factor;
  if (m >= (int64_t)INT32_MAX) return nps_fail(NPS_ERR_INVALID_ARG, "gen_rmat: too many edges");
  memset(out, 0, sizeof(*out));
  std::vector<int32_t> s((size_t)m), d((size_t)m);
  std::vector<uint32_t> w((size_t)m);
  const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < m; ++e) {
    Stream r(seed, kSaltRmat, (uint64_t)e);
    uint32_t u = 0, v = 0;
    for (int l = scale - 1; l >= 0; --l) {  // one quadrant draw per level, most significant first
      double x = r.unit();
      if (x < a) {
      } else if (x < ab) {
        v |= 1u << l;
      } else if (x < abc) {
        u |= 1u << l;
      } else {
        u |= 1u << l;
        v |= 1u << l;
      }
    }
    s[e] = (int32_t)u;
    d[e] = (int32_t)v;
    w[e] = 1 + r.below(wmax);
  }
  nps_status st = nps_build_csr((int32_t)n, m, s.data(), d.data(), w.data(), true, true, out);
  if (st == NPS_OK) out->source = max_degree_vertex(out);
  return st;
}

extern "C" nps_status nps_gen_grid(int32_t rows, int32_t cols, double drop, uint32_t wmax,
                                   uint64_t seed, nps_graph* out) {
  if (!out || rows < 1 || cols < 1 || (int64_t)rows * cols >= (int64_t)INT32_MAX || wmax == 0 ||
      drop < 0 || drop >= 1)
    return nps_fail(NPS_ERR_INVALID_ARG, "gen_grid: bad parameters");
  memset(out, 0, sizeof(*out));
  const int64_t n = (int64_t)rows * cols;
  const uint64_t hpairs = (uint64_t)rows * (cols - 1);
  const uint64_t cut = (uint64_t)(drop * 18446744073709551616.0);
  auto kept_pair = [&](uint64_t pid) {
    Stream r(seed, kSaltGridDrop, pid);
    return r.next() >= cut;
  };
  // pair ids: horizontal (r,c)-(r,c+1) = r*(cols-1)+c ; vertical (r,c)-(r+1,c) = hpairs + r*cols + c
  // insertion order per vertex: north, south, west, east; rows stored reversed (east, west, south, north)
  std::vector<int32_t> deg((size_t)n);
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < n; ++v) {
    int32_t r = (int32_t)(v / cols), c = (int32_t)(v % cols), k = 0;
    if (r > 0 && kept_pair(hpairs + (uint64_t)(r - 1) * cols + c)) k++;
    if (r + 1 < rows && kept_pair(hpairs + (uint64_t)r * cols + c)) k++;
    if (c > 0 && kept_pair((uint64_t)r * (cols - 1) + (c - 1))) k++;
    if (c + 1 < cols && kept_pair((uint64_t)r * (cols - 1) + c)) k++;
    deg[v] = k;
  }
  int64_t m = 0;
  for (int64_t v = 0; v < n; ++v) m += deg[v];
  if (!alloc_graph(out, (int32_t)n, m)) return nps_fail(NPS_ERR_OOM, "gen_grid: allocation failed");
  {
    int64_t acc = 0;
    for (int64_t v = 0; v < n; ++v) {
      out->row_ptr[v] = (int32_t)acc;
      acc += deg[v];
    }
    out->row_ptr[n] = (int32_t)acc;
  }
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < n; ++v) {
    int32_t r = (int32_t)(v / cols), c = (int32_t)(v % cols);
    int32_t o = out->row_ptr[v];
    auto put = [&](int32_t dstv, int dir) {
      Stream rw(seed, kSaltGridW, (uint64_t)v * 4 + dir);
      out->col[o] = dstv;
      out->w[o] = 1 + rw.below(wmax);
      ++o;
    };
    if (c + 1 < cols && kept_pair((uint64_t)r * (cols - 1) + c)) put((int32_t)(v + 1), 3);
    if (c > 0 && kept_pair((uint64_t)r * (cols - 1) + (c - 1))) put((int32_t)(v - 1), 2);
    if (r + 1 < rows && kept_pair(hpairs + (uint64_t)r * cols + c)) put((int32_t)(v + cols), 1);
    if (r > 0 && kept_pair(hpairs + (uint64_t)(r - 1) * cols + c)) put((int32_t)(v - cols), 0);
  }
  out->source = 0;
  return NPS_OK;
}

// ---------------------------------------------------------------------------
// File front-ends.  Each parses into per-vertex adjacency lists in file order
// and then lays rows out in reverse, as readInput*() + convertCSR() do.

namespace {

struct LineReader {
  FILE* f;
  std::vector<char> buf;
  explicit LineReader(FILE* fp) : f(fp), buf(1 << 20) {}
  // reads one line (without size limit); returns false at EOF
  bool next(std::string& line) {
    line.clear();
    while (fgets(buf.data(), (int)buf.size(), f)) {
      line.append(buf.data());
      if (!line.empty() && line.back() == '\n') return true;
    }
    return !line.empty();
  }
};

nps_status lists_to_csr(int32_t n, const std::vector<std::vector<int32_t>>& adj,
                        const std::vector<std::vector<uint32_t>>& wts, nps_graph* out) {
  int64_t m = 0;
  for (auto& a : adj) m += (int64_t)a.size();
  if (m >= (int64_t)INT32_MAX) return nps_fail(NPS_ERR_FORMAT, "reader: too many edges");
  if (!alloc_graph(out, n, m)) return nps_fail(NPS_ERR_OOM, "reader: allocation failed");
  int64_t acc = 0;
  for (int32_t v = 0; v < n; ++v) {
    out->row_ptr[v] = (int32_t)acc;
    const auto& a = adj[v];
    const auto& ww = wts[v];
    for (size_t i = 0; i < a.size(); ++i) {  // back of the list first (global.cpp:217-220)
      out->col[acc + i] = a[a.size() - 1 - i];
      out->w[acc + i] = ww[a.size() - 1 - i];
    }
    acc += (int64_t)a.size();
  }
  out->row_ptr[n] = (int32_t)acc;
  return NPS_OK;
}

}  // namespace

// readInputDIMACS9 (common/global.cpp:29-64): "c" comments, "p sp N M",
// optional "s SRC", "a U V W"; ids 1-based.
extern "C" nps_status nps_read_dimacs9(const char* path, nps_graph* out) {
  if (!path || !out) return nps_fail(NPS_ERR_INVALID_ARG, "dimacs9: null argument");
  memset(out, 0, sizeof(*out));
  FILE* f = fopen(path, "r");
  if (!f) return nps_fail(NPS_ERR_IO, std::string("dimacs9: cannot open ") + path);
  LineReader lr(f);
  std::string line;
  int64_t n = -1, mdecl = 0;
  int32_t source = 0;
  std::vector<std::vector<int32_t>> adj;
  std::vector<std::vector<uint32_t>> wts;
  nps_status st = NPS_OK;
  while (lr.next(line)) {
    if (line.empty() || line[0] == 'c') continue;
    if (line[0] == 'p') {
      char kind[16] = {0};
      long long nn = 0, mm = 0;
      if (sscanf(line.c_str() + 1, "%15s %lld %lld", kind, &nn, &mm) != 3 || nn <= 0 || nn >= INT32_MAX) {
        st = nps_fail(NPS_ERR_FORMAT, "dimacs9: bad problem line");
        break;
      }
      n = nn;
      mdecl = mm;
      adj.assign((size_t)n, {});
      wts.assign((size_t)n, {});
    } else if (line[0] == 's') {
      long long s = 0;
      if (sscanf(line.c_str() + 1, "%lld", &s) != 1) {
        st = nps_fail(NPS_ERR_FORMAT, "dimacs9: bad source line");
        break;
      }
      source = (int32_t)(s - 1);
    } else if (line[0] == 'a') {
      long long u = 0, v = 0, wgt = 0;
      if (n < 0 || sscanf(line.c_str() + 1, "%lld %lld %lld", &u, &v, &wgt) != 3 || u < 1 || v < 1 ||
          u > n || v > n || wgt < 0 || wgt > 0x7fffffffLL) {
        st = nps_fail(NPS_ERR_FORMAT, "dimacs9: bad arc line");
        break;
      }
      adj[u - 1].push_back((int32_t)(v - 1));
      wts[u - 1].push_back((uint32_t)wgt);
    }
  }
  fclose(f);
  if (st != NPS_OK) return st;
  if (n < 0) return nps_fail(NPS_ERR_FORMAT, "dimacs9: missing problem line");
  (void)mdecl;
  st = lists_to_csr((int32_t)n, adj, wts, out);
  if (st == NPS_OK) {
    if (source < 0 || source >= n) {
      nps_graph_free(out);
      return nps_fail(NPS_ERR_FORMAT, "dimacs9: source out of range");
    }
    out->source = source;
  }
  return st;
}

// readInputDIMACS10 (common/global.cpp:66-105): '%' comments, header "N M"
// (undirected M, 2M arcs), then one line per vertex listing 1-based neighbours.
// Weights are rand() % 1000 + 1 after srand(7), drawn in file order; libc's
// rand() is used so the sequence matches a reference build on the same libc.
extern "C" nps_status nps_read_dimacs10(const char* path, nps_graph* out) {
  if (!path || !out) return nps_fail(NPS_ERR_INVALID_ARG, "dimacs10: null argument");
  memset(out, 0, sizeof(*out));
  FILE* f = fopen(path, "r");
  if (!f) return nps_fail(NPS_ERR_IO, std::string("dimacs10: cannot open ") + path);
  LineReader lr(f);
  std::string line;
  bool have_header = false;
  long long n = 0, mu = 0;
  while (lr.next(line)) {
    if (!line.empty() && line[0] == '%') continue;
    if (sscanf(line.c_str(), "%lld %lld", &n, &mu) != 2 || n <= 0 || n >= INT32_MAX) {
      fclose(f);
      return nps_fail(NPS_ERR_FORMAT, "dimacs10: bad header");
    }
    have_header = true;
    break;
  }
  if (!have_header) {
    fclose(f);
    return nps_fail(NPS_ERR_FORMAT, "dimacs10: missing header");
  }
  std::vector<std::vector<int32_t>> adj((size_t)n);
  std::vector<std::vector<uint32_t>> wts((size_t)n);
  srand(7);
  for (long long i = 0; i < n; ++i) {
    if (!lr.next(line)) {
      fclose(f);
      return nps_fail(NPS_ERR_FORMAT, "dimacs10: parsing adjacency list fails");
    }
    const char* p = line.c_str();
    char* endp = nullptr;
    for (;;) {
      while (*p == ' ' || *p == '\t') ++p;
      if (*p == '\n' || *p == '\r' || *p == 0) break;
      long long h = strtoll(p, &endp, 10);
      if (endp == p || h < 1 || h > n) {
        fclose(f);
        return nps_fail(NPS_ERR_FORMAT, "dimacs10: bad neighbour id");
      }
      p = endp;
      adj[i].push_back((int32_t)(h - 1));
      wts[i].push_back((uint32_t)(rand() % 1000 + 1));
    }
  }
  fclose(f);
  int64_t m = 0;
  for (auto& a : adj) m += (int64_t)a.size();
  if (m != 2 * mu) return nps_fail(NPS_ERR_FORMAT, "dimacs10: arc count differs from 2*M in the header");
  nps_status st = lists_to_csr((int32_t)n, adj, wts, out);
  if (st == NPS_OK) out->source = 0;
  return st;
}

// readInputSLNDC (common/global.cpp:107-190): SNAP edge list.  Two comment
// lines, "# Nodes: N Edges: M", one more comment line, then "tail head" pairs.
// Ids that occur are renumbered densely in increasing order; weights are
// rand() % 1000 + 1 after srand(7), drawn per tail id ascending, in file order.
extern "C" nps_status nps_read_slndc(const char* path, nps_graph* out) {
  if (!path || !out) return nps_fail(NPS_ERR_INVALID_ARG, "slndc: null argument");
  memset(out, 0, sizeof(*out));
  FILE* f = fopen(path, "r");
  if (!f) return nps_fail(NPS_ERR_IO, std::string("slndc: cannot open ") + path);
  LineReader lr(f);
  std::string line;
  long long nhdr = 0;
  for (int k = 0; k < 4; ++k) {
    if (!lr.next(line)) {
      fclose(f);
      return nps_fail(NPS_ERR_FORMAT, "slndc: truncated header");
    }
    if (k == 2) {
      const char* p = strstr(line.c_str(), "Nodes:");
      if (!p || sscanf(p + 6, "%lld", &nhdr) != 1 || nhdr <= 0 || nhdr >= INT32_MAX / 2) {
        fclose(f);
        return nps_fail(NPS_ERR_FORMAT, "slndc: parsing total node number fails");
      }
    }
  }
  const int64_t idcap = 2 * nhdr;
  std::vector<std::vector<int32_t>> tmp((size_t)idcap);
  std::vector<char> seen((size_t)idcap, 0);
  long long t = 0, h = 0;
  int64_t maxid = 0;
  while (fscanf(f, "%lld%lld", &t, &h) == 2) {
    if (t < 0 || h < 0 || t >= idcap || h >= idcap) {
      fclose(f);
      return nps_fail(NPS_ERR_FORMAT, "slndc: node id beyond twice the declared node count");
    }
    seen[t] = seen[h] = 1;
    maxid = std::max<int64_t>(maxid, std::max(t, h));
    tmp[t].push_back((int32_t)h);
  }
  fclose(f);
  std::vector<int32_t> map((size_t)idcap, -1);
  int32_t n = 0;
  for (int64_t i = 0; i <= maxid; ++i)
    if (seen[i]) map[i] = n++;
  if (n == 0) return nps_fail(NPS_ERR_FORMAT, "slndc: no edges");
  std::vector<std::vector<int32_t>> adj((size_t)n);
  std::vector<std::vector<uint32_t>> wts((size_t)n);
  srand(7);
  for (int64_t i = 0; i <= maxid; ++i) {
    if (map[i] < 0) continue;
    for (int32_t hh : tmp[i]) {
      adj[map[i]].push_back(map[hh]);
      wts[map[i]].push_back((uint32_t)(rand() % 1000 + 1));
    }
  }
  nps_status st = lists_to_csr(n, adj, wts, out);
  if (st == NPS_OK) out->source = 0;
  return st;
}

// DIMACS9 writer: rows are emitted in insertion order (the reverse of the CSR
// row), so readInputDIMACS9() + convertCSR() rebuild identical arrays.
extern "C" nps_status nps_write_dimacs9(const char* path, const nps_graph* g, int32_t source) {
  if (!path || !g || !g->row_ptr || g->n <= 0) return nps_fail(NPS_ERR_INVALID_ARG, "write_dimacs9: bad argument");
  if (source < 0 || source >= g->n) return nps_fail(NPS_ERR_INVALID_ARG, "write_dimacs9: source out of range");
  FILE* f = fopen(path, "w");
  if (!f) return nps_fail(NPS_ERR_IO, std::string("write_dimacs9: cannot open ") + path);
  std::vector<char> buf(1 << 22);
  setvbuf(f, buf.data(), _IOFBF, buf.size());
  fprintf(f, "c written by libnps\np sp %d %lld\ns %d\n", g->n, (long long)g->m, source + 1);
  for (int32_t v = 0; v < g->n; ++v) {
    for (int32_t e = g->row_ptr[v + 1] - 1; e >= g->row_ptr[v]; --e)
      fprintf(f, "a %d %d %u\n", v + 1, g->col[e] + 1, g->w[e]);
  }
  bool ok = ferror(f) == 0;
  ok = (fclose(f) == 0) && ok;
  return ok ? NPS_OK : nps_fail(NPS_ERR_IO, "write_dimacs9: write failed");
}
