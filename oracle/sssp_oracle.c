/*
 * sssp_oracle.c -- CPU oracle for the SSSP hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: only tests/, the smoke
 * check in __graft_entry__.py and the cpu_baseline / reference legs of bench.py
 * load it.  The library (nested-parallelism_b200/) never links or calls it, and
 * has no CPU fallback.
 *
 * Restated algorithms (paths relative to the dadaism/nested-parallelism tree):
 *
 *   oracle_sssp_heap   SSSP_CPU() in apps/sssp/src/cpu/sssp.cpp:13-47 on the
 *                      Heap class of common/heap.cpp:29-109: lazy-insertion
 *                      binary-heap Dijkstra.  Pop (id, key); if cost[id] is still
 *                      INF, settle it with key and insert (nid, key + w) for every
 *                      out-edge whose head is unsettled (sssp.cpp:29-41).
 *   oracle_sssp_dheap  Dijkstra with decrease-key on a d-ary heap with the item /
 *                      key API of common/dheap.h:55-78 (items 1..N, insert,
 *                      changekey, deletemin, member); the reference ships the heap
 *                      with no SSSP driver, so the driver is written here.
 *   oracle_sssp_state  the label-correcting fixpoint that sssp_np_consolidate_gpu()
 *                      computes from an arbitrary cost[] / update[] state
 *                      (apps/sssp/src/gpu/sssp_wrapper.cu:475-546 with the
 *                      relaxation of sssp_kernel.cu:49-52), as a FIFO worklist.
 *
 *   oracle_bc          bc_cpu() of the bc application (apps/bc/src/cpu/bc.cpp:152-186
 *                      with bc_kernel.cpp:3-106): Brandes betweenness centrality,
 *                      one source after another.  Forward: a level-synchronous BFS
 *                      from the source counting shortest paths, sigma[v] += sigma[u]
 *                      for every edge u -> v with level[v] = level[u] + 1
 *                      (bc_kernel.cpp:29-49; int sums, wrapping like the reference's
 *                      __sync_fetch_and_add).  Backward, deepest level first: for u at
 *                      level L, over its edges in CSR order to v at level L + 1,
 *                      delta[u] = (float)((double)delta[u] + (double)sigma[u] /
 *                      sigma[v] * (1.0f + delta[v])) -- the reference's p[u][v] = 1 is
 *                      exactly "edge u -> v and level[v] = level[u] + 1"
 *                      (bc_kernel.cpp:51-64); then bc[v] += delta[v] in float for every
 *                      reached v other than the source (:83-101).  MAX_LEVEL = 9999
 *                      marks unvisited vertices, as in common/global.h:17.
 *
 *   oracle_color       the coloring of the graph-color application
 *                      (gclr_bitmap_kernel, apps/graph-color/src/gpu/graph_color_kernel.cu:14-35,
 *                      iterated by gclr_nopruning_gpu, graph_color_wrapper.cu:113-130): in iteration c an
 *                      uncolored v takes c unless an out-neighbour u < v is uncolored
 *                      or colored c.  Both block v whatever the order, so v ends with
 *                      1 + the largest color of its smaller out-neighbours; in id order
 *                      those are final when v is reached.  The reference has no CPU
 *                      version of this path; the result is pinned to its GPU program's
 *                      colors (tests/golden/color_reference.json).
 *
 *   oracle_gen_rmat    the benchmark's seeded R-MAT input (a restatement of this
 *                      library's own generator, so the reference's CPU path can be
 *                      timed on the same graph without loading the library).
 *
 * Distances are uint32 with INF = 2^30 (sssp_wrapper.cu:7, common/global.h:19).
 * A tentative distance that reaches 2^30 is treated as unreachable; the
 * reference's int arithmetic never gets there on the inputs it is run on.
 *
 * Pinned by tests/golden/: goldens produced by running the reference's own
 * SSSP_CPU (compiled from its sources by oracle/Makefile into oracle/_ref/).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_INF 0x40000000u

typedef struct {
  uint32_t key;
  int32_t id;
} hitem;

/* binary min-heap on key (ties in any order: they do not change distances) */
typedef struct {
  hitem* a;
  int64_t n, cap;
} bheap;

static int bheap_push(bheap* h, uint32_t key, int32_t id) {
  if (h->n == h->cap) {
    int64_t nc = h->cap ? 2 * h->cap : 1024;
    hitem* na = (hitem*)realloc(h->a, (size_t)nc * sizeof(hitem));
    if (!na) return -1;
    h->a = na;
    h->cap = nc;
  }
  int64_t i = h->n++;
  while (i > 0) {
    int64_t p = (i - 1) >> 1;
    if (h->a[p].key <= key) break;
    h->a[i] = h->a[p];
    i = p;
  }
  h->a[i].key = key;
  h->a[i].id = id;
  return 0;
}

static hitem bheap_pop(bheap* h) {
  hitem top = h->a[0];
  hitem last = h->a[--h->n];
  int64_t i = 0;
  for (;;) {
    int64_t l = 2 * i + 1, r = l + 1, c = i;
    uint32_t ck = last.key;
    if (l < h->n && h->a[l].key < ck) {
      c = l;
      ck = h->a[l].key;
    }
    if (r < h->n && h->a[r].key < ck) c = r;
    if (c == i) break;
    h->a[i] = h->a[c];
    i = c;
  }
  if (h->n > 0) h->a[i] = last;
  return top;
}

/* Returns 0 on success, -1 on bad arguments, -2 on allocation failure. */
int oracle_sssp_heap(int32_t n, const int32_t* row, const int32_t* col, const uint32_t* w, int32_t src,
                     uint32_t* dist) {
  if (n <= 0 || src < 0 || src >= n || !row || !dist) return -1;
  for (int32_t i = 0; i < n; ++i) dist[i] = ORACLE_INF;
  bheap h = {0, 0, 0};
  if (bheap_push(&h, 0u, src)) return -2;
  while (h.n > 0) {
    hitem it = bheap_pop(&h);
    if (dist[it.id] != ORACLE_INF) continue; /* already settled: lazy deletion */
    dist[it.id] = it.key;
    for (int32_t e = row[it.id]; e < row[it.id + 1]; ++e) {
      int32_t v = col[e];
      if (dist[v] != ORACLE_INF) continue;
      uint64_t nd = (uint64_t)it.key + w[e];
      if (nd >= ORACLE_INF) continue;
      if (bheap_push(&h, (uint32_t)nd, v)) {
        free(h.a);
        return -2;
      }
    }
  }
  free(h.a);
  return 0;
}

/* d-ary heap over items 1..N with positions and keys (the dheap.h layout):
 * parent(x) = (x + d - 2) / d, children d(x-1)+2 .. dx+1. */
typedef struct {
  int d;
  int64_t n;
  int64_t* h;   /* h[1..n] items */
  int64_t* pos; /* pos[item], 0 = absent */
  uint64_t* key;
} dheap;

static void dh_siftup(dheap* H, int64_t i, int64_t x) {
  while (x > 1) {
    int64_t px = (x + H->d - 2) / H->d;
    if (H->key[H->h[px]] <= H->key[i]) break;
    H->h[x] = H->h[px];
    H->pos[H->h[x]] = x;
    x = px;
  }
  H->h[x] = i;
  H->pos[i] = x;
}

static int64_t dh_minchild(dheap* H, int64_t x) {
  int64_t first = (int64_t)H->d * (x - 1) + 2;
  if (first > H->n) return 0;
  int64_t last = (int64_t)H->d * x + 1, mc = first;
  for (int64_t y = first + 1; y <= last && y <= H->n; ++y)
    if (H->key[H->h[y]] < H->key[H->h[mc]]) mc = y;
  return mc;
}

static void dh_siftdown(dheap* H, int64_t i, int64_t x) {
  int64_t cx = dh_minchild(H, x);
  while (cx != 0 && H->key[H->h[cx]] < H->key[i]) {
    H->h[x] = H->h[cx];
    H->pos[H->h[x]] = x;
    x = cx;
    cx = dh_minchild(H, x);
  }
  H->h[x] = i;
  H->pos[i] = x;
}

int oracle_sssp_dheap(int32_t n, const int32_t* row, const int32_t* col, const uint32_t* w, int32_t src, int d,
                      uint32_t* dist) {
  if (n <= 0 || src < 0 || src >= n || !row || !dist || d < 2) return -1;
  dheap H;
  H.d = d;
  H.n = 0;
  H.h = (int64_t*)malloc(sizeof(int64_t) * ((size_t)n + 1));
  H.pos = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
  H.key = (uint64_t*)malloc(sizeof(uint64_t) * ((size_t)n + 1));
  char* done = (char*)calloc((size_t)n, 1);
  if (!H.h || !H.pos || !H.key || !done) {
    free(H.h);
    free(H.pos);
    free(H.key);
    free(done);
    return -2;
  }
  for (int32_t i = 0; i < n; ++i) dist[i] = ORACLE_INF;
  dist[src] = 0;
  /* insert: item = vertex + 1 */
  H.key[src + 1] = 0;
  H.n = 1;
  dh_siftup(&H, src + 1, 1);
  while (H.n > 0) {
    int64_t it = H.h[1];
    /* deletemin: move the last item into the root position */
    int64_t j = H.h[H.n--];
    if (it != j) dh_siftdown(&H, j, 1);
    H.pos[it] = 0;
    int32_t u = (int32_t)(it - 1);
    done[u] = 1;
    for (int32_t e = row[u]; e < row[u + 1]; ++e) {
      int32_t v = col[e];
      if (done[v]) continue;
      uint64_t nd = (uint64_t)dist[u] + w[e];
      if (nd >= ORACLE_INF || nd >= dist[v]) continue;
      dist[v] = (uint32_t)nd;
      H.key[v + 1] = nd;
      if (H.pos[v + 1]) {
        dh_siftup(&H, v + 1, H.pos[v + 1]); /* changekey to a smaller key */
      } else {
        H.n++;
        dh_siftup(&H, v + 1, H.n);
      }
    }
  }
  free(H.h);
  free(H.pos);
  free(H.key);
  free(done);
  return 0;
}

/* Label-correcting fixpoint from a state: cost[] is updated in place, update[]
 * flags the initial frontier and is cleared.  FIFO worklist with an in-queue flag. */
int oracle_sssp_state(int32_t n, const int32_t* row, const int32_t* col, const uint32_t* w, uint32_t* cost,
                      uint8_t* update) {
  if (n <= 0 || !row || !cost || !update) return -1;
  int32_t* q = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  char* inq = (char*)calloc((size_t)n, 1);
  if (!q || !inq) {
    free(q);
    free(inq);
    return -2;
  }
  int64_t head = 0, count = 0;
  for (int32_t v = 0; v < n; ++v)
    if (update[v]) {
      update[v] = 0;
      q[(head + count++) % n] = v;
      inq[v] = 1;
    }
  while (count > 0) {
    int32_t u = q[head];
    head = (head + 1) % n;
    count--;
    inq[u] = 0;
    uint32_t du = cost[u];
    if (du >= ORACLE_INF) continue;
    for (int32_t e = row[u]; e < row[u + 1]; ++e) {
      int32_t v = col[e];
      uint64_t nd = (uint64_t)du + w[e];
      if (nd >= ORACLE_INF || nd >= cost[v]) continue;
      cost[v] = (uint32_t)nd;
      if (!inq[v]) {
        inq[v] = 1;
        q[(head + count++) % n] = v;
      }
    }
  }
  free(q);
  free(inq);
  return 0;
}

/* Out-edges of reached vertices (m_r) and reached-vertex count (n_r). */
void oracle_reached(int32_t n, const int32_t* row, const uint32_t* dist, int64_t* n_r, int64_t* m_r) {
  int64_t a = 0, b = 0;
  for (int32_t v = 0; v < n; ++v)
    if (dist[v] < ORACLE_INF) {
      a++;
      b += row[v + 1] - row[v];
    }
  *n_r = a;
  *m_r = b;
}

uint64_t oracle_fnv1a_u32(const uint32_t* a, int64_t n) {
  uint64_t h = 1469598103934665603ull;
  for (int64_t i = 0; i < n; ++i) h = (h ^ (uint64_t)a[i]) * 1099511628211ull;
  return h;
}

/* Betweenness centrality of every vertex over the sources in `sources` (all
 * vertices in id order when sources is NULL), as bc_cpu() accumulates it; see
 * the header for the steps.  bc[n] is overwritten.  Returns 0, or -1 when out of
 * memory. */
#define ORACLE_MAX_LEVEL 9999
int oracle_bc(int32_t n, const int32_t* row, const int32_t* col, int32_t nsrc, const int32_t* sources,
              float* bc) {
  int32_t* level = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  int32_t* sigma = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  float* delta = (float*)malloc(sizeof(float) * (size_t)n);
  int32_t* order = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  int32_t* lb = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n + 2));
  if (!level || !sigma || !delta || !order || !lb) {
    free(level), free(sigma), free(delta), free(order), free(lb);
    return -1;
  }
  for (int32_t v = 0; v < n; ++v) {
    bc[v] = 0.0f;
    level[v] = ORACLE_MAX_LEVEL;
    sigma[v] = 0;
    delta[v] = 0.0f;
  }
  const int32_t count = sources ? nsrc : n;
  for (int32_t k = 0; k < count; ++k) {
    const int32_t s = sources ? sources[k] : k;
    int32_t tail = 0, dist = 0;
    level[s] = 0;
    sigma[s] = 1;
    order[tail++] = s;
    lb[0] = 0;
    lb[1] = 1;
    /* forward: frontier = the vertices of level `dist` */
    while (lb[dist] < lb[dist + 1]) {
      for (int32_t i = lb[dist]; i < lb[dist + 1]; ++i) {
        const int32_t u = order[i];
        for (int32_t e = row[u]; e < row[u + 1]; ++e) {
          const int32_t v = col[e];
          if (level[v] == ORACLE_MAX_LEVEL) {
            level[v] = dist + 1;
            order[tail++] = v;
          }
          if (level[v] == dist + 1) sigma[v] = (int32_t)((uint32_t)sigma[v] + (uint32_t)sigma[u]);
        }
      }
      lb[dist + 2] = tail;
      ++dist;
    }
    /* here dist = deepest level + 1, as the reference's loop leaves it */
    for (int32_t d = dist; d > 1; --d) {
      for (int32_t i = lb[d - 2]; i < lb[d - 1]; ++i) { /* u at level d - 2 */
        const int32_t u = order[i];
        float du = delta[u];
        for (int32_t e = row[u]; e < row[u + 1]; ++e) {
          const int32_t v = col[e];
          if (level[v] == d - 1) du = (float)((double)du + (double)sigma[u] / (double)sigma[v] * (double)(1.0f + delta[v]));
        }
        delta[u] = du;
      }
      for (int32_t i = lb[d - 1]; i < lb[d]; ++i) { /* v at level d - 1 */
        const int32_t v = order[i];
        if (v != s) bc[v] = bc[v] + delta[v];
      }
    }
    for (int32_t i = 0; i < tail; ++i) {
      const int32_t v = order[i];
      level[v] = ORACLE_MAX_LEVEL;
      sigma[v] = 0;
      delta[v] = 0.0f;
    }
  }
  free(level), free(sigma), free(delta), free(order), free(lb);
  return 0;
}

/* Colors of the graph-color application's iterations (see the header); returns
 * the iteration count, the largest color. */
int32_t oracle_color(int32_t n, const int32_t* row, const int32_t* col, int32_t* color) {
  int32_t most = 0;
  for (int32_t v = 0; v < n; ++v) {
    int32_t c = 0;
    for (int32_t e = row[v]; e < row[v + 1]; ++e) {
      const int32_t u = col[e];
      if (u < v && color[u] > c) c = color[u];
    }
    color[v] = c + 1;
    if (c + 1 > most) most = c + 1;
  }
  return most;
}

/* The same by simulating the reference's iterations literally: every iteration
 * tests every uncolored vertex against the colors at that moment (vertices in id
 * order, so a vertex colored earlier in the iteration is seen with color c, as a
 * racing GPU thread may see it).  Returns the iteration count. */
int32_t oracle_color_iterations(int32_t n, const int32_t* row, const int32_t* col, int32_t* color) {
  for (int32_t v = 0; v < n; ++v) color[v] = 0;
  int32_t c = 0, left = n;
  while (left > 0) {
    ++c;
    for (int32_t v = 0; v < n; ++v) {
      if (color[v] != 0) continue;
      int ok = 1;
      for (int32_t e = row[v]; e < row[v + 1] && ok; ++e) {
        const int32_t u = col[e];
        if ((color[u] == 0 || color[u] == c) && u < v) ok = 0;
      }
      if (ok) {
        color[v] = c;
        --left;
      }
    }
  }
  return c;
}

/* ------------------------------------------------------------------------
 * oracle_gen_rmat: the seeded R-MAT input of the benchmark, restated in C so
 * that the reference's CPU path can be run on the very same graph without
 * loading the library under test.  It follows nps_gen_rmat and nps_build_csr
 * (nested-parallelism_b200/csrc/nps_graph.cpp): edge e draws from the counter
 * stream key = splitmix64(splitmix64(seed ^ salt) ^ e * 0xD6E8FEB86659FD93),
 * draw k = splitmix64(key + k * 0x9E3779B97F4A7C15); `scale` quadrant draws
 * (53-bit uniforms, most significant level first), then the weight
 * 1 + ((draw >> 32) * wmax >> 32).  Self-loops are dropped, duplicate
 * (src, dst) pairs keep their earliest edge, rows hold their edges in reverse
 * edge order (the reference's convertCSR convention), and the source is the
 * highest out-degree vertex (lowest id on ties).  The edge draws run on the
 * host's threads; the CSR is built in one O(m) pass: rows are filled in
 * ascending edge order and a per-destination stamp drops repeats.
 * Caller passes row[n+1], col[m], w[m] with m = edge_factor << scale; returns the
 * kept edge count (or -1 on a bad argument) and the source in *src_out.
 */
static uint64_t sm64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

int64_t oracle_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, uint32_t wmax,
                        uint64_t seed, int32_t* row, int32_t* col, uint32_t* w, int32_t* src_out) {
  if (scale < 1 || scale > 30 || edge_factor < 1 || wmax == 0) return -1;
  const int64_t n = (int64_t)1 << scale, m = n * edge_factor;
  const double ab = a + b, abc = a + b + c;
  const uint64_t salt = 0x726D617431323334ull;
  int32_t* es = (int32_t*)malloc(sizeof(int32_t) * (size_t)m);
  int32_t* ed = (int32_t*)malloc(sizeof(int32_t) * (size_t)m);
  uint32_t* ew = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)m);
  int64_t* start = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
  int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
  int64_t* ids = (int64_t*)malloc(sizeof(int64_t) * (size_t)m);
  int32_t* stamp = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  if (!es || !ed || !ew || !start || !fill || !ids || !stamp) {
    free(es); free(ed); free(ew); free(start); free(fill); free(ids); free(stamp);
    return -1;
  }
  const uint64_t base = sm64(seed ^ salt);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < m; ++e) {
    const uint64_t key = sm64(base ^ ((uint64_t)e * 0xD6E8FEB86659FD93ull));
    uint64_t k = 0;
    uint32_t u = 0, v = 0;
    for (int l = scale - 1; l >= 0; --l) {
      const double x = (double)(sm64(key + (k++) * 0x9E3779B97F4A7C15ull) >> 11) * (1.0 / 9007199254740992.0);
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
    es[e] = (int32_t)u;
    ed[e] = (int32_t)v;
    ew[e] = 1u + (uint32_t)(((sm64(key + (k++) * 0x9E3779B97F4A7C15ull) >> 32) * (uint64_t)wmax) >> 32);
  }
  /* bucket edge ids by source, ascending id within a row */
  for (int64_t e = 0; e < m; ++e)
    if (es[e] != ed[e]) start[es[e] + 1]++;
  for (int64_t v = 0; v < n; ++v) start[v + 1] += start[v];
  for (int64_t v = 0; v < n; ++v) fill[v] = start[v];
  for (int64_t e = 0; e < m; ++e)
    if (es[e] != ed[e]) ids[fill[es[e]]++] = e;
  /* per row: keep the first edge to each destination, then write the row reversed */
  for (int64_t v = 0; v < n; ++v) stamp[v] = -1;
  int64_t o = 0;
  int32_t best = 0, bestd = -1;
  for (int64_t v = 0; v < n; ++v) {
    row[v] = (int32_t)o;
    int64_t k = 0;
    for (int64_t i = start[v]; i < start[v + 1]; ++i) {
      const int32_t d = ed[ids[i]];
      if (stamp[d] == (int32_t)v) continue;
      stamp[d] = (int32_t)v;
      ids[start[v] + k++] = ids[i];
    }
    for (int64_t i = 0; i < k; ++i) {
      const int64_t e = ids[start[v] + k - 1 - i];
      col[o + i] = ed[e];
      w[o + i] = ew[e];
    }
    if ((int32_t)k > bestd) {
      bestd = (int32_t)k;
      best = (int32_t)v;
    }
    o += k;
  }
  row[n] = (int32_t)o;
  *src_out = best;
  free(es); free(ed); free(ew); free(start); free(fill); free(ids); free(stamp);
  return o;
}
