/*
 * maxflow_oracle.c — CPU oracle for the grid graph-cut path.  TEST
 * INFRASTRUCTURE ONLY: the tests, the smoke check and the CPU-baseline leg of
 * the benchmark call it as a checker or as the timed CPU reference; the
 * product (libcgc) never links or calls it.
 *
 * What it restates.  The reference's CPU max-flow path is
 * benchmarks/graph_cut/boykov_kolmogorov.cpp:20-83: a Boykov-Kolmogorov
 * solver (external "BK301" = maxflow v3.01, found at ../../BK301 by
 * benchmarks/graph_cut/CMakeLists.txt:10-14, not vendored and absent here) is
 * fed add_tweights(v, capS, capT) (:54) and add_edge(i, j, cap_ij, cap_ji)
 * (:60-64) for every 6-neighbour pair, maxflow() is timed alone (:70-73) and
 * what_segment(v)==SINK becomes the mask (:78-82).  BK301's source is not
 * used: orc_bk_* below is written from the published algorithm (Y. Boykov,
 * V. Kolmogorov, "An Experimental Comparison of Min-Cut/Max-Flow Algorithms
 * for Energy Minimization in Vision", IEEE TPAMI 26(9), 2004: two search
 * trees, growth / augmentation / adoption stages, with the distance and
 * timestamp heuristic of its section 3.3).  An independently written Dinic
 * solver (E. A. Dinic 1970; blocking flows on BFS level graphs) is the second
 * algorithm: both must agree bit for bit on the flow value and on both cut
 * sets before any GPU result is compared with them.
 *
 * Semantics shared with the reference's Graph API:
 *   - t-links: capS (source) and capT (sink) per vertex
 *     (include/cugip/advanced_operations/graph_cut.hpp:64-67);
 *   - n-links: EdgeRecord(a,b) with cap a->b and cap b->a
 *     (graph_cut.hpp:57-62, detail/edge_record.hpp:12-17);
 *   - the flow value is exact (int64 sum of int32 capacities);
 *   - treach = vertices that can reach the sink in the final residual graph
 *     (the set cugip::Graph::fill_segments marks, graph_cut.hpp:304-333, and
 *     BK's what_segment()==SINK, boykov_kolmogorov.cpp:81);
 *   - smin = vertices reachable from the source in the final residual graph.
 *
 * Parity pins: the known answers of the reference's own tests (4x4 grid of
 * test/graph_cut.cu:9-63 -> 4; layered graphs of
 * unit_tests/graph_cut_test.cu:22-67,172-198 -> 8192 and 16384) are checked
 * in tests/test_oracle.py.
 */
#define _POSIX_C_SOURCE 199309L
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* -------------------------------------------------------------------------- */
/* residual graph in CSR form with sister arcs; terminal residual tr[v]:
   tr > 0: residual s->v, tr < 0: residual v->t (after cancelling min(capS,capT)) */
typedef struct {
  int32_t n;
  int64_t narcs;
  int64_t* first;  /* n+1 */
  int32_t* head;   /* narcs */
  int64_t* sister; /* narcs */
  int32_t* rcap;   /* narcs */
  int64_t* tr;     /* n */
  int64_t flow;
} og_graph;

static void og_free(og_graph* g) {
  free(g->first); free(g->head); free(g->sister); free(g->rcap); free(g->tr);
  memset(g, 0, sizeof(*g));
}

static int og_alloc(og_graph* g, int32_t n, int64_t narcs) {
  memset(g, 0, sizeof(*g));
  g->n = n; g->narcs = narcs;
  g->first = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
  g->head = (int32_t*)malloc((size_t)(narcs ? narcs : 1) * sizeof(int32_t));
  g->sister = (int64_t*)malloc((size_t)(narcs ? narcs : 1) * sizeof(int64_t));
  g->rcap = (int32_t*)malloc((size_t)(narcs ? narcs : 1) * sizeof(int32_t));
  g->tr = (int64_t*)calloc((size_t)(n ? n : 1), sizeof(int64_t));
  if (!g->first || !g->head || !g->sister || !g->rcap || !g->tr) { og_free(g); return -1; }
  return 0;
}

static void og_set_tlinks(og_graph* g, const int32_t* capS, const int32_t* capT) {
  int64_t f = 0;
  for (int32_t v = 0; v < g->n; ++v) {
    int64_t s = capS[v], t = capT[v];
    int64_t m = s < t ? s : t;
    f += m;
    g->tr[v] = s - t;
  }
  g->flow = f;
}

/* generic edge list: edge i joins a[i] and b[i]; cab = cap a->b, cba = cap b->a */
static int og_from_edges(og_graph* g, int32_t n, int64_t m, const int32_t* a, const int32_t* b,
                         const int32_t* cab, const int32_t* cba, const int32_t* capS, const int32_t* capT) {
  if (og_alloc(g, n, 2 * m)) return -1;
  for (int64_t i = 0; i < m; ++i) { g->first[a[i] + 1]++; g->first[b[i] + 1]++; }
  for (int32_t v = 0; v < n; ++v) g->first[v + 1] += g->first[v];
  int64_t* fill = (int64_t*)malloc((size_t)(n ? n : 1) * sizeof(int64_t));
  if (!fill) { og_free(g); return -1; }
  for (int32_t v = 0; v < n; ++v) fill[v] = g->first[v];
  for (int64_t i = 0; i < m; ++i) {
    int64_t p = fill[a[i]]++, q = fill[b[i]]++;
    g->head[p] = b[i]; g->rcap[p] = cab[i]; g->sister[p] = q;
    g->head[q] = a[i]; g->rcap[q] = cba[i]; g->sister[q] = p;
  }
  free(fill);
  og_set_tlinks(g, capS, capT);
  return 0;
}

/* 6-connected grid; arcs of a vertex in the order +x,-x,+y,-y,+z,-z (existing only).
   f*[v] = cap v -> v+e, b*[v] = cap v+e -> v. */
static int og_from_grid(og_graph* g, int32_t X, int32_t Y, int32_t Z, const int32_t* capS, const int32_t* capT,
                        const int32_t* const fw[3], const int32_t* const bw[3]) {
  int64_t N = (int64_t)X * Y * Z;
  int64_t narcs = 2 * ((int64_t)(X - 1) * Y * Z + (int64_t)X * (Y - 1) * Z + (int64_t)X * Y * (Z - 1));
  if (og_alloc(g, (int32_t)N, narcs)) return -1;
  const int64_t stride[3] = {1, X, (int64_t)X * Y};
  int64_t p = 0;
  for (int32_t z = 0; z < Z; ++z)
    for (int32_t y = 0; y < Y; ++y)
      for (int32_t x = 0; x < X; ++x) {
        int64_t v = x + (int64_t)X * (y + (int64_t)Y * z);
        g->first[v] = p;
        int32_t c[3] = {x, y, z}, e[3] = {X, Y, Z};
        for (int ax = 0; ax < 3; ++ax) {
          if (c[ax] + 1 < e[ax]) { g->head[p] = (int32_t)(v + stride[ax]); g->rcap[p] = fw[ax][v]; ++p; }
          if (c[ax] > 0) { g->head[p] = (int32_t)(v - stride[ax]); g->rcap[p] = bw[ax][v - stride[ax]]; ++p; }
        }
      }
  g->first[N] = p;
  /* sisters: arcs of u are sorted by direction, so find the arc of u pointing back to v */
  for (int64_t v = 0; v < N; ++v)
    for (int64_t a = g->first[v]; a < g->first[v + 1]; ++a) {
      int32_t u = g->head[a];
      int64_t q = g->first[u];
      while (g->head[q] != v) ++q;
      g->sister[a] = q;
    }
  og_set_tlinks(g, capS, capT);
  return 0;
}

/* -------------------------------------------------------------------------- */
/* Boykov-Kolmogorov (TPAMI 2004).  tree: 0 free, 1 source tree S, 2 sink tree T.
   parent[v] = arc from v to its parent, or P_TERMINAL / P_ORPHAN / P_NONE. */
#define P_NONE (-3)
#define P_ORPHAN (-2)
#define P_TERMINAL (-1)

typedef struct { int32_t* buf; int64_t cap, head, size; } ring_t;
static int ring_init(ring_t* r, int64_t cap) { r->buf = (int32_t*)malloc((size_t)(cap ? cap : 1) * 4); r->cap = cap ? cap : 1; r->head = r->size = 0; return r->buf ? 0 : -1; }
static void ring_push(ring_t* r, int32_t v) { r->buf[(r->head + r->size) % r->cap] = v; r->size++; }
static int32_t ring_pop(ring_t* r) { int32_t v = r->buf[r->head]; r->head = (r->head + 1) % r->cap; r->size--; return v; }

static int bk_run(og_graph* g) {
  const int32_t n = g->n;
  int64_t* parent = (int64_t*)malloc((size_t)(n ? n : 1) * 8);
  uint8_t* tree = (uint8_t*)calloc((size_t)(n ? n : 1), 1);
  uint8_t* inq = (uint8_t*)calloc((size_t)(n ? n : 1), 1);
  int32_t* ts = (int32_t*)calloc((size_t)(n ? n : 1), 4);
  int32_t* dist = (int32_t*)calloc((size_t)(n ? n : 1), 4);
  ring_t active, orphans;
  int ok = parent && tree && inq && ts && dist && !ring_init(&active, n) && !ring_init(&orphans, n);
  if (!ok) { free(parent); free(tree); free(inq); free(ts); free(dist); return -1; }
  const int64_t* first = g->first; const int32_t* head = g->head; const int64_t* sister = g->sister;
  int32_t* rcap = g->rcap; int64_t* tr = g->tr;
  int32_t TIME = 0;

  for (int32_t v = 0; v < n; ++v) {
    if (tr[v] > 0) { tree[v] = 1; parent[v] = P_TERMINAL; dist[v] = 1; inq[v] = 1; ring_push(&active, v); }
    else if (tr[v] < 0) { tree[v] = 2; parent[v] = P_TERMINAL; dist[v] = 1; inq[v] = 1; ring_push(&active, v); }
    else { tree[v] = 0; parent[v] = P_NONE; }
  }
  int32_t cur = -1;
  for (;;) {
    /* pick the current active node */
    if (cur >= 0 && parent[cur] == P_NONE) cur = -1;
    if (cur < 0) {
      while (active.size) {
        int32_t v = ring_pop(&active); inq[v] = 0;
        if (parent[v] != P_NONE) { cur = v; break; }
      }
      if (cur < 0) break;
    }
    /* growth */
    int64_t mid = -1;
    if (tree[cur] == 1) {
      for (int64_t a = first[cur]; a < first[cur + 1]; ++a) {
        if (rcap[a] <= 0) continue;
        int32_t j = head[a];
        if (tree[j] == 0) {
          tree[j] = 1; parent[j] = sister[a]; ts[j] = ts[cur]; dist[j] = dist[cur] + 1;
          if (!inq[j]) { inq[j] = 1; ring_push(&active, j); }
        } else if (tree[j] == 2) { mid = a; break; }
        else if (ts[j] <= ts[cur] && dist[j] > dist[cur]) {
          parent[j] = sister[a]; ts[j] = ts[cur]; dist[j] = dist[cur] + 1;
        }
      }
    } else {
      for (int64_t a = first[cur]; a < first[cur + 1]; ++a) {
        int64_t sa = sister[a];
        if (rcap[sa] <= 0) continue;
        int32_t j = head[a];
        if (tree[j] == 0) {
          tree[j] = 2; parent[j] = sa; ts[j] = ts[cur]; dist[j] = dist[cur] + 1;
          if (!inq[j]) { inq[j] = 1; ring_push(&active, j); }
        } else if (tree[j] == 1) { mid = sa; break; }
        else if (ts[j] <= ts[cur] && dist[j] > dist[cur]) {
          parent[j] = sa; ts[j] = ts[cur]; dist[j] = dist[cur] + 1;
        }
      }
    }
    ++TIME;
    if (mid < 0) { cur = -1; continue; }

    /* augmentation along s -> ... -> p -mid-> q -> ... -> t */
    int32_t p = head[sister[mid]], q = head[mid];
    int64_t delta = rcap[mid];
    for (int32_t i = p; ; ) {
      int64_t b = parent[i];
      if (b == P_TERMINAL) { if (tr[i] < delta) delta = tr[i]; break; }
      if (rcap[sister[b]] < delta) delta = rcap[sister[b]];
      i = head[b];
    }
    for (int32_t i = q; ; ) {
      int64_t b = parent[i];
      if (b == P_TERMINAL) { if (-tr[i] < delta) delta = -tr[i]; break; }
      if (rcap[b] < delta) delta = rcap[b];
      i = head[b];
    }
    rcap[mid] -= (int32_t)delta; rcap[sister[mid]] += (int32_t)delta;
    for (int32_t i = p; ; ) {
      int64_t b = parent[i];
      if (b == P_TERMINAL) {
        tr[i] -= delta;
        if (tr[i] == 0) { parent[i] = P_ORPHAN; ring_push(&orphans, i); }
        break;
      }
      int32_t up = head[b];
      rcap[sister[b]] -= (int32_t)delta; rcap[b] += (int32_t)delta;
      if (rcap[sister[b]] == 0) { parent[i] = P_ORPHAN; ring_push(&orphans, i); }
      i = up;
    }
    for (int32_t i = q; ; ) {
      int64_t b = parent[i];
      if (b == P_TERMINAL) {
        tr[i] += delta;
        if (tr[i] == 0) { parent[i] = P_ORPHAN; ring_push(&orphans, i); }
        break;
      }
      int32_t up = head[b];
      rcap[b] -= (int32_t)delta; rcap[sister[b]] += (int32_t)delta;
      if (rcap[b] == 0) { parent[i] = P_ORPHAN; ring_push(&orphans, i); }
      i = up;
    }
    g->flow += delta;

    /* adoption */
    ++TIME;
    while (orphans.size) {
      int32_t i = ring_pop(&orphans);
      const int in_s = (tree[i] == 1);
      int64_t best = -1; int32_t best_d = 0x7fffffff;
      for (int64_t a = first[i]; a < first[i + 1]; ++a) {
        int32_t j = head[a];
        if (tree[j] != tree[i]) continue;
        if (in_s ? (rcap[sister[a]] <= 0) : (rcap[a] <= 0)) continue;
        /* origin of j: walk to the terminal, using marks set in this TIME */
        int32_t d = 0, k = j, valid = 1;
        for (;;) {
          if (ts[k] == TIME) { d += dist[k]; break; }
          int64_t b = parent[k];
          ++d;
          if (b == P_TERMINAL) { ts[k] = TIME; dist[k] = 1; break; }
          if (b < 0) { valid = 0; break; } /* orphan or free */
          k = head[b];
        }
        if (!valid) continue;
        if (d < best_d) { best_d = d; best = a; }
        for (k = j; ts[k] != TIME; k = head[parent[k]]) { ts[k] = TIME; dist[k] = d--; }
      }
      if (best >= 0) {
        parent[i] = best; ts[i] = TIME; dist[i] = best_d + 1;
        continue;
      }
      /* no parent: i becomes free */
      for (int64_t a = first[i]; a < first[i + 1]; ++a) {
        int32_t j = head[a];
        if (tree[j] != tree[i]) continue;
        if (in_s ? (rcap[sister[a]] > 0) : (rcap[a] > 0)) {
          if (!inq[j]) { inq[j] = 1; ring_push(&active, j); }
        }
        int64_t b = parent[j];
        if (b >= 0 && head[b] == i) { parent[j] = P_ORPHAN; ring_push(&orphans, j); }
      }
      tree[i] = 0; parent[i] = P_NONE;
    }
  }
  free(parent); free(tree); free(inq); free(ts); free(dist); free(active.buf); free(orphans.buf);
  return 0;
}

/* -------------------------------------------------------------------------- */
/* Dinic with the source and sink implicit in tr[] */
static int dinic_run(og_graph* g) {
  const int32_t n = g->n;
  int32_t* level = (int32_t*)malloc((size_t)(n ? n : 1) * 4);
  int64_t* it = (int64_t*)malloc((size_t)(n ? n : 1) * 8);
  int32_t* queue = (int32_t*)malloc((size_t)(n ? n : 1) * 4);
  int64_t* stack = (int64_t*)malloc((size_t)(n ? n : 1) * 8);
  if (!level || !it || !queue || !stack) { free(level); free(it); free(queue); free(stack); return -1; }
  const int64_t* first = g->first; const int32_t* head = g->head; const int64_t* sister = g->sister;
  int32_t* rcap = g->rcap; int64_t* tr = g->tr;
  for (;;) {
    /* BFS level graph from s (level 0) */
    int64_t qh = 0, qt = 0;
    for (int32_t v = 0; v < n; ++v) { level[v] = -1; if (tr[v] > 0) { level[v] = 1; queue[qt++] = v; } }
    int32_t lt = -1; /* level of t */
    while (qh < qt) {
      int32_t v = queue[qh++];
      if (lt >= 0 && level[v] + 1 >= lt) continue;
      if (tr[v] < 0) { if (lt < 0) lt = level[v] + 1; continue; }
      for (int64_t a = first[v]; a < first[v + 1]; ++a) {
        int32_t w = head[a];
        if (rcap[a] > 0 && level[w] < 0) { level[w] = level[v] + 1; queue[qt++] = w; }
      }
    }
    if (lt < 0) break;
    for (int32_t v = 0; v < n; ++v) { it[v] = first[v]; if (level[v] >= lt) level[v] = -1; }
    for (int64_t qi = 0; qi < qt; ++qi) {
      int32_t v0 = queue[qi];
      if (level[v0] != 1) continue;
      while (tr[v0] > 0 && level[v0] == 1) {
        int64_t sp = 0; int32_t u = v0; int found = 0;
        for (;;) {
          if (tr[u] < 0 && level[u] + 1 == lt) { found = 1; break; }
          int adv = 0;
          if (level[u] + 1 < lt) {
            while (it[u] < first[u + 1]) {
              int64_t a = it[u]; int32_t w = head[a];
              if (rcap[a] > 0 && level[w] == level[u] + 1) { stack[sp++] = a; u = w; adv = 1; break; }
              it[u]++;
            }
          }
          if (adv) continue;
          level[u] = -1;
          if (sp == 0) break;
          int64_t a = stack[--sp]; u = head[sister[a]]; it[u]++;
        }
        if (!found) break;
        int64_t d = tr[v0];
        if (-tr[u] < d) d = -tr[u];
        for (int64_t k = 0; k < sp; ++k) if (rcap[stack[k]] < d) d = rcap[stack[k]];
        tr[v0] -= d; tr[u] += d;
        for (int64_t k = 0; k < sp; ++k) { rcap[stack[k]] -= (int32_t)d; rcap[sister[stack[k]]] += (int32_t)d; }
        g->flow += d;
      }
    }
  }
  free(level); free(it); free(queue); free(stack);
  return 0;
}

/* -------------------------------------------------------------------------- */
/* cut sets from the final residual graph */
static int og_cuts(const og_graph* g, uint8_t* smin, uint8_t* treach) {
  const int32_t n = g->n;
  int32_t* queue = (int32_t*)malloc((size_t)(n ? n : 1) * 4);
  if (!queue) return -1;
  if (smin) {
    int64_t qh = 0, qt = 0;
    for (int32_t v = 0; v < n; ++v) { smin[v] = g->tr[v] > 0; if (smin[v]) queue[qt++] = v; }
    while (qh < qt) {
      int32_t v = queue[qh++];
      for (int64_t a = g->first[v]; a < g->first[v + 1]; ++a) {
        int32_t w = g->head[a];
        if (g->rcap[a] > 0 && !smin[w]) { smin[w] = 1; queue[qt++] = w; }
      }
    }
  }
  if (treach) {
    int64_t qh = 0, qt = 0;
    for (int32_t v = 0; v < n; ++v) { treach[v] = g->tr[v] < 0; if (treach[v]) queue[qt++] = v; }
    while (qh < qt) {
      int32_t v = queue[qh++];
      for (int64_t a = g->first[v]; a < g->first[v + 1]; ++a) {
        int32_t w = g->head[a];
        if (g->rcap[g->sister[a]] > 0 && !treach[w]) { treach[w] = 1; queue[qt++] = w; }
      }
    }
  }
  free(queue);
  return 0;
}

static double now_s(void) {
  struct timespec t; clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

static int solve(og_graph* g, int algo, int64_t* flow, uint8_t* smin, uint8_t* treach, double* seconds) {
  double t0 = now_s();
  int rc = (algo == 0) ? bk_run(g) : dinic_run(g);
  double t1 = now_s();
  if (rc) return -1;
  if (seconds) *seconds = t1 - t0;
  if (flow) *flow = g->flow;
  return og_cuts(g, smin, treach);
}

/* algo: 0 = Boykov-Kolmogorov, 1 = Dinic.  Returns 0 on success. */
int orc_maxflow_grid(int algo, int32_t X, int32_t Y, int32_t Z, const int32_t* capS, const int32_t* capT,
                     const int32_t* fx, const int32_t* bx, const int32_t* fy, const int32_t* by,
                     const int32_t* fz, const int32_t* bz, int64_t* flow, uint8_t* smin, uint8_t* treach,
                     double* seconds) {
  og_graph g;
  const int32_t* fw[3] = {fx, fy, fz};
  const int32_t* bw[3] = {bx, by, bz};
  if (X <= 0 || Y <= 0 || Z <= 0) return -2;
  if (og_from_grid(&g, X, Y, Z, capS, capT, fw, bw)) return -1;
  int rc = solve(&g, algo, flow, smin, treach, seconds);
  og_free(&g);
  return rc;
}

int orc_maxflow_edges(int algo, int32_t n, int64_t m, const int32_t* a, const int32_t* b, const int32_t* cab,
                      const int32_t* cba, const int32_t* capS, const int32_t* capT, int64_t* flow, uint8_t* smin,
                      uint8_t* treach, double* seconds) {
  og_graph g;
  if (n < 0 || m < 0) return -2;
  for (int64_t i = 0; i < m; ++i)
    if (a[i] < 0 || a[i] >= n || b[i] < 0 || b[i] >= n) return -2;
  if (og_from_edges(&g, n, m, a, b, cab, cba, capS, capT)) return -1;
  int rc = solve(&g, algo, flow, smin, treach, seconds);
  og_free(&g);
  return rc;
}
