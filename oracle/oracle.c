/*
 * oracle.c -- CPU restatement of the reference's BC hot path (see oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product, never part of it.
 * Each routine cites the reference file:line it restates.  Plain C99 + OpenMP.
 */
#include "oracle.h"

#include <limits.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_INF 999999999 /* TreeDecomp INF / MAXDIS_ (src/TreeCount/Util.h:35, TreeDecomp.h:58) */
#define H2H_INF 0x3f3f3f3f /* include/std.h:15 */

static void *xmalloc(size_t n) {
  void *p = malloc(n ? n : 1);
  if (!p) abort();
  return p;
}
static void *xcalloc(size_t n, size_t s) {
  void *p = calloc(n ? n : 1, s ? s : 1);
  if (!p) abort();
  return p;
}

/* ======================================================================================
 * Graph::ReadGraph (src/Graph.cpp:4-37): ids -1, weight 0 -> 1, a repeated (ID1,ID2) arc is
 * dropped (first kept); arcs of each tail keep file order (Neighbor[ID1].push_back).
 * ====================================================================================== */
int orc_arcs_build(int n, int m_lines, const int *u1, const int *v1, const int *w, orc_arcs **out) {
  if (n <= 0 || m_lines < 0) return -1;
  int *deg = (int *)xcalloc((size_t)n + 1, sizeof(int));
  for (int i = 0; i < m_lines; i++) {
    int a = u1[i] - 1, b = v1[i] - 1;
    if (a < 0 || a >= n || b < 0 || b >= n) { free(deg); return -2; }
    deg[a + 1]++;
  }
  for (int i = 0; i < n; i++) deg[i + 1] += deg[i];
  int *tmp_h = (int *)xmalloc(sizeof(int) * (size_t)m_lines);
  int *tmp_w = (int *)xmalloc(sizeof(int) * (size_t)m_lines);
  int *fill = (int *)xmalloc(sizeof(int) * (size_t)n);
  memcpy(fill, deg, sizeof(int) * (size_t)n);
  for (int i = 0; i < m_lines; i++) {
    int a = u1[i] - 1;
    int ww = w[i] == 0 ? 1 : w[i];
    tmp_h[fill[a]] = v1[i] - 1;
    tmp_w[fill[a]] = ww;
    fill[a]++;
  }
  /* dedupe within each tail, keeping the first occurrence */
  int *stamp = (int *)xmalloc(sizeof(int) * (size_t)n);
  for (int i = 0; i < n; i++) stamp[i] = -1;
  orc_arcs *g = (orc_arcs *)xcalloc(1, sizeof(orc_arcs));
  g->n = n;
  g->off = (int *)xmalloc(sizeof(int) * ((size_t)n + 1));
  g->head = (int *)xmalloc(sizeof(int) * (size_t)m_lines);
  g->w = (int *)xmalloc(sizeof(int) * (size_t)m_lines);
  int m = 0;
  for (int a = 0; a < n; a++) {
    g->off[a] = m;
    for (int e = deg[a]; e < deg[a + 1]; e++) {
      int b = tmp_h[e];
      if (stamp[b] == a) continue;
      stamp[b] = a;
      g->head[m] = b;
      g->w[m] = tmp_w[e];
      m++;
    }
  }
  g->off[n] = m;
  g->m = m;
  free(deg); free(tmp_h); free(tmp_w); free(fill); free(stamp);
  *out = g;
  return 0;
}

void orc_arcs_free(orc_arcs *g) {
  if (!g) return;
  free(g->off); free(g->head); free(g->w); free(g);
}

/* ======================================================================================
 * Ordered adjacency (std::map<int,...> per vertex in the reference): sorted dynamic arrays.
 * ====================================================================================== */
typedef struct { int v, w; uint32_t c, h; } adj_e;
typedef struct { adj_e *e; int n, cap; } adj_t;

static int adj_find(const adj_t *a, int v) {
  int lo = 0, hi = a->n - 1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    if (a->e[mid].v == v) return mid;
    if (a->e[mid].v < v) lo = mid + 1; else hi = mid - 1;
  }
  return -(lo + 1);
}
static void adj_insert_at(adj_t *a, int at, adj_e x) {
  if (a->n == a->cap) {
    a->cap = a->cap ? a->cap * 2 : 4;
    a->e = (adj_e *)realloc(a->e, sizeof(adj_e) * (size_t)a->cap);
    if (!a->e) abort();
  }
  memmove(a->e + at + 1, a->e + at, sizeof(adj_e) * (size_t)(a->n - at));
  a->e[at] = x;
  a->n++;
}
static void adj_erase(adj_t *a, int v) {
  int i = adj_find(a, v);
  if (i < 0) return;
  memmove(a->e + i, a->e + i + 1, sizeof(adj_e) * (size_t)(a->n - i - 1));
  a->n--;
}

/* min-heap standing in for std::set<SelectElement> (TreeDecomp.cpp:65-78): key (DD, DD2, x) */
typedef struct { int dd, dd2, x; } sel_t;
typedef struct { sel_t *a; int n; } heap_t;
static int sel_less(sel_t p, sel_t q) {
  if (p.dd != q.dd) return p.dd < q.dd;
  if (p.dd2 != q.dd2) return p.dd2 < q.dd2;
  return p.x < q.x;
}
static void heap_push(heap_t *h, sel_t s) {
  int i = h->n++;
  h->a[i] = s;
  while (i > 0) {
    int p = (i - 1) >> 1;
    if (!sel_less(h->a[i], h->a[p])) break;
    sel_t t = h->a[i]; h->a[i] = h->a[p]; h->a[p] = t;
    i = p;
  }
}
static void heap_pop(heap_t *h) {
  h->a[0] = h->a[--h->n];
  int i = 0;
  for (;;) {
    int l = 2 * i + 1, r = l + 1, s = i;
    if (l < h->n && sel_less(h->a[l], h->a[s])) s = l;
    if (r < h->n && sel_less(h->a[r], h->a[s])) s = r;
    if (s == i) break;
    sel_t t = h->a[i]; h->a[i] = h->a[s]; h->a[s] = t;
    i = s;
  }
}

/* ======================================================================================
 * TreeDecomp: ReadWeightedGraph + ctor + Reduce + MakeTree + MakeRMQIndex + MakeCountIndex
 * ====================================================================================== */
int orc_tc_build(int n, int m_lines, const int *u1, const int *v1, const int *w, orc_tc **out) {
  if (n <= 0) return -1;
  /* Graph_::ReadWeightedGraph (src/TreeCount/Graph.cpp:55-71): symmetric, keep minimum weight */
  adj_t *E = (adj_t *)xcalloc((size_t)n + 1, sizeof(adj_t));
  for (int i = 0; i < m_lines; i++) {
    int a = u1[i], b = v1[i], ww = w[i];
    if (a < 1 || a > n || b < 1 || b > n) { for (int k = 0; k <= n; k++) free(E[k].e); free(E); return -2; }
    int ia = adj_find(&E[a], b);
    if (ia >= 0) {
      if (E[a].e[ia].w > ww) {
        E[a].e[ia].w = ww;
        int ib = adj_find(&E[b], a);
        E[b].e[ib].w = ww;
      }
    } else {
      adj_e x = {b, ww, 1u, 1u};
      adj_insert_at(&E[a], -(ia + 1), x);
      int ib = adj_find(&E[b], a);
      if (ib < 0) { adj_e y = {a, ww, 1u, 1u}; adj_insert_at(&E[b], -(ib + 1), y); }
    }
  }
  /* TreeDecomp ctor (TreeDecomp.cpp:44-51): C_ = 1 and my_C_ = 1 for every edge (set above) */
  orc_tc *tc = (orc_tc *)xcalloc(1, sizeof(orc_tc));
  tc->n = n;
  int *D = (int *)xmalloc(sizeof(int) * ((size_t)n + 1));
  for (int i = 1; i <= n; i++) D[i] = E[i].n;

  /* ---- Reduce (TreeDecomp.cpp:54-208) ---- */
  int *DD = (int *)xmalloc(sizeof(int) * ((size_t)n + 1));
  int *tDD = (int *)xmalloc(sizeof(int) * ((size_t)n + 1));
  int *DD2 = (int *)xmalloc(sizeof(int) * ((size_t)n + 1));
  int *tDD2 = (int *)xmalloc(sizeof(int) * ((size_t)n + 1));
  char *changed = (char *)xcalloc((size_t)n + 1, 1);
  char *exist = (char *)xmalloc((size_t)n + 1);
  heap_t hp; hp.a = (sel_t *)xmalloc(sizeof(sel_t) * ((size_t)n + 1)); hp.n = 0;
  for (int i = 1; i <= n; i++) {
    DD[i] = tDD[i] = DD2[i] = tDD2[i] = D[i];
    exist[i] = 1;
    sel_t s = {DD[i], DD2[i], i};
    heap_push(&hp, s);
  }
  tc->del_order = (int *)xmalloc(sizeof(int) * (size_t)n);
  /* separator storage per vid, filled in elimination order */
  int64_t *vnb_off = (int64_t *)xcalloc((size_t)n + 2, sizeof(int64_t));
  int64_t cap = 4 * (int64_t)n + 16, used = 0;
  int *vnb = (int *)xmalloc(sizeof(int) * (size_t)cap);
  int *vlen = (int *)xmalloc(sizeof(int) * (size_t)cap);
  uint32_t *vcnt = (uint32_t *)xmalloc(sizeof(uint32_t) * (size_t)cap);
  uint32_t *vhop = (uint32_t *)xmalloc(sizeof(uint32_t) * (size_t)cap);
  int64_t *vstart = (int64_t *)xmalloc(sizeof(int64_t) * ((size_t)n + 1));
  int *vsize = (int *)xmalloc(sizeof(int) * ((size_t)n + 1));
  int ndel = 0;
  adj_e *tmp = (adj_e *)xmalloc(sizeof(adj_e) * ((size_t)n + 1));
  while (hp.n > 0) {
    int x = hp.a[0].x;
    while (changed[x]) { /* TreeDecomp.cpp:104-112 */
      heap_pop(&hp);
      DD[x] = tDD[x];
      DD2[x] = tDD2[x];
      sel_t s = {DD[x], DD2[x], x};
      heap_push(&hp, s);
      changed[x] = 0;
      x = hp.a[0].x;
    }
    tc->del_order[ndel++] = x;
    heap_pop(&hp);
    exist[x] = 0;
    int k = 0;
    for (int i = 0; i < E[x].n; i++)
      if (exist[E[x].e[i].v]) tmp[k++] = E[x].e[i];
    for (int i = 0; i < k; i++) { /* deleteEdge(x, y) TreeDecomp.cpp:151-155 */
      int y = tmp[i].v;
      adj_erase(&E[x], y); adj_erase(&E[y], x);
      D[x]--; D[y]--;
      tDD[y] = D[y];
      changed[y] = 1;
    }
    for (int pu = 0; pu < k; pu++) { /* TreeDecomp.cpp:157-193 */
      for (int pv = pu + 1; pv < k; pv++) {
        int u = tmp[pu].v, v = tmp[pv].v;
        int newlength = tmp[pu].w + tmp[pv].w;
        uint32_t nc = tmp[pu].c * tmp[pv].c;
        uint32_t nh = tmp[pu].h + tmp[pv].h;
        int iu = adj_find(&E[u], v);
        if (iu >= 0) {
          int iv = adj_find(&E[v], u);
          adj_e *eu = &E[u].e[iu], *ev = &E[v].e[iv];
          if (eu->w == newlength) {
            eu->c = ev->c = eu->c + nc;
            if (nh > eu->h) eu->h = ev->h = nh;
          }
          if (eu->w > newlength) {
            eu->w = ev->w = newlength;
            eu->c = ev->c = nc;
            eu->h = ev->h = nh;
          }
        } else {
          adj_e a1 = {v, newlength, nc, nh};
          adj_insert_at(&E[u], -(iu + 1), a1);
          int iv = adj_find(&E[v], u);
          adj_e a2 = {u, newlength, nc, nh};
          adj_insert_at(&E[v], -(iv + 1), a2);
          D[u]++; D[v]++;
          tDD[u] = D[u]; tDD[v] = D[v];
          tDD2[u]++; tDD2[v]++;
          changed[u] = changed[v] = 1;
        }
      }
    }
    if (k > tc->tree_width) tc->tree_width = k;
    if (used + k > cap) {
      while (used + k > cap) cap *= 2;
      vnb = (int *)realloc(vnb, sizeof(int) * (size_t)cap);
      vlen = (int *)realloc(vlen, sizeof(int) * (size_t)cap);
      vcnt = (uint32_t *)realloc(vcnt, sizeof(uint32_t) * (size_t)cap);
      vhop = (uint32_t *)realloc(vhop, sizeof(uint32_t) * (size_t)cap);
      if (!vnb || !vlen || !vcnt || !vhop) abort();
    }
    vstart[x] = used;
    vsize[x] = k;
    for (int i = 0; i < k; i++) {
      vnb[used + i] = tmp[i].v; vlen[used + i] = tmp[i].w;
      vcnt[used + i] = tmp[i].c; vhop[used + i] = tmp[i].h;
    }
    used += k;
  }
  free(tmp); free(hp.a); free(DD); free(tDD); free(DD2); free(tDD2); free(changed); free(exist); free(D);
  for (int i = 0; i <= n; i++) free(E[i].e);
  free(E);
  free(vnb_off);

  /* ---- MakeTree (TreeDecomp.cpp:210-238) + GetParentNode (:630-664) ---- */
  tc->rank = (int *)xmalloc(sizeof(int) * ((size_t)n + 1));
  tc->rank[0] = -1;
  tc->vertex = (int *)xmalloc(sizeof(int) * (size_t)n);
  tc->parent = (int *)xmalloc(sizeof(int) * (size_t)n);
  tc->height = (int *)xmalloc(sizeof(int) * (size_t)n);
  tc->nb_off = (int64_t *)xmalloc(sizeof(int64_t) * ((size_t)n + 1));
  tc->nb = (int *)xmalloc(sizeof(int) * (size_t)(used ? used : 1));
  tc->nb_len = (int *)xmalloc(sizeof(int) * (size_t)(used ? used : 1));
  tc->nb_cnt = (uint32_t *)xmalloc(sizeof(uint32_t) * (size_t)(used ? used : 1));
  tc->nb_hop = (uint32_t *)xmalloc(sizeof(uint32_t) * (size_t)(used ? used : 1));
  int *nchild = (int *)xcalloc((size_t)n + 1, sizeof(int));
  int64_t o = 0;
  tc->tree_height = 0;
  for (int len = n - 1, p = 0; len >= 0; --len, ++p) {
    int vid = tc->del_order[len];
    tc->vertex[p] = vid;
    tc->rank[vid] = p;
    tc->nb_off[p] = o;
    for (int i = 0; i < vsize[vid]; i++) {
      tc->nb[o + i] = vnb[vstart[vid] + i];
      tc->nb_len[o + i] = vlen[vstart[vid] + i];
      tc->nb_cnt[o + i] = vcnt[vstart[vid] + i];
      tc->nb_hop[o + i] = vhop[vstart[vid] + i];
    }
    o += vsize[vid];
    if (len == n - 1) {
      tc->parent[p] = -1;
      tc->height[p] = 1;
      tc->tree_height = 1;
    } else {
      if (vsize[vid] == 0) { /* disconnected: the reference reads neighbors[0] out of range */
        free(nchild); free(vnb); free(vlen); free(vcnt); free(vhop); free(vstart); free(vsize);
        tc->nb_off[p + 1] = o; tc->n = p; orc_tc_free(tc); return -3;
      }
      int best = vnb[vstart[vid]];
      for (int i = 0; i < vsize[vid]; i++) {
        int nbv = vnb[vstart[vid] + i];
        if (tc->rank[nbv] > tc->rank[best]) best = nbv;
      }
      int pp = tc->rank[best];
      tc->parent[p] = pp;
      nchild[pp]++;
      tc->height[p] = tc->height[pp] + 1;
      if (tc->height[p] > tc->tree_height) tc->tree_height = tc->height[p];
    }
  }
  tc->nb_off[n] = o;
  free(vnb); free(vlen); free(vcnt); free(vhop); free(vstart); free(vsize);
  tc->child_off = (int *)xmalloc(sizeof(int) * ((size_t)n + 1));
  tc->child_off[0] = 0;
  for (int p = 0; p < n; p++) tc->child_off[p + 1] = tc->child_off[p] + nchild[p];
  tc->child = (int *)xmalloc(sizeof(int) * (size_t)(n > 1 ? n - 1 : 1));
  memset(nchild, 0, sizeof(int) * ((size_t)n + 1));
  for (int p = 1; p < n; p++) { /* children appended in tree-position order (push_back at :229) */
    int pp = tc->parent[p];
    tc->child[tc->child_off[pp] + nchild[pp]++] = p;
  }
  free(nchild);

  /* ---- EulerTour + MakeRMQIndex (TreeDecomp.cpp:248-257, 324-345) ---- */
  int m = 2 * n - 1;
  int *euler = (int *)xmalloc(sizeof(int) * (size_t)m);
  tc->euler_pos = (int *)xmalloc(sizeof(int) * (size_t)n);
  {
    int *stk = (int *)xmalloc(sizeof(int) * (size_t)n), *it = (int *)xmalloc(sizeof(int) * (size_t)n);
    int sp = 0, el = 0;
    stk[sp] = 0; it[sp] = 0; sp++;
    tc->euler_pos[0] = el; euler[el++] = 0;
    while (sp > 0) {
      int p = stk[sp - 1];
      if (it[sp - 1] < tc->child_off[p + 1] - tc->child_off[p]) {
        int c = tc->child[tc->child_off[p] + it[sp - 1]++];
        tc->euler_pos[c] = el; euler[el++] = c;
        stk[sp] = c; it[sp] = 0; sp++;
      } else {
        sp--;
        if (sp > 0) euler[el++] = stk[sp - 1];
      }
    }
    free(stk); free(it);
    m = el;
  }
  tc->euler_len = m;
  int levels = 1;
  for (int i = 2; i < m; i *= 2) levels++;
  tc->rmq_levels = levels;
  tc->rmq = (int *)xcalloc((size_t)levels * (size_t)m, sizeof(int));
  memcpy(tc->rmq, euler, sizeof(int) * (size_t)m);
  for (int i = 2, k = 1; i < m; i *= 2, ++k) {
    int *prev = tc->rmq + (size_t)(k - 1) * m, *cur = tc->rmq + (size_t)k * m;
    for (int j = 0; j < m - i; ++j) {
      int x = prev[j], y = prev[j + i / 2];
      cur[j] = tc->height[x] < tc->height[y] ? x : y;
    }
  }
  free(euler);

  /* ---- MakeCountIndex / makeIndexDFS (TreeDecomp.cpp:355-511) ----
   * A node's label only reads its ancestors' labels and every ancestor has a smaller tree
   * position, so tree-position order replaces the recursive DFS.  The DFS ancestor list
   * `list` is the root-first chain; toList[vid] is the vertex's height-1. */
  tc->pos_off = (int64_t *)xmalloc(sizeof(int64_t) * ((size_t)n + 1));
  tc->lab_off = (int64_t *)xmalloc(sizeof(int64_t) * ((size_t)n + 1));
  int64_t po = 0, lo = 0;
  for (int p = 0; p < n; p++) {
    tc->pos_off[p] = po;
    tc->lab_off[p] = lo;
    po += (p == 0) ? 1 : (tc->nb_off[p + 1] - tc->nb_off[p]) + 1;
    lo += tc->height[p] - 1;
  }
  tc->pos_off[n] = po;
  tc->lab_off[n] = lo;
  tc->pos = (int *)xmalloc(sizeof(int) * (size_t)(po ? po : 1));
  tc->dis = (int *)xmalloc(sizeof(int) * (size_t)(lo ? lo : 1));
  tc->cnt = (uint32_t *)xmalloc(sizeof(uint32_t) * (size_t)(lo ? lo : 1));
  tc->hop = (uint32_t *)xmalloc(sizeof(uint32_t) * (size_t)(lo ? lo : 1));
  tc->pos[0] = 0; /* root: pos = {0}, empty labels (:490-494) */
  for (int p = 1; p < n; p++) {
    int64_t nb0 = tc->nb_off[p];
    int nX = (int)(tc->nb_off[p + 1] - nb0);
    int L = tc->height[p] - 1; /* list.size() */
    int *pos = tc->pos + tc->pos_off[p];
    int *dis = tc->dis + tc->lab_off[p];
    uint32_t *cnt = tc->cnt + tc->lab_off[p];
    uint32_t *hop = tc->hop + tc->lab_off[p];
    for (int i = 0; i < nX; i++) pos[i] = tc->height[tc->rank[tc->nb[nb0 + i]]] - 1;
    pos[nX] = L;
    for (int j = 0; j < L; j++) { dis[j] = ORC_INF; cnt[j] = 0; hop[j] = 0; }
    for (int i = 0; i < nX; i++) { /* direct edges (:379-386) */
      int j = pos[i];
      if (dis[j] > tc->nb_len[nb0 + i]) {
        dis[j] = tc->nb_len[nb0 + i];
        cnt[j] = tc->nb_cnt[nb0 + i];
        hop[j] = tc->nb_hop[nb0 + i];
      }
    }
    for (int i = 0; i < nX; ++i) { /* (:388-450) */
      int xk = tc->rank[tc->nb[nb0 + i]];
      int k = pos[i];
      for (int j = 0; j < L; j++) {
        if (k == j) continue;
        int dis_new;
        uint32_t route_new, hop_new;
        if (k < j) {
          dis_new = ORC_INF; route_new = 0; hop_new = 0;
        } else {
          /* DistanceQueryAncestorToPosterity(list[j], x) = tree_[x].dis[j] (:347-353) */
          int z = tc->dis[tc->lab_off[xk] + j];
          dis_new = tc->nb_len[nb0 + i] + z;
          route_new = tc->nb_cnt[nb0 + i] * tc->cnt[tc->lab_off[xk] + j];
          hop_new = tc->nb_hop[nb0 + i] + tc->hop[tc->lab_off[xk] + j];
        }
        if (dis[j] > dis_new) {
          dis[j] = dis_new; cnt[j] = route_new; hop[j] = hop_new;
        } else if (dis[j] == dis_new) {
          cnt[j] = cnt[j] + route_new;
          if (hop_new > hop[j]) hop[j] = hop_new;
        }
      }
    }
  }
  *out = tc;
  return 0;
}

void orc_tc_free(orc_tc *tc) {
  if (!tc) return;
  free(tc->del_order); free(tc->rank); free(tc->vertex); free(tc->parent); free(tc->height);
  free(tc->child_off); free(tc->child); free(tc->nb_off); free(tc->nb); free(tc->nb_len);
  free(tc->nb_cnt); free(tc->nb_hop); free(tc->pos_off); free(tc->pos); free(tc->lab_off);
  free(tc->dis); free(tc->cnt); free(tc->hop); free(tc->euler_pos); free(tc->rmq);
  free(tc);
}

/* LCA by Euler-tour RMQ with floor(log2) window (MHLQBC.cu:305-330). */
static inline int tc_lca(const orc_tc *tc, int p, int q) {
  if (p > q) { int t = p; p = q; q = t; }
  int len = q - p + 1;
  int k = 31 - __builtin_clz((unsigned)len);
  int i = 1 << k;
  q = q - i + 1;
  const int *lv = tc->rmq + (size_t)k * tc->euler_len;
  int a = lv[p], b = lv[q];
  return tc->height[a] < tc->height[b] ? a : b;
}

/* dist/count/hop row of one source (MHLQBC.cu:302-412); lca scratch has n ints. */
static void tc_rows(const orc_tc *tc, int source, int *lcaq, int *distance, uint32_t *count, int *layer,
                    int *max_layer) {
  const int n = tc->n;
  const int x1 = tc->rank[source + 1];
  const int p1 = tc->euler_pos[x1];
  for (int idx = 0; idx < n; idx++) lcaq[idx] = tc_lca(tc, p1, tc->euler_pos[idx]);
  int ml = 0;
  for (int idx = 0; idx < n; idx++) {
    int p = source + 1, q = idx + 1, x = x1;
    (void)p;
    if (p == q) {
      count[idx] = 1; distance[idx] = 0; layer[idx] = 0;
      continue;
    }
    int y = tc->rank[q];
    int lca = lcaq[y];
    int dis = ORC_INF;
    uint32_t ret = 0, cnt = 0;
    int my_ret = 0, my_cnt = 0;
    int ps = (int)(tc->pos_off[lca + 1] - tc->pos_off[lca]);
    int position = tc->pos[tc->pos_off[lca] + ps - 1];
    if (lca == x || lca == y) {
      if (lca == y) { int v = y; y = x; x = v; }
      int a = (int)(tc->pos_off[x + 1] - tc->pos_off[x]) - 1;
      int pp = tc->pos[tc->pos_off[x] + a];
      dis = tc->dis[tc->lab_off[y] + pp];
      ret = tc->cnt[tc->lab_off[y] + pp];
      my_ret = (int)tc->hop[tc->lab_off[y] + pp];
      position--;
    }
    int tmp_dis = ORC_INF;
    const int *dx = tc->dis + tc->lab_off[x], *dy = tc->dis + tc->lab_off[y];
    const uint32_t *cx = tc->cnt + tc->lab_off[x], *cy = tc->cnt + tc->lab_off[y];
    const uint32_t *hx = tc->hop + tc->lab_off[x], *hy = tc->hop + tc->lab_off[y];
    for (int i = 0; i <= position; i++) {
      int t = dx[i] + dy[i];
      if (tmp_dis > t) {
        tmp_dis = t;
        cnt = cx[i] * cy[i];
        my_cnt = (int)(hx[i] + hy[i]);
      } else if (tmp_dis == t) {
        cnt += cx[i] * cy[i];
        if ((int)(hx[i] + hy[i]) > my_cnt) my_cnt = (int)(hx[i] + hy[i]);
      }
    }
    if (dis > tmp_dis) {
      dis = tmp_dis; ret = cnt; my_ret = my_cnt;
    } else if (dis == tmp_dis) {
      ret += cnt;
      if (my_cnt > my_ret) my_ret = my_cnt;
    }
    if (my_ret > ml) ml = my_ret;
    layer[idx] = my_ret;
    count[idx] = ret;
    distance[idx] = dis;
  }
  *max_layer = ml;
}

int orc_mhl_rows(const orc_tc *tc, int source, int *dist, uint32_t *cnt, int *hop) {
  if (source < 0 || source >= tc->n) return -1;
  int *lcaq = (int *)xmalloc(sizeof(int) * (size_t)tc->n);
  int ml;
  tc_rows(tc, source, lcaq, dist, cnt, hop, &ml);
  free(lcaq);
  return 0;
}

/* Per-source SP-DAG, layer queue and backprop (MHLQBC.cu:415-472). */
typedef struct {
  int *lcaq, *dist, *layer, *layer_edge, *layer_size, *layer_start, *queue;
  uint32_t *cnt;
  double *delta;
} mhl_scratch;

static void mhl_one(const orc_tc *tc, const orc_arcs *g, int source, mhl_scratch *s, double *bc) {
  const int n = tc->n, m = g->m;
  int maxLayer;
  tc_rows(tc, source, s->lcaq, s->dist, s->cnt, s->layer, &maxLayer);
  for (int i = 0; i <= maxLayer + 1 && i < n + 2; i++) s->layer_size[i] = 0;
  /* 3. successors + edge layers (:416-431) */
  for (int t = 0; t < n; t++) {
    for (int e = g->off[t]; e < g->off[t + 1]; e++) {
      int h = g->head[e];
      if (s->dist[h] == s->dist[t] + g->w[e]) {
        if (t != source) {
          s->layer_edge[e] = s->layer[h];
          s->layer_size[s->layer[h]]++;
        } else {
          s->layer_edge[e] = 1;
        }
      } else {
        s->layer_edge[e] = 1;
      }
    }
  }
  /* 4. layer starts packed at the end of the queue (:435-440) */
  if (maxLayer >= 2) {
    s->layer_start[maxLayer] = m - s->layer_size[maxLayer];
    for (int i = maxLayer - 1; i >= 2; --i) s->layer_start[i] = s->layer_start[i + 1] - s->layer_size[i];
  }
  /* 5. scatter (:443-449): ascending arc order stands in for the atomic order */
  for (int e = 0; e < m; e++) {
    int L = s->layer_edge[e];
    if (L > 1) s->queue[s->layer_start[L]++] = e;
  }
  /* 6. backprop (:452-466) */
  int tmp_back = m - 1;
  for (int i = 0; i < n; i++) s->delta[i] = 0.0;
  for (int i = maxLayer; i > 1; --i) {
    for (int idx = 0; idx < s->layer_size[i]; idx++) {
      int e = s->queue[tmp_back - idx];
      /* tail of arc e: arcs are grouped by tail */
      int lo = 0, hi = n - 1;
      while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (g->off[mid] <= e) lo = mid; else hi = mid - 1; }
      int t = lo, h = g->head[e];
      double tmp2 = (double)(int)s->cnt[t] * (1 + s->delta[h]) / (double)(int)s->cnt[h];
      s->delta[t] += tmp2;
    }
    tmp_back -= s->layer_size[i];
  }
  /* 7. add BC (:469-472) */
  for (int v = 0; v < n; v++) bc[v] += s->delta[v] * 0.5;
}

static int resolve_threads(int nthreads) {
#ifdef _OPENMP
  return nthreads > 0 ? nthreads : omp_get_max_threads();
#else
  (void)nthreads;
  return 1;
#endif
}

int orc_mhl_bc(const orc_tc *tc, const orc_arcs *g, const int *sources, int ns, double *bc_out, int nthreads) {
  const int n = tc->n;
  if (g->n != n) return -1;
  if (!sources) ns = n;
  int nt = resolve_threads(nthreads);
  double *part = (double *)xcalloc((size_t)nt * (size_t)n, sizeof(double));
#pragma omp parallel num_threads(nt)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    mhl_scratch s;
    s.lcaq = (int *)xmalloc(sizeof(int) * (size_t)n);
    s.dist = (int *)xmalloc(sizeof(int) * (size_t)n);
    s.layer = (int *)xmalloc(sizeof(int) * (size_t)n);
    s.cnt = (uint32_t *)xmalloc(sizeof(uint32_t) * (size_t)n);
    s.layer_edge = (int *)xmalloc(sizeof(int) * (size_t)(g->m ? g->m : 1));
    s.queue = (int *)xmalloc(sizeof(int) * (size_t)(g->m ? g->m : 1));
    s.layer_size = (int *)xcalloc((size_t)n + 2, sizeof(int));
    s.layer_start = (int *)xcalloc((size_t)n + 2, sizeof(int));
    s.delta = (double *)xmalloc(sizeof(double) * (size_t)n);
#pragma omp for schedule(dynamic, 1)
    for (int k = 0; k < ns; k++) {
      int src = sources ? sources[k] : k;
      mhl_one(tc, g, src, &s, part + (size_t)tid * n);
    }
    free(s.lcaq); free(s.dist); free(s.layer); free(s.cnt); free(s.layer_edge); free(s.queue);
    free(s.layer_size); free(s.layer_start); free(s.delta);
  }
  for (int v = 0; v < n; v++) {
    double acc = 0.0;
    for (int t = 0; t < nt; t++) acc += part[(size_t)t * n + v];
    bc_out[v] = acc;
  }
  free(part);
  return 0;
}

/* ======================================================================================
 * RQ pair formula (RQ.cu:201-291 rows of each query vertex, :354-459 pair kernel,
 * :516-520 host sum).  Each pair term is (int)(sigma_vs*sigma_vt) * (1.0/sigma_st).
 * ====================================================================================== */
static void tc_rows_rq(const orc_tc *tc, int source, int *lcaq, int *distance, uint32_t *count) {
  /* Same scan as tc_rows; RQ.cu uses INT_MAX as the starting value (:400,424), which only
   * differs from 999999999 when no label entry exists (a disconnected graph). */
  int *layer = (int *)xmalloc(sizeof(int) * (size_t)tc->n);
  int ml;
  tc_rows(tc, source, lcaq, distance, count, layer, &ml);
  free(layer);
}

int orc_rq_bc(const orc_tc *tc, const int *points, int q, double *out, int nthreads) {
  const int n = tc->n;
  int *pd = (int *)xmalloc(sizeof(int) * (size_t)q * (size_t)n);
  uint32_t *pc = (uint32_t *)xmalloc(sizeof(uint32_t) * (size_t)q * (size_t)n);
  int *lcaq = (int *)xmalloc(sizeof(int) * (size_t)n);
  for (int i = 0; i < q; i++) {
    if (points[i] < 0 || points[i] >= n) { free(pd); free(pc); free(lcaq); return -1; }
    tc_rows_rq(tc, points[i], lcaq, pd + (size_t)i * n, pc + (size_t)i * n);
  }
  free(lcaq);
  int nt = resolve_threads(nthreads);
  double *part = (double *)xcalloc((size_t)nt * (size_t)q, sizeof(double));
#pragma omp parallel num_threads(nt)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    int *lq = (int *)xmalloc(sizeof(int) * (size_t)n);
    int *d = (int *)xmalloc(sizeof(int) * (size_t)n);
    uint32_t *c = (uint32_t *)xmalloc(sizeof(uint32_t) * (size_t)n);
    double *acc = part + (size_t)tid * q;
#pragma omp for schedule(dynamic, 1)
    for (int s = 0; s < n; s++) {
      tc_rows_rq(tc, s, lq, d, c);
      for (int t = s + 1; t < n; t++) {
        double sigma_t = 1.0 / (double)(int)c[t];
        int distance_t = d[t];
        for (int i = 0; i < q; i++) {
          const int *pdi = pd + (size_t)i * n;
          const uint32_t *pci = pc + (size_t)i * n;
          if (s != points[i] && t != points[i] && distance_t == pdi[s] + pdi[t]) {
            int prod = (int)(pci[s] * pci[t]);
            acc[i] += prod * sigma_t;
          }
        }
      }
    }
    free(lq); free(d); free(c);
  }
  for (int i = 0; i < q; i++) {
    double a = 0.0;
    for (int t = 0; t < nt; t++) a += part[(size_t)t * q + i];
    out[i] = a;
  }
  free(part); free(pd); free(pc);
  return 0;
}

/* ======================================================================================
 * H2H index of QBC (buildIndex.cpp) and QBC per-source loop (QBC.cu)
 * ====================================================================================== */
int orc_h2h_build(const orc_arcs *g, const int *node_order, orc_h2h **out) {
  const int n = g->n;
  int *vorder = (int *)xmalloc(sizeof(int) * (size_t)n);
  for (int i = 0; i < n; i++) vorder[i] = -1;
  for (int v = 0; v < n; v++) { /* CHconsorderMT (:10-20) */
    int o = node_order[v];
    if (o < 0 || o >= n) { free(vorder); return -1; }
    vorder[o] = v;
  }
  for (int i = 0; i < n; i++) if (vorder[i] < 0) { free(vorder); return -1; }
  /* E (Graph::ReadGraph :31): map per tail of (head, weight) */
  adj_t *E = (adj_t *)xcalloc((size_t)n, sizeof(adj_t));
  for (int t = 0; t < n; t++)
    for (int e = g->off[t]; e < g->off[t + 1]; e++) {
      int at = adj_find(&E[t], g->head[e]);
      if (at < 0) { adj_e x = {g->head[e], g->w[e], 1u, 0u}; adj_insert_at(&E[t], -(at + 1), x); }
    }
  char *exist = (char *)xmalloc((size_t)n);
  memset(exist, 1, (size_t)n);
  int64_t *ncon_start = (int64_t *)xmalloc(sizeof(int64_t) * (size_t)n);
  int *ncon_size = (int *)xmalloc(sizeof(int) * (size_t)n);
  int64_t cap = 4 * (int64_t)n + 16, used = 0;
  int *nc_v = (int *)xmalloc(sizeof(int) * (size_t)cap), *nc_w = (int *)xmalloc(sizeof(int) * (size_t)cap);
  adj_e *tmp = (adj_e *)xmalloc(sizeof(adj_e) * (size_t)n);
  for (int no = 0; no < n; no++) { /* contraction loop (:29-110) */
    int x = vorder[no];
    exist[x] = 0;
    int k = 0;
    for (int i = 0; i < E[x].n; i++)
      if (exist[E[x].e[i].v]) tmp[k++] = E[x].e[i];
    for (int i = 0; i < k; i++) { adj_erase(&E[x], tmp[i].v); adj_erase(&E[tmp[i].v], x); }
    if (used + k > cap) {
      while (used + k > cap) cap *= 2;
      nc_v = (int *)realloc(nc_v, sizeof(int) * (size_t)cap);
      nc_w = (int *)realloc(nc_w, sizeof(int) * (size_t)cap);
      if (!nc_v || !nc_w) abort();
    }
    ncon_start[x] = used; ncon_size[x] = k;
    for (int i = 0; i < k; i++) { nc_v[used + i] = tmp[i].v; nc_w[used + i] = tmp[i].w; }
    used += k;
    for (int i = 0; i < k; i++)
      for (int j = i + 1; j < k; j++) { /* insertEorder (:125-149) */
        int u = tmp[i].v, v = tmp[j].v, ww = tmp[i].w + tmp[j].w;
        int a = adj_find(&E[u], v);
        if (a < 0) { adj_e y = {v, ww, 1u, 0u}; adj_insert_at(&E[u], -(a + 1), y); }
        else if (E[u].e[a].w > ww) E[u].e[a].w = ww;
        int b = adj_find(&E[v], u);
        if (b < 0) { adj_e y = {u, ww, 1u, 0u}; adj_insert_at(&E[v], -(b + 1), y); }
        else if (E[v].e[b].w > ww) E[v].e[b].w = ww;
      }
  }
  free(tmp);
  for (int i = 0; i < n; i++) free(E[i].e);
  free(E); free(exist);

  orc_h2h *h = (orc_h2h *)xcalloc(1, sizeof(orc_h2h));
  h->n = n;
  h->rank = (int *)xmalloc(sizeof(int) * (size_t)n);
  h->uvertex = (int *)xmalloc(sizeof(int) * (size_t)n);
  h->parent = (int *)xmalloc(sizeof(int) * (size_t)n);
  h->height = (int *)xmalloc(sizeof(int) * (size_t)n);
  h->vert_off = (int64_t *)xmalloc(sizeof(int64_t) * ((size_t)n + 1));
  h->vert = (int *)xmalloc(sizeof(int) * (size_t)(used ? used : 1));
  h->vert_w = (int *)xmalloc(sizeof(int) * (size_t)(used ? used : 1));
  /* makeTree (:151-196) */
  int64_t o = 0;
  int *nchild = (int *)xcalloc((size_t)n + 1, sizeof(int));
  int rc = 0;
  for (int len = n - 1, p = 0; len >= 0; len--, p++) {
    int x = vorder[len];
    h->uvertex[p] = x;
    h->vert_off[p] = o;
    for (int i = 0; i < ncon_size[x]; i++) { h->vert[o + i] = nc_v[ncon_start[x] + i]; h->vert_w[o + i] = nc_w[ncon_start[x] + i]; }
    o += ncon_size[x];
    if (len == n - 1) {
      h->parent[p] = -1; h->height[p] = 1;
    } else {
      if (ncon_size[x] == 0) { rc = -3; h->parent[p] = 0; h->height[p] = 2; }
      else {
        int nearest = nc_v[ncon_start[x]]; /* match (:197-207) */
        for (int i = 1; i < ncon_size[x]; i++)
          if (h->rank[nc_v[ncon_start[x] + i]] > h->rank[nearest]) nearest = nc_v[ncon_start[x] + i];
        int pa = h->rank[nearest];
        h->parent[p] = pa;
        h->height[p] = h->height[pa] + 1;
      }
      nchild[h->parent[p]]++;
    }
    h->rank[x] = p;
  }
  h->vert_off[n] = o;
  free(nc_v); free(nc_w); free(ncon_start); free(ncon_size); free(vorder);
  h->child_off = (int *)xmalloc(sizeof(int) * ((size_t)n + 1));
  h->child_off[0] = 0;
  for (int p = 0; p < n; p++) h->child_off[p + 1] = h->child_off[p] + nchild[p];
  h->child = (int *)xmalloc(sizeof(int) * (size_t)(n > 1 ? n - 1 : 1));
  memset(nchild, 0, sizeof(int) * ((size_t)n + 1));
  for (int p = 1; p < n; p++) { int pp = h->parent[p]; h->child[h->child_off[pp] + nchild[pp]++] = p; }
  free(nchild);
  if (rc) { *out = h; orc_h2h_free(h); *out = NULL; return rc; }

  /* makeRMQ (:279-310) */
  int m = 2 * n - 1;
  int *euler = (int *)xmalloc(sizeof(int) * (size_t)m);
  h->to_rmq = (int *)xmalloc(sizeof(int) * (size_t)n);
  {
    int *stk = (int *)xmalloc(sizeof(int) * (size_t)n), *it = (int *)xmalloc(sizeof(int) * (size_t)n);
    int sp = 0, el = 0;
    stk[sp] = 0; it[sp] = 0; sp++;
    h->to_rmq[0] = el; euler[el++] = 0;
    while (sp > 0) {
      int p = stk[sp - 1];
      if (it[sp - 1] < h->child_off[p + 1] - h->child_off[p]) {
        int c = h->child[h->child_off[p] + it[sp - 1]++];
        h->to_rmq[c] = el; euler[el++] = c;
        stk[sp] = c; it[sp] = 0; sp++;
      } else {
        sp--;
        if (sp > 0) euler[el++] = stk[sp - 1];
      }
    }
    free(stk); free(it);
    m = el;
  }
  h->euler_len = m;
  int levels = 1;
  for (int i = 2; i < m; i *= 2) levels++;
  h->rmq_levels = levels;
  h->rmq = (int *)xcalloc((size_t)levels * (size_t)m, sizeof(int));
  memcpy(h->rmq, euler, sizeof(int) * (size_t)m);
  for (int i = 2, k = 1; i < m; i *= 2, ++k) {
    int *prev = h->rmq + (size_t)(k - 1) * m, *cur = h->rmq + (size_t)k * m;
    for (int j = 0; j < m - i; j++) {
      int x = prev[j], y = prev[j + i / 2];
      cur[j] = h->height[x] < h->height[y] ? x : y;
    }
  }
  free(euler);

  /* makeIndex / makeIndexDFS (:208-278): H2H distance labels, in tree-position order */
  h->pos_off = (int64_t *)xmalloc(sizeof(int64_t) * ((size_t)n + 1));
  h->dis_off = (int64_t *)xmalloc(sizeof(int64_t) * ((size_t)n + 1));
  int64_t po = 0, dlo = 0;
  for (int p = 0; p < n; p++) {
    h->pos_off[p] = po; h->dis_off[p] = dlo;
    po += (h->vert_off[p + 1] - h->vert_off[p]) + 1;
    dlo += h->height[p] - 1;
  }
  h->pos_off[n] = po; h->dis_off[n] = dlo;
  h->pos = (int *)xmalloc(sizeof(int) * (size_t)po);
  h->dis = (int *)xmalloc(sizeof(int) * (size_t)(dlo ? dlo : 1));
  h->pos[0] = 0;
  for (int p = 1; p < n; p++) {
    int nX = (int)(h->vert_off[p + 1] - h->vert_off[p]);
    int L = h->height[p] - 1;
    int *pos = h->pos + h->pos_off[p], *dis = h->dis + h->dis_off[p];
    const int *vv = h->vert + h->vert_off[p], *vw = h->vert_w + h->vert_off[p];
    for (int j = 0; j < L; j++) dis[j] = H2H_INF;
    for (int i = 0; i < nX; i++) { pos[i] = h->height[h->rank[vv[i]]] - 1; dis[pos[i]] = vw[i]; }
    pos[nX] = L;
    /* ancestors by depth: walk parents */
    int *anc = (int *)xmalloc(sizeof(int) * (size_t)(L ? L : 1));
    for (int a = h->parent[p], d = L - 1; d >= 0; a = h->parent[a], d--) anc[d] = a;
    for (int i = 0; i < nX; i++) {
      int xk = h->rank[vv[i]], disvb = vw[i], k = pos[i];
      for (int j = 0; j < L; j++) {
        if (k == j) continue;
        int z = (k < j) ? h->dis[h->dis_off[anc[j]] + k] : h->dis[h->dis_off[xk] + j];
        if (dis[j] > z + disvb) dis[j] = z + disvb;
      }
    }
    free(anc);
  }

  /* optimizeVS (:313-386); the unordered_map iteration order is replaced by ascending
   * position order, which only permutes the scanned set. */
  h->popt_off = (int64_t *)xmalloc(sizeof(int64_t) * ((size_t)n + 1));
  int64_t pcap = 2 * (int64_t)n + 16, pu = 0;
  h->popt = (int *)xmalloc(sizeof(int) * (size_t)pcap);
  int *cnt = (int *)xcalloc((size_t)n + 1, sizeof(int));
  for (int v = 0; v < n; v++) {
    h->popt_off[v] = pu;
    int nch = h->child_off[v + 1] - h->child_off[v];
    int back = h->pos[h->pos_off[v + 1] - 1];
    int64_t need = pu + (int64_t)h->height[v] + 2;
    if (need > pcap) { while (need > pcap) pcap *= 2; h->popt = (int *)realloc(h->popt, sizeof(int) * (size_t)pcap); if (!h->popt) abort(); }
    if (nch < 2) {
      h->popt[pu++] = back;
    } else if (nch == 2) {
      int c1 = h->child[h->child_off[v]], c2 = h->child[h->child_off[v] + 1];
      int64_t s1 = h->pos_off[c1 + 1] - h->pos_off[c1], s2 = h->pos_off[c2 + 1] - h->pos_off[c2];
      int t = s1 < s2 ? c1 : c2;
      int64_t ts = h->pos_off[t + 1] - h->pos_off[t];
      for (int64_t kk = ts - 2; kk >= 0; --kk) {
        int pk = h->pos[h->pos_off[t] + kk];
        if (pk != back) h->popt[pu++] = pk;
      }
      h->popt[pu++] = back;
    } else {
      int bestA = -1, bi = 0;
      for (int c = 0; c < nch; c++) {
        int ch = h->child[h->child_off[v] + c];
        for (int64_t kk = h->pos_off[ch + 1] - h->pos_off[ch] - 2; kk >= 0; --kk) cnt[h->pos[h->pos_off[ch] + kk]]++;
      }
      for (int c = 0; c < nch; c++) {
        int ch = h->child[h->child_off[v] + c], A = 0;
        for (int64_t kk = h->pos_off[ch + 1] - h->pos_off[ch] - 2; kk >= 0; --kk)
          if (cnt[h->pos[h->pos_off[ch] + kk]] == 1) A++;
        if (bestA < 0 || A > bestA) { bestA = A; bi = c; }
      }
      {
        int ch = h->child[h->child_off[v] + bi];
        for (int64_t kk = h->pos_off[ch + 1] - h->pos_off[ch] - 2; kk >= 0; --kk) cnt[h->pos[h->pos_off[ch] + kk]]--;
      }
      for (int key = 0; key < h->height[v]; key++)
        if (cnt[key] > 0 && key != back) h->popt[pu++] = key;
      h->popt[pu++] = back;
      for (int c = 0; c < nch; c++) { /* clear */
        int ch = h->child[h->child_off[v] + c];
        for (int64_t kk = h->pos_off[ch + 1] - h->pos_off[ch] - 2; kk >= 0; --kk) cnt[h->pos[h->pos_off[ch] + kk]] = 0;
      }
    }
  }
  h->popt_off[n] = pu;
  free(cnt);
  *out = h;
  return 0;
}

void orc_h2h_free(orc_h2h *h) {
  if (!h) return;
  free(h->rank); free(h->uvertex); free(h->parent); free(h->height); free(h->child_off); free(h->child);
  free(h->vert_off); free(h->vert); free(h->vert_w); free(h->pos_off); free(h->pos); free(h->dis_off);
  free(h->dis); free(h->popt_off); free(h->popt); free(h->to_rmq); free(h->rmq);
  free(h);
}

/* LCA with the CPU `while (i*2 < len)` window (QBC.cu:247-267). */
static inline int h2h_lca(const orc_h2h *h, int p, int q) {
  if (p > q) { int t = p; p = q; q = t; }
  int len = q - p + 1, i = 1, k = 0;
  while (i * 2 < len) { i *= 2; k++; }
  q = q - i + 1;
  const int *lv = h->rmq + (size_t)k * h->euler_len;
  int a = lv[p], b = lv[q];
  return h->height[a] < h->height[b] ? a : b;
}

static void h2h_row(const orc_h2h *h, int source, int *lcaq, int *distance) {
  const int n = h->n;
  int x1 = h->rank[source], p1 = h->to_rmq[x1];
  for (int idx = 0; idx < n; idx++) lcaq[idx] = h2h_lca(h, p1, h->to_rmq[idx]);
  for (int idx = 0; idx < n; idx++) { /* QBC.cu:272-331 */
    if (idx == source) { distance[idx] = 0; continue; }
    int r1 = x1, r2 = h->rank[idx], LCA = lcaq[r2], t = H2H_INF;
    if (LCA == r1) {
      int r1_idx = h->popt[h->popt_off[r1 + 1] - 1];
      t = h->dis[h->dis_off[r2] + r1_idx];
    } else if (LCA == r2) {
      int r2_idx = h->popt[h->popt_off[r2 + 1] - 1];
      t = h->dis[h->dis_off[r1] + r2_idx];
    } else {
      const int *d1 = h->dis + h->dis_off[r1], *d2 = h->dis + h->dis_off[r2];
      for (int64_t i = h->popt_off[LCA + 1] - 1; i >= h->popt_off[LCA]; --i) {
        int off = h->popt[i];
        int sum = d1[off] + d2[off];
        if (t > sum) t = sum;
      }
    }
    distance[idx] = t;
  }
}

int orc_qbc_dist(const orc_h2h *h, int source, int *dist) {
  if (source < 0 || source >= h->n) return -1;
  int *lcaq = (int *)xmalloc(sizeof(int) * (size_t)h->n);
  h2h_row(h, source, lcaq, dist);
  free(lcaq);
  return 0;
}

/* QBC.cu:335-344 successors/indegree, :485-555 host Kahn sigma + edge layers,
 * :379-397 backprop and 0.5*delta. */
int orc_qbc_bc(const orc_h2h *h, const orc_arcs *g, const int *sources, int ns, double *bc_out, int nthreads) {
  const int n = h->n, m = g->m;
  if (g->n != n) return -1;
  if (!sources) ns = n;
  int nt = resolve_threads(nthreads);
  double *part = (double *)xcalloc((size_t)nt * (size_t)n, sizeof(double));
  int bad = 0;
#pragma omp parallel num_threads(nt)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    int *lcaq = (int *)xmalloc(sizeof(int) * (size_t)n);
    int *dist = (int *)xmalloc(sizeof(int) * (size_t)n);
    int *indeg = (int *)xmalloc(sizeof(int) * (size_t)n);
    unsigned char *succ = (unsigned char *)xmalloc((size_t)(m ? m : 1));
    int *sigma = (int *)xmalloc(sizeof(int) * (size_t)n);
    int *queue = (int *)xmalloc(sizeof(int) * (size_t)n);
    int *qedge = (int *)xmalloc(sizeof(int) * (size_t)(m ? m : 1));
    int *lstart = (int *)xmalloc(sizeof(int) * ((size_t)n + 2));
    double *delta = (double *)xmalloc(sizeof(double) * (size_t)n);
    int *tail = (int *)xmalloc(sizeof(int) * (size_t)(m ? m : 1));
    for (int t = 0; t < n; t++) for (int e = g->off[t]; e < g->off[t + 1]; e++) tail[e] = t;
    double *acc = part + (size_t)tid * n;
#pragma omp for schedule(dynamic, 1)
    for (int k = 0; k < ns; k++) {
      int source = sources ? sources[k] : k;
      h2h_row(h, source, lcaq, dist);
      for (int i = 0; i < n; i++) indeg[i] = 0;
      for (int e = 0; e < m; e++) {
        int t = tail[e], hh = g->head[e];
        if (dist[hh] == dist[t] + g->w[e]) { succ[e] = 1; indeg[hh]++; } else succ[e] = 0;
      }
      for (int i = 0; i < n; i++) sigma[i] = 0;
      sigma[source] = 1;
      int layerQueueStart, layerSize, h_cnt = 0, total_edge = 0, nlayer = 0;
      lstart[0] = 0;
      queue[0] = source;
      for (int j = g->off[source]; j < g->off[source + 1]; ++j) {
        if (succ[j]) {
          int NN = g->head[j];
          sigma[NN] = (int)((uint32_t)sigma[NN] + (uint32_t)sigma[source]);
          if (--indeg[NN] == 0) queue[1 + h_cnt++] = NN;
        }
      }
      layerQueueStart = 1; layerSize = h_cnt;
      int guard = 0;
      while (layerQueueStart + layerSize != n) {
        if (layerSize == 0 || ++guard > n) { bad = 1; break; } /* the reference spins here */
        h_cnt = 0;
        int h_cnt_edge = 0;
        for (int idx = 0; idx < layerSize; ++idx) {
          int nodeID = queue[idx + layerQueueStart];
          for (int j = g->off[nodeID]; j < g->off[nodeID + 1]; ++j) {
            if (succ[j]) {
              int NN = g->head[j];
              sigma[NN] = (int)((uint32_t)sigma[NN] + (uint32_t)sigma[nodeID]);
              if (--indeg[NN] == 0) queue[layerQueueStart + layerSize + h_cnt++] = NN;
              qedge[total_edge + h_cnt_edge++] = j;
            }
          }
        }
        layerQueueStart += layerSize;
        layerSize = h_cnt;
        total_edge += h_cnt_edge;
        lstart[++nlayer] = total_edge;
      }
      int maxLayer = nlayer;
      for (int i = 0; i < n; i++) delta[i] = 0.0;
      for (int i = maxLayer - 1; i >= 0; --i) {
        for (int idx = lstart[i]; idx < lstart[i + 1]; idx++) {
          int e = qedge[idx];
          int t = tail[e], hh = g->head[e];
          delta[t] += (double)sigma[t] * (1 + delta[hh]) / (double)sigma[hh];
        }
      }
      for (int v = 0; v < n; v++) acc[v] += delta[v] * 0.5;
    }
    free(lcaq); free(dist); free(indeg); free(succ); free(sigma); free(queue); free(qedge);
    free(lstart); free(delta); free(tail);
  }
  for (int v = 0; v < n; v++) {
    double a = 0.0;
    for (int t = 0; t < nt; t++) a += part[(size_t)t * n + v];
    bc_out[v] = a;
  }
  free(part);
  return bad ? -4 : 0;
}

/* ======================================================================================
 * Independent witness: Dijkstra (binary heap) + Brandes dependency accumulation.
 * ====================================================================================== */
typedef struct { int64_t key; int v; } dh_e;
static void dh_push(dh_e *a, int *n, dh_e x) {
  int i = (*n)++;
  a[i] = x;
  while (i > 0) {
    int p = (i - 1) >> 1;
    if (a[p].key <= a[i].key) break;
    dh_e t = a[p]; a[p] = a[i]; a[i] = t; i = p;
  }
}
static dh_e dh_pop(dh_e *a, int *n) {
  dh_e top = a[0];
  a[0] = a[--(*n)];
  int i = 0;
  for (;;) {
    int l = 2 * i + 1, r = l + 1, s = i;
    if (l < *n && a[l].key < a[s].key) s = l;
    if (r < *n && a[r].key < a[s].key) s = r;
    if (s == i) break;
    dh_e t = a[s]; a[s] = a[i]; a[i] = t; i = s;
  }
  return top;
}

/* settles vertices in nondecreasing distance; order[] receives settle order */
static int dijkstra(const orc_arcs *g, int source, int *dist, uint32_t *cnt, int *hop, int *order, dh_e *heap,
                    char *done) {
  const int n = g->n;
  for (int i = 0; i < n; i++) { dist[i] = INT_MAX; cnt[i] = 0; hop[i] = 0; done[i] = 0; }
  int hn = 0, no = 0;
  dist[source] = 0; cnt[source] = 1; hop[source] = 0;
  dh_e s0 = {0, source};
  dh_push(heap, &hn, s0);
  while (hn > 0) {
    dh_e t = dh_pop(heap, &hn);
    int v = t.v;
    if (done[v] || t.key != dist[v]) continue;
    done[v] = 1;
    order[no++] = v;
    for (int e = g->off[v]; e < g->off[v + 1]; e++) {
      int w = g->head[e];
      int64_t nd = (int64_t)dist[v] + g->w[e];
      if (nd < dist[w]) {
        dist[w] = (int)nd; cnt[w] = cnt[v]; hop[w] = hop[v] + 1;
        dh_e x = {nd, w};
        dh_push(heap, &hn, x);
      } else if (nd == dist[w]) {
        cnt[w] += cnt[v];
        if (hop[v] + 1 > hop[w]) hop[w] = hop[v] + 1;
      }
    }
  }
  return no;
}

int orc_dijkstra_rows(const orc_arcs *g, int source, int *dist, uint32_t *cnt, int *hop) {
  const int n = g->n;
  if (source < 0 || source >= n) return -1;
  int *order = (int *)xmalloc(sizeof(int) * (size_t)n);
  dh_e *heap = (dh_e *)xmalloc(sizeof(dh_e) * ((size_t)g->m + 1));
  char *done = (char *)xmalloc((size_t)n);
  dijkstra(g, source, dist, cnt, hop, order, heap, done);
  free(order); free(heap); free(done);
  return 0;
}

int orc_brandes_bc(const orc_arcs *g, const int *sources, int ns, double *bc_out, int nthreads) {
  const int n = g->n;
  if (!sources) ns = n;
  int nt = resolve_threads(nthreads);
  double *part = (double *)xcalloc((size_t)nt * (size_t)n, sizeof(double));
#pragma omp parallel num_threads(nt)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    int *dist = (int *)xmalloc(sizeof(int) * (size_t)n), *hop = (int *)xmalloc(sizeof(int) * (size_t)n);
    uint32_t *cnt = (uint32_t *)xmalloc(sizeof(uint32_t) * (size_t)n);
    int *order = (int *)xmalloc(sizeof(int) * (size_t)n);
    dh_e *heap = (dh_e *)xmalloc(sizeof(dh_e) * ((size_t)g->m + 1));
    char *done = (char *)xmalloc((size_t)n);
    double *delta = (double *)xmalloc(sizeof(double) * (size_t)n);
    double *acc = part + (size_t)tid * n;
#pragma omp for schedule(dynamic, 1)
    for (int k = 0; k < ns; k++) {
      int s = sources ? sources[k] : k;
      int no = dijkstra(g, s, dist, cnt, hop, order, heap, done);
      for (int i = 0; i < n; i++) delta[i] = 0.0;
      for (int i = no - 1; i >= 1; i--) { /* reverse settle order; pull from DAG successors */
        int v = order[i];
        double d = 0.0;
        for (int e = g->off[v]; e < g->off[v + 1]; e++) {
          int w = g->head[e];
          if (dist[w] != INT_MAX && (int64_t)dist[w] == (int64_t)dist[v] + g->w[e])
            d += (double)(int)cnt[v] * (1 + delta[w]) / (double)(int)cnt[w];
        }
        delta[v] = d;
      }
      for (int v = 0; v < n; v++) if (v != s) acc[v] += delta[v] * 0.5;
    }
    free(dist); free(hop); free(cnt); free(order); free(heap); free(done); free(delta);
  }
  for (int v = 0; v < n; v++) {
    double a = 0.0;
    for (int t = 0; t < nt; t++) a += part[(size_t)t * n + v];
    bc_out[v] = a;
  }
  free(part);
  return 0;
}
