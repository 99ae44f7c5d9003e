// host.cpp -- readers, validation and the tree-decomposition index builders of libqbc_b200.
//
// The index builders are this library's own design: a min-degree elimination (any elimination
// order yields the same distances, path counts and hop layers; only the index size depends on it),
// a DFS-preorder renumbering so every subtree is a contiguous id range, and label rows that
// include the node itself so one prefix scan covers the reference's ancestor/descendant special
// cases (MHLQBC.cu:356-373).  Rows are filled in parallel: a row reads only its ancestors' rows.
#include "host.h"

#include "../../include/qbc_b200.h"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <thread>

#include <omp.h>

namespace qbc {

// separators at least this large are merged into their neighbours' lists in parallel
constexpr int32_t kParallelSeparator = 32;

int hardware_threads(int requested) {
  if (requested > 0) return requested;
  unsigned h = std::thread::hardware_concurrency();
  return h ? (int)h : 1;
}

template <class F>
static void parallel_for(int64_t count, int nthreads, F &&f) {
  nthreads = (int)std::min<int64_t>(std::max(1, nthreads), std::max<int64_t>(1, count));
  if (nthreads <= 1) {
    for (int64_t i = 0; i < count; i++) f(i);
    return;
  }
  std::atomic<int64_t> next{0};
  std::vector<std::thread> th;
  for (int t = 0; t < nthreads; t++)
    th.emplace_back([&]() {
      for (;;) {
        int64_t i = next.fetch_add(1, std::memory_order_relaxed);
        if (i >= count) break;
        f(i);
      }
    });
  for (auto &t : th) t.join();
}

// ------------------------------------------------------------------------------------ readers
namespace {
struct Reader {
  std::vector<char> buf;
  size_t p = 0;
  explicit Reader(const std::string &path) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) throw Error(QBC_EIO, "cannot open " + path);
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    buf.resize((size_t)std::max<long>(sz, 0) + 1);
    size_t got = sz > 0 ? fread(buf.data(), 1, (size_t)sz, f) : 0;
    fclose(f);
    buf[got] = 0;
    buf.resize(got + 1);
  }
  bool next(int64_t &v) {
    while (p < buf.size() && buf[p] && (buf[p] == ' ' || buf[p] == '\n' || buf[p] == '\r' || buf[p] == '\t')) p++;
    if (p >= buf.size() || !buf[p]) return false;
    bool neg = false;
    if (buf[p] == '-' || buf[p] == '+') { neg = buf[p] == '-'; p++; }
    if (buf[p] < '0' || buf[p] > '9') return false;
    int64_t x = 0;
    while (buf[p] >= '0' && buf[p] <= '9') { x = x * 10 + (buf[p] - '0'); p++; }
    v = neg ? -x : x;
    return true;
  }
};
}  // namespace

Graph graph_read(const std::string &path) {
  Reader r(path);
  int64_t n, m;
  if (!r.next(n) || !r.next(m)) throw Error(QBC_EIO, path + ": missing 'n m' header");
  if (n <= 0 || n > INT32_MAX - 2 || m < 0) throw Error(QBC_EIO, path + ": bad header");
  std::vector<int32_t> u((size_t)m), v((size_t)m), w((size_t)m);
  for (int64_t i = 0; i < m; i++) {
    int64_t a, b, c;
    if (!r.next(a) || !r.next(b) || !r.next(c))
      throw Error(QBC_EIO, path + ": expected " + std::to_string(m) + " arc lines, found " + std::to_string(i));
    if (c < INT32_MIN || c > INT32_MAX || a < INT32_MIN || a > INT32_MAX || b < INT32_MIN || b > INT32_MAX)
      throw Error(QBC_EIO, path + ": value out of int32 range at arc " + std::to_string(i));
    u[i] = (int32_t)a; v[i] = (int32_t)b; w[i] = (int32_t)c;
  }
  return graph_from_lines((int32_t)n, m, u.data(), v.data(), w.data());
}

Graph graph_from_lines(int32_t n, int64_t m, const int32_t *u1, const int32_t *v1, const int32_t *w) {
  if (n <= 0) throw Error(QBC_EINVAL, "n must be positive");
  if (m < 0) throw Error(QBC_EINVAL, "m must be non-negative");
  std::vector<int32_t> deg((size_t)n + 1, 0);
  for (int64_t i = 0; i < m; i++) {
    if (u1[i] < 1 || u1[i] > n || v1[i] < 1 || v1[i] > n)
      throw Error(QBC_EIO, "arc " + std::to_string(i) + ": vertex id out of range 1.." + std::to_string(n));
    if (u1[i] == v1[i]) throw Error(QBC_EGRAPH, "arc " + std::to_string(i) + ": self loop");
    if (w[i] < 0) throw Error(QBC_EGRAPH, "arc " + std::to_string(i) + ": negative weight");
    deg[u1[i]]++;
  }
  for (int32_t i = 0; i < n; i++) deg[i + 1] += deg[i];
  // stable bucket by tail: position k of tail a holds file line order
  std::vector<int64_t> line((size_t)m);
  {
    std::vector<int32_t> fill(deg.begin(), deg.end() - 1);
    for (int64_t i = 0; i < m; i++) line[fill[u1[i] - 1]++] = i;
  }
  Graph g;
  g.n = n;
  g.off.assign((size_t)n + 1, 0);
  g.head.reserve((size_t)m);
  g.w.reserve((size_t)m);
  std::vector<int64_t> tmp;
  std::vector<char> keep;
  int64_t wsum = 0;
  for (int32_t a = 0; a < n; a++) {
    g.off[a] = (int32_t)g.head.size();
    int32_t lo = deg[a], hi = deg[a + 1];
    tmp.assign(line.begin() + lo, line.begin() + hi);
    // detect duplicates: sort by head, stable so the file-first arc leads each run
    std::vector<int64_t> byh = tmp;
    std::stable_sort(byh.begin(), byh.end(), [&](int64_t x, int64_t y) { return v1[x] < v1[y]; });
    keep.assign((size_t)(hi - lo), 0);
    std::vector<int64_t> kept_lines;
    for (size_t k = 0; k < byh.size(); k++) {
      if (k > 0 && v1[byh[k]] == v1[byh[k - 1]]) {
        int32_t w0 = w[byh[k - 1]] == 0 ? 1 : w[byh[k - 1]], w1 = w[byh[k]] == 0 ? 1 : w[byh[k]];
        if (w0 != w1)
          throw Error(QBC_EGRAPH, "arc " + std::to_string(u1[byh[k]]) + "->" + std::to_string(v1[byh[k]]) +
                                      " repeated with a different weight");
        continue;
      }
      kept_lines.push_back(byh[k]);
    }
    std::sort(kept_lines.begin(), kept_lines.end());  // back to file order
    for (int64_t li : kept_lines) {
      g.head.push_back(v1[li] - 1);
      int32_t ww = w[li] == 0 ? 1 : w[li];  // src/Graph.cpp:27-28
      g.w.push_back(ww);
      wsum += ww;
    }
  }
  g.off[n] = (int32_t)g.head.size();
  // symmetry: every arc needs its reverse with the same weight
  std::vector<int32_t> sorted_head(g.head.size()), sorted_w(g.head.size());
  for (int32_t a = 0; a < n; a++) {
    std::vector<std::pair<int32_t, int32_t>> hw;
    for (int32_t e = g.off[a]; e < g.off[a + 1]; e++) hw.push_back({g.head[e], g.w[e]});
    std::sort(hw.begin(), hw.end());
    for (size_t k = 0; k < hw.size(); k++) {
      sorted_head[g.off[a] + k] = hw[k].first;
      sorted_w[g.off[a] + k] = hw[k].second;
    }
  }
  for (int32_t a = 0; a < n; a++)
    for (int32_t e = g.off[a]; e < g.off[a + 1]; e++) {
      int32_t b = g.head[e];
      auto first = sorted_head.begin() + g.off[b], last = sorted_head.begin() + g.off[b + 1];
      auto it = std::lower_bound(first, last, a);
      if (it == last || *it != a)
        throw Error(QBC_EGRAPH, "arc " + std::to_string(a + 1) + "->" + std::to_string(b + 1) + " has no reverse arc");
      if (sorted_w[it - sorted_head.begin()] != g.w[e])
        throw Error(QBC_EGRAPH, "arcs " + std::to_string(a + 1) + "<->" + std::to_string(b + 1) + " differ in weight");
    }
  if (wsum / 2 >= (int64_t)kInf) throw Error(QBC_EGRAPH, "total edge weight reaches the distance sentinel 999999999");
  return g;
}

std::vector<int32_t> read_order(const std::string &path, int32_t n) {
  Reader r(path);
  int64_t num;
  if (!r.next(num)) throw Error(QBC_EIO, path + ": missing vertex count");
  if (num != n) throw Error(QBC_EIO, path + ": order file lists " + std::to_string(num) + " vertices, graph has " + std::to_string(n));
  std::vector<int32_t> order((size_t)n, -1);
  std::vector<char> seen((size_t)n, 0);
  for (int64_t i = 0; i < num; i++) {
    int64_t id, o;
    if (!r.next(id) || !r.next(o)) throw Error(QBC_EIO, path + ": truncated at entry " + std::to_string(i));
    if (id < 0 || id >= n || o < 0 || o >= n) throw Error(QBC_EIO, path + ": entry " + std::to_string(i) + " out of range");
    if (seen[o]) throw Error(QBC_EIO, path + ": order " + std::to_string(o) + " repeated");
    seen[o] = 1;
    order[id] = (int32_t)o;
  }
  for (int32_t v = 0; v < n; v++)
    if (order[v] < 0) throw Error(QBC_EIO, path + ": vertex " + std::to_string(v) + " has no order");
  return order;
}

std::vector<int32_t> read_query(const std::string &path, int32_t n) {
  Reader r(path);
  int64_t q;
  if (!r.next(q) || q < 0) throw Error(QBC_EIO, path + ": missing query count");
  std::vector<int32_t> ids;
  ids.reserve((size_t)q);
  for (int64_t i = 0; i < q; i++) {
    int64_t id;
    if (!r.next(id)) throw Error(QBC_EIO, path + ": expected " + std::to_string(q) + " ids, found " + std::to_string(i));
    if (id < 1 || id > n) throw Error(QBC_EIO, path + ": id " + std::to_string(id) + " out of range");
    ids.push_back((int32_t)(id - 1));
  }
  return ids;
}

// ------------------------------------------------------------------------------- elimination
namespace {
struct Adj {
  int32_t v, len;
  uint32_t cnt;
  int32_t hop;
};

// Eliminates every vertex (in `fixed_order` if given, else by minimum current degree with the
// smaller id first).  For each vertex records its separator X(x): the neighbours still present,
// with the shortcut (length, path count, max hop) over already-eliminated vertices.
struct Elimination {
  std::vector<int32_t> order;     // elimination sequence
  std::vector<int32_t> rank;      // vid -> position in order
  std::vector<int64_t> x_off;     // separator lists in elimination order
  std::vector<Adj> x;
  int32_t width = 0;
};

// The vertices still to eliminate, by least current degree, then least id: per degree value a
// three-level 64-ary bitmap over vertex ids (a set bit at each level marks a nonzero word below),
// so the least id of a degree is three count-trailing-zeros and a degree change is a clear and a
// set.  An indexed binary heap's sift chains wander over 12 MB of arrays at 1M vertices; here the
// hot low-degree bitmaps stay in cache.  Bitmaps are made on first use (n/8 bytes each).
struct MinDegreeBuckets {
  struct Bits {
    std::vector<uint64_t> w0, w1, w2;
    int64_t count = 0;
  };
  std::vector<std::unique_ptr<Bits>> by_deg;
  std::vector<int32_t> deg;
  std::vector<char> live;
  size_t n0 = 0, n1 = 0, n2 = 0;
  int32_t lb = 0;  // no live vertex has a degree below lb

  Bits &at(int32_t d) {
    if ((size_t)d >= by_deg.size()) by_deg.resize((size_t)d + 1);
    if (!by_deg[d]) {
      by_deg[d] = std::make_unique<Bits>();
      by_deg[d]->w0.assign(n0, 0);
      by_deg[d]->w1.assign(n1, 0);
      by_deg[d]->w2.assign(n2, 0);
    }
    return *by_deg[d];
  }
  void insert(int32_t d, int32_t v) {
    Bits &b = at(d);
    const size_t i0 = (size_t)v >> 6, i1 = i0 >> 6, i2 = i1 >> 6;
    if (b.w0[i0] == 0) {
      if (b.w1[i1] == 0) b.w2[i2] |= 1ull << (i1 & 63);
      b.w1[i1] |= 1ull << (i0 & 63);
    }
    b.w0[i0] |= 1ull << (v & 63);
    b.count++;
    if (d < lb) lb = d;
  }
  void erase(int32_t d, int32_t v) {
    Bits &b = *by_deg[d];
    const size_t i0 = (size_t)v >> 6, i1 = i0 >> 6, i2 = i1 >> 6;
    b.w0[i0] &= ~(1ull << (v & 63));
    if (b.w0[i0] == 0) {
      b.w1[i1] &= ~(1ull << (i0 & 63));
      if (b.w1[i1] == 0) b.w2[i2] &= ~(1ull << (i1 & 63));
    }
    b.count--;
  }
  void init(std::vector<int32_t> d) {
    deg = std::move(d);
    const size_t n = deg.size();
    n0 = (n + 63) / 64;
    n1 = (n0 + 63) / 64;
    n2 = (n1 + 63) / 64;
    live.assign(n, 1);
    lb = 0;
    for (size_t v = 0; v < n; v++) insert(deg[v], (int32_t)v);
    lb = 0;
  }
  int32_t pop() {
    while ((size_t)lb < by_deg.size() && (!by_deg[lb] || by_deg[lb]->count == 0)) lb++;
    if ((size_t)lb >= by_deg.size()) throw Error(QBC_EGRAPH, "min-degree elimination ran out of vertices");
    const Bits &b = *by_deg[lb];
    size_t i2 = 0;
    while (b.w2[i2] == 0) i2++;
    const size_t i1 = (i2 << 6) | (size_t)__builtin_ctzll(b.w2[i2]);
    const size_t i0 = (i1 << 6) | (size_t)__builtin_ctzll(b.w1[i1]);
    const int32_t v = (int32_t)((i0 << 6) | (size_t)__builtin_ctzll(b.w0[i0]));
    erase(lb, v);
    live[v] = 0;
    return v;
  }
  void update(int32_t v, int32_t d) {
    if (!live[v] || deg[v] == d) return;
    erase(deg[v], v);
    deg[v] = d;
    insert(d, v);
  }
};

// The last tail_r steps handed to `tail` (min-degree elimination only): the vertices still present
// and their adjacency go out in local ids, the rest of the order and its separators come back.
static void run_tail(Elimination &el, std::vector<std::vector<Adj>> &adj, int32_t n, int32_t step,
                     const TailEngine &tail) {
  DenseTail dt;
  std::vector<int32_t> loc((size_t)n, -1);
  for (int32_t v = 0; v < n; v++)
    if (el.rank[v] < 0) {
      loc[v] = (int32_t)dt.ids.size();
      dt.ids.push_back(v);
    }
  dt.r = (int32_t)dt.ids.size();
  dt.off.assign((size_t)dt.r + 1, 0);
  for (int32_t i = 0; i < dt.r; i++) dt.off[i + 1] = dt.off[i] + (int64_t)adj[dt.ids[i]].size();
  dt.ent.resize((size_t)dt.off[dt.r] * 4);
  for (int32_t i = 0; i < dt.r; i++) {
    int64_t o = dt.off[i] * 4;
    for (const Adj &a : adj[dt.ids[i]]) {
      dt.ent[o++] = loc[a.v];
      dt.ent[o++] = a.len;
      dt.ent[o++] = (int32_t)a.cnt;
      dt.ent[o++] = a.hop;
    }
  }
  {
    TraceScope t("dense elimination tail");
    tail(dt);
  }
  if ((int32_t)dt.order.size() != dt.r || (int32_t)dt.x_off.size() != dt.r + 1)
    throw Error(QBC_ECUDA, "dense elimination returned a wrong-sized result");
  for (int32_t s = 0; s < dt.r; s++) {
    const int32_t x = dt.ids[dt.order[s]];
    el.rank[x] = step + s;
    el.order.push_back(x);
    const int64_t b = dt.x_off[s], e = dt.x_off[s + 1];
    el.width = std::max(el.width, (int32_t)(e - b));
    for (int64_t i = b; i < e; i++)
      el.x.push_back({dt.ids[dt.x[4 * i]], dt.x[4 * i + 1], (uint32_t)dt.x[4 * i + 2], dt.x[4 * i + 3]});
    el.x_off.push_back((int64_t)el.x.size());
  }
}

Elimination eliminate(const Graph &g, const std::vector<int32_t> *fixed_order, int32_t tail_r = 0,
                      const TailEngine &tail = {}) {
  const int32_t n = g.n;
  const int nthreads = hardware_threads(0);
  std::vector<std::vector<int32_t>> stamp_t, where_t;  // per-thread stamps for large separators
  std::vector<std::vector<Adj>> adj((size_t)n);
  for (int32_t a = 0; a < n; a++)
    for (int32_t e = g.off[a]; e < g.off[a + 1]; e++) adj[a].push_back({g.head[e], g.w[e], 1u, 1});
  Elimination el;
  el.order.reserve((size_t)n);
  el.rank.assign((size_t)n, -1);
  el.x_off.reserve((size_t)n + 1);
  el.x_off.push_back(0);
  std::vector<int32_t> stamp((size_t)n, -1), where((size_t)n, 0);
  MinDegreeBuckets pq;
  std::vector<int32_t> by_rank;
  if (fixed_order) {
    by_rank.assign((size_t)n, -1);
    for (int32_t v = 0; v < n; v++) by_rank[(*fixed_order)[v]] = v;
  } else {
    std::vector<int32_t> deg0((size_t)n);
    for (int32_t v = 0; v < n; v++) deg0[v] = (int32_t)adj[v].size();
    pq.init(std::move(deg0));
  }
  std::vector<Adj> X;
  for (int32_t step = 0; step < n; step++) {
    if (tail && !fixed_order && tail_r > 0 && n - step == tail_r) {
      run_tail(el, adj, n, step, tail);
      break;
    }
    int32_t x;
    if (fixed_order) {
      x = by_rank[step];
    } else {
      x = pq.pop();
    }
    el.rank[x] = step;
    el.order.push_back(x);
    X.swap(adj[x]);
    adj[x].clear();
    adj[x].shrink_to_fit();
    const int32_t k = (int32_t)X.size();
    el.width = std::max(el.width, k);
    // Neighbour u of x gets the shortcuts through x to every other neighbour.  stamp/where mark u's
    // current neighbours; a stale stamp (v marked for u earlier, v no longer in u's list) can only
    // belong to an eliminated v, which never reappears in a separator, so stamps are not cleared.
    auto merge = [&](int32_t i, std::vector<int32_t> &stp, std::vector<int32_t> &whr) {
      const int32_t u = X[i].v;
      std::vector<Adj> &au = adj[u];
      // drop x from u
      for (size_t e = 0; e < au.size(); e++)
        if (au[e].v == x) { au[e] = au.back(); au.pop_back(); break; }
      for (size_t e = 0; e < au.size(); e++) { stp[au[e].v] = u; whr[au[e].v] = (int32_t)e; }
      for (int32_t j = 0; j < k; j++) {
        if (j == i) continue;
        const int32_t v = X[j].v;
        const int32_t nl = X[i].len + X[j].len;
        const uint32_t nc = X[i].cnt * X[j].cnt;
        const int32_t nh = X[i].hop + X[j].hop;
        if (stp[v] == u) {
          Adj &a = au[whr[v]];
          if (nl < a.len) { a.len = nl; a.cnt = nc; a.hop = nh; }
          else if (nl == a.len) { a.cnt += nc; if (nh > a.hop) a.hop = nh; }
        } else {
          stp[v] = u;
          whr[v] = (int32_t)au.size();
          au.push_back({v, nl, nc, nh});
        }
      }
    };
    if (k >= kParallelSeparator && nthreads > 1) {
      // the large separators near the top of the tree dominate the elimination: their neighbours'
      // lists are updated in parallel (each neighbour by one thread, with its own stamp arrays)
      if (stamp_t.empty()) {
        stamp_t.assign((size_t)nthreads, std::vector<int32_t>((size_t)n, -1));
        where_t.assign((size_t)nthreads, std::vector<int32_t>((size_t)n, 0));
      }
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
      for (int32_t i = 0; i < k; i++) {
        const int t = omp_get_thread_num();
        merge(i, stamp_t[t], where_t[t]);
      }
    } else {
      for (int32_t i = 0; i < k; i++) merge(i, stamp, where);
    }
    if (!fixed_order)
      for (int32_t i = 0; i < k; i++) pq.update(X[i].v, (int32_t)adj[X[i].v].size());
    // any stamps left by neighbours-of-neighbours are harmless: they compare against a vertex id
    el.x.insert(el.x.end(), X.begin(), X.end());
    el.x_off.push_back((int64_t)el.x.size());
    X.clear();
  }
  return el;
}

// Tree from an elimination: parent(x) = the separator vertex eliminated first.  Renumbers
// vertices in DFS preorder and fills depth / parent / subtree end.
void make_tree(const Graph &g, const Elimination &el, Index &ix, bool host_rows = true) {
  const int32_t n = g.n;
  std::vector<int32_t> par((size_t)n, -1);
  int32_t roots = 0, root = -1;
  for (int32_t s = 0; s < n; s++) {
    int32_t x = el.order[s];
    int64_t b = el.x_off[s], e = el.x_off[s + 1];
    if (b == e) {
      roots++;
      root = x;
      continue;
    }
    int32_t best = el.x[b].v;
    for (int64_t i = b + 1; i < e; i++)
      if (el.rank[el.x[i].v] < el.rank[best]) best = el.x[i].v;
    par[x] = best;
  }
  if (roots != 1) throw Error(QBC_EGRAPH, "graph is not connected (" + std::to_string(roots) + " components)");
  // children, in decreasing elimination rank (the reference's tree-position order)
  std::vector<int32_t> cnt((size_t)n + 1, 0);
  for (int32_t v = 0; v < n; v++)
    if (par[v] >= 0) cnt[par[v] + 1]++;
  for (int32_t v = 0; v < n; v++) cnt[v + 1] += cnt[v];
  std::vector<int32_t> kids((size_t)std::max(n - 1, 1)), fill(cnt.begin(), cnt.end() - 1);
  for (int32_t s = n - 1; s >= 0; s--) {
    int32_t x = el.order[s];
    if (par[x] >= 0) kids[fill[par[x]]++] = x;
  }
  ix.n = n;
  ix.vid_of.assign((size_t)n, 0);
  ix.tid_of.assign((size_t)n, 0);
  ix.depth.assign((size_t)n, 0);
  ix.parent.assign((size_t)n, -1);
  ix.send.assign((size_t)n, 0);
  std::vector<int32_t> stk, it;
  stk.push_back(root);
  it.push_back(0);
  int32_t next = 0;
  ix.tid_of[root] = next;
  ix.vid_of[next] = root;
  ix.depth[next] = 1;
  next++;
  while (!stk.empty()) {
    int32_t v = stk.back();
    int32_t &k = it.back();
    if (cnt[v] + k < cnt[v + 1]) {
      int32_t c = kids[cnt[v] + k];
      k++;
      int32_t t = next++;
      ix.tid_of[c] = t;
      ix.vid_of[t] = c;
      ix.parent[t] = ix.tid_of[v];
      ix.depth[t] = ix.depth[ix.tid_of[v]] + 1;
      stk.push_back(c);
      it.push_back(0);
    } else {
      ix.send[ix.tid_of[v]] = next;
      stk.pop_back();
      it.pop_back();
    }
  }
  ix.tree_height = *std::max_element(ix.depth.begin(), ix.depth.end());
  ix.tree_width = el.width;
  ix.lab_off.assign((size_t)n + 1, 0);
  int64_t o = 0;
  ix.depth_sum = 0;
  for (int32_t t = 0; t < n; t++) {
    ix.lab_off[t] = o;
    o += (ix.depth[t] + 3) & ~3;
    ix.depth_sum += ix.depth[t];
  }
  ix.lab_off[n] = o;
  if (host_rows) fill_ancestor_rows(ix);
  // arcs in tid space
  ix.arc_off.assign((size_t)n + 1, 0);
  ix.arc_head.resize(g.head.size());
  ix.arc_w.resize(g.head.size());
  int32_t ao = 0;
  for (int32_t t = 0; t < n; t++) {
    ix.arc_off[t] = ao;
    int32_t v = ix.vid_of[t];
    for (int32_t e = g.off[v]; e < g.off[v + 1]; e++) {
      ix.arc_head[ao] = ix.tid_of[g.head[e]];
      ix.arc_w[ao] = g.w[e];
      ao++;
    }
  }
  ix.arc_off[n] = ao;
}

// Runs f(t) for every tid with all ancestors' rows finished first: tids are handed out in
// increasing order and a row only depends on its ancestors, which have smaller tids.
template <class F>
void fill_rows(const Index &ix, int nthreads, F &&f) {
  const int32_t n = ix.n;
  std::vector<std::atomic<uint8_t>> done((size_t)n);
  for (auto &d : done) d.store(0, std::memory_order_relaxed);
  auto wait = [&](int32_t t) {
    while (!done[t].load(std::memory_order_acquire)) std::this_thread::yield();
  };
  parallel_for(n, nthreads, [&](int64_t t) {
    f((int32_t)t, wait);
    done[t].store(1, std::memory_order_release);
  });
}
}  // namespace

void fill_ancestor_rows(Index &ix) {
  const int32_t n = ix.n;
  const int64_t o = ix.lab_off.empty() ? 0 : ix.lab_off[n];
  // a row is its parent's row plus the node itself (preorder: parent first)
  ix.anc.assign((size_t)o, 0);
  for (int32_t t = 0; t < n; t++) {
    const int32_t h = ix.depth[t];
    if (h <= 0) continue;
    int32_t *row = ix.anc.data() + ix.lab_off[t];
    if (ix.parent[t] >= 0) {
      const int32_t *prow = ix.anc.data() + ix.lab_off[ix.parent[t]];
      std::copy(prow, prow + (h - 1), row);
    }
    row[h - 1] = t;
  }
  ix.aend.assign((size_t)o, 0);
  for (int32_t t = 0; t < n; t++) {
    const int64_t b = ix.lab_off[t];
    for (int32_t j = 0; j < ix.depth[t]; j++) ix.aend[b + j] = ix.send[ix.anc[b + j]];
  }
}

// Elimination (min-degree for MHL, the order file's for H2H) and tree, without label rows; the
// separator list of each tree node goes to `seps` in tid space for the device row fill.
Index prepare_index(const Graph &g, IndexKind kind, const std::vector<int32_t> *node_order, Separators &seps,
                    int32_t tail_r, const TailEngine &tail) {
  if (kind == IndexKind::H2H) {
    if (!node_order || (int32_t)node_order->size() != g.n) throw Error(QBC_EINVAL, "order has wrong length");
    std::vector<char> seen((size_t)g.n, 0);
    for (int32_t v = 0; v < g.n; v++) {
      int32_t o = (*node_order)[v];
      if (o < 0 || o >= g.n || seen[o]) throw Error(QBC_EINVAL, "order is not a permutation of 0..n-1");
      seen[o] = 1;
    }
  }
  Elimination el;
  {
    TraceScope t("elimination");
    el = eliminate(g, kind == IndexKind::H2H ? node_order : nullptr, std::min(tail_r, g.n), tail);
  }
  Index ix;
  ix.kind = kind;
  TraceScope t("tree and separators");
  make_tree(g, el, ix, false);
  const int32_t n = g.n;
  std::vector<int64_t> xs((size_t)n, 0);
  for (int32_t s = 0; s < n; s++) xs[ix.tid_of[el.order[s]]] = s;
  seps.off.assign((size_t)n + 1, 0);
  for (int32_t t = 0; t < n; t++) seps.off[t + 1] = seps.off[t] + (el.x_off[xs[t] + 1] - el.x_off[xs[t]]);
  seps.ent.assign((size_t)seps.off[n] * 4, 0);
  for (int32_t t = 0; t < n; t++) {
    int64_t o = seps.off[t] * 4;
    for (int64_t i = el.x_off[xs[t]]; i < el.x_off[xs[t] + 1]; i++) {
      const Adj &a = el.x[i];
      seps.ent[o++] = ix.tid_of[a.v];
      seps.ent[o++] = a.len;
      seps.ent[o++] = (int32_t)a.cnt;
      seps.ent[o++] = a.hop;
    }
  }
  return ix;
}

Index build_mhl(const Graph &g, int nthreads) {
  Elimination el = eliminate(g, nullptr);
  Index ix;
  ix.kind = IndexKind::MHL;
  make_tree(g, el, ix);
  const int64_t L = ix.lab_off[g.n];
  ix.dis.assign((size_t)L, 0);
  ix.ch.assign((size_t)L * 2, 0);
  // separator list of each tid: (tid of x_i, len, cnt, hop)
  std::vector<int64_t> xs((size_t)g.n + 1, 0);
  for (int32_t s = 0; s < g.n; s++) xs[ix.tid_of[el.order[s]]] = s;
  fill_rows(ix, hardware_threads(nthreads), [&](int32_t p, auto &&wait) {
    const int32_t h = ix.depth[p];
    int32_t *dis = ix.dis.data() + ix.lab_off[p];
    int32_t *ch = ix.ch.data() + 2 * ix.lab_off[p];
    for (int32_t j = 0; j < h - 1; j++) { dis[j] = kInf; ch[2 * j] = 0; ch[2 * j + 1] = 0; }
    dis[h - 1] = 0;
    ch[2 * (h - 1)] = 1;
    ch[2 * (h - 1) + 1] = 0;
    const int64_t s = xs[p];
    for (int64_t i = el.x_off[s]; i < el.x_off[s + 1]; i++) {
      const Adj &a = el.x[i];
      const int32_t xt = ix.tid_of[a.v];
      wait(xt);
      const int32_t k = ix.depth[xt] - 1;
      const int32_t *xd = ix.dis.data() + ix.lab_off[xt];
      const int32_t *xc = ix.ch.data() + 2 * ix.lab_off[xt];
      for (int32_t j = 0; j <= k; j++) {
        const int32_t nd = a.len + xd[j];
        const uint32_t nc = a.cnt * (uint32_t)xc[2 * j];
        const int32_t nh = a.hop + xc[2 * j + 1];
        if (nd < dis[j]) { dis[j] = nd; ch[2 * j] = (int32_t)nc; ch[2 * j + 1] = nh; }
        else if (nd == dis[j]) {
          ch[2 * j] = (int32_t)((uint32_t)ch[2 * j] + nc);
          if (nh > ch[2 * j + 1]) ch[2 * j + 1] = nh;
        }
      }
    }
  });
  ix.max_label = 0;
  for (int32_t t = 0; t < ix.n; t++)
    for (int32_t j = 0; j < ix.depth[t]; j++) ix.max_label = std::max(ix.max_label, ix.dis[ix.lab_off[t] + j]);
  return ix;
}

Index build_h2h(const Graph &g, const std::vector<int32_t> &node_order, int nthreads) {
  if ((int32_t)node_order.size() != g.n) throw Error(QBC_EINVAL, "order has wrong length");
  {
    std::vector<char> seen((size_t)g.n, 0);
    for (int32_t v = 0; v < g.n; v++) {
      int32_t o = node_order[v];
      if (o < 0 || o >= g.n || seen[o]) throw Error(QBC_EINVAL, "order is not a permutation of 0..n-1");
      seen[o] = 1;
    }
  }
  Elimination el = eliminate(g, &node_order);
  Index ix;
  ix.kind = IndexKind::H2H;
  make_tree(g, el, ix);
  const int64_t L = ix.lab_off[g.n];
  ix.dis.assign((size_t)L, 0);
  std::vector<int64_t> xs((size_t)g.n + 1, 0);
  for (int32_t s = 0; s < g.n; s++) xs[ix.tid_of[el.order[s]]] = s;
  fill_rows(ix, hardware_threads(nthreads), [&](int32_t p, auto &&wait) {
    const int32_t h = ix.depth[p];
    int32_t *dis = ix.dis.data() + ix.lab_off[p];
    std::vector<int32_t> anc((size_t)h);
    for (int32_t a = p, d = h - 1; d >= 0; a = ix.parent[a], d--) anc[d] = a;
    for (int32_t j = 0; j < h - 1; j++) dis[j] = kInf;
    dis[h - 1] = 0;
    const int64_t s = xs[p];
    for (int64_t i = el.x_off[s]; i < el.x_off[s + 1]; i++) wait(ix.tid_of[el.x[i].v]);
    for (int32_t j = 0; j < h - 1; j++) wait(anc[j]);
    // true distance to ancestor j through the separator (H2H, src/buildIndex.cpp:246-270)
    for (int64_t i = el.x_off[s]; i < el.x_off[s + 1]; i++) {
      const Adj &a = el.x[i];
      const int32_t xt = ix.tid_of[a.v];
      const int32_t k = ix.depth[xt] - 1;
      const int32_t *xd = ix.dis.data() + ix.lab_off[xt];
      for (int32_t j = 0; j <= k; j++) {
        int32_t nd = a.len + xd[j];
        if (nd < dis[j]) dis[j] = nd;
      }
      for (int32_t j = k + 1; j < h - 1; j++) {
        int32_t nd = a.len + ix.dis[ix.lab_off[anc[j]] + k];
        if (nd < dis[j]) dis[j] = nd;
      }
    }
  });
  ix.max_label = 0;
  for (int32_t t = 0; t < ix.n; t++)
    for (int32_t j = 0; j < ix.depth[t]; j++) ix.max_label = std::max(ix.max_label, ix.dis[ix.lab_off[t] + j]);
  return ix;
}

// Label-free index (IndexKind::CSR): the per-source rows come from shortest-path sweeps over the
// arc list on the device, so the index is the arc list itself, kept in vertex-id order (tid = vid:
// the file's own numbering, which for road graphs is usually spatially coherent, so a sweep's
// frontier touches nearby rows).  No tree: depth 0, no parent, one-vertex "subtrees", no rows.
// The graph must be connected (every BC path here assumes it, QBC.cu:525).
Index build_csr(const Graph &g) {
  const int32_t n = g.n;
  if (n <= 0) throw Error(QBC_EGRAPH, "empty graph");
  {
    std::vector<int32_t> stack{0};
    std::vector<char> seen((size_t)n, 0);
    seen[0] = 1;
    int32_t reached = 1;
    while (!stack.empty()) {
      const int32_t v = stack.back();
      stack.pop_back();
      for (int32_t e = g.off[v]; e < g.off[v + 1]; e++)
        if (!seen[g.head[e]]) {
          seen[g.head[e]] = 1;
          reached++;
          stack.push_back(g.head[e]);
        }
    }
    if (reached != n)
      throw Error(QBC_EGRAPH, "graph is not connected (" + std::to_string(n - reached) + " vertices unreachable from vertex 1)");
  }
  Index ix;
  ix.kind = IndexKind::CSR;
  ix.n = n;
  ix.vid_of.resize((size_t)n);
  ix.tid_of.resize((size_t)n);
  ix.send.resize((size_t)n);
  for (int32_t v = 0; v < n; v++) {
    ix.vid_of[v] = ix.tid_of[v] = v;
    ix.send[v] = v + 1;
  }
  ix.depth.assign((size_t)n, 0);
  ix.parent.assign((size_t)n, -1);
  ix.lab_off.assign((size_t)n + 1, 0);
  ix.arc_off = g.off;
  ix.arc_head = g.head;
  ix.arc_w = g.w;
  return ix;
}

std::vector<int32_t> min_degree_order(const Graph &g) {
  Elimination el = eliminate(g, nullptr);
  return el.rank;
}

int64_t scan_entries(const Index &ix, const int32_t *sources0, int32_t ns) {
  int64_t total = 0;
  for (int32_t k = 0; k < ns; k++) {
    int32_t s = ix.tid_of[sources0[k]];
    int64_t below = 0;  // targets already attributed to a deeper ancestor
    for (int32_t a = s; a >= 0; a = ix.parent[a]) {
      int64_t size = (int64_t)ix.send[a] - a;
      total += (int64_t)ix.depth[a] * (size - below);
      below = size;
    }
  }
  return total;
}

// Label entries the packed-key scan copies from target rows: sources sorted by tid form CTAs of
// `group` consecutive sources, and a CTA copies each target row t up to the deepest LCA depth of t
// with any of its sources -- the depth of t's deepest ancestor-or-self that lies on some source's
// root path (a preorder pass per group: parent before child).
int64_t group_entries(const Index &ix, const int32_t *sources0, int32_t ns, int32_t group) {
  std::vector<int32_t> tids((size_t)ns);
  for (int32_t k = 0; k < ns; k++) tids[k] = ix.tid_of[sources0[k]];
  std::sort(tids.begin(), tids.end());
  std::vector<int32_t> mark((size_t)ix.n, -1), best((size_t)ix.n, 0);
  int64_t total = 0;
  for (int32_t g0 = 0; g0 < ns; g0 += group) {
    for (int32_t k = g0; k < std::min(ns, g0 + group); k++)
      for (int32_t a = tids[k]; a >= 0 && mark[a] != g0; a = ix.parent[a]) mark[a] = g0;
    for (int32_t t = 0; t < ix.n; t++) {
      best[t] = mark[t] == g0 ? ix.depth[t] : (ix.parent[t] >= 0 ? best[ix.parent[t]] : 0);
      total += best[t];
    }
  }
  return total;
}

}  // namespace qbc
