// host.h -- host-side types of libqbc_b200: graph, tree-decomposition index, errors.
#pragma once

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

namespace qbc {

// Wall-clock time of a scope on stderr ("qbc: <name> <ms> ms") when the environment variable
// QBC_TRACE is set and not "0": the phases of an index build (elimination, dense tail, tree, row
// fill, scratch) for a user sizing a deployment.  Phases that enqueue device work end with a
// synchronisation, so their times include it.
struct TraceScope {
  explicit TraceScope(const char *name) : name_(name) {
    if (enabled()) t0_ = std::chrono::steady_clock::now(), on_ = true;
  }
  ~TraceScope() {
    if (on_)
      std::fprintf(stderr, "qbc: %s %.1f ms\n", name_,
                   std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0_).count());
  }
  TraceScope(const TraceScope &) = delete;
  TraceScope &operator=(const TraceScope &) = delete;
  static bool enabled() {
    static const bool on = [] {
      const char *e = std::getenv("QBC_TRACE");
      return e && *e && std::string(e) != "0";
    }();
    return on;
  }

 private:
  const char *name_;
  std::chrono::steady_clock::time_point t0_{};
  bool on_ = false;
};

constexpr int32_t kInf = 999999999;  // TreeDecomp INF (src/TreeCount/TreeDecomp.h:58)

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// Arc list as Graph::ReadGraph keeps it (src/Graph.cpp:22-36): 0-based, first duplicate kept,
// weight 0 read as 1, arcs of each tail in file order.
struct Graph {
  int32_t n = 0;
  std::vector<int32_t> off;   // n+1
  std::vector<int32_t> head;  // arcs
  std::vector<int32_t> w;     // arcs
  int32_t arcs() const { return (int32_t)head.size(); }
};

// Builds the arc list from raw file lines and validates it (symmetric, simple, weights >= 1,
// bounded total weight).  Connectivity is checked by the index builder.
Graph graph_from_lines(int32_t n, int64_t m, const int32_t *u1, const int32_t *v1, const int32_t *w);
Graph graph_read(const std::string &path);
std::vector<int32_t> read_order(const std::string &path, int32_t n);
std::vector<int32_t> read_query(const std::string &path, int32_t n);

// MHL: TreeCount distance + count + hop labels; H2H: distance labels from an order file; CSR: no
// labels (graphs whose tree decomposition is too wide), the per-source rows come from
// shortest-path sweeps over the arc list.
enum class IndexKind : int { MHL = 0, H2H = 1, CSR = 2 };

// Tree-decomposition index in DFS-preorder numbering ("tid").  Row p holds one entry per
// ancestor, root first, plus the node itself last (dis 0, cnt 1, hop 0); rows start on 4-entry
// boundaries so 16-byte vector loads stay aligned.
struct Index {
  IndexKind kind = IndexKind::MHL;
  int32_t n = 0;
  int32_t tree_height = 0, tree_width = 0;
  std::vector<int32_t> vid_of;   // tid -> 0-based vid
  std::vector<int32_t> tid_of;   // vid -> tid
  std::vector<int32_t> depth;    // tid -> depth (root 1) = row length
  std::vector<int32_t> parent;   // tid -> parent tid (-1 root)
  std::vector<int32_t> send;     // tid -> tid + subtree size (ancestor test a <= t < send[a])
  std::vector<int64_t> lab_off;  // n+1, entry offsets (multiples of 4)
  std::vector<int32_t> dis;      // lab_off[n]
  std::vector<int32_t> ch;       // 2*lab_off[n]: (cnt bits, hop) pairs; MHL only
  std::vector<int32_t> anc;      // lab_off[n]: tid of the ancestor each row entry refers to
  std::vector<int32_t> aend;     // lab_off[n]: subtree end (send) of that ancestor
  int32_t max_label = 0;         // largest label distance (decides the packed-key scan)
  // arcs in tid space, each tail's arcs in file order
  std::vector<int32_t> arc_off, arc_head, arc_w;
  int64_t depth_sum = 0;
  bool rows_on_host = true;  // false: label rows (dis/ch/anc/aend) exist only on the device
};

// Separator lists in tid space, for the device row fill: node t's entries are
// ent[4*off[t] .. 4*off[t+1]), each (tid of x, shortcut length, path count bits, max hop), in
// elimination order of the separator.
struct Separators {
  std::vector<int64_t> off;
  std::vector<int32_t> ent;
};
// The last r vertices of a min-degree elimination, handed to another engine (the device's dense
// elimination, device_dense_eliminate): the vertices still present, ascending (local id = index),
// with their current adjacency in local ids.  The engine returns the rest of the elimination: the
// local ids in elimination order (minimum current degree, smaller id first, as the host) and each
// step's separator, (local column, shortcut length, path count bits, max hop) per entry.
struct DenseTail {
  int32_t r = 0;
  std::vector<int32_t> ids;  // global vertex ids, ascending
  std::vector<int64_t> off;  // r + 1: vertex i's entries are ent[4*off[i] .. 4*off[i+1])
  std::vector<int32_t> ent;  // (local column, length, count bits, max hop)
  std::vector<int32_t> order;  // result: local ids in elimination order
  std::vector<int64_t> x_off;  // result: r + 1
  std::vector<int32_t> x;      // result: separator entries as in `ent`
};
using TailEngine = std::function<void(DenseTail &)>;

// Elimination and tree only (no label rows: dis/ch/anc/aend stay empty); max_label is unknown (0).
// With `tail` (min-degree elimination only), the last `tail_r` vertices are eliminated by it.
Index prepare_index(const Graph &g, IndexKind kind, const std::vector<int32_t> *node_order, Separators &seps,
                    int32_t tail_r = 0, const TailEngine &tail = {});

// Per-entry ancestor ids (anc) and their subtree ends (aend) of every row, from the tree links
// (a row is its parent's row plus the node itself).
void fill_ancestor_rows(Index &ix);
// TreeCount-equivalent index (distance + count + max hop) by min-degree elimination.
Index build_mhl(const Graph &g, int nthreads);
// H2H distance index from an order file (node_order[vid] = contraction rank).
Index build_h2h(const Graph &g, const std::vector<int32_t> &node_order, int nthreads);
// Label-free index: the arc list in vertex-id order (tid = vid), connectivity checked, no tree.
Index build_csr(const Graph &g);
// Min-degree contraction order (node_order[vid] = rank).
std::vector<int32_t> min_degree_order(const Graph &g);

// sum over targets of h(lca(s, t)) for each listed source (0-based vids)
int64_t scan_entries(const Index &ix, const int32_t *sources0, int32_t ns);
// label entries the packed-key scan copies from target rows for CTAs of `group` consecutive
// sources (tid order): sum over groups and targets of the deepest LCA depth within the group
int64_t group_entries(const Index &ix, const int32_t *sources0, int32_t ns, int32_t group);

int hardware_threads(int requested);

// On-disk index (index_file.cpp): the host index, rows included, with a header and a checksum.
void index_save(const Index &ix, const std::string &path);
Index index_load(const std::string &path);

}  // namespace qbc
