// qbc_graph.hpp -- C++ host-side mirror of the reference's `Graph` driver API over the C ABI.
//
// The reference's drivers are methods of `class Graph` (include/Graph.h:64-200):
//   ReadGraph(path)                                  src/Graph.cpp:4
//   brandesBCIndexGPU_5(roadName)        -> BC       MHLQBC.cu:495 (TreeCount index) / QBC.cu:419 (H2H + order file)
//   brandesBCIndexGPU_PointBatch(roadName, points, querySize) -> h_PointBC   RQ.cu:465
// This header keeps those names, argument meanings and result members; the work goes through
// libqbc_b200 (include/qbc_b200.h).  The reference reads the graph/order paths from globals
// (roadDataPath, orderFile); here they are arguments.  Failures throw std::runtime_error with the
// library's message instead of continuing silently.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "qbc_b200.h"

namespace qbc_b200 {

inline void check(int rc) {
  if (rc != QBC_OK) throw std::runtime_error(std::string("qbc: ") + qbc_last_error());
}

class Graph {
 public:
  int nodenum = 0;
  int edgenum = 0;          // arcs kept by the reader
  int device = 0;           // cudaSetDevice target (QBC.cu:601-602)
  int nthreads = 0;         // kept for source compatibility; the elimination uses all host threads
  std::vector<double> BC;         // include/Graph.h:71
  std::vector<double> h_PointBC;  // include/Graph.h:198

  Graph() = default;
  Graph(const Graph &) = delete;
  Graph &operator=(const Graph &) = delete;
  ~Graph() {
    if (idx_) qbc_index_free(idx_);
    if (g_) qbc_graph_free(g_);
  }

  void ReadGraph(const std::string &graphname) {
    if (g_) { qbc_graph_free(g_); g_ = nullptr; }
    check(qbc_graph_read(graphname.c_str(), &g_));
    check(qbc_graph_info(g_, &nodenum, &edgenum));
  }

  // MHL-QBC: TreeCount-style index, all-vertex BC.
  void brandesBCIndexGPU_5(const std::string & /*roadName*/) {
    build(QBC_INDEX_MHL, nullptr);
    BC.assign((size_t)nodenum, 0.0);
    check(qbc_bc_all(idx_, BC.data()));
  }

  // QBC: H2H index from an order file, all-vertex BC.
  void brandesBCIndexGPU_5(const std::string & /*roadName*/, const std::string &orderFile) {
    std::vector<int32_t> order((size_t)nodenum);
    check(qbc_read_order(orderFile.c_str(), nodenum, order.data()));
    build(QBC_INDEX_H2H, order.data());
    BC.assign((size_t)nodenum, 0.0);
    check(qbc_bc_all(idx_, BC.data()));
  }

  // RQ: BC of the query vertices (0-based ids).
  void brandesBCIndexGPU_PointBatch(const std::string & /*roadName*/, std::vector<int> &points, const int querySize) {
    if (querySize < 0 || (size_t)querySize > points.size()) throw std::runtime_error("qbc: querySize out of range");
    build(QBC_INDEX_MHL, nullptr);
    h_PointBC.assign((size_t)querySize, 0.0);
    std::vector<int32_t> p(points.begin(), points.begin() + querySize);
    check(qbc_bc_query(idx_, p.data(), querySize, h_PointBC.data()));
  }

  qbc_index *index() { return idx_; }
  qbc_graph *graph() { return g_; }

 private:
  qbc_graph *g_ = nullptr;
  qbc_index *idx_ = nullptr;

  void build(int kind, const int32_t *order) {
    if (!g_) throw std::runtime_error("qbc: ReadGraph first");
    if (idx_) { qbc_index_free(idx_); idx_ = nullptr; }
    // elimination on the host, label rows filled on the GPU (qbc_index_build_device)
    check(qbc_index_build_device(g_, kind, order, device, &idx_));
  }
};

}  // namespace qbc_b200
