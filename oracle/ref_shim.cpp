// ref_shim.cpp -- exports the reference's own CPU index structures as plain arrays.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with the
// reference's unmodified CPU sources (src/TreeCount/TreeDecomp.cpp, src/TreeCount/Graph.cpp,
// src/Graph.cpp, src/buildIndex.cpp) into oracle/_ref/libref_cpu.so.  The tests use it to pin
// the C restatement in oracle.c; nothing in the product loads it.
#include "include/Graph.h"

#include <cstdint>
#include <cstdio>

extern "C" {

// TreeDecomp pipeline as the drivers run it (MHLQBC.cu:497-501, RQ.cu:470-474).
void *ref_tc_new(const char *graph_path, const char *index_dump_path) {
  TreeDecomp *td = new TreeDecomp(graph_path, index_dump_path);
  td->Reduce();
  td->MakeTree();
  td->MakeIndex();
  fflush(td->fout_);
  return td;
}

void ref_tc_free(void *h) { delete static_cast<TreeDecomp *>(h); }

// sizes[0]=n, [1]=label entries, [2]=pos entries, [3]=tree width, [4]=tree height,
// [5]=euler length, [6]=rmq levels
void ref_tc_sizes(void *h, int64_t *sizes) {
  TreeDecomp *td = static_cast<TreeDecomp *>(h);
  int64_t lab = 0, pos = 0;
  for (auto &nd : td->tree_) {
    lab += (int64_t)nd.dis.size();
    pos += (int64_t)nd.pos.size();
  }
  sizes[0] = td->G_.n();
  sizes[1] = lab;
  sizes[2] = pos;
  sizes[3] = td->tree_width_;
  sizes[4] = td->tree_height_;
  sizes[5] = (int64_t)td->euler_tour_.size();
  sizes[6] = (int64_t)td->rmq_index_.size();
}

void ref_tc_export(void *h, int *del_order, int *rank, int *parent, int *height, int64_t *lab_off, int *dis,
                   uint32_t *cnt, uint32_t *hop, int64_t *pos_off, int *pos, int *euler_pos) {
  TreeDecomp *td = static_cast<TreeDecomp *>(h);
  const int n = td->G_.n();
  for (int i = 0; i < n; i++) del_order[i] = td->delete_vertex_order_[i];
  for (int i = 0; i <= n; i++) rank[i] = (i == 0) ? -1 : td->rank_[i];
  int64_t lo = 0, po = 0;
  for (int p = 0; p < n; p++) {
    const Node_ &nd = td->tree_[p];
    parent[p] = nd.parent;
    height[p] = nd.height;
    euler_pos[p] = td->euler_tour_pos_[p];
    lab_off[p] = lo;
    pos_off[p] = po;
    for (size_t j = 0; j < nd.dis.size(); j++) {
      dis[lo + j] = nd.dis[j];
      cnt[lo + j] = nd.cnt[j];
      hop[lo + j] = nd.my_cnt[j];
    }
    for (size_t j = 0; j < nd.pos.size(); j++) pos[po + j] = nd.pos[j];
    lo += (int64_t)nd.dis.size();
    po += (int64_t)nd.pos.size();
  }
  lab_off[n] = lo;
  pos_off[n] = po;
}

// TreeDecomp::DistanceCountQuery (TreeDecomp.cpp:568-628): separator-only scan; returns the
// max-hop count and writes the path count.  1-based vids.
int ref_tc_count_hop(void *h, int p, int q, uint32_t *count) {
  TreeDecomp *td = static_cast<TreeDecomp *>(h);
  count_t c = 0;
  int hop = td->DistanceCountQuery(p, q, c);
  *count = c;
  return hop;
}

// H2H pipeline of QBC (QBC.cu:421-429) without the time-seeded P2H step.
void *ref_h2h_new(const char *graph_path, const char *order_path) {
  Graph *g = new Graph();
  g->ReadGraph(graph_path);
  g->CHconsorderMT(order_path);
  g->makeTree();
  g->makeIndex();
  g->optimizeVS();
  return g;
}

void ref_h2h_free(void *h) { delete static_cast<Graph *>(h); }

// sizes[0]=n, [1]=dis entries, [2]=posOptimize entries, [3]=height max
void ref_h2h_sizes(void *h, int64_t *sizes) {
  Graph *g = static_cast<Graph *>(h);
  int64_t d = 0, po = 0;
  for (auto &nd : g->Tree) {
    d += (int64_t)nd.dis.size();
    po += (int64_t)nd.posOptimize.size();
  }
  sizes[0] = g->nodenum;
  sizes[1] = d;
  sizes[2] = po;
  sizes[3] = g->heightMax;
}

void ref_h2h_export(void *h, int *rank, int *uvertex, int *parent, int *height, int64_t *dis_off, int *dis,
                    int64_t *popt_off, int *popt) {
  Graph *g = static_cast<Graph *>(h);
  const int n = g->nodenum;
  for (int v = 0; v < n; v++) rank[v] = g->rank[v];
  int64_t d = 0, po = 0;
  for (int p = 0; p < n; p++) {
    const Node &nd = g->Tree[p];
    uvertex[p] = nd.uniqueVertex;
    parent[p] = nd.pa;
    height[p] = nd.height;
    dis_off[p] = d;
    popt_off[p] = po;
    for (size_t j = 0; j < nd.dis.size(); j++) dis[d + j] = nd.dis[j];
    for (size_t j = 0; j < nd.posOptimize.size(); j++) popt[po + j] = nd.posOptimize[j];
    d += (int64_t)nd.dis.size();
    po += (int64_t)nd.posOptimize.size();
  }
  dis_off[n] = d;
  popt_off[n] = po;
}

}  // extern "C"
