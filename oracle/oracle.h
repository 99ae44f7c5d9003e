/*
 * oracle.h -- CPU restatement of the reference's betweenness-centrality hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: tests/, the smoke check in
 * __graft_entry__.py and the cpu_baseline / --impl reference legs of bench.py may load it.
 * The product (gpu_betweennesscentrality_b200) never links, loads or calls it.
 *
 * Every function restates a reference routine (paths relative to the reference project):
 *   orc_arcs_build     src/Graph.cpp:4-37             Graph::ReadGraph (0-based arcs, first duplicate kept, w 0 -> 1)
 *   orc_tc_build       src/TreeCount/Graph.cpp:41-81  Graph_::ReadWeightedGraph (symmetrised, min weight)
 *                      src/TreeCount/TreeDecomp.cpp:12-52   TreeDecomp ctor (count 1, hop 1 per edge)
 *                      src/TreeCount/TreeDecomp.cpp:54-208  Reduce (min-degree elimination, count/hop shortcuts)
 *                      src/TreeCount/TreeDecomp.cpp:210-238 MakeTree, :630-664 GetParentNode
 *                      src/TreeCount/TreeDecomp.cpp:248-257,324-345 EulerTour / MakeRMQIndex
 *                      src/TreeCount/TreeDecomp.cpp:355-511 makeIndexDFS / MakeCountIndex (dis/cnt/my_cnt labels)
 *   orc_mhl_rows       MHLQBC.cu:302-412   LCA + dist/count/hop row of one source
 *   orc_mhl_bc         MHLQBC.cu:237-494   full per-source loop (SP-DAG, layers, backprop, 0.5*delta)
 *   orc_h2h_build      src/buildIndex.cpp:4-111 CHconsorderMT, :151-207 makeTree/match,
 *                      :208-310 makeIndex/makeRMQ (H2H distance labels), :313-386 optimizeVS
 *   orc_qbc_dist       QBC.cu:243-331      LCA + H2H distance row (posOptimize scan; P2H branch not restated)
 *   orc_qbc_bc         QBC.cu:335-400,485-555  SP-DAG, host Kahn sigma/layers, backprop
 *   orc_rq_bc          RQ.cu:201-291,307-463,513-521  per-pair dependency test of a query set
 *   orc_brandes_bc     independent Dijkstra-Brandes witness (int32-wrapping sigma, same FP64 step)
 *
 * Integer semantics follow the reference: distances int32, path counts uint32 bits that wrap
 * (the reference stores them in int), hop counts int32, BC in FP64.
 */
#ifndef QBC_ORACLE_H
#define QBC_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Directed arc list as Graph::ReadGraph keeps it (src/Graph.cpp:22-36). */
typedef struct orc_arcs {
  int n, m;      /* vertices (0-based ids), arcs kept */
  int *off;      /* n+1 CSR offsets; arcs of a tail stay in file order */
  int *head;     /* m */
  int *w;        /* m */
} orc_arcs;

/* TreeCount index (TreeDecomp after Reduce/MakeTree/MakeIndex). Arrays are indexed by tree
 * position p (rank_[vid] = p) unless stated; vertex ids are 1-based as in TreeDecomp. */
typedef struct orc_tc {
  int n;
  int tree_width, tree_height;
  int *del_order;          /* n   delete_vertex_order_ */
  int *rank;               /* n+1 vid -> tree position */
  int *vertex;             /* n   tree position -> vid */
  int *parent, *height;    /* n */
  int *child_off, *child;  /* children per tree position, in insertion order */
  int64_t *nb_off;         /* n+1 separator (vertices/vertices_length/edge_count_/my_edge_count_) */
  int *nb, *nb_len;
  uint32_t *nb_cnt, *nb_hop;
  int64_t *pos_off;        /* n+1 pos lists (|X|+1 entries, last = own position) */
  int *pos;
  int64_t *lab_off;        /* n+1 labels: height-1 entries (one per ancestor) */
  int *dis;
  uint32_t *cnt, *hop;
  int euler_len, rmq_levels;
  int *euler_pos;          /* n   tree position -> first Euler index */
  int *rmq;                /* rmq_levels * euler_len */
} orc_tc;

/* H2H index of QBC (buildIndex.cpp). Indexed by tree position; vertex ids 0-based. */
typedef struct orc_h2h {
  int n;
  int *rank, *uvertex, *parent, *height;
  int *child_off, *child;
  int64_t *vert_off;       /* NeighborCon per tree position */
  int *vert, *vert_w;
  int64_t *pos_off;
  int *pos;
  int64_t *dis_off;
  int *dis;
  int64_t *popt_off;       /* posOptimize */
  int *popt;
  int euler_len, rmq_levels;
  int *to_rmq;
  int *rmq;
} orc_h2h;

/* ---- construction ---- */
int  orc_arcs_build(int n, int m_lines, const int *u1, const int *v1, const int *w, orc_arcs **out);
void orc_arcs_free(orc_arcs *g);
int  orc_tc_build(int n, int m_lines, const int *u1, const int *v1, const int *w, orc_tc **out);
void orc_tc_free(orc_tc *tc);
/* node_order[vid] = contraction order (order-file semantics, buildIndex.cpp:13-20) */
int  orc_h2h_build(const orc_arcs *g, const int *node_order, orc_h2h **out);
void orc_h2h_free(orc_h2h *h);

/* ---- per-source rows ---- */
/* dist/count/hop of 0-based source to every 0-based vid (MHLQBC.cu:302-412). */
int orc_mhl_rows(const orc_tc *tc, int source, int *dist, uint32_t *cnt, int *hop);
/* H2H distance row (QBC.cu:243-331 without the P2H branch). */
int orc_qbc_dist(const orc_h2h *h, int source, int *dist);

/* ---- BC ----
 * bc_out (n doubles) receives sum over the listed sources of 0.5*delta_s(v).
 * sources == NULL means all n sources.  nthreads <= 0 uses every OpenMP thread. */
int orc_mhl_bc(const orc_tc *tc, const orc_arcs *g, const int *sources, int ns, double *bc_out, int nthreads);
int orc_qbc_bc(const orc_h2h *h, const orc_arcs *g, const int *sources, int ns, double *bc_out, int nthreads);
/* RQ pair formula; points are 0-based vids; out has q doubles. O(n^2 q): small graphs only. */
int orc_rq_bc(const orc_tc *tc, const int *points, int q, double *out, int nthreads);
/* Independent witness: Dijkstra + Brandes on the arc list. */
int orc_brandes_bc(const orc_arcs *g, const int *sources, int ns, double *bc_out, int nthreads);
/* Dijkstra row (dist, wrapping path count, max hop over shortest paths). */
int orc_dijkstra_rows(const orc_arcs *g, int source, int *dist, uint32_t *cnt, int *hop);

#ifdef __cplusplus
}
#endif
#endif
