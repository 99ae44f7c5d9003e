// ref_harness.cu -- runs the reference's own GPU drivers and dumps full-precision results.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles the unmodified reference .cu file with
// -Dmain=ref_main and links it with this harness into oracle/_ref/ref_{mhlqbc,qbc,rq}.  The
// reference CLIs print BC with %.2f (MHLQBC.cu:570, QBC.cu:617) or %.8f (RQ.cu:583); this
// harness calls the same Graph methods and writes %.17g instead, plus wall times of the
// CPU index build alone and of the whole driver call (index build + GPU), so that the GPU
// share can be read as the difference.
//
//   ref_mhlqbc <graph> <out>            Graph::brandesBCIndexGPU_5   (MHLQBC.cu:495)
//   ref_qbc    <graph> <order> <out>    Graph::brandesBCIndexGPU_5   (QBC.cu:419)
//   ref_rq     <graph> <query> <out>    Graph::brandesBCIndexGPU_PointBatch (RQ.cu:465)
#include "include/Graph.h"

#include <chrono>
#include <cstdio>

extern string roadDataPath;
#if defined(REF_QBC)
extern string orderFile;
#endif
#if defined(REF_RQ)
extern string queryBatchPath;
void processBactch(int nodenum, int &batckSize, vector<int> &randNumber);
#endif

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int main(int argc, char **argv) {
#if defined(REF_MHL)
  if (argc < 3) { fprintf(stderr, "usage: %s graph out\n", argv[0]); return 2; }
  const char *out_path = argv[2];
#else
  if (argc < 4) { fprintf(stderr, "usage: %s graph order|query out\n", argv[0]); return 2; }
  const char *out_path = argv[3];
#endif
  roadDataPath = argv[1];
  cudaSetDevice(0);
  Graph g;
  g.ReadGraph(roadDataPath);
  double t_idx = 0.0, t0, t1;
#if defined(REF_MHL) || defined(REF_RQ)
  {
    t0 = now_s();
    TreeDecomp td(roadDataPath.c_str(), "tmpRoadCountIndex_probe");
    td.Reduce();
    td.MakeTree();
    td.MakeIndex();
    t_idx = now_s() - t0;
  }
#endif
  FILE *f = fopen(out_path, "w");
  if (!f) { fprintf(stderr, "cannot open %s\n", out_path); return 2; }
#if defined(REF_MHL)
  t0 = now_s();
  g.brandesBCIndexGPU_5(roadDataPath);
  t1 = now_s();
  for (int i = 0; i < g.nodenum; i++) fprintf(f, "%d %.17g\n", i + 1, g.BC[i]);
#elif defined(REF_QBC)
  orderFile = argv[2];
  {
    Graph g2;
    g2.ReadGraph(roadDataPath);
    t0 = now_s();
    g2.CHconsorderMT(orderFile);
    g2.makeTree();
    g2.makeIndex();
    g2.optimizeVS();
    vector<int> ress;
    g2.SVSP_P2H(10, 5, 1000000, ress);
    t_idx = now_s() - t0;
  }
  t0 = now_s();
  g.brandesBCIndexGPU_5(roadDataPath);
  t1 = now_s();
  for (int i = 0; i < g.nodenum; i++) fprintf(f, "%d %.17g\n", i + 1, g.BC[i]);
#elif defined(REF_RQ)
  queryBatchPath = argv[2];
  int topk;
  vector<int> pts;
  processBactch(g.nodenum, topk, pts);
  if (topk >= g.nodenum) topk = g.nodenum;
  t0 = now_s();
  g.brandesBCIndexGPU_PointBatch(roadDataPath, pts, topk);
  t1 = now_s();
  for (int i = 0; i < topk; i++) fprintf(f, "%d %.17g\n", pts[i] + 1, g.h_PointBC[i]);
#endif
  fclose(f);
  cudaError_t err = cudaGetLastError();
  printf("{\"n\": %d, \"arcs\": %d, \"index_s\": %.6f, \"total_s\": %.6f, \"cuda\": \"%s\"}\n", g.nodenum,
         g.edgenum, t_idx, t1 - t0, cudaGetErrorString(err));
  return err == cudaSuccess ? 0 : 1;
}
