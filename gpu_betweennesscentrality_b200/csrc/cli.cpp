// cli.cpp -- drop-in command lines of the reference, built three times (QBC_CLI_MHL / _QBC / _RQ):
//
//   MHLQBC <graph> <device> [out]                  MHLQBC.cu:547-579
//   QBC    <graph> <order> <device> [out [stdBC]]  QBC.cu:593-647
//   RQ     <graph> <queryBatch> <device>           RQ.cu:542-587, batch reader RQ.cu:589-610
//
// Same positional arguments, stdout lines and output files ("vertexID  BCValue", 1-based ids,
// %.2f; RQ's table with %.8f).  QBC_OUTPUT_DIGITS=17 in the environment switches the BC file to
// %.17g for full-precision comparisons.  Errors go to stderr with exit status 1.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/qbc_graph.hpp"

using std::cout;
using std::endl;
using std::string;

static void write_bc(const string &path, const std::vector<double> &bc) {
  FILE *f = fopen(path.c_str(), "w");
  if (!f) throw std::runtime_error("cannot open " + path);
  const char *dg = getenv("QBC_OUTPUT_DIGITS");
  const bool full = dg && atoi(dg) >= 17;
  fprintf(f, "vertexID  BCValue\n");
  for (size_t i = 0; i < bc.size(); i++) {
    if (full) fprintf(f, "%zu %.17g\n", i + 1, bc[i]);
    else fprintf(f, "%zu %.2f\n", i + 1, bc[i]);
  }
  fclose(f);
  cout << "The BC value has been save: " << path << endl;
}

int main(int argc, char **argv) {
  cout.precision(8);
  cout << std::fixed;
  try {
#if defined(QBC_CLI_MHL)
    if (argc < 3) { fprintf(stderr, "usage: %s <graph> <device> [out]\n", argv[0]); return 2; }
    const string road = argv[1];
    qbc_b200::Graph g;
    g.device = std::stoi(argv[2]);
    g.ReadGraph(road);
    cout << "roadDataPath:" << road << "\t" << g.nodenum << "\t" << g.edgenum << "\n";
    auto t1 = std::chrono::high_resolution_clock::now();
    g.brandesBCIndexGPU_5(road);
    auto t2 = std::chrono::high_resolution_clock::now();
    cout << std::chrono::duration<double>(t2 - t1).count() << "  seconds (---totalTime---)" << endl;
    if (argc >= 4) write_bc(argv[3], g.BC);
#elif defined(QBC_CLI_QBC)
    if (argc < 4) { fprintf(stderr, "usage: %s <graph> <order> <device> [out [stdBC]]\n", argv[0]); return 2; }
    const string road = argv[1], order = argv[2];
    qbc_b200::Graph g;
    g.device = std::stoi(argv[3]);
    g.ReadGraph(road);
    cout << "roadDataPath:" << road << "\t" << g.nodenum << "\t" << g.edgenum << "\n";
    auto t1 = std::chrono::high_resolution_clock::now();
    g.brandesBCIndexGPU_5(road, order);
    auto t2 = std::chrono::high_resolution_clock::now();
    cout << std::chrono::duration<double>(t2 - t1).count() << "  seconds (---totalTime---)" << endl;
    if (argc >= 5) write_bc(argv[4], g.BC);
    if (argc >= 6) {  // standard-BC self-check (QBC.cu:628-647): 1e-1 absolute, or QBC_STD_TOL
      double tol = 1e-1;
      if (const char *e = std::getenv("QBC_STD_TOL")) tol = std::atof(e);
      std::ifstream ifs(argv[5]);
      if (!ifs) throw std::runtime_error(string("cannot open ") + argv[5]);
      int nn, mm, vid;
      double v;
      ifs >> nn >> mm;
      std::vector<double> stdbc((size_t)std::max(nn, 0), 0.0);
      while (ifs >> vid >> v)
        if (vid >= 1 && vid <= nn) stdbc[vid - 1] = v;
      for (int i = 0; i < g.nodenum && i < nn; i++) {
        if (std::fabs(g.BC[i] - stdbc[i]) > tol) {
          cout << "BC value is not correct for node " << i << "\t" << g.BC[i] << "\t" << stdbc[i] << endl;
          return 1;
        }
      }
      cout << "BC value is correct\n\n" << endl;
    }
#elif defined(QBC_CLI_RQ)
    if (argc < 4) { fprintf(stderr, "usage: %s <graph> <queryBatch> <device>\n", argv[0]); return 2; }
    const string road = argv[1], qpath = argv[2];
    qbc_b200::Graph g;
    g.device = std::stoi(argv[3]);
    g.ReadGraph(road);
    cout << "roadName:" << road << "\t" << g.nodenum << "\t" << g.edgenum << "\n";
    int32_t q = 0;
    qbc_b200::check(qbc_read_query(qpath.c_str(), g.nodenum, 0, &q, nullptr));
    std::vector<int32_t> ids((size_t)q);
    qbc_b200::check(qbc_read_query(qpath.c_str(), g.nodenum, q, &q, ids.data()));
    cout << "The number of vertices to query: " << q << endl;
    int topk = q < g.nodenum ? q : g.nodenum;
    std::vector<int> pts(ids.begin(), ids.end());
    auto t1 = std::chrono::high_resolution_clock::now();
    g.brandesBCIndexGPU_PointBatch(road, pts, topk);
    auto t2 = std::chrono::high_resolution_clock::now();
    cout << std::chrono::duration<double>(t2 - t1).count() << "  seconds (---totalTime---)" << endl;
    cout << std::left << endl;
    cout << std::setw(10) << "vertexID" << std::setw(10) << "BCValue" << endl;
    cout << string(20, '-') << endl;
    for (int i = 0; i < topk; ++i) cout << std::setw(10) << (pts[i] + 1) << std::setw(10) << g.h_PointBC[i] << endl;
    cout << endl;
#endif
  } catch (const std::exception &e) {
    fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
