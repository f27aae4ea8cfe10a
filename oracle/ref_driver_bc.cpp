// ref_driver_bc.cpp -- drives the reference's own CPU betweenness centrality.
//
// TEST INFRASTRUCTURE ONLY (the checker of the BC path).  Built by oracle/Makefile
// together with the reference's unmodified sources, compiled where they lie:
//   apps/bc/src/cpu/bc.cpp    bc_cpu() and, through its #include, bc_kernel.cpp;
//                             its main() renamed by -Dmain=...
//   common/global.cpp         graph / noNodeTotal / noEdgeTotal / source / bc globals
// The output goes to oracle/_ref/libref_bc.so only; nothing is copied.
#include <omp.h>

#include <chrono>
#include <cstdint>
#include <cstring>

#include "global.h"

void bc_cpu();  // apps/bc/src/cpu/bc.cpp:152
extern int* sigma;
extern float* delta;
extern char* p;
extern int* p_idx;
extern int* p_data;

// bc_cpu() over every vertex as source, on one OpenMP thread: its loop over
// sources shares the level, sigma, delta and p arrays, so it is only well
// defined on one thread.  It keeps an n x n byte matrix, so n must be small.
// Returns the seconds bc_cpu() took; bc_out[n] receives the centralities.
extern "C" double nps_ref_bc_cpu(int32_t n, int32_t m, const int32_t* row, const int32_t* col, float* bc_out) {
  const _GRAPH_ saved = graph;
  const int sn = noNodeTotal, sm = noEdgeTotal;
  graph.vertexArray = const_cast<int*>(row);
  graph.edgeArray = const_cast<int*>(col);
  graph.levelArray = new int[n]();
  graph.frontier = new char[n]();
  graph.update = new char[n]();
  noNodeTotal = n;
  noEdgeTotal = m;
  omp_set_dynamic(0);
  omp_set_num_threads(1);
  const auto t0 = std::chrono::steady_clock::now();
  bc_cpu();
  const auto t1 = std::chrono::steady_clock::now();
  memcpy(bc_out, bc, sizeof(float) * (size_t)n);
  delete[] bc;
  delete[] delta;
  delete[] sigma;
  delete[] p;
  delete[] p_idx;
  delete[] p_data;
  delete[] graph.levelArray;
  delete[] graph.frontier;
  delete[] graph.update;
  graph = saved;
  noNodeTotal = sn;
  noEdgeTotal = sm;
  return std::chrono::duration<double>(t1 - t0).count();
}
