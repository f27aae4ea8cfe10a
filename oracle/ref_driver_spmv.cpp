// ref_driver_spmv.cpp -- drives the reference's own CPU SpMV from plain arrays.
//
// TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline of the SpMV
// workload).  Built by oracle/Makefile together with the reference's unmodified
// sources, compiled where they lie:
//   apps/SpMV/src/cpu/SpMV.cpp         data / x / y globals, its main() renamed by -Dmain=...
//   apps/SpMV/src/cpu/SpMV_kernel.cpp  prepare_cpu() (the data and x it multiplies),
//                                      spmv_omp() (the OpenMP row loop), clean_cpu()
//   common/global.cpp                  graph / noNodeTotal / noEdgeTotal globals
// The output goes to oracle/_ref/libref_spmv.so only; nothing is copied.
#include <omp.h>

#include <chrono>
#include <cstdint>
#include <cstring>

#include "SpMV.h"

void prepare_cpu();  // apps/SpMV/src/cpu/SpMV_kernel.cpp:4
void spmv_omp();     // apps/SpMV/src/cpu/SpMV_kernel.cpp:26
void clean_cpu();    // apps/SpMV/src/cpu/SpMV_kernel.cpp:19

// y = A x as SpMV_CPU() computes it (SpMV_kernel.cpp:45-61): prepare_cpu() fills
// the values and x, spmv_omp() runs with `threads` OpenMP threads (0 = the
// default).  Copies y, and x and the values when asked, then frees them as
// clean_cpu() does.  Returns the seconds spmv_omp() took.
extern "C" double nps_ref_spmv_cpu(int32_t n, int32_t m, const int32_t* row, const int32_t* col, int32_t threads,
                                   double* y_out, double* x_out, double* val_out) {
  const _GRAPH_ saved = graph;
  const int sn = noNodeTotal, sm = noEdgeTotal;
  graph.vertexArray = const_cast<int*>(row);
  graph.edgeArray = const_cast<int*>(col);
  noNodeTotal = n;
  noEdgeTotal = m;
  prepare_cpu();
  if (threads > 0) omp_set_num_threads(threads);
  const auto t0 = std::chrono::steady_clock::now();
  spmv_omp();
  const auto t1 = std::chrono::steady_clock::now();
  if (y_out) memcpy(y_out, y, sizeof(double) * (size_t)n);
  if (x_out) memcpy(x_out, x, sizeof(double) * (size_t)n);
  if (val_out) memcpy(val_out, data, sizeof(double) * (size_t)m);
  clean_cpu();
  graph = saved;
  noNodeTotal = sn;
  noEdgeTotal = sm;
  return std::chrono::duration<double>(t1 - t0).count();
}
