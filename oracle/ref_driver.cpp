// ref_driver.cpp -- drives the reference's own CPU SSSP code from plain arrays.
//
// TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline).  Built by
// oracle/Makefile together with the reference's unmodified sources, compiled
// where they lie:
//   apps/sssp/src/cpu/sssp.cpp         SSSP_CPU(), its main() renamed by -Dmain=...
//   common/heap.cpp                    Heap (lazy-insertion binary heap)
//   common/global.cpp                  graph / noNodeTotal / noEdgeTotal / source globals
//   apps/sssp/src/cpu/sssp_kernel.cpp  usssp_cpu(), the OpenMP frontier sweep
//   common/dheap.cpp                   dheap, the d-ary heap with decrease-key
//                                      (driven from ref_driver_dheap.cpp: heap.h and
//                                      dheap.h both define a type named item)
// The output goes to oracle/_ref/libref_sssp.so only; nothing is copied.
//
// The reference code reads and writes the globals of common/global.h:28-58, so
// these entry points fill them from the caller's arrays, run, and restore them.
#include <fcntl.h>
#include <unistd.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "global.h"
#include "heap.h"

int SSSP_CPU();     // apps/sssp/src/cpu/sssp.cpp:13
void usssp_cpu();   // apps/sssp/src/cpu/sssp_kernel.cpp:14

namespace {

// SSSP_CPU() prints an iteration count on stdout; keep the caller's stdout clean.
struct QuietStdout {
  int saved = -1;
  QuietStdout() {
    fflush(stdout);
    saved = dup(1);
    int dn = open("/dev/null", O_WRONLY);
    if (dn >= 0) {
      dup2(dn, 1);
      close(dn);
    }
  }
  ~QuietStdout() {
    fflush(stdout);
    if (saved >= 0) {
      dup2(saved, 1);
      close(saved);
    }
  }
};

struct Globals {
  _GRAPH_ g;
  int n, m, s;
  Globals() : g(graph), n(noNodeTotal), m(noEdgeTotal), s(source) {}
  ~Globals() {
    graph = g;
    noNodeTotal = n;
    noEdgeTotal = m;
    source = s;
  }
};

void bind(int32_t n, int32_t m, const int32_t* row, const int32_t* col, const int32_t* w, int32_t src,
          int32_t* cost) {
  noNodeTotal = n;
  noEdgeTotal = m;
  source = src;
  graph.vertexArray = const_cast<int32_t*>(row);
  graph.edgeArray = const_cast<int32_t*>(col);
  graph.weightArray = const_cast<int32_t*>(w);
  graph.costArray = cost;
}

}  // namespace

extern "C" {

// Reference heap Dijkstra.  Returns wall seconds of SSSP_CPU() (which includes
// its own `new Heap()` of a 102.4 MB bitmask, common/heap.cpp:3-10).
double nps_ref_sssp_cpu(int32_t n, int32_t m, const int32_t* row, const int32_t* col, const int32_t* w,
                        int32_t src, int32_t* cost) {
  Globals keep;
  bind(n, m, row, col, w, src, cost);
  QuietStdout q;
  auto t0 = std::chrono::steady_clock::now();
  SSSP_CPU();
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

// Wall seconds of the Heap constructor alone (the bitmask zero-fill).
double nps_ref_heap_init_seconds(void) {
  auto t0 = std::chrono::steady_clock::now();
  Heap* h = new Heap();
  auto t1 = std::chrono::steady_clock::now();
  delete h;
  return std::chrono::duration<double>(t1 - t0).count();
}

// Reference OpenMP frontier sweep (racy: unsynchronised writes to costArray,
// apps/sssp/src/cpu/sssp_kernel.cpp:42-44).  Timing baseline only.
double nps_ref_usssp_cpu(int32_t n, int32_t m, const int32_t* row, const int32_t* col, const int32_t* w,
                         int32_t src, int32_t threads, int32_t* cost) {
  Globals keep;
  bind(n, m, row, col, w, src, cost);
  if (threads > 0) omp_set_num_threads(threads);
  auto t0 = std::chrono::steady_clock::now();
  usssp_cpu();
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

// The reference's own file front-end: readInputDIMACS9 / readInputDIMACS10 /
// readInputSLNDC (format 0 / 1 / 2, common/global.cpp:29-190) followed by
// convertCSR() (:192-235).  On success *n, *m, *source are set and the CSR is
// copied into caller buffers of capacity cap_n+1 / cap_m (pass null buffers to
// query the sizes).  Returns 0, -1 (cannot open), -2 (buffers too small).
int nps_ref_read_graph(const char* path, int32_t format, int32_t* n, int32_t* m, int32_t* src,
                       int32_t* row, int32_t* col, int32_t* w, int32_t cap_n, int32_t cap_m) {
  Globals keep;
  fp = fopen(path, "r");
  if (!fp) return -1;
  source = 0;
  {
    QuietStdout q;
    if (format == 0) readInputDIMACS9();
    else if (format == 1) readInputDIMACS10();
    else readInputSLNDC();
  }
  fclose(fp);
  fp = nullptr;
  convertCSR();
  *n = noNodeTotal;
  *m = noEdgeTotal;
  *src = source;
  int rc = 0;
  if (row && col && w) {
    if (cap_n < noNodeTotal || cap_m < noEdgeTotal) {
      rc = -2;
    } else {
      memcpy(row, graph.vertexArray, sizeof(int32_t) * (noNodeTotal + 1));
      memcpy(col, graph.edgeArray, sizeof(int32_t) * noEdgeTotal);
      memcpy(w, graph.weightArray, sizeof(int32_t) * noEdgeTotal);
    }
  }
  delete[] graph.vertexArray;
  delete[] graph.edgeArray;
  delete[] graph.weightArray;
  delete[] graph.costArray;
  delete[] graph.levelArray;
  delete[] graph.frontier;
  delete[] graph.update;
  delete[] graph.visited;
  return rc;
}

}  // extern "C"
