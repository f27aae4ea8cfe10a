// ref_driver_bfs.cpp -- drives the reference's own CPU BFS from plain arrays.
//
// TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline of the BFS
// workload).  Built by oracle/Makefile together with the reference's unmodified
// sources, compiled where they lie:
//   apps/bfs-rec/src/gpu/bfs_rec.cpp   bfs_cpu() (:100-119), its main() renamed by -Dmain=...
//   common/global.cpp                  graph / noNodeTotal / noEdgeTotal / source globals
// The output goes to oracle/_ref/libref_bfs.so only; nothing is copied.
#include <chrono>
#include <cstdint>

#include "bfs_rec.h"

void bfs_cpu(int* levelArray);  // apps/bfs-rec/src/gpu/bfs_rec.cpp:100

// bfs_rec.cpp's main() calls the GPU path; that path is not part of this library.
void BFS_REC_GPU() {}

// Levels from src (UNDEFINED = 0x7FFFFFFF for unreachable vertices) as the
// reference's validation run computes them (bfs_rec.cpp:194-197); returns the
// seconds bfs_cpu() took.  The globals bfs_cpu() reads are set from the caller's
// arrays and restored afterwards.
extern "C" double nps_ref_bfs_cpu(int32_t n, int32_t m, const int32_t* row, const int32_t* col, int32_t src,
                                  int32_t* level) {
  const _GRAPH_ saved = graph;
  const int sn = noNodeTotal, sm = noEdgeTotal, ss = source;
  graph.vertexArray = const_cast<int*>(row);
  graph.edgeArray = const_cast<int*>(col);
  noNodeTotal = n;
  noEdgeTotal = m;
  source = src;
  for (int32_t i = 0; i < n; ++i) level[i] = UNDEFINED;
  level[src] = 0;
  const auto t0 = std::chrono::steady_clock::now();
  bfs_cpu(level);
  const auto t1 = std::chrono::steady_clock::now();
  graph = saved;
  noNodeTotal = sn;
  noEdgeTotal = sm;
  source = ss;
  return std::chrono::duration<double>(t1 - t0).count();
}
