// Drop-in definition of the bfs-rec application's `void bfs_rec_dp_cons_gpu(void)`
// (apps/bfs-rec/src/gpu/bfs_rec_wrapper.cu:170-229) on libnps's SSSP engine.
//
// A bfs-rec build links this file in place of its own definition and links
// libnps.so.  It reads the globals that application's prepare_gpu() fills
// (d_vertexArray, d_edgeArray, d_levelArray, bfs_rec_wrapper.cu:28-30, :80-95)
// and noNodeTotal / noEdgeTotal / source (common/global.h:53-55), and leaves
// d_levelArray as the reference does: the hop count from the source, UNDEFINED
// (0x7FFFFFFF) for unreachable vertices.  The engine runs with unit edge weights
// on the unordered frontier; CONSOLIDATE_LEVEL 0/1/2 selects the consolidation level
// as in the reference's compile-time switch (default 2, bfs_rec_wrapper.cu:20-22).
//
// Unlike the reference, errors do not exit(): the status is printed to stderr
// and kept in nps_compat_bfs_last_status.
#include <cstdio>

#include "nps.h"

#ifndef CONSOLIDATE_LEVEL
#define CONSOLIDATE_LEVEL 2
#endif

extern int* d_vertexArray;
extern int* d_edgeArray;
extern int* d_levelArray;
extern int noNodeTotal;
extern int noEdgeTotal;
extern int source;

nps_status nps_compat_bfs_last_status = NPS_OK;

void bfs_rec_dp_cons_gpu() {
  nps_params p;
  nps_params_default(&p);
  p.level = CONSOLIDATE_LEVEL;
  p.delta = 0;
  p.threshold = 32;     // the tuned BFS configuration (nps.bfs_params)
  p.block_size = 512;
  p.device_ptrs = 1;
  nps_stats st;
  nps_compat_bfs_last_status = nps_bfs(reinterpret_cast<const int32_t*>(d_vertexArray),
                                       reinterpret_cast<const int32_t*>(d_edgeArray), noNodeTotal, noEdgeTotal,
                                       source, &p, reinterpret_cast<int32_t*>(d_levelArray), &st);
  if (nps_compat_bfs_last_status != NPS_OK)
    fprintf(stderr, "bfs_rec_dp_cons_gpu: %s\n", nps_last_error_string());
}
