// Drop-in definition of the reference's `void sssp_np_consolidate_gpu(void)`
// (apps/sssp/src/gpu/sssp_wrapper.cu:475-546) on top of libnps.
//
// A reference build links this file in place of its own definition (delete or
// rename the one in sssp_wrapper.cu) and links libnps.so.  It reads the same
// file-scope globals the reference function uses -- the device CSR, cost and
// update arrays that prepare_gpu() filled (sssp_wrapper.cu:22-30, :98-113) and
// noNodeTotal / noEdgeTotal (common/global.h:53-54) -- and leaves them as the
// reference does: d_costArray holds the distances (int32, INF = 2^30 for
// unreachable vertices), d_update is all zero, and `iteration` counts the
// frontier iterations.  CONSOLIDATE_LEVEL 0/1/2 (warp/block/grid) selects the
// consolidation level as in the reference's compile-time switch.
//
// Unlike the reference, errors do not exit(): the status is printed to stderr
// and kept in nps_compat_last_status for the caller to inspect.
#include <cstdio>

#include "nps.h"

#ifndef CONSOLIDATE_LEVEL
#define CONSOLIDATE_LEVEL 0  // same default as sssp_wrapper.cu:14-16
#endif

// the reference's globals (defined by the reference's sssp_wrapper.cu / global.cpp)
extern int* d_vertexArray;
extern int* d_costArray;
extern int* d_edgeArray;
extern int* d_weightArray;
extern char* d_update;
extern int noNodeTotal;
extern int noEdgeTotal;
extern unsigned int iteration;

nps_status nps_compat_last_status = NPS_OK;

void sssp_np_consolidate_gpu() {
  nps_params p;
  nps_params_default(&p);
  p.level = CONSOLIDATE_LEVEL;
  p.device_ptrs = 1;
  nps_stats st;
  nps_compat_last_status = nps_sssp_state(
      reinterpret_cast<const int32_t*>(d_vertexArray), reinterpret_cast<const int32_t*>(d_edgeArray),
      reinterpret_cast<const uint32_t*>(d_weightArray), noNodeTotal, noEdgeTotal,
      reinterpret_cast<uint32_t*>(d_costArray), reinterpret_cast<uint8_t*>(d_update), &p, &st);
  if (nps_compat_last_status != NPS_OK) {
    fprintf(stderr, "sssp_np_consolidate_gpu: %s\n", nps_last_error_string());
    return;
  }
  iteration += st.iterations;
}
