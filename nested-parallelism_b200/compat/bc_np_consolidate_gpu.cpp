// Drop-in definition of the bc application's `void bc_np_consolidate_gpu(void)`
// (apps/bc/src/gpu/bc_wrapper.cu:678-741) on libnps's nps_bc.
//
// It reads the globals the bc application's prepare_gpu() fills -- d_vertexArray,
// d_edgeArray and d_bc (bc_wrapper.cu:14-21) and noNodeTotal / noEdgeTotal
// (common/global.h:53-54) -- and leaves d_bc with the betweenness centrality of
// every vertex over every source in id order, as the reference's loop over
// sources does (its result equals the CPU version bc_cpu bit for bit).  Errors
// do not exit(): they are printed and kept in nps_compat_bc_last_status.
#include <cstdio>

#include "nps.h"

extern int* d_vertexArray;
extern int* d_edgeArray;
extern float* d_bc;
extern int noNodeTotal;
extern int noEdgeTotal;

nps_status nps_compat_bc_last_status = NPS_OK;

void bc_np_consolidate_gpu() {
  nps_params p;
  nps_params_default(&p);
  p.device_ptrs = 1;
  nps_compat_bc_last_status = nps_bc(reinterpret_cast<const int32_t*>(d_vertexArray),
                                     reinterpret_cast<const int32_t*>(d_edgeArray), noNodeTotal, noEdgeTotal,
                                     nullptr, 0, &p, d_bc, nullptr);
  if (nps_compat_bc_last_status != NPS_OK) fprintf(stderr, "bc_np_consolidate_gpu: %s\n", nps_last_error_string());
}
