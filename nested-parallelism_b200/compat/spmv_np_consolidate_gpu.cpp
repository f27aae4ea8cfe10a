// Drop-in definition of the SpMV application's `void spmv_np_consolidate_gpu(void)`
// (apps/SpMV/src/gpu/SpMV_wrapper.cu:285-311) on libnps's nps_spmv.
//
// It reads the globals the SpMV application's prepare_gpu() fills -- d_vertexArray,
// d_edgeArray, d_data, d_x, d_y (SpMV_wrapper.cu:18-26) and noNodeTotal /
// noEdgeTotal (common/global.h:53-54) -- and leaves d_y = A x as the reference
// does.  CONSOLIDATE_LEVEL 0/1/2 selects the consolidation level as in the
// reference's compile-time switch (default 2 here).  FLOAT_T is double
// (apps/SpMV/src/gpu/SpMV.h:13).  Errors do not exit(): they are printed and kept
// in nps_compat_spmv_last_status.
#include <cstdio>

#include "nps.h"

#ifndef CONSOLIDATE_LEVEL
#define CONSOLIDATE_LEVEL 2
#endif

extern int* d_vertexArray;
extern int* d_edgeArray;
extern double* d_data;
extern double* d_x;
extern double* d_y;
extern int noNodeTotal;
extern int noEdgeTotal;

nps_status nps_compat_spmv_last_status = NPS_OK;

void spmv_np_consolidate_gpu() {
  nps_params p;
  nps_params_default(&p);
  p.level = CONSOLIDATE_LEVEL;
  p.device_ptrs = 1;
  nps_compat_spmv_last_status = nps_spmv(reinterpret_cast<const int32_t*>(d_vertexArray),
                                         reinterpret_cast<const int32_t*>(d_edgeArray), d_data, d_x, d_y,
                                         noNodeTotal, noEdgeTotal, &p, nullptr);
  if (nps_compat_spmv_last_status != NPS_OK)
    fprintf(stderr, "spmv_np_consolidate_gpu: %s\n", nps_last_error_string());
}
