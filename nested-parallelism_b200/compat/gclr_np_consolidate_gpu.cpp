// Drop-in definition of the graph-color application's
// `void gclr_np_consolidate_gpu(void)` (apps/graph-color/src/gpu/graph_color_wrapper.cu:368-412)
// on libnps's nps_color.
//
// It reads the globals the graph-color application's prepare_gpu() fills --
// d_vertexArray, d_edgeArray, d_colorArray (graph_color_wrapper.cu:16-18) and
// noNodeTotal / noEdgeTotal (common/global.h:53-54) -- and leaves d_colorArray
// with the colors the reference's iterations assign.  Errors do not exit():
// they are printed and kept in nps_compat_color_last_status, and the
// reference's iteration count is kept in nps_compat_color_iterations.
#include <cstdio>

#include "nps.h"

extern int* d_vertexArray;
extern int* d_edgeArray;
extern int* d_colorArray;
extern int noNodeTotal;
extern int noEdgeTotal;

nps_status nps_compat_color_last_status = NPS_OK;
unsigned int nps_compat_color_iterations = 0;

void gclr_np_consolidate_gpu() {
  nps_params p;
  nps_params_default(&p);
  p.device_ptrs = 1;
  nps_stats st;
  nps_compat_color_last_status = nps_color(reinterpret_cast<const int32_t*>(d_vertexArray),
                                           reinterpret_cast<const int32_t*>(d_edgeArray), noNodeTotal, noEdgeTotal,
                                           &p, reinterpret_cast<int32_t*>(d_colorArray), &st);
  if (nps_compat_color_last_status != NPS_OK) {
    fprintf(stderr, "gclr_np_consolidate_gpu: %s\n", nps_last_error_string());
    return;
  }
  nps_compat_color_iterations = st.iterations;
}
