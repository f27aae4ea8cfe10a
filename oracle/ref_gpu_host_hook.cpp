// Linked into the reference's own SSSP command-line program (built by
// oracle/Makefile from apps/sssp/src/gpu/sssp.cpp, sssp_wrapper.cu and
// common/global.cpp where they lie).  TEST INFRASTRUCTURE ONLY.
//
// The program's main() (sssp.cpp:102-156) reads a graph file, converts it to CSR,
// runs SSSP_GPU() ten times -- each prepare_gpu() (sssp_wrapper.cu:58-140)
// resets the device and uploads graph.costArray, case 6 of the switch
// (sssp_wrapper.cu:566) calls sssp_np_consolidate_gpu(), and the costs are copied
// back into graph.costArray (:576) -- and finally calls clear() (global.cpp:401)
// without printing anything.  The build renames global.o's clear() to
// nps_ref_clear_original (objcopy --redefine-sym), so the clear() below runs in
// its place: it writes the last run's graph.costArray (noNodeTotal int32 values)
// to the file named by NPS_REF_COSTS, then frees the graph as the reference does.
#include <cstdio>
#include <cstdlib>

#include "global.h"

int nps_ref_clear_original();

int clear() {
  const char* path = std::getenv("NPS_REF_COSTS");
  if (path && graph.costArray) {
    if (FILE* f = std::fopen(path, "wb")) {
      std::fwrite(graph.costArray, sizeof(int), (size_t)noNodeTotal, f);
      std::fclose(f);
    }
  }
  return nps_ref_clear_original();
}
