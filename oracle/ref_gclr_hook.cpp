// Linked into the reference's graph-coloring program gpu-graph-color (built by
// oracle/Makefile from apps/graph-color/src/gpu where the sources lie).
// TEST INFRASTRUCTURE ONLY.
//
// The program's main() (graph_color.cpp:113-158) colors the graph on the GPU,
// copies the colors back into graph.colorArray (graph_color_wrapper.cu:700) and
// frees them in clean_gclr_cpu() (graph_color.cpp:107-111); it prints them only
// through outputColor() with -d, which has no return statement
// (common/global.cpp:392-398) and traps when built with a current GCC.  The build
// makes graph_color.o's clean_gclr_cpu() weak (objcopy --weaken-symbol) so the one
// below runs in its place: it writes the colors (noNodeTotal int32 values) to the
// file named by NPS_REF_COLORS, then frees them as the reference's does.
#include <cstdio>
#include <cstdlib>

#include "global.h"

void clean_gclr_cpu() {
  const char* path = std::getenv("NPS_REF_COLORS");
  if (path && graph.colorArray) {
    if (FILE* f = std::fopen(path, "wb")) {
      std::fwrite(graph.colorArray, sizeof(int), (size_t)noNodeTotal, f);
      std::fclose(f);
    }
  }
  delete[] graph.colorArray;
}
