// Test harness standing in for the bfs-rec application's bfs_rec.cpp +
// bfs_rec_wrapper.cu around the drop-in bfs_rec_dp_cons_gpu(): it owns the
// globals that application defines (apps/bfs-rec/src/gpu/bfs_rec_wrapper.cu:28-30,
// common/global.h:53-55), fills them as its main() and prepare_gpu() do (levels
// UNDEFINED except level[source] = 0; bfs_rec.cpp:189-190, bfs_rec_wrapper.cu:80-95),
// calls the shim once and prints the FNV-1a hash of the levels and the status.
//
//   harness_bfs <graph: uniform|rmat> <size> <seed>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "nps.h"

int* d_vertexArray = nullptr;
int* d_edgeArray = nullptr;
int* d_levelArray = nullptr;
int noNodeTotal = 0;
int noEdgeTotal = 0;
int source = 0;

void bfs_rec_dp_cons_gpu();
extern nps_status nps_compat_bfs_last_status;

#define CK(x)                                                              \
  do {                                                                     \
    cudaError_t e = (x);                                                   \
    if (e != cudaSuccess) {                                                \
      fprintf(stderr, "%s: %s\n", #x, cudaGetErrorString(e));              \
      return 2;                                                            \
    }                                                                      \
  } while (0)

int main(int argc, char** argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: harness_bfs uniform|rmat size seed\n");
    return 1;
  }
  const bool rmat = strcmp(argv[1], "rmat") == 0;
  const int size = atoi(argv[2]);
  const unsigned long long seed = strtoull(argv[3], nullptr, 10);
  nps_graph g;
  nps_status s = rmat ? nps_gen_rmat(size, 16, 0.57, 0.19, 0.19, 255, seed, &g)
                      : nps_gen_uniform(size, 8LL * size, 100, seed, &g);
  if (s != NPS_OK) {
    fprintf(stderr, "generator: %s\n", nps_last_error_string());
    return 1;
  }
  noNodeTotal = g.n;
  noEdgeTotal = (int)g.m;
  source = g.source;
  CK(cudaMalloc(&d_vertexArray, sizeof(int) * (g.n + 1)));
  CK(cudaMalloc(&d_edgeArray, sizeof(int) * (g.m ? g.m : 1)));
  CK(cudaMalloc(&d_levelArray, sizeof(int) * g.n));
  CK(cudaMemcpy(d_vertexArray, g.row_ptr, sizeof(int) * (g.n + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_edgeArray, g.col, sizeof(int) * g.m, cudaMemcpyHostToDevice));
  std::vector<int> level(g.n, NPS_BFS_UNDEFINED);
  level[source] = 0;
  CK(cudaMemcpy(d_levelArray, level.data(), sizeof(int) * g.n, cudaMemcpyHostToDevice));

  bfs_rec_dp_cons_gpu();

  CK(cudaMemcpy(level.data(), d_levelArray, sizeof(int) * g.n, cudaMemcpyDeviceToHost));
  printf("status %d source %d n %d fnv1a %016llx\n", (int)nps_compat_bfs_last_status, source, g.n,
         (unsigned long long)nps_fnv1a_u32((const uint32_t*)level.data(), g.n));
  cudaFree(d_vertexArray);
  cudaFree(d_edgeArray);
  cudaFree(d_levelArray);
  nps_graph_free(&g);
  return nps_compat_bfs_last_status == NPS_OK ? 0 : 3;
}
