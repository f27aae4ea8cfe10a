// Test harness standing in for the reference's sssp.cpp + sssp_wrapper.cu around
// the drop-in solutions (sssp_np_consolidate_gpu() and the six earlier ones of
// SSSP_GPU()'s switch, sssp_wrapper.cu:554-566): it owns the file-scope globals the
// reference defines (apps/sssp/src/gpu/sssp_wrapper.cu:22-30, common/global.h:53-54),
// fills them the way prepare_gpu() does (cost = INF except cost[src] = 0,
// update[src] = 1; sssp_wrapper.cu:98-113), calls the chosen solution once, as
// SSSP_GPU() would, and prints the FNV-1a hash of the distances, the iteration
// count and the shim's status.
//
//   harness <graph: uniform|rmat> <size> <seed> [solution 0-6, default 6]
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "nps.h"

int* d_vertexArray = nullptr;
int* d_costArray = nullptr;
int* d_edgeArray = nullptr;
int* d_weightArray = nullptr;
char* d_update = nullptr;
int noNodeTotal = 0;
int noEdgeTotal = 0;
unsigned int iteration = 0;

void sssp_tqueue_gpu();
void sssp_dual_queue_gpu();
void sssp_shared_delayed_buffer_gpu();
void sssp_global_delayed_buffer_gpu();
void sssp_np_naive_gpu();
void sssp_np_opt_gpu();
void sssp_np_consolidate_gpu();
extern nps_status nps_compat_last_status;

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
    fprintf(stderr, "usage: harness uniform|rmat size seed\n");
    return 1;
  }
  const bool rmat = strcmp(argv[1], "rmat") == 0;
  const int size = atoi(argv[2]);
  const unsigned long long seed = strtoull(argv[3], nullptr, 10);
  const int solution = argc > 4 ? atoi(argv[4]) : 6;
  nps_graph g;
  nps_status s = rmat ? nps_gen_rmat(size, 16, 0.57, 0.19, 0.19, 255, seed, &g)
                      : nps_gen_uniform(size, 8LL * size, 100, seed, &g);
  if (s != NPS_OK) {
    fprintf(stderr, "generator: %s\n", nps_last_error_string());
    return 1;
  }
  noNodeTotal = g.n;
  noEdgeTotal = (int)g.m;
  const int src = g.source;
  CK(cudaMalloc(&d_vertexArray, sizeof(int) * (g.n + 1)));
  CK(cudaMalloc(&d_edgeArray, sizeof(int) * (g.m ? g.m : 1)));
  CK(cudaMalloc(&d_weightArray, sizeof(int) * (g.m ? g.m : 1)));
  CK(cudaMalloc(&d_costArray, sizeof(int) * g.n));
  CK(cudaMalloc(&d_update, g.n));
  CK(cudaMemcpy(d_vertexArray, g.row_ptr, sizeof(int) * (g.n + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_edgeArray, g.col, sizeof(int) * g.m, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_weightArray, g.w, sizeof(int) * g.m, cudaMemcpyHostToDevice));
  std::vector<int> cost(g.n, NPS_INF);
  std::vector<char> upd(g.n, 0);
  cost[src] = 0;
  upd[src] = 1;
  CK(cudaMemcpy(d_costArray, cost.data(), sizeof(int) * g.n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_update, upd.data(), g.n, cudaMemcpyHostToDevice));

  switch (solution) {  // SSSP_GPU()'s dispatch, sssp_wrapper.cu:552-570
    case 0: sssp_tqueue_gpu(); break;
    case 1: sssp_dual_queue_gpu(); break;
    case 2: sssp_shared_delayed_buffer_gpu(); break;
    case 3: sssp_global_delayed_buffer_gpu(); break;
    case 4: sssp_np_naive_gpu(); break;
    case 5: sssp_np_opt_gpu(); break;
    case 6: sssp_np_consolidate_gpu(); break;
    default: fprintf(stderr, "solution must be 0..6\n"); return 1;
  }

  CK(cudaMemcpy(cost.data(), d_costArray, sizeof(int) * g.n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(upd.data(), d_update, g.n, cudaMemcpyDeviceToHost));
  int upd_left = 0;
  for (char c : upd) upd_left += c != 0;
  printf("status %d iterations %u source %d n %d fnv1a %016llx update_left %d\n", (int)nps_compat_last_status,
         iteration, src, g.n, (unsigned long long)nps_fnv1a_u32((const uint32_t*)cost.data(), g.n), upd_left);
  cudaFree(d_vertexArray);
  cudaFree(d_edgeArray);
  cudaFree(d_weightArray);
  cudaFree(d_costArray);
  cudaFree(d_update);
  nps_graph_free(&g);
  return nps_compat_last_status == NPS_OK ? 0 : 3;
}
