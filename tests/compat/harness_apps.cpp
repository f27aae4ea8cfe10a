// Test harness standing in for the SpMV, bc and graph-color applications around
// their drop-in shims (nested-parallelism_b200/compat/{spmv,bc,gclr}_np_consolidate_gpu.cpp):
// it owns the globals those applications define (SpMV_wrapper.cu:18-26,
// bc_wrapper.cu:14-21, graph_color_wrapper.cu:16-18, common/global.h:53-54), fills
// them as their prepare_gpu() does, calls one shim and prints the FNV-1a hash
// of the result array and the shim's status.
//
//   harness_apps spmv|bc|color <R-MAT scale> <seed>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "nps.h"

int* d_vertexArray = nullptr;
int* d_edgeArray = nullptr;
double* d_data = nullptr;
double* d_x = nullptr;
double* d_y = nullptr;
float* d_bc = nullptr;
int* d_colorArray = nullptr;
int noNodeTotal = 0;
int noEdgeTotal = 0;

void spmv_np_consolidate_gpu();
void bc_np_consolidate_gpu();
void gclr_np_consolidate_gpu();
extern nps_status nps_compat_spmv_last_status;
extern nps_status nps_compat_bc_last_status;
extern nps_status nps_compat_color_last_status;
extern unsigned int nps_compat_color_iterations;

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
    fprintf(stderr, "usage: harness_apps spmv|bc|color scale seed\n");
    return 1;
  }
  const char* app = argv[1];
  nps_graph g;
  if (nps_gen_rmat(atoi(argv[2]), 16, 0.57, 0.19, 0.19, 255, strtoull(argv[3], nullptr, 10), &g) != NPS_OK) {
    fprintf(stderr, "generator: %s\n", nps_last_error_string());
    return 1;
  }
  noNodeTotal = g.n;
  noEdgeTotal = (int)g.m;
  CK(cudaMalloc(&d_vertexArray, sizeof(int) * (g.n + 1)));
  CK(cudaMalloc(&d_edgeArray, sizeof(int) * (g.m ? g.m : 1)));
  CK(cudaMemcpy(d_vertexArray, g.row_ptr, sizeof(int) * (g.n + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_edgeArray, g.col, sizeof(int) * g.m, cudaMemcpyHostToDevice));
  nps_status status = NPS_OK;
  unsigned long long hash = 0;
  unsigned int extra = 0;
  if (strcmp(app, "spmv") == 0) {
    // the reference's data: val[i] = i % 13 + 0.5, x[i] = i % 17 + 0.5 (SpMV_wrapper.cu:105-113)
    std::vector<double> val(g.m), x(g.n), y(g.n);
    for (int64_t i = 0; i < g.m; ++i) val[i] = i % 13 + 0.5;
    for (int i = 0; i < g.n; ++i) x[i] = i % 17 + 0.5;
    CK(cudaMalloc(&d_data, sizeof(double) * (g.m ? g.m : 1)));
    CK(cudaMalloc(&d_x, sizeof(double) * g.n));
    CK(cudaMalloc(&d_y, sizeof(double) * g.n));
    CK(cudaMemcpy(d_data, val.data(), sizeof(double) * g.m, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_x, x.data(), sizeof(double) * g.n, cudaMemcpyHostToDevice));
    spmv_np_consolidate_gpu();
    status = nps_compat_spmv_last_status;
    CK(cudaMemcpy(y.data(), d_y, sizeof(double) * g.n, cudaMemcpyDeviceToHost));
    hash = nps_fnv1a_u32(reinterpret_cast<const uint32_t*>(y.data()), 2LL * g.n);
  } else if (strcmp(app, "bc") == 0) {
    std::vector<float> bc(g.n);
    CK(cudaMalloc(&d_bc, sizeof(float) * g.n));
    CK(cudaMemset(d_bc, 0, sizeof(float) * g.n));
    bc_np_consolidate_gpu();
    status = nps_compat_bc_last_status;
    CK(cudaMemcpy(bc.data(), d_bc, sizeof(float) * g.n, cudaMemcpyDeviceToHost));
    hash = nps_fnv1a_u32(reinterpret_cast<const uint32_t*>(bc.data()), g.n);
  } else {
    std::vector<int> color(g.n, 0);
    CK(cudaMalloc(&d_colorArray, sizeof(int) * g.n));
    CK(cudaMemcpy(d_colorArray, color.data(), sizeof(int) * g.n, cudaMemcpyHostToDevice));
    gclr_np_consolidate_gpu();
    status = nps_compat_color_last_status;
    extra = nps_compat_color_iterations;
    CK(cudaMemcpy(color.data(), d_colorArray, sizeof(int) * g.n, cudaMemcpyDeviceToHost));
    hash = nps_fnv1a_u32(reinterpret_cast<const uint32_t*>(color.data()), g.n);
  }
  printf("status %d n %d fnv1a %016llx iterations %u\n", (int)status, g.n, hash, extra);
  nps_graph_free(&g);
  return status == NPS_OK ? 0 : 3;
}
