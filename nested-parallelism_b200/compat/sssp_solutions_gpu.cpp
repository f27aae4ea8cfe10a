// Drop-in definitions of the reference dispatcher's other solutions on top of
// libnps: sssp_tqueue_gpu, sssp_dual_queue_gpu, sssp_shared_delayed_buffer_gpu,
// sssp_global_delayed_buffer_gpu, sssp_np_naive_gpu and sssp_np_opt_gpu
// (apps/sssp/src/gpu/sssp_wrapper.cu:151-473), cases 0-5 of SSSP_GPU()'s switch
// (:554-564).
//
// Linked together with sssp_np_consolidate_gpu.cpp (whose nps_compat_last_status
// they share) in place of the reference's definitions.  Each reads the globals
// prepare_gpu() filled (the device CSR, d_costArray with INF except the source,
// d_update with the source flagged) and leaves them as the reference does:
// distances in d_costArray, d_update all zero, `iteration` advanced by the
// number of frontier iterations.  Large rows are those of at least THRESHOLD =
// 64 edges and row-per-thread CTAs have 192 threads, the reference's THRESHOLD
// and THREADS_PER_BLOCK (sssp_kernel.cu:7, sssp_wrapper.cu:12).
//
// Unlike the reference, errors do not exit(): the status is printed to stderr
// and kept in nps_compat_last_status.
#include <cstdio>

#include "nps.h"

extern int* d_vertexArray;
extern int* d_costArray;
extern int* d_edgeArray;
extern int* d_weightArray;
extern char* d_update;
extern int noNodeTotal;
extern int noEdgeTotal;
extern unsigned int iteration;
extern nps_status nps_compat_last_status;

namespace {

void run_solution(int32_t solution, const char* name) {
  nps_params p;
  nps_params_default(&p);
  p.threshold = 64;
  p.block_size = 192;
  p.device_ptrs = 1;
  nps_stats st;
  nps_compat_last_status = nps_sssp_solution_state(
      solution, reinterpret_cast<const int32_t*>(d_vertexArray), reinterpret_cast<const int32_t*>(d_edgeArray),
      reinterpret_cast<const uint32_t*>(d_weightArray), noNodeTotal, noEdgeTotal,
      reinterpret_cast<uint32_t*>(d_costArray), reinterpret_cast<uint8_t*>(d_update), &p, &st, nullptr);
  if (nps_compat_last_status != NPS_OK) {
    fprintf(stderr, "%s: %s\n", name, nps_last_error_string());
    return;
  }
  iteration += st.iterations;
}

}  // namespace

void sssp_tqueue_gpu() { run_solution(NPS_SOLUTION_TQUEUE, "sssp_tqueue_gpu"); }
void sssp_dual_queue_gpu() { run_solution(NPS_SOLUTION_DUAL_QUEUE, "sssp_dual_queue_gpu"); }
void sssp_shared_delayed_buffer_gpu() { run_solution(NPS_SOLUTION_SHARED_DELAYED, "sssp_shared_delayed_buffer_gpu"); }
void sssp_global_delayed_buffer_gpu() { run_solution(NPS_SOLUTION_GLOBAL_DELAYED, "sssp_global_delayed_buffer_gpu"); }
void sssp_np_naive_gpu() { run_solution(NPS_SOLUTION_NP_NAIVE, "sssp_np_naive_gpu"); }
void sssp_np_opt_gpu() { run_solution(NPS_SOLUTION_NP_OPT, "sssp_np_opt_gpu"); }
