// Degree statistics of a CSR graph on the GPU: the numbers the reference's graph
// analyzer prints (utility/graph-analyzer/analyzer.cpp:75-138, getStatInfo()):
// vertex and edge counts, total / average / maximum / minimum out-degree with the
// lowest vertex id attaining the maximum and the minimum, and the distribution
// (how many vertices have each degree).  It also returns the 8-bin histogram
// [4^k - 1, 4^(k+1) - 1) that the learned policy's frontier features use.
//
// Two streaming passes over row_ptr (4 (n + 1) bytes each, HBM-bound):
//   pass 1  per-thread extremes, sums and 8 bins, reduced per warp and CTA, then
//           one 64-bit atomic per CTA per quantity.  Extremes are packed so one
//           atomicMax / atomicMin also picks the lowest id on ties:
//           max key = degree << 32 | ~id, min key = degree << 32 | id;
//   pass 2  the distribution: degrees below kSmemBins count in a shared-memory
//           histogram per CTA (power-law graphs put most vertices on a few small
//           degrees, which would serialise on global atomics), larger degrees go
//           straight to the global counts.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "nps.h"
#include "nps_internal.h"

namespace {

constexpr int kThreads = 512;
constexpr int kSmemBins = 2048;
constexpr int32_t kRefMinStart = 999999;  // the reference's initial minDegree (analyzer.cpp:85)

struct DegAcc {
  unsigned long long max_key;   // degree << 32 | ~id
  unsigned long long min_key;   // degree << 32 | id
  unsigned long long total;
  unsigned long long bins[8];
  unsigned int bad;             // a row with end < start was seen
};

__device__ __forceinline__ int deg_bin8(int32_t d) {
  const int l = 31 - __clz((uint32_t)d + 1);
  const int b = l >> 1;
  return b > 7 ? 7 : b;
}

__device__ __forceinline__ int32_t rp_load(const int32_t* p) {
  int32_t v;
  asm volatile("ld.global.nc.L1::no_allocate.s32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

__global__ void __launch_bounds__(kThreads) degree_pass1(const int32_t* __restrict__ row_ptr, int32_t n, DegAcc* acc) {
  unsigned long long mx = 0, mn = ~0ull, tot = 0;
  unsigned long long bins[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  unsigned int bad = 0;
  const int stride = gridDim.x * blockDim.x;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    const int32_t d = rp_load(row_ptr + v + 1) - rp_load(row_ptr + v);
    if (d < 0) {
      bad = 1;
      continue;
    }
    const unsigned long long kmax = ((unsigned long long)(uint32_t)d << 32) | (uint32_t)~(uint32_t)v;
    const unsigned long long kmin = ((unsigned long long)(uint32_t)d << 32) | (uint32_t)v;
    mx = kmax > mx ? kmax : mx;
    mn = kmin < mn ? kmin : mn;
    tot += (unsigned long long)d;
    bins[deg_bin8(d)] += 1;
  }
  // warp reduction, then one atomic per warp leader into shared memory, one per CTA to global
  for (int o = 16; o >= 1; o >>= 1) {
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    tot += __shfl_xor_sync(0xffffffffu, tot, o);
#pragma unroll
    for (int b = 0; b < 8; ++b) bins[b] += __shfl_xor_sync(0xffffffffu, bins[b], o);
    bad |= __shfl_xor_sync(0xffffffffu, bad, o);
  }
  __shared__ DegAcc s;
  if (threadIdx.x == 0) {
    s.max_key = 0;
    s.min_key = ~0ull;
    s.total = 0;
    for (int b = 0; b < 8; ++b) s.bins[b] = 0;
    s.bad = 0;
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&s.max_key, mx);
    atomicMin(&s.min_key, mn);
    atomicAdd(&s.total, tot);
    for (int b = 0; b < 8; ++b)
      if (bins[b]) atomicAdd(&s.bins[b], bins[b]);
    if (bad) atomicOr(&s.bad, 1u);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicMax(&acc->max_key, s.max_key);
    atomicMin(&acc->min_key, s.min_key);
    atomicAdd(&acc->total, s.total);
    for (int b = 0; b < 8; ++b)
      if (s.bins[b]) atomicAdd(&acc->bins[b], s.bins[b]);
    if (s.bad) atomicOr(&acc->bad, 1u);
  }
}

__global__ void __launch_bounds__(kThreads) degree_pass2(const int32_t* __restrict__ row_ptr, int32_t n,
                                                         unsigned long long* dist, int64_t dist_len) {
  __shared__ unsigned int h[kSmemBins];
  for (int i = threadIdx.x; i < kSmemBins; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const int stride = gridDim.x * blockDim.x;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    const int32_t d = rp_load(row_ptr + v + 1) - rp_load(row_ptr + v);
    if (d < 0 || (int64_t)d >= dist_len) continue;  // rejected by pass 1 / by the caller's length check
    if (d < kSmemBins) atomicAdd(&h[d], 1u);
    else atomicAdd(&dist[d], 1ull);
  }
  __syncthreads();
  const int lim = dist_len < kSmemBins ? (int)dist_len : kSmemBins;
  for (int i = threadIdx.x; i < lim; i += blockDim.x)
    if (h[i]) atomicAdd(&dist[i], (unsigned long long)h[i]);
}


// Per-device cached buffers: the staged row_ptr (host-pointer calls), the
// accumulators and the distribution.
struct DegWork {
  unsigned long long ctx_id = 0;  // context the cached buffers live in (nps_context_id)
  int32_t* rp = nullptr;
  size_t rp_n = 0;
  DegAcc* acc = nullptr;
  unsigned long long* dist = nullptr;
  size_t dist_n = 0;
  cudaStream_t stream = nullptr;
  std::mutex mu;
};

std::mutex g_deg_mu;
std::vector<DegWork*> g_deg;

DegWork* deg_work(int device) {
  std::lock_guard<std::mutex> lk(g_deg_mu);
  if ((int)g_deg.size() <= device) g_deg.resize(device + 1, nullptr);
  {
    const unsigned long long id = nps_context_id(device);
    if (g_deg[device] && id != 0 && g_deg[device]->ctx_id != id) g_deg[device] = nullptr;  // device reset: abandoned
    if (!g_deg[device]) {
      g_deg[device] = new DegWork();
      g_deg[device]->ctx_id = id;
    }
  }
  return g_deg[device];
}


}  // namespace

extern "C" nps_status nps_degree_stats(const int32_t* row_ptr, int32_t n, int32_t device_ptrs, int32_t device,
                                       nps_degree_info* info, int64_t* dist, int64_t dist_len) {
  nps_clear_error();
  if (!row_ptr || !info || n <= 0) return nps_fail(NPS_ERR_INVALID_ARG, "degree stats: need row_ptr, info and n > 0");
  if (dist_len < 0 || (dist_len > 0 && !dist))
    return nps_fail(NPS_ERR_INVALID_ARG, "degree stats: dist_len > 0 needs a dist array");
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return nps_fail(NPS_ERR_NO_DEVICE, "degree stats: no CUDA device");
  }
  if (device < 0 || device >= count) return nps_fail(NPS_ERR_INVALID_ARG, "degree stats: device ordinal out of range");
  NPS_CUDA_RETURN(cudaSetDevice(device));
  DegWork* w = deg_work(device);
  std::lock_guard<std::mutex> lk(w->mu);
  if (!w->stream) NPS_CUDA_RETURN(cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking));
  cudaStream_t s = w->stream;
  nps_status e;
  const int32_t* rp = row_ptr;
  if (!device_ptrs) {
    if ((e = nps_ensure(&w->rp, &w->rp_n, (size_t)n + 1, s, "degree stats"))) return e;
    NPS_CUDA_RETURN(cudaMemcpyAsync(w->rp, row_ptr, sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice, s));
    rp = w->rp;
  }
  size_t one = 0;
  if (!w->acc) {
    if ((e = nps_ensure(&w->acc, &one, 1, s, "degree stats"))) return e;
  }
  DegAcc init;
  memset(&init, 0, sizeof(init));
  init.min_key = ~0ull;
  NPS_CUDA_RETURN(cudaMemcpyAsync(w->acc, &init, sizeof(init), cudaMemcpyHostToDevice, s));
  int sms = 0;
  NPS_CUDA_RETURN(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const int blocks = (int)std::min<int64_t>((int64_t)sms * 4, ((int64_t)n + kThreads - 1) / kThreads);
  degree_pass1<<<blocks, kThreads, 0, s>>>(rp, n, w->acc);
  NPS_CUDA_RETURN(cudaGetLastError());
  DegAcc out;
  NPS_CUDA_RETURN(cudaMemcpyAsync(&out, w->acc, sizeof(out), cudaMemcpyDeviceToHost, s));
  NPS_CUDA_RETURN(cudaStreamSynchronize(s));
  if (out.bad) return nps_fail(NPS_ERR_FORMAT, "degree stats: row_ptr decreases (malformed CSR)");

  memset(info, 0, sizeof(*info));
  info->n = n;
  int32_t m_last = 0;
  if (device_ptrs) NPS_CUDA_RETURN(cudaMemcpy(&m_last, row_ptr + n, sizeof(int32_t), cudaMemcpyDeviceToHost));
  else m_last = row_ptr[n];
  info->m = m_last;
  info->total_degree = (int64_t)out.total;
  info->edges_by_degree = (int64_t)(out.total / 2);
  info->avg_degree = (float)(int64_t)out.total / (float)n;
  info->max_degree = (int32_t)(out.max_key >> 32);
  info->max_degree_node = (int32_t)~(uint32_t)out.max_key;
  const int32_t dmin = (int32_t)(out.min_key >> 32);
  if (dmin < kRefMinStart) {
    info->min_degree = dmin;
    info->min_degree_node = (int32_t)(uint32_t)out.min_key;
  } else {
    info->min_degree = kRefMinStart;  // no degree below the reference's start value
    info->min_degree_node = -1;
  }
  for (int b = 0; b < 8; ++b) info->bins[b] = (int64_t)out.bins[b];

  if (dist_len > 0) {
    if (dist_len < (int64_t)info->max_degree + 1)
      return nps_fail(NPS_ERR_CAPACITY, "degree stats: dist_len must be at least max_degree + 1 (info is filled)");
    if ((e = nps_ensure(&w->dist, &w->dist_n, (size_t)dist_len, s, "degree stats"))) return e;
    NPS_CUDA_RETURN(cudaMemsetAsync(w->dist, 0, sizeof(unsigned long long) * (size_t)dist_len, s));
    degree_pass2<<<blocks, kThreads, 0, s>>>(rp, n, w->dist, dist_len);
    NPS_CUDA_RETURN(cudaGetLastError());
    NPS_CUDA_RETURN(cudaMemcpyAsync(dist, w->dist, sizeof(int64_t) * (size_t)dist_len,
                            device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
    NPS_CUDA_RETURN(cudaStreamSynchronize(s));
  }
  return NPS_OK;
}
