// Betweenness centrality: the bc application (bc_np_consolidate_gpu,
// apps/bc/src/gpu/bc_wrapper.cu:678-741) with the results of its CPU version
// bc_cpu (apps/bc/src/cpu/bc.cpp:152-186, bc_kernel.cpp:3-106), bit for bit.
//
// Brandes' algorithm, one source per CTA.  The reference launches grid-wide
// kernels per BFS level of one source at a time, with a host round trip per
// level; here each source's levels run inside one CTA separated by
// __syncthreads (no grid barrier and no host round trip), and the grid works on
// many sources at once.
//
// Per source s (CTA-private scratch: level, sigma, the vertices in BFS order and
// the level bounds in that order; the source's delta row of a block buffer):
//   forward   level-synchronous BFS.  For an edge u -> v from the frontier
//             (level L), an unvisited v (level = MAX_LEVEL) takes level L + 1 by
//             atomicCAS and is appended to the order; if v is at level L + 1,
//             sigma[v] += sigma[u] (int, wrapping like the reference's
//             __sync_fetch_and_add; integer sums do not depend on order).
//             Rows of 32 edges or more are walked by a whole warp.
//   backward  deepest level first, one thread per vertex u of level L, its
//             edges in CSR order: for v at level L + 1,
//             delta[u] = (float)((double)delta[u] + (double)sigma[u] / sigma[v]
//                                 * (1.0f + delta[v]))
//             with the rounding of every step made explicit (no fused
//             multiply-add), as the reference's x86 code rounds it.
//   sum       bc[v] += delta_s[v] for every reached v other than s, in float, in
//             source order: a second kernel folds the block's delta rows into
//             bc in order, so the result equals the reference's sequential loop
//             over sources exactly.
//
// MAX_LEVEL = 9999 marks unvisited vertices as in the reference
// (common/global.h:17).  Path counts wrap as the reference's int sums do; where
// that gives 0 / 0 the result is NaN on both sides, but with different payloads
// (x86 writes 0xFFC00000, the GPU 0x7FFFFFFF), so NaNs match as NaNs only.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "nps.h"
#include "nps_internal.h"

namespace {

// 256-thread CTAs: 87.9 ms for every source of R-MAT scale 14, against 106 ms with
// 512 (fewer threads per source, more sources in flight; 128 gave 87.5 ms)
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int32_t kMaxLevel = 9999;
constexpr int32_t kWarpRow = 32;  // rows of at least this many edges are walked by a warp (forward)

struct BcArgs {
  const int32_t* row;
  const int32_t* col;
  int32_t n;
  int64_t m;
  const int32_t* sources;  // null: source k is vertex k
  int32_t src_base;        // this block's sources are entries [src_base, src_base + count)
  int32_t count;
  int32_t* level;          // per CTA: n entries each
  int32_t* sigma;
  int32_t* order;
  int32_t* lb;             // per CTA: n + 2 level bounds
  float* delta;            // count rows of n
  uint32_t* status;
};

__device__ __forceinline__ void flag_format(uint32_t* status) { atomicCAS(status, 0u, (uint32_t)NPS_ERR_FORMAT); }

__device__ __forceinline__ bool row_ok(const BcArgs& a, int32_t u, int32_t& s, int32_t& e) {
  s = a.row[u];
  e = a.row[u + 1];
  if (s < 0 || e < s || (int64_t)e > a.m) {
    flag_format(a.status);
    s = e = 0;
    return false;
  }
  return true;
}

// Forward relaxation of edge k from a vertex of level L with path count su.
__device__ __forceinline__ void forward_edge(const BcArgs& a, int32_t* level, int32_t* sigma, int32_t* order,
                                             int* s_tail, int64_t k, int32_t L, int32_t su) {
  const int32_t v = __ldg(a.col + k);
  if ((uint32_t)v >= (uint32_t)a.n) {
    flag_format(a.status);
    return;
  }
  int32_t lv = __ldcg(level + v);
  if (lv == kMaxLevel) {
    lv = atomicCAS(level + v, kMaxLevel, L + 1);
    if (lv == kMaxLevel) {
      lv = L + 1;
      order[atomicAdd(s_tail, 1)] = v;
    }
  }
  if (lv == L + 1) atomicAdd(sigma + v, su);  // wraps as the reference's int sum does
}

__global__ void __launch_bounds__(kThreads) bc_sources_kernel(BcArgs a) {
  __shared__ int s_tail;
  __shared__ int s_nbig[2];  // per sweep parity: a count is reset one sweep after its last read
  __shared__ int32_t s_big[kThreads];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const size_t n = (size_t)a.n;
  int32_t* level = a.level + blockIdx.x * n;
  int32_t* sigma = a.sigma + blockIdx.x * n;
  int32_t* order = a.order + blockIdx.x * n;
  int32_t* lb = a.lb + blockIdx.x * (n + 2);
  int sweep = 0;  // the same count in every thread
  if (tid == 0) s_nbig[0] = s_nbig[1] = 0;
  for (int j = blockIdx.x; j < a.count; j += gridDim.x) {
    const int32_t s = a.sources ? a.sources[a.src_base + j] : a.src_base + j;
    float* delta = a.delta + (size_t)j * n;
    for (size_t v = tid; v < n; v += kThreads) delta[v] = 0.0f;
    if (tid == 0) {
      level[s] = 0;
      sigma[s] = 1;
      order[0] = s;
      lb[0] = 0;
      lb[1] = 1;
      s_tail = 1;
    }
    __syncthreads();
    // ---- forward: the frontier is order[lb[L], lb[L + 1])
    int32_t L = 0;
    for (;;) {
      const int32_t lo = __ldcg(lb + L), hi = __ldcg(lb + L + 1);
      if (lo >= hi) break;
      for (int32_t base = lo; base < hi; base += kThreads, ++sweep) {  // the same sweeps for every thread
        const int par = sweep & 1;
        const int32_t i = base + tid;
        if (i < hi) {
          const int32_t u = __ldcg(order + i);
          int32_t rs, re;
          if (row_ok(a, u, rs, re)) {
            if (re - rs >= kWarpRow) {
              s_big[atomicAdd(&s_nbig[par], 1)] = u;  // at most one per thread per sweep
            } else {
              const int32_t su = __ldcg(sigma + u);
              for (int64_t k = rs; k < re; ++k) forward_edge(a, level, sigma, order, &s_tail, k, L, su);
            }
          }
        }
        __syncthreads();
        const int nbig = s_nbig[par];
        if (tid == 0) s_nbig[par ^ 1] = 0;  // last read in the previous sweep, before the barrier above
        for (int b = warp; b < nbig; b += kWarps) {
          const int32_t u = s_big[b];
          const int32_t rs = a.row[u], re = a.row[u + 1];  // checked when listed
          const int32_t su = __ldcg(sigma + u);
          for (int64_t k = (int64_t)rs + lane; k < re; k += 32) forward_edge(a, level, sigma, order, &s_tail, k, L, su);
        }
        __syncthreads();
      }
      __syncthreads();
      if (tid == 0) lb[L + 2] = s_tail;
      __syncthreads();
      ++L;
    }
    // here L = deepest level + 1.  ---- backward: levels L - 2 down to 1 (level 0 is
    // the source alone, whose delta is never summed; the deepest level's delta is 0)
    for (int32_t d = L - 2; d >= 1; --d) {
      const int32_t lo = __ldcg(lb + d), hi = __ldcg(lb + d + 1);
      for (int32_t i = lo + tid; i < hi; i += kThreads) {
        const int32_t u = __ldcg(order + i);
        const int32_t rs = a.row[u], re = a.row[u + 1];  // checked in the forward pass (else empty)
        if (rs < 0 || re < rs || (int64_t)re > a.m) continue;
        const double su = (double)__ldcg(sigma + u);
        float du = 0.0f;
        for (int64_t k = rs; k < re; ++k) {
          const int32_t v = __ldg(a.col + k);
          if ((uint32_t)v >= (uint32_t)a.n) continue;  // reported in the forward pass
          if (__ldcg(level + v) == d + 1) {
            const double q = __ddiv_rn(su, (double)__ldcg(sigma + v));
            const double t = __dmul_rn(q, (double)__fadd_rn(1.0f, __ldcg(delta + v)));
            du = __double2float_rn(__dadd_rn((double)du, t));
          }
        }
        delta[u] = du;
      }
      __syncthreads();
    }
    // ---- leave the scratch as found: every reached vertex back to unvisited
    const int32_t reached = s_tail;
    for (int32_t i = tid; i < reached; i += kThreads) {
      const int32_t v = __ldcg(order + i);
      level[v] = kMaxLevel;
      sigma[v] = 0;
    }
    __syncthreads();
  }
}

// bc[v] += delta_j[v] for the block's sources j in order (float, one rounding per add).
__global__ void bc_fold_kernel(float* bc, const float* delta, int32_t n, int32_t count) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    float acc = bc[v];
    for (int32_t j = 0; j < count; ++j) acc = __fadd_rn(acc, __ldcs(delta + (size_t)j * n + v));
    bc[v] = acc;
  }
}

__global__ void bc_fill_kernel(int32_t* level, int32_t* sigma, size_t total) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    level[i] = kMaxLevel;
    sigma[i] = 0;
  }
}

__global__ void bc_check_sources_kernel(const int32_t* sources, int32_t nsrc, int32_t n, uint32_t* status) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nsrc; i += gridDim.x * blockDim.x)
    if ((uint32_t)sources[i] >= (uint32_t)n) atomicCAS(status, 0u, (uint32_t)NPS_ERR_INVALID_ARG);
}


struct BcWork {
  unsigned long long ctx_id = 0;  // context the cached buffers live in (nps_context_id)
  std::mutex mu;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[4] = {};
  int sms = 0;
  uint32_t* status = nullptr;
  int32_t* scratch = nullptr;  // level, sigma, order, lb for every CTA
  size_t scratch_n = 0;
  float* delta = nullptr;
  size_t delta_n = 0;
  int32_t* row = nullptr;
  size_t row_n = 0;
  int32_t* col = nullptr;
  size_t col_n = 0;
  int32_t* src = nullptr;
  size_t src_n = 0;
  float* bc = nullptr;
  size_t bc_n = 0;
};

std::mutex g_bc_mu;
std::vector<BcWork*> g_bc;


}  // namespace

extern "C" nps_status nps_bc(const int32_t* row_ptr, const int32_t* col, int32_t n, int64_t m,
                             const int32_t* sources, int32_t nsrc, const nps_params* pin, float* bc_out,
                             nps_stats* st) {
  nps_clear_error();
  nps_params p;
  if (pin) p = *pin;
  else nps_params_default(&p);
  if (n <= 0) return nps_fail(NPS_ERR_INVALID_ARG, "n must be positive");
  if (m < 0 || m >= (int64_t)INT32_MAX) return nps_fail(NPS_ERR_INVALID_ARG, "m must be in [0, 2^31-1)");
  if (!row_ptr || !bc_out || (m > 0 && !col)) return nps_fail(NPS_ERR_INVALID_ARG, "null array");
  if (sources && nsrc < 0) return nps_fail(NPS_ERR_INVALID_ARG, "nsrc must be >= 0");
  if (!p.device_ptrs && (row_ptr[0] != 0 || row_ptr[n] != (int32_t)m))
    return nps_fail(NPS_ERR_FORMAT, "malformed CSR: row_ptr[0] must be 0 and row_ptr[n] must be m");
  if (!p.device_ptrs && sources)
    for (int32_t i = 0; i < nsrc; ++i)
      if (sources[i] < 0 || sources[i] >= n) return nps_fail(NPS_ERR_INVALID_ARG, "bc: source out of range");
  const int32_t count_all = sources ? nsrc : n;
  int dcount = 0;
  if (cudaGetDeviceCount(&dcount) != cudaSuccess || dcount == 0) {
    cudaGetLastError();
    return nps_fail(NPS_ERR_NO_DEVICE, "no CUDA device");
  }
  if (p.device < 0 || p.device >= dcount) return nps_fail(NPS_ERR_INVALID_ARG, "device ordinal out of range");
  NPS_CUDA_RETURN(cudaSetDevice(p.device));
  BcWork* W;
  {
    std::lock_guard<std::mutex> lk(g_bc_mu);
    if ((int)g_bc.size() <= p.device) g_bc.resize(p.device + 1, nullptr);
    {
    const unsigned long long id = nps_context_id(p.device);
    if (g_bc[p.device] && id != 0 && g_bc[p.device]->ctx_id != id) g_bc[p.device] = nullptr;  // device reset: abandoned
    if (!g_bc[p.device]) {
      g_bc[p.device] = new BcWork();
      g_bc[p.device]->ctx_id = id;
    }
  }
    W = g_bc[p.device];
  }
  std::lock_guard<std::mutex> lk(W->mu);
  if (!W->stream) NPS_CUDA_RETURN(cudaStreamCreateWithFlags(&W->stream, cudaStreamNonBlocking));
  if (!W->ev[0])
    for (auto& ev : W->ev) NPS_CUDA_RETURN(cudaEventCreate(&ev));
  if (!W->status) NPS_CUDA_RETURN(cudaMalloc((void**)&W->status, sizeof(uint32_t)));
  if (!W->sms) NPS_CUDA_RETURN(cudaDeviceGetAttribute(&W->sms, cudaDevAttrMultiProcessorCount, p.device));
  cudaStream_t s = p.stream ? (cudaStream_t)p.stream : W->stream;
  if (st) memset(st, 0, sizeof(*st));
  nps_status e;
  NPS_CUDA_RETURN(cudaEventRecord(W->ev[0], s));
  const int32_t* drow = row_ptr;
  const int32_t* dcol = col;
  const int32_t* dsrc = sources;
  float* dbc = bc_out;
  if (!p.device_ptrs) {
    if ((e = nps_ensure(&W->row, &W->row_n, (size_t)n + 1, s, "bc")) || (e = nps_ensure(&W->col, &W->col_n, (size_t)m, s, "bc")) ||
        (e = nps_ensure(&W->bc, &W->bc_n, (size_t)n, s, "bc")))
      return e;
    NPS_CUDA_RETURN(cudaMemcpyAsync(W->row, row_ptr, sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice, s));
    if (m > 0) NPS_CUDA_RETURN(cudaMemcpyAsync(W->col, col, sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice, s));
    if (sources && nsrc > 0) {
      if ((e = nps_ensure(&W->src, &W->src_n, (size_t)nsrc, s, "bc"))) return e;
      NPS_CUDA_RETURN(cudaMemcpyAsync(W->src, sources, sizeof(int32_t) * (size_t)nsrc, cudaMemcpyHostToDevice, s));
      dsrc = W->src;
    }
    drow = W->row;
    dcol = W->col;
    dbc = W->bc;
  }
  // one CTA per source at a time, as many CTAs as are resident; a block of
  // sources shares one delta buffer
  int per_sm = 0;
  NPS_CUDA_RETURN(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bc_sources_kernel, kThreads, 0));
  const size_t per_cta = 4 * (size_t)n + 2;
  // at most 8 GB of CTA scratch (16 n bytes each): large graphs run fewer sources at once
  const int64_t by_memory = std::max<int64_t>(W->sms, (int64_t)((8ull << 30) / (per_cta * sizeof(int32_t))));
  const int grid = (int)std::max<int64_t>(
      1, std::min<int64_t>(std::min<int64_t>((int64_t)W->sms * std::max(1, per_sm), by_memory), count_all));
  if ((e = nps_ensure(&W->scratch, &W->scratch_n, per_cta * (size_t)grid, s, "bc"))) return e;
  const size_t budget = (size_t)1 << 31;  // bytes of delta rows per block
  int64_t cap = std::max<int64_t>(grid, budget / (4 * (size_t)n));
  if (p.reserved[1] > 0) cap = p.reserved[1];
  const int32_t block = (int32_t)std::max<int64_t>(1, std::min<int64_t>(count_all, cap));
  if ((e = nps_ensure(&W->delta, &W->delta_n, (size_t)block * (size_t)n, s, "bc"))) return e;
  NPS_CUDA_RETURN(cudaMemsetAsync(W->status, 0, sizeof(uint32_t), s));
  NPS_CUDA_RETURN(cudaMemsetAsync(dbc, 0, sizeof(float) * (size_t)n, s));
  if (dsrc && nsrc > 0 && p.device_ptrs) {
    bc_check_sources_kernel<<<(int)std::min<int64_t>(1024, ((int64_t)nsrc + 255) / 256), 256, 0, s>>>(dsrc, nsrc, n,
                                                                                               W->status);
    NPS_CUDA_RETURN(cudaGetLastError());
  }
  BcArgs a;
  a.row = drow;
  a.col = dcol;
  a.n = n;
  a.m = m;
  a.sources = dsrc;
  a.level = W->scratch;
  a.sigma = W->scratch + (size_t)n * grid;
  a.order = W->scratch + 2 * (size_t)n * grid;
  a.lb = W->scratch + 3 * (size_t)n * grid;
  a.delta = W->delta;
  a.status = W->status;
  bc_fill_kernel<<<W->sms * 4, 256, 0, s>>>(a.level, a.sigma, (size_t)n * grid);
  NPS_CUDA_RETURN(cudaGetLastError());
  uint32_t h_status = 0;
  if (dsrc && p.device_ptrs) {  // a bad device-side source list stops the call before any kernel reads it
    NPS_CUDA_RETURN(cudaMemcpyAsync(&h_status, W->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    NPS_CUDA_RETURN(cudaStreamSynchronize(s));
    if (h_status) return nps_fail(NPS_ERR_INVALID_ARG, "bc: source out of range");
  }
  NPS_CUDA_RETURN(cudaEventRecord(W->ev[1], s));
  const int fold_grid = (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)n + 255) / 256, (int64_t)W->sms * 8));
  for (int32_t base = 0; base < count_all; base += block) {
    a.src_base = base;
    a.count = std::min<int32_t>(block, count_all - base);
    bc_sources_kernel<<<grid, kThreads, 0, s>>>(a);
    NPS_CUDA_RETURN(cudaGetLastError());
    bc_fold_kernel<<<fold_grid, 256, 0, s>>>(dbc, W->delta, n, a.count);
    NPS_CUDA_RETURN(cudaGetLastError());
  }
  NPS_CUDA_RETURN(cudaEventRecord(W->ev[2], s));
  if (!p.device_ptrs) NPS_CUDA_RETURN(cudaMemcpyAsync(bc_out, dbc, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, s));
  NPS_CUDA_RETURN(cudaMemcpyAsync(&h_status, W->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  NPS_CUDA_RETURN(cudaEventRecord(W->ev[3], s));
  NPS_CUDA_RETURN(cudaStreamSynchronize(s));
  if (st) {
    st->status = (int32_t)h_status;
    st->grid_ctas = grid;
    st->vertices_processed = (uint64_t)count_all;
    cudaEventElapsedTime(&st->kernel_ms, W->ev[1], W->ev[2]);
    cudaEventElapsedTime(&st->total_ms, W->ev[0], W->ev[3]);
  }
  if (h_status == NPS_ERR_FORMAT)
    return nps_fail(NPS_ERR_FORMAT, "malformed CSR: a row range or column index is out of bounds");
  return NPS_OK;
}
