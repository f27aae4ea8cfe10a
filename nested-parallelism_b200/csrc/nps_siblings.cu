// The reference dispatcher's other solutions, 0-5 of SSSP_GPU()'s `solution`
// switch (apps/sssp/src/gpu/sssp_wrapper.cu:151-473, kernels
// apps/sssp/src/gpu/sssp_kernel.cu:34-327 and :626-658), on libnps's graph
// arrays, for ablation against workload consolidation (solution 6, the
// persistent engine in nps_engine.cu).
//
// Every solution iterates the reference's unordered frontier: an iteration
// walks the rows of a queue of vertices, relaxing cost[v] > cost[u] + w with
// atomicMin and flagging v in update[]; a generation kernel then turns the flags
// into the next queue (unorder_generateQueue_kernel, sssp_kernel.cu:648).  They
// differ only in which threads walk a queued row u of degree d:
//
//   0 thread queue          one thread walks the row, whatever d
//                           (unorder_threadQueue_kernel, sssp_kernel.cu:34)
//   1 dual queue            the generation kernel splits the queue at d = threshold;
//                           small rows by a thread, large rows by a 64-thread CTA each
//                           (unorder_gen_multiQueue_kernel :626, unorder_blockQueue_kernel :57)
//   2 shared delayed buffer d >= threshold is deferred into the CTA's shared buffer,
//                           which the whole CTA then walks row by row (:112)
//   3 global delayed buffer d >= threshold is deferred into one device buffer, walked
//                           by a second kernel with a 64-thread CTA per row (:179, :57)
//   4 naive nested launch   each row with d >= threshold gets its own child grid of
//                           one 64-thread CTA (unorder_threadQueue_multiple_dp_kernel :233,
//                           sssp_process_neighbors :216)
//   5 per-block nested      each CTA gathers its rows with d >= threshold and launches
//                           one child grid, a 64-thread CTA per row
//                           (unorder_threadQueue_single_dp_kernel :279, sssp_process_buffer :82)
//
// How this differs from the reference, and why:
//   - The host does not read the queue length back after every iteration.  It
//     enqueues chunks of iterations (4, 8, 16, then 32 at a time) and reads the
//     counters once per chunk, one chunk behind, so the read overlaps the next
//     chunk.  Every kernel of an iteration whose queue is empty returns at once.
//   - Grids are fixed (full occupancy on this device) and stride over the queue,
//     so they can be enqueued before the queue length is known.
//   - Queue and buffer appends are warp-aggregated: one atomic per warp.
//   - A vertex is flagged only when its atomicMin lowered the cost.
//   - Nested launches use the CUDA 12 device runtime: child grids go to the
//     fire-and-forget stream, and a parent grid completes only after its children.
//     A launch the device runtime refuses (its pending-launch limit) is walked by
//     the launching thread and counted in nps_solution_info.launch_fallbacks.
//   - The queue never overflows: a vertex enters it at most once per generation,
//     so n entries suffice (the reference has a fixed 10,240,000-entry queue).
//   - A neighbour id outside [0, n) or a malformed row is skipped and reported as
//     NPS_ERR_FORMAT, as in the persistent engine.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "nps.h"
#include "nps_internal.h"

namespace {

constexpr uint32_t kInf = NPS_INF;
constexpr int kRowCta = 64;  // threads of a row-per-CTA walker and of a child grid's CTAs
                             // (NESTED_BLOCK_SIZE, sssp_kernel.cu:9)
constexpr int kGenThreads = 256;
constexpr int kMaxBlock = 1024;
constexpr int kMaxChunk = 32;
constexpr size_t kPendingLaunches = 1 << 16;  // device-runtime pending-launch limit set for 4 and 5

// Device counters of one call, zeroed by the host before the first kernel.
// Queue lengths are kept per iteration parity: iteration i walks parity i & 1,
// its generation kernel fills parity (i + 1) & 1, which the first kernel of
// iteration i zeroes.
struct SibCtr {
  uint32_t qlo[2];      // queue length (solution 1: small rows, from the front of the queue)
  uint32_t qhi[2];      // solution 1: large rows, from the back of the queue
  uint32_t hlen;        // solution 3: rows in the device delayed buffer
  uint32_t iterations;  // iterations whose queue was not empty
  uint32_t status;      // NPS_ERR_FORMAT on a malformed row or neighbour id
  uint32_t reached;
  unsigned long long processed;  // queued rows
  unsigned long long edges;      // out-edges of the queued rows
  unsigned long long deferred;
  unsigned long long launches;
  unsigned long long fallbacks;
  unsigned long long reached_edges;
};

struct Graph {
  const int32_t* row;
  const int32_t* col;
  const uint32_t* w;
  uint32_t* dist;
  uint8_t* upd;
  int32_t n;
  int64_t m;
};

__device__ __forceinline__ void relax_edge(const Graph& g, uint32_t du, int64_t k, SibCtr* c) {
  const int32_t v = g.col[k];
  if ((uint32_t)v >= (uint32_t)g.n) {
    atomicCAS(&c->status, 0u, (uint32_t)NPS_ERR_FORMAT);
    return;
  }
  const uint32_t wk = g.w[k];
  const uint32_t alt = (wk >= kInf || du >= kInf) ? kInf : du + wk;  // both < 2^30: no wrap
  if (g.dist[v] > alt && atomicMin(&g.dist[v], alt) > alt) g.upd[v] = 1;
}

// Row bounds of u; false (and status FORMAT) on a malformed row.
__device__ __forceinline__ bool row_of(const Graph& g, int32_t u, int32_t& s, int32_t& e, SibCtr* c) {
  s = g.row[u];
  e = g.row[u + 1];
  if (s < 0 || e < s || (int64_t)e > g.m) {
    atomicCAS(&c->status, 0u, (uint32_t)NPS_ERR_FORMAT);
    return false;
  }
  return true;
}

__device__ __forceinline__ void walk_row_serial(const Graph& g, int32_t u, int32_t s, int32_t e, SibCtr* c) {
  const uint32_t du = g.dist[u];
  for (int64_t k = s; k < e; ++k) relax_edge(g, du, k, c);
}

// Child grid of solution 4: the edges [s, e) of one row, strided over the grid
// (sssp_process_neighbors, sssp_kernel.cu:216).
__global__ void child_row_kernel(Graph g, uint32_t du, int32_t s, int32_t e, SibCtr* c) {
  for (int64_t k = (int64_t)s + blockIdx.x * blockDim.x + threadIdx.x; k < e; k += (int64_t)gridDim.x * blockDim.x)
    relax_edge(g, du, k, c);
}

// One CTA per listed row, threads strided over the row's edges
// (unorder_blockQueue_kernel, sssp_kernel.cu:57; sssp_process_buffer, :82).
// Entry b of the list is list[b * dir]; the length is *len_ptr when given.
__global__ void __launch_bounds__(kRowCta) row_per_cta_kernel(Graph g, const int32_t* list, int dir,
                                                               const uint32_t* len_ptr, uint32_t len_fixed,
                                                               SibCtr* c) {
  const uint32_t len = len_ptr ? *len_ptr : len_fixed;
  for (uint32_t b = blockIdx.x; b < len; b += gridDim.x) {
    const int32_t u = list[(int64_t)dir * b];
    int32_t s, e;
    if (!row_of(g, u, s, e, c)) continue;
    const uint32_t du = g.dist[u];
    for (int64_t k = (int64_t)s + threadIdx.x; k < e; k += blockDim.x) relax_edge(g, du, k, c);
  }
}

// One slot of a device array for every lane with want = true, reserved with one
// atomic per warp; returns this lane's slot (unspecified where want = false).
// All 32 lanes of the warp must call it.
__device__ __forceinline__ uint32_t warp_reserve(uint32_t* ctr, bool want) {
  const unsigned lane = threadIdx.x & 31;
  const unsigned mask = __ballot_sync(0xffffffffu, want);
  uint32_t base = 0;
  if (mask) {
    const int leader = __ffs(mask) - 1;
    if ((int)lane == leader) base = atomicAdd(ctr, (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
  }
  return base + __popc(mask & ((1u << lane) - 1));
}

enum Mode { kThreadOnly = 0, kSharedDelayed = 2, kGlobalDelayed = 3, kNestedNaive = 4, kNestedPerBlock = 5 };

// Row-per-thread pass over the queue of iteration `it` (parity it & 1), with
// the large-row handling of MODE.  Queue entry i is walked by thread i of the
// grid-stride sweep; every CTA runs the same number of sweeps, so the CTA-wide
// barriers of MODE 2 and 5 are reached by all threads.
template <int MODE>
__global__ void __launch_bounds__(kMaxBlock) row_per_thread_kernel(Graph g, const int32_t* q, int it,
                                                                    int32_t threshold, int32_t* buf,
                                                                    uint32_t slice, SibCtr* c) {
  const int cur = it & 1, nxt = cur ^ 1;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    c->qlo[nxt] = 0;
    c->qhi[nxt] = 0;
  }
  const uint32_t len = c->qlo[cur];
  if (len == 0) return;
  __shared__ int32_t s_rows[kMaxBlock];
  __shared__ uint32_t s_count;
  if (MODE == kSharedDelayed || MODE == kNestedPerBlock) {
    if (threadIdx.x == 0) s_count = 0;
    __syncthreads();
  }
  unsigned long long deferred = 0, launches = 0, fallbacks = 0;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x; base < len; base += stride) {
    const uint32_t i = base + threadIdx.x;
    int32_t u = -1, s = 0, e = 0;
    if (i < len) {
      u = q[i];
      if (!row_of(g, u, s, e, c)) u = -1;
    }
    const bool large = MODE != kThreadOnly && u >= 0 && e - s >= threshold;
    if (u >= 0 && !large) walk_row_serial(g, u, s, e, c);
    if (MODE == kSharedDelayed) {
      if (large) s_rows[atomicAdd(&s_count, 1u)] = u;  // at most blockDim.x rows per sweep
      __syncthreads();
      const uint32_t cnt = s_count;
      for (uint32_t j = 0; j < cnt; ++j) {
        const int32_t r = s_rows[j];
        int32_t rs = g.row[r], re = g.row[r + 1];  // checked when deferred
        const uint32_t dr = g.dist[r];
        for (int64_t k = (int64_t)rs + threadIdx.x; k < re; k += blockDim.x) relax_edge(g, dr, k, c);
      }
      deferred += (threadIdx.x == 0) ? cnt : 0;
      __syncthreads();
      if (threadIdx.x == 0) s_count = 0;
      __syncthreads();
    } else if (MODE == kGlobalDelayed) {
      const uint32_t slot = warp_reserve(&c->hlen, large);  // hlen <= len <= n entries
      if (large) {
        buf[slot] = u;
        ++deferred;
      }
    } else if (MODE == kNestedNaive) {
      if (large) {
        ++deferred;
        child_row_kernel<<<1, kRowCta, 0, cudaStreamFireAndForget>>>(g, g.dist[u], s, e, c);
        if (cudaGetLastError() == cudaSuccess) {
          ++launches;
        } else {
          ++fallbacks;
          walk_row_serial(g, u, s, e, c);
        }
      }
    } else if (MODE == kNestedPerBlock) {
      if (large) {
        buf[(size_t)blockIdx.x * slice + atomicAdd(&s_count, 1u)] = u;  // < slice: rows this CTA sweeps
        ++deferred;
      }
    }
  }
  if (MODE == kNestedPerBlock) {
    __syncthreads();
    if (threadIdx.x == 0 && s_count > 0) {
      const int32_t* list = buf + (size_t)blockIdx.x * slice;
      __threadfence();  // the CTA's list entries (ordered by the barrier) before the child reads them
      row_per_cta_kernel<<<s_count, kRowCta, 0, cudaStreamFireAndForget>>>(g, list, 1, nullptr, s_count, c);
      if (cudaGetLastError() == cudaSuccess) {
        ++launches;
      } else {
        ++fallbacks;
        for (uint32_t j = 0; j < s_count; ++j) {
          int32_t rs, re;
          if (row_of(g, list[j], rs, re, c)) walk_row_serial(g, list[j], rs, re, c);
        }
      }
    }
  }
  if (deferred) atomicAdd(&c->deferred, deferred);
  if (launches) atomicAdd(&c->launches, launches);
  if (fallbacks) atomicAdd(&c->fallbacks, fallbacks);
}

// The flags -> queue step of iteration `it` (it = -1: the initial queue from
// the caller's flags).  Clears each flag it reads; appends to parity
// (it + 1) & 1; DUAL splits at `threshold` into the front (small) and back
// (large) of the queue.  Also counts the queued rows and their edges, and
// zeroes the solution-3 buffer length for the next iteration.
template <bool DUAL>
__global__ void __launch_bounds__(kGenThreads) gen_queue_kernel(Graph g, int32_t* q, int it, int32_t threshold,
                                                                SibCtr* c) {
  const int nxt = (it + 1) & 1;
  if (it >= 0) {
    const int cur = it & 1;
    const uint32_t len = c->qlo[cur] + (DUAL ? c->qhi[cur] : 0u);
    if (len == 0) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      c->iterations += 1;
      c->processed += len;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) c->hlen = 0;
  const int32_t n = g.n;
  // every thread of a warp runs the same number of sweeps (the bound is warp-uniform)
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t span = (((int64_t)n + 31) / 32) * 32;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < span; v += stride) {
    bool flag = false;
    uint32_t deg = 0;
    if (v < n && g.upd[v]) {
      g.upd[v] = 0;
      flag = true;
      const int32_t s = g.row[v], e = g.row[v + 1];
      deg = (e >= s) ? (uint32_t)(e - s) : 0u;
    }
    if (DUAL) {
      const bool large = flag && (int64_t)deg >= threshold;
      const bool small = flag && !large;
      const uint32_t a = warp_reserve(&c->qlo[nxt], small);
      const uint32_t b = warp_reserve(&c->qhi[nxt], large);
      if (small) q[a] = (int32_t)v;
      if (large) q[(int64_t)n - 1 - b] = (int32_t)v;  // small + large <= n: the ends never meet
      const unsigned lm = __ballot_sync(0xffffffffu, large);
      if ((threadIdx.x & 31) == 0 && lm) atomicAdd(&c->deferred, (unsigned long long)__popc(lm));
    } else {
      const uint32_t a = warp_reserve(&c->qlo[nxt], flag);
      if (flag) q[a] = (int32_t)v;
    }
    const uint32_t dsum = __reduce_add_sync(0xffffffffu, deg);
    if ((threadIdx.x & 31) == 0 && dsum) atomicAdd(&c->edges, (unsigned long long)dsum);
  }
}

__global__ void init_kernel(uint32_t* dist, uint8_t* upd, int32_t n, int32_t src) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    dist[v] = v == src ? 0u : kInf;
    upd[v] = v == src ? 1 : 0;
  }
}

// Reached vertices and their out-edges (m_r), for the stats.
__global__ void __launch_bounds__(kGenThreads) reached_kernel(Graph g, SibCtr* c) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t span = (((int64_t)g.n + 31) / 32) * 32;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < span; v += stride) {
    uint32_t r = 0, deg = 0;
    if (v < g.n && g.dist[v] < kInf) {
      r = 1;
      const int32_t s = g.row[v], e = g.row[v + 1];
      deg = (e >= s) ? (uint32_t)(e - s) : 0u;
    }
    const uint32_t rs = __reduce_add_sync(0xffffffffu, r);
    const uint32_t ds = __reduce_add_sync(0xffffffffu, deg);
    if ((threadIdx.x & 31) == 0) {
      if (rs) atomicAdd(&c->reached, rs);
      if (ds) atomicAdd(&c->reached_edges, (unsigned long long)ds);
    }
  }
}


// Per-device cached workspace.
struct SibWork {
  unsigned long long ctx_id = 0;  // context the cached buffers live in (nps_context_id)
  std::mutex mu;
  cudaStream_t stream = nullptr;
  int32_t* q = nullptr;
  size_t q_n = 0;
  int32_t* buf = nullptr;
  size_t buf_n = 0;
  uint8_t* upd = nullptr;
  size_t upd_n = 0;
  int32_t* row = nullptr;
  size_t row_n = 0;
  int32_t* col = nullptr;
  size_t col_n = 0;
  uint32_t* w = nullptr;
  size_t w_n = 0;
  uint32_t* dist = nullptr;
  size_t dist_n = 0;
  SibCtr* ctr = nullptr;
  SibCtr* snap = nullptr;  // pinned: [0], [1] per-chunk snapshots, [2] final
  cudaEvent_t ev[4] = {};
  cudaEvent_t chunk_ev[2] = {};
  bool pending_limit = false;
  int sms = 0;
};

std::mutex g_sib_mu;
std::vector<SibWork*> g_sib;

SibWork* sib_work(int device) {
  std::lock_guard<std::mutex> lk(g_sib_mu);
  if ((int)g_sib.size() <= device) g_sib.resize(device + 1, nullptr);
  {
    const unsigned long long id = nps_context_id(device);
    if (g_sib[device] && id != 0 && g_sib[device]->ctx_id != id) g_sib[device] = nullptr;  // device reset: abandoned
    if (!g_sib[device]) {
      g_sib[device] = new SibWork();
      g_sib[device]->ctx_id = id;
    }
  }
  return g_sib[device];
}


nps_status setup(SibWork* W, int device) {
  if (!W->stream) NPS_CUDA_RETURN(cudaStreamCreateWithFlags(&W->stream, cudaStreamNonBlocking));
  if (!W->ctr) NPS_CUDA_RETURN(cudaMalloc((void**)&W->ctr, sizeof(SibCtr)));
  if (!W->snap) NPS_CUDA_RETURN(cudaMallocHost((void**)&W->snap, 3 * sizeof(SibCtr)));
  if (!W->ev[0]) {
    for (auto& e : W->ev) NPS_CUDA_RETURN(cudaEventCreate(&e));
    for (auto& e : W->chunk_ev) NPS_CUDA_RETURN(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  if (!W->sms) NPS_CUDA_RETURN(cudaDeviceGetAttribute(&W->sms, cudaDevAttrMultiProcessorCount, device));
  return NPS_OK;
}

struct Launch {
  int sol;
  Graph g;
  int32_t* q;
  int32_t* buf;
  uint32_t slice;
  int32_t threshold;
  int bs, grid, row_grid, gen_grid;
  SibCtr* c;
};

// Enqueue iteration `it` of solution L.sol.
nps_status enqueue_iteration(const Launch& L, int it, cudaStream_t s) {
  const int cur = it & 1;
  switch (L.sol) {
    case NPS_SOLUTION_TQUEUE:
      row_per_thread_kernel<kThreadOnly><<<L.grid, L.bs, 0, s>>>(L.g, L.q, it, L.threshold, nullptr, 0, L.c);
      gen_queue_kernel<false><<<L.gen_grid, kGenThreads, 0, s>>>(L.g, L.q, it, L.threshold, L.c);
      break;
    case NPS_SOLUTION_DUAL_QUEUE:
      // small rows: the front of the queue (qlo); large rows: the back (qhi), one CTA each
      row_per_thread_kernel<kThreadOnly><<<L.grid, L.bs, 0, s>>>(L.g, L.q, it, L.threshold, nullptr, 0, L.c);
      row_per_cta_kernel<<<L.row_grid, kRowCta, 0, s>>>(L.g, L.q + (L.g.n - 1), -1, &L.c->qhi[cur], 0, L.c);
      gen_queue_kernel<true><<<L.gen_grid, kGenThreads, 0, s>>>(L.g, L.q, it, L.threshold, L.c);
      break;
    case NPS_SOLUTION_SHARED_DELAYED:
      row_per_thread_kernel<kSharedDelayed><<<L.grid, L.bs, 0, s>>>(L.g, L.q, it, L.threshold, nullptr, 0, L.c);
      gen_queue_kernel<false><<<L.gen_grid, kGenThreads, 0, s>>>(L.g, L.q, it, L.threshold, L.c);
      break;
    case NPS_SOLUTION_GLOBAL_DELAYED:
      row_per_thread_kernel<kGlobalDelayed><<<L.grid, L.bs, 0, s>>>(L.g, L.q, it, L.threshold, L.buf, 0, L.c);
      row_per_cta_kernel<<<L.row_grid, kRowCta, 0, s>>>(L.g, L.buf, 1, &L.c->hlen, 0, L.c);
      gen_queue_kernel<false><<<L.gen_grid, kGenThreads, 0, s>>>(L.g, L.q, it, L.threshold, L.c);
      break;
    case NPS_SOLUTION_NP_NAIVE:
      row_per_thread_kernel<kNestedNaive><<<L.grid, L.bs, 0, s>>>(L.g, L.q, it, L.threshold, nullptr, 0, L.c);
      gen_queue_kernel<false><<<L.gen_grid, kGenThreads, 0, s>>>(L.g, L.q, it, L.threshold, L.c);
      break;
    case NPS_SOLUTION_NP_OPT:
      row_per_thread_kernel<kNestedPerBlock><<<L.grid, L.bs, 0, s>>>(L.g, L.q, it, L.threshold, L.buf, L.slice,
                                                                     L.c);
      gen_queue_kernel<false><<<L.gen_grid, kGenThreads, 0, s>>>(L.g, L.q, it, L.threshold, L.c);
      break;
    default:
      return nps_fail(NPS_ERR_INVALID_ARG, "solution must be 0..6");
  }
  NPS_CUDA_RETURN(cudaGetLastError());
  return NPS_OK;
}

nps_status check_solution_params(int32_t solution, const nps_params& p) {
  if (solution < 0 || solution > 6) return nps_fail(NPS_ERR_INVALID_ARG, "solution must be 0..6");
  if (p.threshold < 1) return nps_fail(NPS_ERR_INVALID_ARG, "threshold must be >= 1");
  if (p.block_size < 64 || p.block_size > kMaxBlock || p.block_size % 32)
    return nps_fail(NPS_ERR_INVALID_ARG, "block_size must be a multiple of 32 in [64, 1024]");
  if (!(p.timeout_s > 0) || p.timeout_s > 3600) return nps_fail(NPS_ERR_INVALID_ARG, "timeout_s must be in (0, 3600]");
  return NPS_OK;
}

// The iteration loop on device arrays; dist/upd hold the initial state.
nps_status run(SibWork* W, int32_t sol, const Graph& g, const nps_params& p, cudaStream_t s, nps_stats* st,
               nps_solution_info* info) {
  const auto t0 = std::chrono::steady_clock::now();
  const int bs = p.block_size;
  const int64_t n = g.n;
  Launch L;
  L.sol = sol;
  L.g = g;
  L.threshold = p.threshold;
  L.bs = bs;
  L.grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + bs - 1) / bs, (int64_t)W->sms * (2048 / bs)));
  L.row_grid = (int)std::max<int64_t>(1, std::min<int64_t>(n, (int64_t)W->sms * 32));
  L.gen_grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + kGenThreads - 1) / kGenThreads, (int64_t)W->sms * 8));
  L.c = W->ctr;
  nps_status e;
  if ((e = nps_ensure(&W->q, &W->q_n, (size_t)n, s, "solution"))) return e;
  L.q = W->q;
  L.buf = nullptr;
  L.slice = 0;
  if (sol == NPS_SOLUTION_GLOBAL_DELAYED) {
    if ((e = nps_ensure(&W->buf, &W->buf_n, (size_t)n, s, "solution"))) return e;
    L.buf = W->buf;
  } else if (sol == NPS_SOLUTION_NP_OPT) {
    // a CTA sweeps at most bs * ceil(n / (grid * bs)) queue entries
    const int64_t sweeps = (n + (int64_t)L.grid * bs - 1) / ((int64_t)L.grid * bs);
    L.slice = (uint32_t)(sweeps * bs);
    if ((e = nps_ensure(&W->buf, &W->buf_n, (size_t)L.grid * L.slice, s, "solution"))) return e;
    L.buf = W->buf;
  }
  if ((sol == NPS_SOLUTION_NP_NAIVE || sol == NPS_SOLUTION_NP_OPT) && !W->pending_limit) {
    size_t have = 0;
    NPS_CUDA_RETURN(cudaDeviceGetLimit(&have, cudaLimitDevRuntimePendingLaunchCount));
    // not fatal: with the default limit more launches are refused and walked by their parent thread
    if (have < kPendingLaunches && cudaDeviceSetLimit(cudaLimitDevRuntimePendingLaunchCount, kPendingLaunches) != cudaSuccess)
      cudaGetLastError();
    W->pending_limit = true;
  }
  NPS_CUDA_RETURN(cudaMemsetAsync(W->ctr, 0, sizeof(SibCtr), s));
  NPS_CUDA_RETURN(cudaEventRecord(W->ev[1], s));
  if (sol == NPS_SOLUTION_DUAL_QUEUE)
    gen_queue_kernel<true><<<L.gen_grid, kGenThreads, 0, s>>>(g, L.q, -1, L.threshold, L.c);
  else
    gen_queue_kernel<false><<<L.gen_grid, kGenThreads, 0, s>>>(g, L.q, -1, L.threshold, L.c);
  NPS_CUDA_RETURN(cudaGetLastError());

  // chunks of iterations; the counters of chunk k are read while chunk k + 1 runs
  const int64_t max_iter = 2 * n + 64;
  int64_t it = 0;
  int chunk = 4, k = 0;
  uint32_t reads = 0;
  bool done = false;
  while (!done) {
    for (int j = 0; j < chunk; ++j)
      if ((e = enqueue_iteration(L, (int)((it + j) & 1), s))) return e;  // kernels use the parity only
    it += chunk;
    NPS_CUDA_RETURN(cudaMemcpyAsync(&W->snap[k & 1], W->ctr, sizeof(SibCtr), cudaMemcpyDeviceToHost, s));
    NPS_CUDA_RETURN(cudaEventRecord(W->chunk_ev[k & 1], s));
    if (k > 0) {
      NPS_CUDA_RETURN(cudaEventSynchronize(W->chunk_ev[(k - 1) & 1]));
      ++reads;
      const SibCtr& sn = W->snap[(k - 1) & 1];
      const int par = (int)((it - chunk) & 1);  // parity of the first iteration of chunk k
      if (sn.status) break;
      if (sn.qlo[par] + sn.qhi[par] == 0) done = true;
    }
    ++k;
    chunk = std::min(chunk * 2, kMaxChunk);
    if (!done && it > max_iter) {
      cudaStreamSynchronize(s);
      return nps_fail(NPS_ERR_CAPACITY, "solution did not converge within 2n + 64 iterations");
    }
    if (!done && std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > p.timeout_s) {
      cudaStreamSynchronize(s);
      return nps_fail(NPS_ERR_TIMEOUT, "solution exceeded timeout_s");
    }
  }
  NPS_CUDA_RETURN(cudaEventRecord(W->ev[2], s));
  reached_kernel<<<L.gen_grid, kGenThreads, 0, s>>>(g, L.c);
  NPS_CUDA_RETURN(cudaGetLastError());
  NPS_CUDA_RETURN(cudaMemcpyAsync(&W->snap[2], W->ctr, sizeof(SibCtr), cudaMemcpyDeviceToHost, s));
  NPS_CUDA_RETURN(cudaStreamSynchronize(s));
  const SibCtr& f = W->snap[2];
  if (st) {
    st->iterations = f.iterations;
    st->edges_scanned = f.edges;
    st->vertices_processed = f.processed;
    st->reached = f.reached;
    st->reached_edges = f.reached_edges;
    st->status = (int32_t)f.status;
    st->grid_ctas = L.grid;
    cudaEventElapsedTime(&st->kernel_ms, W->ev[1], W->ev[2]);
  }
  if (info) {
    info->deferred = f.deferred;
    info->child_launches = f.launches;
    info->launch_fallbacks = f.fallbacks;
    info->host_reads = reads + 1;
  }
  if (f.status == NPS_ERR_FORMAT)
    return nps_fail(NPS_ERR_FORMAT, "malformed CSR: a row range or neighbour id is out of bounds");
  return NPS_OK;
}

nps_status device_setup(int device, SibWork** out) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return nps_fail(NPS_ERR_NO_DEVICE, "no CUDA device");
  }
  if (device < 0 || device >= count) return nps_fail(NPS_ERR_INVALID_ARG, "device ordinal out of range");
  NPS_CUDA_RETURN(cudaSetDevice(device));
  *out = sib_work(device);
  return NPS_OK;
}

}  // namespace

extern "C" nps_status nps_sssp_solution_state(int32_t solution, const int32_t* d_row_ptr, const int32_t* d_col,
                                              const uint32_t* d_w, int32_t n, int64_t m, uint32_t* d_cost,
                                              uint8_t* d_update, const nps_params* pin, nps_stats* st,
                                              nps_solution_info* info) {
  nps_clear_error();
  nps_params p;
  if (pin) p = *pin;
  else nps_params_default(&p);
  if (info) memset(info, 0, sizeof(*info));
  if (solution == NPS_SOLUTION_CONSOLIDATE) {
    p.device_ptrs = 1;
    return nps_sssp_state(d_row_ptr, d_col, d_w, n, m, d_cost, d_update, &p, st);
  }
  nps_status e = check_solution_params(solution, p);
  if (e) return e;
  if (n <= 0) return nps_fail(NPS_ERR_INVALID_ARG, "n must be positive");
  if (m < 0 || m >= (int64_t)INT32_MAX) return nps_fail(NPS_ERR_INVALID_ARG, "m must be in [0, 2^31-1)");
  if (!d_row_ptr || !d_cost || !d_update || (m > 0 && (!d_col || !d_w))) return nps_fail(NPS_ERR_INVALID_ARG, "null array");
  SibWork* W = nullptr;
  if ((e = device_setup(p.device, &W))) return e;
  std::lock_guard<std::mutex> lk(W->mu);
  if ((e = setup(W, p.device))) return e;
  cudaStream_t s = p.stream ? (cudaStream_t)p.stream : W->stream;
  if (st) memset(st, 0, sizeof(*st));
  NPS_CUDA_RETURN(cudaEventRecord(W->ev[0], s));
  Graph g{d_row_ptr, d_col, d_w, d_cost, d_update, n, m};
  if ((e = run(W, solution, g, p, s, st, info))) return e;
  NPS_CUDA_RETURN(cudaEventRecord(W->ev[3], s));
  NPS_CUDA_RETURN(cudaStreamSynchronize(s));
  if (st) cudaEventElapsedTime(&st->total_ms, W->ev[0], W->ev[3]);
  return NPS_OK;
}

extern "C" nps_status nps_sssp_solution(int32_t solution, const int32_t* row_ptr, const int32_t* col,
                                        const uint32_t* w, int32_t n, int64_t m, int32_t src, const nps_params* pin,
                                        uint32_t* dist_out, nps_stats* st, nps_solution_info* info) {
  nps_clear_error();
  nps_params p;
  if (pin) p = *pin;
  else nps_params_default(&p);
  if (info) memset(info, 0, sizeof(*info));
  if (solution == NPS_SOLUTION_CONSOLIDATE) return nps_sssp(row_ptr, col, w, n, m, src, &p, dist_out, st);
  nps_status e = check_solution_params(solution, p);
  if (e) return e;
  if (n <= 0) return nps_fail(NPS_ERR_INVALID_ARG, "n must be positive");
  if (m < 0 || m >= (int64_t)INT32_MAX) return nps_fail(NPS_ERR_INVALID_ARG, "m must be in [0, 2^31-1)");
  if (src < 0 || src >= n) return nps_fail(NPS_ERR_INVALID_ARG, "source vertex out of range");
  if (!row_ptr || !dist_out || (m > 0 && (!col || !w))) return nps_fail(NPS_ERR_INVALID_ARG, "null array");
  if (!p.device_ptrs && (row_ptr[0] != 0 || row_ptr[n] != (int32_t)m))
    return nps_fail(NPS_ERR_FORMAT, "malformed CSR: row_ptr[0] must be 0 and row_ptr[n] must be m");
  SibWork* W = nullptr;
  if ((e = device_setup(p.device, &W))) return e;
  std::lock_guard<std::mutex> lk(W->mu);
  if ((e = setup(W, p.device))) return e;
  cudaStream_t s = p.stream ? (cudaStream_t)p.stream : W->stream;
  if (st) memset(st, 0, sizeof(*st));
  NPS_CUDA_RETURN(cudaEventRecord(W->ev[0], s));
  const int32_t *drow = row_ptr, *dcol = col;
  const uint32_t* dw = w;
  uint32_t* ddist = dist_out;
  if (!p.device_ptrs) {
    if ((e = nps_ensure(&W->row, &W->row_n, (size_t)n + 1, s, "solution")) || (e = nps_ensure(&W->col, &W->col_n, (size_t)m, s, "solution")) ||
        (e = nps_ensure(&W->w, &W->w_n, (size_t)m, s, "solution")) || (e = nps_ensure(&W->dist, &W->dist_n, (size_t)n, s, "solution")))
      return e;
    NPS_CUDA_RETURN(cudaMemcpyAsync(W->row, row_ptr, sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice, s));
    if (m > 0) {
      NPS_CUDA_RETURN(cudaMemcpyAsync(W->col, col, sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice, s));
      NPS_CUDA_RETURN(cudaMemcpyAsync(W->w, w, sizeof(uint32_t) * (size_t)m, cudaMemcpyHostToDevice, s));
    }
    drow = W->row;
    dcol = W->col;
    dw = W->w;
    ddist = W->dist;
  }
  if ((e = nps_ensure(&W->upd, &W->upd_n, (size_t)n, s, "solution"))) return e;
  const int ig = (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)n + 255) / 256, (int64_t)W->sms * 8));
  init_kernel<<<ig, 256, 0, s>>>(ddist, W->upd, n, src);
  NPS_CUDA_RETURN(cudaGetLastError());
  Graph g{drow, dcol, dw, ddist, W->upd, n, m};
  if ((e = run(W, solution, g, p, s, st, info))) return e;
  if (!p.device_ptrs)
    NPS_CUDA_RETURN(cudaMemcpyAsync(dist_out, ddist, sizeof(uint32_t) * (size_t)n, cudaMemcpyDeviceToHost, s));
  NPS_CUDA_RETURN(cudaEventRecord(W->ev[3], s));
  NPS_CUDA_RETURN(cudaStreamSynchronize(s));
  if (st) cudaEventElapsedTime(&st->total_ms, W->ev[0], W->ev[3]);
  return NPS_OK;
}
