// Host engine of the SSSP library: contexts, workspaces, the cooperative
// launch of the persistent kernel and the C ABI of include/nps.h.
//
// Boundary.  nps_sssp()/nps_sssp_ctx() take the place of the reference's
// SSSP_GPU() + sssp_np_consolidate_gpu() pair (apps/sssp/src/gpu/
// sssp_wrapper.cu:548-583, :475-546): where the reference resets the device,
// allocates five arrays and two queues, and loops on the host until the queue
// is empty, a call here reuses a cached per-context workspace and makes exactly
// one persistent launch.  Errors come back as status codes instead of exit().
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <queue>
#include <set>
#include <string>
#include <vector>

#include "nps.h"
#include "nps_device.cuh"
#include "nps_internal.h"

using nps::Counters;
using nps::InstDesc;
using nps::LaunchParams;
using nps::PolicyDev;
using nps::TeamDesc;

// ---------------------------------------------------------------------------
// errors

namespace {
thread_local std::string g_last_error;
}

nps_status nps_fail(nps_status code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
void nps_clear_error() { g_last_error.clear(); }

extern "C" const char* nps_last_error_string(void) { return g_last_error.c_str(); }

// Driver entry points through the runtime (the library links no libcuda).
unsigned long long nps_context_id(int device) {
  using GetCurrentFn = CUresult (*)(CUcontext*);
  using GetIdFn = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrentFn get_current = nullptr;
  static GetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetIdFn>(f);
    cudaGetLastError();
  });
  if (!get_current || !get_id) return 0;
  if (cudaSetDevice(device) != cudaSuccess || cudaFree(nullptr) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  CUcontext cu = nullptr;
  unsigned long long id = 0;
  if (get_current(&cu) != CUDA_SUCCESS || !cu || get_id(cu, &id) != CUDA_SUCCESS) return 0;
  return id;
}
extern "C" int32_t nps_abi_version(void) { return NPS_ABI_VERSION; }

#define NPS_CUDA(call)                                                                       \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return nps_fail(NPS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)

extern "C" void nps_params_default(nps_params* p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->level = NPS_LEVEL_BLOCK;
  p->threshold = 64;
  p->block_threshold = 256;
  p->grid_threshold = 4096;
  p->block_size = 256;
  p->ctas_per_sm = 0;
  p->delta = 0;
  p->policy = NPS_POLICY_PLAIN;
  p->device_ptrs = 0;
  p->device = 0;
  p->stream = nullptr;
  p->timeout_s = 10.0;
  p->trace = 0;
  p->light_heavy = 1;
}

namespace {

// ---------------------------------------------------------------------------
// device properties

struct DevInfo {
  bool ok = false;
  int sms = 0;
  int major = 0, minor = 0;
  bool coop = false;
};

nps_status device_info(int dev, DevInfo* out) {
  static std::mutex mu;
  static std::vector<DevInfo> cache;
  std::lock_guard<std::mutex> lk(mu);
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return nps_fail(NPS_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
  }
  if (dev < 0 || dev >= count) return nps_fail(NPS_ERR_INVALID_ARG, "device ordinal out of range");
  if ((int)cache.size() < count) cache.resize(count);
  if (!cache[dev].ok) {
    cudaDeviceProp pr;
    NPS_CUDA(cudaGetDeviceProperties(&pr, dev));
    int coop = 0;
    NPS_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    cache[dev].sms = pr.multiProcessorCount;
    cache[dev].major = pr.major;
    cache[dev].minor = pr.minor;
    cache[dev].coop = coop != 0;
    cache[dev].ok = true;
  }
  *out = cache[dev];
  if (out->major != 10)
    return nps_fail(NPS_ERR_NO_DEVICE, "libnps is built for sm_100a (B200); device has compute capability " +
                                           std::to_string(out->major) + "." + std::to_string(out->minor));
  if (!out->coop) return nps_fail(NPS_ERR_NO_DEVICE, "device does not support cooperative launch");
  return NPS_OK;
}

// ---------------------------------------------------------------------------
// kernel selection

using KernelFn = void (*)(const LaunchParams, const InstDesc);

KernelFn pick_kernel(int bs, bool single, bool async = false) {
  switch (bs) {
    case 128:
      return async ? nps::sssp_persistent_kernel<128, true, true>
                   : (single ? nps::sssp_persistent_kernel<128, true> : nps::sssp_persistent_kernel<128, false>);
    case 256:
      return async ? nps::sssp_persistent_kernel<256, true, true>
                   : (single ? nps::sssp_persistent_kernel<256, true> : nps::sssp_persistent_kernel<256, false>);
    case 512:
      return async ? nps::sssp_persistent_kernel<512, true, true>
                   : (single ? nps::sssp_persistent_kernel<512, true> : nps::sssp_persistent_kernel<512, false>);
    default: return nullptr;
  }
}

// Shared-memory carveout: the smallest split that still holds `nb` resident
// CTAs, so the rest of the SM's 256 KB of L1/shared storage caches the
// distance array (the pre-check loads of hub vertices hit in L1 instead of
// queueing on one L2 slice).  Done once per (device, kernel); occupancy is
// checked again and the default restored if the split would lower it.
cudaError_t set_carveout(int dev, KernelFn k, int bs, int nb) {
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  std::lock_guard<std::mutex> lk(mu);
  if (!done.insert({dev, (const void*)k}).second) return cudaSuccess;
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, (const void*)k);
  if (e != cudaSuccess) return e;
  int smem_sm = 0, reserved = 0;
  if ((e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev)) != cudaSuccess) return e;
  if (smem_sm <= 0) return cudaSuccess;
  const size_t need = (size_t)nb * (fa.sharedSizeBytes + (size_t)reserved);
  int pct = (int)((need * 100 + (size_t)smem_sm - 1) / (size_t)smem_sm);
  pct = std::min(100, std::max(1, pct));
  if ((e = cudaFuncSetAttribute((const void*)k, cudaFuncAttributePreferredSharedMemoryCarveout, pct)) != cudaSuccess)
    return e;
  int nb2 = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb2, (const void*)k, bs, 0)) != cudaSuccess) return e;
  if (nb2 < nb) return cudaFuncSetAttribute((const void*)k, cudaFuncAttributePreferredSharedMemoryCarveout, -1);
  return cudaSuccess;
}

nps_status grid_size(int dev, const DevInfo& di, int bs, bool single, int ctas_per_sm, int* grid,
                     bool async = false) {
  KernelFn k = pick_kernel(bs, single, async);
  if (!k) return nps_fail(NPS_ERR_INVALID_ARG, "block_size must be 128, 256 or 512");
  int nb = 0;
  NPS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void*)k, bs, 0));
  if (nb <= 0) return nps_fail(NPS_ERR_CUDA, "persistent kernel does not fit on an SM");
  NPS_CUDA(set_carveout(dev, k, bs, nb));
  if (ctas_per_sm > 0) nb = std::min(nb, ctas_per_sm);
  *grid = nb * di.sms;
  (void)dev;
  return NPS_OK;
}

// ---------------------------------------------------------------------------
// device buffers

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  nps_status ensure(size_t count, bool zero, cudaStream_t s) {
    if (count <= n && p) return NPS_OK;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      return nps_fail(NPS_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    n = count;
    if (zero) {
      e = cudaMemsetAsync(p, 0, std::max<size_t>(count, 1) * sizeof(T), s);
      if (e != cudaSuccess) return nps_fail(NPS_ERR_CUDA, cudaGetErrorString(e));
    }
    return NPS_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

// Control block: counters, barrier words and the abort flag share one
// allocation so a single memset clears them before each launch.  Layout:
//   Counters[n_inst] | barrier words, `stride` per team | abort flag (128 B) | team table (128 B)
struct Control {
  size_t n_inst = 0, n_teams = 0, stride = 0;
  char* base = nullptr;
  Control(size_t ni, size_t nt, int max_team_ctas)
      : n_inst(ni), n_teams(nt), stride(32 * (2 + (size_t)(max_team_ctas + nps::kBarGroup - 1) / nps::kBarGroup)) {}
  size_t counters_bytes() const { return n_inst * sizeof(Counters); }
  size_t bar_bytes() const { return n_teams * stride * sizeof(uint32_t); }
  Counters* ctr() const { return (Counters*)base; }
  uint32_t* bar() const { return (uint32_t*)(base + counters_bytes()); }
  uint32_t* abort_flag() const { return (uint32_t*)(base + counters_bytes() + bar_bytes()); }
  TeamDesc* team_table() const { return (TeamDesc*)(base + counters_bytes() + bar_bytes() + 128); }
  size_t clear_bytes() const { return counters_bytes() + bar_bytes() + 128; }
  size_t bytes() const { return clear_bytes() + 128; }
};

struct PolicyState {
  PolicyDev* dev = nullptr;
  PolicyDev host;                 // kept to upload again after a device reset
  unsigned long long ctx_id = 0;  // context `dev` was allocated in
  bool set = false;
};

std::mutex g_policy_mu;
std::vector<PolicyState> g_policy;

}  // namespace

struct nps_ctx {
  int device = 0;
  unsigned long long ctx_id = 0;  // context the cached state below lives in (nps_context_id)
  cudaStream_t stream = nullptr;
  DevInfo di;
  // per-instance workspace (single-instance calls)
  DevBuf<int32_t> q0, q1, f0, f1, s0, s1;
  DevBuf<uint32_t> mark, fmark, smark, stamp;
  DevBuf<int4> heavy;
  // work rings of the asynchronous schedule (tags and head/tail persist across runs)
  DevBuf<unsigned long long> nq;
  DevBuf<int4> segs;
  DevBuf<nps::RingState> rstate;
  bool rings_ready = false;
  DevBuf<char> control;
  DevBuf<nps_trace_rec> trace;
  uint32_t trace_count = 0;
  // graph staging for host-pointer calls
  DevBuf<int32_t> g_row, g_col;
  DevBuf<uint32_t> g_w, g_dist;
  DevBuf<uint8_t> g_wpack;     // weights packed to 1 or 2 bytes, widened into g_w
  uint8_t* h_wpack = nullptr;  // pinned staging of the packed weights
  size_t h_wpack_n = 0;
  // batch workspace
  DevBuf<int32_t> b_pool;
  DevBuf<uint32_t> b_stamp;
  DevBuf<int4> b_heavy;
  DevBuf<InstDesc> b_inst;
  DevBuf<TeamDesc> b_teams;
  DevBuf<int32_t> b_order;
  DevBuf<char> b_control;
  std::vector<InstDesc> b_inst_host;
  std::vector<nps_instance> b_key;
  nps_params b_params_key{};
  int b_grid = 0, b_bs = 0;
  int b_nteams = 0;
  cudaGraphExec_t b_graph = nullptr;
  // Re-balancing of the teams of an unchanged instance set (one instance per team):
  // stage 0 splits CTAs by work; the solve times of the first two calls (taken with
  // different splits) calibrate a per-team model, after which the split is fixed.
  int b_stage = 0;
  std::vector<int> b_inst_ctas;   // CTAs of each instance's team in the current split
  std::vector<double> b_t1, b_t2; // measured solve times (ms) of the first two calls
  std::vector<int> b_c1, b_c2;    // ... and their teams' CTAs
  std::vector<uint32_t> b_it1;    // iterations in the first call
  Counters* h_ctr = nullptr;  // pinned
  size_t h_ctr_n = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  std::mutex mu;
};

namespace {

nps_status ctx_init(nps_ctx* c, int device) {
  nps_status st = device_info(device, &c->di);
  if (st != NPS_OK) return st;
  c->device = device;
  NPS_CUDA(cudaSetDevice(device));
  NPS_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  for (auto& e : c->ev) NPS_CUDA(cudaEventCreate(&e));
  return NPS_OK;
}

void ctx_release(nps_ctx* c) {
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto* b : {&c->q0, &c->q1, &c->f0, &c->f1, &c->s0, &c->s1, &c->g_row, &c->g_col, &c->b_pool, &c->b_order})
    b->release();
  for (auto* b : {&c->mark, &c->fmark, &c->smark, &c->stamp, &c->g_w, &c->g_dist, &c->b_stamp}) b->release();
  c->heavy.release();
  c->nq.release();
  c->segs.release();
  c->rstate.release();
  c->b_heavy.release();
  c->control.release();
  c->b_control.release();
  c->trace.release();
  c->b_inst.release();
  c->b_teams.release();
  if (c->b_graph) cudaGraphExecDestroy(c->b_graph);
  c->b_graph = nullptr;
  if (c->h_ctr) cudaFreeHost(c->h_ctr);
  c->h_ctr = nullptr;
  if (c->h_wpack) cudaFreeHost(c->h_wpack);
  c->h_wpack = nullptr;
  c->h_wpack_n = 0;
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  c->stream = nullptr;
}

nps_status ensure_pinned_counters(nps_ctx* c, size_t n) {
  if (c->h_ctr_n >= n && c->h_ctr) return NPS_OK;
  if (c->h_ctr) cudaFreeHost(c->h_ctr);
  c->h_ctr = nullptr;
  c->h_ctr_n = 0;
  NPS_CUDA(cudaMallocHost(&c->h_ctr, n * sizeof(Counters)));
  c->h_ctr_n = n;
  return NPS_OK;
}

// Default context per device (created on first use, lives until exit).
std::mutex g_ctx_mu;
std::vector<nps_ctx*> g_default_ctx;

nps_status default_ctx(int device, nps_ctx** out) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (device < 0) return nps_fail(NPS_ERR_INVALID_ARG, "device ordinal out of range");
  if ((int)g_default_ctx.size() <= device) g_default_ctx.resize(device + 1, nullptr);
  const unsigned long long id = nps_context_id(device);
  if (g_default_ctx[device] && id != 0 && g_default_ctx[device]->ctx_id != id) {
    // the device was reset: its buffers, stream and events died with the old
    // context, so the cached state is dropped without being freed
    g_default_ctx[device] = nullptr;
  }
  if (!g_default_ctx[device]) {
    auto* c = new nps_ctx();
    nps_status st = ctx_init(c, device);
    if (st != NPS_OK) {
      delete c;
      return st;
    }
    c->ctx_id = id;
    g_default_ctx[device] = c;
  }
  *out = g_default_ctx[device];
  return NPS_OK;
}

nps_status check_params(const nps_params& p) {
  if (p.level < 0 || p.level > 3) return nps_fail(NPS_ERR_INVALID_ARG, "level must be 0..3");
  if (p.threshold < 1) return nps_fail(NPS_ERR_INVALID_ARG, "threshold must be >= 1");
  if (p.level == NPS_LEVEL_HYBRID && (p.block_threshold < p.threshold || p.grid_threshold < p.block_threshold))
    return nps_fail(NPS_ERR_INVALID_ARG, "hybrid thresholds must satisfy threshold <= block_threshold <= grid_threshold");
  if (p.block_size != 128 && p.block_size != 256 && p.block_size != 512)
    return nps_fail(NPS_ERR_INVALID_ARG, "block_size must be 128, 256 or 512");
  if (p.ctas_per_sm < 0) return nps_fail(NPS_ERR_INVALID_ARG, "ctas_per_sm must be >= 0");
  if (p.policy != NPS_POLICY_PLAIN && p.policy != NPS_POLICY_LEARNED)
    return nps_fail(NPS_ERR_INVALID_ARG, "policy must be 0 (plain) or 1 (learned)");
  if (!(p.timeout_s > 0) || p.timeout_s > 3600) return nps_fail(NPS_ERR_INVALID_ARG, "timeout_s must be in (0, 3600]");
  if (p.delta >= NPS_INF) return nps_fail(NPS_ERR_INVALID_ARG, "delta must be < 2^30");
  if (p.local_rounds < 0 || p.local_rounds > 1024) return nps_fail(NPS_ERR_INVALID_ARG, "local_rounds must be in [0, 1024]");
  if (p.order_degree < 0) return nps_fail(NPS_ERR_INVALID_ARG, "order_degree must be >= 0");
  if (p.sort_at_push < -1 || p.sort_at_push > 1) return nps_fail(NPS_ERR_INVALID_ARG, "sort_at_push must be -1, 0 or 1");
  if (p.reserved2 != 0) return nps_fail(NPS_ERR_INVALID_ARG, "reserved2 must be 0");
  return NPS_OK;
}

// Smallest degree that can reach the grid tier under these parameters
// (bounds the number of grid-tier entries per iteration by m / t + 1).
int32_t min_grid_threshold(const nps_params& p) {
  int32_t t = p.level == NPS_LEVEL_HYBRID ? p.grid_threshold : p.threshold;
  if (p.policy == NPS_POLICY_LEARNED) t = std::min(t, p.threshold);
  return std::max(t, 1);
}

uint32_t heavy_capacity(int32_t n, int64_t m, const nps_params& p) {
  // two halves (iteration parity), each bounded by the vertex count and m / t
  int64_t per = std::min<int64_t>((int64_t)n, m / min_grid_threshold(p) + 1);
  return (uint32_t)std::max<int64_t>(2 * per, 2);
}

PolicyDev* policy_ptr(int device) {
  std::lock_guard<std::mutex> lk(g_policy_mu);
  if ((int)g_policy.size() <= device || !g_policy[device].set) return nullptr;
  PolicyState& ps = g_policy[device];
  const unsigned long long id = nps_context_id(device);
  if (id != 0 && id != ps.ctx_id) {
    // the device was reset since the weights were uploaded: upload them again
    ps.dev = nullptr;
    if (cudaMalloc(&ps.dev, sizeof(PolicyDev)) != cudaSuccess ||
        cudaMemcpy(ps.dev, &ps.host, sizeof(PolicyDev), cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaGetLastError();
      ps.dev = nullptr;
      ps.set = false;
      return nullptr;
    }
    ps.ctx_id = id;
  }
  return ps.dev;
}

void fill_thresholds(const nps_params& p, InstDesc& d) {
  d.level = p.level;
  d.t1 = p.threshold;
  d.t2 = p.block_threshold;
  d.t3 = p.grid_threshold;
  d.delta = p.delta;
  d.policy = p.policy;
  d.light_heavy = p.light_heavy != 0;
  d.local_rounds = p.local_rounds;
  d.order_degree = p.order_degree;
  d.dsched = p.delta_schedule;
  d.sort_push = p.sort_at_push;
}

// Whether a single-instance call runs the asynchronous schedule: requested, tiers
// at the grid level (or chosen by the learned policy, which then runs grid tiers),
// no warp-local rounds and no light/heavy split in effect.
bool use_async(const nps_params& p) {
  if (p.schedule != NPS_SCHEDULE_ASYNC) return false;
  if (p.level != NPS_LEVEL_GRID && p.policy != NPS_POLICY_LEARNED) return false;
  if (p.local_rounds != 0) return false;
  const bool split = p.light_heavy && (p.delta != 0 || p.delta_schedule != 0 || p.policy == NPS_POLICY_LEARNED);
  return !split;
}

size_t pow2_at_least(size_t x) {
  size_t r = 1;
  while (r < x) r <<= 1;
  return r;
}

// Ring capacities: the near ring holds every vertex at most once at a time plus the
// claims of every warp, so 2n + 2^18 slots leave it at most half full; the segment
// ring is sized so that half of it holds 2 m / 256 + 2^11 segments (pushes back off
// to the pushing warp beyond half).
size_t near_ring_slots(int32_t n) { return pow2_at_least((size_t)2 * (size_t)n + ((size_t)1 << 18)); }
size_t seg_ring_slots(int64_t m) { return pow2_at_least(std::max<size_t>((size_t)1 << 14, (size_t)m / 64 + 4096)); }

// Tags to their first lap (slot i free for index i), heads and tails to zero.
__global__ void ring_init_kernel(unsigned long long* nq, uint32_t qc, int4* seg, uint32_t sc, nps::RingState* rs) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < qc; i += stride)
    nq[i] = ((unsigned long long)i << 32) | 0xffffffffull;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < sc; i += stride) seg[i] = make_int4(0, 0, 0, (int)i);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    rs->nq_head = rs->nq_tail = 0;
    rs->seg_head = rs->seg_tail = 0;
  }
}

// Whole-launch bound: 30 per-wait timeouts, at least 60 s.
unsigned long long run_budget_ns(const nps_params& p) {
  return (unsigned long long)(std::max(60.0, 30.0 * p.timeout_s) * 1e9);
}

nps_status launch(nps_ctx* c, cudaStream_t s, int bs, bool single, int grid, const LaunchParams& lp,
                  const InstDesc& inst) {
  KernelFn k = pick_kernel(bs, single, single && inst.async != 0);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)bs);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  (void)c;
  NPS_CUDA(cudaLaunchKernelEx(&cfg, k, lp, inst));
  return NPS_OK;
}

nps_status status_from_device(uint32_t st) {
  switch (st) {
    case NPS_OK: return NPS_OK;
    case NPS_ERR_CAPACITY: return nps_fail(NPS_ERR_CAPACITY, "device queue capacity exceeded");
    case NPS_ERR_TIMEOUT: return nps_fail(NPS_ERR_TIMEOUT, "a bounded wait in the persistent kernel timed out");
    case NPS_ERR_FORMAT: return nps_fail(NPS_ERR_FORMAT, "malformed CSR: a row range or neighbour id is out of bounds");
    case NPS_ERR_INTERNAL:
      return nps_fail(NPS_ERR_INTERNAL, "the persistent kernel's CTAs took different schedule decisions");
    default: return nps_fail((nps_status)st, "device reported error " + std::to_string(st));
  }
}

// Core single-instance run on device-resident arrays.
nps_status run_single(nps_ctx* c, cudaStream_t s, const int32_t* row, const int32_t* col, const uint32_t* w,
                      int32_t n, int64_t m, int32_t src, uint32_t* dist, uint8_t* update, int mode,
                      const nps_params& p, nps_stats* st, bool time_it) {
  const size_t nn = (size_t)n;
  nps_status e;
  if ((e = c->q0.ensure(nn, false, s)) || (e = c->q1.ensure(nn, false, s)) || (e = c->f0.ensure(nn, false, s)) ||
      (e = c->f1.ensure(nn, false, s)) || (e = c->s0.ensure(nn, false, s)) || (e = c->s1.ensure(nn, false, s)))
    return e;
  const bool grow_marks = c->mark.n < nn;
  if ((e = c->mark.ensure(nn, true, s)) || (e = c->fmark.ensure(nn, true, s)) || (e = c->smark.ensure(nn, true, s)))
    return e;
  if ((e = c->stamp.ensure(1, grow_marks || !c->stamp.p, s))) return e;
  if (grow_marks) NPS_CUDA(cudaMemsetAsync(c->stamp.p, 0, sizeof(uint32_t), s));
  const uint32_t hcap = heavy_capacity(n, m, p);
  uint32_t icap = 0, ishift = 0;
  nps_heavy_items(m, hcap / 2, 0, &icap, &ishift);
  if ((e = c->heavy.ensure(nps_heavy_slots(hcap, icap), false, s))) return e;
  int grid = 0;
  if ((e = grid_size(c->device, c->di, p.block_size, true, p.ctas_per_sm, &grid, use_async(p)))) return e;
  Control ctl(1, 1, grid);
  if ((e = c->control.ensure(ctl.bytes(), false, s))) return e;
  ctl.base = c->control.p;
  if (p.trace) {
    if ((e = c->trace.ensure(1 << 16, false, s))) return e;
  }
  if ((e = ensure_pinned_counters(c, 1))) return e;
  const bool async = use_async(p);
  size_t qc = 0, sc = 0;
  if (async) {
    qc = near_ring_slots(n);
    sc = seg_ring_slots(m);
    if (qc > ((size_t)1 << 31) || sc > ((size_t)1 << 31))
      return nps_fail(NPS_ERR_INVALID_ARG, "asynchronous schedule: graph too large for 32-bit ring indices");
    const void *q0 = c->nq.p, *s0 = c->segs.p;
    if ((e = c->nq.ensure(qc, false, s)) || (e = c->segs.ensure(sc, false, s)) || (e = c->rstate.ensure(1, false, s)))
      return e;
    if (c->nq.p != q0 || c->segs.p != s0) c->rings_ready = false;
    qc = c->nq.n;
    sc = c->segs.n;
    if (!c->rings_ready) {
      ring_init_kernel<<<c->di.sms * 4, 256, 0, s>>>(c->nq.p, (uint32_t)qc, c->segs.p, (uint32_t)sc, c->rstate.p);
      NPS_CUDA(cudaGetLastError());
      c->rings_ready = true;
    }
  }

  InstDesc d;
  memset(&d, 0, sizeof(d));
  d.row_ptr = row;
  d.col = col;
  d.w = w;
  d.dist = dist;
  d.update = update;
  d.n = n;
  d.m = (int32_t)m;
  d.src = src;
  d.mode = mode;
  d.q[0] = c->q0.p;
  d.q[1] = c->q1.p;
  d.fq[0] = c->f0.p;
  d.fq[1] = c->f1.p;
  d.mark = c->mark.p;
  d.fmark = c->fmark.p;
  d.smark = c->smark.p;
  d.sq[0] = c->s0.p;
  d.sq[1] = c->s1.p;
  d.heavy = c->heavy.p;
  d.hitem = (int32_t*)(c->heavy.p + hcap);
  d.icap = icap;
  d.item_shift = ishift;
  d.qcap = (uint32_t)n;
  d.hcap = hcap;
  d.ctr = ctl.ctr();
  d.stamp_base = c->stamp.p;
  d.trace = p.trace ? c->trace.p : nullptr;
  d.trace_cap = p.trace ? (uint32_t)c->trace.n : 0;
  d.vec_ok = (((uintptr_t)col | (uintptr_t)w) & 15) == 0;
  fill_thresholds(p, d);
  d.policy = nps_policy_for(p, m);  // the learned policy only where it gains
  if (st) st->policy_used = (uint32_t)d.policy;
  if (async) {
    d.async = 1;
    d.nq = c->nq.p;
    d.nq_mask = (uint32_t)(qc - 1);
    d.seg = c->segs.p;
    d.seg_mask = (uint32_t)(sc - 1);
    d.rs = c->rstate.p;
    d.wait_ns = (unsigned long long)(p.timeout_s * 1e9);
  }

  TeamDesc td{0, grid, 0, 1};
  // single-instance launches read the team table from a small device buffer
  static_assert(sizeof(TeamDesc) == 16, "team descriptor layout");
  LaunchParams lp;
  memset(&lp, 0, sizeof(lp));
  lp.inst = nullptr;
  lp.order = nullptr;
  lp.n_teams = 1;
  lp.fault_inject_wait = p.reserved[0] == 1;
  lp.test_disagree = p.reserved[0] == 2;
  lp.bar = ctl.bar();
  lp.bar_stride = (uint32_t)ctl.stride;
  lp.abort_flag = ctl.abort_flag();
  lp.timeout_ns = (unsigned long long)(p.timeout_s * 1e9);
  lp.run_budget_ns = run_budget_ns(p);
  lp.policy = policy_ptr(c->device);
  if (p.policy == NPS_POLICY_LEARNED && !lp.policy)
    return nps_fail(NPS_ERR_INVALID_ARG, "learned policy requested but no weights loaded (nps_policy_set_weights)");
  TeamDesc* d_team = ctl.team_table();
  lp.teams = d_team;

  NPS_CUDA(cudaMemsetAsync(ctl.base, 0, ctl.clear_bytes(), s));
  NPS_CUDA(cudaMemcpyAsync(d_team, &td, sizeof(td), cudaMemcpyHostToDevice, s));
  if (time_it) NPS_CUDA(cudaEventRecord(c->ev[1], s));
  if ((e = launch(c, s, p.block_size, true, grid, lp, d))) return e;
  if (time_it) NPS_CUDA(cudaEventRecord(c->ev[2], s));
  NPS_CUDA(cudaMemcpyAsync(c->h_ctr, ctl.ctr(), sizeof(Counters), cudaMemcpyDeviceToHost, s));
  if (st) st->grid_ctas = grid;
  return NPS_OK;
}

// A launch that stopped early never advanced its stamp base, so its stamps
// could collide with the next run's: clear marks and base after any failure.
void reset_stamps(nps_ctx* c, cudaStream_t s) {
  c->rings_ready = false;  // a stopped asynchronous run leaves its ring claims unreleased
  if (c->mark.p) cudaMemsetAsync(c->mark.p, 0, c->mark.n * sizeof(uint32_t), s);
  if (c->fmark.p) cudaMemsetAsync(c->fmark.p, 0, c->fmark.n * sizeof(uint32_t), s);
  if (c->smark.p) cudaMemsetAsync(c->smark.p, 0, c->smark.n * sizeof(uint32_t), s);
  if (c->stamp.p) cudaMemsetAsync(c->stamp.p, 0, sizeof(uint32_t), s);
  cudaStreamSynchronize(s);
}

void fill_stats(const Counters& k, nps_stats* st) {
  if (!st) return;
  st->iterations = k.iterations;
  st->buckets = k.buckets;
  st->edges_scanned = k.edges;
  st->improvements = k.improvements;
  st->vertices_processed = k.processed;
  st->status = (int32_t)k.status;
  for (int i = 0; i < 9; ++i) st->phase_cycles[i] = k.prof[i];
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI

extern "C" nps_status nps_ctx_create(int32_t device, nps_ctx** out) {
  if (!out) return nps_fail(NPS_ERR_INVALID_ARG, "ctx_create: null output");
  auto* c = new nps_ctx();
  nps_status st = ctx_init(c, device);
  if (st != NPS_OK) {
    ctx_release(c);
    delete c;
    return st;
  }
  *out = c;
  return NPS_OK;
}

extern "C" nps_status nps_ctx_destroy(nps_ctx* ctx) {
  if (!ctx) return NPS_OK;
  ctx_release(ctx);
  delete ctx;
  return NPS_OK;
}

namespace {

// Breadth-first levels from unit-weight distances: unreachable vertices (NPS_INF)
// get the reference's UNDEFINED (apps/bfs-rec/src/gpu/bfs_rec.h:13).
__global__ void bfs_levels_kernel(uint32_t* d, int32_t n) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
    if (d[v] >= NPS_INF) d[v] = (uint32_t)NPS_BFS_UNDEFINED;
}

// Host-pointer calls move weights that fit in 8 or 16 bits across PCIe packed:
// one host pass (OpenMP) finds the largest weight and writes the low bytes to
// pinned staging while the row and column copies are in flight, and the device
// widens them back to 32 bits.  The kernel reads the same 32-bit weights either
// way.  On R-MAT 22 (weights in [1, 255]) the weight copy shrinks from 261 to
// 65 MB; the pass takes 2.7 ms on 16 cores, inside the 4.8 ms column copy.
constexpr int64_t kPackMinEdges = 1 << 20;  // below this the pass and the extra launch cost more

// Largest weight decides the width: 1 (all < 256), 2 (all < 65536) or 4 (no packing).
// h receives m bytes (width 1) or 2m bytes (width 2).
int pack_weights(const uint32_t* w, int64_t m, uint8_t* h) {
  uint32_t mx = 0;
#pragma omp parallel for reduction(max : mx) schedule(static)
  for (int64_t i = 0; i < m; ++i) {
    const uint32_t x = w[i];
    mx = x > mx ? x : mx;
    h[i] = (uint8_t)x;
  }
  if (mx <= 0xFFu) return 1;
  if (mx > 0xFFFFu) return 4;
  uint16_t* h16 = reinterpret_cast<uint16_t*>(h);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m; ++i) h16[i] = (uint16_t)w[i];
  return 2;
}

// dst[i] = src[i] for m packed weights of `bytes` (1 or 2) bytes each; four per thread.
__global__ void widen_weights_kernel(const uint8_t* __restrict__ src, int bytes, uint32_t* __restrict__ dst,
                                     int64_t m) {
  const int64_t q = m / 4;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < q; i += stride) {
    uint4 o;
    if (bytes == 1) {
      const uchar4 b = reinterpret_cast<const uchar4*>(src)[i];
      o = make_uint4(b.x, b.y, b.z, b.w);
    } else {
      const ushort4 b = reinterpret_cast<const ushort4*>(src)[i];
      o = make_uint4(b.x, b.y, b.z, b.w);
    }
    reinterpret_cast<uint4*>(dst)[i] = o;
  }
  for (int64_t i = 4 * q + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride)
    dst[i] = bytes == 1 ? src[i] : reinterpret_cast<const uint16_t*>(src)[i];
}

nps_status ensure_pinned_wpack(nps_ctx* c, size_t bytes) {
  if (c->h_wpack_n >= bytes && c->h_wpack) return NPS_OK;
  if (c->h_wpack) cudaFreeHost(c->h_wpack);
  c->h_wpack = nullptr;
  c->h_wpack_n = 0;
  const cudaError_t err = cudaMallocHost(&c->h_wpack, bytes);
  if (err != cudaSuccess) {
    cudaGetLastError();
    c->h_wpack = nullptr;
    return nps_fail(NPS_ERR_OOM, std::string("pinned weight staging: cudaMallocHost: ") + cudaGetErrorString(err));
  }
  c->h_wpack_n = bytes;
  return NPS_OK;
}

// nps_sssp_ctx, and with bfs = true nps_bfs (w unused: every edge weighs 1).
nps_status sssp_ctx_impl(nps_ctx* c, const int32_t* row_ptr, const int32_t* col, const uint32_t* w, int32_t n,
                         int64_t m, int32_t src, const nps_params* pin, uint32_t* dist_out, nps_stats* st,
                         bool bfs) {
  nps_clear_error();
  nps_params p;
  if (pin) p = *pin;
  else nps_params_default(&p);
  if (!c) return nps_fail(NPS_ERR_INVALID_ARG, "null context");
  nps_status e = check_params(p);
  if (e) return e;
  if (n <= 0) return nps_fail(NPS_ERR_INVALID_ARG, "n must be positive");
  if (m < 0 || m >= (int64_t)INT32_MAX) return nps_fail(NPS_ERR_INVALID_ARG, "m must be in [0, 2^31-1)");
  if (src < 0 || src >= n) return nps_fail(NPS_ERR_INVALID_ARG, "source vertex out of range");
  if (bfs) w = nullptr;
  if (!row_ptr || !dist_out || (m > 0 && (!col || (!w && !bfs)))) return nps_fail(NPS_ERR_INVALID_ARG, "null array");
  std::lock_guard<std::mutex> lk(c->mu);
  NPS_CUDA(cudaSetDevice(c->device));
  cudaStream_t s = p.stream ? (cudaStream_t)p.stream : c->stream;
  if (st) memset(st, 0, sizeof(*st));

  const int32_t *drow = row_ptr, *dcol = col;
  const uint32_t* dw = w;
  uint32_t* ddist = dist_out;
  NPS_CUDA(cudaEventRecord(c->ev[0], s));
  if (!p.device_ptrs) {
    // host arrays: validate the CSR shape on the host, then stage on the device
    if (row_ptr[0] != 0 || row_ptr[n] != (int32_t)m)
      return nps_fail(NPS_ERR_FORMAT, "malformed CSR: row_ptr[0] must be 0 and row_ptr[n] must be m");
    if ((e = c->g_row.ensure((size_t)n + 1, false, s)) || (e = c->g_col.ensure((size_t)m, false, s)) ||
        (!bfs && (e = c->g_w.ensure((size_t)m, false, s))) || (e = c->g_dist.ensure((size_t)n, false, s)))
      return e;
    NPS_CUDA(cudaMemcpyAsync(c->g_row.p, row_ptr, sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice, s));
    if (m > 0) {
      NPS_CUDA(cudaMemcpyAsync(c->g_col.p, col, sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice, s));
      if (!bfs) {
        int wb = 4;
        if (m >= kPackMinEdges) {
          if (ensure_pinned_wpack(c, 2 * (size_t)m) == NPS_OK) {
            wb = pack_weights(w, m, c->h_wpack);  // overlaps the copies queued above
          } else {
            // no pinned staging of that size: copy the weights as they are
            cudaGetLastError();
            nps_clear_error();
          }
        }
        if (wb == 4) {
          NPS_CUDA(cudaMemcpyAsync(c->g_w.p, w, sizeof(uint32_t) * (size_t)m, cudaMemcpyHostToDevice, s));
        } else {
          if ((e = c->g_wpack.ensure((size_t)wb * (size_t)m, false, s))) return e;
          NPS_CUDA(cudaMemcpyAsync(c->g_wpack.p, c->h_wpack, (size_t)wb * (size_t)m, cudaMemcpyHostToDevice, s));
          const int wg = (int)std::min<int64_t>(((int64_t)m / 4 + 255) / 256 + 1, (int64_t)c->di.sms * 8);
          widen_weights_kernel<<<wg, 256, 0, s>>>(c->g_wpack.p, wb, c->g_w.p, m);
          NPS_CUDA(cudaGetLastError());
        }
      }
    }
    drow = c->g_row.p;
    dcol = c->g_col.p;
    dw = bfs ? nullptr : c->g_w.p;
    ddist = c->g_dist.p;
  }
  if ((e = run_single(c, s, drow, dcol, dw, n, m, src, ddist, nullptr, 0, p, st, true))) return e;
  if (bfs) {
    const int lg = (int)std::min<int64_t>(((int64_t)n + 255) / 256, (int64_t)c->di.sms * 8);
    bfs_levels_kernel<<<lg, 256, 0, s>>>(ddist, n);
    NPS_CUDA(cudaGetLastError());
  }
  if (!p.device_ptrs)
    NPS_CUDA(cudaMemcpyAsync(dist_out, ddist, sizeof(uint32_t) * (size_t)n, cudaMemcpyDeviceToHost, s));
  NPS_CUDA(cudaEventRecord(c->ev[3], s));
  NPS_CUDA(cudaStreamSynchronize(s));
  const Counters& k = *c->h_ctr;
  c->trace_count = p.trace ? std::min<uint32_t>(k.iterations, (uint32_t)c->trace.n) : 0;
  if (st) {
    fill_stats(k, st);
    cudaEventElapsedTime(&st->kernel_ms, c->ev[1], c->ev[2]);
    cudaEventElapsedTime(&st->total_ms, c->ev[0], c->ev[3]);
    st->reached = k.reached + 1;
  }
  if (k.status) reset_stamps(c, s);
  return status_from_device(k.status);
}

}  // namespace

extern "C" nps_status nps_sssp_ctx(nps_ctx* c, const int32_t* row_ptr, const int32_t* col,
                                   const uint32_t* w, int32_t n, int64_t m, int32_t src,
                                   const nps_params* pin, uint32_t* dist_out, nps_stats* st) {
  return sssp_ctx_impl(c, row_ptr, col, w, n, m, src, pin, dist_out, st, false);
}

extern "C" nps_status nps_bfs(const int32_t* row_ptr, const int32_t* col, int32_t n, int64_t m, int32_t src,
                              const nps_params* p, int32_t* level_out, nps_stats* st) {
  nps_clear_error();
  // arguments first, so a bad call is reported as such even without a device
  nps_status e0 = p ? check_params(*p) : NPS_OK;
  if (e0) return e0;
  if (n <= 0 || src < 0 || src >= n) return nps_fail(NPS_ERR_INVALID_ARG, "bfs: n must be positive and src in [0, n)");
  nps_ctx* c = nullptr;
  nps_status e = default_ctx(p ? p->device : 0, &c);
  if (e) return e;
  return sssp_ctx_impl(c, row_ptr, col, nullptr, n, m, src, p, reinterpret_cast<uint32_t*>(level_out), st, true);
}

extern "C" nps_status nps_sssp(const int32_t* row_ptr, const int32_t* col, const uint32_t* w, int32_t n,
                               int64_t m, int32_t src, const nps_params* p, uint32_t* dist_out,
                               nps_stats* st) {
  nps_clear_error();
  nps_ctx* c = nullptr;
  nps_status e = default_ctx(p ? p->device : 0, &c);
  if (e) return e;
  return nps_sssp_ctx(c, row_ptr, col, w, n, m, src, p, dist_out, st);
}

extern "C" nps_status nps_sssp_state(const int32_t* d_row_ptr, const int32_t* d_col, const uint32_t* d_w,
                                     int32_t n, int64_t m, uint32_t* d_cost, uint8_t* d_update,
                                     const nps_params* pin, nps_stats* st) {
  nps_clear_error();
  nps_params p;
  if (pin) p = *pin;
  else nps_params_default(&p);
  nps_status e = check_params(p);
  if (e) return e;
  if (n <= 0) return nps_fail(NPS_ERR_INVALID_ARG, "n must be positive");
  if (m < 0 || m >= (int64_t)INT32_MAX) return nps_fail(NPS_ERR_INVALID_ARG, "m must be in [0, 2^31-1)");
  if (!d_row_ptr || !d_cost || !d_update || (m > 0 && (!d_col || !d_w)))
    return nps_fail(NPS_ERR_INVALID_ARG, "null array");
  nps_ctx* c = nullptr;
  if ((e = default_ctx(p.device, &c))) return e;
  std::lock_guard<std::mutex> lk(c->mu);
  NPS_CUDA(cudaSetDevice(c->device));
  cudaStream_t s = p.stream ? (cudaStream_t)p.stream : c->stream;
  if (st) memset(st, 0, sizeof(*st));
  NPS_CUDA(cudaEventRecord(c->ev[0], s));
  if ((e = run_single(c, s, d_row_ptr, d_col, d_w, n, m, 0, d_cost, d_update, 1, p, st, true))) return e;
  NPS_CUDA(cudaEventRecord(c->ev[3], s));
  NPS_CUDA(cudaStreamSynchronize(s));
  const Counters& k = *c->h_ctr;
  c->trace_count = p.trace ? std::min<uint32_t>(k.iterations, (uint32_t)c->trace.n) : 0;
  if (st) {
    fill_stats(k, st);
    cudaEventElapsedTime(&st->kernel_ms, c->ev[1], c->ev[2]);
    cudaEventElapsedTime(&st->total_ms, c->ev[0], c->ev[3]);
    st->reached = k.reached;
  }
  if (k.status) reset_stamps(c, s);
  return status_from_device(k.status);
}

extern "C" nps_status nps_trace_read(int32_t device, nps_trace_rec* out, int32_t cap, int32_t* count) {
  nps_clear_error();
  if (!out || !count || cap < 0) return nps_fail(NPS_ERR_INVALID_ARG, "trace_read: bad argument");
  nps_ctx* c = nullptr;
  nps_status e = default_ctx(device, &c);
  if (e) return e;
  std::lock_guard<std::mutex> lk(c->mu);
  NPS_CUDA(cudaSetDevice(c->device));
  int32_t k = (int32_t)std::min<uint32_t>(c->trace_count, (uint32_t)cap);
  if (k > 0) NPS_CUDA(cudaMemcpy(out, c->trace.p, sizeof(nps_trace_rec) * (size_t)k, cudaMemcpyDeviceToHost));
  *count = k;
  return NPS_OK;
}

// ---------------------------------------------------------------------------
// batch

extern "C" nps_status nps_sssp_batch(const nps_instance* inst, int32_t count, const nps_params* pin,
                                     int32_t use_graph, nps_stats* per_instance, float* kernel_ms) {
  nps_clear_error();
  nps_params p;
  if (pin) p = *pin;
  else nps_params_default(&p);
  nps_status e = check_params(p);
  if (e) return e;
  if (!inst || count <= 0 || count > 65536) return nps_fail(NPS_ERR_INVALID_ARG, "batch: need 1..65536 instances");
  for (int i = 0; i < count; ++i) {
    const nps_instance& x = inst[i];
    if (x.n <= 0 || x.m < 0 || x.m >= (int64_t)INT32_MAX || x.src < 0 || x.src >= x.n || !x.row_ptr || !x.dist ||
        (x.m > 0 && (!x.col || !x.w)))
      return nps_fail(NPS_ERR_INVALID_ARG, "batch: instance " + std::to_string(i) + " is invalid");
  }
  nps_ctx* c = nullptr;
  if ((e = default_ctx(p.device, &c))) return e;
  std::lock_guard<std::mutex> lk(c->mu);
  NPS_CUDA(cudaSetDevice(c->device));
  cudaStream_t s = p.stream ? (cudaStream_t)p.stream : c->stream;
  int grid = 0;
  if ((e = grid_size(c->device, c->di, p.block_size, false, p.ctas_per_sm, &grid))) return e;

  const bool same_set = (int)c->b_key.size() == count && c->b_grid == grid && c->b_bs == p.block_size &&
                        memcmp(c->b_key.data(), inst, sizeof(nps_instance) * count) == 0 &&
                        memcmp(&c->b_params_key, &p, sizeof(p)) == 0;
  const int nteams = std::min(count, grid);
  if (!same_set || nteams != count) c->b_stage = 0;
  // stages 1 and 2 form the teams anew (a captured graph is captured again); stage 3
  // keeps the last split
  const bool rebalance = c->b_stage == 1 || c->b_stage == 2;
  const bool same = same_set && c->b_graph && !rebalance;
  Control ctl((size_t)count, (size_t)nteams, grid);

  if (!same) {
    if (c->b_graph) cudaGraphExecDestroy(c->b_graph);
    c->b_graph = nullptr;
    // workspace: per instance 4 queues of n int32 + marks carved from pools
    size_t q_total = 0, h_total = 0;
    std::vector<uint32_t> hcap(count), icap(count), ishift(count);
    for (int i = 0; i < count; ++i) {
      q_total += 6 * (size_t)inst[i].n;
      hcap[i] = heavy_capacity(inst[i].n, inst[i].m, p);
      nps_heavy_items(inst[i].m, hcap[i] / 2, 0, &icap[i], &ishift[i]);
      h_total += nps_heavy_slots(hcap[i], icap[i]);
    }
    size_t mk_total = 0;
    for (int i = 0; i < count; ++i) mk_total += 3 * (size_t)inst[i].n;
    if ((e = c->b_pool.ensure(q_total, false, s))) return e;
    const bool regrow = c->b_stamp.n < mk_total + (size_t)count;
    if ((e = c->b_stamp.ensure(mk_total + (size_t)count, true, s))) return e;
    if (!regrow) NPS_CUDA(cudaMemsetAsync(c->b_stamp.p, 0, sizeof(uint32_t) * (mk_total + count), s));
    if ((e = c->b_heavy.ensure(h_total, false, s))) return e;
    if ((e = c->b_control.ensure(ctl.bytes(), false, s))) return e;
    if ((e = c->b_inst.ensure((size_t)count, false, s))) return e;
    if ((e = c->b_teams.ensure((size_t)nteams, false, s))) return e;
    if ((e = c->b_order.ensure((size_t)count, false, s))) return e;
    ctl.base = c->b_control.p;

    // team formation: longest-processing-time assignment of instances to
    // nteams teams by work (m + n), then CTAs by water-filling on work per CTA
    std::vector<int> idx(count);
    for (int i = 0; i < count; ++i) idx[i] = i;
    auto work = [&](int i) { return (double)inst[i].m + (double)inst[i].n; };
    std::sort(idx.begin(), idx.end(), [&](int a, int b) { return work(a) > work(b) || (work(a) == work(b) && a < b); });
    std::vector<double> tw(nteams, 0.0);
    std::vector<std::vector<int>> members(nteams);
    for (int i : idx) {
      int t = (int)(std::min_element(tw.begin(), tw.end()) - tw.begin());
      tw[t] += work(i);
      members[t].push_back(i);
    }
    // CTAs: one per team, then each further CTA to the team whose predicted time is
    // largest.  The prediction is a + b / CTAs per team:
    //   stage 0   a = 0, b = work (m + n): minimises the largest work / CTAs ratio;
    //   stage 1   from the first call's solve time T1 with c1 CTAs: a = iterations x
    //             kIterFloorMs (the latency floor more CTAs do not shorten),
    //             b = (T1 - a) x c1;
    //   stage 2+  fitted through the first two calls' (c1, T1) and (c2, T2).
    constexpr double kIterFloorMs = 0.008;
    std::vector<double> fa(nteams, 0.0), fb(nteams, 0.0);
    for (int t = 0; t < nteams; ++t) {
      if (c->b_stage == 0) {
        fb[t] = tw[t];
        continue;
      }
      const int i = members[t][0];
      const double t1 = c->b_t1[i], c1 = std::max(c->b_c1[i], 1);
      fa[t] = c->b_it1[i] * kIterFloorMs;
      fb[t] = std::max(t1 - fa[t], 0.05 * t1) * c1;
      if (c->b_stage >= 2 && c->b_c2[i] != c->b_c1[i]) {
        const double t2 = c->b_t2[i], c2 = std::max(c->b_c2[i], 1);
        const double b = (t1 - t2) / (1.0 / c1 - 1.0 / c2);
        const double a = t1 - b / c1;
        if (b > 0 && a >= 0) {
          fa[t] = a;
          fb[t] = b;
        }
      }
    }
    std::vector<int> ctas(nteams, 1);
    {
      using Q = std::pair<double, int>;
      std::priority_queue<Q> pq;
      for (int t = 0; t < nteams; ++t) pq.push({fa[t] + fb[t], t});
      for (int left = grid - nteams; left > 0; --left) {
        const int t = pq.top().second;
        pq.pop();
        ctas[t] += 1;
        pq.push({fa[t] + fb[t] / ctas[t], t});
      }
    }
    c->b_inst_ctas.assign(count, 0);
    for (int t = 0; t < nteams; ++t)
      for (int i : members[t]) c->b_inst_ctas[i] = ctas[t];
    std::vector<TeamDesc> teams(nteams);
    std::vector<int32_t> order;
    int cb = 0;
    for (int t = 0; t < nteams; ++t) {
      teams[t].cta_begin = cb;
      teams[t].cta_count = ctas[t];
      teams[t].inst_begin = (int32_t)order.size();
      teams[t].inst_count = (int32_t)members[t].size();
      for (int i : members[t]) order.push_back(i);
      cb += ctas[t];
    }
    // descriptors
    c->b_inst_host.assign(count, InstDesc{});
    size_t qo = 0, ho = 0, mo = 0;
    uint32_t* stamps = c->b_stamp.p + mk_total;
    for (int i = 0; i < count; ++i) {
      InstDesc& d = c->b_inst_host[i];
      memset(&d, 0, sizeof(d));
      const nps_instance& x = inst[i];
      d.row_ptr = x.row_ptr;
      d.col = x.col;
      d.w = x.w;
      d.dist = x.dist;
      d.n = x.n;
      d.m = (int32_t)x.m;
      d.src = x.src;
      d.mode = 0;
      for (int k = 0; k < 2; ++k) {
        d.q[k] = c->b_pool.p + qo;
        qo += x.n;
        d.fq[k] = c->b_pool.p + qo;
        qo += x.n;
        d.sq[k] = c->b_pool.p + qo;
        qo += x.n;
      }
      d.mark = c->b_stamp.p + mo;
      mo += x.n;
      d.fmark = c->b_stamp.p + mo;
      mo += x.n;
      d.smark = c->b_stamp.p + mo;
      mo += x.n;
      d.heavy = c->b_heavy.p + ho;
      d.hitem = (int32_t*)(c->b_heavy.p + ho + hcap[i]);
      d.icap = icap[i];
      d.item_shift = ishift[i];
      d.hcap = hcap[i];
      ho += nps_heavy_slots(hcap[i], icap[i]);
      d.qcap = (uint32_t)x.n;
      d.ctr = ctl.ctr() + i;
      d.stamp_base = stamps + i;
      d.vec_ok = (((uintptr_t)x.col | (uintptr_t)x.w) & 15) == 0;
      fill_thresholds(p, d);
      d.policy = nps_policy_for(p, x.m);
    }
    NPS_CUDA(cudaMemcpyAsync(c->b_inst.p, c->b_inst_host.data(), sizeof(InstDesc) * count, cudaMemcpyHostToDevice, s));
    NPS_CUDA(cudaMemcpyAsync(c->b_teams.p, teams.data(), sizeof(TeamDesc) * nteams, cudaMemcpyHostToDevice, s));
    NPS_CUDA(cudaMemcpyAsync(c->b_order.p, order.data(), sizeof(int32_t) * count, cudaMemcpyHostToDevice, s));
    NPS_CUDA(cudaStreamSynchronize(s));  // host vectors above go out of scope
    c->b_key.assign(inst, inst + count);
    c->b_params_key = p;
    c->b_grid = grid;
    c->b_bs = p.block_size;
    c->b_nteams = nteams;
  }
  ctl.base = c->b_control.p;
  LaunchParams lp;
  memset(&lp, 0, sizeof(lp));
  lp.inst = c->b_inst.p;
  lp.order = c->b_order.p;
  lp.teams = c->b_teams.p;
  lp.n_teams = c->b_nteams;
  lp.fault_inject_wait = p.reserved[0] == 1;
  lp.test_disagree = p.reserved[0] == 2;
  lp.bar = ctl.bar();
  lp.bar_stride = (uint32_t)ctl.stride;
  lp.abort_flag = ctl.abort_flag();
  lp.timeout_ns = (unsigned long long)(p.timeout_s * 1e9);
  lp.run_budget_ns = run_budget_ns(p);
  lp.policy = policy_ptr(c->device);
  if (p.policy == NPS_POLICY_LEARNED && !lp.policy)
    return nps_fail(NPS_ERR_INVALID_ARG, "learned policy requested but no weights loaded (nps_policy_set_weights)");
  InstDesc dummy;
  memset(&dummy, 0, sizeof(dummy));
  if ((e = ensure_pinned_counters(c, (size_t)count))) return e;

  NPS_CUDA(cudaEventRecord(c->ev[1], s));
  if (use_graph) {
    if (!c->b_graph) {
      cudaGraph_t g = nullptr;
      NPS_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      cudaError_t ce = cudaMemsetAsync(ctl.base, 0, ctl.clear_bytes(), s);
      nps_status le = ce == cudaSuccess ? launch(c, s, p.block_size, false, grid, lp, dummy) : NPS_ERR_CUDA;
      cudaError_t ee = cudaStreamEndCapture(s, &g);
      if (ce != cudaSuccess) return nps_fail(NPS_ERR_CUDA, std::string("capture memset: ") + cudaGetErrorString(ce));
      if (le) {
        if (g) cudaGraphDestroy(g);
        return le;
      }
      if (ee != cudaSuccess) return nps_fail(NPS_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(ee));
      cudaError_t ie = cudaGraphInstantiate(&c->b_graph, g, 0);
      cudaGraphDestroy(g);
      if (ie != cudaSuccess) {
        c->b_graph = nullptr;
        return nps_fail(NPS_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ie));
      }
      NPS_CUDA(cudaEventRecord(c->ev[1], s));
    }
    NPS_CUDA(cudaGraphLaunch(c->b_graph, s));
  } else {
    NPS_CUDA(cudaMemsetAsync(ctl.base, 0, ctl.clear_bytes(), s));
    if ((e = launch(c, s, p.block_size, false, grid, lp, dummy))) return e;
  }
  NPS_CUDA(cudaEventRecord(c->ev[2], s));
  NPS_CUDA(cudaMemcpyAsync(c->h_ctr, ctl.ctr(), sizeof(Counters) * count, cudaMemcpyDeviceToHost, s));
  NPS_CUDA(cudaStreamSynchronize(s));
  if (kernel_ms) cudaEventElapsedTime(kernel_ms, c->ev[1], c->ev[2]);
  uint32_t first_err = 0;
  for (int i = 0; i < count; ++i) {
    const Counters& k = c->h_ctr[i];
    if (per_instance) {
      memset(&per_instance[i], 0, sizeof(nps_stats));
      fill_stats(k, &per_instance[i]);
      per_instance[i].reached = k.reached + 1;
      per_instance[i].grid_ctas = grid;
      per_instance[i].kernel_ms = (float)((double)k.solve_ns * 1e-6);  // device time to this instance's end
      per_instance[i].policy_used = (uint32_t)c->b_inst_host[i].policy;
    }
    if (k.status && !first_err) first_err = k.status;
  }
  if (!first_err && nteams == count && c->b_stage < 2) {
    std::vector<double>& t = c->b_stage == 0 ? c->b_t1 : c->b_t2;
    t.resize(count);
    for (int i = 0; i < count; ++i) t[i] = (double)c->h_ctr[i].solve_ns * 1e-6;
    if (c->b_stage == 0) {
      c->b_it1.resize(count);
      for (int i = 0; i < count; ++i) c->b_it1[i] = c->h_ctr[i].iterations;
      c->b_c1 = c->b_inst_ctas;
    } else {
      c->b_c2 = c->b_inst_ctas;
    }
  }
  if (!first_err && nteams == count && c->b_stage < 3) c->b_stage += 1;
  if (first_err) {  // stamps of an aborted batch may collide with the next run's
    cudaMemsetAsync(c->b_stamp.p, 0, c->b_stamp.n * sizeof(uint32_t), s);
    cudaStreamSynchronize(s);
  }
  return status_from_device(first_err);
}

// ---------------------------------------------------------------------------
// policy weights

extern "C" nps_status nps_policy_set_weights(int32_t device, const float* w1, const float* b1, const float* w2,
                                             const float* b2, const float* mean, const float* istd) {
  nps_clear_error();
  if (!w1 || !b1 || !w2 || !b2 || !mean || !istd) return nps_fail(NPS_ERR_INVALID_ARG, "policy: null array");
  DevInfo di;
  nps_status e = device_info(device, &di);
  if (e) return e;
  PolicyDev h;
  memset(&h, 0, sizeof(h));
  auto to_bf16 = [](float f) -> uint16_t {  // round to nearest even
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)(u >> 16);
    u += 0x7fffu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
  };
  for (int i = 0; i < NPS_MLP_HID * NPS_MLP_IN; ++i) h.w1[i] = to_bf16(w1[i]);
  for (int i = 0; i < NPS_MLP_OUT * NPS_MLP_HID; ++i) h.w2[i] = to_bf16(w2[i]);
  memcpy(h.b1, b1, sizeof(h.b1));
  memcpy(h.b2, b2, sizeof(h.b2));
  memcpy(h.mean, mean, sizeof(h.mean));
  memcpy(h.istd, istd, sizeof(h.istd));
  const unsigned long long id = nps_context_id(device);
  std::lock_guard<std::mutex> lk(g_policy_mu);
  if ((int)g_policy.size() <= device) g_policy.resize(device + 1);
  PolicyState& ps = g_policy[device];
  NPS_CUDA(cudaSetDevice(device));
  if (ps.dev && ps.ctx_id != id) ps.dev = nullptr;  // allocated before a device reset: gone
  if (!ps.dev) NPS_CUDA(cudaMalloc(&ps.dev, sizeof(PolicyDev)));
  NPS_CUDA(cudaMemcpy(ps.dev, &h, sizeof(h), cudaMemcpyHostToDevice));
  ps.host = h;
  ps.ctx_id = id;
  ps.set = true;
  return NPS_OK;
}

// Device copy of the learned-policy weights of `device`, or null when none were
// loaded (used by entry points in other translation units; allocates nothing).
const void* nps_policy_device_weights(int device) { return policy_ptr(device); }
