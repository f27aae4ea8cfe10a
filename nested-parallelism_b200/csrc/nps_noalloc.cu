// nps_sssp_noalloc(): single-source shortest paths without any allocation.
//
// Who needs it.  Some callers cannot allocate device memory at the moment they
// want a shortest-path answer: services that reserve all device memory up front
// in their own pool and must not let a library grow its footprint or stall
// other streams with a device-synchronising cudaMalloc, and plug-in hosts that
// forbid allocator calls from their callbacks.  The regular entry points keep a
// per-context workspace that grows with cudaMalloc the first time a larger
// graph arrives; this one never calls cudaMalloc, cudaFree, cudaMallocHost,
// stream or event creation.
//
// The call waits for its kernel: it copies the run's counters to the host and
// synchronises the stream to return a status.  On a stream that is being captured
// it returns NPS_ERR_INVALID_ARG before doing anything.
//
// How.  The workspace the persistent kernel needs (queues, dedupe stamps, the
// grid-tier list, counters, barrier words) lives in one file-scope
// `static __device__` array of NPS_NOALLOC_SCRATCH_BYTES (10 MiB), sized for
// graphs of up to NPS_NOALLOC_MAX_VERTICES vertices (edges are not limited).
// Every GPU that loads libnps holds this array until the process exits.  The
// array's host-side name is only a stand-in for the symbol, not a device
// address, so the first call on each device resolves the address with
// cudaGetSymbolAddress (that device current) and caches it; make that first call
// before any stream capture begins.  After a cudaDeviceReset() of that device the
// module is loaded anew, so the address is resolved again on the next call.
//
// Sharing.  All calls on a device share the one array and it keeps the state of
// the last call: counters and barrier words are cleared at the start of each
// call; the dedupe stamps carry a base that advances from call to call (and are
// cleared after a call that failed).  Two calls whose kernels overlap on the GPU
// (different streams or host threads without ordering) race on the array and
// give wrong results; order them on one stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "nps.h"
#include "nps_device.cuh"
#include "nps_internal.h"

namespace {

using nps::Counters;
using nps::InstDesc;
using nps::LaunchParams;
using nps::TeamDesc;

constexpr size_t kMaxV = NPS_NOALLOC_MAX_VERTICES;
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Layout of the scratch array (byte offsets, 256-byte aligned).
constexpr size_t kBarWords = 4096;  // one team of up to 2032 CTAs (2 + 2032/16 lines of 32 words)
constexpr size_t kOffCtr = 0;
constexpr size_t kOffBar = align256(kOffCtr + sizeof(Counters));
constexpr size_t kOffAbort = align256(kOffBar + kBarWords * sizeof(uint32_t));
constexpr size_t kOffTeam = align256(kOffAbort + 128);
constexpr size_t kClearBytes = kOffTeam;  // counters, barrier words, abort flag
constexpr size_t kOffStamp = align256(kOffTeam + sizeof(TeamDesc));
constexpr size_t kOffMarks = align256(kOffStamp + sizeof(uint32_t));
constexpr size_t kOffQueues = align256(kOffMarks + 3 * kMaxV * sizeof(uint32_t));
constexpr size_t kOffHeavy = align256(kOffQueues + 6 * kMaxV * sizeof(int32_t));
constexpr size_t kItemCap = 65536;  // grid-tier work items per half (larger items for larger m)
constexpr size_t kOffItems = align256(kOffHeavy + 2 * kMaxV * sizeof(int4));
constexpr size_t kScratchBytes = align256(kOffItems + 2 * kItemCap * sizeof(int32_t));
static_assert(kScratchBytes <= NPS_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds NPS_NOALLOC_SCRATCH_BYTES");

}  // namespace

// The scratch, NPS_NOALLOC_SCRATCH_BYTES long (the layout above uses the first
// kScratchBytes).  Host code must not take its address directly (that would be
// the host shadow, not device memory); see scratch_address().
static __device__ __align__(256) unsigned char g_nps_noalloc_scratch[NPS_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_addr[kMaxDevices] = {nullptr};
unsigned long long g_addr_ctx[kMaxDevices] = {0};  // context each address was resolved in

// Device address of the scratch on `device` (which must be current), resolved
// again when the device was reset since (the module is loaded anew then).
nps_status scratch_address(int device, unsigned char** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  const unsigned long long id = nps_context_id(device);
  if (!g_addr[device] || (id != 0 && id != g_addr_ctx[device])) {
    g_addr[device] = nullptr;
    g_addr_ctx[device] = id;
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_nps_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return nps_fail(NPS_ERR_CUDA, std::string("noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_addr[device] = (unsigned char*)p;
  }
  *out = g_addr[device];
  return NPS_OK;
}

using KernelFn = void (*)(const LaunchParams, const InstDesc);

KernelFn pick(int bs) {
  switch (bs) {
    case 128: return nps::sssp_persistent_kernel<128, true>;
    case 256: return nps::sssp_persistent_kernel<256, true>;
    case 512: return nps::sssp_persistent_kernel<512, true>;
    default: return nullptr;
  }
}

// Restores the caller's current device on every return path.
struct DeviceGuard {
  int prev = -1;
  DeviceGuard() { cudaGetDevice(&prev); }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

#define NA_CUDA(call)                                                                   \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return nps_fail(NPS_ERR_CUDA, std::string("noalloc: " #call ": ") + cudaGetErrorString(e_)); \
  } while (0)

}  // namespace

extern "C" nps_status nps_sssp_noalloc(const int32_t* d_row_ptr, const int32_t* d_col, const uint32_t* d_w,
                                       int32_t n, int64_t m, int32_t src, uint32_t* d_dist,
                                       const nps_params* pin, nps_stats* st) {
  nps_clear_error();
  nps_params p;
  if (pin) p = *pin;
  else nps_params_default(&p);
  if (st) memset(st, 0, sizeof(*st));
  if (n <= 0) return nps_fail(NPS_ERR_INVALID_ARG, "noalloc: n must be positive");
  if ((size_t)n > kMaxV)
    return nps_fail(NPS_ERR_CAPACITY, "noalloc: graph has " + std::to_string(n) +
                                          " vertices; this entry point's static scratch holds at most " +
                                          std::to_string(kMaxV) + " (use nps_sssp for larger graphs)");
  if (m < 0 || m >= (int64_t)INT32_MAX) return nps_fail(NPS_ERR_INVALID_ARG, "noalloc: m must be in [0, 2^31-1)");
  if (src < 0 || src >= n) return nps_fail(NPS_ERR_INVALID_ARG, "noalloc: source vertex out of range");
  if (!d_row_ptr || !d_dist || (m > 0 && (!d_col || !d_w))) return nps_fail(NPS_ERR_INVALID_ARG, "noalloc: null array");
  if (p.level < 0 || p.level > 3 || p.threshold < 1 || p.delta >= NPS_INF || !(p.timeout_s > 0) ||
      p.timeout_s > 3600 || p.ctas_per_sm < 0 ||
      (p.level == NPS_LEVEL_HYBRID && (p.block_threshold < p.threshold || p.grid_threshold < p.block_threshold)))
    return nps_fail(NPS_ERR_INVALID_ARG, "noalloc: invalid parameters");
  if (p.device < 0 || p.device >= kMaxDevices) return nps_fail(NPS_ERR_INVALID_ARG, "noalloc: device out of range");
  KernelFn k = pick(p.block_size);
  if (!k) return nps_fail(NPS_ERR_INVALID_ARG, "noalloc: block_size must be 128, 256 or 512");

  DeviceGuard guard;
  NA_CUDA(cudaSetDevice(p.device));
  cudaStream_t s = (cudaStream_t)p.stream;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  NA_CUDA(cudaStreamIsCapturing(s, &cap));
  if (cap != cudaStreamCaptureStatusNone)
    return nps_fail(NPS_ERR_INVALID_ARG,
                    "noalloc: the stream is being captured; this call synchronises the stream to return its "
                    "status, which a capture does not allow");
  int major = 0, sms = 0, coop = 0;
  NA_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, p.device));
  NA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p.device));
  NA_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, p.device));
  if (major != 10 || !coop) return nps_fail(NPS_ERR_NO_DEVICE, "noalloc: needs an sm_100a device with cooperative launch");
  const void* policy = nps_policy_device_weights(p.device);
  if (p.policy == NPS_POLICY_LEARNED && !policy)
    return nps_fail(NPS_ERR_INVALID_ARG, "noalloc: learned policy requested but no weights loaded");

  unsigned char* base = nullptr;
  nps_status e = scratch_address(p.device, &base);
  if (e) return e;
  int nb = 0;
  NA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void*)k, p.block_size, 0));
  if (nb <= 0) return nps_fail(NPS_ERR_CUDA, "noalloc: kernel does not fit on an SM");
  if (p.ctas_per_sm > 0 && p.ctas_per_sm < nb) nb = p.ctas_per_sm;
  const int grid = nb * sms;
  const size_t stride = 32 * (2 + (size_t)(grid + nps::kBarGroup - 1) / nps::kBarGroup);
  if (stride > kBarWords) return nps_fail(NPS_ERR_CAPACITY, "noalloc: too many CTAs for the barrier area");

  Counters* ctr = (Counters*)(base + kOffCtr);
  uint32_t* marks = (uint32_t*)(base + kOffMarks);
  int32_t* queues = (int32_t*)(base + kOffQueues);
  const size_t nn = (size_t)n;

  InstDesc d;
  memset(&d, 0, sizeof(d));
  d.row_ptr = d_row_ptr;
  d.col = d_col;
  d.w = d_w;
  d.dist = d_dist;
  d.n = n;
  d.m = (int32_t)m;
  d.src = src;
  d.mode = 0;
  for (int j = 0; j < 2; ++j) {
    d.q[j] = queues + (0 + j) * kMaxV;
    d.fq[j] = queues + (2 + j) * kMaxV;
    d.sq[j] = queues + (4 + j) * kMaxV;
  }
  d.mark = marks;
  d.fmark = marks + kMaxV;
  d.smark = marks + 2 * kMaxV;
  d.heavy = (int4*)(base + kOffHeavy);
  d.qcap = (uint32_t)nn;
  d.hcap = (uint32_t)(2 * nn);  // two halves of up to n grid-tier rows each
  nps_heavy_items(m, nn, kItemCap, &d.icap, &d.item_shift);
  d.hitem = (int32_t*)(base + kOffItems);
  d.ctr = ctr;
  d.stamp_base = (uint32_t*)(base + kOffStamp);
  d.trace = nullptr;  // no trace buffer: that would need an allocation
  d.vec_ok = (((uintptr_t)d_col | (uintptr_t)d_w) & 15) == 0;
  d.level = p.level;
  d.t1 = p.threshold;
  d.t2 = p.block_threshold;
  d.t3 = p.grid_threshold;
  d.delta = p.delta;
  d.policy = nps_policy_for(p, m);
  d.light_heavy = p.light_heavy != 0;
  d.local_rounds = p.local_rounds < 0 ? 0 : (p.local_rounds > 1024 ? 1024 : p.local_rounds);
  d.order_degree = p.order_degree < 0 ? 0 : p.order_degree;
  d.dsched = p.delta_schedule;
  d.sort_push = p.sort_at_push < -1 ? -1 : (p.sort_at_push > 1 ? 1 : p.sort_at_push);

  const TeamDesc td{0, grid, 0, 1};
  LaunchParams lp;
  memset(&lp, 0, sizeof(lp));
  lp.teams = (const TeamDesc*)(base + kOffTeam);
  lp.n_teams = 1;
  lp.fault_inject_wait = p.reserved[0] == 1;
  lp.test_disagree = p.reserved[0] == 2;
  lp.bar = (uint32_t*)(base + kOffBar);
  lp.bar_stride = (uint32_t)stride;
  lp.abort_flag = (uint32_t*)(base + kOffAbort);
  lp.timeout_ns = (unsigned long long)(p.timeout_s * 1e9);
  lp.run_budget_ns = (unsigned long long)(std::max(60.0, 30.0 * p.timeout_s) * 1e9);
  lp.policy = (const nps::PolicyDev*)policy;

  // counters, barrier words and the abort flag start at zero on every call
  NA_CUDA(cudaMemsetAsync(base + kOffCtr, 0, kClearBytes, s));
  NA_CUDA(cudaMemcpyAsync(base + kOffTeam, &td, sizeof(td), cudaMemcpyHostToDevice, s));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)p.block_size);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  NA_CUDA(cudaLaunchKernelEx(&cfg, k, lp, d));
  Counters h;
  NA_CUDA(cudaMemcpyAsync(&h, ctr, sizeof(h), cudaMemcpyDeviceToHost, s));
  NA_CUDA(cudaStreamSynchronize(s));
  if (h.status != NPS_OK) {
    // a stopped launch never advanced the stamp base: clear stamps and base
    NA_CUDA(cudaMemsetAsync(marks, 0, 3 * kMaxV * sizeof(uint32_t), s));
    NA_CUDA(cudaMemsetAsync(base + kOffStamp, 0, sizeof(uint32_t), s));
    NA_CUDA(cudaStreamSynchronize(s));
  }
  if (st) {
    st->iterations = h.iterations;
    st->buckets = h.buckets;
    st->edges_scanned = h.edges;
    st->improvements = h.improvements;
    st->vertices_processed = h.processed;
    st->reached = h.reached + 1;
    st->status = (int32_t)h.status;
    st->grid_ctas = grid;
    st->policy_used = (uint32_t)d.policy;
  }
  switch (h.status) {
    case NPS_OK: return NPS_OK;
    case NPS_ERR_TIMEOUT: return nps_fail(NPS_ERR_TIMEOUT, "noalloc: a bounded wait in the persistent kernel timed out");
    case NPS_ERR_FORMAT: return nps_fail(NPS_ERR_FORMAT, "noalloc: malformed CSR");
    case NPS_ERR_CAPACITY: return nps_fail(NPS_ERR_CAPACITY, "noalloc: device queue capacity exceeded");
    default: return nps_fail((nps_status)h.status, "noalloc: device reported error " + std::to_string(h.status));
  }
}
