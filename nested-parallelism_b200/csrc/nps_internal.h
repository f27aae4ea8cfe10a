// Internal helpers shared by the host translation units of libnps.
#ifndef NPS_INTERNAL_H_
#define NPS_INTERNAL_H_

#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "nps.h"

// Records `msg` as this thread's last error (nps_last_error_string) and
// returns `code`, so call sites read `return nps_fail(NPS_ERR_..., "...")`.
nps_status nps_fail(nps_status code, const std::string& msg);
void nps_clear_error();

nps_status nps_build_csr(int32_t n, int64_t m, const int32_t* src, const int32_t* dst,
                         const uint32_t* w, bool dedupe, bool drop_self, nps_graph* out);

// Work items of one half of the grid-tier list: its flat chunk space holds at
// most m/4 + 2*entries chunks (row_chunks(s, e) <= (e - s)/4 + 2); an item is
// 2^shift chunks, shift >= 5 (6 from 10 M edges), the smallest that keeps the
// items within `cap` (0 = no limit).
inline void nps_heavy_items(int64_t m, uint64_t entries, uint64_t cap, uint32_t* icap, uint32_t* shift) {
  const uint64_t chunks = (uint64_t)(m < 0 ? 0 : m) / 4 + 2 * entries + 1;
  // 32-chunk items for graphs of under 10 M edges (more items to spread over the
  // team's warps), 64-chunk items above (less per-item overhead); measured on R-MAT 16-22
  uint32_t sh = m < 10000000 ? 5 : 6;
  while (cap && (chunks >> sh) + 2 > cap) ++sh;
  *shift = sh;
  *icap = (uint32_t)((chunks >> sh) + 2);
}

// int4 slots of the grid-tier buffer: hcap entries, then 2 * icap item starts.
inline size_t nps_heavy_slots(uint32_t hcap, uint32_t icap) { return (size_t)hcap + ((size_t)2 * icap + 3) / 4; }

// Returns NPS_ERR_CUDA, with the call and CUDA's message, when `call` fails.
#define NPS_CUDA_RETURN(call)                                                                  \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess)                                                                     \
      return nps_fail(NPS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));       \
  } while (0)

// Grows the device buffer *p (capacity *have elements) to hold `want` elements:
// a smaller buffer is freed -- after `s` drains, so no queued work still uses
// it -- and a new one allocated; its contents are not kept.  NPS_ERR_OOM (naming
// `what`) when the allocation fails.
template <class T>
nps_status nps_ensure(T** p, size_t* have, size_t want, cudaStream_t s, const char* what) {
  if (*p && *have >= want) return NPS_OK;
  if (*p) {
    cudaStreamSynchronize(s);
    cudaFree(*p);
  }
  *p = nullptr;
  *have = 0;
  cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(want, 1) * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return nps_fail(NPS_ERR_OOM, std::string(what) + " workspace: cudaMalloc: " + cudaGetErrorString(e));
  }
  *have = want;
  return NPS_OK;
}

// Identifier of the context current on `device` (made current, and created if a
// reset destroyed it), 0 if it cannot be read.  Every per-device cache of the
// library remembers the identifier it was built under: a different one means the
// device was reset since -- the reference's prepare_gpu() calls cudaDeviceReset()
// before every run -- and the cached device memory, streams and events are gone,
// so the cache is abandoned (not freed) and built again.
unsigned long long nps_context_id(int device);

// The policy a run on a graph of m edges uses: NPS_POLICY_LEARNED only from
// p.policy_min_edges edges (0 = NPS_POLICY_MIN_EDGES, negative = any size).
inline int32_t nps_policy_for(const nps_params& p, int64_t m) {
  if (p.policy != NPS_POLICY_LEARNED) return p.policy;
  const int64_t lim = p.policy_min_edges == 0 ? (int64_t)NPS_POLICY_MIN_EDGES : p.policy_min_edges;
  return (lim > 0 && m < lim) ? (int32_t)NPS_POLICY_PLAIN : (int32_t)NPS_POLICY_LEARNED;
}

// Device copy of the learned-policy weights of `device` (null if none loaded).
const void* nps_policy_device_weights(int device);

#endif  // NPS_INTERNAL_H_
