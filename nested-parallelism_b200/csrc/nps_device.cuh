// Device side of the B200 SSSP engine: one persistent cooperative kernel that
// runs the whole shortest-path computation of one or many graph instances with
// no host round trip.
//
// What it replaces (apps/sssp/src/gpu/ in the reference):
//   * the host loop of sssp_np_consolidate_gpu() (sssp_wrapper.cu:475-546), which
//     regenerates the frontier from the update[] byte map with an O(n) scan
//     (unorder_generateQueue_kernel, sssp_kernel.cu:648-658) and copies the queue
//     length to the host after every iteration;
//   * the consolidation kernels consolidate_{warp,block,grid}_dp_kernel
//     (sssp_kernel.cu:330-541), which buffer vertices of degree >= THRESHOLD per
//     warp / block / grid and launch a dynamic-parallelism child grid
//     (sssp_process_buffer, :82-104, or unorder_blockQueue_kernel, :57-78) per buffer.
// Here the buffers are consumed in-kernel by the warp, the CTA or every CTA of
// the team, and the frontier is a device queue filled by warp-aggregated
// appends, deduplicated with per-vertex stamps.
//
// Relaxation is the reference's (sssp_kernel.cu:49-52): alt = cost[u] + w;
// if (cost[v] > alt) atomicMin(&cost[v], alt) -- on uint32 distances, exact.
//
// Ordering is near-far delta stepping (Davidson et al., IPDPS 2014): vertices
// improved below the bucket bound T go to the near queue, the rest to a far
// pile that is filtered when the near queue drains (T += delta).  delta = 0
// gives the reference's unordered frontier order.  Any delta yields the same
// exact distances; it only changes the work and the number of iterations.
//
// Iteration protocol (per team of co-resident CTAs, one barrier per iteration):
//   iteration it consumes either the near queue Q[it&1] or, on a bucket advance,
//   the far pile of the previous epoch, plus the grid-tier list H[(it-1)%3] that
//   the previous iteration collected.  It appends to Q[(it+1)&1], to the far pile
//   of the current epoch and to H[it%3].  All counters live in 3-slot rings so a
//   slot is reset at least one barrier before it is reused.
#pragma once

#include <cstdint>

#include "nps.h"

namespace nps {

constexpr uint32_t kFull = 0xffffffffu;
constexpr uint32_t kInf = NPS_INF;
constexpr int kHeavyShift = 36;  // heavy counter packs (count << 36) | chunk_offset
constexpr unsigned long long kHeavyMask = (1ull << kHeavyShift) - 1;

// Per-instance device counters.  Zeroed by the host before a launch.
struct __align__(128) Counters {
  uint32_t qtail[3];   // near-queue tails, slot = iteration % 3
  uint32_t ftail[3];   // far-pile tails,   slot = epoch % 3
  uint32_t work[3];    // dynamic work-item counters, slot = iteration % 3
  uint32_t fmin[3];    // min distance pushed into the far pile on an advance, slot = epoch % 3
  unsigned long long heavy[3];  // grid-tier list counter, slot = iteration % 3
  uint32_t status;     // NPS_OK or the first error
  uint32_t iterations;
  uint32_t buckets;
  uint32_t reached;    // vertices whose distance left INF during the run
  unsigned long long edges;
  unsigned long long improvements;
  unsigned long long processed;
  // per-iteration ring used by the learned policy and the trace
  uint32_t hist[3][8];
  unsigned long long it_edges[3];
  unsigned long long it_impr[3];
  uint32_t it_reached[3];
  uint32_t pad[5];
};

struct InstDesc {
  const int32_t* row_ptr;
  const int32_t* col;
  const uint32_t* w;
  uint32_t* dist;
  uint8_t* update;      // state mode: initial frontier flags, cleared in place
  int32_t n;
  int32_t m;
  int32_t src;
  int32_t mode;         // 0: single source, 1: start from dist[] + update[]
  int32_t* q[2];        // near queues (capacity qcap)
  int32_t* fq[2];       // far piles   (capacity qcap)
  uint32_t* mark;       // near-queue dedupe stamps
  uint32_t* fmark;      // far-pile dedupe stamps
  int4* heavy;          // grid-tier entries {row start, row end, vertex, chunk offset}
  uint32_t qcap;
  uint32_t hcap;
  Counters* ctr;
  uint32_t* stamp_base; // device word carried across runs on this workspace
  nps_trace_rec* trace;
  uint32_t trace_cap;
  uint32_t delta;
  int32_t level;
  int32_t t1, t2, t3;   // tier thresholds: [t1,t2) warp, [t2,t3) block, >= t3 grid; < t1 small
  int32_t policy;
  int32_t vec_ok;       // col / w are 16-byte aligned
  int32_t pad0;
};

struct TeamDesc {
  int32_t cta_begin;
  int32_t cta_count;
  int32_t inst_begin;   // into LaunchParams::order
  int32_t inst_count;
};

// Policy weights in device memory: bf16 weights, fp32 biases and feature scaling.
struct PolicyDev {
  uint16_t w1[NPS_MLP_HID * NPS_MLP_IN];
  uint16_t w2[NPS_MLP_OUT * NPS_MLP_HID];
  float b1[NPS_MLP_HID];
  float b2[NPS_MLP_OUT];
  float mean[NPS_MLP_IN];
  float istd[NPS_MLP_IN];
};

struct LaunchParams {
  InstDesc* inst;
  const int32_t* order;
  const TeamDesc* teams;
  int32_t n_teams;
  int32_t fault_inject_wait;  // 1: the first barrier waits for an arrival that never comes
  uint32_t* bar;              // per-team barrier counters, 32 words apart
  uint32_t* abort_flag;
  unsigned long long timeout_ns;     // bound on each wait
  unsigned long long run_budget_ns;  // bound on the whole launch
  const PolicyDev* policy;
};

// ---------------------------------------------------------------------------
// small device helpers

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Read-only graph streams (CSR columns and weights): no L1 allocation.
__device__ __forceinline__ int4 ld_stream_v4(const int32_t* p) {
  int4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.s32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}
__device__ __forceinline__ int32_t ld_stream(const int32_t* p) {
  int32_t v;
  asm volatile("ld.global.nc.L1::no_allocate.s32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ int deg_bin(int32_t d) {
  // bins [4^k - 1, 4^(k+1) - 1): 0..2, 3..14, 15..62, ... , >= 16383
  int l = 31 - __clz((uint32_t)d + 1);
  int b = l >> 1;
  return b > 7 ? 7 : b;
}

// ---------------------------------------------------------------------------
// Per-iteration context, identical in every CTA of a team.
struct IterCtx {
  uint32_t T;        // bucket upper bound
  uint32_t snear;    // stamp for pushes into the next near queue
  uint32_t sfar;     // stamp for pushes into the current far pile
  int32_t* qn;       // next near queue
  uint32_t* qn_tail;
  int32_t* fp;       // far pile receiving pushes
  uint32_t* fp_tail;
  uint32_t* fp_min;  // non-null on a bucket advance
  int4* heavy;       // grid-tier list receiving appends
  unsigned long long* heavy_ctr;
  uint32_t hcap;     // capacity of that list
  int32_t t1, t2, t3;
};

// Thread-local accumulators, reduced per CTA.
struct Acc {
  uint32_t edges;
  uint32_t impr;
  uint32_t reached;
  uint32_t processed;
};

// Relax one candidate edge u->v with tentative distance nd.  Returns which
// queue (if any) v must be appended to.  Exact: atomicMin decides.
__device__ __forceinline__ void relax_one(const InstDesc& I, const IterCtx& C, bool valid, int32_t v,
                                          uint32_t nd, bool& pn, bool& pf, Acc& acc) {
  pn = false;
  pf = false;
  if (!valid) return;
  acc.edges++;
  if ((uint32_t)v >= (uint32_t)I.n) {  // neighbour id outside [0, n): record and skip
    atomicCAS(&I.ctr->status, 0u, (uint32_t)NPS_ERR_FORMAT);
    return;
  }
  if (nd >= kInf) return;
  uint32_t cur = __ldcg(I.dist + v);
  if (nd >= cur) return;
  uint32_t old = atomicMin(I.dist + v, nd);
  if (nd >= old) return;
  acc.impr++;
  if (old == kInf) acc.reached++;
  if (nd < C.T) {
    if (__ldcg(I.mark + v) != C.snear) pn = atomicExch(I.mark + v, C.snear) != C.snear;
  } else {
    if (__ldcg(I.fmark + v) != C.sfar) {
      pf = atomicExch(I.fmark + v, C.sfar) != C.sfar;
      if (pf && C.fp_min) atomicMin(C.fp_min, nd);
    }
  }
}

__device__ __forceinline__ uint32_t tent(uint32_t du, uint32_t w) {
  return (w >= kInf || du >= kInf) ? kInf : du + w;  // both < 2^30, so no wrap
}

// Warp-aggregated append of one item per lane.
__device__ __forceinline__ void append1(int32_t* q, uint32_t* tail, uint32_t cap, bool f, int32_t v,
                                        uint32_t* status, int lane) {
  uint32_t b = __ballot_sync(kFull, f);
  if (b == 0) return;
  uint32_t base = 0;
  int leader = __ffs(b) - 1;
  if (lane == leader) base = atomicAdd(tail, (uint32_t)__popc(b));
  base = __shfl_sync(kFull, base, leader);
  uint32_t pos = base + __popc(b & lanemask_lt());
  if (f) {
    if (pos < cap) q[pos] = v;
    else atomicCAS(status, 0u, (uint32_t)NPS_ERR_CAPACITY);
  }
}

// Warp-aggregated append of up to four items per lane (one ballot per slot).
__device__ __forceinline__ void append4(int32_t* q, uint32_t* tail, uint32_t cap, bool f0, bool f1,
                                        bool f2, bool f3, int32_t v0, int32_t v1, int32_t v2,
                                        int32_t v3, uint32_t* status, int lane) {
  uint32_t b0 = __ballot_sync(kFull, f0), b1 = __ballot_sync(kFull, f1);
  uint32_t b2 = __ballot_sync(kFull, f2), b3 = __ballot_sync(kFull, f3);
  uint32_t tot = __popc(b0) + __popc(b1) + __popc(b2) + __popc(b3);
  if (tot == 0) return;
  uint32_t base = 0;
  if (lane == 0) base = atomicAdd(tail, tot);
  base = __shfl_sync(kFull, base, 0);
  uint32_t lt = lanemask_lt();
  uint32_t o = base;
  bool over = false;
  if (f0) { uint32_t p = o + __popc(b0 & lt); if (p < cap) q[p] = v0; else over = true; }
  o += __popc(b0);
  if (f1) { uint32_t p = o + __popc(b1 & lt); if (p < cap) q[p] = v1; else over = true; }
  o += __popc(b1);
  if (f2) { uint32_t p = o + __popc(b2 & lt); if (p < cap) q[p] = v2; else over = true; }
  o += __popc(b2);
  if (f3) { uint32_t p = o + __popc(b3 & lt); if (p < cap) q[p] = v3; else over = true; }
  if (over) atomicCAS(status, 0u, (uint32_t)NPS_ERR_CAPACITY);
}

// Relax the (up to) four edges of the 16-byte chunk starting at edge index c
// that fall inside [s, e).  Loads the column and weight chunks with one int4
// load each when aligned and in bounds.  Warp-collective (ballots inside).
__device__ __forceinline__ void relax_chunk(const InstDesc& I, const IterCtx& C, bool act, int32_t c,
                                            int32_t s, int32_t e, uint32_t du, Acc& acc, int lane) {
  int4 cv = make_int4(0, 0, 0, 0), wv = make_int4(0, 0, 0, 0);
  if (act) {
    if (I.vec_ok && c + 4 <= I.m) {
      cv = ld_stream_v4(I.col + c);
      wv = ld_stream_v4((const int32_t*)I.w + c);
    } else {
      if (c >= s && c < e) { cv.x = ld_stream(I.col + c); wv.x = ld_stream((const int32_t*)I.w + c); }
      if (c + 1 >= s && c + 1 < e) { cv.y = ld_stream(I.col + c + 1); wv.y = ld_stream((const int32_t*)I.w + c + 1); }
      if (c + 2 >= s && c + 2 < e) { cv.z = ld_stream(I.col + c + 2); wv.z = ld_stream((const int32_t*)I.w + c + 2); }
      if (c + 3 >= s && c + 3 < e) { cv.w = ld_stream(I.col + c + 3); wv.w = ld_stream((const int32_t*)I.w + c + 3); }
    }
  }
  bool n0, n1, n2, n3, f0, f1, f2, f3;
  relax_one(I, C, act && c >= s && c < e, cv.x, tent(du, (uint32_t)wv.x), n0, f0, acc);
  relax_one(I, C, act && c + 1 >= s && c + 1 < e, cv.y, tent(du, (uint32_t)wv.y), n1, f1, acc);
  relax_one(I, C, act && c + 2 >= s && c + 2 < e, cv.z, tent(du, (uint32_t)wv.z), n2, f2, acc);
  relax_one(I, C, act && c + 3 >= s && c + 3 < e, cv.w, tent(du, (uint32_t)wv.w), n3, f3, acc);
  append4(C.qn, C.qn_tail, I.qcap, n0, n1, n2, n3, cv.x, cv.y, cv.z, cv.w, &I.ctr->status, lane);
  append4(C.fp, C.fp_tail, I.qcap, f0, f1, f2, f3, cv.x, cv.y, cv.z, cv.w, &I.ctr->status, lane);
}

__device__ __forceinline__ uint32_t row_chunks(int32_t s, int32_t e) {
  return (uint32_t)(((e - 1) >> 2) - (s >> 2) + 1);
}

// ---------------------------------------------------------------------------
// CTA shared state

template <int BS>
struct Smem {
  unsigned long long blk_ctr;  // (count << 32) | chunk offset
  uint32_t item;
  int32_t ok;
  uint32_t hist[8];
  int4 blk[BS];                // block-tier entries {s, e, du, chunk offset}
  uint32_t red[4][BS / 32];
  float feat[NPS_MLP_IN];
  float hid[NPS_MLP_HID];
  int32_t pol_choice[2];
  TeamDesc team;
  int32_t team_id;
  unsigned long long t_start;
};

// Team barrier over the CTAs of one team.  Bounded: gives up after timeout_ns
// (setting NPS_ERR_TIMEOUT and the abort flag) or when the abort flag is set.
// Returns false when the computation must stop.
template <int BS>
__device__ __forceinline__ bool team_barrier(const LaunchParams& P, Smem<BS>& sm, uint32_t* bar,
                                             uint32_t& epoch, uint32_t team_size,
                                             uint32_t* status, bool inject) {
  __syncthreads();
  if (threadIdx.x == 0) {
    if (globaltimer_ns() - sm.t_start > P.run_budget_ns) {
      atomicCAS(status, 0u, (uint32_t)NPS_ERR_TIMEOUT);
      atomicExch(P.abort_flag, 1u);
    }
    epoch += 1;
    uint32_t target = epoch * team_size + (inject ? 1u : 0u);
    __threadfence();
    atomicAdd(bar, 1u);
    unsigned long long t0 = globaltimer_ns();
    int ok = 1;
    uint32_t spins = 0;
    while ((int32_t)(ld_acquire_u32(bar) - target) < 0) {
      if (ld_relaxed_u32(P.abort_flag)) { ok = 0; break; }
      if ((++spins & 15u) == 0 && globaltimer_ns() - t0 > P.timeout_ns) {
        atomicCAS(status, 0u, (uint32_t)NPS_ERR_TIMEOUT);
        atomicExch(P.abort_flag, 1u);
        ok = 0;
        break;
      }
      __nanosleep(20);
    }
    __threadfence();
    if (ok && ld_relaxed_u32(status) != 0) ok = 0;
    if (!ok) atomicExch(P.abort_flag, 1u);
    sm.ok = ok;
  }
  __syncthreads();
  return sm.ok != 0;
}

// Block-wide sum of four counters; result valid in thread 0.
template <int BS>
__device__ __forceinline__ void block_sum4(Smem<BS>& sm, uint32_t a, uint32_t b, uint32_t c, uint32_t d,
                                           uint32_t out[4]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(kFull, a, o);
    b += __shfl_xor_sync(kFull, b, o);
    c += __shfl_xor_sync(kFull, c, o);
    d += __shfl_xor_sync(kFull, d, o);
  }
  __syncthreads();
  if (lane == 0) {
    sm.red[0][warp] = a;
    sm.red[1][warp] = b;
    sm.red[2][warp] = c;
    sm.red[3][warp] = d;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    out[0] = out[1] = out[2] = out[3] = 0;
    for (int i = 0; i < BS / 32; ++i) {
      out[0] += sm.red[0][i];
      out[1] += sm.red[1][i];
      out[2] += sm.red[2][i];
      out[3] += sm.red[3][i];
    }
  }
}

// ---------------------------------------------------------------------------
// Process one frontier chunk of BS vertices (or far-pile entries on a bucket
// advance).  Degree tiers:
//   deg <  t1       : warp-flat loop (warp scan of degrees, one edge per lane)
//   [t1, t2)        : warp tier  -- the owning warp walks the row with int4 chunks
//   [t2, t3)        : block tier -- appended to the CTA list, walked by all warps
//   >= t3           : grid tier  -- appended to H, walked by every CTA next iteration
template <int BS>
__device__ __forceinline__ void process_vertices(const InstDesc& I, const IterCtx& C, Smem<BS>& sm,
                                                 const int32_t* src_q, uint32_t idx_base,
                                                 uint32_t src_len, bool advance, uint32_t T_old,
                                                 bool want_hist, Acc& acc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = BS / 32;
  uint32_t idx = idx_base + threadIdx.x;
  int32_t v = -1, s = 0, e = 0;
  uint32_t du = 0;
  bool repush = false;
  int32_t rv = 0;
  if (idx < src_len) {
    v = src_q[idx];
    du = __ldcg(I.dist + v);
    if (advance) {
      // far-pile entry: stale below the old bound, deferred again at/above the new one
      if (du < T_old) {
        v = -1;
      } else if (du >= C.T) {
        if (__ldcg(I.fmark + v) != C.sfar) {
          repush = atomicExch(I.fmark + v, C.sfar) != C.sfar;
          if (repush) atomicMin(C.fp_min, du);
        }
        rv = v;
        v = -1;
      }
    }
    if (v >= 0) {
      s = __ldg(I.row_ptr + v);
      e = __ldg(I.row_ptr + v + 1);
      if (s < 0 || e < s || e > I.m) {  // malformed CSR row: record and skip
        atomicCAS(&I.ctr->status, 0u, (uint32_t)NPS_ERR_FORMAT);
        s = e = 0;
      }
      acc.processed++;
      if (want_hist) atomicAdd(&sm.hist[deg_bin(e - s)], 1u);
    }
  }
  if (advance) append1(C.fp, C.fp_tail, I.qcap, repush, rv, &I.ctr->status, lane);
  const int32_t deg = e - s;
  const bool small = deg > 0 && deg < C.t1;
  const bool wtier = deg >= C.t1 && deg < C.t2 && deg > 0;
  const bool btier = deg >= C.t2 && deg < C.t3 && deg > 0;
  const bool gtier = deg >= C.t3 && deg > 0;
  if (btier) {
    uint32_t nch = row_chunks(s, e);
    unsigned long long old = atomicAdd(&sm.blk_ctr, (1ull << 32) | nch);
    sm.blk[old >> 32] = make_int4(s, e, (int32_t)du, (int32_t)(uint32_t)old);
  }
  if (gtier) {
    uint32_t nch = row_chunks(s, e);
    unsigned long long old = atomicAdd(C.heavy_ctr, (1ull << kHeavyShift) | nch);
    uint32_t slot = (uint32_t)(old >> kHeavyShift);
    if (slot < C.hcap) C.heavy[slot] = make_int4(s, e, v, (int32_t)(uint32_t)(old & kHeavyMask));
    else atomicCAS(&I.ctr->status, 0u, (uint32_t)NPS_ERR_CAPACITY);
  }

  // ---- small vertices: warp-flat edge loop
  {
    uint32_t d = small ? (uint32_t)deg : 0u;
    uint32_t incl = d;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t;
    }
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    const uint32_t excl = incl - d;
    for (uint32_t k0 = 0; k0 < total; k0 += 32) {
      const uint32_t k = k0 + lane;
      const bool valid = k < total;
      int j = 0;
#pragma unroll
      for (int step = 16; step >= 1; step >>= 1) {
        uint32_t x = __shfl_sync(kFull, excl, j + step);
        if (x <= k) j += step;
      }
      const int32_t sj = __shfl_sync(kFull, s, j);
      const uint32_t duj = __shfl_sync(kFull, du, j);
      const uint32_t exj = __shfl_sync(kFull, excl, j);
      int32_t nb = 0;
      uint32_t wt = 0;
      if (valid) {
        int32_t ei = sj + (int32_t)(k - exj);
        nb = ld_stream(I.col + ei);
        wt = (uint32_t)ld_stream((const int32_t*)I.w + ei);
      }
      bool pn, pf;
      relax_one(I, C, valid, nb, tent(duj, wt), pn, pf, acc);
      append1(C.qn, C.qn_tail, I.qcap, pn, nb, &I.ctr->status, lane);
      append1(C.fp, C.fp_tail, I.qcap, pf, nb, &I.ctr->status, lane);
    }
  }

  // ---- warp tier: the warp walks each of its rows, 128 edges per step
  {
    uint32_t wb = __ballot_sync(kFull, wtier);
    while (wb) {
      const int src_lane = __ffs(wb) - 1;
      wb &= wb - 1;
      const int32_t rs = __shfl_sync(kFull, s, src_lane);
      const int32_t re = __shfl_sync(kFull, e, src_lane);
      const uint32_t rdu = __shfl_sync(kFull, du, src_lane);
      for (int32_t c0 = rs & ~3; c0 < re; c0 += 128) {
        const int32_t c = c0 + lane * 4;
        relax_chunk(I, C, c < re, c, rs, re, rdu, acc, lane);
      }
    }
  }

  // ---- block tier: every warp of the CTA walks the flat chunk space of the list
  __syncthreads();
  const unsigned long long bc = sm.blk_ctr;
  const uint32_t bcnt = (uint32_t)(bc >> 32), btot = (uint32_t)bc;
  for (uint32_t k0 = warp * 32; k0 < btot; k0 += NW * 32) {
    const uint32_t k = k0 + lane;
    const bool act = k < btot;
    int lo = 0, hi = (int)bcnt - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if ((uint32_t)sm.blk[mid].w <= k) lo = mid;
      else hi = mid - 1;
    }
    const int4 ent = sm.blk[lo];
    const int32_t c = (ent.x & ~3) + 4 * (int32_t)(k - (uint32_t)ent.w);
    relax_chunk(I, C, act, c, ent.x, ent.y, (uint32_t)ent.z, acc, lane);
  }
}

// Grid-tier work item: BS chunks of the flat chunk space of list H.
template <int BS>
__device__ __forceinline__ void process_heavy(const InstDesc& I, const IterCtx& C, const int4* H,
                                              uint32_t hcnt, unsigned long long htot,
                                              unsigned long long k_base, Acc& acc) {
  const int lane = threadIdx.x & 31;
  const unsigned long long k = k_base + threadIdx.x;
  const bool act = k < htot;
  // largest j with offset(j) <= k
  int lo = 0, hi = (int)hcnt - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    int4 em = H[mid];
    if ((unsigned long long)(uint32_t)em.w <= k) lo = mid;
    else hi = mid - 1;
  }
  int4 ent = H[lo];
  uint32_t du = act ? __ldcg(I.dist + ent.z) : 0u;
  const int32_t c = (ent.x & ~3) + 4 * (int32_t)(k - (uint32_t)ent.w);
  relax_chunk(I, C, act, c, ent.x, ent.y, du, acc, lane);
}

// ---------------------------------------------------------------------------
// Learned policy: 12 features -> 32 ReLU -> 14 logits (bf16 weights, fp32 math).
// Evaluated redundantly by every CTA of a team on identical inputs, so every
// CTA takes the same decision without another barrier.
__device__ __forceinline__ float bf16_bits_to_float(uint16_t b) {
  return __uint_as_float(((uint32_t)b) << 16);
}

template <int BS>
__device__ __forceinline__ void policy_eval(const PolicyDev* pol, Smem<BS>& sm) {
  const int t = threadIdx.x;
  __syncthreads();
  if (t < NPS_MLP_HID) {
    float a = pol->b1[t];
#pragma unroll
    for (int i = 0; i < NPS_MLP_IN; ++i) a = fmaf(bf16_bits_to_float(pol->w1[t * NPS_MLP_IN + i]), sm.feat[i], a);
    sm.hid[t] = a > 0.f ? a : 0.f;
  }
  __syncthreads();
  if (t == 0) {
    float best = -3.0e38f;
    int bd = 0;
    float lg[NPS_MLP_OUT];
    for (int o = 0; o < NPS_MLP_OUT; ++o) {
      float a = pol->b2[o];
      for (int h = 0; h < NPS_MLP_HID; ++h) a = fmaf(bf16_bits_to_float(pol->w2[o * NPS_MLP_HID + h]), sm.hid[h], a);
      lg[o] = a;
    }
    for (int o = 0; o < 11; ++o)
      if (lg[o] > best) { best = lg[o]; bd = o; }
    int bl = 0;
    best = lg[11];
    for (int o = 1; o < 3; ++o)
      if (lg[11 + o] > best) { best = lg[11 + o]; bl = o; }
    sm.pol_choice[0] = bd;
    sm.pol_choice[1] = bl;
  }
  __syncthreads();
}

// Thresholds (t1, t2, t3) for a consolidation level.
__device__ __forceinline__ void level_thresholds(int level, int32_t thr, int32_t bthr, int32_t gthr,
                                                 int32_t& t1, int32_t& t2, int32_t& t3) {
  const int32_t big = 0x7fffffff;
  switch (level) {
    case NPS_LEVEL_WARP: t1 = thr; t2 = big; t3 = big; break;
    case NPS_LEVEL_GRID: t1 = thr; t2 = thr; t3 = thr; break;
    case NPS_LEVEL_HYBRID: t1 = thr; t2 = bthr; t3 = gthr; break;
    default: t1 = thr; t2 = thr; t3 = big; break;  // block
  }
}

// Solve one instance with the CTAs of one team.  I refers to kernel-parameter
// space (single-instance launches) or to a shared-memory copy (batches).
template <int BS>
__device__ void solve_instance(const LaunchParams& P, const InstDesc& I, Smem<BS>& sm, uint32_t* bar,
                               uint32_t& bar_epoch, uint32_t rank, uint32_t team_size,
                               bool& inject) {
  Counters* ctr = I.ctr;
  const uint32_t gthreads = team_size * BS;
  const uint32_t gtid = rank * BS + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool learned = I.policy == NPS_POLICY_LEARNED && P.policy != nullptr;
  const bool want_iter = learned || (I.trace != nullptr);

  // ---- prologue: distances, stamps, initial frontier
  uint32_t base = __ldcg(I.stamp_base);
  const bool wrap = base > 0xF0000000u;
  if (wrap) base = 0;
  if (I.mode == 0) {
    for (uint32_t v = gtid; v < (uint32_t)I.n; v += gthreads) {
      I.dist[v] = (v == (uint32_t)I.src) ? 0u : kInf;
      if (wrap) { I.mark[v] = 0; I.fmark[v] = 0; }
    }
    if (rank == 0 && threadIdx.x == 0) {
      I.q[0][0] = I.src;
      ctr->qtail[0] = 1;
    }
  } else {
    // state mode: frontier = vertices with update[v] != 0 (cleared), distances kept
    const uint32_t nr = ((uint32_t)I.n + 31u) & ~31u;
    for (uint32_t v = gtid; v < nr; v += gthreads) {
      bool f = false;
      if (v < (uint32_t)I.n) {
        f = I.update[v] != 0;
        if (f) I.update[v] = 0;
        if (wrap) { I.mark[v] = 0; I.fmark[v] = 0; }
      }
      append1(I.q[0], &ctr->qtail[0], I.qcap, f, (int32_t)v, &ctr->status, lane);
    }
  }
  if (rank == 0 && threadIdx.x == 0) {
    ctr->fmin[0] = ctr->fmin[1] = ctr->fmin[2] = 0xffffffffu;
  }
  const bool inj = inject;
  inject = false;
  if (!team_barrier<BS>(P, sm, bar, bar_epoch, team_size, &ctr->status, inj)) return;

  uint32_t qlen = min(__ldcg(&ctr->qtail[0]), I.qcap);
  uint32_t it = 0, ep = 0;
  uint32_t delta = I.delta;
  uint32_t T = delta == 0 ? 0xffffffffu : delta;
  bool advance = false;
  uint32_t adv_len = 0, T_old = 0;
  uint32_t hprev_cnt = 0;
  unsigned long long hprev_tot = 0;
  int level = I.level;
  Acc tot = {0, 0, 0, 0};
  uint32_t buckets = 0;
  uint32_t reached_total = 1;
  const uint32_t hhalf = I.hcap / 2;

  for (;;) {
    // ---- iteration set-up (identical in every CTA)
    const uint32_t E = advance ? ep + 1 : ep;  // far epoch receiving pushes
    IterCtx C;
    C.T = T;
    C.snear = base + it + 1;
    C.sfar = base + E + 1;
    C.qn = I.q[(it + 1) & 1];
    C.qn_tail = &ctr->qtail[(it + 1) % 3];
    C.fp = I.fq[E & 1];
    C.fp_tail = &ctr->ftail[E % 3];
    C.fp_min = advance ? &ctr->fmin[E % 3] : nullptr;
    // grid-tier lists alternate halves of the heavy buffer by iteration parity
    C.heavy = I.heavy + ((it & 1) ? hhalf : 0);
    C.heavy_ctr = &ctr->heavy[it % 3];
    C.hcap = hhalf;
    level_thresholds(level, I.t1, I.t2, I.t3, C.t1, C.t2, C.t3);
    const int4* Hprev = I.heavy + ((it & 1) ? 0 : hhalf);

    if (rank == 0 && threadIdx.x == 0) {
      ctr->qtail[(it + 2) % 3] = 0;
      ctr->work[(it + 1) % 3] = 0;
      ctr->heavy[(it + 1) % 3] = 0;
      ctr->ftail[(E + 1) % 3] = 0;
      ctr->fmin[(E + 1) % 3] = 0xffffffffu;
      if (want_iter) {
        const uint32_t sl = (it + 1) % 3;
        for (int b = 0; b < 8; ++b) ctr->hist[sl][b] = 0;
        ctr->it_edges[sl] = 0;
        ctr->it_impr[sl] = 0;
        ctr->it_reached[sl] = 0;
      }
    }
    if (threadIdx.x < 8) sm.hist[threadIdx.x] = 0;

    const int32_t* srcq = advance ? I.fq[ep & 1] : I.q[it & 1];
    const uint32_t srclen = advance ? adv_len : qlen;
    const uint32_t n_heavy_items = (uint32_t)((hprev_tot + BS - 1) / BS);
    const uint32_t n_items = n_heavy_items + (srclen + BS - 1) / BS;
    Acc acc = {0, 0, 0, 0};

    // ---- work loop: dynamic items (grid-tier chunks first, then frontier chunks)
    for (;;) {
      if (threadIdx.x == 0) {
        sm.item = atomicAdd(&ctr->work[it % 3], 1u);
        sm.blk_ctr = 0ull;
      }
      __syncthreads();
      const uint32_t item = sm.item;
      if (item >= n_items) break;
      if (item < n_heavy_items) {
        process_heavy<BS>(I, C, Hprev, hprev_cnt, hprev_tot, (unsigned long long)item * BS, acc);
      } else {
        process_vertices<BS>(I, C, sm, srcq, (item - n_heavy_items) * BS, srclen, advance, T_old,
                             want_iter, acc);
      }
      __syncthreads();
    }

    // ---- per-CTA flush of iteration counters
    if (want_iter) {
      uint32_t r[4];
      block_sum4<BS>(sm, acc.edges, acc.impr, acc.reached, acc.processed, r);
      if (threadIdx.x == 0) {
        const uint32_t sl = it % 3;
        if (r[0]) atomicAdd(&ctr->it_edges[sl], (unsigned long long)r[0]);
        if (r[1]) atomicAdd(&ctr->it_impr[sl], (unsigned long long)r[1]);
        if (r[2]) atomicAdd(&ctr->it_reached[sl], r[2]);
        for (int b = 0; b < 8; ++b)
          if (sm.hist[b]) atomicAdd(&ctr->hist[sl][b], sm.hist[b]);
      }
    }
    tot.edges += acc.edges;
    tot.impr += acc.impr;
    tot.reached += acc.reached;
    tot.processed += acc.processed;

    if (!team_barrier<BS>(P, sm, bar, bar_epoch, team_size, &ctr->status, false)) return;

    // ---- decide the next iteration (every CTA reads the same values)
    if (advance) {
      ep += 1;
      buckets += 1;
    }
    const uint32_t qn = min(__ldcg(&ctr->qtail[(it + 1) % 3]), I.qcap);
    const unsigned long long hc = ld_relaxed_u64(&ctr->heavy[it % 3]);
    const uint32_t hn = min((uint32_t)(hc >> kHeavyShift), hhalf);
    const uint32_t fl = min(__ldcg(&ctr->ftail[ep % 3]), I.qcap);
    const bool will_advance = qn == 0 && hn == 0 && fl != 0;

    if (want_iter) {
      const uint32_t sl = it % 3;
      reached_total += __ldcg(&ctr->it_reached[sl]);
      if (learned) {
        // 12 features: log2 next frontier, 8 degree-histogram fractions of this
        // iteration's frontier, log2 bucket index, reached fraction, improvements per edge
        if (threadIdx.x == 0) {
          float h[8], hs = 0.f;
          for (int b = 0; b < 8; ++b) { h[b] = (float)__ldcg(&ctr->hist[sl][b]); hs += h[b]; }
          const float inv = hs > 0.f ? 1.f / hs : 0.f;
          float f[NPS_MLP_IN];
          f[0] = log2f(1.f + (float)(will_advance ? fl : qn));
          for (int b = 0; b < 8; ++b) f[1 + b] = h[b] * inv;
          f[9] = log2f(1.f + (float)buckets);
          f[10] = (float)reached_total / (float)I.n;
          const unsigned long long ie = __ldcg(&ctr->it_edges[sl]);
          f[11] = ie ? (float)__ldcg(&ctr->it_impr[sl]) / (float)ie : 0.f;
          for (int i = 0; i < NPS_MLP_IN; ++i) sm.feat[i] = (f[i] - P.policy->mean[i]) * P.policy->istd[i];
        }
        policy_eval<BS>(P.policy, sm);
        level = sm.pol_choice[1];
      }
      if (I.trace && rank == 0 && threadIdx.x == 0 && it < I.trace_cap) {
        nps_trace_rec* tr = I.trace + it;
        tr->iteration = it;
        tr->frontier = srclen;
        tr->far_len = fl;
        tr->bucket_hi = T;
        tr->delta = delta;
        tr->level = (uint32_t)level;
        for (int b = 0; b < 8; ++b) tr->hist[b] = __ldcg(&ctr->hist[sl][b]);
        tr->edges = __ldcg(&ctr->it_edges[sl]);
        tr->improvements = __ldcg(&ctr->it_impr[sl]);
        tr->reached = reached_total;
        tr->pad = hn;
      }
    }

    hprev_cnt = hn;
    hprev_tot = hc & kHeavyMask;
    advance = false;
    if (qn == 0 && hn == 0) {
      if (fl == 0) {
        it += 1;
        break;
      }
      // bucket advance: the next iteration filters the far pile of epoch ep
      if (learned) delta = 1u << sm.pol_choice[0];
      const uint32_t fm = __ldcg(&ctr->fmin[ep % 3]);
      const uint32_t dstep = delta ? delta : 1u;
      unsigned long long nt = (unsigned long long)T + dstep;
      if (fm != 0xffffffffu && (unsigned long long)fm + dstep > nt) nt = (unsigned long long)fm + dstep;
      T_old = T;
      T = nt >= 0xffffffffull ? 0xfffffffeu : (uint32_t)nt;
      advance = true;
      adv_len = fl;
    }
    qlen = qn;
    it += 1;
  }

  // ---- epilogue: totals and the stamp base for the next run on this workspace
  uint32_t r[4];
  block_sum4<BS>(sm, tot.edges, tot.impr, tot.reached, tot.processed, r);
  if (threadIdx.x == 0) {
    atomicAdd(&ctr->edges, (unsigned long long)r[0]);
    atomicAdd(&ctr->improvements, (unsigned long long)r[1]);
    atomicAdd(&ctr->reached, r[2]);
    atomicAdd(&ctr->processed, (unsigned long long)r[3]);
    if (rank == 0) {
      ctr->iterations = it;
      ctr->buckets = buckets;
      *I.stamp_base = base + (it > ep ? it : ep) + 4;
    }
  }
}

// The persistent kernel.  SINGLE: one instance whose descriptor is the kernel
// parameter `single` (constant-bank reads in the hot loops); otherwise the
// team's instances are staged one at a time in shared memory.
template <int BS, bool SINGLE>
__global__ void __launch_bounds__(BS) sssp_persistent_kernel(const __grid_constant__ LaunchParams P,
                                                             const __grid_constant__ InstDesc single) {
  __shared__ Smem<BS> sm;
  __shared__ InstDesc sinst;
  if (threadIdx.x == 0) {
    sm.t_start = globaltimer_ns();
    sm.team_id = -1;
    for (int t = 0; t < P.n_teams; ++t) {
      TeamDesc td = P.teams[t];
      if ((int)blockIdx.x >= td.cta_begin && (int)blockIdx.x < td.cta_begin + td.cta_count) {
        sm.team = td;
        sm.team_id = t;
        break;
      }
    }
  }
  __syncthreads();
  if (sm.team_id < 0) return;
  const TeamDesc td = sm.team;
  uint32_t* bar = P.bar + 32 * sm.team_id;
  uint32_t bar_epoch = 0;
  const uint32_t rank = blockIdx.x - td.cta_begin;
  bool inject = P.fault_inject_wait != 0;
  if constexpr (SINGLE) {
    solve_instance<BS>(P, single, sm, bar, bar_epoch, rank, (uint32_t)td.cta_count, inject);
    return;
  } else {
  for (int k = 0; k < td.inst_count; ++k) {
    __syncthreads();
    if (threadIdx.x == 0) sinst = P.inst[P.order[td.inst_begin + k]];
    __syncthreads();
    solve_instance<BS>(P, sinst, sm, bar, bar_epoch, rank, (uint32_t)td.cta_count, inject);
    if (ld_relaxed_u32(P.abort_flag)) return;
    // instances of a team are separated by a barrier so every CTA sees the previous one done
    if (!team_barrier<BS>(P, sm, bar, bar_epoch, (uint32_t)td.cta_count, &sinst.ctr->status, false)) return;
  }
  }
}

}  // namespace nps
