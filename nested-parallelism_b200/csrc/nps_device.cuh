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
// Here the buffers are consumed in-kernel by the warp, the CTA or every warp of
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
// Work distribution.  Inside an iteration every warp pulls its own work items
// from 8 striped atomic counters (no CTA-wide synchronisation on the hot path):
//   heavy items   128 16-byte chunks (512 edges) of the flat chunk space of the
//                 grid-tier list H that the previous iteration collected;
//   vertex items  32 frontier vertices, one per lane.
// A vertex of out-degree d is handled by tier:
//   d < threshold                     small: warp-flat loop over the warp's small rows
//   WARP  level, or HYBRID d < block  warp tier: the warp walks the row, 128 edges a step
//   BLOCK level, or HYBRID d < grid   block tier: appended to the CTA list in shared
//                                     memory, walked by all of the CTA's warps once per
//                                     iteration (the warp tier takes it if the list is full)
//   GRID  level, or HYBRID d >= grid  grid tier: appended to H, walked next iteration by
//                                     every warp of the team
//
// Iteration protocol (per team of co-resident CTAs, one barrier per iteration):
//   iteration it consumes either the near queue Q[it&1] or, on a bucket advance,
//   the far pile of the previous epoch, plus H of iteration it-1.  It appends to
//   Q[(it+1)&1], to the far pile of the current epoch and to H of iteration it.
//   All counters live in 3-slot rings so a slot is reset at least one barrier
//   before it is reused.
#pragma once

#include <cstdint>

#include "nps.h"

namespace nps {

constexpr uint32_t kFull = 0xffffffffu;
constexpr uint32_t kInf = NPS_INF;
constexpr int kHeavyShift = 36;  // heavy counter packs (count << 36) | chunk_offset
constexpr unsigned long long kHeavyMask = (1ull << kHeavyShift) - 1;
#ifndef NPS_STRIPES
#define NPS_STRIPES 8
#endif
#ifndef NPS_FLUSH_AT
#define NPS_FLUSH_AT 64
#endif
constexpr int kStripes = NPS_STRIPES;  // striped work counters (at most 32: one per lane when probed)
static_assert(kStripes >= 1 && kStripes <= 32, "stripes are probed one per lane");
constexpr uint32_t kStripeMask = kStripes >= 32 ? 0xffffffffu : ((1u << kStripes) - 1u);
constexpr int kBlockListCap = 512;     // CTA list entries (block tier)

// Per-instance device counters.  Zeroed by the host before a launch.
struct __align__(128) Counters {
  uint32_t qtail[3];   // near-queue tails, slot = iteration % 3
  uint32_t ftail[3];   // far-pile tails,   slot = epoch % 3
  uint32_t fmin[3];    // min distance pushed into the far pile on an advance, slot = epoch % 3
  uint32_t stail[3];   // settle-list tails, slot = heavy generation % 3
  uint32_t status;     // NPS_OK or the first error
  unsigned long long heavy[3];  // grid-tier list counter, slot = iteration % 3
  uint32_t iterations;
  uint32_t buckets;
  uint32_t reached;    // vertices whose distance left INF during the run
  uint32_t pad0;
  unsigned long long edges;
  unsigned long long improvements;
  unsigned long long processed;
  // per-iteration ring used by the learned policy and the trace
  uint32_t hist[3][8];
  unsigned long long it_edges[3];
  unsigned long long it_impr[3];
  uint32_t it_reached[3];
  uint32_t it_early[3];  // rows sorted into the grid-tier list when pushed (part of the next frontier)
  unsigned long long prof[9];   // NPS_PROFILE builds: SM cycles per phase, summed over warps
  unsigned long long solve_ns;  // end of this instance's solve, from its team CTA 0's start
  // asynchronous buckets: ring units (near-ring vertices and segments) pushed and not yet
  // processed, and the phase's static items claimed and done, slot = phase % 3
  uint32_t pend;
  uint32_t swork[3];
  uint32_t sdone[3];
  // settle-list entries appended in each iteration, slot = iteration % 3.  The decision
  // after an iteration reads its own slot, which the next iteration leaves alone (that
  // iteration may already be appending while a slower CTA decides: a bucket advance
  // appends the far-pile vertices it processes)
  uint32_t sadd[3];
  uint32_t pad2[2];
  // striped work counters, one 128-byte line each: work[slot][stripe * 32]
  // decision agreement: every CTA adds a hash of the counters its decision after iteration
  // i read to slot i % 4, and checks the sum one iteration later (team size x its own hash)
  uint32_t agree[4];
  alignas(128) uint32_t work[3][kStripes * 32];
};

// Work rings of the asynchronous buckets.  Head and tail counters persist across
// runs on a workspace (like the stamp base), each on its own 128-byte line.
struct __align__(128) RingState {
  uint32_t nq_head, pad0[31];
  uint32_t nq_tail, pad1[31];
  uint32_t seg_head, pad2[31];
  uint32_t seg_tail, pad3[31];
};

struct InstDesc {
  const int32_t* row_ptr;
  const int32_t* col;
  const uint32_t* w;     // null: every edge weighs 1 (breadth-first levels)
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
  int4* heavy;          // grid-tier entries {row start, row end, vertex | heavy flag, chunk offset}
  int32_t* hitem;       // per half: entry holding the first chunk of each grid-tier work item
  uint32_t icap;        // work items per half
  uint32_t item_shift;  // log2 chunks per grid-tier work item (5 or more)
  int32_t* sq[2];       // settle lists (light/heavy split): vertices processed in the bucket
  uint32_t* smark;      // settle-list dedupe stamps
  uint32_t qcap;
  uint32_t hcap;
  Counters* ctr;
  uint32_t* stamp_base; // device word carried across runs on this workspace
  nps_trace_rec* trace;
  uint32_t trace_cap;
  uint32_t delta;
  int32_t level;
  int32_t t1, t2, t3;   // threshold, block_threshold, grid_threshold
  int32_t policy;
  int32_t vec_ok;       // col / w are 16-byte aligned
  int32_t light_heavy;  // 1: split edges at delta (relax w >= delta once per settled vertex)
  int32_t local_rounds; // warp-local processing rounds per vertex item (0 = none)
  int32_t order_degree; // rows below this degree ignore the bucket bound (0 = none)
  uint32_t dsched;      // per-bucket log2 widths, 4 bits each (0 = fixed delta)
  int32_t sort_push;    // grid-tier rows sorted at push: 1 on, -1 off, 0 by the grid threshold
  int32_t async;        // 1: buckets are processed without per-iteration barriers (GRID tiers)
  unsigned long long* nq;  // near ring: slot = (tag << 32) | vertex, tag = index + 1 when filled
  uint32_t nq_mask;        // ring capacity - 1 (a power of two)
  int4* seg;               // segment ring: {start, end, vertex | heavy flag, tag}
  uint32_t seg_mask;
  RingState* rs;
  unsigned long long wait_ns;  // bound on one wait for a ring slot
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
  int32_t test_disagree;      // 1: CTA 1 reports another hash for the first decision (agreement check test)
  uint32_t* bar;              // per-team barrier words (see team_barrier), bar_stride words per team
  uint32_t bar_stride;
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

__device__ __forceinline__ unsigned long long ld_relaxed_u64p(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int4 ld_relaxed_v4(const int4* p) {
  int4 v;
  asm volatile("ld.relaxed.gpu.global.v4.s32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p)
               : "memory");
  return v;
}

__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void st_relaxed_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t atom_exch_release(uint32_t* p, uint32_t v) {
  uint32_t old;
  asm volatile("atom.release.gpu.global.exch.b32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

__device__ __forceinline__ uint32_t atom_exch_acquire(uint32_t* p, uint32_t v) {
  uint32_t old;
  asm volatile("atom.acquire.gpu.global.exch.b32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Zero that the compiler cannot see through: adding it to an address makes a
// later access wait for the value it was made from (a data dependency, so the
// access is issued only after that value has returned from memory).
__device__ __forceinline__ uint32_t dep_zero(uint32_t x) {
  uint32_t z;
  asm volatile("and.b32 %0, %1, 0;" : "=r"(z) : "r"(x));
  return z;
}

// L2 cache policies (createpolicy, sm_80+): the CSR column/weight stream is
// read once per scan and should leave L2 first; the per-vertex arrays touched at
// random (distances) should stay.  Without the hint the stream (8 bytes per
// scanned edge) evicts the distance array although both would fit in L2.
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t pol;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t pol;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

// Read-only graph streams (CSR columns and weights): no L1 allocation, L2 evict-first.
__device__ __forceinline__ int4 ld_stream_v4(const int32_t* p) {
  int4 v;
#ifdef NPS_NO_L2_HINTS
  asm volatile("ld.global.nc.L1::no_allocate.v4.s32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
#else
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0,%1,%2,%3}, [%4], %5;"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p), "l"(policy_evict_first()));
#endif
  return v;
}
__device__ __forceinline__ int32_t ld_stream(const int32_t* p) {
  int32_t v;
#ifdef NPS_NO_L2_HINTS
  asm volatile("ld.global.nc.L1::no_allocate.s32 %0, [%1];" : "=r"(v) : "l"(p));
#else
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;"
               : "=r"(v)
               : "l"(p), "l"(policy_evict_first()));
#endif
  return v;
}

// Read-only index data (row_ptr) read once per visit: no L1 allocation, so L1
// keeps the distance lines.
__device__ __forceinline__ int32_t ld_index(const int32_t* p) {
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

// Distance read for the pre-check `nd < dist[v]` before atomicMin: cached in L1
// (`.ca`) with the L2 evict-last policy.  An L1 copy may be stale, but within a
// launch distances only decrease, and L1 lines of global data do not survive
// from one launch to the next (PTX ISA, ld cache operators: the driver
// invalidates them between dependent grids), so a stale value is never below
// the current one: the pre-check can only let an extra candidate through to the
// atomicMin, whose returned old value decides.  On R-MAT graphs
// the heads of most edges are a few thousand hub vertices; serving their
// distances from L1 takes that load off a handful of L2 slices.
__device__ __forceinline__ uint32_t ld_dist(const uint32_t* p) {
#ifdef NPS_NO_L2_HINTS
  return __ldca(p);
#else
  uint32_t v;
  asm volatile("ld.global.ca.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(policy_evict_last()));
  return v;
#endif
}

__device__ __forceinline__ uint32_t tent(uint32_t du, uint32_t w) {
  return (w >= kInf || du >= kInf) ? kInf : du + w;  // both < 2^30, so no wrap
}

__device__ __forceinline__ uint32_t row_chunks(int32_t s, int32_t e) {
  return (uint32_t)(((e - 1) >> 2) - (s >> 2) + 1);
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
  int32_t* hitem;    // its work-item start entries
  int32_t t_warp;    // degree >= t_warp leaves the small path
  int32_t t_block;   // degree >= t_block goes to the CTA list
  int32_t t_grid;    // degree >= t_grid goes to H
  uint32_t split;    // light/heavy split weight (0: no split, every edge is relaxed)
  bool heavy_iter;   // this iteration relaxes heavy edges of the settle list
  int32_t* sq;       // settle list receiving processed vertices (null: no settle appends)
  uint32_t* sq_tail;
  uint32_t sstamp;
  int32_t local_rounds;  // rounds of warp-local processing per vertex item
  int32_t order_deg;     // improved vertices below this degree join the near queue at any distance
  bool ring;             // asynchronous bucket: near pushes go to the near ring, grid-tier rows
                         // to the segment ring (qn, heavy and the item tables are unused)
  uint32_t* sadd;        // counts this iteration's settle-list appends
  bool early;            // near pushes of at least t_grid edges join this iteration's grid-tier
                         // list when their staging buffer is flushed (walked next iteration)
  bool want_hist;        // policy features or trace: count the degrees of those rows
};

// Whether an edge of weight w is relaxed by a pass over light (heavy = false)
// or heavy (heavy = true) edges.
__device__ __forceinline__ bool edge_in_pass(const IterCtx& C, uint32_t w, bool heavy) {
  return C.split == 0u || (heavy ? w >= C.split : w < C.split);
}

// Append the lanes' rows with `g` set ({s, e, vtag}) to this iteration's grid-tier
// list.  One atomicAdd per warp reserves list slots and chunk offsets for all of
// them (a per-row atomic on this one counter serialises large frontiers); within
// the warp, slots and offsets follow lane order, so offsets still grow with the
// slot across the list.  The entry holds the first chunk of every work item that
// starts inside it; the warp then writes those item starts together, one row at a
// time.  Warp-collective.
__device__ __forceinline__ void grid_append(const InstDesc& I, const IterCtx& C, bool g, int32_t s, int32_t e,
                                            int32_t vtag, int lane) {
  const uint32_t gmask = __ballot_sync(kFull, g);
  if (!gmask) return;
  uint32_t slot = 0xffffffffu, b0 = 0, b1 = 0;  // list slot and work items [b0, b1) starting in it
  const uint32_t nch = g ? row_chunks(s, e) : 0u;
  uint32_t incl = nch;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += t;
  }
  const uint32_t wtot = __shfl_sync(kFull, incl, 31);
  const int leader = __ffs(gmask) - 1;
  unsigned long long old = 0;
  if (lane == leader) old = atomicAdd(C.heavy_ctr, ((unsigned long long)__popc(gmask) << kHeavyShift) | wtot);
  old = __shfl_sync(kFull, old, leader);
  const uint32_t off = (uint32_t)(old & kHeavyMask) + (incl - nch);
  if (g) {
    slot = (uint32_t)(old >> kHeavyShift) + (uint32_t)__popc(gmask & lanemask_lt());
    if (slot < C.hcap) {
      C.heavy[slot] = make_int4(s, e, vtag, (int32_t)off);
      const uint32_t sh = I.item_shift;
      b0 = (off + (1u << sh) - 1) >> sh;
      b1 = ((off + nch - 1) >> sh) + 1;
      if (b1 > I.icap) atomicCAS(&I.ctr->status, 0u, (uint32_t)NPS_ERR_CAPACITY);
    } else {
      atomicCAS(&I.ctr->status, 0u, (uint32_t)NPS_ERR_CAPACITY);
    }
  }
  uint32_t wb = __ballot_sync(kFull, b1 > b0);
  while (wb) {
    const int src_lane = __ffs(wb) - 1;
    wb &= wb - 1;
    const uint32_t rs = __shfl_sync(kFull, slot, src_lane);
    const uint32_t r0 = __shfl_sync(kFull, b0, src_lane);
    const uint32_t r1 = min(__shfl_sync(kFull, b1, src_lane), I.icap);
    for (uint32_t b = r0 + lane; b < r1; b += 32) C.hitem[b] = (int32_t)rs;
  }
}

// Thread-local accumulators, reduced per CTA.
struct Acc {
  uint32_t edges;
  uint32_t impr;
  uint32_t reached;
  uint32_t processed;
};

// Phase timers of an NPS_PROFILE build: each warp's lane 0 sums clock64()
// deltas per phase; the sums reach Counters::prof at the end of the launch.
#ifdef NPS_PROFILE
struct PhaseClock {
  unsigned long long acc[9];
  long long t;
  __device__ __forceinline__ void reset() {
    for (int i = 0; i < 9; ++i) acc[i] = 0;
    t = clock64();
  }
  __device__ __forceinline__ void lap(int phase) {
    const long long now = clock64();
    acc[phase] += (unsigned long long)(now - t);
    t = now;
  }
};
#define NPS_LAP(pc, phase) (pc).lap(phase)
#else
struct PhaseClock {
  __device__ __forceinline__ void reset() {}
  __device__ __forceinline__ void lap(int) {}
};
#define NPS_LAP(pc, phase) ((void)0)
#endif

// ---------------------------------------------------------------------------
// Batched relaxation: K candidate edges per lane.  All K distance loads are
// issued before any is used and all K atomicMin before any result is used, so
// one lane keeps K independent L2 requests in flight.  Returns, per candidate,
// whether the head must be appended to the near queue (pn) or far pile (pf).
template <int K>
__device__ __forceinline__ void relax_batch(const InstDesc& I, const IterCtx& C, const bool (&valid)[K],
                                            const int32_t (&v)[K], const uint32_t (&nd)[K], bool (&pn)[K],
                                            bool (&pf)[K], Acc& acc) {
  uint32_t cur[K];
  bool go[K];
#pragma unroll
  for (int j = 0; j < K; ++j) {
    go[j] = valid[j];
    if (valid[j]) {
      acc.edges++;
      if ((uint32_t)v[j] >= (uint32_t)I.n) {  // neighbour id outside [0, n): record and skip
        atomicCAS(&I.ctr->status, 0u, (uint32_t)NPS_ERR_FORMAT);
        go[j] = false;
      } else if (nd[j] >= kInf) {
        go[j] = false;
      }
    }
  }
#pragma unroll
  for (int j = 0; j < K; ++j) cur[j] = go[j] ? ld_dist(I.dist + v[j]) : 0u;
  uint32_t old[K];
#pragma unroll
  for (int j = 0; j < K; ++j) {
    go[j] = go[j] && nd[j] < cur[j];
    old[j] = go[j] ? atomicMin(I.dist + v[j], nd[j]) : 0u;
  }
#pragma unroll
  for (int j = 0; j < K; ++j) {
    pn[j] = false;
    pf[j] = false;
    if (go[j] && nd[j] < old[j]) {
      acc.impr++;
      if (old[j] == kInf) acc.reached++;
      // one exchange decides whether this improvement is the first of the iteration
      bool near = nd[j] < C.T;
      if (!near && C.order_deg > 0) near = __ldg(I.row_ptr + v[j] + 1) - __ldg(I.row_ptr + v[j]) < C.order_deg;
      if (near) {
        // ring mode: a consumer resets the mark before it reads the distance, so the
        // mark is set with release semantics -- whoever sees it set sees this atomicMin
        // (ordering by the dependency on the returned value alone lost updates on B200)
        pn[j] = (C.ring ? atom_exch_release(I.mark + v[j], C.snear) : atomicExch(I.mark + v[j], C.snear)) != C.snear;
      } else {
        pf[j] = atomicExch(I.fmark + v[j], C.sfar) != C.sfar;
      }
    }
  }
  if (C.fp_min) {
    // smallest distance pushed into the far pile: one atomicMin per warp (all lanes
    // take part; a single per-push atomic on this one word serialises an advance)
    uint32_t mn = 0xffffffffu;
#pragma unroll
    for (int j = 0; j < K; ++j)
      if (pf[j]) mn = min(mn, nd[j]);
    mn = __reduce_min_sync(kFull, mn);
    if ((threadIdx.x & 31) == 0 && mn != 0xffffffffu) atomicMin(C.fp_min, mn);
  }
}

// Warp-aggregated append of up to K items per lane: one ballot per slot, one
// atomicAdd per warp.  Warp-collective.
template <int K>
__device__ __forceinline__ void append_k(int32_t* q, uint32_t* tail, uint32_t cap, const bool (&f)[K],
                                         const int32_t (&v)[K], uint32_t* status, int lane) {
  uint32_t b[K];
  uint32_t tot = 0;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    b[j] = __ballot_sync(kFull, f[j]);
    tot += __popc(b[j]);
  }
  if (tot == 0) return;
  uint32_t base = 0;
  if (lane == 0) base = atomicAdd(tail, tot);
  base = __shfl_sync(kFull, base, 0);
  const uint32_t lt = lanemask_lt();
  bool over = false;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    if (f[j]) {
      const uint32_t p = base + __popc(b[j] & lt);
      if (p < cap) q[p] = v[j];
      else over = true;
    }
    base += __popc(b[j]);
  }
  if (over) atomicCAS(status, 0u, (uint32_t)NPS_ERR_CAPACITY);
}

// Per-warp staging of queue appends in shared memory.  A warp collects the
// vertices it pushes and moves them to the global queue 32 at a time (one
// atomicAdd on the queue tail per >= 32 entries, one coalesced 128-byte store
// per 32), so warps do not serialise on the tail counter every round.
// A warp moves its staged appends to the global queue once kFlushAt are waiting,
// in multiples of 32, with one atomicAdd on the queue tail: fewer, larger flushes
// keep the single tail counter of each queue from serialising the improvements
// of a large iteration.
constexpr int kFlushAt = NPS_FLUSH_AT;
constexpr int kStage = kFlushAt + 4 * 32;  // >= kFlushAt - 1 left over + 4 * 32 from one append

struct Stage {
  int32_t* nbuf;   // near-queue staging (kStage entries, shared memory)
  int32_t* fbuf;   // far-pile staging
  int32_t* sbuf;   // settle-list staging
  uint32_t ncnt;   // warp-uniform fill counts
  uint32_t fcnt;
  uint32_t scnt;
  uint32_t fmin;   // per lane: smallest distance pushed into the far pile (ring mode)
  uint32_t* credit;  // ring mode: pending-total credits this warp holds (shared memory, lane 0)
  uint32_t* hnext;   // push-time sorting: degree histogram of the rows sorted (next iteration's)
  uint32_t* enext;   // push-time sorting: rows sorted in this iteration
};

// Move the first `nflush` staged entries to q and shift the rest down.
__device__ __forceinline__ void stage_flush(int32_t* buf, uint32_t& cnt, uint32_t nflush, int32_t* q,
                                            uint32_t* tail, uint32_t cap, uint32_t* status, int lane,
                                            uint32_t* count = nullptr) {
  __syncwarp();
  uint32_t base = 0;
  if (lane == 0) {
    base = atomicAdd(tail, nflush);
    if (count) atomicAdd(count, nflush);
  }
  base = __shfl_sync(kFull, base, 0);
  for (uint32_t i = lane; i < nflush; i += 32) {
    if (base + i < cap) q[base + i] = buf[i];
    else atomicCAS(status, 0u, (uint32_t)NPS_ERR_CAPACITY);
  }
  const uint32_t rem = cnt - nflush;
  int32_t t = 0;
  if ((uint32_t)lane < rem) t = buf[nflush + lane];
  __syncwarp();
  if ((uint32_t)lane < rem) buf[lane] = t;
  __syncwarp();
  cnt = rem;
}

// Wait (bounded by I.wait_ns) until the previous user of a ring slot has released it,
// i.e. its tag equals `want`.  False, with NPS_ERR_TIMEOUT recorded, when the bound
// runs out or another error already stopped the run.
static __device__ __noinline__ bool ring_wait_tag(const uint32_t* tag, uint32_t want, const InstDesc& I) {
  const unsigned long long t0 = globaltimer_ns();
  for (;;) {
    if (ld_relaxed_u32(tag) == want) return true;
    if (ld_relaxed_u32(&I.ctr->status) != 0) return false;
    if (globaltimer_ns() - t0 > I.wait_ns) {
      atomicCAS(&I.ctr->status, 0u, (uint32_t)NPS_ERR_TIMEOUT);
      return false;
    }
    __nanosleep(64);
  }
}

// Ring mode: units this warp makes visible are first covered by credits it holds
// in the pending total.  Lane 0 takes `k` credits, adding a batch of at least
// kCreditBatch to the pending total when its own run out (one atomic per batch,
// not per flush); the returned value orders the addition before anything made
// visible from it (callers add dep_zero of the result to their next address).
constexpr uint32_t kCreditBatch = 1024;
__device__ __forceinline__ uint32_t take_credits(const InstDesc& I, uint32_t* credit, uint32_t k) {
  uint32_t c = *credit, x = 0;
  if (c < k) {
    const uint32_t add = max(k - c, kCreditBatch);
    x = atomicAdd(&I.ctr->pend, add);
    c += add;
  }
  *credit = c - k;
  return x;
}

// Move the first `nflush` staged entries to the near ring and shift the rest down.
// The entries are covered by pending-total credits before they become visible (the
// ring reservation waits for the credits), so the total cannot reach zero while one
// of them waits or is being processed.  Slot = (index + 1) << 32 | vertex, one
// 8-byte store, written once its previous user released it (tag == index).
__device__ __forceinline__ void ring_flush(const InstDesc& I, int32_t* buf, uint32_t& cnt, uint32_t nflush,
                                           int lane, uint32_t* credit) {
  __syncwarp();
  uint32_t base = 0;
  if (lane == 0) {
    const uint32_t x = take_credits(I, credit, nflush);
    base = atomicAdd(&I.rs->nq_tail + dep_zero(x), nflush);
  }
  base = __shfl_sync(kFull, base, 0);
  for (uint32_t i = lane; i < nflush; i += 32) {
    const uint32_t idx = base + i;
    unsigned long long* slot = I.nq + (idx & I.nq_mask);
    const uint32_t* tag = reinterpret_cast<const uint32_t*>(slot) + 1;  // high word (little-endian)
    if (ld_relaxed_u32(tag) == idx || ring_wait_tag(tag, idx, I))
      st_relaxed_u64(slot, ((unsigned long long)(idx + 1) << 32) | (uint32_t)buf[i]);
  }
  const uint32_t rem = cnt - nflush;
  int32_t t = 0;
  if ((uint32_t)lane < rem) t = buf[nflush + lane];
  __syncwarp();
  if ((uint32_t)lane < rem) buf[lane] = t;
  __syncwarp();
  cnt = rem;
}

template <int K>
__device__ __forceinline__ void stage_k(int32_t* buf, uint32_t& cnt, const bool (&f)[K], const int32_t (&v)[K],
                                        int32_t* q, uint32_t* tail, uint32_t cap, uint32_t* status, int lane,
                                        const InstDesc* ring = nullptr, uint32_t* credit = nullptr,
                                        uint32_t* count = nullptr) {
  uint32_t b[K];
  uint32_t tot = 0;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    b[j] = __ballot_sync(kFull, f[j]);
    tot += __popc(b[j]);
  }
  if (tot == 0) return;
  const uint32_t lt = lanemask_lt();
  uint32_t base = cnt;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    if (f[j]) buf[base + __popc(b[j] & lt)] = v[j];
    base += __popc(b[j]);
  }
  cnt += tot;
  if (cnt >= (uint32_t)kFlushAt) {
    if (ring) ring_flush(*ring, buf, cnt, cnt & ~31u, lane, credit);
    else stage_flush(buf, cnt, cnt & ~31u, q, tail, cap, status, lane, count);
  }
}

// Near-queue flush with push-time sorting: the first `nflush` staged vertices are
// looked up in row_ptr (32 at a time, one per lane); rows of at least t_grid edges
// join this iteration's grid-tier list, so the next iteration walks them (sorted
// when they are taken from the queue instead, they would wait one iteration more),
// and the others go to the near queue with one atomicAdd on its tail.  The rest of
// the buffer moves down.  Warp-collective.
__device__ __forceinline__ void sort_flush(const InstDesc& I, const IterCtx& C, Stage& S, uint32_t nflush,
                                               int lane) {
  __syncwarp();
  uint32_t kept = 0, nsorted = 0;
  const uint32_t lt = lanemask_lt();
  for (uint32_t g0 = 0; g0 < nflush; g0 += 32) {
    const uint32_t i = g0 + lane;
    const int32_t v = i < nflush ? S.nbuf[i] : -1;
    int32_t s = 0, e = 0;
    if (v >= 0) {
      s = ld_index(I.row_ptr + v);
      e = ld_index(I.row_ptr + v + 1);
      if (s < 0 || e < s || e > I.m) {  // malformed CSR row: record; the queue entry reports it again
        atomicCAS(&I.ctr->status, 0u, (uint32_t)NPS_ERR_FORMAT);
        s = e = 0;
      }
    }
    const bool g = v >= 0 && e > s && e - s >= C.t_grid;
    grid_append(I, C, g, s, e, v, lane);
    if (C.want_hist) {
      const int bin = g ? deg_bin(e - s) : 8;
      const uint32_t grp = __match_any_sync(kFull, bin);
      if (g && lane == __ffs(grp) - 1) atomicAdd(&S.hnext[bin], (uint32_t)__popc(grp));
    }
    nsorted += __popc(__ballot_sync(kFull, g));
    const bool keep = v >= 0 && !g;
    const uint32_t b = __ballot_sync(kFull, keep);
    __syncwarp();  // every lane has read its entry of this group
    // compaction in place: kept + rank <= g0 + lane, so no entry of a later group is overwritten
    if (keep) S.nbuf[kept + __popc(b & lt)] = v;
    kept += __popc(b);
  }
  __syncwarp();
  if (C.want_hist && lane == 0 && nsorted) atomicAdd(S.enext, nsorted);
  if (kept) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(C.qn_tail, kept);
    base = __shfl_sync(kFull, base, 0);
    for (uint32_t i = lane; i < kept; i += 32) {
      if (base + i < I.qcap) C.qn[base + i] = S.nbuf[i];
      else atomicCAS(&I.ctr->status, 0u, (uint32_t)NPS_ERR_CAPACITY);
    }
  }
  const uint32_t rem = S.ncnt - nflush;
  int32_t t = 0;
  if ((uint32_t)lane < rem) t = S.nbuf[nflush + lane];
  __syncwarp();
  if ((uint32_t)lane < rem) S.nbuf[lane] = t;
  __syncwarp();
  S.ncnt = rem;
}

// Stage near-queue pushes (four per lane) and flush once kFlushAt are waiting.
__device__ __forceinline__ void stage_near(const InstDesc& I, const IterCtx& C, Stage& S, const bool (&f)[4],
                                           const int32_t (&v)[4], int lane) {
  if (!C.early) {
    stage_k<4>(S.nbuf, S.ncnt, f, v, C.qn, C.qn_tail, I.qcap, &I.ctr->status, lane, C.ring ? &I : nullptr,
               S.credit);
    return;
  }
  uint32_t b[4];
  uint32_t tot = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    b[j] = __ballot_sync(kFull, f[j]);
    tot += __popc(b[j]);
  }
  if (tot == 0) return;
  const uint32_t lt = lanemask_lt();
  uint32_t base = S.ncnt;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (f[j]) S.nbuf[base + __popc(b[j] & lt)] = v[j];
    base += __popc(b[j]);
  }
  S.ncnt += tot;
  if (S.ncnt >= (uint32_t)kFlushAt) sort_flush(I, C, S, S.ncnt & ~31u, lane);
}

// End of an iteration: everything staged goes to the global queues (near pushes to
// the near ring in ring mode).
__device__ __forceinline__ void stage_drain(const InstDesc& I, Stage& S, const IterCtx& C, uint32_t qcap,
                                            uint32_t* status, int lane) {
  if (S.ncnt) {
    if (C.ring) ring_flush(I, S.nbuf, S.ncnt, S.ncnt, lane, S.credit);
    else if (C.early) sort_flush(I, C, S, S.ncnt, lane);
    else stage_flush(S.nbuf, S.ncnt, S.ncnt, C.qn, C.qn_tail, qcap, status, lane);
  }
  if (S.fcnt) stage_flush(S.fbuf, S.fcnt, S.fcnt, C.fp, C.fp_tail, qcap, status, lane);
  if (S.scnt) stage_flush(S.sbuf, S.scnt, S.scnt, C.sq, C.sq_tail, qcap, status, lane, C.sadd);
}

template <int K>
__device__ __forceinline__ void relax_and_push(const InstDesc& I, const IterCtx& C, const bool (&valid)[K],
                                               const int32_t (&v)[K], const uint32_t (&nd)[K], Acc& acc,
                                               Stage& S, int lane) {
  static_assert(K == 4 || K == 8, "candidates per lane");
  bool pn[K], pf[K];
  relax_batch<K>(I, C, valid, v, nd, pn, pf, acc);
  // staged four per lane at a time: a staging buffer holds one such append beyond its flush point
#pragma unroll
  for (int h = 0; h < K; h += 4) {
    const bool fn[4] = {pn[h], pn[h + 1], pn[h + 2], pn[h + 3]};
    const bool ff[4] = {pf[h], pf[h + 1], pf[h + 2], pf[h + 3]};
    const int32_t vv[4] = {v[h], v[h + 1], v[h + 2], v[h + 3]};
    stage_near(I, C, S, fn, vv, lane);
    stage_k<4>(S.fbuf, S.fcnt, ff, vv, C.fp, C.fp_tail, I.qcap, &I.ctr->status, lane);
  }
  if (C.ring) {
#pragma unroll
    for (int j = 0; j < K; ++j)
      if (pf[j]) S.fmin = min(S.fmin, nd[j]);
  }
}

// Load the 16-byte chunk at edge index c (4-aligned) of the column and weight
// arrays: one int4 load each when aligned and in bounds, else element-wise
// loads of the positions inside [s, e).  A null weight array means every edge
// weighs 1 (breadth-first levels), and no weight is read.
__device__ __forceinline__ void load_chunk(const InstDesc& I, bool act, int32_t c, int32_t s, int32_t e,
                                           int4& cv, int4& wv) {
  cv = make_int4(0, 0, 0, 0);
  wv = make_int4(0, 0, 0, 0);
  if (!act) return;
  if (I.vec_ok && c + 4 <= I.m) {
    cv = ld_stream_v4(I.col + c);
    wv = I.w ? ld_stream_v4((const int32_t*)I.w + c) : make_int4(1, 1, 1, 1);
  } else {
    const int32_t* wp = (const int32_t*)I.w;
    if (c >= s && c < e) { cv.x = ld_stream(I.col + c); wv.x = wp ? ld_stream(wp + c) : 1; }
    if (c + 1 >= s && c + 1 < e) { cv.y = ld_stream(I.col + c + 1); wv.y = wp ? ld_stream(wp + c + 1) : 1; }
    if (c + 2 >= s && c + 2 < e) { cv.z = ld_stream(I.col + c + 2); wv.z = wp ? ld_stream(wp + c + 2) : 1; }
    if (c + 3 >= s && c + 3 < e) { cv.w = ld_stream(I.col + c + 3); wv.w = wp ? ld_stream(wp + c + 3) : 1; }
  }
}

// Relax the edges of an already loaded chunk c that fall inside [s, e).
// Warp-collective.
__device__ __forceinline__ void relax_loaded(const InstDesc& I, const IterCtx& C, bool act, int32_t c,
                                             int32_t s, int32_t e, uint32_t du, bool heavy, const int4& cv,
                                             const int4& wv, Acc& acc, Stage& S, int lane) {
  const bool valid[4] = {act && c >= s && c < e && edge_in_pass(C, (uint32_t)wv.x, heavy),
                         act && c + 1 >= s && c + 1 < e && edge_in_pass(C, (uint32_t)wv.y, heavy),
                         act && c + 2 >= s && c + 2 < e && edge_in_pass(C, (uint32_t)wv.z, heavy),
                         act && c + 3 >= s && c + 3 < e && edge_in_pass(C, (uint32_t)wv.w, heavy)};
  const int32_t v[4] = {cv.x, cv.y, cv.z, cv.w};
  const uint32_t nd[4] = {tent(du, (uint32_t)wv.x), tent(du, (uint32_t)wv.y), tent(du, (uint32_t)wv.z),
                          tent(du, (uint32_t)wv.w)};
  relax_and_push<4>(I, C, valid, v, nd, acc, S, lane);
}

// ---------------------------------------------------------------------------
// CTA shared state

template <int BS>
struct Smem {
  unsigned long long blk_ctr;  // CTA list (block tier): (entries << 32) | chunks, one atomic
  int32_t ok;
  uint32_t hist[8];
  int4 blk[kBlockListCap];     // block-tier entries {s, e, vertex, chunk offset}
  int32_t stage[BS / 32][3][kStage];  // per-warp append staging: [near, far, settle]
  uint32_t red[4][BS / 32];
  float feat[NPS_MLP_IN];
  int32_t pol_choice[2];
  PolicyDev pol;               // the policy's weights, copied once per solve (learned runs only)
  uint32_t it_acc[4];          // this CTA's edges, improvements, first reaches, rows sorted at push
  uint32_t hist_next[8];       // degree histogram of rows sorted at push (the next iteration's frontier)
  uint32_t credit[BS / 32];    // ring mode: pending-total credits held per warp
  uint32_t phase_flag;         // ring mode: set by the CTA's warp 0 when the bucket ends (p + 1) or
                               // must stop (0xffffffff); the CTA's other warps read it, not global memory
  TeamDesc team;
  int32_t team_id;
  uint32_t rank;
  uint32_t bc_q, bc_f, bc_m, bc_s;   // counters broadcast after a barrier
  unsigned long long bc_h;
  unsigned long long t_start;
  uint32_t agree_prev;         // thread 0: hash of this CTA's last schedule decision
  uint32_t bc_ag;              // the agreement slot of the decision before it
};

// Team barrier over the CTAs of one team.  Bounded: gives up after timeout_ns
// (setting NPS_ERR_TIMEOUT and the abort flag) or when the abort flag is set.
// Returns false when the computation must stop.
//
// Arrival is one `red.release.gpu` add per CTA on the team's counter (release:
// the CTA's writes, made thread 0's by the preceding bar.sync, become visible
// with the arrival); thread 0 then polls the counter with `ld.acquire.gpu` until
// it reaches epoch * team_size.  With check_status = false the caller reads the
// status word itself, together with the counters it needs after the barrier.
constexpr uint32_t kBarGroup = 16;  // barrier-area sizing granule (words per team = 32 * (2 + CTAs / 16))

template <int BS>
__device__ __forceinline__ bool team_barrier(const LaunchParams& P, Smem<BS>& sm, uint32_t* bar,
                                             uint32_t& epoch, uint32_t team_size,
                                             uint32_t* status, bool inject, bool check_status = true,
                                             Counters* flush = nullptr, uint32_t flush_slot = 0) {
  __syncthreads();
  if (threadIdx.x == 0) {
    if (flush) {
      // this CTA's iteration statistics, ordered before the arrival by the release
      if (sm.it_acc[0]) atomicAdd(&flush->it_edges[flush_slot], (unsigned long long)sm.it_acc[0]);
      if (sm.it_acc[1]) atomicAdd(&flush->it_impr[flush_slot], (unsigned long long)sm.it_acc[1]);
      if (sm.it_acc[2]) atomicAdd(&flush->it_reached[flush_slot], sm.it_acc[2]);
      if (sm.it_acc[3]) atomicAdd(&flush->it_early[flush_slot], sm.it_acc[3]);
      for (int b = 0; b < 8; ++b)
        if (sm.hist[b]) atomicAdd(&flush->hist[flush_slot][b], sm.hist[b]);
    }
    if (globaltimer_ns() - sm.t_start > P.run_budget_ns) {
      atomicCAS(status, 0u, (uint32_t)NPS_ERR_TIMEOUT);
      atomicExch(P.abort_flag, 1u);
    }
    epoch += 1;
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar) : "memory");
    const uint32_t target = epoch * team_size + (inject ? 1u : 0u);
    const unsigned long long t0 = globaltimer_ns();
    int ok = 1;
    uint32_t spins = 0;
    // Spin with relaxed loads and acquire once the count is reached: an acquire
    // at GPU scope makes the SM drop its L1 copies of global data, which would
    // also throw away the distance lines the SM's other CTAs are still using.
    while ((int32_t)(ld_relaxed_u32(bar) - target) < 0) {
      if ((++spins & 15u) == 0) {
        if (ld_relaxed_u32(P.abort_flag)) { ok = 0; break; }
        if (globaltimer_ns() - t0 > P.timeout_ns) {
          atomicCAS(status, 0u, (uint32_t)NPS_ERR_TIMEOUT);
          atomicExch(P.abort_flag, 1u);
          ok = 0;
          break;
        }
      }
      __nanosleep(20);
    }
    if (ok) (void)ld_acquire_u32(bar);  // synchronises with every arrival's release
    if (ok && check_status && ld_relaxed_u32(status) != 0) ok = 0;
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
// Walk one row [s, e) with the whole warp, 128 edges (one int4 per lane) a step.
__device__ __forceinline__ void warp_row(const InstDesc& I, const IterCtx& C, int32_t s, int32_t e, uint32_t du,
                                         Acc& acc, Stage& S, int lane) {
  for (int32_t c0 = s & ~3; c0 < e; c0 += 128) {
    const int32_t c = c0 + lane * 4;
    int4 cv, wv;
    load_chunk(I, c < e, c, s, e, cv, wv);
    relax_loaded(I, C, c < e, c, s, e, du, C.heavy_iter, cv, wv, acc, S, lane);
  }
}

constexpr int kSegEdges = 1024;  // edges per segment: four 256-edge rounds of one warp

// Ring mode: the grid-tier rows of a warp become segments of at most kSegEdges
// edges (from the row's 4-aligned start) on the segment ring.  The segments
// are covered by pending-total credits before they are visible; one reservation
// per warp.
// Returns false, pushing nothing, when the ring is more than half full: the rows
// are then walked by the warp itself.  Warp-collective.
__device__ __forceinline__ bool push_segments(const InstDesc& I, bool gtier, int32_t s, int32_t e, int32_t vtag,
                                              int lane, uint32_t* credit) {
  const uint32_t nseg = gtier ? (uint32_t)(((int64_t)e - (s & ~3) + kSegEdges - 1) / kSegEdges) : 0u;
  uint32_t incl = nseg;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += t;
  }
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  if (total == 0) return true;
  uint32_t base = 0, ok = 1;
  if (lane == 0) {
    const int32_t used = (int32_t)(ld_relaxed_u32(&I.rs->seg_tail) - ld_relaxed_u32(&I.rs->seg_head));
    if ((int64_t)max(used, 0) + total > (int64_t)(I.seg_mask + 1) / 2) {
      ok = 0;
    } else {
      const uint32_t x = take_credits(I, credit, total);
      base = atomicAdd(&I.rs->seg_tail + dep_zero(x), total);
    }
  }
  if (!__shfl_sync(kFull, ok, 0)) return false;
  base = __shfl_sync(kFull, base, 0);
  const uint32_t excl = incl - nseg;
  uint32_t wb = __ballot_sync(kFull, nseg > 0);
  while (wb) {
    const int src = __ffs(wb) - 1;
    wb &= wb - 1;
    const int32_t rs = __shfl_sync(kFull, s, src), re = __shfl_sync(kFull, e, src);
    const int32_t rz = __shfl_sync(kFull, vtag, src);
    const uint32_t rn = __shfl_sync(kFull, nseg, src), rx = __shfl_sync(kFull, excl, src);
    const int64_t c0 = rs & ~3;
    for (uint32_t j = lane; j < rn; j += 32) {
      const uint32_t idx = base + rx + j;
      int4* slot = I.seg + (idx & I.seg_mask);
      uint32_t* tag = reinterpret_cast<uint32_t*>(slot) + 3;
      if (ld_relaxed_u32(tag) == idx || ring_wait_tag(tag, idx, I)) {
        int32_t* w = reinterpret_cast<int32_t*>(slot);
        st_relaxed_u32(reinterpret_cast<uint32_t*>(w), (uint32_t)max((int64_t)rs, c0 + kSegEdges * (int64_t)j));
        st_relaxed_u32(reinterpret_cast<uint32_t*>(w) + 1,
                       (uint32_t)min((int64_t)re, c0 + kSegEdges * ((int64_t)j + 1)));
        st_relaxed_u32(reinterpret_cast<uint32_t*>(w) + 2, (uint32_t)rz);
      }
    }
  }
  // every payload is in place before any tag says so: one fence, then the tags
  __threadfence();
  wb = __ballot_sync(kFull, nseg > 0);
  while (wb) {
    const int src = __ffs(wb) - 1;
    wb &= wb - 1;
    const uint32_t rn = __shfl_sync(kFull, nseg, src), rx = __shfl_sync(kFull, excl, src);
    for (uint32_t j = lane; j < rn; j += 32) {
      const uint32_t idx = base + rx + j;
      uint32_t* tag = reinterpret_cast<uint32_t*>(I.seg + (idx & I.seg_mask)) + 3;
      if (ld_relaxed_u32(&I.ctr->status) == 0) st_relaxed_u32(tag, idx + 1);
    }
  }
  return true;
}

// 256 edges from chunk r0 of the row range [s, e): two chunks per lane, their
// column and weight loads issued together, one batch of eight candidates.
__device__ __forceinline__ void walk_round(const InstDesc& I, const IterCtx& C, int32_t r0, int32_t s, int32_t e,
                                           uint32_t du, bool heavy, Acc& acc, Stage& S, int lane) {
  bool act[2];
  int32_t c[2];
  int4 cv[2], wv[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    c[h] = r0 + 128 * h + 4 * lane;
    act[h] = c[h] < e;
    load_chunk(I, act[h], c[h], s, e, cv[h], wv[h]);
  }
  bool valid[8];
  int32_t vv[8];
  uint32_t nd[8];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int32_t cc[4] = {cv[h].x, cv[h].y, cv[h].z, cv[h].w};
    const uint32_t ww[4] = {(uint32_t)wv[h].x, (uint32_t)wv[h].y, (uint32_t)wv[h].z, (uint32_t)wv[h].w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int32_t ei = c[h] + q;
      valid[4 * h + q] = act[h] && ei >= s && ei < e && edge_in_pass(C, ww[q], heavy);
      vv[4 * h + q] = cc[q];
      nd[4 * h + q] = tent(du, ww[q]);
    }
  }
  relax_and_push<8>(I, C, valid, vv, nd, acc, S, lane);
}

// One segment {start, end, vertex | heavy flag} of at most kSegEdges edges from a
// 4-aligned chunk, in rounds of 256 edges: two chunks per lane, one batch of eight
// candidates per round.  The owner's distance is read now, by a load that sees the
// latest value (a weak load could return a copy older than the one the owner's
// consumer read, and the edges would miss that improvement).  Warp-collective.
__device__ __forceinline__ void walk_segment(const InstDesc& I, const IterCtx& C, int4 sg, Acc& acc, Stage& S,
                                             int lane) {
  const int32_t s = sg.x, e = sg.y;
  const uint32_t v = (uint32_t)sg.z & 0x7fffffffu;
  if (s < 0 || e > I.m || v >= (uint32_t)I.n) {  // never pushed by a producer: record and skip
    if (lane == 0) atomicCAS(&I.ctr->status, 0u, (uint32_t)NPS_ERR_CAPACITY);
    return;
  }
  const uint32_t du = ld_relaxed_u32(I.dist + v);
  for (int32_t r0 = s & ~3; r0 < e; r0 += 256) walk_round(I, C, r0, s, e, du, sg.z < 0, acc, S, lane);
}

// Vertex work item: up to 32 frontier entries (or far-pile entries on a bucket
// advance), one per lane; lanes without one pass vin = -1.  Warp-collective.
template <int BS>
__device__ __forceinline__ void process_vertex_item(const InstDesc& I, const IterCtx& C, Smem<BS>& sm,
                                                    int32_t vin, bool advance, uint32_t T_old, bool want_hist,
                                                    Acc& acc, Stage& S, PhaseClock& pc, int lane,
                                                    bool local = false) {
  int32_t v = vin, s = 0, e = 0;
  uint32_t du = 0;
  bool repush = false;
  int32_t rv = 0;
  if (v >= 0) {
    // ring mode: a load that sees the latest distance (the mark-reset protocol needs
    // the value as of the reset; a weak load may return an older copy)
    du = C.ring ? ld_relaxed_u32(I.dist + v) : __ldcg(I.dist + v);
    if (advance) {
      // far-pile entry: stale below the old bound, deferred again at/above the new one
      if (du < T_old) {
        v = -1;
      } else if (du >= C.T) {
        if (__ldcg(I.fmark + v) != C.sfar) {
          repush = atomicExch(I.fmark + v, C.sfar) != C.sfar;
        }
        rv = v;
        v = -1;
      }
    }
    if (v >= 0) {
      s = ld_index(I.row_ptr + v);
      e = ld_index(I.row_ptr + v + 1);
      if (s < 0 || e < s || e > I.m) {  // malformed CSR row: record and skip
        atomicCAS(&I.ctr->status, 0u, (uint32_t)NPS_ERR_FORMAT);
        s = e = 0;
      }
      acc.processed++;
    }
  }
  if (want_hist) {
    // frontier degree histogram: one shared atomic per distinct bin in the warp
    const bool has = v >= 0;
    const int bin = has ? deg_bin(e - s) : 8;
    const uint32_t grp = __match_any_sync(kFull, bin);
    if (has && lane == __ffs(grp) - 1) atomicAdd(&sm.hist[bin], (uint32_t)__popc(grp));
  }
  if (advance) {
    if (C.fp_min) {
      const uint32_t mn = __reduce_min_sync(kFull, repush ? du : 0xffffffffu);
      if (lane == 0 && mn != 0xffffffffu) atomicMin(C.fp_min, mn);
    } else if (repush) {
      S.fmin = min(S.fmin, du);
    }
    const bool f[1] = {repush};
    const int32_t vv[1] = {rv};
    stage_k<1>(S.fbuf, S.fcnt, f, vv, C.fp, C.fp_tail, I.qcap, &I.ctr->status, lane);
  }
  const int32_t deg = e - s;
  if (C.sq) {
    // light pass: the vertex joins the bucket's settle list once, for its heavy edges
    bool f[1] = {false};
    if (deg > 0 && __ldcg(I.smark + v) != C.sstamp) f[0] = atomicExch(I.smark + v, C.sstamp) != C.sstamp;
    const int32_t vv[1] = {v};
    stage_k<1>(S.sbuf, S.scnt, f, vv, C.sq, C.sq_tail, I.qcap, &I.ctr->status, lane, nullptr, nullptr, C.sadd);
  }
  // deferred entries remember which edges they relax in the top bit of the vertex id
  // deferred entries remember which edges they relax in the top bit of the vertex id
  const int32_t vtag = C.heavy_iter ? (int32_t)((uint32_t)v | 0x80000000u) : v;
  const bool small = deg > 0 && deg < C.t_warp;
  // A vertex taken back by a warp-local round is walked by that warp: the CTA and grid
  // lists then hold each vertex at most once per iteration, which bounds their size.
  bool wtier = local ? deg >= C.t_warp : (deg >= C.t_warp && deg < C.t_block);
  const bool btier = !local && deg >= C.t_block && deg < C.t_grid;
  bool gtier = !local && deg >= C.t_grid && deg > 0;
  if (btier) {
    // slot and chunk offset from one atomic, so offsets increase with the slot
    const unsigned long long old = atomicAdd(&sm.blk_ctr, (1ull << 32) | row_chunks(s, e));
    const uint32_t slot = (uint32_t)(old >> 32);
    if (slot < (uint32_t)kBlockListCap) sm.blk[slot] = make_int4(s, e, vtag, (int32_t)(uint32_t)old);
    else wtier = true;  // CTA list full: the warp walks the row itself
  }
  if (C.ring) {
    if (!push_segments(I, gtier, s, e, vtag, lane, S.credit)) wtier = wtier || gtier;  // ring half full: walk it here
  } else {
    // with push-time sorting a row may already be in this iteration's list (pushed and
    // sorted earlier in it): the near stamp decides which of the two appends it
    if (C.early && gtier) gtier = atomicExch(I.mark + v, C.snear) != C.snear;
    grid_append(I, C, gtier, s, e, vtag, lane);
  }

  NPS_LAP(pc, 1);
  // ---- small rows: warp-flat loop, four edges per lane per round
  {
    const uint32_t d = small ? (uint32_t)deg : 0u;
    uint32_t incl = d;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t;
    }
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    const uint32_t excl = incl - d;
    for (uint32_t k0 = 0; k0 < total; k0 += 128) {
      bool valid[4];
      int32_t ei[4];
      uint32_t dj[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const uint32_t k = k0 + j * 32 + lane;
        valid[j] = k < total;
        int o = 0;
#pragma unroll
        for (int step = 16; step >= 1; step >>= 1) {
          const uint32_t x = __shfl_sync(kFull, excl, o + step);
          if (x <= k) o += step;
        }
        const int32_t so = __shfl_sync(kFull, s, o);
        const uint32_t eo = __shfl_sync(kFull, excl, o);
        dj[j] = __shfl_sync(kFull, du, o);
        ei[j] = so + (int32_t)(k - eo);
      }
      int32_t nb[4];
      uint32_t nd[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        nb[j] = valid[j] ? ld_stream(I.col + ei[j]) : 0;
        nd[j] = valid[j] ? (I.w ? (uint32_t)ld_stream((const int32_t*)I.w + ei[j]) : 1u) : 0u;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        valid[j] = valid[j] && edge_in_pass(C, nd[j], C.heavy_iter);
        nd[j] = tent(dj[j], nd[j]);
      }
      relax_and_push<4>(I, C, valid, nb, nd, acc, S, lane);
    }
  }

  NPS_LAP(pc, 2);
  // ---- warp tier: the warp walks each of its rows
  {
    uint32_t wb = __ballot_sync(kFull, wtier);
    while (wb) {
      const int src_lane = __ffs(wb) - 1;
      wb &= wb - 1;
      const int32_t rs = __shfl_sync(kFull, s, src_lane);
      const int32_t re = __shfl_sync(kFull, e, src_lane);
      const uint32_t rdu = __shfl_sync(kFull, du, src_lane);
      warp_row(I, C, rs, re, rdu, acc, S, lane);
    }
  }
  NPS_LAP(pc, 3);
}

// Flat chunk-space walk of a list of rows {s, e, vertex, chunk offset} sorted by
// offset: chunks [k_begin, k_end) are handled by this warp, each lane takes
// every 32nd chunk.  Distances of the row owners are re-read here (the list may
// have been built an iteration earlier).  Warp-collective.
__device__ __forceinline__ void walk_chunks(const InstDesc& I, const IterCtx& C, const int4* L, uint32_t cnt,
                                            unsigned long long k_begin, unsigned long long k_end, Acc& acc,
                                            Stage& S, int lane) {
  if (k_begin >= k_end || cnt == 0) return;
  // owner of the lane's first chunk: largest j with offset(j) <= k
  unsigned long long k = k_begin + lane;
  int lo = 0, hi = (int)cnt - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if ((unsigned long long)(uint32_t)L[mid].w <= k) lo = mid;
    else hi = mid - 1;
  }
  int j = lo;
  int4 ent = L[j];
  uint32_t nxt = (j + 1 < (int)cnt) ? (uint32_t)L[j + 1].w : 0xffffffffu;
  // The owner's distance is read when the owner changes.  A value that has
  // dropped since only makes this walk relax with a larger tentative distance,
  // and the owner is back in a queue for every drop.
  uint32_t du = (k < k_end) ? __ldcg(I.dist + (ent.z & 0x7fffffff)) : 0u;
  for (unsigned long long k0 = k_begin; k0 < k_end; k0 += 32) {
    k = k0 + lane;
    const bool act = k < k_end;
    bool moved = false;
    while (act && j + 1 < (int)cnt && (unsigned long long)nxt <= k) {
      ++j;
      ent = L[j];
      nxt = (j + 1 < (int)cnt) ? (uint32_t)L[j + 1].w : 0xffffffffu;
      moved = true;
    }
    if (moved) du = __ldcg(I.dist + (ent.z & 0x7fffffff));
    const int32_t c = (ent.x & ~3) + 4 * (int32_t)(k - (uint32_t)ent.w);
    int4 cv, wv;
    load_chunk(I, act, c, ent.x, ent.y, cv, wv);
    relax_loaded(I, C, act, c, ent.x, ent.y, du, ent.z < 0, cv, wv, acc, S, lane);
  }
}

// One work item of the grid-tier list L (cnt entries sorted by chunk offset):
// chunks [kb, ke) of its flat chunk space, whose first chunk lies in entry js.
// The warp loads 32 consecutive entries at a time (one coalesced load); each
// lane finds the owner of its chunks among them with a 5-step shuffle search.
// The owners' distances are read at walk time, one per window lane.
// Every entry has at least one chunk, so a window of 32 entries covers any 32
// consecutive chunks that start in its first entry.
//
// A round takes 64 chunks, two per lane (chunks k0 + lane and k0 + 32 + lane):
// both chunks' column and weight loads are issued together, then their eight
// distance loads, then their eight atomicMin, so one round costs one dependent
// chain for 256 edges.  Warp-collective.
__device__ __forceinline__ void walk_item(const InstDesc& I, const IterCtx& C, const int4* L, uint32_t cnt,
                                          uint32_t kb, uint32_t ke, uint32_t js, Acc& acc, Stage& S, int lane) {
  uint32_t k = kb;
  while (k < ke) {
    const uint32_t jl = js + lane;
    int4 E = make_int4(0, 0, 0, 0);
    uint32_t off = 0xffffffffu, cov = 0xffffffffu, dv = kInf;
    if (jl < cnt) {
      E = __ldcg(L + jl);  // written last iteration; read at L2, not kept in L1
      off = (uint32_t)E.w;
      cov = off + row_chunks(E.x, E.y);
      const uint32_t v = (uint32_t)E.z & 0x7fffffffu;
      if (v < (uint32_t)I.n) dv = __ldcg(I.dist + v);
    }
    const uint32_t lim = min(ke, __shfl_sync(kFull, cov, 31));  // end of the window's chunks
    for (uint32_t k0 = k; k0 < lim; k0 += 64) {
      bool act[2];
      int32_t s[2], e[2], z[2], c[2];
      uint32_t du[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const uint32_t kk = k0 + 32 * h + lane;
        int o = 0;  // largest window index whose first chunk is <= kk (entry 0's is <= k0)
#pragma unroll
        for (int step = 16; step >= 1; step >>= 1) {
          const uint32_t x = __shfl_sync(kFull, off, o + step);
          if (x <= kk) o += step;
        }
        s[h] = __shfl_sync(kFull, E.x, o);
        e[h] = __shfl_sync(kFull, E.y, o);
        z[h] = __shfl_sync(kFull, E.z, o);
        du[h] = __shfl_sync(kFull, dv, o);
        const uint32_t oo = __shfl_sync(kFull, off, o);
        // the owner must hold chunk kk (it always does unless the list is inconsistent)
        const bool own = kk >= oo && e[h] > s[h] && kk - oo < row_chunks(s[h], e[h]);
        if (kk < lim && !own) atomicCAS(&I.ctr->status, 0u, (uint32_t)NPS_ERR_CAPACITY);
        act[h] = kk < lim && own;
        c[h] = (s[h] & ~3) + 4 * (int32_t)(kk - oo);
      }
      int4 cv[2], wv[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) load_chunk(I, act[h], c[h], s[h], e[h], cv[h], wv[h]);
      bool valid[8];
      int32_t v[8];
      uint32_t nd[8];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int32_t cc[4] = {cv[h].x, cv[h].y, cv[h].z, cv[h].w};
        const uint32_t ww[4] = {(uint32_t)wv[h].x, (uint32_t)wv[h].y, (uint32_t)wv[h].z, (uint32_t)wv[h].w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int32_t ei = c[h] + q;
          valid[4 * h + q] = act[h] && ei >= s[h] && ei < e[h] && edge_in_pass(C, ww[q], z[h] < 0);
          v[4 * h + q] = cc[q];
          nd[4 * h + q] = tent(du[h], ww[q]);
        }
      }
      relax_and_push<8>(I, C, valid, v, nd, acc, S, lane);
    }
    k = lim;
    js += 32;
  }
}

// ---------------------------------------------------------------------------
// Learned policy: 12 features -> 32 ReLU -> 14 logits (bf16 weights, fp32 math).
// Evaluated redundantly by every CTA of a team on identical inputs, so every
// CTA takes the same decision without another barrier.
__device__ __forceinline__ float bf16_bits_to_float(uint16_t b) {
  return __uint_as_float(((uint32_t)b) << 16);
}

// One warp evaluates the MLP on the normalised features in shared memory: lane h
// computes hidden unit h, lanes 0..13 the logits (the hidden layer reaches them
// by shuffles), then two shuffle arg-max reductions (lowest index on ties) give
// the width exponent (logits 0..10) and the level (logits 11..13), written to
// choice[0] and choice[1].  Called by all 32 lanes of one warp.
static __device__ __noinline__ void policy_eval_warp(const PolicyDev* pol, const float* feat, int32_t* choice, int lane) {
  static_assert(NPS_MLP_HID == 32 && NPS_MLP_OUT <= 32, "one lane per hidden unit and per logit");
  float a = pol->b1[lane];
#pragma unroll
  for (int i = 0; i < NPS_MLP_IN; ++i) a = fmaf(bf16_bits_to_float(pol->w1[lane * NPS_MLP_IN + i]), feat[i], a);
  const float hid = a > 0.f ? a : 0.f;
  const int o = lane < NPS_MLP_OUT ? lane : 0;
  float lg = pol->b2[o];
#pragma unroll
  for (int h = 0; h < NPS_MLP_HID; ++h)
    lg = fmaf(bf16_bits_to_float(pol->w2[o * NPS_MLP_HID + h]), __shfl_sync(kFull, hid, h), lg);
  // arg-max over [lo, hi): the larger value wins, the lower index on equal values
  auto argmax = [&](int lo, int hi) {
    float v = (lane >= lo && lane < hi) ? lg : -INFINITY;
    int ix = (lane >= lo && lane < hi) ? lane : 0x7fffffff;
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) {
      const float v2 = __shfl_xor_sync(kFull, v, d);
      const int i2 = __shfl_xor_sync(kFull, ix, d);
      if (v2 > v || (v2 == v && i2 < ix)) { v = v2; ix = i2; }
    }
    return ix;
  };
  const int bd = argmax(0, 11);
  const int bl = argmax(11, NPS_MLP_OUT) - 11;
  if (lane == 0) {
    choice[0] = bd;
    choice[1] = bl;
  }
}

// Tier thresholds (warp, block, grid) for a consolidation level.
__device__ __forceinline__ void level_thresholds(int level, int32_t thr, int32_t bthr, int32_t gthr,
                                                 int32_t& tw, int32_t& tb, int32_t& tg) {
  const int32_t big = 0x7fffffff;
  switch (level) {
    case NPS_LEVEL_WARP: tw = thr; tb = big; tg = big; break;
    case NPS_LEVEL_BLOCK: tw = thr; tb = thr; tg = big; break;
    case NPS_LEVEL_GRID: tw = thr; tb = thr; tg = thr; break;
    default: tw = thr; tb = bthr; tg = gthr; break;  // hybrid
  }
}

// Decision agreement (thread 0 of each CTA).  After a barrier every CTA reads the
// counters its next decision depends on; they must be identical in every CTA (the
// decision also depends on per-CTA state, which stays identical as long as every earlier
// decision was).  Each CTA adds a hash of what it read to slot it % 4 and checks, one
// iteration later, that the slot of the previous decision holds team_size times its own
// hash (prev_sum: that slot, loaded by the caller with its other counters).  False on a
// mismatch.  Out of line, so the hot loop's register allocation does not pay for it.
static __device__ __noinline__ bool agree_step(Counters* ctr, uint32_t it, uint32_t team_size, uint32_t* prev,
                                               uint32_t prev_sum, uint32_t a, uint32_t b, uint32_t c, uint32_t d,
                                               uint32_t e, uint32_t f) {
  const bool ok = it == 0 || prev_sum == *prev * team_size;
  uint32_t h = 0x811C9DC5u;  // FNV-1a over the words
  h = (h ^ a) * 0x01000193u;
  h = (h ^ b) * 0x01000193u;
  h = (h ^ c) * 0x01000193u;
  h = (h ^ d) * 0x01000193u;
  h = (h ^ e) * 0x01000193u;
  h = (h ^ f) * 0x01000193u;
  atomicAdd(&ctr->agree[it % 4], h);
  *prev = h;
  return ok;
}

// Start of a solve, shared by both schedules: distances and stamps, the initial
// frontier in q[0] (the source, or the state form's flagged vertices), a team
// barrier, then the first bucket's width and level (from the policy's start state
// when the learned policy runs).  Returns false when the run must stop.
template <int BS>
__device__ bool start_instance(const LaunchParams& P, const InstDesc& I, Smem<BS>& sm, uint32_t* bar,
                               uint32_t& bar_epoch, uint32_t rank, uint32_t team_size, bool& inject, bool learned,
                               uint32_t& base_out, uint32_t& qlen, uint32_t& delta, int& level) {
  Counters* ctr = I.ctr;
  const uint32_t gthreads = team_size * BS;
  const uint32_t gtid = rank * BS + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t base = __ldcg(I.stamp_base);
  const bool wrap = base > 0xF0000000u;
  if (wrap) base = 0;
  if (I.mode == 0) {
    for (uint32_t v = gtid; v < (uint32_t)I.n; v += gthreads) {
      I.dist[v] = (v == (uint32_t)I.src) ? 0u : kInf;
      if (wrap) { I.mark[v] = 0; I.fmark[v] = 0; I.smark[v] = 0; }
      if ((v & 7u) == 0) {
        // the stamps and row offsets are read at random for the whole run: bring them into
        // L2 with the evict-last priority while the distances are written (R-MAT 22: DRAM
        // bytes 1.383 -> 1.359 GB, 1 % faster)
        asm volatile("prefetch.global.L2::evict_last [%0];" ::"l"(I.mark + v));
        asm volatile("prefetch.global.L2::evict_last [%0];" ::"l"(I.fmark + v));
        asm volatile("prefetch.global.L2::evict_last [%0];" ::"l"(I.row_ptr + v));
      }
    }
    if (rank == 0 && threadIdx.x == 0) {
      I.q[0][0] = I.src;
      ctr->qtail[0] = 1;
    }
  } else {
    // state mode: frontier = vertices with update[v] != 0 (cleared), distances kept
    const uint32_t nr = ((uint32_t)I.n + 31u) & ~31u;
    for (uint32_t v = gtid; v < nr; v += gthreads) {
      bool f[1] = {false};
      if (v < (uint32_t)I.n) {
        f[0] = I.update[v] != 0;
        if (f[0]) I.update[v] = 0;
        if (wrap) { I.mark[v] = 0; I.fmark[v] = 0; I.smark[v] = 0; }
      }
      const int32_t vv[1] = {(int32_t)v};
      append_k<1>(I.q[0], &ctr->qtail[0], I.qcap, f, vv, &ctr->status, lane);
    }
  }
  if (rank == 0 && threadIdx.x == 0) ctr->fmin[0] = ctr->fmin[1] = ctr->fmin[2] = 0xffffffffu;
  if (threadIdx.x == 0) sm.blk_ctr = 0ull;
  const bool inj = inject;
  inject = false;
  if (!team_barrier<BS>(P, sm, bar, bar_epoch, team_size, &ctr->status, inj)) return false;

  if (threadIdx.x == 0) sm.bc_q = __ldcg(&ctr->qtail[0]);
  if (learned) {
    // the weights move to shared memory once, so each evaluation reads no global memory
    static_assert(sizeof(PolicyDev) % 4 == 0, "word copy");
    const uint32_t* src = reinterpret_cast<const uint32_t*>(P.policy);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&sm.pol);
    for (uint32_t i = threadIdx.x; i < sizeof(PolicyDev) / 4; i += BS) dst[i] = __ldg(src + i);
  }
  __syncthreads();
  qlen = min(sm.bc_q, I.qcap);
  delta = I.dsched ? 1u << (I.dsched & 15u) : I.delta;
  level = I.level;
  if (learned) {
    // the first bucket's width and the first level come from the policy too, on the
    // start state.  The first bucket is filled by the source's out-neighbours, so a
    // single-source start reports that frontier: log2(1 + out-degree of the source)
    // and the source's degree bin; the state form reports its initial frontier size
    // and no histogram.  No advances, 1 of n reached.
    if (threadIdx.x == 0) {
      int sbin = -1;
      float f0 = log2f(1.f + (float)qlen);
      if (I.mode == 0 && qlen == 1) {
        const int32_t sd = __ldg(I.row_ptr + I.src + 1) - __ldg(I.row_ptr + I.src);
        sbin = deg_bin(sd);
        f0 = log2f(1.f + (float)sd);
      }
      for (int i = 0; i < NPS_MLP_IN; ++i) {
        float f = 0.f;
        if (i == 0) f = f0;
        if (i >= 1 && i <= 8 && i - 1 == sbin) f = 1.f;
        if (i == 10) f = 1.f / (float)I.n;
        sm.feat[i] = (f - sm.pol.mean[i]) * sm.pol.istd[i];
      }
    }
    if (warp == 0) {
      __syncwarp();
      policy_eval_warp(&sm.pol, sm.feat, sm.pol_choice, lane);
    }
    __syncthreads();
    delta = 1u << sm.pol_choice[0];
    level = sm.pol_choice[1];
  }
  base_out = base;
  return true;
}

// ---------------------------------------------------------------------------
// Solve one instance with the CTAs of one team.  I refers to kernel-parameter
// space (single-instance launches) or to a shared-memory copy (batches).
template <int BS>
__device__ void solve_instance(const LaunchParams& P, const InstDesc& I, Smem<BS>& sm, uint32_t* bar,
                               uint32_t& bar_epoch, uint32_t rank, uint32_t team_size, bool& inject) {
  constexpr int NW = BS / 32;
  Counters* ctr = I.ctr;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t gwarp = rank * NW + warp;
  const bool learned = I.policy == NPS_POLICY_LEARNED && P.policy != nullptr;
  const bool want_iter = learned || (I.trace != nullptr);

  // ---- prologue: distances, stamps, initial frontier, first bucket
  uint32_t base = 0, qlen = 0, delta = 0;
  int level = 0;
  if (!start_instance<BS>(P, I, sm, bar, bar_epoch, rank, team_size, inject, learned, base, qlen, delta, level))
    return;
  uint32_t it = 0, ep = 0;
  uint32_t T = delta == 0 ? 0xffffffffu : delta;
  bool advance = false;
  bool heavy_it = false;  // this iteration relaxes the heavy edges of the settle list
  uint32_t hg = 0;        // settle-list generation
  uint32_t slen = 0;
  uint32_t s_gen = 0;     // entries appended to the settle list of generation hg so far
  uint32_t adv_len = 0, T_old = 0;
  uint32_t hprev_cnt = 0;
  unsigned long long hprev_tot = 0;
  Acc tot = {0, 0, 0, 0};
  PhaseClock pc;
  pc.reset();
  uint32_t buckets = 0;
  uint32_t reached_total = 1;
  const uint32_t hhalf = I.hcap / 2;
  if (threadIdx.x < 8) sm.hist_next[threadIdx.x] = 0;

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
    C.hitem = I.hitem + ((it & 1) ? I.icap : 0);
    C.split = (I.light_heavy && delta != 0) ? delta : 0u;
    C.heavy_iter = heavy_it;
    C.sq = (C.split != 0u && !heavy_it) ? I.sq[hg & 1] : nullptr;
    C.sq_tail = &ctr->stail[hg % 3];
    C.sstamp = base + hg + 1;
    C.sadd = &ctr->sadd[it % 3];
    C.local_rounds = heavy_it ? 0 : I.local_rounds;  // a heavy pass only relaxes heavy edges
    C.order_deg = I.order_degree;
    C.ring = false;  // queues and lists of the iteration schedule
    level_thresholds(level, I.t1, I.t2, I.t3, C.t_warp, C.t_block, C.t_grid);
    // push-time sorting into the grid-tier list: plain iterations at the grid level
    C.early = !heavy_it && C.sq == nullptr && C.t_grid != 0x7fffffff &&
              (I.sort_push > 0 ||
               (I.sort_push == 0 && C.t_grid <= NPS_SORT_AT_PUSH_AUTO_MAX && I.w != nullptr));
    C.want_hist = want_iter;
    const int4* Hprev = I.heavy + ((it & 1) ? 0 : hhalf);
    const int32_t* Hitem = I.hitem + ((it & 1) ? 0 : I.icap);

    if (rank == 0 && threadIdx.x < kStripes) {
      ctr->work[(it + 1) % 3][threadIdx.x * 32] = 0;
      if (threadIdx.x == 0) {
        ctr->qtail[(it + 2) % 3] = 0;
        ctr->heavy[(it + 1) % 3] = 0;
        ctr->ftail[(E + 1) % 3] = 0;
        ctr->fmin[(E + 1) % 3] = 0xffffffffu;
        ctr->sadd[(it + 1) % 3] = 0;
        ctr->agree[(it + 1) % 4] = 0;  // last read by the decision after iteration it - 2
        if (heavy_it) ctr->stail[(hg + 1) % 3] = 0;
        if (want_iter) {
          const uint32_t sl = (it + 1) % 3;
          for (int b = 0; b < 8; ++b) ctr->hist[sl][b] = 0;
          ctr->it_edges[sl] = 0;
          ctr->it_impr[sl] = 0;
          ctr->it_reached[sl] = 0;
          ctr->it_early[sl] = 0;
        }
      }
    }
    if (threadIdx.x < 8) {
      // rows sorted at push in the last iteration belong to this iteration's frontier
      sm.hist[threadIdx.x] = sm.hist_next[threadIdx.x];
      sm.hist_next[threadIdx.x] = 0;
    }
    if (threadIdx.x < 4) sm.it_acc[threadIdx.x] = 0;
    __syncthreads();
    if (threadIdx.x == 0 && it > 0 &&
        !agree_step(ctr, it - 1, team_size, &sm.agree_prev, sm.bc_ag,
                    sm.bc_q + ((P.test_disagree && rank == 1 && it == 1) ? 1u : 0u), (uint32_t)sm.bc_h,
                    (uint32_t)(sm.bc_h >> 32), sm.bc_m, sm.bc_s, advance ? sm.bc_f : 0u)) {
      // the decision that opened this iteration was not the same in every CTA.  It is
      // checked here, off the decision's path, while the other warps start working; the
      // far-pile tail counts only after an advance, the one decision after which it is stable
      atomicCAS(&ctr->status, 0u, (uint32_t)NPS_ERR_INTERNAL);
      atomicExch(P.abort_flag, 1u);
    }

    const int32_t* srcq = advance ? I.fq[ep & 1] : (heavy_it ? I.sq[hg & 1] : I.q[it & 1]);
    const uint32_t srclen = advance ? adv_len : (heavy_it ? slen : qlen);
    const uint32_t n_heavy_items = (uint32_t)((hprev_tot + (1ull << I.item_shift) - 1) >> I.item_shift);
    // vertex items hold 32 frontier entries, or 16 / 8 / 4 when the frontier is small
    // against the team's warps: a small frontier's rows then spread over more warps
    // instead of leaving a few warps with 32 rows each
    uint32_t vper = 32;
    while (vper > 4 && (unsigned long long)srclen < (unsigned long long)vper * team_size * NW) vper >>= 1;
    const uint32_t n_items = n_heavy_items + (srclen + vper - 1) / vper;
    Acc acc = {0, 0, 0, 0};
    Stage S;
    S.nbuf = sm.stage[warp][0];
    S.fbuf = sm.stage[warp][1];
    S.sbuf = sm.stage[warp][2];
    S.ncnt = 0;
    S.fcnt = 0;
    S.scnt = 0;
    S.fmin = 0xffffffffu;
    S.credit = nullptr;  // ring mode only
    S.hnext = sm.hist_next;
    S.enext = &sm.it_acc[3];

    // ---- work loop: heavy chunk items, then vertex items.  With no more items than
    // warps, warp w takes item w (no atomics); otherwise items come from striped
    // counters, the next index requested before the current item is processed, and
    // an exhausted stripe answered by a parallel probe of all stripes.
    {
      const uint32_t team_warps = team_size * NW;
      const bool static_items = n_items <= team_warps;
      uint32_t* wc = &ctr->work[it % 3][0];
      int stripe = (int)(gwarp % kStripes);
      uint32_t t_next = 0;
      bool have_next = false;
      bool static_done = false;
      for (;;) {
        unsigned long long item;
        if (static_items) {
          if (static_done || gwarp >= n_items) break;
          static_done = true;
          item = gwarp;
        } else {
          uint32_t t = 0;
          if (lane == 0) t = have_next ? t_next : atomicAdd(&wc[stripe * 32], 1u);
          t = __shfl_sync(kFull, t, 0);
          have_next = false;
          const uint32_t my_items = n_items > (uint32_t)stripe ? (n_items - stripe + kStripes - 1) / kStripes : 0u;
          if (t >= my_items) {
            // probe every stripe at once; continue on the first one with items left
            const uint32_t li = n_items > (uint32_t)lane ? (n_items - lane + kStripes - 1) / kStripes : 0u;
            const bool avail = lane < kStripes && ld_relaxed_u32(&wc[lane * 32]) < li;
            const uint32_t m = __ballot_sync(kFull, avail);
            if (m == 0) break;
            const unsigned long long mm = (unsigned long long)m | ((unsigned long long)m << kStripes);
            const uint32_t rot = (uint32_t)(mm >> (stripe + 1)) & kStripeMask;  // m rotated right by stripe + 1
            stripe = (stripe + __ffs(rot)) % kStripes;
            continue;
          }
          if (lane == 0) t_next = atomicAdd(&wc[stripe * 32], 1u);
          have_next = true;
          item = (unsigned long long)t * kStripes + stripe;
        }
        NPS_LAP(pc, 0);
        if (item < n_heavy_items) {
          const uint32_t kb = (uint32_t)item << I.item_shift;
          const uint32_t ke = (uint32_t)min((unsigned long long)kb + (1ull << I.item_shift), hprev_tot);
          const int32_t js = __ldcg(Hitem + item);
          walk_item(I, C, Hprev, hprev_cnt, kb, ke, (uint32_t)js, acc, S, lane);
          NPS_LAP(pc, 4);
        } else {
          const uint32_t idx = (uint32_t)(item - n_heavy_items) * vper + lane;
          process_vertex_item<BS>(I, C, sm, ((uint32_t)lane < vper && idx < srclen) ? __ldcg(srcq + idx) : -1, advance,
                                  T_old, want_iter, acc, S, pc, lane);
          // warp-local rounds: vertices this warp just queued for the next iteration are
          // taken back from its staging buffer and processed now, up to local_rounds times;
          // their stamp is reset so a later improvement in this iteration queues them again
          for (int r = 0; r < C.local_rounds && S.ncnt > 0; ++r) {
            const uint32_t k = min(S.ncnt, 32u);
            int32_t lv = -1;
            if ((uint32_t)lane < k) {
              lv = S.nbuf[S.ncnt - k + lane];
              atomicExch(I.mark + lv, 0u);
              __threadfence();  // the reset is visible before lv's distance is read
            }
            __syncwarp();
            S.ncnt -= k;
            process_vertex_item<BS>(I, C, sm, lv, false, T_old, want_iter, acc, S, pc, lane, true);
          }
        }
      }
    }
    NPS_LAP(pc, 0);
    // ---- block tier: the CTA's warps walk the CTA list once
    __syncthreads();
    const uint32_t bcnt = min((uint32_t)(sm.blk_ctr >> 32), (uint32_t)kBlockListCap);
    if (bcnt) {
      // chunks of the stored entries only (overflowed entries were walked by their warp)
      const int4 last = sm.blk[bcnt - 1];
      const uint32_t btot = (uint32_t)last.w + row_chunks(last.x, last.y);
      const uint32_t per = (btot + NW - 1) / NW;
      const unsigned long long kb = (unsigned long long)warp * per;
      const unsigned long long ke = min((unsigned long long)btot, kb + per);
      walk_chunks(I, C, sm.blk, bcnt, kb, ke, acc, S, lane);
      __syncthreads();
      if (threadIdx.x == 0) sm.blk_ctr = 0ull;
    }
    NPS_LAP(pc, 5);
    stage_drain(I, S, C, I.qcap, &ctr->status, lane);
    NPS_LAP(pc, 6);

    // ---- iteration counters (policy features, trace): warp sums into shared
    // memory; thread 0 adds the CTA's totals to the instance counters just before
    // it arrives at the barrier, so the release orders them before the arrival
    if (want_iter) {
      const uint32_t e = __reduce_add_sync(kFull, acc.edges);
      const uint32_t im = __reduce_add_sync(kFull, acc.impr);
      const uint32_t rc = __reduce_add_sync(kFull, acc.reached);
      if (lane == 0) {
        if (e) atomicAdd(&sm.it_acc[0], e);
        if (im) atomicAdd(&sm.it_acc[1], im);
        if (rc) atomicAdd(&sm.it_acc[2], rc);
      }
    }
    tot.edges += acc.edges;
    tot.impr += acc.impr;
    tot.reached += acc.reached;
    tot.processed += acc.processed;

    NPS_LAP(pc, 8);
    if (!team_barrier<BS>(P, sm, bar, bar_epoch, team_size, &ctr->status, false, false,
                          want_iter ? ctr : nullptr, it % 3))
      return;
    NPS_LAP(pc, 7);

    // ---- decide the next iteration (every CTA reads the same values)
    if (advance) {
      ep += 1;
      buckets += 1;
    }
    if (heavy_it) hg += 1;
    // thread 0 reads the shared counters, the status word and (for the policy or
    // the trace) this iteration's statistics in one batch of loads, and
    // broadcasts them; with the learned policy, warp 0 then evaluates the MLP on
    // the features thread 0 computed (every CTA reads the same counters, so every
    // CTA takes the same decision)
    if (threadIdx.x == 0) {
      const uint32_t sl = it % 3;
      const uint32_t q1 = __ldcg(&ctr->qtail[(it + 1) % 3]);
      const uint32_t ag = __ldcg(&ctr->agree[(it + 3) % 4]);
      const unsigned long long h1 = ld_relaxed_u64(&ctr->heavy[it % 3]);
      const uint32_t f1 = __ldcg(&ctr->ftail[ep % 3]);
      const uint32_t m1 = __ldcg(&ctr->fmin[ep % 3]);
      const uint32_t s1 = __ldcg(&ctr->sadd[it % 3]);
      const uint32_t st1 = ld_relaxed_u32(&ctr->status);
      uint32_t hb[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      unsigned long long ie = 0, ii = 0;
      uint32_t ir = 0, ea = 0;
      if (want_iter) {
        for (int b = 0; b < 8; ++b) hb[b] = __ldcg(&ctr->hist[sl][b]);
        ie = __ldcg(&ctr->it_edges[sl]);
        ii = __ldcg(&ctr->it_impr[sl]);
        ir = __ldcg(&ctr->it_reached[sl]);
        ea = __ldcg(&ctr->it_early[sl]);
      }
      sm.bc_q = q1;
      sm.bc_h = h1;
      sm.bc_f = f1;
      sm.bc_m = m1;
      sm.bc_s = s1;
      sm.bc_ag = ag;
      if (st1 != 0) {
        atomicExch(P.abort_flag, 1u);
        sm.ok = 0;
      }
      if (want_iter) {
        // The 12 policy features: log2 of the next frontier, the out-degree histogram
        // of this iteration's frontier as 8 fractions, log2(1 + bucket advances), the
        // reached fraction, improvements per scanned edge.
        reached_total += ir;
        const uint32_t qn0 = min(q1, I.qcap);
        const uint32_t fl0 = min(f1, I.qcap);
        const uint32_t hn0 = min((uint32_t)(h1 >> kHeavyShift), hhalf);
        // an advance follows only when no heavy pass does (the far-pile length is stable only
        // then: a light or heavy pass may already be pushing to it in a faster CTA)
        const bool heavy0 = I.light_heavy && delta != 0 && min(s_gen + s1, I.qcap) != 0;
        const bool adv0 = qn0 == 0 && hn0 == 0 && !heavy0 && fl0 != 0;
        float hs = 0.f;
        for (int b = 0; b < 8; ++b) hs += (float)hb[b];
        const float inv = hs > 0.f ? 1.f / hs : 0.f;
        float f[NPS_MLP_IN];
        // the next frontier: its queue and the rows sorted into the grid-tier list at push
        f[0] = log2f(1.f + (float)(adv0 ? fl0 : qn0 + ea));
        for (int b = 0; b < 8; ++b) f[1 + b] = (float)hb[b] * inv;
        f[9] = log2f(1.f + (float)buckets);
        f[10] = (float)reached_total / (float)I.n;
        f[11] = ie ? (float)ii / (float)ie : 0.f;
        if (learned)
          for (int i = 0; i < NPS_MLP_IN; ++i) sm.feat[i] = (f[i] - sm.pol.mean[i]) * sm.pol.istd[i];
        if (I.trace && rank == 0 && it < I.trace_cap) {
          nps_trace_rec* tr = I.trace + it;
          tr->iteration = it;
          tr->frontier = srclen;
          tr->far_len = fl0;
          tr->bucket_hi = T;
          tr->delta = delta;
          tr->level = (uint32_t)level | (heavy_it ? 0x100u : 0u) | (advance ? 0x200u : 0u);
          for (int b = 0; b < 8; ++b) tr->hist[b] = hb[b];
          tr->edges = ie;
          tr->improvements = ii;
          tr->reached = reached_total;
          tr->heavy = hn0;
          tr->t_ns = globaltimer_ns() - sm.t_start;
          for (int i = 0; i < NPS_MLP_IN; ++i) tr->feat[i] = f[i];
        }
      }
    }
    if (learned && warp == 0) {
      __syncwarp();
      if (sm.ok) policy_eval_warp(&sm.pol, sm.feat, sm.pol_choice, lane);
    }
    __syncthreads();
    if (!sm.ok) return;
    const uint32_t qn = min(sm.bc_q, I.qcap);
    const unsigned long long hc = sm.bc_h;
    const uint32_t hn = min((uint32_t)(hc >> kHeavyShift), hhalf);
    const uint32_t fl = min(sm.bc_f, I.qcap);
    if (learned) level = sm.pol_choice[1];

    hprev_cnt = hn;
    hprev_tot = hc & kHeavyMask;
    advance = false;
    // entries of the current settle list: every CTA adds the same per-iteration counts
    s_gen += sm.bc_s;
    const uint32_t sn = min(s_gen, I.qcap);
    const bool split_now = I.light_heavy && delta != 0;
    heavy_it = false;
    if (qn == 0 && hn == 0 && split_now && sn != 0) {
      // bucket drained: relax the heavy edges of every vertex it settled, once
      heavy_it = true;
      slen = sn;
      s_gen = 0;  // the heavy iteration appends nothing; the next list starts empty
    } else if (qn == 0 && hn == 0) {
      if (fl == 0) {
        it += 1;
        break;
      }
      // bucket advance: the next iteration filters the far pile of epoch ep
      if (learned) {
        delta = 1u << sm.pol_choice[0];
      } else if (I.dsched) {
        const uint32_t b = min(buckets + 1u, 7u);  // index of the bucket this advance opens
        delta = 1u << ((I.dsched >> (4u * b)) & 15u);
      }
      const uint32_t fm = sm.bc_m;
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
  }
#ifdef NPS_PROFILE
  if (lane == 0)
    for (int i = 0; i < 9; ++i) atomicAdd(&ctr->prof[i], pc.acc[i]);
#endif
  if (threadIdx.x == 0) {
    if (rank == 0) {
      ctr->iterations = it;
      ctr->solve_ns = globaltimer_ns() - sm.t_start;
      ctr->buckets = buckets;
      *I.stamp_base = base + (it > ep ? it : ep) + 4;
    }
  }
}

// ---------------------------------------------------------------------------
// Asynchronous buckets (InstDesc::async).  Inside a bucket nothing waits for a
// barrier: a vertex improved below the bucket bound goes to the near ring, a row
// of at least `threshold` edges becomes 256-edge segments on the segment ring,
// and every warp takes work as soon as it appears -- a segment first, then one of
// the bucket's static items (32 entries of the far pile being filtered on an
// advance, or of the initial frontier), then up to 32 near-ring vertices.
//
// The bucket ends when its static items are done and the pending total is zero.
// Ring units (vertices and segments) join the pending total before they become
// visible, and a warp subtracts the units it took only after everything they
// pushed has been counted, so the total is zero only when no unit is queued or
// being processed.  Only then does the team meet at a barrier, to pick the next
// bucket (the far pile's smallest distance, the policy's width).  Results are
// exact for the reason the iteration schedule's are: the scheme is
// label-correcting, and a vertex whose distance drops after it was taken from the
// ring is queued again -- its mark is reset (an acquire) before its distance is
// read, and the mark is set (a release) after the atomicMin that improved the
// distance.
//
// Ring slots carry tags (Vyukov's bounded queue): index i may be written once its
// slot holds tag i and read once it holds i + 1; a reader then writes i + capacity.
// Head and tail persist across runs.  Every warp holds one claimed segment index
// and one claimed window of 32 near-ring indices, and polls only those slots; it
// claims again when it takes a filled segment, or the last entry of its window,
// while it still holds that unit (so the bucket cannot end between).  Claims
// beyond the tail are filled by later pushes; those still empty when the bucket
// ends are handed back by their warp, and after the team barrier the tails are
// moved up to the heads, one more barrier ahead of the next bucket.
template <int BS>
__device__ void solve_instance_async(const LaunchParams& P, const InstDesc& I, Smem<BS>& sm, uint32_t* bar,
                                     uint32_t& bar_epoch, uint32_t rank, uint32_t team_size, bool& inject) {
  Counters* ctr = I.ctr;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool learned = I.policy == NPS_POLICY_LEARNED && P.policy != nullptr;
  const bool want_iter = learned || (I.trace != nullptr);
  const uint32_t QC = I.nq_mask + 1, SC = I.seg_mask + 1;

  uint32_t base = 0, srclen = 0, delta = 0;
  int level = 0;
  if (!start_instance<BS>(P, I, sm, bar, bar_epoch, rank, team_size, inject, learned, base, srclen, delta, level))
    return;
  const int32_t* srcq = I.q[0];
  bool advance = false;
  uint32_t p = 0;  // bucket (phase) index; its far pushes go to epoch p
  uint32_t T = delta == 0 ? 0xffffffffu : delta, T_old = 0;
  Acc tot = {0, 0, 0, 0};
  PhaseClock pc;
  pc.reset();
  uint32_t reached_total = 1;

  for (;;) {
    IterCtx C;
    C.T = T;
    C.snear = base + p + 1;
    C.sfar = base + p + 1;
    C.qn = nullptr;
    C.qn_tail = nullptr;
    C.fp = I.fq[p & 1];
    C.fp_tail = &ctr->ftail[p % 3];
    C.fp_min = nullptr;  // kept per lane in Stage::fmin
    C.heavy = nullptr;
    C.heavy_ctr = nullptr;
    C.hcap = 0;
    C.hitem = nullptr;
    C.t_warp = C.t_block = C.t_grid = I.t1;  // GRID tiers: rows of >= threshold edges become segments
    C.split = 0u;
    C.heavy_iter = false;
    C.sq = nullptr;
    C.sq_tail = &ctr->stail[0];
    C.sstamp = 0;
    C.local_rounds = 0;
    C.order_deg = I.order_degree;
    C.ring = true;
    C.sadd = nullptr;
    C.early = false;
    C.want_hist = false;
    if (rank == 0 && threadIdx.x == 0) {
      // slots of the next bucket (their last user ended two barriers ago)
      const uint32_t sl = (p + 1) % 3;
      ctr->ftail[sl] = 0;
      ctr->fmin[sl] = 0xffffffffu;
      ctr->swork[sl] = 0;
      ctr->sdone[sl] = 0;
      if (want_iter) {
        for (int b = 0; b < 8; ++b) ctr->hist[sl][b] = 0;
        ctr->it_edges[sl] = 0;
        ctr->it_impr[sl] = 0;
        ctr->it_reached[sl] = 0;
      }
    }
    if (threadIdx.x < 8) sm.hist[threadIdx.x] = 0;
    if (threadIdx.x < 4) sm.it_acc[threadIdx.x] = 0;
    if (threadIdx.x == 0) sm.phase_flag = 0;
    __syncthreads();

    const uint32_t n_static = (srclen + 31) / 32;
    Acc acc = {0, 0, 0, 0};
    Stage S;
    S.nbuf = sm.stage[warp][0];
    S.fbuf = sm.stage[warp][1];
    S.sbuf = sm.stage[warp][2];
    S.ncnt = S.fcnt = S.scnt = 0;
    S.fmin = 0xffffffffu;
    S.credit = &sm.credit[warp];
    S.hnext = sm.hist_next;
    S.enext = &sm.it_acc[3];
    if (lane == 0) sm.credit[warp] = 0;
    uint32_t D = 0;        // ring units taken and processed, not yet subtracted from the pending total
    uint32_t sdone_w = 0;  // static items processed, not yet added to sdone
    bool static_left = n_static > 0;
    uint32_t wb = 0, om = 0;  // claimed near-ring window and its lanes still to read
    bool has_seg = false;
    uint32_t sidx = 0;
    uint32_t idle = 0;
    unsigned long long t_idle = 0;
    bool fin = false;
    for (;;) {
      bool did = false;
      // (1) a segment.  The warp always holds one claimed index of the segment ring and
      // polls only that slot's tag (no shared counter is read while waiting); taking a
      // filled slot claims the next index at once, so the claim's round trip overlaps
      // the walk.  Claims beyond the tail wait for later pushes -- at most one per warp.
      if (!has_seg) {
        uint32_t si = 0;
        if (lane == 0) si = atomicAdd(&I.rs->seg_head, 1u);
        sidx = __shfl_sync(kFull, si, 0);
        has_seg = true;
      }
      {
        int4 sg = make_int4(0, 0, 0, 0);
        uint32_t ready = 0, next = 0;
        if (lane == 0) {
          int4* slot = I.seg + (sidx & I.seg_mask);
          uint32_t* tag = reinterpret_cast<uint32_t*>(slot) + 3;
          const uint32_t tg = ld_relaxed_u32(tag);
          if (tg == sidx + 1) {
            sg = ld_relaxed_v4(slot + dep_zero(tg));  // the payload, read after the tag ...
            // ... and back before the slot is handed back (the store waits for it)
            st_relaxed_u32(tag + dep_zero((uint32_t)sg.x ^ (uint32_t)sg.y ^ (uint32_t)sg.z), sidx + SC);
            next = atomicAdd(&I.rs->seg_head, 1u);
            ready = 1;
          }
        }
        if (__shfl_sync(kFull, ready, 0)) {
          sg.x = __shfl_sync(kFull, sg.x, 0);
          sg.y = __shfl_sync(kFull, sg.y, 0);
          sg.z = __shfl_sync(kFull, sg.z, 0);
          walk_segment(I, C, sg, acc, S, lane);
          sidx = __shfl_sync(kFull, next, 0);
          D += 1;
          did = true;
        }
      }
      // (2) a static item
      if (!did && static_left) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(&ctr->swork[p % 3], 1u);
        t = __shfl_sync(kFull, t, 0);
        if (t < n_static) {
          const uint32_t idx = t * 32 + lane;
          process_vertex_item<BS>(I, C, sm, idx < srclen ? __ldcg(srcq + idx) : -1, advance, T_old, want_iter, acc,
                                  S, pc, lane);
          sdone_w += 1;
          did = true;
        } else {
          static_left = false;
        }
      }
      // (3) near-ring vertices
      if (!did) {
        if (om == 0) {
          // a new window once every slot of the last one was taken (as for segments,
          // at most one claimed window per warp, polled slot by slot)
          uint32_t b = 0;
          if (lane == 0) b = atomicAdd(&I.rs->nq_head, 32u);
          wb = __shfl_sync(kFull, b, 0);
          om = kFull;
        }
        if (om) {
          int32_t v = -1;
          if (om & (1u << lane)) {
            const uint32_t idx = wb + lane;
            unsigned long long* slot = I.nq + (idx & I.nq_mask);
            const unsigned long long x = ld_relaxed_u64p(slot);
            if ((uint32_t)(x >> 32) == idx + 1) {
              v = (int32_t)(uint32_t)x;
              st_relaxed_u64(slot, ((unsigned long long)(idx + QC) << 32) | 0xffffffffull);
              if ((uint32_t)v >= (uint32_t)I.n) {  // never pushed by a producer: record and drop
                atomicCAS(&ctr->status, 0u, (uint32_t)NPS_ERR_CAPACITY);
                v = -1;
              }
            }
          }
          const uint32_t tm = __ballot_sync(kFull, v >= 0);
          om &= ~tm;
          if (tm) {
            if (v >= 0) {
              // the mark is reset before the distance is read: a drop after this
              // exchange queues v again, one before it is seen by the read.  The reset
              // is an acquire, paired with the producer's release: a relaxed reset
              // followed by a dependent load still returned a stale distance on B200
              // (a few vertices in a thousand runs came out too long)
              const uint32_t old = atom_exch_acquire(I.mark + v, 0u);
              v += (int32_t)dep_zero(old);
            }
            process_vertex_item<BS>(I, C, sm, v, false, T_old, want_iter, acc, S, pc, lane);
            D += __popc(tm);
            did = true;
          }
        }
      }
      if (did) {
        idle = 0;
        continue;
      }
      // (4) no work at hand: publish what this warp holds, then test for the end of the
      // bucket.  Only the CTA's warp 0 reads the shared counters; it tells the CTA's
      // other warps through shared memory, so idle warps do not crowd those lines.
      stage_drain(I, S, C, I.qcap, &ctr->status, lane);
      uint32_t f = 0, stop = 0;
      if (lane == 0) {
        const uint32_t back = D + sm.credit[warp];  // processed units and unused credits
        if (sdone_w || back) {
          __threadfence();  // this warp's pushes are covered before its items and units are done
          if (sdone_w) atomicAdd(&ctr->sdone[p % 3], sdone_w);
          if (back) atomicSub(&ctr->pend, back);
          sm.credit[warp] = 0;
        }
        const unsigned long long now = globaltimer_ns();
        if (idle == 0) t_idle = now;
        const uint32_t flag = *(volatile uint32_t*)&sm.phase_flag;
        if (flag == p + 1) {
          f = 1;
        } else if (flag == 0xffffffffu) {
          stop = 1;
        } else if (warp == 0) {
          if (idle >= 1) {
            const uint32_t sd = ld_relaxed_u32(&ctr->sdone[p % 3]);
            if (sd >= n_static) f = ld_relaxed_u32(&ctr->pend + dep_zero(sd)) == 0;
          }
          if (!f && (idle & 15) == 15 &&
              (ld_relaxed_u32(&ctr->status) != 0 || ld_relaxed_u32(P.abort_flag) != 0))
            stop = 1;
          if (f || stop) *(volatile uint32_t*)&sm.phase_flag = f ? p + 1 : 0xffffffffu;
        }
        if (!f && !stop && (now - t_idle > P.timeout_ns || now - sm.t_start > P.run_budget_ns)) {
          atomicCAS(&ctr->status, 0u, (uint32_t)NPS_ERR_TIMEOUT);
          atomicExch(P.abort_flag, 1u);
          *(volatile uint32_t*)&sm.phase_flag = 0xffffffffu;
          stop = 1;
        }
      }
      sdone_w = 0;
      D = 0;
      if (__shfl_sync(kFull, f, 0)) {
        fin = true;
        break;
      }
      if (__shfl_sync(kFull, stop, 0)) break;
      ++idle;
      __nanosleep(idle < 4 ? 64u : (idle < 12 ? 256u : 1024u));  // idle warps back off the shared counters
    }
    if (fin) {
      // claims never filled: nothing more arrives in this bucket, hand the slots back
      if (has_seg && lane == 0) st_release_u32(reinterpret_cast<uint32_t*>(I.seg + (sidx & I.seg_mask)) + 3, sidx + SC);
      if (om & (1u << lane))
        st_relaxed_u64(I.nq + ((wb + lane) & I.nq_mask), ((unsigned long long)(wb + lane + QC) << 32) | 0xffffffffull);
    }
    {
      const uint32_t fm = __reduce_min_sync(kFull, S.fmin);
      if (lane == 0 && fm != 0xffffffffu) atomicMin(&ctr->fmin[p % 3], fm);
    }
    if (want_iter) {
      const uint32_t e = __reduce_add_sync(kFull, acc.edges);
      const uint32_t im = __reduce_add_sync(kFull, acc.impr);
      const uint32_t rc = __reduce_add_sync(kFull, acc.reached);
      if (lane == 0) {
        if (e) atomicAdd(&sm.it_acc[0], e);
        if (im) atomicAdd(&sm.it_acc[1], im);
        if (rc) atomicAdd(&sm.it_acc[2], rc);
      }
    }
    tot.edges += acc.edges;
    tot.impr += acc.impr;
    tot.reached += acc.reached;
    tot.processed += acc.processed;
    __syncthreads();
    if (!team_barrier<BS>(P, sm, bar, bar_epoch, team_size, &ctr->status, false, false,
                          want_iter ? ctr : nullptr, p % 3))
      return;
    if (rank == 0 && threadIdx.x == 0) {
      // every warp of the team has left the bucket and handed back its unfilled
      // claims: move the tails up to the heads, past every claim, before anything
      // is pushed again (the next bucket starts after one more barrier; the next
      // run, after the launch ends)
      const uint32_t nh = ld_relaxed_u32(&I.rs->nq_head), nt = ld_relaxed_u32(&I.rs->nq_tail);
      if ((int32_t)(nh - nt) > 0) atomicExch(&I.rs->nq_tail, nh);
      const uint32_t sh = ld_relaxed_u32(&I.rs->seg_head), st = ld_relaxed_u32(&I.rs->seg_tail);
      if ((int32_t)(sh - st) > 0) atomicExch(&I.rs->seg_tail, sh);
    }

    // ---- the next bucket (every CTA reads the same values)
    if (threadIdx.x == 0) {
      const uint32_t sl = p % 3;
      const uint32_t f1 = __ldcg(&ctr->ftail[sl]);
      const uint32_t m1 = __ldcg(&ctr->fmin[sl]);
      const uint32_t st1 = ld_relaxed_u32(&ctr->status);
      sm.bc_f = f1;
      sm.bc_m = m1;
      if (st1 != 0) {
        atomicExch(P.abort_flag, 1u);
        sm.ok = 0;
      }
      if (want_iter) {
        uint32_t hb[8];
        for (int b = 0; b < 8; ++b) hb[b] = __ldcg(&ctr->hist[sl][b]);
        const unsigned long long ie = __ldcg(&ctr->it_edges[sl]);
        const unsigned long long ii = __ldcg(&ctr->it_impr[sl]);
        const uint32_t ir = __ldcg(&ctr->it_reached[sl]);
        // the iteration schedule's 12 features, over the whole bucket: the next
        // frontier (the far pile), the degree histogram of the bucket's vertices,
        // log2(1 + advances), the reached fraction, improvements per scanned edge
        reached_total += ir;
        const uint32_t fl0 = min(f1, I.qcap);
        float hs = 0.f;
        for (int b = 0; b < 8; ++b) hs += (float)hb[b];
        const float inv = hs > 0.f ? 1.f / hs : 0.f;
        float fv[NPS_MLP_IN];
        fv[0] = log2f(1.f + (float)fl0);
        for (int b = 0; b < 8; ++b) fv[1 + b] = (float)hb[b] * inv;
        fv[9] = log2f(1.f + (float)p);
        fv[10] = (float)reached_total / (float)I.n;
        fv[11] = ie ? (float)ii / (float)ie : 0.f;
        if (learned)
          for (int i = 0; i < NPS_MLP_IN; ++i) sm.feat[i] = (fv[i] - sm.pol.mean[i]) * sm.pol.istd[i];
        if (I.trace && rank == 0 && p < I.trace_cap) {
          nps_trace_rec* tr = I.trace + p;
          tr->iteration = p;
          tr->frontier = srclen;
          tr->far_len = fl0;
          tr->bucket_hi = T;
          tr->delta = delta;
          tr->level = (uint32_t)NPS_LEVEL_GRID | (advance ? 0x200u : 0u) | 0x400u;  // 0x400: asynchronous bucket
          for (int b = 0; b < 8; ++b) tr->hist[b] = hb[b];
          tr->edges = ie;
          tr->improvements = ii;
          tr->reached = reached_total;
          tr->heavy = 0;
          tr->t_ns = globaltimer_ns() - sm.t_start;
          for (int i = 0; i < NPS_MLP_IN; ++i) tr->feat[i] = fv[i];
        }
      }
    }
    if (learned && warp == 0) {
      __syncwarp();
      if (sm.ok) policy_eval_warp(&sm.pol, sm.feat, sm.pol_choice, lane);
    }
    __syncthreads();
    if (!sm.ok) return;
    const uint32_t fl = min(sm.bc_f, I.qcap);
    p += 1;
    if (fl == 0) break;
    // bucket advance: the next bucket filters the far pile of this one
    if (learned) {
      delta = 1u << sm.pol_choice[0];
    } else if (I.dsched) {
      const uint32_t b = min(p, 7u);  // index of the bucket this advance opens
      delta = 1u << ((I.dsched >> (4u * b)) & 15u);
    }
    const uint32_t fm = sm.bc_m;
    const uint32_t dstep = delta ? delta : 1u;
    unsigned long long nt = (unsigned long long)T + dstep;
    if (fm != 0xffffffffu && (unsigned long long)fm + dstep > nt) nt = (unsigned long long)fm + dstep;
    T_old = T;
    T = nt >= 0xffffffffull ? 0xfffffffeu : (uint32_t)nt;
    advance = true;
    srcq = I.fq[(p - 1) & 1];
    srclen = fl;
    // the ring counters are set before the next bucket pushes or claims anything
    if (!team_barrier<BS>(P, sm, bar, bar_epoch, team_size, &ctr->status, false)) return;
  }
  (void)level;

  // ---- epilogue: totals and the stamp base for the next run on this workspace
  uint32_t r[4];
  block_sum4<BS>(sm, tot.edges, tot.impr, tot.reached, tot.processed, r);
  if (threadIdx.x == 0) {
    atomicAdd(&ctr->edges, (unsigned long long)r[0]);
    atomicAdd(&ctr->improvements, (unsigned long long)r[1]);
    atomicAdd(&ctr->reached, r[2]);
    atomicAdd(&ctr->processed, (unsigned long long)r[3]);
    if (rank == 0) {
      ctr->iterations = p;
      ctr->solve_ns = globaltimer_ns() - sm.t_start;
      ctr->buckets = p - 1;
      *I.stamp_base = base + p + 4;
    }
  }
}

// Resident CTAs per SM the register budget is sized for (about 768-1024
// threads per SM: enough warps in flight to cover L2 and HBM latency).
template <int BS>
constexpr int kMinBlocks = BS >= 512 ? 2 : (BS >= 256 ? 3 : 6);

// The persistent kernel.  SINGLE: one instance whose descriptor is the kernel
// parameter `single` (constant-bank reads in the hot loops); otherwise the
// team's instances are staged one at a time in shared memory.  ASYNC (single
// instances only): the asynchronous bucket schedule, in a kernel of its own so
// that each schedule gets its own register allocation.
template <int BS, bool SINGLE, bool ASYNC = false>
__global__ void __launch_bounds__(BS, kMinBlocks<BS>) sssp_persistent_kernel(const __grid_constant__ LaunchParams P,
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
  uint32_t* bar = P.bar + (size_t)P.bar_stride * sm.team_id;
  uint32_t bar_epoch = 0;
  const uint32_t rank = blockIdx.x - td.cta_begin;
  if (threadIdx.x == 0) sm.rank = rank;
  __syncthreads();
  bool inject = P.fault_inject_wait != 0;
  if constexpr (SINGLE && ASYNC) {
    solve_instance_async<BS>(P, single, sm, bar, bar_epoch, rank, (uint32_t)td.cta_count, inject);
  } else if constexpr (SINGLE) {
    solve_instance<BS>(P, single, sm, bar, bar_epoch, rank, (uint32_t)td.cta_count, inject);
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
