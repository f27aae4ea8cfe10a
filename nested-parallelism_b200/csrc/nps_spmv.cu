// Sparse matrix-vector product y = A x in double precision on a CSR matrix: the
// SpMV application's consolidated kernel (spmv_np_consolidate_gpu,
// apps/SpMV/src/gpu/SpMV_wrapper.cu:285-311; csr_spmv_warp_dp_kernel,
// csr_spmv_block_dp_kernel and csr_spmv_grid_dp_kernel, SpMV_kernel.cu:353-541),
// the same degree-based consolidation as the SSSP engine applied to a single
// pass over the rows.  FLOAT_T is double in the reference (SpMV.h:13).
//
// Rows below `threshold` nonzeros ("small") are walked flat: a warp takes 32
// consecutive rows, concatenates their small rows' nonzeros and walks them 64 at
// a time (two rounds of 32 with their loads in flight together), so consecutive
// lanes read consecutive nonzeros (coalesced) whatever the row lengths.  Each lane finds the row of its nonzero by a 5-step shuffle
// search over the warp's exclusive prefix of row lengths, and every round ends
// in a segmented shuffle reduction that hands each row's share to the lane that
// owns the row.  Rows of at least `threshold` nonzeros ("large") are
// consolidated at the requested level, as the reference's CONSOLIDATE_LEVEL:
//   WARP   the warp that met the row walks it, 32 lanes strided
//   BLOCK  the CTA lists its large rows in shared memory and walks each with
//          all its threads
//   GRID   large rows go to one device list, split into 1024-nonzero chunks
//          described in a chunk table; a second kernel gives each chunk to a
//          warp, and the warp that finishes a row's last chunk adds the row's
//          chunk sums in chunk order
//
// Every y[r] is summed in an order fixed by the matrix alone (round by round,
// then a fixed shuffle tree; chunk by chunk for GRID rows), so results repeat
// bit for bit from run to run, unlike the reference's scheduling-dependent
// order.  With the reference's data (val[i] = i % 13 + 0.5, x[i] = i % 17 + 0.5,
// SpMV_wrapper.cu:105-113) every partial sum is a multiple of 0.25 far below
// 2^50, so any order gives the same, exact y.
//
// HBM traffic: 12 bytes per nonzero (column index and value, streamed once with
// evict-first loads), row offsets, y, and x (read through L2, 8 n bytes when it
// stays resident).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "nps.h"
#include "nps_internal.h"

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kChunk = 1024;  // nonzeros per grid-level chunk
constexpr int kStripes = 8;
// Loads in flight per lane in a grid-level chunk, and the resident CTAs per SM
// the chunk kernel is built for.  On R-MAT scale 22 the pairs (8, 4), (4, 5),
// (4, 6) and (2, 8) all take 0.56-0.58 ms: the kernel is bound by L2 sector
// traffic for the x gathers, not by loads in flight.
constexpr int kBatch = 8;
constexpr int kChunkCtas = 4;        // row-group counters, so CTAs do not queue on one address
constexpr unsigned kFull = 0xffffffffu;

struct SpmvCtr {
  unsigned long long list;  // grid level: (large rows << 32) | chunks, reserved together
  uint32_t status;
  uint32_t next[kStripes];  // next unit of kWarps row groups, per stripe
};

struct LargeRow {
  int32_t row;
  uint32_t chunk_begin;
  uint32_t chunks;
  uint32_t done;  // chunks finished
};

struct ChunkDesc {
  int32_t row;
  int32_t start;  // nonzero range [start, end)
  int32_t end;
  int32_t entry;  // list entry of the row when it has more than one chunk, else -1
};

struct Mat {
  const int32_t* row;
  const int32_t* col;
  const double* val;
  const double* x;
  double* y;
  int32_t n;
  int64_t m;
};

__device__ __forceinline__ double warp_sum(double v) {
  // butterfly: a + b == b + a, so every lane ends with the same, fixed-order sum
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ void flag_format(SpmvCtr* c) { atomicCAS(&c->status, 0u, (uint32_t)NPS_ERR_FORMAT); }

// x[j] for a column index read from the matrix (0 and FORMAT when out of range).
__device__ __forceinline__ double x_at(const Mat& A, int32_t j, SpmvCtr* c) {
  if ((uint32_t)j >= (uint32_t)A.n) {
    flag_format(c);
    return 0.0;
  }
  return __ldg(A.x + j);
}

// Sum of the nonzeros [s, e) by one warp, lanes strided by 32, in batches of
// 256: each lane loads up to eight column indices and values (predicated at the
// end of the range) before any x, so a batch costs one round trip for the index
// and one for x however short the range.  Column indices and values are read
// once (evict-first), x through L2.  Every lane returns the same sum.
template <int B>
__device__ __forceinline__ double warp_range(const Mat& A, int64_t s, int64_t e, int lane, SpmvCtr* c) {
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t k = s + lane; k - lane < e; k += B * 32) {
    int32_t cj[B];
    double v[B];
#pragma unroll
    for (int i = 0; i < B; ++i) {
      const bool in = k + 32 * i < e;
      cj[i] = in ? __ldcs(A.col + k + 32 * i) : 0;
      v[i] = in ? __ldcs(A.val + k + 32 * i) : 0.0;
    }
#pragma unroll
    for (int i = 0; i < B; ++i)
      if (k + 32 * i < e) acc[i & 3] += v[i] * x_at(A, cj[i], c);
  }
  return warp_sum((acc[0] + acc[1]) + (acc[2] + acc[3]));
}

// Row bounds; a malformed row is reported and treated as empty.
__device__ __forceinline__ void row_bounds(const Mat& A, int64_t r, int32_t& s, int32_t& e, SpmvCtr* c) {
  s = A.row[r];
  e = A.row[r + 1];
  if (s < 0 || e < s || (int64_t)e > A.m) {
    flag_format(c);
    s = e = 0;
  }
}

// Lane of the warp whose small rows hold flat position k: the last lane whose
// exclusive prefix is <= k (rows are contiguous in k).
__device__ __forceinline__ int owner_of(uint32_t excl, uint32_t k) {
  int o = 0;
#pragma unroll
  for (int step = 16; step >= 1; step >>= 1) {
    const uint32_t x = __shfl_sync(kFull, excl, o + step);
    if (x <= k) o += step;
  }
  return o;
}

// Segmented sum toward each segment's first lane; `own` labels the segments
// (equal labels are contiguous).
__device__ __forceinline__ double seg_sum(double v, int own, int lane) {
#pragma unroll
  for (int dd = 1; dd < 32; dd <<= 1) {
    const double vo = __shfl_down_sync(kFull, v, dd);
    const int oo = __shfl_down_sync(kFull, own, dd);
    if (lane + dd < 32 && oo == own) v += vo;
  }
  return v;
}

// The share of this lane's row in the round of flat positions [base, base + 32):
// the segment sum held by the segment's first lane.
__device__ __forceinline__ double my_share(double seg, uint32_t d, uint32_t excl, uint32_t base) {
  const bool mine = d > 0 && excl < base + 32 && excl + d > base;
  const int h = mine ? (int)(max(excl, base) - base) : 0;
  const double got = __shfl_sync(kFull, seg, h);
  return mine ? got : 0.0;
}

// The small rows of group g (rows [32 g, 32 g + 32), bounds s, e of this lane's
// row): walked flat, two rounds of 32 positions per step so both rounds' loads
// are in flight together; writes y for them and returns whether this lane's row
// is large.
__device__ __forceinline__ bool small_rows(const Mat& A, int64_t g, int32_t s, int32_t e, int32_t threshold,
                                           int lane, SpmvCtr* c) {
  const int64_t r = g * 32 + lane;
  const int32_t deg = e - s;
  const bool large = deg >= threshold;
  const uint32_t d = large ? 0u : (uint32_t)deg;
  uint32_t incl = d;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += t;
  }
  const uint32_t excl = incl - d;
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  double acc = 0.0;
  for (uint32_t base = 0; base < total; base += 64) {
    const uint32_t k0 = base + lane, k1 = k0 + 32;
    const int o0 = owner_of(excl, k0), o1 = owner_of(excl, k1);
    const int32_t s0 = __shfl_sync(kFull, s, o0), s1 = __shfl_sync(kFull, s, o1);
    const uint32_t e0 = __shfl_sync(kFull, excl, o0), e1 = __shfl_sync(kFull, excl, o1);
    const bool ok0 = k0 < total, ok1 = k1 < total;
    const int64_t i0 = (int64_t)s0 + (k0 - e0), i1 = (int64_t)s1 + (k1 - e1);
    const int32_t c0 = ok0 ? __ldcs(A.col + i0) : 0, c1 = ok1 ? __ldcs(A.col + i1) : 0;
    const double w0 = ok0 ? __ldcs(A.val + i0) : 0.0, w1 = ok1 ? __ldcs(A.val + i1) : 0.0;
    const double v0 = ok0 ? w0 * x_at(A, c0, c) : 0.0;
    const double v1 = ok1 ? w1 * x_at(A, c1, c) : 0.0;
    const double g0 = seg_sum(v0, ok0 ? o0 : 32 + lane, lane);
    const double g1 = seg_sum(v1, ok1 ? o1 : 32 + lane, lane);
    acc += my_share(g0, d, excl, base);
    acc += my_share(g1, d, excl, base + 32);
  }
  if (r < A.n && !large) A.y[r] = acc;
  return large;
}

// Next row group for a warp from kStripes striped counters: one atomic, issued
// by lane 0, whose result is used one group later so its latency overlaps the
// walk.  A stripe that runs dry sends the warp to the next stripe.
struct GroupFeed {
  int stripe, tried;
  int64_t per_stripe, groups;
  __device__ __forceinline__ uint32_t issue(SpmvCtr* c, int lane) const {
    return lane == 0 && tried < kStripes ? atomicAdd(&c->next[stripe], 1u) : 0u;
  }
  // the group a ticket from issue() stands for, or -1 when every stripe is dry
  __device__ __forceinline__ int64_t resolve(uint32_t ticket, SpmvCtr* c, int lane) {
    int64_t g = -1;
    if (lane == 0) {
      uint32_t t = ticket;
      while (tried < kStripes) {
        const int64_t lo = (int64_t)stripe * per_stripe, hi = min(groups, lo + per_stripe);
        if (lo + (int64_t)t < hi) {
          g = lo + t;
          break;
        }
        stripe = (stripe + 1) % kStripes;
        ++tried;
        if (tried < kStripes) t = atomicAdd(&c->next[stripe], 1u);
      }
    }
    stripe = __shfl_sync(kFull, stripe, 0);
    tried = __shfl_sync(kFull, tried, 0);
    return __shfl_sync(kFull, g, 0);
  }
};

// WARP and GRID levels: warps take row groups on their own.  The group after
// the current one is known and its row bounds are loading while the current
// group is walked, and the ticket for the one after that is in flight.
template <int LEVEL>
__global__ void __launch_bounds__(kThreads) spmv_rows_kernel(Mat A, int32_t threshold, LargeRow* L, ChunkDesc* D,
                                                             SpmvCtr* c) {
  const int lane = threadIdx.x & 31;
  const int gw = blockIdx.x * kWarps + (threadIdx.x >> 5);
  GroupFeed f;
  f.groups = ((int64_t)A.n + 31) / 32;
  f.per_stripe = (f.groups + kStripes - 1) / kStripes;
  f.stripe = gw % kStripes;
  f.tried = 0;
  int64_t g = f.resolve(f.issue(c, lane), c, lane);
  int64_t gn = f.resolve(f.issue(c, lane), c, lane);
  int32_t s = 0, e = 0;
  if (g >= 0 && g * 32 + lane < A.n) row_bounds(A, g * 32 + lane, s, e, c);
  while (g >= 0) {
    const uint32_t ticket = f.issue(c, lane);  // for the group after gn
    int32_t sn = 0, en = 0;
    if (gn >= 0 && gn * 32 + lane < A.n) row_bounds(A, gn * 32 + lane, sn, en, c);
    const bool large = small_rows(A, g, s, e, threshold, lane, c);
    const int32_t deg = e - s;
    if (LEVEL == NPS_LEVEL_WARP) {
      unsigned lm = __ballot_sync(kFull, large);
      while (lm) {
        const int j = __ffs(lm) - 1;
        lm &= lm - 1;
        const int32_t rs = __shfl_sync(kFull, s, j), re = __shfl_sync(kFull, e, j);
        const double t = warp_range<8>(A, rs, re, lane, c);
        if (lane == 0) A.y[g * 32 + j] = t;
      }
    } else {
      // one 64-bit atomic per warp reserves list entries and chunks together, so
      // list order is chunk order
      const uint32_t nch = large ? ((uint32_t)deg + kChunk - 1) / kChunk : 0u;
      const unsigned lm = __ballot_sync(kFull, large);
      if (lm) {
        uint32_t cincl = nch;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t t = __shfl_up_sync(kFull, cincl, o);
          if (lane >= o) cincl += t;
        }
        const uint32_t ctot = __shfl_sync(kFull, cincl, 31);
        const int leader = __ffs(lm) - 1;
        unsigned long long base = 0;
        if (lane == leader) base = atomicAdd(&c->list, ((unsigned long long)__popc(lm) << 32) | ctot);
        base = __shfl_sync(kFull, base, leader);
        const uint32_t slot = (uint32_t)(base >> 32) + __popc(lm & ((1u << lane) - 1));
        const uint32_t cb = (uint32_t)base + (cincl - nch);
        if (large && nch > 1) L[slot] = LargeRow{(int32_t)(g * 32 + lane), cb, nch, 0u};
        // the chunk table, written by the whole warp one large row at a time
        unsigned todo = lm;
        while (todo) {
          const int j = __ffs(todo) - 1;
          todo &= todo - 1;
          const uint32_t js = __shfl_sync(kFull, slot, j), jcb = __shfl_sync(kFull, cb, j);
          const uint32_t jn = __shfl_sync(kFull, nch, j);
          const int32_t rs = __shfl_sync(kFull, s, j), re = __shfl_sync(kFull, e, j);
          for (uint32_t i = lane; i < jn; i += 32) {
            const int64_t cs = (int64_t)rs + (int64_t)i * kChunk;
            D[jcb + i] = ChunkDesc{(int32_t)(g * 32 + j), (int32_t)cs, (int32_t)min((int64_t)re, cs + kChunk),
                                   jn > 1 ? (int32_t)js : -1};
          }
        }
      }
    }
    g = gn;
    s = sn;
    e = en;
    gn = f.resolve(ticket, c, lane);
  }
}

// BLOCK level: CTAs take units of kWarps row groups (one atomic per unit, on
// kStripes striped counters); each CTA lists its large rows in shared memory and
// walks each with all its threads.  The unit loop is the same for every thread
// of the CTA, so its barriers are reached by all.
__global__ void __launch_bounds__(kThreads) spmv_rows_block_kernel(Mat A, int32_t threshold, SpmvCtr* c) {
  __shared__ int32_t s_rows[kThreads];
  __shared__ uint32_t s_count[2];  // per unit parity, like s_unit: reset two units after its last read
  __shared__ double s_part[kWarps];
  __shared__ int64_t s_unit[2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t groups = ((int64_t)A.n + 31) / 32;
  const int64_t units = (groups + kWarps - 1) / kWarps;
  const int64_t per_stripe = (units + kStripes - 1) / kStripes;
  int stripe = blockIdx.x % kStripes, tried = 0;
  for (int it = 0;; ++it) {
    if (threadIdx.x == 0) {
      int64_t u = -1;
      while (tried < kStripes) {
        const int64_t lo = (int64_t)stripe * per_stripe, hi = min(units, lo + per_stripe);
        const int64_t cand = lo + (int64_t)atomicAdd(&c->next[stripe], 1u);
        if (cand < hi) {
          u = cand;
          break;
        }
        stripe = (stripe + 1) % kStripes;
        ++tried;
      }
      s_unit[it & 1] = u;
      s_count[it & 1] = 0;
    }
    __syncthreads();
    const int64_t unit = s_unit[it & 1];  // slot it & 1 is rewritten only after the next barrier
    if (unit < 0) break;
    const int64_t g = unit * kWarps + warp;
    if (g < groups) {  // warp-uniform
      const int64_t r = g * 32 + lane;
      int32_t s = 0, e = 0;
      if (r < A.n) row_bounds(A, r, s, e, c);
      if (small_rows(A, g, s, e, threshold, lane, c)) s_rows[atomicAdd(&s_count[it & 1], 1u)] = (int32_t)r;
    }
    __syncthreads();
    const uint32_t cnt = s_count[it & 1];
    for (uint32_t j = 0; j < cnt; ++j) {
      const int32_t r = s_rows[j];
      int32_t s, e;
      row_bounds(A, r, s, e, c);
      double a0 = 0.0, a1 = 0.0;
      int64_t k = (int64_t)s + threadIdx.x;
      for (; k + kThreads < e; k += 2 * kThreads) {
        const int32_t ca = __ldcs(A.col + k), cb = __ldcs(A.col + k + kThreads);
        const double va = __ldcs(A.val + k), vb = __ldcs(A.val + k + kThreads);
        a0 += va * x_at(A, ca, c);
        a1 += vb * x_at(A, cb, c);
      }
      if (k < e) a0 += __ldcs(A.val + k) * x_at(A, __ldcs(A.col + k), c);
      const double ws = warp_sum(a0 + a1);
      if (lane == 0) s_part[warp] = ws;
      __syncthreads();
      if (threadIdx.x == 0) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) t += s_part[w];
        A.y[r] = t;
      }
      __syncthreads();
    }
  }
}

// Grid level, second pass: one warp per chunk of the listed rows, the next
// chunk's descriptor loading while the current one is walked.  A row of one
// chunk is written at once; for longer rows the warp that finishes the last
// chunk adds the row's chunk sums in chunk order.
__global__ void __launch_bounds__(kThreads, kChunkCtas) spmv_chunks_kernel(Mat A, LargeRow* L, const ChunkDesc* D, double* part,
                                                               SpmvCtr* c) {
  const uint32_t nc = (uint32_t)c->list;
  const int lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * kWarps;
  uint32_t q = blockIdx.x * kWarps + (threadIdx.x >> 5);
  ChunkDesc cd = q < nc ? D[q] : ChunkDesc{0, 0, 0, -1};
  for (; q < nc; q += warps) {
    const ChunkDesc nx = q + warps < nc ? D[q + warps] : ChunkDesc{0, 0, 0, -1};
    const double t = warp_range<kBatch>(A, cd.start, cd.end, lane, c);
    if (lane == 0) {
      if (cd.entry < 0) {
        A.y[cd.row] = t;
      } else {
        const LargeRow lr = L[cd.entry];
        part[q] = t;
        __threadfence();
        if (atomicAdd(&L[cd.entry].done, 1u) == lr.chunks - 1) {  // the row's last chunk
          __threadfence();
          double sum = 0.0;
          for (uint32_t i = 0; i < lr.chunks; ++i) sum += __ldcg(part + lr.chunk_begin + i);
          A.y[lr.row] = sum;
        }
      }
    }
    cd = nx;
  }
}


struct SpmvWork {
  unsigned long long ctx_id = 0;  // context the cached buffers live in (nps_context_id)
  std::mutex mu;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[4] = {};
  int sms = 0;
  SpmvCtr* ctr = nullptr;
  SpmvCtr* h_ctr = nullptr;  // pinned
  LargeRow* list = nullptr;
  size_t list_n = 0;
  double* part = nullptr;
  size_t part_n = 0;
  ChunkDesc* chunks = nullptr;
  size_t chunks_n = 0;
  int32_t* row = nullptr;
  size_t row_n = 0;
  int32_t* col = nullptr;
  size_t col_n = 0;
  double* val = nullptr;
  size_t val_n = 0;
  double* x = nullptr;
  size_t x_n = 0;
  double* y = nullptr;
  size_t y_n = 0;
};

std::mutex g_spmv_mu;
std::vector<SpmvWork*> g_spmv;


nps_status spmv_work(int device, SpmvWork** out) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return nps_fail(NPS_ERR_NO_DEVICE, "no CUDA device");
  }
  if (device < 0 || device >= count) return nps_fail(NPS_ERR_INVALID_ARG, "device ordinal out of range");
  NPS_CUDA_RETURN(cudaSetDevice(device));
  SpmvWork* w;
  {
    std::lock_guard<std::mutex> lk(g_spmv_mu);
    if ((int)g_spmv.size() <= device) g_spmv.resize(device + 1, nullptr);
    {
    const unsigned long long id = nps_context_id(device);
    if (g_spmv[device] && id != 0 && g_spmv[device]->ctx_id != id) g_spmv[device] = nullptr;  // device reset: abandoned
    if (!g_spmv[device]) {
      g_spmv[device] = new SpmvWork();
      g_spmv[device]->ctx_id = id;
    }
  }
    w = g_spmv[device];
  }
  *out = w;
  return NPS_OK;
}

}  // namespace

extern "C" nps_status nps_spmv(const int32_t* row_ptr, const int32_t* col, const double* val, const double* x,
                               double* y, int32_t n, int64_t m, const nps_params* pin, nps_stats* st) {
  nps_clear_error();
  nps_params p;
  if (pin) p = *pin;
  else nps_params_default(&p);
  if (p.level < NPS_LEVEL_WARP || p.level > NPS_LEVEL_GRID) return nps_fail(NPS_ERR_INVALID_ARG, "spmv: level must be 0..2");
  if (p.threshold < 1) return nps_fail(NPS_ERR_INVALID_ARG, "threshold must be >= 1");
  if (n <= 0) return nps_fail(NPS_ERR_INVALID_ARG, "n must be positive");
  if (m < 0 || m >= (int64_t)INT32_MAX) return nps_fail(NPS_ERR_INVALID_ARG, "m must be in [0, 2^31-1)");
  if (!row_ptr || !x || !y || (m > 0 && (!col || !val))) return nps_fail(NPS_ERR_INVALID_ARG, "null array");
  if (!p.device_ptrs && (row_ptr[0] != 0 || row_ptr[n] != (int32_t)m))
    return nps_fail(NPS_ERR_FORMAT, "malformed CSR: row_ptr[0] must be 0 and row_ptr[n] must be m");
  SpmvWork* W = nullptr;
  nps_status e = spmv_work(p.device, &W);
  if (e) return e;
  std::lock_guard<std::mutex> lk(W->mu);
  if (!W->stream) NPS_CUDA_RETURN(cudaStreamCreateWithFlags(&W->stream, cudaStreamNonBlocking));
  if (!W->ev[0])
    for (auto& ev : W->ev) NPS_CUDA_RETURN(cudaEventCreate(&ev));
  if (!W->ctr) NPS_CUDA_RETURN(cudaMalloc((void**)&W->ctr, sizeof(SpmvCtr)));
  if (!W->h_ctr) NPS_CUDA_RETURN(cudaMallocHost((void**)&W->h_ctr, sizeof(SpmvCtr)));
  if (!W->sms) NPS_CUDA_RETURN(cudaDeviceGetAttribute(&W->sms, cudaDevAttrMultiProcessorCount, p.device));
  cudaStream_t s = p.stream ? (cudaStream_t)p.stream : W->stream;
  if (st) memset(st, 0, sizeof(*st));
  NPS_CUDA_RETURN(cudaEventRecord(W->ev[0], s));
  Mat A{row_ptr, col, val, x, y, n, m};
  if (!p.device_ptrs) {
    if ((e = nps_ensure(&W->row, &W->row_n, (size_t)n + 1, s, "spmv")) || (e = nps_ensure(&W->col, &W->col_n, (size_t)m, s, "spmv")) ||
        (e = nps_ensure(&W->val, &W->val_n, (size_t)m, s, "spmv")) || (e = nps_ensure(&W->x, &W->x_n, (size_t)n, s, "spmv")) ||
        (e = nps_ensure(&W->y, &W->y_n, (size_t)n, s, "spmv")))
      return e;
    NPS_CUDA_RETURN(cudaMemcpyAsync(W->row, row_ptr, sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice, s));
    if (m > 0) {
      NPS_CUDA_RETURN(cudaMemcpyAsync(W->col, col, sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice, s));
      NPS_CUDA_RETURN(cudaMemcpyAsync(W->val, val, sizeof(double) * (size_t)m, cudaMemcpyHostToDevice, s));
    }
    NPS_CUDA_RETURN(cudaMemcpyAsync(W->x, x, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, s));
    A = Mat{W->row, W->col, W->val, W->x, W->y, n, m};
  }
  const int grid = (int)std::max<int64_t>(
      1, std::min<int64_t>(((int64_t)n + kThreads - 1) / kThreads, (int64_t)W->sms * (2048 / kThreads)));
  LargeRow* L = nullptr;
  ChunkDesc* D = nullptr;
  if (p.level == NPS_LEVEL_GRID) {
    // large rows <= m / threshold; chunks <= m / kChunk + large rows
    const size_t nl = std::min<size_t>((size_t)n, (size_t)m / (size_t)p.threshold + 1);
    const size_t nc = (size_t)m / kChunk + nl + 1;
    if ((e = nps_ensure(&W->list, &W->list_n, nl, s, "spmv")) || (e = nps_ensure(&W->part, &W->part_n, nc, s, "spmv")) ||
        (e = nps_ensure(&W->chunks, &W->chunks_n, nc, s, "spmv")))
      return e;
    L = W->list;
    D = W->chunks;
  }
  NPS_CUDA_RETURN(cudaMemsetAsync(W->ctr, 0, sizeof(SpmvCtr), s));
  NPS_CUDA_RETURN(cudaEventRecord(W->ev[1], s));
  switch (p.level) {
    case NPS_LEVEL_WARP:
      spmv_rows_kernel<NPS_LEVEL_WARP><<<grid, kThreads, 0, s>>>(A, p.threshold, L, D, W->ctr);
      break;
    case NPS_LEVEL_BLOCK:
      spmv_rows_block_kernel<<<grid, kThreads, 0, s>>>(A, p.threshold, W->ctr);
      break;
    default:
      spmv_rows_kernel<NPS_LEVEL_GRID><<<grid, kThreads, 0, s>>>(A, p.threshold, L, D, W->ctr);
      NPS_CUDA_RETURN(cudaGetLastError());
      spmv_chunks_kernel<<<grid, kThreads, 0, s>>>(A, L, D, W->part, W->ctr);
      break;
  }
  NPS_CUDA_RETURN(cudaGetLastError());
  NPS_CUDA_RETURN(cudaEventRecord(W->ev[2], s));
  if (!p.device_ptrs) NPS_CUDA_RETURN(cudaMemcpyAsync(y, A.y, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, s));
  NPS_CUDA_RETURN(cudaMemcpyAsync(W->h_ctr, W->ctr, sizeof(SpmvCtr), cudaMemcpyDeviceToHost, s));
  NPS_CUDA_RETURN(cudaEventRecord(W->ev[3], s));
  NPS_CUDA_RETURN(cudaStreamSynchronize(s));
  if (st) {
    st->status = (int32_t)W->h_ctr->status;
    st->grid_ctas = grid;
    st->edges_scanned = (uint64_t)m;
    st->vertices_processed = (uint64_t)n;
    st->buckets = (uint32_t)(W->h_ctr->list >> 32);  // grid level: rows consolidated device-wide
    cudaEventElapsedTime(&st->kernel_ms, W->ev[1], W->ev[2]);
    cudaEventElapsedTime(&st->total_ms, W->ev[0], W->ev[3]);
  }
  if (W->h_ctr->status == NPS_ERR_FORMAT)
    return nps_fail(NPS_ERR_FORMAT, "malformed CSR: a row range or column index is out of bounds");
  return NPS_OK;
}
