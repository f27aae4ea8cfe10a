// Training and inference kernels of the SSSP policy network: a 2-layer MLP
// 12 -> 32 (ReLU) -> 14 with bf16 weights and fp32 accumulation.  Outputs are
// 11 logits over the bucket width delta = 2^k (k = 0..10) and 3 logits over the
// consolidation level (warp, block, grid).  The same weights, rounded to bf16,
// run inside the persistent SSSP kernel (policy_eval in nps_device.cuh).
//
// The network has 832 multiply-adds per sample, so these kernels are
// latency-bound one-thread-per-sample loops with the weights staged in shared
// memory; tensor cores would not be fed by a 12x32 layer.
#include <cuda_runtime.h>

#include <string>

#include "nps.h"
#include "nps_internal.h"

namespace {

constexpr int IN = NPS_MLP_IN, HID = NPS_MLP_HID, OUT = NPS_MLP_OUT;
constexpr int ND = 11;  // delta head
constexpr int NL = 3;   // level head
constexpr int TPB = 128;

__device__ __forceinline__ float bf16f(uint16_t b) { return __uint_as_float(((uint32_t)b) << 16); }

__device__ __forceinline__ uint16_t f2bf16(float f) {  // round to nearest even
  uint32_t u = __float_as_uint(f);
  if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)(u >> 16);
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

struct SW {
  float w1[HID * IN];
  float b1[HID];
  float w2[OUT * HID];
  float b2[OUT];
};

__device__ void stage_weights(SW& s, const uint16_t* w1, const float* b1, const uint16_t* w2, const float* b2) {
  for (int i = threadIdx.x; i < HID * IN; i += blockDim.x) s.w1[i] = bf16f(w1[i]);
  for (int i = threadIdx.x; i < OUT * HID; i += blockDim.x) s.w2[i] = bf16f(w2[i]);
  for (int i = threadIdx.x; i < HID; i += blockDim.x) s.b1[i] = b1[i];
  for (int i = threadIdx.x; i < OUT; i += blockDim.x) s.b2[i] = b2[i];
  __syncthreads();
}

__device__ __forceinline__ void forward_one(const SW& s, const float* x, float* h, float* o) {
#pragma unroll 4
  for (int j = 0; j < HID; ++j) {
    float a = s.b1[j];
#pragma unroll
    for (int i = 0; i < IN; ++i) a = fmaf(s.w1[j * IN + i], x[i], a);
    h[j] = a > 0.f ? a : 0.f;
  }
#pragma unroll 2
  for (int k = 0; k < OUT; ++k) {
    float a = s.b2[k];
#pragma unroll
    for (int j = 0; j < HID; ++j) a = fmaf(s.w2[k * HID + j], h[j], a);
    o[k] = a;
  }
}

__global__ void mlp_forward_kernel(const uint16_t* w1, const float* b1, const uint16_t* w2, const float* b2,
                                   const float* X, int B, float* logits) {
  __shared__ SW s;
  stage_weights(s, w1, b1, w2, b2);
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < B; r += gridDim.x * blockDim.x) {
    float x[IN], h[HID], o[OUT];
#pragma unroll
    for (int i = 0; i < IN; ++i) x[i] = X[(size_t)r * IN + i];
    forward_one(s, x, h, o);
#pragma unroll
    for (int k = 0; k < OUT; ++k) logits[(size_t)r * OUT + k] = o[k];
  }
}

// softmax cross-entropy over a head; writes dlogits = wt * (p - onehot) / wsum
__device__ __forceinline__ float ce_head(const float* o, int n, int label, float scale, float* d) {
  float mx = o[0];
  for (int k = 1; k < n; ++k) mx = fmaxf(mx, o[k]);
  float z = 0.f;
  for (int k = 0; k < n; ++k) z += __expf(o[k] - mx);
  const float lz = __logf(z) + mx;
  for (int k = 0; k < n; ++k) d[k] = scale * (__expf(o[k] - lz) - (k == label ? 1.f : 0.f));
  return scale * (lz - o[label]);
}

// Butterfly transpose-sum over a warp: on return lane L holds the sum over all
// 32 lanes of v[L].  31 shuffles for 32 sums (v is overwritten).
__device__ __forceinline__ float transpose_sum32(float (&v)[32], int lane) {
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    const bool hi = (lane & off) != 0;
#pragma unroll
    for (int i = 0; i < off; ++i) {
      const float send = hi ? v[i] : v[i + off];
      const float keep = hi ? v[i + off] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, off);
    }
  }
  return v[0];
}

// Mean weighted cross-entropy of both heads; gradients accumulate (fp32) into
// g_* which the caller zeroes.  Labels < 0 drop that head for the sample.
// One sample per lane.  A warp's 32 per-sample outer products are summed with
// transpose-sums, so lane j ends up owning hidden unit j's gradients (column j
// of w2, row j of w1, b1[j]; lane k < 14 also b2[k]) and adds them to the CTA's
// shared accumulators without contention inside the warp.
static_assert(HID == 32 && OUT <= 32, "one lane per hidden unit");
__global__ void mlp_loss_backward_kernel(const uint16_t* w1, const float* b1, const uint16_t* w2,
                                         const float* b2, const float* X, const int32_t* yd,
                                         const int32_t* yl, const float* wt, int B, float inv_wsum,
                                         float* g_w1, float* g_b1, float* g_w2, float* g_b2, float* loss) {
  __shared__ SW s;
  __shared__ SW g;
  __shared__ float sl;
  stage_weights(s, w1, b1, w2, b2);
  for (int i = threadIdx.x; i < HID * IN; i += blockDim.x) g.w1[i] = 0.f;
  for (int i = threadIdx.x; i < OUT * HID; i += blockDim.x) g.w2[i] = 0.f;
  for (int i = threadIdx.x; i < HID; i += blockDim.x) g.b1[i] = 0.f;
  for (int i = threadIdx.x; i < OUT; i += blockDim.x) g.b2[i] = 0.f;
  if (threadIdx.x == 0) sl = 0.f;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  float my_loss = 0.f;
  // the bound is uniform per warp: every lane takes part in the transpose-sums
  for (int r0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); r0 < B; r0 += gridDim.x * blockDim.x) {
    const int r = r0 + lane;
    const bool act = r < B;
    float x[IN], h[HID], o[OUT], d[OUT];
#pragma unroll
    for (int i = 0; i < IN; ++i) x[i] = act ? X[(size_t)r * IN + i] : 0.f;
    forward_one(s, x, h, o);
#pragma unroll
    for (int k = 0; k < OUT; ++k) d[k] = 0.f;
    if (act) {
      const float sc = (wt ? wt[r] : 1.f) * inv_wsum;
      if (yd[r] >= 0 && yd[r] < ND) my_loss += ce_head(o, ND, yd[r], sc, d);
      if (yl[r] >= 0 && yl[r] < NL) my_loss += ce_head(o + ND, NL, yl[r], sc, d + ND);
    }
    float v[32];
    // b2: lanes 0..OUT-1
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = k < OUT ? d[k] : 0.f;
    const float gb2 = transpose_sum32(v, lane);
    if (lane < OUT && gb2 != 0.f) atomicAdd(&g.b2[lane], gb2);
    // w2[k][j] += d[k] h[j]: lane j owns column j
#pragma unroll 1
    for (int k = 0; k < OUT; ++k) {
#pragma unroll
      for (int j = 0; j < HID; ++j) v[j] = d[k] * h[j];
      const float t = transpose_sum32(v, lane);
      if (t != 0.f) atomicAdd(&g.w2[k * HID + lane], t);
    }
    // back through the ReLU: dh[j] = (h[j] > 0) * sum_k w2[k][j] d[k]
    float dh[HID];
#pragma unroll
    for (int j = 0; j < HID; ++j) {
      float a = 0.f;
#pragma unroll
      for (int k = 0; k < OUT; ++k) a = fmaf(s.w2[k * HID + j], d[k], a);
      dh[j] = h[j] > 0.f ? a : 0.f;
    }
#pragma unroll
    for (int j = 0; j < HID; ++j) v[j] = dh[j];
    const float gb1 = transpose_sum32(v, lane);
    if (gb1 != 0.f) atomicAdd(&g.b1[lane], gb1);
    // w1[j][i] += dh[j] x[i]: lane j owns row j
#pragma unroll 1
    for (int i = 0; i < IN; ++i) {
#pragma unroll
      for (int j = 0; j < HID; ++j) v[j] = dh[j] * x[i];
      const float t = transpose_sum32(v, lane);
      if (t != 0.f) atomicAdd(&g.w1[lane * IN + i], t);
    }
  }
  atomicAdd(&sl, my_loss);
  __syncthreads();
  for (int i = threadIdx.x; i < HID * IN; i += blockDim.x) atomicAdd(&g_w1[i], g.w1[i]);
  for (int i = threadIdx.x; i < OUT * HID; i += blockDim.x) atomicAdd(&g_w2[i], g.w2[i]);
  for (int i = threadIdx.x; i < HID; i += blockDim.x) atomicAdd(&g_b1[i], g.b1[i]);
  for (int i = threadIdx.x; i < OUT; i += blockDim.x) atomicAdd(&g_b2[i], g.b2[i]);
  if (threadIdx.x == 0 && loss) atomicAdd(loss, sl);
}

// Adam (Kingma & Ba 2015) on fp32 master weights; bf16_out (optional) receives
// the rounded copy used by the forward kernels.
__global__ void adam_kernel(float* master, uint16_t* bf16_out, const float* grad, float* m1, float* m2, int count,
                            float lr, float beta1, float beta2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const float gr = grad[i];
    const float a = beta1 * m1[i] + (1.f - beta1) * gr;
    const float b = beta2 * m2[i] + (1.f - beta2) * gr * gr;
    m1[i] = a;
    m2[i] = b;
    const float mhat = a / c1, vhat = b / c2;
    const float w = master[i] - lr * mhat / (sqrtf(vhat) + eps);
    master[i] = w;
    if (bf16_out) bf16_out[i] = f2bf16(w);
  }
}

// Sum of the sample weights (so the loss is a weighted mean).
__global__ void wsum_kernel(const float* wt, int B, float* out) {
  float a = 0.f;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < B; r += gridDim.x * blockDim.x) a += wt[r];
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, a);
}

int blocks_for(int B) {
  int b = (B + TPB - 1) / TPB;
  return b < 1 ? 1 : (b > 1184 ? 1184 : b);
}

}  // namespace

#define NPS_CUDA_LAST(what)                                                                 \
  do {                                                                                      \
    cudaError_t e_ = cudaGetLastError();                                                    \
    if (e_ != cudaSuccess) return nps_fail(NPS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e_)); \
  } while (0)

extern "C" nps_status nps_mlp_forward(const uint16_t* w1, const float* b1, const uint16_t* w2, const float* b2,
                                      const float* X, int32_t B, float* logits, void* stream) {
  nps_clear_error();
  if (!w1 || !b1 || !w2 || !b2 || !X || !logits || B <= 0) return nps_fail(NPS_ERR_INVALID_ARG, "mlp_forward: bad argument");
  mlp_forward_kernel<<<blocks_for(B), TPB, 0, (cudaStream_t)stream>>>(w1, b1, w2, b2, X, B, logits);
  NPS_CUDA_LAST("mlp_forward_kernel");
  return NPS_OK;
}

extern "C" nps_status nps_mlp_loss_backward(const uint16_t* w1, const float* b1, const uint16_t* w2, const float* b2,
                                            const float* X, const int32_t* label_delta, const int32_t* label_level,
                                            const float* wt, int32_t B, float* g_w1, float* g_b1, float* g_w2,
                                            float* g_b2, float* loss, void* stream) {
  nps_clear_error();
  if (!w1 || !b1 || !w2 || !b2 || !X || !label_delta || !label_level || B <= 0 || !g_w1 || !g_b1 || !g_w2 || !g_b2)
    return nps_fail(NPS_ERR_INVALID_ARG, "mlp_loss_backward: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  // weighted mean: the host passes the sample weights; their sum is formed on the device
  float inv = 1.0f / (float)B;
  if (wt) {
    float* d_sum = nullptr;
    if (cudaMallocAsync(&d_sum, sizeof(float), s) != cudaSuccess) return nps_fail(NPS_ERR_OOM, "mlp: wsum buffer");
    cudaMemsetAsync(d_sum, 0, sizeof(float), s);
    wsum_kernel<<<blocks_for(B), TPB, 0, s>>>(wt, B, d_sum);
    float h = 0.f;
    cudaMemcpyAsync(&h, d_sum, sizeof(float), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(d_sum, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) NPS_CUDA_LAST("wsum_kernel");
    inv = h > 0.f ? 1.0f / h : 0.f;
  }
  mlp_loss_backward_kernel<<<blocks_for(B), TPB, 0, s>>>(w1, b1, w2, b2, X, label_delta, label_level, wt, B, inv,
                                                        g_w1, g_b1, g_w2, g_b2, loss);
  NPS_CUDA_LAST("mlp_loss_backward_kernel");
  return NPS_OK;
}

extern "C" nps_status nps_mlp_adam_step(float* master, uint16_t* bf16_out, const float* grad, float* m1, float* m2,
                                        int32_t count, float lr, float beta1, float beta2, float eps, int32_t step,
                                        void* stream) {
  nps_clear_error();
  if (!master || !grad || !m1 || !m2 || count <= 0 || step < 1) return nps_fail(NPS_ERR_INVALID_ARG, "adam: bad argument");
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  adam_kernel<<<blocks_for(count), TPB, 0, (cudaStream_t)stream>>>(master, bf16_out, grad, m1, m2, count, lr, beta1,
                                                                  beta2, eps, c1, c2);
  NPS_CUDA_LAST("adam_kernel");
  return NPS_OK;
}
