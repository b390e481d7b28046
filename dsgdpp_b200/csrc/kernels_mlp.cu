// kernels_mlp.cu -- the step-size controller network: 16 -> 64 -> 64 -> 1, GELU.
//
// No reference counterpart: the reference's only adaptive step rule is
// BoldDriver (mf/sgd/decay/decay_bolddriver.h:59-67).  The controller maps 16
// features of the run's recent history to a log step multiplier clipped to
// [-1, 1]; BoldDriver stays the fallback.  Everything is FP32 and tiny (5,313
// parameters), so one CTA of 64 threads handles one sample: thread j owns
// hidden unit j of both layers.  Per-sample gradients are written to a
// [batch][params] buffer and reduced in a fixed order, so training is
// deterministic.
#include "kernels.cuh"

namespace dsgdpp {
namespace {

constexpr int kIn = 16, kHid = 64;
// parameter layout
constexpr int kW1 = 0;                      // [kHid][kIn]
constexpr int kB1 = kW1 + kHid * kIn;       // [kHid]
constexpr int kW2 = kB1 + kHid;             // [kHid][kHid]
constexpr int kB2 = kW2 + kHid * kHid;      // [kHid]
constexpr int kW3 = kB2 + kHid;             // [kHid]
constexpr int kB3 = kW3 + kHid;             // [1]
constexpr int kParams = kB3 + 1;            // 5313

__device__ __forceinline__ float gelu(float x) {
  return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f));
}
// d/dx [x Phi(x)] = Phi(x) + x phi(x)
__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
  return cdf + x * pdf;
}

__device__ __forceinline__ float block_sum64(float v, float* sh) {
  // 64 threads = 2 warps
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(kFullMask, v, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  const float t = sh[0] + sh[1];
  __syncthreads();
  return t;
}

// One CTA (64 threads) per sample.  out[b] = clip(net(x_b), -1, 1).  With
// grads != null, also the gradient of (net(x_b) - y)^2 / batch (unclipped
// output) into grads[b][kParams] and the sample's loss.
__global__ void __launch_bounds__(kHid) mlp_kernel(const float* __restrict__ P, const float* X,
                                                   const float* Y, int batch, float* out,
                                                   float* grads, float* losses) {
  const int b = blockIdx.x, j = threadIdx.x;
  if (b >= batch) return;
  __shared__ float x[kIn], h1[kHid], z1[kHid], dz2[kHid], sh[2];
  if (j < kIn) x[j] = X[(size_t)b * kIn + j];
  __syncthreads();
  float a = P[kB1 + j];
#pragma unroll
  for (int k = 0; k < kIn; ++k) a += P[kW1 + j * kIn + k] * x[k];
  z1[j] = a;
  h1[j] = gelu(a);
  __syncthreads();
  float a2 = P[kB2 + j];
  for (int k = 0; k < kHid; ++k) a2 += P[kW2 + j * kHid + k] * h1[k];
  const float h2 = gelu(a2);
  const float raw = block_sum64(P[kW3 + j] * h2, sh) + P[kB3];
  const float clipped = fminf(1.0f, fmaxf(-1.0f, raw));
  if (j == 0 && out) out[b] = clipped;
  if (!grads) return;
  // the loss is taken on the unclipped output (the clip applies to the
  // proposed multiplier only), so a saturated output still gets a gradient
  const float y = Y[b];
  const float dout = 2.0f * (raw - y) / (float)batch;
  if (j == 0 && losses) losses[b] = (raw - y) * (raw - y) / (float)batch;
  float* g = grads + (size_t)b * kParams;
  g[kW3 + j] = dout * h2;
  if (j == 0) g[kB3] = dout;
  const float d2 = dout * P[kW3 + j] * gelu_grad(a2);
  dz2[j] = d2;
  g[kB2 + j] = d2;
  for (int k = 0; k < kHid; ++k) g[kW2 + j * kHid + k] = d2 * h1[k];
  __syncthreads();
  // thread j now owns unit j of the first layer: dh1[j] = sum_i W2[i][j] dz2[i]
  float dh1 = 0;
  for (int i = 0; i < kHid; ++i) dh1 += P[kW2 + i * kHid + j] * dz2[i];
  const float d1 = dh1 * gelu_grad(z1[j]);
  g[kB1 + j] = d1;
#pragma unroll
  for (int k = 0; k < kIn; ++k) g[kW1 + j * kIn + k] = d1 * x[k];
}

// grad[p] = sum over samples of per-sample grads, in sample order
__global__ void mlp_reduce_kernel(const float* grads, int batch, float* grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kParams) return;
  float s = 0;
  for (int b = 0; b < batch; ++b) s += grads[(size_t)b * kParams + p];
  grad[p] = s;
}

// Adam (Kingma & Ba, ICLR 2015) with bias correction
__global__ void adam_kernel(float* P, const float* g, float* m, float* v, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kParams) return;
  const float gp = g[p];
  const float mp = b1 * m[p] + (1 - b1) * gp;
  const float vp = b2 * v[p] + (1 - b2) * gp * gp;
  m[p] = mp;
  v[p] = vp;
  P[p] -= lr * (mp / c1) / (sqrtf(vp / c2) + eps);
}

}  // namespace

int mlp_param_count() { return kParams; }
int mlp_input_count() { return kIn; }

cudaError_t launch_mlp(const float* P, const float* X, const float* Y, int batch, float* out,
                       float* grads, float* losses, cudaStream_t st) {
  if (batch <= 0) return cudaSuccess;
  mlp_kernel<<<batch, kHid, 0, st>>>(P, X, Y, batch, out, grads, losses);
  return cudaGetLastError();
}

cudaError_t launch_mlp_reduce(const float* grads, int batch, float* grad, cudaStream_t st) {
  mlp_reduce_kernel<<<(kParams + 255) / 256, 256, 0, st>>>(grads, batch, grad);
  return cudaGetLastError();
}

cudaError_t launch_adam(float* P, const float* g, float* m, float* v, float lr, float b1,
                        float b2, float eps, int step, cudaStream_t st) {
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  adam_kernel<<<(kParams + 255) / 256, 256, 0, st>>>(P, g, m, v, lr, b1, b2, eps, c1, c2);
  return cudaGetLastError();
}

}  // namespace dsgdpp
