// kernels_loss.cu -- FP64 loss reductions of DSGD++ on sm_100a.
//
// Reference: nzsl (mf/loss/nzsl.h:29-52), l2 (mf/loss/l2.h:39-48) and nzl2
// (mf/loss/nzl2.h:29-87), summed over blocks (mf/matrix/op/sum.h:27-30).
// Every term is formed exactly as the reference forms it (the inner product
// summed in z order in FP64, no FMA contraction); the terms are then reduced
// by a fixed two-level tree (per-CTA partials, then one CTA), so the result is
// deterministic run to run and within a few ulps of any summation order.
#include "kernels.cuh"

namespace dsgdpp {
namespace {

__device__ __forceinline__ double block_reduce(double v, double* sh) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(kFullMask, v, off);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double t = 0;
  if (warp == 0) {
    t = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(kFullMask, t, off);
  }
  return t;  // valid in thread 0
}

template <typename T, typename V>
__global__ void __launch_bounds__(256) nzsl_partials_kernel(const uint32_t* row, const uint32_t* col,
                                                            const V* val, uint64_t nnz, const T* W,
                                                            const T* H, uint32_t r, uint32_t rp,
                                                            double* partials) {
  using E = Elem<T>;
  constexpr int VW = E::VW;
  __shared__ double sh[32];
  double acc = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nnz; k += stride) {
    const T* w = W + (size_t)row[k] * rp;
    const T* h = H + (size_t)col[k] * rp;
    double ip = 0;
    for (uint32_t z0 = 0; z0 < r; z0 += VW) {
      typename E::C wf[VW], hf[VW];
      E::unpack(*reinterpret_cast<const uint4*>(w + z0), wf);
      E::unpack(*reinterpret_cast<const uint4*>(h + z0), hf);
#pragma unroll
      for (int e = 0; e < VW; ++e)
        if (z0 + e < r) ip = __dadd_rn(ip, __dmul_rn((double)wf[e], (double)hf[e]));
    }
    const double diff = __dsub_rn((double)val[k], ip);
    acc = __dadd_rn(acc, __dmul_rn(diff, diff));
  }
  const double t = block_reduce(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

template <typename T>
__global__ void __launch_bounds__(256) sumsq_partials_kernel(const T* X, uint64_t count,
                                                             double* partials) {
  __shared__ double sh[32];
  double acc = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < count; k += stride) {
    const double v = (double)(float)X[k];
    acc = __dadd_rn(acc, __dmul_rn(v, v));
  }
  const double t = block_reduce(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
}
template <>
__global__ void __launch_bounds__(256) sumsq_partials_kernel<double>(const double* X,
                                                                     uint64_t count,
                                                                     double* partials) {
  __shared__ double sh[32];
  double acc = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < count; k += stride)
    acc = __dadd_rn(acc, __dmul_rn(X[k], X[k]));
  const double t = block_reduce(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

template <typename T>
__device__ __forceinline__ double as_double(T v) { return (double)(float)v; }
template <>
__device__ __forceinline__ double as_double<double>(double v) { return v; }

template <typename T>
__global__ void __launch_bounds__(256) nzl2_partials_kernel(const T* X, uint64_t rows, uint32_t rp,
                                                            const uint32_t* cnt,
                                                            double* partials) {
  __shared__ double sh[32];
  double acc = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < rows; i += stride) {
    double v = 0;
    for (uint32_t z = 0; z < rp; ++z) {
      const double e = as_double(X[i * rp + z]);
      v = __dadd_rn(v, __dmul_rn(e, e));
    }
    acc = __dadd_rn(acc, __dmul_rn((double)cnt[i], v));
  }
  const double t = block_reduce(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

__global__ void __launch_bounds__(1024) sum_partials_kernel(const double* partials, uint32_t count,
                                                            double* out) {
  __shared__ double sh[32];
  double acc = 0;
  for (uint32_t k = threadIdx.x; k < count; k += blockDim.x) acc = __dadd_rn(acc, partials[k]);
  const double t = block_reduce(acc, sh);
  if (threadIdx.x == 0) out[0] = t;
}

}  // namespace

cudaError_t launch_nzsl_partials(int precision, const uint32_t* row, const uint32_t* col,
                                 const void* val, uint64_t nnz, const void* W, const void* H,
                                 uint32_t r, uint32_t rp, double* partials, uint32_t grid,
                                 cudaStream_t st) {
  if (precision == kFp64)
    nzsl_partials_kernel<double, double><<<grid, 256, 0, st>>>(
        row, col, (const double*)val, nnz, (const double*)W, (const double*)H, r, rp, partials);
  else if (precision == kFp32)
    nzsl_partials_kernel<float, float><<<grid, 256, 0, st>>>(
        row, col, (const float*)val, nnz, (const float*)W, (const float*)H, r, rp, partials);
  else
    nzsl_partials_kernel<__nv_bfloat16, float><<<grid, 256, 0, st>>>(
        row, col, (const float*)val, nnz, (const __nv_bfloat16*)W, (const __nv_bfloat16*)H, r,
        rp, partials);
  return cudaGetLastError();
}

cudaError_t launch_sumsq_partials(int precision, const void* X, uint64_t count,
                                  double* partials, uint32_t grid, cudaStream_t st) {
  if (precision == kFp64)
    sumsq_partials_kernel<double><<<grid, 256, 0, st>>>((const double*)X, count, partials);
  else if (precision == kFp32)
    sumsq_partials_kernel<float><<<grid, 256, 0, st>>>((const float*)X, count, partials);
  else
    sumsq_partials_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>((const __nv_bfloat16*)X, count,
                                                               partials);
  return cudaGetLastError();
}

cudaError_t launch_nzl2_partials(int precision, const void* X, uint64_t rows, uint32_t rp,
                                 const uint32_t* cnt, double* partials, uint32_t grid,
                                 cudaStream_t st) {
  if (precision == kFp64)
    nzl2_partials_kernel<double><<<grid, 256, 0, st>>>((const double*)X, rows, rp, cnt, partials);
  else if (precision == kFp32)
    nzl2_partials_kernel<float><<<grid, 256, 0, st>>>((const float*)X, rows, rp, cnt, partials);
  else
    nzl2_partials_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>((const __nv_bfloat16*)X, rows, rp,
                                                              cnt, partials);
  return cudaGetLastError();
}

cudaError_t launch_sum_partials(const double* partials, uint32_t count, double* out,
                                cudaStream_t st) {
  sum_partials_kernel<<<1, 1024, 0, st>>>(partials, count, out);
  return cudaGetLastError();
}

}  // namespace dsgdpp

// ---- factor-update norms (controller features) -------------------------------------
namespace dsgdpp {
namespace {

// Per row: the Euclidean norm of (X - Xold) over the rp entries; per CTA the sum
// and the maximum of those norms go to partials[blockIdx.x] and
// partials[gridDim.x + blockIdx.x].
template <typename T>
__global__ void __launch_bounds__(256) update_norm_partials_kernel(const T* X, const T* Xold,
                                                                   uint64_t rows, uint32_t rp,
                                                                   double* partials) {
  __shared__ double sh[32];
  __shared__ double shm[32];
  double sum = 0, mx = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < rows; i += stride) {
    double s = 0;
    for (uint32_t z = 0; z < rp; ++z) {
      const double dlt = as_double(X[i * rp + z]) - as_double(Xold[i * rp + z]);
      s += dlt * dlt;
    }
    const double nrm = sqrt(s);
    sum += nrm;
    mx = fmax(mx, nrm);
  }
  const double t = block_reduce(sum, sh);
  // block max
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(kFullMask, mx, off));
  if ((threadIdx.x & 31) == 0) shm[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m2 = 0;
    for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) m2 = fmax(m2, shm[w]);
    partials[blockIdx.x] = t;
    partials[gridDim.x + blockIdx.x] = m2;
  }
}

__global__ void max_partials_kernel(const double* partials, uint32_t count, double* out) {
  __shared__ double sh[32];
  double mx = 0;
  for (uint32_t k = threadIdx.x; k < count; k += blockDim.x) mx = fmax(mx, partials[k]);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(kFullMask, mx, off));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m2 = 0;
    for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) m2 = fmax(m2, sh[w]);
    out[0] = m2;
  }
}

}  // namespace

cudaError_t launch_update_norms(int precision, const void* X, const void* Xold, uint64_t rows,
                                uint32_t rp, double* partials, uint32_t grid, double* out2,
                                cudaStream_t st) {
  if (precision == kFp64)
    update_norm_partials_kernel<double><<<grid, 256, 0, st>>>((const double*)X, (const double*)Xold,
                                                              rows, rp, partials);
  else if (precision == kFp32)
    update_norm_partials_kernel<float><<<grid, 256, 0, st>>>((const float*)X, (const float*)Xold,
                                                             rows, rp, partials);
  else
    update_norm_partials_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>(
        (const __nv_bfloat16*)X, (const __nv_bfloat16*)Xold, rows, rp, partials);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = launch_sum_partials(partials, grid, out2, st);
  if (e != cudaSuccess) return e;
  max_partials_kernel<<<1, 1024, 0, st>>>(partials + grid, grid, out2 + 1);
  return cudaGetLastError();
}

}  // namespace dsgdpp
