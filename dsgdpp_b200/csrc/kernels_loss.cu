// kernels_loss.cu -- FP64 loss reductions of DSGD++ on sm_100a.
//
// Reference: nzsl (mf/loss/nzsl.h:29-52), l2 (mf/loss/l2.h:39-48) and nzl2
// (mf/loss/nzl2.h:29-87), summed over blocks (mf/matrix/op/sum.h:27-30).
// With FP64 factors every term is formed exactly as the reference forms it
// (the inner product summed in z order, no FMA contraction).  With FP32/BF16
// factors a group of lanes shares an entry (coalesced row loads); products of
// floats are exact in FP64 and only the order of the inner product's additions
// differs.  Terms are reduced by a fixed two-level tree (per-CTA partials,
// then one CTA), so every result is deterministic run to run.
#include "kernels.cuh"

namespace dsgdpp {
namespace {

inline uint32_t vec_width_of(int precision) {
  return precision == kFp64 ? 2 : (precision == kFp32 ? 4 : 8);
}

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

// FP32 / BF16 factors: LPN lanes per entry, each lane loading VPL 16-byte
// vectors of the W row and H column, so a row is one coalesced request.  A
// warp takes 32 consecutive entries (one index load per lane), then walks
// them in LPN rounds of 32 / LPN entries, the factor loads of U rounds issued
// before any is used.  Products of two floats are exact in FP64; each lane
// sums its elements in z order and the group adds the lane sums by a fixed
// butterfly.  Entries [begin, end) are dealt to warps warp, warp + nwarps, ...
// 32 at a time; a warp loads its next 32 entries before it sums the current
// ones.  Training loss on 100M entries at rank 32: 2.97 -> 2.30 ms (FP32) and
// 2.21 -> 2.10 ms (BF16) with the entries in flight, then 2.15 and 1.83 ms
// with H built by f32_scaled (99M entries at rank 128: 8.17 -> 6.97 ms FP32,
// 6.81 -> 5.05 ms BF16).
// f * 2^-896 as a double, exactly, built from the float's bits with integer
// operations: the 8-bit exponent field and 23-bit fraction move into the low
// bits of the double's exponent field and the top of its fraction, so an
// exponent field e reads as 2^(e-1023) where the float meant 2^(e-127) --
// for normal and subnormal floats alike.  The conversion unit, which bounds
// the loss kernels (two conversions per product), then converts only W.
__device__ __forceinline__ double f32_scaled(float f) {
  const uint32_t b = __float_as_uint(f);
  const uint32_t hi = ((b >> 3) & 0x0fffffffu) | (b & 0x80000000u);
  return __hiloint2double((int)hi, (int)(b << 29));
}

template <typename T, int LPN, int VPL>
__device__ __forceinline__ double nzsl_lanes(const uint32_t* row, const uint32_t* col,
                                             const float* val, const T* W, const T* H,
                                             uint32_t r, uint32_t rp, uint64_t begin,
                                             uint64_t end, uint64_t warp, uint64_t nwarps) {
  using E = Elem<T>;
  constexpr int VW = E::VW;
  constexpr int NG = 32 / LPN;          // entries per round
  // rounds with loads in flight together (bounded by the registers they hold)
  constexpr int U = VPL == 1 ? (LPN < 4 ? LPN : 4) : (VPL == 2 ? 2 : 1);
  const uint32_t lane = threadIdx.x & 31u, grp = lane / LPN, gl = lane % LPN;
  const uint32_t nvec = rp / VW;
  double acc = 0;
  uint64_t base = begin + warp * 32;
  uint32_t n_row = 0, n_col = 0;
  float n_val = 0;
  if (base + lane < end) {
    n_row = row[base + lane];
    n_col = col[base + lane];
    n_val = val[base + lane];
  }
  for (; base < end; base += nwarps * 32) {
    const uint32_t my_row = n_row, my_col = n_col;
    const float my_val = n_val;
    // the next 32 entries travel while these are summed
    const uint64_t nk = base + nwarps * 32 + lane;
    if (nk < end) {
      n_row = row[nk];
      n_col = col[nk];
      n_val = val[nk];
    }
    const uint32_t nrec = (uint32_t)min((uint64_t)32, end - base);
#pragma unroll 1
    for (uint32_t t0 = 0; t0 < (uint32_t)LPN; t0 += U) {
      uint4 wv[U][VPL], hv[U][VPL];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const uint32_t ri = (t0 + u) * NG + grp;
        const uint32_t rr = __shfl_sync(kFullMask, my_row, ri);
        const uint32_t cc = __shfl_sync(kFullMask, my_col, ri);
        const bool valid = ri < nrec;
#pragma unroll
        for (int v = 0; v < VPL; ++v) {
          const uint32_t vi = v * LPN + gl;
          if (valid && vi < nvec) {
            wv[u][v] = __ldg(reinterpret_cast<const uint4*>(W + (size_t)rr * rp + vi * VW));
            hv[u][v] = __ldg(reinterpret_cast<const uint4*>(H + (size_t)cc * rp + vi * VW));
          } else {
            wv[u][v] = make_uint4(0, 0, 0, 0);
            hv[u][v] = make_uint4(0, 0, 0, 0);
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const uint32_t ri = (t0 + u) * NG + grp;
        double ip = 0;
#pragma unroll
        for (int v = 0; v < VPL; ++v) {
          float wf[VW], hf[VW];
          E::unpack(wv[u][v], wf);
          E::unpack(hv[u][v], hf);
          const uint32_t z0 = (v * LPN + gl) * VW;
          // The product of two floats is exact in FP64, so the fused
          // multiply-add rounds exactly like the separate add.  The sum is
          // formed with H scaled by 2^-896 and scaled back once: a power of
          // two, so it rounds exactly as unscaled wherever the scaled terms
          // stay normal doubles (magnitudes of 2^-126 and up; below that the
          // absolute error stays under 2^-178).
          if (z0 + VW <= r) {
#pragma unroll
            for (int e = 0; e < VW; ++e) ip = fma((double)wf[e], f32_scaled(hf[e]), ip);
          } else {
#pragma unroll
            for (int e = 0; e < VW; ++e)
              if (z0 + e < r) ip = fma((double)wf[e], f32_scaled(hf[e]), ip);
          }
        }
        ip = __dmul_rn(ip, 0x1p896);
#pragma unroll
        for (int off = LPN / 2; off > 0; off >>= 1)
          ip = __dadd_rn(ip, __shfl_xor_sync(kFullMask, ip, off));
        const float x = __shfl_sync(kFullMask, my_val, ri);
        if (ri < nrec && gl == 0) {
          const double diff = __dsub_rn((double)x, ip);
          acc = __dadd_rn(acc, __dmul_rn(diff, diff));
        }
      }
    }
  }
  return acc;
}

template <typename T, int LPN, int VPL>
__global__ void __launch_bounds__(256, 3)
    nzsl_lanes_kernel(const uint32_t* row, const uint32_t* col, const float* val, uint64_t nnz,
                      const T* W, const T* H, uint32_t r, uint32_t rp, double* partials) {
  __shared__ double sh[32];
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  const uint64_t warp = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const double acc = nzsl_lanes<T, LPN, VPL>(row, col, val, W, H, r, rp, 0, nnz, warp, warps);
  const double t = block_reduce(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

// FP64 factors: one thread per entry, the inner product in z order (as the
// reference forms it) over entries [begin, end) dealt by `stride`.
__device__ __forceinline__ double nzsl_exact(const uint32_t* row, const uint32_t* col,
                                             const double* val, const double* W, const double* H,
                                             uint32_t r, uint32_t rp, uint64_t first,
                                             uint64_t end, uint64_t stride) {
  double acc = 0;
  for (uint64_t k = first; k < end; k += stride) {
    const double* w = W + (size_t)row[k] * rp;
    const double* h = H + (size_t)col[k] * rp;
    double ip = 0;
    for (uint32_t z = 0; z < r; ++z) ip = __dadd_rn(ip, __dmul_rn(w[z], h[z]));
    const double diff = __dsub_rn(val[k], ip);
    acc = __dadd_rn(acc, __dmul_rn(diff, diff));
  }
  return acc;
}

// ---- per-problem (segmented) reductions of the batched form ----------------------
// One CTA per chunk of a problem's range; owner_sums then adds each problem's
// chunk partials in chunk order, so every per-problem sum is deterministic.
template <typename T, int LPN, int VPL>
__global__ void __launch_bounds__(256, 3) nzsl_chunks_kernel(const RangeChunk* chunks,
                                                          const uint32_t* row, const uint32_t* col,
                                                          const float* val, const T* W,
                                                          const T* H, uint32_t r, uint32_t rp,
                                                          double* partials) {
  __shared__ double sh[32];
  const RangeChunk c = chunks[blockIdx.x];
  const double acc = nzsl_lanes<T, LPN, VPL>(row, col, val, W, H, r, rp, c.begin, c.end,
                                             threadIdx.x >> 5, blockDim.x >> 5);
  const double t = block_reduce(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
}
__global__ void __launch_bounds__(256) nzsl_chunks_exact_kernel(
    const RangeChunk* chunks, const uint32_t* row, const uint32_t* col, const double* val,
    const double* W, const double* H, uint32_t r, uint32_t rp, double* partials) {
  __shared__ double sh[32];
  const RangeChunk c = chunks[blockIdx.x];
  const double acc =
      nzsl_exact(row, col, val, W, H, r, rp, c.begin + threadIdx.x, c.end, blockDim.x);
  const double t = block_reduce(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
}
template <typename T>
__global__ void __launch_bounds__(256) sumsq_chunks_kernel(const RangeChunk* chunks, const T* X,
                                                           double* partials) {
  __shared__ double sh[32];
  const RangeChunk c = chunks[blockIdx.x];
  double acc = 0;
  for (uint64_t k = c.begin + threadIdx.x; k < c.end; k += blockDim.x) {
    const double v = (double)(float)X[k];
    acc = __dadd_rn(acc, __dmul_rn(v, v));
  }
  const double t = block_reduce(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
}
template <>
__global__ void __launch_bounds__(256) sumsq_chunks_kernel<double>(const RangeChunk* chunks,
                                                                   const double* X,
                                                                   double* partials) {
  __shared__ double sh[32];
  const RangeChunk c = chunks[blockIdx.x];
  double acc = 0;
  for (uint64_t k = c.begin + threadIdx.x; k < c.end; k += blockDim.x)
    acc = __dadd_rn(acc, __dmul_rn(X[k], X[k]));
  const double t = block_reduce(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
}
__global__ void __launch_bounds__(256) owner_sums_kernel(const double* partials,
                                                         const uint32_t* owner_begin,
                                                         double* out) {
  __shared__ double sh[32];
  const uint32_t p = blockIdx.x;
  double acc = 0;
  for (uint32_t k = owner_begin[p] + threadIdx.x; k < owner_begin[p + 1]; k += blockDim.x)
    acc = __dadd_rn(acc, partials[k]);
  const double t = block_reduce(acc, sh);
  if (threadIdx.x == 0) out[p] = t;
}

// lane mapping of the FP32 / BF16 loss kernels: LPN = the power of two
// covering the row's vectors (at most 32), VPL = vectors per lane
struct LossShape {
  uint32_t lanes, vecs;
};
LossShape loss_shape(uint32_t nvec) {
  // rows of up to 4 vectors: one vector per lane; longer rows: 4 vectors per
  // lane, so fewer lanes share an entry and the butterfly is shorter (measured
  // faster at rank 32 FP32 and rank 128, slower at rank 32 BF16)
  LossShape s{2, 1};
  s.vecs = nvec > 4 ? 4 : 1;
  while (s.lanes * s.vecs < nvec && s.lanes < 32) s.lanes <<= 1;
  s.vecs = (nvec + s.lanes - 1) / s.lanes;
  if (s.vecs == 3) s.vecs = 4;
  return s;
}

template <typename T>
void* nzsl_lanes_fn(LossShape s, bool chunks) {
#define DSGDPP_CASE(L, V)                                                            \
  if (s.lanes == L && s.vecs == V)                                                   \
    return chunks ? reinterpret_cast<void*>(&nzsl_chunks_kernel<T, L, V>)            \
                  : reinterpret_cast<void*>(&nzsl_lanes_kernel<T, L, V>);
  DSGDPP_CASE(2, 1) DSGDPP_CASE(4, 1) DSGDPP_CASE(2, 4) DSGDPP_CASE(4, 4)
  DSGDPP_CASE(8, 4) DSGDPP_CASE(16, 4) DSGDPP_CASE(32, 4)
#undef DSGDPP_CASE
  return nullptr;
}

void* nzsl_fn(int precision, uint32_t rp, bool chunks) {
  const LossShape s = loss_shape(rp / vec_width_of(precision));
  return precision == kFp32 ? nzsl_lanes_fn<float>(s, chunks)
                            : nzsl_lanes_fn<__nv_bfloat16>(s, chunks);
}

// Squares of the elements of one 16-byte vector, added in element order.
// The square of a float is exact in FP64, so the fused multiply-add rounds as
// the separate add does; FP64 elements keep the separate multiply and add.
template <typename T>
__device__ __forceinline__ double add_squares(double acc, const uint4& v) {
  typename Elem<T>::C f[Elem<T>::VW];
  Elem<T>::unpack(v, f);
#pragma unroll
  for (int e = 0; e < Elem<T>::VW; ++e) {
    if constexpr (sizeof(T) == 8) {
      acc = __dadd_rn(acc, __dmul_rn(f[e], f[e]));
    } else {
      const double x = (double)f[e];
      acc = fma(x, x, acc);
    }
  }
  return acc;
}

// Sum of squares of `count` factor entries (L2Loss, mf/loss/l2.h) in FP64:
// 16-byte vector loads dealt grid-stride to the threads, four vectors in
// flight per thread; the elements past the last whole vector (none when rows
// are padded to a vector) go to the first threads.
template <typename T>
__global__ void __launch_bounds__(256) sumsq_partials_kernel(const T* X, uint64_t count,
                                                             double* partials) {
  __shared__ double sh[32];
  constexpr int VW = Elem<T>::VW;
  const uint4* V = reinterpret_cast<const uint4*>(X);
  const uint64_t nvec = count / VW;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  double acc = 0;
  uint64_t k = tid;
  for (; k + 3 * stride < nvec; k += 4 * stride) {
    uint4 v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) v[u] = __ldcs(V + k + u * stride);
#pragma unroll
    for (int u = 0; u < 4; ++u) acc = add_squares<T>(acc, v[u]);
  }
  for (; k < nvec; k += stride) acc = add_squares<T>(acc, __ldcs(V + k));
  for (uint64_t j = nvec * VW + tid; j < count; j += stride) {
    const double x = (double)(typename Elem<T>::C)X[j];
    acc = __dadd_rn(acc, __dmul_rn(x, x));
  }
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
  if (precision == kFp64) {
    nzsl_partials_kernel<double, double><<<grid, 256, 0, st>>>(
        row, col, (const double*)val, nnz, (const double*)W, (const double*)H, r, rp, partials);
    return cudaGetLastError();
  }
  void* fn = nzsl_fn(precision, rp, false);
  if (!fn) return cudaErrorInvalidValue;
  const float* v = static_cast<const float*>(val);
  void* params[] = {&row, &col, &v, &nnz, &W, &H, &r, &rp, &partials};
  return cudaLaunchKernel(fn, dim3(grid), dim3(256), params, 0, st);
}

int nzsl_ctas_per_sm(int precision, uint32_t rp) {
  void* fn = precision == kFp64 ? reinterpret_cast<void*>(&nzsl_partials_kernel<double, double>)
                                : nzsl_fn(precision, rp, false);
  int n = 0;
  if (!fn || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, 256, 0) != cudaSuccess) return 0;
  return n;
}

cudaError_t launch_nzsl_chunks(int precision, const RangeChunk* chunks, uint32_t nchunks,
                               const uint32_t* row, const uint32_t* col, const void* val,
                               const void* W, const void* H, uint32_t r, uint32_t rp,
                               double* partials, cudaStream_t st) {
  if (nchunks == 0) return cudaSuccess;
  if (precision == kFp64) {
    nzsl_chunks_exact_kernel<<<nchunks, 256, 0, st>>>(chunks, row, col, (const double*)val,
                                                      (const double*)W, (const double*)H, r, rp,
                                                      partials);
    return cudaGetLastError();
  }
  void* fn = nzsl_fn(precision, rp, true);
  if (!fn) return cudaErrorInvalidValue;
  const float* v = static_cast<const float*>(val);
  void* params[] = {&chunks, &row, &col, &v, &W, &H, &r, &rp, &partials};
  return cudaLaunchKernel(fn, dim3(nchunks), dim3(256), params, 0, st);
}

cudaError_t launch_sumsq_chunks(int precision, const RangeChunk* chunks, uint32_t nchunks,
                                const void* X, double* partials, cudaStream_t st) {
  if (nchunks == 0) return cudaSuccess;
  if (precision == kFp64)
    sumsq_chunks_kernel<double><<<nchunks, 256, 0, st>>>(chunks, (const double*)X, partials);
  else if (precision == kFp32)
    sumsq_chunks_kernel<float><<<nchunks, 256, 0, st>>>(chunks, (const float*)X, partials);
  else
    sumsq_chunks_kernel<__nv_bfloat16><<<nchunks, 256, 0, st>>>(
        chunks, (const __nv_bfloat16*)X, partials);
  return cudaGetLastError();
}

cudaError_t launch_owner_sums(const double* partials, const uint32_t* owner_begin,
                              uint32_t owners, double* out, cudaStream_t st) {
  if (owners == 0) return cudaSuccess;
  owner_sums_kernel<<<owners, 256, 0, st>>>(partials, owner_begin, out);
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
