// kernels_data.cu -- blocking of the input matrices and factor conversion.
//
// Reference: ReadMatrixBlocksMm (mf/matrix/io/read_impl.h:364-486) routes
// every entry to its block of the d x 2d grid and stores block-local
// coordinates; coordinate_matrix::sort (read_impl.h:162-164) orders each block
// by (i, j) and sums duplicate entries.  Here the entries arrive as one
// global COO array and are blocked on the GPU: a 64-bit key
// (block, local row, local column) -- for the Hogwild training records
// (block, position in the in-block layout), a permutation of the same
// positions -- is radix-sorted stably, runs of equal keys are merged, and
// block boundaries are found by binary search.
#include <algorithm>

#include "kernels.cuh"

namespace dsgdpp {
namespace {

__device__ __forceinline__ uint32_t find_block(const uint64_t* off, uint32_t nb, uint64_t x) {
  uint32_t lo = 0, hi = nb - 1;
  while (lo < hi) {
    uint32_t mid = (lo + hi + 1) >> 1;
    if (off[mid] <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// A keyed permutation of [0, 2^b): xor with the key, then three rounds of a
// multiply by an odd constant and a xor-shift by half the width, all modulo
// 2^b -- each step is invertible on b-bit values, so distinct positions keep
// distinct images.
__device__ __forceinline__ uint64_t permute_bits(uint64_t x, int b, uint64_t key) {
  if (b == 0) return 0;
  const uint64_t mask = b >= 64 ? ~0ull : (1ull << b) - 1;
  const int s = (b + 1) / 2;
  x = (x ^ key) & mask;
  x = (x * 0x9E3779B97F4A7C15ull) & mask;
  x ^= x >> s;
  x = (x * ((key >> 1) | 1ull)) & mask;
  x ^= x >> s;
  x = (x * 0xBF58476D1CE4E5B9ull) & mask;
  x ^= x >> s;
  return x;
}

__global__ void make_keys_kernel(BlockingGeom g, const uint32_t* rows, const uint32_t* cols,
                                 uint64_t nnz, uint64_t* keys, uint32_t* idx,
                                 unsigned long long* bad) {
  extern __shared__ uint64_t offs[];
  uint64_t* o1 = offs;
  uint64_t* o2 = offs + g.nb1 + 1;
  for (uint32_t k = threadIdx.x; k <= g.nb1; k += blockDim.x) o1[k] = g.off1[k];
  for (uint32_t k = threadIdx.x; k <= g.nb2; k += blockDim.x) o2[k] = g.off2[k];
  __syncthreads();
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nnz; k += stride) {
    const uint64_t i = rows[k], j = cols[k];
    if (i >= g.m || j >= g.n) {
      atomicAdd(bad, 1ull);
      keys[k] = ~0ull;
      idx[k] = (uint32_t)k;
      continue;
    }
    const uint32_t b1 = find_block(o1, g.nb1, i), b2 = find_block(o2, g.nb2, j);
    const uint64_t blk = (uint64_t)b1 * g.nb2 + b2;
    const uint64_t li = i - o1[b1], lj = j - o2[b2];
    uint64_t pos;
    if (g.layout == kLayoutColRuns)  // a column's records together, its rows permuted
      pos = lj << g.pbits | permute_bits(li, g.pbits, mix64(g.seed ^ (j * 0xD6E8FEB86659FD93ull)));
    else if (g.layout == kLayoutRowRuns)
      pos = li << g.pbits | permute_bits(lj, g.pbits, mix64(g.seed ^ (i * 0xD6E8FEB86659FD93ull)));
    else if (g.layout == kLayoutShuffled)
      pos = permute_bits(li * g.nB + lj, g.pbits, mix64(g.seed));
    else
      pos = li * g.nB + lj;
    keys[k] = blk * g.stride + pos;
    idx[k] = (uint32_t)k;
  }
}

__global__ void head_flags_kernel(const uint64_t* keys, uint64_t nnz, uint32_t* flags) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nnz; k += stride)
    flags[k] = (k == 0 || keys[k] != keys[k - 1]) ? 1u : 0u;
}

// Runs of equal keys in the sorted order -> one record each, in run order:
// its key, its coordinates and the sorted position where the run starts (the
// values are summed later, once they have arrived: gather_values_kernel).
__global__ void merge_keys_kernel(const uint64_t* keys, const uint32_t* idx, const uint32_t* pos,
                                  uint64_t nnz, const uint32_t* rows_in, const uint32_t* cols_in,
                                  uint64_t* ukeys, uint32_t* urow, uint32_t* ucol,
                                  uint32_t* head_at) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nnz; k += stride) {
    if (!(k == 0 || keys[k] != keys[k - 1])) continue;
    const uint64_t o = pos[k];
    ukeys[o] = keys[k];
    urow[o] = rows_in[idx[k]];
    ucol[o] = cols_in[idx[k]];
    head_at[o] = (uint32_t)k;
  }
}

__global__ void block_ptr_kernel(const uint64_t* ukeys, uint64_t u, uint64_t span,
                                 uint32_t nblocks, uint64_t* ptr) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b > nblocks) return;
  if (b == nblocks) { ptr[b] = u; return; }
  const uint64_t target = (uint64_t)b * span;
  uint64_t lo = 0, hi = u;  // first key >= target
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (ukeys[mid] < target) lo = mid + 1; else hi = mid;
  }
  ptr[b] = lo;
}

// 32 low bits of the key: a hash of the record (shuffled), or the local
// column / row in the high `side_bits` bits above 32 - side_bits hash bits
__global__ void shuffle_keys_kernel(const uint64_t* ukeys, uint64_t u, uint64_t span, uint64_t nB,
                                    int mode, int side_bits, uint64_t seed, uint64_t* keys2,
                                    uint32_t* idx2) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < u; k += stride) {
    const uint64_t blk = ukeys[k] / span, local = ukeys[k] % span;
    const uint32_t hash = (uint32_t)(mix64(seed ^ (k * 0xD6E8FEB86659FD93ull)) >> 32);
    uint32_t low = hash;
    if (mode != kLayoutShuffled) {
      const uint64_t side = mode == kLayoutColRuns ? local % nB : local / nB;
      low = side_bits >= 32 ? (uint32_t)side
                            : (uint32_t)(side << (32 - side_bits)) | (hash >> side_bits);
    }
    keys2[k] = (blk << 32) | low;
    idx2[k] = (uint32_t)k;
  }
}

// Record k of the final order is merged record perm[k] (k without perm).
__global__ void gather_coords_kernel(const uint32_t* perm, uint64_t u, const uint32_t* urow,
                                     const uint32_t* ucol, uint32_t* row, uint32_t* col) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < u; k += stride) {
    const uint32_t q = perm ? perm[k] : (uint32_t)k;
    row[k] = urow[q];
    col[k] = ucol[q];
  }
}

// The value of record k: the sum of its run's values in sorted (stable, so
// input) order, as ReadMatrixBlocksMm's coordinate sort sums duplicates.
__global__ void gather_values_kernel(const uint32_t* perm, uint64_t u, const uint32_t* head_at,
                                     const uint64_t* keys, const uint32_t* idx, uint64_t nnz,
                                     const double* vals_in, void* val, int val_is_double) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < u; k += stride) {
    const uint32_t q = perm ? perm[k] : (uint32_t)k;
    const uint64_t s = head_at[q];
    double v = vals_in[idx[s]];
    for (uint64_t t = s + 1; t < nnz && keys[t] == keys[s]; ++t) v += vals_in[idx[t]];
    if (val_is_double) reinterpret_cast<double*>(val)[k] = v;
    else reinterpret_cast<float*>(val)[k] = (float)v;
  }
}

__global__ void offset_copy_kernel(const uint32_t* rows_in, const uint32_t* cols_in, uint64_t nnz,
                                   uint32_t row0, uint32_t col0, uint32_t* rows_out,
                                   uint32_t* cols_out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nnz; k += stride) {
    rows_out[k] = rows_in[k] + row0;
    cols_out[k] = cols_in[k] + col0;
  }
}

// Block-local coordinates of blocks stored one after another (block b holds
// entries [start[b], start[b+1])) -> global ones; entries outside their block
// are counted in *bad and left as they are.
__global__ void shift_blocks_kernel(const uint64_t* start, uint32_t nblocks, uint32_t nb2,
                                    const uint64_t* off1, const uint64_t* off2, uint64_t nnz,
                                    uint32_t* rows, uint32_t* cols, unsigned long long* bad) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nnz; k += stride) {
    const uint32_t b = find_block(start, nblocks, k);
    const uint32_t b1 = b / nb2, b2 = b - b1 * nb2;
    const uint64_t i = rows[k], j = cols[k];
    if (i >= off1[b1 + 1] - off1[b1] || j >= off2[b2 + 1] - off2[b2]) {
      atomicAdd(bad, 1ull);
      continue;
    }
    rows[k] = (uint32_t)(i + off1[b1]);
    cols[k] = (uint32_t)(j + off2[b2]);
  }
}

__global__ void counts_to_u32_kernel(const uint64_t* in, uint64_t len, uint32_t* out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < len; k += stride)
    out[k] = (uint32_t)in[k];
}

__global__ void count_nnz12_kernel(const uint32_t* row, const uint32_t* col, uint64_t nnz,
                                   uint32_t* cnt1, uint32_t* cnt2) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nnz; k += stride) {
    atomicAdd(cnt1 + row[k], 1u);
    atomicAdd(cnt2 + col[k], 1u);
  }
}

__global__ void inverse_counts_kernel(const uint32_t* cnt, uint64_t len, void* inv, int as_double) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < len; k += stride) {
    const uint32_t c = cnt[k];
    if (as_double) reinterpret_cast<double*>(inv)[k] = c ? 1.0 / (double)c : 0.0;
    else reinterpret_cast<float*>(inv)[k] = c ? 1.0f / (float)c : 0.0f;
  }
}

template <typename T>
__device__ __forceinline__ T from_double(double x);
template <> __device__ __forceinline__ double from_double<double>(double x) { return x; }
template <> __device__ __forceinline__ float from_double<float>(double x) { return (float)x; }
template <> __device__ __forceinline__ __nv_bfloat16 from_double<__nv_bfloat16>(double x) {
  return __double2bfloat16(x);
}
template <typename T>
__device__ __forceinline__ double to_double(T x) { return (double)(float)x; }
template <> __device__ __forceinline__ double to_double<double>(double x) { return x; }

template <typename T>
__global__ void factor_to_device_kernel(const double* src, uint64_t rows, uint32_t r,
                                        uint32_t rp, T* dst) {
  const uint64_t total = rows * rp, stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < total; q += stride) {
    const uint64_t i = q / rp;
    const uint32_t z = (uint32_t)(q % rp);
    dst[q] = z < r ? from_double<T>(src[i * r + z]) : from_double<T>(0.0);
  }
}

template <typename T>
__global__ void factor_to_host_kernel(const T* src, uint64_t rows, uint32_t r, uint32_t rp,
                                      double* dst) {
  const uint64_t total = rows * r, stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < total; q += stride) {
    const uint64_t i = q / r;
    const uint32_t z = (uint32_t)(q % r);
    dst[q] = to_double<T>(src[i * rp + z]);
  }
}

constexpr uint32_t kGrid = 1184;  // 148 SMs x 8

}  // namespace

cudaError_t launch_make_keys(const BlockingGeom& g, const uint32_t* rows, const uint32_t* cols,
                             uint64_t nnz, uint64_t* keys, uint32_t* idx,
                             unsigned long long* bad, cudaStream_t st) {
  if (nnz == 0) return cudaSuccess;
  const size_t sm = sizeof(uint64_t) * (g.nb1 + g.nb2 + 2);
  make_keys_kernel<<<kGrid, 256, sm, st>>>(g, rows, cols, nnz, keys, idx, bad);
  return cudaGetLastError();
}

cudaError_t launch_head_flags(const uint64_t* keys, uint64_t nnz, uint32_t* flags,
                              cudaStream_t st) {
  if (nnz == 0) return cudaSuccess;
  head_flags_kernel<<<kGrid, 256, 0, st>>>(keys, nnz, flags);
  return cudaGetLastError();
}

cudaError_t launch_merge_keys(const uint64_t* keys, const uint32_t* idx, const uint32_t* pos,
                              uint64_t nnz, const uint32_t* rows_in, const uint32_t* cols_in,
                              uint64_t* ukeys, uint32_t* urow, uint32_t* ucol, uint32_t* head_at,
                              cudaStream_t st) {
  if (nnz == 0) return cudaSuccess;
  merge_keys_kernel<<<kGrid, 256, 0, st>>>(keys, idx, pos, nnz, rows_in, cols_in, ukeys, urow,
                                           ucol, head_at);
  return cudaGetLastError();
}

cudaError_t launch_block_ptr(const uint64_t* ukeys, uint64_t u, uint64_t block_span,
                             uint32_t nblocks, uint64_t* block_ptr, cudaStream_t st) {
  block_ptr_kernel<<<(nblocks + 1 + 255) / 256, 256, 0, st>>>(ukeys, u, block_span, nblocks,
                                                               block_ptr);
  return cudaGetLastError();
}

cudaError_t launch_shuffle_keys(const uint64_t* ukeys, uint64_t u, uint64_t block_span,
                                uint64_t nB, int mode, uint64_t seed, uint64_t* keys2,
                                uint32_t* idx2, cudaStream_t st) {
  const uint64_t side_extent = mode == kLayoutColRuns ? nB : (nB ? block_span / nB : 1);
  int side_bits = 0;
  while (side_bits < 32 && (1ull << side_bits) < side_extent) ++side_bits;
  if (u == 0) return cudaSuccess;
  shuffle_keys_kernel<<<kGrid, 256, 0, st>>>(ukeys, u, block_span, nB, mode, side_bits, seed,
                                             keys2, idx2);
  return cudaGetLastError();
}

cudaError_t launch_gather_coords(const uint32_t* perm, uint64_t u, const uint32_t* urow,
                                 const uint32_t* ucol, uint32_t* row, uint32_t* col,
                                 cudaStream_t st) {
  if (u == 0) return cudaSuccess;
  gather_coords_kernel<<<kGrid, 256, 0, st>>>(perm, u, urow, ucol, row, col);
  return cudaGetLastError();
}

cudaError_t launch_gather_values(const uint32_t* perm, uint64_t u, const uint32_t* head_at,
                                 const uint64_t* keys, const uint32_t* idx, uint64_t nnz,
                                 const double* vals_in, void* val, int val_is_double,
                                 cudaStream_t st) {
  if (u == 0) return cudaSuccess;
  gather_values_kernel<<<kGrid, 256, 0, st>>>(perm, u, head_at, keys, idx, nnz, vals_in, val,
                                              val_is_double);
  return cudaGetLastError();
}

cudaError_t launch_offset_copy(const uint32_t* rows_in, const uint32_t* cols_in, uint64_t nnz,
                               uint32_t row0, uint32_t col0, uint32_t* rows_out,
                               uint32_t* cols_out, cudaStream_t st) {
  if (nnz == 0) return cudaSuccess;
  const uint64_t blocks = std::min<uint64_t>((nnz + 255) / 256, 4096);
  offset_copy_kernel<<<(unsigned)blocks, 256, 0, st>>>(rows_in, cols_in, nnz, row0, col0,
                                                       rows_out, cols_out);
  return cudaGetLastError();
}

cudaError_t launch_shift_blocks(const uint64_t* start, uint32_t nblocks, uint32_t nb2,
                                const uint64_t* off1, const uint64_t* off2, uint64_t nnz,
                                uint32_t* rows, uint32_t* cols, unsigned long long* bad,
                                cudaStream_t st) {
  if (nnz == 0) return cudaSuccess;
  shift_blocks_kernel<<<kGrid, 256, 0, st>>>(start, nblocks, nb2, off1, off2, nnz, rows, cols, bad);
  return cudaGetLastError();
}

cudaError_t launch_counts_to_u32(const uint64_t* in, uint64_t len, uint32_t* out,
                                 cudaStream_t st) {
  if (len == 0) return cudaSuccess;
  counts_to_u32_kernel<<<kGrid, 256, 0, st>>>(in, len, out);
  return cudaGetLastError();
}

cudaError_t launch_count_nnz12(const uint32_t* row, const uint32_t* col, uint64_t nnz,
                               uint32_t* cnt1, uint32_t* cnt2, cudaStream_t st) {
  if (nnz == 0) return cudaSuccess;
  count_nnz12_kernel<<<kGrid, 256, 0, st>>>(row, col, nnz, cnt1, cnt2);
  return cudaGetLastError();
}

cudaError_t launch_inverse_counts(const uint32_t* cnt, uint64_t len, void* inv, int as_double,
                                  cudaStream_t st) {
  if (len == 0) return cudaSuccess;
  inverse_counts_kernel<<<kGrid, 256, 0, st>>>(cnt, len, inv, as_double);
  return cudaGetLastError();
}

cudaError_t launch_factor_to_device(int precision, const double* src, uint64_t rows,
                                    uint32_t r, uint32_t rp, void* dst, cudaStream_t st) {
  if (rows == 0) return cudaSuccess;
  if (precision == kFp64)
    factor_to_device_kernel<double><<<kGrid, 256, 0, st>>>(src, rows, r, rp, (double*)dst);
  else if (precision == kFp32)
    factor_to_device_kernel<float><<<kGrid, 256, 0, st>>>(src, rows, r, rp, (float*)dst);
  else
    factor_to_device_kernel<__nv_bfloat16><<<kGrid, 256, 0, st>>>(src, rows, r, rp,
                                                                  (__nv_bfloat16*)dst);
  return cudaGetLastError();
}

cudaError_t launch_factor_to_host(int precision, const void* src, uint64_t rows, uint32_t r,
                                  uint32_t rp, double* dst, cudaStream_t st) {
  if (rows == 0) return cudaSuccess;
  if (precision == kFp64)
    factor_to_host_kernel<double><<<kGrid, 256, 0, st>>>((const double*)src, rows, r, rp, dst);
  else if (precision == kFp32)
    factor_to_host_kernel<float><<<kGrid, 256, 0, st>>>((const float*)src, rows, r, rp, dst);
  else
    factor_to_host_kernel<__nv_bfloat16><<<kGrid, 256, 0, st>>>((const __nv_bfloat16*)src, rows,
                                                                r, rp, dst);
  return cudaGetLastError();
}

}  // namespace dsgdpp
