// noalloc.cu -- an FP32 sum-of-squared-errors entry point that allocates nothing.
//
// Some callers cannot call cudaMalloc: code that runs inside another
// framework's memory pool, or in a process whose allocator is owned by
// someone else, must not grow the device heap behind the owner's back.  This
// entry point serves them.  The caller passes device buffers for the inputs
// and the output; the scratch the reduction needs (one FP64 partial sum per
// CTA) lives in a fixed array in this library's device image, so the call
// itself never allocates or frees device memory.
//
// The scratch array is file-scope device memory.  In host code its name is
// only a host-side stand-in, not a device address, so the first call on each
// device (with that device current) looks its address up once with
// cudaGetSymbolAddress and keeps it.  Every call on a device shares the one
// array and leaves its last contents behind; each partial slot the kernel
// uses is written before it is read, so nothing needs clearing.  Calls that
// overlap on the GPU (for instance on two streams at once) race on the array.
#include <cstdio>
#include <mutex>

#include "../../include/dsgdpp.h"
#include "kernels.cuh"

namespace {

// one partial sum per CTA of the reduction; the grid never exceeds this
static __device__ __align__(256) double g_noalloc_partials[DSGDPP_NOALLOC_MAX_PARTIALS];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_scratch[kMaxDevices] = {};
int g_sms[kMaxDevices] = {};

// Once per device, with that device current: the device address of the
// scratch array and the SM count.
cudaError_t device_setup(int dev, double** scratch, int* sms) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess) return e;
    int n = 0;
    e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    g_sms[dev] = n;
    g_scratch[dev] = static_cast<double*>(p);
  }
  *scratch = g_scratch[dev];
  *sms = g_sms[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" int dsgdpp_nzsl_fp32_noalloc(const uint32_t* rows, const uint32_t* cols,
                                        const float* vals, uint64_t nnz, const float* W,
                                        const float* H, uint32_t rank, uint32_t ld,
                                        uint32_t partials, double* out, void* stream) {
  if (!out || (nnz > 0 && (!rows || !cols || !vals || !W || !H)) || rank == 0)
    return DSGDPP_E_INVALID;
  // rows of W and H are read as 16-byte vectors
  if (ld % 4 != 0 || ld < (rank + 3) / 4 * 4 || (reinterpret_cast<uintptr_t>(W) & 15u) ||
      (reinterpret_cast<uintptr_t>(H) & 15u))
    return DSGDPP_E_INVALID;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return DSGDPP_E_CUDA;
  double* scratch = nullptr;
  int sms = 0;
  if (device_setup(dev, &scratch, &sms) != cudaSuccess) return DSGDPP_E_CUDA;
  const uint32_t grid = partials ? partials : (uint32_t)sms * 4;
  if (grid > DSGDPP_NOALLOC_MAX_PARTIALS) {
    std::fprintf(stderr,
                 "dsgdpp_nzsl_fp32_noalloc: %u partial sums requested, the fixed scratch holds "
                 "at most %d\n",
                 grid, DSGDPP_NOALLOC_MAX_PARTIALS);
    return DSGDPP_E_INVALID;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (nnz == 0) {
    // an empty matrix: write 0 through the same reduction over zero partials
    if (dsgdpp::launch_sum_partials(scratch, 0, out, st) != cudaSuccess) return DSGDPP_E_CUDA;
    return DSGDPP_OK;
  }
  if (dsgdpp::launch_nzsl_partials(dsgdpp::kFp32, rows, cols, vals, nnz, W, H, rank, ld, scratch,
                                   grid, st) != cudaSuccess)
    return DSGDPP_E_CUDA;
  if (dsgdpp::launch_sum_partials(scratch, grid, out, st) != cudaSuccess) return DSGDPP_E_CUDA;
  return DSGDPP_OK;
}
