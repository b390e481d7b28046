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
// only a host-side stand-in, not a device address, so the first call in each
// CUDA context (with that context's device current) looks its address up once
// with cudaGetSymbolAddress and keeps it.  The address belongs to the context
// the module was loaded into, so it is kept per context, not per device
// number: a caller that makes its own context current gets that context's
// copy of the array.  Every call in a context shares the one array and leaves
// its last contents behind; each partial slot the kernel uses is written
// before it is read, so nothing needs clearing.  Calls that overlap on the GPU
// (for instance on two streams at once) race on the array.
#include <cuda.h>

#include <cstdio>
#include <mutex>

#include "../../include/dsgdpp.h"
#include "kernels.cuh"

namespace {

// one partial sum per CTA of the reduction; the grid never exceeds this
static __device__ __align__(256) double g_noalloc_partials[DSGDPP_NOALLOC_MAX_PARTIALS];

struct Setup {
  CUcontext ctx;
  double* scratch;
  int sms;
};
constexpr int kMaxContexts = 64;
std::mutex g_setup_mutex;
Setup g_setup[kMaxContexts] = {};
int g_nsetup = 0;
using CtxGetCurrent = CUresult (*)(CUcontext*);
CtxGetCurrent g_ctx_get_current = nullptr;

// The current context, through the driver entry point the runtime exposes
// (the library links no driver library of its own).
cudaError_t current_context(CUcontext* ctx) {
  if (!g_ctx_get_current) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    const cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
      return e != cudaSuccess ? e : cudaErrorSymbolNotFound;
    g_ctx_get_current = reinterpret_cast<CtxGetCurrent>(fn);
  }
  return g_ctx_get_current(ctx) == CUDA_SUCCESS && *ctx ? cudaSuccess : cudaErrorDeviceUninitialized;
}

// Once per context, with its device current: the device address of the
// scratch array and the SM count.
cudaError_t context_setup(int dev, double** scratch, int* sms) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  // a runtime call first, so the device's primary context exists and is current
  int n = 0;
  cudaError_t e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  CUcontext ctx = nullptr;
  e = current_context(&ctx);
  if (e != cudaSuccess) return e;
  for (int k = 0; k < g_nsetup; ++k)
    if (g_setup[k].ctx == ctx) {
      *scratch = g_setup[k].scratch;
      *sms = g_setup[k].sms;
      return cudaSuccess;
    }
  if (g_nsetup == kMaxContexts) return cudaErrorDeviceUninitialized;
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_noalloc_partials);
  if (e != cudaSuccess) return e;
  g_setup[g_nsetup++] = Setup{ctx, static_cast<double*>(p), n};
  *scratch = static_cast<double*>(p);
  *sms = n;
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
      (reinterpret_cast<uintptr_t>(H) & 15u)) {
    std::fprintf(stderr,
                 "dsgdpp_nzsl_fp32_noalloc: ld %u must be a multiple of 4 and at least the "
                 "rank %u rounded up to 4, and W and H 16-byte aligned\n",
                 ld, rank);
    return DSGDPP_E_INVALID;
  }
  if (ld > DSGDPP_NOALLOC_MAX_LD) {
    std::fprintf(stderr,
                 "dsgdpp_nzsl_fp32_noalloc: ld %u is above the widest row the loss kernel "
                 "takes (%d floats)\n",
                 ld, DSGDPP_NOALLOC_MAX_LD);
    return DSGDPP_E_INVALID;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DSGDPP_E_CUDA;
  double* scratch = nullptr;
  int sms = 0;
  if (context_setup(dev, &scratch, &sms) != cudaSuccess) return DSGDPP_E_CUDA;
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
