// capi_rm.cu -- C ABI of the .rm descriptors and of their stand-alone generation.
#include <cstring>
#include <string>

#include "../../include/dsgdpp.h"
#include "mmio.h"
#include "rm_device.h"

namespace {

thread_local std::string g_rm_error;

template <typename F>
int rm_guard(F&& f) {
  try {
    g_rm_error.clear();
    return f();
  } catch (const dsgdpp::MmError& e) {
    g_rm_error = e.what();
    return DSGDPP_E_IO;
  } catch (const std::invalid_argument& e) {
    g_rm_error = e.what();
    return DSGDPP_E_INVALID;
  } catch (const std::bad_alloc&) {
    g_rm_error = "out of memory";
    return DSGDPP_E_CUDA;
  } catch (const std::exception& e) {
    g_rm_error = e.what();
    return DSGDPP_E_CUDA;
  }
}

// device buffers for the stand-alone generators, freed on scope exit
struct Scratch {
  void* p = nullptr;
  explicit Scratch(size_t bytes) {
    if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) throw std::runtime_error("cudaMalloc failed");
  }
  ~Scratch() { cudaFree(p); }
};

}  // namespace

extern "C" {

const char* dsgdpp_rm_error(void) { return g_rm_error.c_str(); }

int dsgdpp_rm_load(const char* path, dsgdpp_rm** out) {
  if (!path || !out) return DSGDPP_E_INVALID;
  *out = nullptr;
  return rm_guard([&]() {
    dsgdpp_rm* h = new dsgdpp_rm;
    try {
      h->d = dsgdpp::rm_load(path);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return DSGDPP_OK;
  });
}

int dsgdpp_rm_create(uint64_t size1, uint64_t size2, uint32_t blocks1, uint32_t blocks2,
                     uint64_t nnz, uint64_t nnz_test, uint32_t rank, const char* values,
                     const char* noise, dsgdpp_rm** out) {
  if (!values || !out) return DSGDPP_E_INVALID;
  *out = nullptr;
  return rm_guard([&]() {
    dsgdpp_rm* h = new dsgdpp_rm;
    try {
      h->d = dsgdpp::rm_create(size1, size2, blocks1, blocks2, nnz, nnz_test, rank, values,
                               noise ? noise : "");
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return DSGDPP_OK;
  });
}

int dsgdpp_rm_save(const dsgdpp_rm* rm, const char* path) {
  if (!rm || !path) return DSGDPP_E_INVALID;
  return rm_guard([&]() {
    dsgdpp::rm_save(path, rm->d);
    return DSGDPP_OK;
  });
}

void dsgdpp_rm_destroy(dsgdpp_rm* rm) { delete rm; }

int dsgdpp_rm_info(const dsgdpp_rm* rm, uint64_t* out) {
  if (!rm || !out) return DSGDPP_E_INVALID;
  const dsgdpp::RmDesc& d = rm->d;
  const uint64_t v[9] = {d.size1, d.size2, d.rank, d.chunks1, d.chunks2, d.nnz, d.nnz_test,
                         dsgdpp::rm_count(d, 0), dsgdpp::rm_count(d, 1)};
  std::memcpy(out, v, sizeof(v));
  return DSGDPP_OK;
}

int dsgdpp_rm_generate(const dsgdpp_rm* rm, int which, int device, uint32_t* rows,
                       uint32_t* cols, double* vals) {
  if (!rm || (which != DSGDPP_TRAIN && which != DSGDPP_TEST)) return DSGDPP_E_INVALID;
  return rm_guard([&]() {
    const uint64_t n = dsgdpp::rm_count(rm->d, which);
    if (!rm->d.has_data()) throw std::invalid_argument("the descriptor holds no data matrix");
    if (n && (!rows || !cols || !vals)) throw std::invalid_argument("null output array");
    if (cudaSetDevice(device) != cudaSuccess) throw std::runtime_error("cudaSetDevice failed");
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
      throw std::runtime_error("cudaStreamCreate failed");
    struct S {
      cudaStream_t s;
      ~S() { cudaStreamDestroy(s); }
    } guard{st};
    Scratch r(n * 4), c(n * 4), v(n * 8);
    dsgdpp::rm_data_device(rm->d, which, (uint32_t*)r.p, (uint32_t*)c.p, (double*)v.p, st);
    if (n) {
      if (cudaMemcpyAsync(rows, r.p, n * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaMemcpyAsync(cols, c.p, n * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaMemcpyAsync(vals, v.p, n * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess)
        throw std::runtime_error("copy of the generated matrix failed");
    }
    return DSGDPP_OK;
  });
}

int dsgdpp_rm_generate_factors(const dsgdpp_rm* rm, int device, double* W, double* H) {
  if (!rm || !W || !H) return DSGDPP_E_INVALID;
  return rm_guard([&]() {
    const dsgdpp::RmDesc& d = rm->d;
    if (cudaSetDevice(device) != cudaSuccess) throw std::runtime_error("cudaSetDevice failed");
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
      throw std::runtime_error("cudaStreamCreate failed");
    struct S {
      cudaStream_t s;
      ~S() { cudaStreamDestroy(s); }
    } guard{st};
    Scratch f((d.size1 + d.size2) * d.rank * 8);
    double* fw = (double*)f.p;
    dsgdpp::rm_factors_device(d, fw, fw + d.size1 * d.rank, st);
    if (cudaMemcpyAsync(W, fw, d.size1 * d.rank * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(H, fw + d.size1 * d.rank, d.size2 * d.rank * 8, cudaMemcpyDeviceToHost,
                        st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      throw std::runtime_error("copy of the generated factors failed");
    return DSGDPP_OK;
  });
}

}  // extern "C"
