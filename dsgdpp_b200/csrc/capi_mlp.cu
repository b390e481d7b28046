// capi_mlp.cu -- C ABI of the step-size controller network (include/dsgdpp.h).
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/dsgdpp.h"
#include "kernels.cuh"
#include "schedule.h"

using namespace dsgdpp;

struct dsgdpp_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  float* P = nullptr;  // parameters
  float* m = nullptr;  // Adam moments
  float* v = nullptr;
  float* g = nullptr;  // reduced gradient
  float* X = nullptr;  // batch buffers (grown on demand)
  float* Y = nullptr;
  float* out = nullptr;
  float* grads = nullptr;  // per-sample gradients
  float* losses = nullptr;
  int cap = 0;
  int step = 0;
};

namespace {

bool ok(cudaError_t e) { return e == cudaSuccess; }

int grow(dsgdpp_mlp* n, int batch) {
  if (batch <= n->cap) return DSGDPP_OK;
  const int np = mlp_param_count();
  cudaFree(n->X); cudaFree(n->Y); cudaFree(n->out); cudaFree(n->grads); cudaFree(n->losses);
  n->X = n->Y = n->out = n->grads = n->losses = nullptr;
  n->cap = 0;
  if (!ok(cudaMalloc(&n->X, (size_t)batch * mlp_input_count() * 4)) ||
      !ok(cudaMalloc(&n->Y, (size_t)batch * 4)) || !ok(cudaMalloc(&n->out, (size_t)batch * 4)) ||
      !ok(cudaMalloc(&n->grads, (size_t)batch * np * 4)) ||
      !ok(cudaMalloc(&n->losses, (size_t)batch * 4)))
    return DSGDPP_E_NOMEM;
  n->cap = batch;
  return DSGDPP_OK;
}

int upload(dsgdpp_mlp* n, const float* x, const float* y, int batch) {
  if (batch <= 0 || !x) return DSGDPP_E_INVALID;
  if (cudaSetDevice(n->device) != cudaSuccess) return DSGDPP_E_CUDA;
  int rc = grow(n, batch);
  if (rc != DSGDPP_OK) return rc;
  if (!ok(cudaMemcpyAsync(n->X, x, (size_t)batch * mlp_input_count() * 4, cudaMemcpyHostToDevice,
                          n->stream)))
    return DSGDPP_E_CUDA;
  if (y && !ok(cudaMemcpyAsync(n->Y, y, (size_t)batch * 4, cudaMemcpyHostToDevice, n->stream)))
    return DSGDPP_E_CUDA;
  return DSGDPP_OK;
}

// loss and gradient of the batch already uploaded; sums stay on the device
int gradient(dsgdpp_mlp* n, int batch, float* loss_out) {
  if (!ok(launch_mlp(n->P, n->X, n->Y, batch, n->out, n->grads, n->losses, n->stream)) ||
      !ok(launch_mlp_reduce(n->grads, batch, n->g, n->stream)))
    return DSGDPP_E_CUDA;
  if (loss_out) {
    std::vector<float> l(batch);
    if (!ok(cudaMemcpyAsync(l.data(), n->losses, (size_t)batch * 4, cudaMemcpyDeviceToHost,
                            n->stream)) ||
        !ok(cudaStreamSynchronize(n->stream)))
      return DSGDPP_E_CUDA;
    float s = 0;
    for (float v : l) s += v;
    *loss_out = s;
  }
  return DSGDPP_OK;
}

}  // namespace

extern "C" {

int dsgdpp_mlp_param_count(void) { return mlp_param_count(); }

int dsgdpp_mlp_create(int device, uint64_t seed, dsgdpp_mlp** out) {
  if (!out) return DSGDPP_E_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return DSGDPP_E_CUDA;
  auto* n = new (std::nothrow) dsgdpp_mlp();
  if (!n) return DSGDPP_E_NOMEM;
  n->device = device;
  const int np = mlp_param_count();
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking) != cudaSuccess ||
      !ok(cudaMalloc(&n->P, np * 4)) || !ok(cudaMalloc(&n->m, np * 4)) ||
      !ok(cudaMalloc(&n->v, np * 4)) || !ok(cudaMalloc(&n->g, np * 4))) {
    dsgdpp_mlp_destroy(n);
    return DSGDPP_E_CUDA;
  }
  // Glorot-uniform weights from the pinned Random32, zero biases
  std::vector<float> p(np, 0.0f);
  Random32 rng((uint32_t)(seed ^ (seed >> 32)));
  auto fill = [&](int off, int fan_in, int fan_out, int count) {
    const double lim = std::sqrt(6.0 / (fan_in + fan_out));
    for (int k = 0; k < count; ++k) p[off + k] = (float)((rng.next() / 4294967296.0 * 2 - 1) * lim);
  };
  fill(0, 16, 64, 64 * 16);             // W1
  fill(64 * 16 + 64, 64, 64, 64 * 64);  // W2
  fill(64 * 16 + 64 + 64 * 64 + 64, 64, 1, 64);  // W3
  if (!ok(cudaMemcpy(n->P, p.data(), np * 4, cudaMemcpyHostToDevice)) ||
      !ok(cudaMemset(n->m, 0, np * 4)) || !ok(cudaMemset(n->v, 0, np * 4))) {
    dsgdpp_mlp_destroy(n);
    return DSGDPP_E_CUDA;
  }
  *out = n;
  return DSGDPP_OK;
}

void dsgdpp_mlp_destroy(dsgdpp_mlp* n) {
  if (!n) return;
  cudaSetDevice(n->device);
  if (n->stream) cudaStreamSynchronize(n->stream);
  for (float* p : {n->P, n->m, n->v, n->g, n->X, n->Y, n->out, n->grads, n->losses}) cudaFree(p);
  if (n->stream) cudaStreamDestroy(n->stream);
  delete n;
}

int dsgdpp_mlp_get_params(dsgdpp_mlp* n, float* params) {
  if (!n || !params) return DSGDPP_E_INVALID;
  if (cudaSetDevice(n->device) != cudaSuccess ||
      !ok(cudaMemcpy(params, n->P, mlp_param_count() * 4, cudaMemcpyDeviceToHost)))
    return DSGDPP_E_CUDA;
  return DSGDPP_OK;
}

int dsgdpp_mlp_set_params(dsgdpp_mlp* n, const float* params) {
  if (!n || !params) return DSGDPP_E_INVALID;
  const int np = mlp_param_count();
  if (cudaSetDevice(n->device) != cudaSuccess ||
      !ok(cudaMemcpy(n->P, params, np * 4, cudaMemcpyHostToDevice)) ||
      !ok(cudaMemset(n->m, 0, np * 4)) || !ok(cudaMemset(n->v, 0, np * 4)))
    return DSGDPP_E_CUDA;
  n->step = 0;
  return DSGDPP_OK;
}

int dsgdpp_mlp_forward(dsgdpp_mlp* n, const float* x, int batch, float* out) {
  if (!n || !out) return DSGDPP_E_INVALID;
  int rc = upload(n, x, nullptr, batch);
  if (rc != DSGDPP_OK) return rc;
  if (!ok(launch_mlp(n->P, n->X, nullptr, batch, n->out, nullptr, nullptr, n->stream)) ||
      !ok(cudaMemcpyAsync(out, n->out, (size_t)batch * 4, cudaMemcpyDeviceToHost, n->stream)) ||
      !ok(cudaStreamSynchronize(n->stream)))
    return DSGDPP_E_CUDA;
  return DSGDPP_OK;
}

int dsgdpp_mlp_gradient(dsgdpp_mlp* n, const float* x, const float* y, int batch, float* loss,
                        float* grad) {
  if (!n || !y) return DSGDPP_E_INVALID;
  int rc = upload(n, x, y, batch);
  if (rc != DSGDPP_OK) return rc;
  rc = gradient(n, batch, loss);
  if (rc != DSGDPP_OK) return rc;
  if (grad && (!ok(cudaMemcpyAsync(grad, n->g, mlp_param_count() * 4, cudaMemcpyDeviceToHost,
                                   n->stream)) ||
               !ok(cudaStreamSynchronize(n->stream))))
    return DSGDPP_E_CUDA;
  return DSGDPP_OK;
}

int dsgdpp_mlp_train_step(dsgdpp_mlp* n, const float* x, const float* y, int batch, float lr,
                          float* loss) {
  if (!n || !y) return DSGDPP_E_INVALID;
  int rc = upload(n, x, y, batch);
  if (rc != DSGDPP_OK) return rc;
  rc = gradient(n, batch, loss);
  if (rc != DSGDPP_OK) return rc;
  n->step += 1;
  if (!ok(launch_adam(n->P, n->g, n->m, n->v, lr, 0.9f, 0.999f, 1e-8f, n->step, n->stream)) ||
      !ok(cudaStreamSynchronize(n->stream)))
    return DSGDPP_E_CUDA;
  return DSGDPP_OK;
}

void dsgdpp_controller_features(const double* tr, const double* te, double eps, double upd_mean,
                                double upd_max, double epoch_frac, double last_log_mult,
                                double fail_eps, float* f) {
  auto lr = [](double a, double b) -> float {  // log-ratio of two losses, 0 if missing
    if (!(a > 0) || !(b > 0) || std::isnan(a) || std::isnan(b)) return 0.0f;
    double v = std::log(a / b);
    return (float)std::fmax(-5.0, std::fmin(5.0, v));
  };
  for (int k = 0; k < 4; ++k) {
    f[k] = lr(tr[k], tr[k + 1]) * 10.0f;
    f[4 + k] = lr(te[k], te[k + 1]) * 10.0f;
  }
  // log10 of a positive quantity / 3, bounded to [-10, 10]; a non-finite or
  // huge value (a diverging run) maps to the upper bound
  auto lg = [](double v) -> float {
    if (!(v == v) || v > 1e30) return 10.0f;
    return (float)std::fmax(-10.0, std::fmin(10.0, std::log10(std::fmax(v, 1e-30)) / 3.0));
  };
  f[8] = lg(eps);
  f[9] = lg(upd_mean);
  f[10] = lg(upd_max);
  f[11] = (float)std::fmax(0.0, std::fmin(1.0, epoch_frac));
  f[12] = lr(tr[0], te[0]);
  f[13] = (float)std::fmax(-1.0, std::fmin(1.0, last_log_mult));
  f[14] = (tr[0] > 0 && tr[1] > 0) ? (tr[0] < tr[1] ? 1.0f : -1.0f) : 0.0f;
  // distance (log units, as the multiplier) to the smallest step that raised
  // the loss; 3 when none has (or the ratio is not a finite positive number)
  const double ratio = fail_eps / eps;
  f[15] = (fail_eps > 0 && ratio > 0 && std::isfinite(ratio))
              ? (float)std::fmax(-3.0, std::fmin(3.0, std::log(ratio)))
              : 3.0f;
}

}  // extern "C"
