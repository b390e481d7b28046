// kernels_rm.cu -- matrices of a .rm descriptor generated on the device.
//
// Every value is a counter-based draw (SplitMix64 outputs at a computed
// position), so one thread makes one factor element or one nonzero with no
// sequential stream to walk; the scheme is stated in rm.h.  HBM-bound: a
// nonzero reads one Worig row and one Horig row (2 * rank * 8 bytes, mostly
// from L2 for the hot rows of a chunk) and writes 16 bytes.
#include <algorithm>
#include <stdexcept>
#include <string>

#include "rm_device.h"
#include "schedule.h"

namespace dsgdpp {
namespace {

constexpr uint64_t kGolden = 0x9e3779b97f4a7c15ull;

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ uint64_t stream_at(uint64_t key, uint64_t n) {
  return mix64(key + (n + 1) * kGolden);
}
__device__ __forceinline__ uint64_t rm_key(uint32_t seed, uint32_t tag) {
  return mix64(((uint64_t)tag << 32) | seed);
}
__device__ __forceinline__ double unit53(uint64_t x) { return (double)(x >> 11) * 0x1.0p-53; }

struct DevDist {
  int kind;
  double a, b;
};

// value draw n of `key` (two stream outputs per draw)
__device__ __forceinline__ double draw(const DevDist& d, uint64_t key, uint64_t n) {
  const double u = unit53(stream_at(key, 2 * n));
  if (d.kind == 1) return __dadd_rn(d.a, __dmul_rn(__dsub_rn(d.b, d.a), u));
  const double u1 = __dsub_rn(1.0, u);  // (0, 1]
  const double u2 = unit53(stream_at(key, 2 * n + 1));
  const double r = sqrt(__dmul_rn(-2.0, log(u1)));
  return __dmul_rn(d.b, __dmul_rn(r, cospi(__dmul_rn(2.0, u2))));
}

__device__ __forceinline__ uint32_t find_chunk(const uint64_t* start, uint32_t n, uint64_t x) {
  // largest c < n with start[c] <= x (start is non-decreasing, start[0] = 0)
  uint32_t lo = 0, hi = n - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (start[mid] <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__global__ void rm_factor_kernel(DevDist dist, const uint32_t* seeds, const uint64_t* off,
                                 uint32_t nchunks, uint64_t rows, uint32_t rank, uint32_t tag,
                                 double* out) {
  const uint64_t total = rows * rank, stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total; e += stride) {
    const uint64_t i = e / rank, z = e - i * rank;
    const uint32_t b = find_chunk(off, nchunks, i);
    out[e] = draw(dist, rm_key(seeds[b], tag), (i - off[b]) * rank + z);
  }
}

__global__ void rm_data_kernel(DevDist noise, const uint32_t* seeds, const uint64_t* start,
                               const uint64_t* off1, const uint64_t* off2, uint32_t c2,
                               uint32_t nc, const double* W, const double* H, uint32_t rank,
                               uint64_t total, uint32_t* rows, uint32_t* cols, double* vals) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < total; k += stride) {
    const uint32_t c = find_chunk(start, nc, k);
    const uint32_t b1 = c / c2, b2 = c - b1 * c2;
    const uint64_t r0 = off1[b1], c0 = off2[b2];
    const uint64_t ncols = off2[b2 + 1] - c0;
    const uint64_t N = (off1[b1 + 1] - r0) * ncols;
    // Feistel permutation of [0, 2^(2h)) restricted to [0, N) by cycle walking
    const uint64_t key = rm_key(seeds[c], kTagCells);
    const int bits = N > 1 ? 64 - __clzll((long long)(N - 1)) : 1;
    const int h = max(1, (bits + 1) >> 1);
    const uint64_t mask = (h >= 64) ? ~0ull : ((1ull << h) - 1);
    uint64_t rk[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) rk[r] = stream_at(key, r);
    uint64_t x = k - start[c];
    do {
      uint64_t L = x >> h, R = x & mask;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const uint64_t F = mix64(R ^ rk[r]) & mask;
        const uint64_t nl = R;
        R = L ^ F;
        L = nl;
      }
      x = (L << h) | R;
    } while (x >= N);  // ends: x lies on a cycle of the permutation through a value below N
    const uint64_t i = r0 + x / ncols, j = c0 + x % ncols;
    const double* w = W + i * rank;
    const double* hh = H + j * rank;
    double v = 0.0;
    for (uint32_t z = 0; z < rank; ++z) v = __dadd_rn(v, __dmul_rn(w[z], hh[z]));
    if (noise.kind >= 0) v = __dadd_rn(v, draw(noise, rm_key(seeds[c], kTagNoise), x));
    rows[k] = (uint32_t)i;
    cols[k] = (uint32_t)j;
    vals[k] = v;
  }
}

void cu(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

DevDist dev_dist(const std::string& name, const std::string& spec) {
  DevDist d{-1, 0, 0};
  const RmDist p = parse_dist(name, spec);
  d.kind = p.kind;
  d.a = p.a;
  d.b = p.b;
  return d;
}

// offsets with the total appended (nchunks + 1 entries)
std::vector<uint64_t> offsets_with_end(uint64_t size, uint64_t chunks) {
  std::vector<uint64_t> o = block_offsets(size, (uint32_t)chunks);
  o.push_back(size);
  return o;
}

// device copies of small host arrays, freed on scope exit
struct DevArrays {
  std::vector<void*> ptrs;
  template <typename T>
  T* put(const std::vector<T>& h, cudaStream_t st) {
    void* p = nullptr;
    cu(cudaMalloc(&p, std::max<size_t>(1, h.size()) * sizeof(T)), "cudaMalloc");
    ptrs.push_back(p);
    if (!h.empty())
      cu(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st), "H2D");
    return static_cast<T*>(p);
  }
  ~DevArrays() {
    for (void* p : ptrs) cudaFree(p);
  }
};

uint32_t grid_for(uint64_t work) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint64_t want = (work + 255) / 256;
  return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sms * 8));
}

}  // namespace

uint64_t rm_count(const RmDesc& d, int which) {
  if (!d.has_data()) return 0;
  uint64_t s = 0;
  for (uint64_t c : which == 0 ? d.nnz_v : d.nnz_vtest) s += c;
  return s;
}

void rm_factors_device(const RmDesc& d, double* W, double* H, cudaStream_t st) {
  const DevDist dist = dev_dist("values", d.values);
  DevArrays a;
  const uint32_t* sw = a.put(d.seeds_w, st);
  const uint32_t* sh = a.put(d.seeds_h, st);
  const uint64_t* o1 = a.put(offsets_with_end(d.size1, d.chunks1), st);
  const uint64_t* o2 = a.put(offsets_with_end(d.size2, d.chunks2), st);
  const uint32_t rank = (uint32_t)d.rank;
  rm_factor_kernel<<<grid_for(d.size1 * rank), 256, 0, st>>>(dist, sw, o1, (uint32_t)d.chunks1,
                                                             d.size1, rank, kTagW, W);
  cu(cudaGetLastError(), "rm_factor_kernel");
  rm_factor_kernel<<<grid_for(d.size2 * rank), 256, 0, st>>>(dist, sh, o2, (uint32_t)d.chunks2,
                                                             d.size2, rank, kTagH, H);
  cu(cudaGetLastError(), "rm_factor_kernel");
  cu(cudaStreamSynchronize(st), "sync");
}

uint64_t rm_data_device(const RmDesc& d, int which, uint32_t* rows, uint32_t* cols, double* vals,
                        cudaStream_t st) {
  if (!d.has_data()) throw std::invalid_argument("the descriptor holds no data matrix (nnz or nnzTest is 0)");
  const uint64_t total = rm_count(d, which);
  if (total == 0) return 0;
  // the test matrix has no noise (generateDistributedMatrix_impl.h:641-643)
  DevDist noise{-1, 0, 0};
  if (which == 0 && d.noise.find_first_not_of(" \t\r\n") != std::string::npos)
    noise = dev_dist("noise", d.noise);
  const uint64_t nc = d.chunks1 * d.chunks2;
  std::vector<uint64_t> start(nc + 1, 0);
  const std::vector<uint64_t>& cnt = which == 0 ? d.nnz_v : d.nnz_vtest;
  for (uint64_t c = 0; c < nc; ++c) start[c + 1] = start[c] + cnt[c];
  double* fac = nullptr;
  cu(cudaMalloc(&fac, (d.size1 + d.size2) * d.rank * sizeof(double)), "cudaMalloc Worig/Horig");
  struct Free {
    double* p;
    ~Free() { cudaFree(p); }
  } free_fac{fac};
  rm_factors_device(d, fac, fac + d.size1 * d.rank, st);
  DevArrays a;
  const uint32_t* seeds = a.put(which == 0 ? d.seeds_v : d.seeds_vtest, st);
  const uint64_t* dstart = a.put(start, st);
  const uint64_t* o1 = a.put(offsets_with_end(d.size1, d.chunks1), st);
  const uint64_t* o2 = a.put(offsets_with_end(d.size2, d.chunks2), st);
  rm_data_kernel<<<grid_for(total), 256, 0, st>>>(noise, seeds, dstart, o1, o2, (uint32_t)d.chunks2,
                                                  (uint32_t)nc, fac, fac + d.size1 * d.rank,
                                                  (uint32_t)d.rank, total, rows, cols, vals);
  cu(cudaGetLastError(), "rm_data_kernel");
  cu(cudaStreamSynchronize(st), "sync");
  return total;
}

}  // namespace dsgdpp
