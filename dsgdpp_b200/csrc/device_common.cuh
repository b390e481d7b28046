// device_common.cuh -- shared device-side types of the DSGD++ kernels.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace dsgdpp {

constexpr unsigned kFullMask = 0xffffffffu;
constexpr int kChunk = 32;  // records per Hogwild chunk (one per lane)

// Element traits of the three factor storage types.  Factors move as 16-byte
// vectors: VW elements per vector.
template <typename T> struct Elem;
template <> struct Elem<double> {
  using C = double;  // compute type
  static constexpr int VW = 2;
  __device__ static inline void unpack(const uint4& v, double (&f)[2]) {
    f[0] = __hiloint2double((int)v.y, (int)v.x);
    f[1] = __hiloint2double((int)v.w, (int)v.z);
  }
  __device__ static inline uint4 pack(const double (&f)[2]) {
    uint4 v;
    v.x = (unsigned)__double2loint(f[0]); v.y = (unsigned)__double2hiint(f[0]);
    v.z = (unsigned)__double2loint(f[1]); v.w = (unsigned)__double2hiint(f[1]);
    return v;
  }
};
template <> struct Elem<float> {
  using C = float;
  static constexpr int VW = 4;
  __device__ static inline void unpack(const uint4& v, float (&f)[4]) {
    f[0] = __uint_as_float(v.x); f[1] = __uint_as_float(v.y);
    f[2] = __uint_as_float(v.z); f[3] = __uint_as_float(v.w);
  }
  __device__ static inline uint4 pack(const float (&f)[4]) {
    return make_uint4(__float_as_uint(f[0]), __float_as_uint(f[1]), __float_as_uint(f[2]),
                      __float_as_uint(f[3]));
  }
};
template <> struct Elem<__nv_bfloat16> {
  using C = float;
  static constexpr int VW = 8;
  __device__ static inline void unpack(const uint4& v, float (&f)[8]) {
    const unsigned w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      f[2 * k] = __uint_as_float(w[k] << 16);
      f[2 * k + 1] = __uint_as_float(w[k] & 0xffff0000u);
    }
  }
};

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): 10 rounds of the 4x32 bijection with the
// published multipliers and Weyl key increments.
struct Philox4 {
  uint32_t v[4];
};
__host__ __device__ inline uint32_t mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}
__host__ __device__ inline Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2,
                                                 uint32_t c3, uint32_t k0, uint32_t k1) {
  constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int round = 0; round < 10; ++round) {
    uint32_t hi0 = mulhi32(M0, c0), lo0 = M0 * c0;
    uint32_t hi1 = mulhi32(M1, c2), lo1 = M1 * c2;
    uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += W0; k1 += W1;
  }
  Philox4 r;
  r.v[0] = c0; r.v[1] = c1; r.v[2] = c2; r.v[3] = c3;
  return r;
}

// Random bits of one stochastically rounded vector write: a Philox-4x32-10
// block drawn once per chunk and lane (`base`) is expanded per write by one
// multiply and xor-shift of (word xor tag * golden ratio), the tag distinct
// per record, vector and side within the chunk.  For each tag the map is a
// bijection of the uniform Philox word, so every write's bits are uniform;
// the xor-shift folds the product's well-mixed high half into the low half
// that rounds the lower value of each pair.  (MurmurHash3's 32-bit
// finalizer per word -- two multiplies and three xor-shifts -- cost the
// BF16 epochs 7-19%: C2 5.90 vs 5.50 ms, C3 16.1 vs 13.5 ms, C5 29.2 vs
// 23.6 ms, at the same test RMSE.)
__host__ __device__ inline Philox4 sr_expand(const Philox4& base, uint32_t tag) {
  Philox4 r;
  const uint32_t tg = tag * 0x9E3779B9u;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint32_t x = (base.v[k] ^ tg) * 0x85EBCA6Bu;
    r.v[k] = x ^ (x >> 16);
  }
  return r;
}

// Two fp32 values -> packed bf16x2 with stochastic rounding, one sm_100a
// instruction: each value gets 16 random bits added below the bf16 mantissa
// and is truncated, so its magnitude rounds up with probability equal to the
// discarded fraction.  The lower half comes from `lo` with the lower 16 bits
// of `rbits`, the upper half from `hi` with the upper 16 (measured on B200:
// identical, for finite values, to (bits(x) + r16) >> 16 per half).
__device__ __forceinline__ uint32_t bf16x2_sr(float lo, float hi, uint32_t rbits) {
  uint32_t d;
  asm("cvt.rs.satfinite.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
  return d;
}

// a - b on packed bf16x2, rounded to nearest (the exact difference when the
// two values lie a few ulps apart)
__device__ __forceinline__ uint32_t bf16x2_sub(uint32_t a, uint32_t b) {
  uint32_t d;
  asm("sub.rn.bf16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}

// One sub-epoch segment: the records of block (id, schedule[s][id]).
struct Segment {
  uint64_t rec_begin;    // first record of the block in the record arrays
  uint32_t count;        // records in the block
  uint32_t chunk_begin;  // exclusive prefix of chunks over the sub-epoch's segments
  float cwh;             // lazy L2 scale of w.h   (sigma_W * sigma_H)
  float rho_w;           // sigma_H / sigma_W
  float rho_h;           // sigma_W / sigma_H
  uint32_t col_block;    // b2
  double eps;            // step size of the segment's problem
};

// One Hogwild launch: segments [seg_begin, seg_begin + nseg) of the segment
// array (entry nseg holds the chunk total) and its work counter.
struct LaunchDesc {
  uint64_t seg_begin;
  uint32_t nseg;
  uint32_t counter;
};

}  // namespace dsgdpp
