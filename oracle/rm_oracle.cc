// rm_oracle.cc -- TEST INFRASTRUCTURE ONLY: CPU restatement of the .rm
// generator (parity checker for dsgdpp_b200's device generation; never part
// of the product path).
//
// Follows the generation model of the reference (Worig and Horig per chunk,
// V = sampled cells of Worig * Horig plus noise, the test matrix without
// noise: mf/matrix/io/generateDistributedMatrix_impl.h:94-175,598-647) with
// the library's own counter-based draws, restated here from their published
// definitions: SplitMix64 (Steele, Lea, Flood, OOPSLA 2014), a 4-round Feistel
// permutation with cycle walking (Black, Rogaway, CT-RSA 2002), Box-Muller.
// The reference's own draws (rg::skipSequential, Boost distributions) are in
// unvendored, unpinned libraries: parity with them is unpinned.
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

const uint64_t kGolden = 0x9e3779b97f4a7c15ull;

uint64_t mix(uint64_t z) {
  z ^= z >> 30;
  z *= 0xbf58476d1ce4e5b9ull;
  z ^= z >> 27;
  z *= 0x94d049bb133111ebull;
  z ^= z >> 31;
  return z;
}

uint64_t nth(uint64_t state, uint64_t n) { return mix(state + kGolden * (n + 1)); }

uint64_t key_of(uint32_t seed, uint32_t tag) { return mix((uint64_t(tag) << 32) | seed); }

double unit(uint64_t x) { return double(x >> 11) / 9007199254740992.0; }  // 2^53

double value(int kind, double a, double b, uint64_t key, uint64_t n) {
  double u = unit(nth(key, 2 * n));
  if (kind == 1) return a + (b - a) * u;
  double u1 = 1.0 - u;
  double u2 = unit(nth(key, 2 * n + 1));
  return b * (std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2));
}

// computeDefaultBlockOffsets (mf/matrix/distributed_matrix_impl.cc:24-40),
// with the size appended
std::vector<uint64_t> offsets(uint64_t size, uint64_t blocks) {
  std::vector<uint64_t> o;
  uint64_t q = size / blocks, extra = size % blocks, at = 0;
  for (uint64_t b = 0; b < blocks; b++) {
    o.push_back(at);
    at += q + (b < extra ? 1 : 0);
  }
  o.push_back(size);
  return o;
}

// image of t under the chunk's permutation of [0, N)
uint64_t cell(uint64_t key, uint64_t N, uint64_t t) {
  int bits = 1;
  if (N > 1) {
    bits = 0;
    for (uint64_t v = N - 1; v; v >>= 1) bits++;
  }
  int h = (bits + 1) / 2;
  if (h < 1) h = 1;
  uint64_t mask = h >= 64 ? ~0ull : ((1ull << h) - 1);
  uint64_t rk[4];
  for (int r = 0; r < 4; r++) rk[r] = nth(key, r);
  uint64_t x = t;
  for (;;) {
    uint64_t L = x >> h, R = x & mask;
    for (int r = 0; r < 4; r++) {
      uint64_t nr = L ^ (mix(R ^ rk[r]) & mask);
      L = R;
      R = nr;
    }
    x = (L << h) | R;
    if (x < N) return x;
  }
}

}  // namespace

extern "C" {

// Worig (tag 1) or Horig (tag 2): rows x rank, row-major
void orc_rm_factor(int kind, double a, double b, const uint32_t* seeds, uint64_t chunks,
                   uint64_t rows, uint32_t rank, uint32_t tag, double* out) {
  std::vector<uint64_t> o = offsets(rows, chunks);
  for (uint64_t c = 0; c < chunks; c++) {
    uint64_t key = key_of(seeds[c], tag);
    for (uint64_t i = o[c]; i < o[c + 1]; i++)
      for (uint32_t z = 0; z < rank; z++)
        out[i * rank + z] = value(kind, a, b, key, (i - o[c]) * rank + z);
  }
}

// data (noise_kind >= 0) or test (noise_kind = -1) matrix, chunk by chunk;
// returns the number of entries written
uint64_t orc_rm_data(int noise_kind, double na, double nb, const uint32_t* seeds,
                     const uint64_t* counts, uint64_t c1, uint64_t c2, uint64_t size1,
                     uint64_t size2, const double* W, const double* H, uint32_t rank,
                     uint32_t* rows, uint32_t* cols, double* vals) {
  std::vector<uint64_t> o1 = offsets(size1, c1), o2 = offsets(size2, c2);
  uint64_t k = 0;
  for (uint64_t b1 = 0; b1 < c1; b1++)
    for (uint64_t b2 = 0; b2 < c2; b2++) {
      uint64_t ch = b1 * c2 + b2;
      uint64_t nc = o2[b2 + 1] - o2[b2];
      uint64_t N = (o1[b1 + 1] - o1[b1]) * nc;
      uint64_t kc = key_of(seeds[ch], 3), kn = key_of(seeds[ch], 4);
      for (uint64_t t = 0; t < counts[ch]; t++, k++) {
        uint64_t x = cell(kc, N, t);
        uint64_t i = o1[b1] + x / nc, j = o2[b2] + x % nc;
        double v = 0.0;
        for (uint32_t z = 0; z < rank; z++) v = v + W[i * rank + z] * H[j * rank + z];
        if (noise_kind >= 0) v = v + value(noise_kind, na, nb, kn, x);
        rows[k] = (uint32_t)i;
        cols[k] = (uint32_t)j;
        vals[k] = v;
      }
    }
  return k;
}

}  // extern "C"
