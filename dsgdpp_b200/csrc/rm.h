// rm.h -- random-matrix descriptors (.rm) and the generator that turns them
// into data and factor matrices on the device.
//
// The reference generates synthetic matrices on the fly from an XML
// descriptor (mf/matrix/io/randomMatrixDescriptor.h, _impl.cc:21-113): sizes,
// a chunks1 x chunks2 grid, the rank and two distribution specs, one seed per
// row chunk of the original W, per column chunk of the original H, per chunk
// of the data matrix V and of the test matrix, and the nonzeros per chunk.
// getDataMatrices / getFactors (generateDistributedMatrix_impl.h:655-744)
// accept such a file wherever a matrix file is expected.  V is a sample of
// chunk cells of Worig * Horig plus noise; the test matrix the same from its
// own seeds without noise (generateDistributedMatrix_impl.h:127-175,615-647);
// factors read from a descriptor are Worig and Horig themselves (:598-613).
//
// The descriptor format, the chunk grid (computeDefaultBlockOffsets), the
// nonzeros per chunk and the value model are the reference's.  The random
// draws are not: the reference walks one Mersenne-Twister stream per chunk
// through rg::skipSequential and Boost distributions (unpinned versions),
// a sequential process.  Here every draw is a counter-based value, so each
// nonzero is generated by its own thread:
//   * stream(key, n) = SplitMix64 output n of state `key` (Steele, Lea and
//     Flood, OOPSLA 2014): mix64(key + (n + 1) * 0x9e3779b97f4a7c15);
//   * key(seed, tag) = mix64(tag << 32 | seed), tags below;
//   * the cells of a chunk with N cells and k nonzeros are the images of
//     0..k-1 under a pseudo-random permutation of [0, N): a 4-round Feistel
//     network on 2h bits (2^(2h) >= N) with round keys stream(key, r) and
//     round function mix64(R ^ round key), restricted to [0, N) by cycle
//     walking (Black and Rogaway, CT-RSA 2002) -- k distinct cells, exactly;
//   * Uniform(a, b): a + (b - a) * u, u = (x >> 11) * 2^-53;
//     Normal(mean, s): s * sqrt(-2 log u1) * cos(2 pi u2) (Box-Muller) with
//     u1 = 1 - u, the mean ignored as the reference ignores it
//     (tools/parse.h:80-88);
//   * Worig[i][z] (row chunk b): value draw n = (i - offset_b) * rank + z of
//     key(seedsWorig[b], kTagW); Horig the same per column chunk (kTagH);
//   * V[i][j] = sum over z of Worig[i][z] * Horig[j][z] (in z order, no
//     fused multiply-add) plus the noise draw n = local cell of the chunk
//     (key(seed of the chunk, kTagNoise)).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace dsgdpp {

enum RmTag : uint32_t { kTagW = 1, kTagH = 2, kTagCells = 3, kTagNoise = 4 };

// Normal(mean, stddev) or Uniform(min, max) (tools/parse.h:75-110)
struct RmDist {
  int kind = -1;  // -1 none, 0 Normal, 1 Uniform
  double a = 0, b = 0;
};
RmDist parse_dist(const std::string& arg_name, const std::string& spec);

struct RmDesc {
  uint64_t size1 = 0, size2 = 0, rank = 0, chunks1 = 0, chunks2 = 0, nnz = 0, nnz_test = 0;
  std::string values, noise;
  std::vector<uint32_t> seeds_w, seeds_h;          // chunks1, chunks2
  std::vector<uint32_t> seeds_v, seeds_vtest;      // chunks1 x chunks2, row-major
  std::vector<uint64_t> nnz_v, nnz_vtest;          // empty when the file has no data part
  bool has_data() const { return !nnz_v.empty(); }
};

// Reads / writes the property_tree XML of randomMatrixDescriptor_impl.cc:21-113.
RmDesc rm_load(const std::string& path);
void rm_save(const std::string& path, const RmDesc& d);
// RandomMatrixDescriptor::create (randomMatrixDescriptor.h:27-77): seeds
// from one generator seeded 123 in the reference's order; nonzeros per chunk
// split off one chunk at a time, each a binomial draw of the remaining count
// with probability 1 / (chunks left) from the chunk's V seed, as the reference
// does (randomMatrixDescriptor_impl.cc:115-176) but with this file's own
// binomial sampler.
RmDesc rm_create(uint64_t size1, uint64_t size2, uint64_t chunks1, uint64_t chunks2,
                 uint64_t nnz, uint64_t nnz_test, uint64_t rank, const std::string& values,
                 const std::string& noise);
// Checks sizes, grid and counts; throws MmError.
void rm_validate(const RmDesc& d);

}  // namespace dsgdpp
