// mfdblock.cc -- the drop-in for tools/mfdblock.cc: splits a MatrixMarket
// matrix into blocks1 x blocks2 blocks at the default block offsets
// (computeDefaultBlockOffsets, mf/matrix/distributed_matrix_impl.cc:24-40)
// and writes one file per block plus the .xml descriptor that mfdsgdpp and
// mfdsgd read (BlockedMatrixFileDescriptor, mf/matrix/io/descriptor_impl.cc).
//
//   mfdblock [options] <input-file> <output-base-file>
//     --blocks1 N   row blocks (1)        --blocks2 N   column blocks (1)
//     --threads N   block writers (1)     --format F    block format ("": mmc
//                                                       for a sparse matrix,
//                                                       mma for a dense one)
//
// A sparse matrix (.mmc, or an .xml of .mmc blocks) is blocked as the
// reference's loader blocks it (ReadMatrixBlocksMm, mf/matrix/io/read_impl.h:
// 364-486): each block's entries sorted by (i, j), duplicates summed in file
// order, written as .mmc with block-local coordinates.  A dense matrix (.mma,
// or an .xml of .mma blocks) is written as .mma blocks.  Blocks are named
// <base>-<b1>-<b2>.<ext> in the output directory; the descriptor
// <output-base-file>.xml is saved with an empty path, as the reference saves
// it (tools/mfdblock.cc:88-90), so a reader resolves the block names against
// its own working directory.  Binary block formats are not written here.
#include <algorithm>
#include <cstdint>
#include <iostream>
#include <map>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dsgdpp.h"
#include "mmio.h"

using namespace dsgdpp;

namespace {

void usage() {
  std::cout << "mfdblock [options] <input-file> <output-base-file>\n\n"
            << "Options:\n"
            << "  --help                produce help message\n"
            << "  --blocks1 arg (=1)    number of row blocks\n"
            << "  --blocks2 arg (=1)    number of column blocks\n"
            << "  --threads arg (=1)    number of threads per node\n"
            << "  --format arg          file format of blocks (default: one of the matrix market\n"
            << "                        formats)\n"
            << "  --input-file arg      input file\n"
            << "  --output-base-file arg output file (no ending)\n"
            << std::endl;
}

std::vector<uint64_t> offsets(uint64_t size, uint64_t blocks) {
  std::vector<uint64_t> o(blocks);
  dsgdpp_block_offsets(size, (uint32_t)blocks, o.data());
  return o;
}

// end of block b of a dimension of `size` split at `off`
uint64_t block_end(const std::vector<uint64_t>& off, uint64_t b, uint64_t size) {
  return b + 1 < off.size() ? off[b + 1] : size;
}

size_t block_of(const std::vector<uint64_t>& off, uint64_t x) {
  return (size_t)(std::upper_bound(off.begin(), off.end(), x) - off.begin() - 1);
}

// Runs f(k) for k < count on `threads` threads, blocks dealt in turn.
template <typename F>
void for_blocks(size_t count, unsigned threads, F&& f) {
  threads = std::max(1u, std::min<unsigned>(threads, (unsigned)std::max<size_t>(1, count)));
  if (threads == 1) {
    for (size_t k = 0; k < count; ++k) f(k);
    return;
  }
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < threads; ++t)
    pool.emplace_back([&, t]() {
      for (size_t k = t; k < count; k += threads) f(k);
    });
  for (auto& th : pool) th.join();
}

// The blocks of a sparse matrix, row-major: block-local coordinates, each
// block sorted by (i, j) with the values of equal coordinates summed in the
// order the entries came.
std::vector<Coo> block_sparse(const Coo& m, const std::vector<uint64_t>& o1,
                              const std::vector<uint64_t>& o2, unsigned threads) {
  const size_t b1n = o1.size(), b2n = o2.size(), nb = b1n * b2n, nnz = m.vals.size();
  std::vector<uint32_t> blk(nnz);
  std::vector<uint64_t> start(nb + 1, 0);
  for (size_t k = 0; k < nnz; ++k) {
    blk[k] = (uint32_t)(block_of(o1, m.rows[k]) * b2n + block_of(o2, m.cols[k]));
    ++start[blk[k] + 1];
  }
  std::partial_sum(start.begin(), start.end(), start.begin());
  std::vector<uint64_t> fill(start.begin(), start.end() - 1), order(nnz);
  for (size_t k = 0; k < nnz; ++k) order[fill[blk[k]]++] = k;  // stable: file order per block
  std::vector<Coo> out(nb);
  for_blocks(nb, threads, [&](size_t b) {
    const size_t i = b / b2n, j = b % b2n;
    Coo& c = out[b];
    c.size1 = block_end(o1, i, m.size1) - o1[i];
    c.size2 = block_end(o2, j, m.size2) - o2[j];
    std::vector<uint64_t> idx(order.begin() + start[b], order.begin() + start[b + 1]);
    std::stable_sort(idx.begin(), idx.end(), [&](uint64_t x, uint64_t y) {
      return m.rows[x] != m.rows[y] ? m.rows[x] < m.rows[y] : m.cols[x] < m.cols[y];
    });
    for (size_t t = 0; t < idx.size(); ++t) {
      const uint64_t k = idx[t];
      if (t > 0 && m.rows[k] == m.rows[idx[t - 1]] && m.cols[k] == m.cols[idx[t - 1]]) {
        c.vals.back() += m.vals[k];
        continue;
      }
      c.rows.push_back((uint32_t)(m.rows[k] - o1[i]));
      c.cols.push_back((uint32_t)(m.cols[k] - o2[j]));
      c.vals.push_back(m.vals[k]);
    }
  });
  return out;
}

// The blocks of a dense matrix, row-major, each column by column.
std::vector<Dense> block_dense(const Dense& m, const std::vector<uint64_t>& o1,
                               const std::vector<uint64_t>& o2) {
  const size_t b1n = o1.size(), b2n = o2.size();
  std::vector<Dense> out(b1n * b2n);
  for (size_t i = 0; i < b1n; ++i)
    for (size_t j = 0; j < b2n; ++j) {
      Dense& d = out[i * b2n + j];
      d.size1 = block_end(o1, i, m.size1) - o1[i];
      d.size2 = block_end(o2, j, m.size2) - o2[j];
      d.colmajor.resize(d.size1 * d.size2);
      for (uint64_t c = 0; c < d.size2; ++c)
        for (uint64_t r = 0; r < d.size1; ++r)
          d.colmajor[c * d.size1 + r] = m.colmajor[(o2[j] + c) * m.size1 + o1[i] + r];
    }
  return out;
}

}  // namespace

int main(int argc, char** argv) {
  std::map<std::string, std::string> vm;
  std::vector<std::string> positional;
  const std::vector<std::string> known = {"help", "blocks1", "blocks2", "threads",
                                          "format", "input-file", "output-base-file"};
  for (int k = 1; k < argc; ++k) {
    std::string a = argv[k];
    if (a.rfind("--", 0) != 0) {
      positional.push_back(a);
      continue;
    }
    std::string key = a.substr(2), val;
    const size_t eq = key.find('=');
    if (eq != std::string::npos) {
      val = key.substr(eq + 1);
      key = key.substr(0, eq);
    } else if (key != "help") {
      if (k + 1 >= argc) {
        std::cerr << "the required argument for option '--" << key << "' is missing" << std::endl;
        return 1;
      }
      val = argv[++k];
    }
    if (std::find(known.begin(), known.end(), key) == known.end()) {
      std::cerr << "unrecognised option '--" << key << "'" << std::endl;
      return 1;
    }
    vm[key] = val;
  }
  if (positional.size() > 0 && !vm.count("input-file")) vm["input-file"] = positional[0];
  if (positional.size() > 1 && !vm.count("output-base-file")) vm["output-base-file"] = positional[1];
  if (vm.count("help") || !vm.count("input-file") || !vm.count("output-base-file")) {
    usage();
    return 1;
  }
  try {
    auto count = [&](const char* key) -> uint64_t {
      if (!vm.count(key)) return 1;
      const std::string& t = vm[key];
      size_t used = 0;
      unsigned long long v = 0;
      try {
        v = std::stoull(t, &used);
      } catch (const std::exception&) {
        used = 0;
      }
      if (used != t.size() || t.empty() || t[0] == '-' || v == 0)
        throw std::invalid_argument(std::string("invalid value for --") + key + ": " + t);
      return v;
    };
    const uint64_t blocks1 = count("blocks1"), blocks2 = count("blocks2");
    if (blocks1 > (1u << 24) || blocks2 > (1u << 24) || blocks1 * blocks2 > (1u << 24))
      throw std::invalid_argument("at most 2^24 blocks");
    const unsigned threads = (unsigned)std::min<uint64_t>(count("threads"), 1024);
    const std::string in = vm["input-file"], outBase = vm["output-base-file"];
    const std::string format = vm.count("format") ? vm["format"] : "";
    const size_t slash = outBase.find_last_of('/');
    const std::string outFile = slash == std::string::npos ? outBase : outBase.substr(slash + 1);
    std::string outDir = slash == std::string::npos ? "" : outBase.substr(0, slash);
    if (!outDir.empty()) outDir += "/";
    std::cout << "Input file        : " << in << "\n"
              << "Output directory  : " << outDir << "\n"
              << "Output file       : " << outFile << ".xml (+ blocks)\n"
              << "Output format     : " << (format.empty() ? "AUTOMATIC" : format) << "\n"
              << "Blocks            : " << blocks1 << "x" << blocks2 << "\n"
              << "Threads@nodes     : " << threads << "@1\n\n";

    // sparse or dense, from the extension (or the descriptor's block format)
    std::string kind;
    if (ends_with(in, ".mmc")) kind = "mmc";
    else if (ends_with(in, ".mma")) kind = "mma";
    else if (ends_with(in, ".xml")) kind = read_descriptor(in).format;
    if (kind != "mmc" && kind != "mma")
      throw std::invalid_argument("unsupported input file " + in +
                                  " (a .mmc or .mma file, or an .xml of .mmc or .mma blocks)");
    if (!format.empty() && format != kind)
      throw std::invalid_argument("unsupported block format " + format + ": a " +
                                  (kind == "mmc" ? "sparse" : "dense") +
                                  " matrix is written in " + kind + " blocks");

    BlockedDescriptor desc;
    desc.blocks1 = blocks1;
    desc.blocks2 = blocks2;
    desc.format = kind;
    for (uint64_t i = 0; i < blocks1; ++i)
      for (uint64_t j = 0; j < blocks2; ++j)
        desc.filenames.push_back(outFile + "-" + std::to_string(i) + "-" + std::to_string(j) +
                                 "." + kind);
    std::cout << "Reading " << in << "... " << std::endl << std::endl;
    if (kind == "mmc") {
      const Coo m = read_sparse(in);
      desc.size1 = m.size1;
      desc.size2 = m.size2;
      desc.offsets1 = offsets(m.size1, blocks1);
      desc.offsets2 = offsets(m.size2, blocks2);
      std::cout << "Writing blocks ... " << std::endl;
      const std::vector<Coo> blocks = block_sparse(m, desc.offsets1, desc.offsets2, threads);
      for_blocks(blocks.size(), threads,
                 [&](size_t b) { write_mm_coord(outDir + desc.filenames[b], blocks[b]); });
    } else {
      const Dense m = read_dense(in);
      desc.size1 = m.size1;
      desc.size2 = m.size2;
      desc.offsets1 = offsets(m.size1, blocks1);
      desc.offsets2 = offsets(m.size2, blocks2);
      std::cout << "Writing blocks ... " << std::endl;
      const std::vector<Dense> blocks = block_dense(m, desc.offsets1, desc.offsets2);
      for_blocks(blocks.size(), threads,
                 [&](size_t b) { write_mm_array(outDir + desc.filenames[b], blocks[b]); });
    }
    desc.path = "";  // as the reference saves it: block names relative to the reader
    write_descriptor(outDir + outFile + ".xml", desc);
  } catch (const std::exception& e) {
    std::cerr << "mfdblock: " << e.what() << std::endl;
    return 1;
  }
  return 0;
}
