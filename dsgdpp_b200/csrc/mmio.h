// mmio.h -- MatrixMarket (.mmc/.mma) and blocked-matrix descriptor (.xml) I/O.
//
// Formats of the reference (drop-in):
//  * .mmc  "%%MatrixMarket matrix coordinate real general", 1-based
//          coordinates (mf/matrix/io/read_impl.h:45-116, write_impl.h:42-88);
//  * .mma  "%%MatrixMarket matrix array real general", entries listed column
//          by column (read_impl.h:194-256, write_impl.h:92-118); written with
//          16 significant digits (write_impl.h:98);
//  * .xml  BlockedMatrixFileDescriptor (mf/matrix/io/descriptor_impl.cc:25-75):
//          <matrix> with size1, size2, blocks1, blocks2, blockOffsets1/offset,
//          blockOffsets2/offset, path, filenames/filename (row-major blocks),
//          format; each block file holds block-local coordinates.
// Parse errors throw MmError with the reference's messages.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace dsgdpp {

struct MmError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

struct Coo {
  uint64_t size1 = 0, size2 = 0;
  std::vector<uint32_t> rows, cols;  // 0-based
  std::vector<double> vals;
};

struct Dense {
  uint64_t size1 = 0, size2 = 0;
  std::vector<double> colmajor;  // size1 * size2, column by column
};

struct BlockedDescriptor {
  uint64_t size1 = 0, size2 = 0, blocks1 = 0, blocks2 = 0;
  std::vector<uint64_t> offsets1, offsets2;
  std::string path, format;
  std::vector<std::string> filenames;  // blocks1 x blocks2, row-major
};

bool ends_with(const std::string& s, const std::string& suffix);

// Element tree of the small XML files the reference writes with Boost's
// property_tree (text trimmed, entities decoded, attributes ignored).
struct XmlNode {
  std::string name, text;
  std::vector<XmlNode> kids;
  const XmlNode* child(const std::string& n) const;
};
// top-level elements in file order (property_tree writes several roots)
std::vector<XmlNode> parse_xml(const std::string& text);

// Reads a coordinate file with several threads; entries keep file order.
Coo read_mm_coord(const std::string& path, unsigned threads = 0);
Dense read_mm_array(const std::string& path);
void write_mm_coord(const std::string& path, const Coo& m);
void write_mm_array(const std::string& path, const Dense& m);

BlockedDescriptor read_descriptor(const std::string& path);
void write_descriptor(const std::string& path, const BlockedDescriptor& d);

// A sparse matrix file: .mmc, or .xml whose blocks are .mmc files (block-local
// coordinates are shifted by the block offsets to global ones).
Coo read_sparse(const std::string& path, BlockedDescriptor* desc_out = nullptr);
// A dense matrix file: .mma, or .xml whose blocks are .mma files (each block
// placed at its offsets).
Dense read_dense(const std::string& path);

}  // namespace dsgdpp
