// rm.cc -- .rm descriptor I/O and creation (host side of the generator).
#include "rm.h"

#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <sstream>

#include "mmio.h"
#include "schedule.h"

namespace dsgdpp {

namespace {

std::string trim(const std::string& t) {
  size_t a = t.find_first_not_of(" \t\r\n"), b = t.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? std::string() : t.substr(a, b - a + 1);
}

uint64_t rm_u64(const std::string& t, const std::string& what) {
  char* q = nullptr;
  errno = 0;
  const std::string s = trim(t);
  unsigned long long v = std::strtoull(s.c_str(), &q, 10);
  if (s.empty() || *q || errno || s[0] == '-') throw MmError("bad number in random matrix descriptor (" + what + "): " + t);
  return v;
}

const XmlNode& rm_need(const std::vector<XmlNode>& top, const std::string& name) {
  for (auto& n : top)
    if (n.name == name) return n;
  throw MmError("random matrix descriptor lacks " + name);
}

const XmlNode& rm_need(const XmlNode& n, const std::string& name) {
  const XmlNode* c = n.child(name);
  if (!c) throw MmError("random matrix descriptor lacks " + n.name + "." + name);
  return *c;
}

// uniform on [0, 1) from two raw draws (53 bits)
double uniform53(Random32& rng) {
  const uint64_t hi = rng.next() >> 5, lo = rng.next() >> 6;  // 27 + 26 bits
  return (double)((hi << 26) | lo) * 0x1.0p-53;
}

// Binomial(n, p): inversion for small means, else the normal approximation
// rounded and clamped (own sampler; the reference calls Boost's).
uint64_t binomial(uint64_t n, double p, Random32& rng) {
  if (n == 0 || p <= 0) return 0;
  if (p >= 1) return n;
  const double mean = (double)n * p;
  if (mean < 30) {
    const double u = uniform53(rng);
    double prob = std::pow(1 - p, (double)n), cdf = prob;
    uint64_t k = 0;
    while (u > cdf && k < n) {
      prob *= (double)(n - k) / (double)(k + 1) * p / (1 - p);
      ++k;
      cdf += prob;
      if (prob == 0 && cdf < u) break;
    }
    return k;
  }
  const double u1 = 1 - uniform53(rng), u2 = uniform53(rng);
  const double z = std::sqrt(-2 * std::log(u1)) * std::cos(2 * M_PI * u2);
  const double k = std::floor(mean + z * std::sqrt(mean * (1 - p)) + 0.5);
  if (k <= 0) return 0;
  if (k >= (double)n) return n;
  return (uint64_t)k;
}

// RandomMatrixDescriptor::calculateNnzPerBlock (randomMatrixDescriptor_impl.cc:115-176):
// chunk (i, j) takes a binomial share of what is left with probability
// 1 / (chunks left), from a generator seeded with that chunk's V seed.
std::vector<uint64_t> split_nnz(uint64_t nnz, uint64_t c1, uint64_t c2,
                                const std::vector<uint32_t>& seeds_v) {
  std::vector<uint64_t> out(c1 * c2);
  uint64_t left = nnz, done = 0;
  for (uint64_t k = 0; k < c1 * c2; ++k, ++done) {
    Random32 rng(seeds_v[k]);
    const double p = 1.0 / (double)(c1 * c2 - done);
    out[k] = binomial(left, p, rng);
    left -= out[k];
  }
  return out;
}

}  // namespace

RmDist parse_dist(const std::string& arg_name, const std::string& spec) {
  // parse::parseArg + parseDistribution (tools/parse.h:38-110)
  RmDist d;
  const std::string s = trim(spec);
  const size_t lp = s.find('('), rp = s.rfind(')');
  std::string name = trim(s.substr(0, lp));
  std::vector<std::string> args;
  bool ok = lp != std::string::npos && rp == s.size() - 1 && rp > lp;
  if (ok) {
    std::string inner = s.substr(lp + 1, rp - lp - 1);
    size_t a = 0;
    for (;;) {
      size_t c = inner.find(',', a);
      args.push_back(trim(inner.substr(a, c == std::string::npos ? std::string::npos : c - a)));
      if (c == std::string::npos) break;
      a = c + 1;
    }
  }
  auto num = [&](const std::string& t, double& v) {
    char* q = nullptr;
    errno = 0;
    v = std::strtod(t.c_str(), &q);
    return !t.empty() && !*q && !errno;
  };
  if (ok && args.size() == 2 && (name == "Normal" || name == "Uniform") && num(args[0], d.a) &&
      num(args[1], d.b)) {
    d.kind = name == "Normal" ? 0 : 1;
    return d;
  }
  throw MmError("Error in argument '" + arg_name + "': Unknown or invalid distribution '" + spec +
                "'. Valid choices are: Normal(<mean>,<stddev>), Uniform(<min>,<max>)");
}

void rm_validate(const RmDesc& d) {
  if (d.size1 == 0 || d.size2 == 0 || d.size1 >= (1ull << 32) || d.size2 >= (1ull << 32))
    throw MmError("random matrix descriptor: sizes must lie in [1, 2^32)");
  if (d.rank == 0 || d.rank > 4096) throw MmError("random matrix descriptor: rank must lie in [1, 4096]");
  if (d.chunks1 == 0 || d.chunks2 == 0 || d.chunks1 > d.size1 || d.chunks2 > d.size2)
    throw MmError("random matrix descriptor: blocks1/blocks2 must lie in [1, size]");
  if (d.chunks1 * d.chunks2 >= (1ull << 31))
    throw MmError("random matrix descriptor: blocks1 x blocks2 must stay below 2^31");
  if (d.seeds_w.size() != d.chunks1 || d.seeds_h.size() != d.chunks2)
    throw MmError("random matrix descriptor: one Worig seed per row block and one Horig seed per column block are required");
  parse_dist("values", d.values);
  if (!d.has_data()) return;
  const uint64_t nc = d.chunks1 * d.chunks2;
  if (d.seeds_v.size() != nc || d.seeds_vtest.size() != nc || d.nnz_v.size() != nc ||
      d.nnz_vtest.size() != nc)
    throw MmError("random matrix descriptor: V and Vtest need one seed and one count per block");
  if (!trim(d.noise).empty()) parse_dist("noise", d.noise);
  const auto o1 = block_offsets(d.size1, (uint32_t)d.chunks1);
  const auto o2 = block_offsets(d.size2, (uint32_t)d.chunks2);
  for (uint64_t b1 = 0; b1 < d.chunks1; ++b1)
    for (uint64_t b2 = 0; b2 < d.chunks2; ++b2) {
      const uint64_t r = (b1 + 1 < d.chunks1 ? o1[b1 + 1] : d.size1) - o1[b1];
      const uint64_t c = (b2 + 1 < d.chunks2 ? o2[b2 + 1] : d.size2) - o2[b2];
      const uint64_t k = b1 * d.chunks2 + b2;
      if (d.nnz_v[k] > r * c || d.nnz_vtest[k] > r * c)
        throw MmError("nnz must be less than matrix size");  // mf/matrix/op/generate.h:258
    }
}

RmDesc rm_load(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f.is_open()) throw MmError("Cannot open file " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  const std::vector<XmlNode> top = parse_xml(ss.str());
  RmDesc d;
  d.size1 = rm_u64(rm_need(top, "size1").text, "size1");
  d.size2 = rm_u64(rm_need(top, "size2").text, "size2");
  d.chunks1 = rm_u64(rm_need(top, "blocks1").text, "blocks1");
  d.chunks2 = rm_u64(rm_need(top, "blocks2").text, "blocks2");
  d.nnz = rm_u64(rm_need(top, "nnz").text, "nnz");
  d.nnz_test = rm_u64(rm_need(top, "nnzTest").text, "nnzTest");
  d.values = rm_need(top, "values").text;
  d.noise = rm_need(top, "noise").text;
  d.rank = rm_u64(rm_need(top, "rank").text, "rank");
  for (auto& k : rm_need(top, "Worig").kids) d.seeds_w.push_back((uint32_t)rm_u64(k.text, "Worig"));
  for (auto& k : rm_need(top, "Horig").kids) d.seeds_h.push_back((uint32_t)rm_u64(k.text, "Horig"));
  if (d.nnz != 0 && d.nnz_test != 0) {  // randomMatrixDescriptor_impl.cc:46-91
    const XmlNode& v = rm_need(top, "V");
    const XmlNode& t = rm_need(top, "Vtest");
    for (auto& k : rm_need(v, "seeds").kids) d.seeds_v.push_back((uint32_t)rm_u64(k.text, "V.seeds"));
    for (auto& k : rm_need(v, "nnzs").kids) d.nnz_v.push_back(rm_u64(k.text, "V.nnzs"));
    for (auto& k : rm_need(t, "seeds").kids) d.seeds_vtest.push_back((uint32_t)rm_u64(k.text, "Vtest.seeds"));
    for (auto& k : rm_need(t, "nnzs").kids) d.nnz_vtest.push_back(rm_u64(k.text, "Vtest.nnzs"));
  }
  rm_validate(d);
  return d;
}

void rm_save(const std::string& path, const RmDesc& d) {
  // the layout property_tree's write_xml gives with 4-space indentation
  std::ostringstream o;
  o << "<?xml version=\"1.0\" encoding=\"utf-8\"?>\n";
  o << "<size1>" << d.size1 << "</size1>\n<size2>" << d.size2 << "</size2>\n";
  o << "<blocks1>" << d.chunks1 << "</blocks1>\n<blocks2>" << d.chunks2 << "</blocks2>\n";
  o << "<nnz>" << d.nnz << "</nnz>\n<nnzTest>" << d.nnz_test << "</nnzTest>\n";
  o << "<values>" << d.values << "</values>\n<noise>" << d.noise << "</noise>\n";
  o << "<rank>" << d.rank << "</rank>\n<Worig>\n";
  for (uint32_t s : d.seeds_w) o << "    <seed>" << s << "</seed>\n";
  o << "</Worig>\n<Horig>\n";
  for (uint32_t s : d.seeds_h) o << "    <seed>" << s << "</seed>\n";
  o << "</Horig>\n";
  if (d.has_data()) {
    const char* names[2] = {"V", "Vtest"};
    const std::vector<uint32_t>* seeds[2] = {&d.seeds_v, &d.seeds_vtest};
    const std::vector<uint64_t>* counts[2] = {&d.nnz_v, &d.nnz_vtest};
    for (int w = 0; w < 2; ++w) {
      o << "<" << names[w] << ">\n    <seeds>\n";
      for (uint32_t s : *seeds[w]) o << "        <seed>" << s << "</seed>\n";
      o << "    </seeds>\n    <nnzs>\n";
      for (uint64_t c : *counts[w]) o << "        <nnz>" << c << "</nnz>\n";
      o << "    </nnzs>\n</" << names[w] << ">\n";
    }
  }
  std::ofstream f(path, std::ios::binary);
  if (!f.is_open()) throw MmError("Cannot open file " + path);
  const std::string s = o.str();
  f.write(s.data(), (std::streamsize)s.size());
  if (!f) throw MmError("Cannot write file " + path);
}

RmDesc rm_create(uint64_t size1, uint64_t size2, uint64_t chunks1, uint64_t chunks2,
                 uint64_t nnz, uint64_t nnz_test, uint64_t rank, const std::string& values,
                 const std::string& noise) {
  if (chunks1 == 0 || chunks2 == 0 || size1 % chunks1 != 0 || size2 % chunks2 != 0)
    throw MmError("size1 and size2 must be multiples of blocks1 and blocks2");  // randomMatrixDescriptor.h:31-32
  RmDesc d;
  d.size1 = size1; d.size2 = size2; d.chunks1 = chunks1; d.chunks2 = chunks2;
  d.nnz = nnz; d.nnz_test = nnz_test; d.rank = rank; d.values = values; d.noise = noise;
  Random32 rng(123);  // randomMatrixDescriptor.h:36
  d.seeds_v.assign(chunks1 * chunks2, 0);
  d.seeds_vtest.assign(chunks1 * chunks2, 0);
  for (uint64_t b1 = 0; b1 < chunks1; ++b1) {  // randomMatrixDescriptor.h:54-68
    d.seeds_w.push_back(rng.next());
    for (uint64_t b2 = 0; b2 < chunks2; ++b2) {
      if (b1 == 0) d.seeds_h.push_back(rng.next());
      d.seeds_v[b1 * chunks2 + b2] = rng.next();
      d.seeds_vtest[b1 * chunks2 + b2] = rng.next();
    }
  }
  if (nnz != 0 && nnz_test != 0) {
    // both counts are split with the V seeds (randomMatrixDescriptor_impl.cc:145,163)
    d.nnz_v = split_nnz(nnz, chunks1, chunks2, d.seeds_v);
    d.nnz_vtest = split_nnz(nnz_test, chunks1, chunks2, d.seeds_v);
  } else {
    d.seeds_v.clear();
    d.seeds_vtest.clear();
  }
  rm_validate(d);
  return d;
}

}  // namespace dsgdpp
