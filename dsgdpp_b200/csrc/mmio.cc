// mmio.cc -- see mmio.h.
#include "mmio.h"

#include "../../include/dsgdpp.h"

#include <algorithm>
#include <cerrno>
#include <charconv>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <thread>

namespace dsgdpp {

bool ends_with(const std::string& s, const std::string& suffix) {
  return s.size() > suffix.size() && s.compare(s.size() - suffix.size(), suffix.size(), suffix) == 0;
}

namespace {

std::string read_file(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in.is_open()) throw MmError("Cannot open file " + path);
  std::string s;
  in.seekg(0, std::ios::end);
  s.resize((size_t)in.tellg());
  in.seekg(0);
  in.read(&s[0], (std::streamsize)s.size());
  return s;
}

std::string rtrim(std::string s) {
  while (!s.empty() && std::isspace((unsigned char)s.back())) s.pop_back();
  return s;
}

bool blank(const char* a, const char* b) {
  for (; a < b; ++a)
    if (!std::isspace((unsigned char)*a)) return false;
  return true;
}

// Number fields of one line, parsed in place: std::from_chars for the usual
// forms, and strtoul / strtod on a copy of the token for anything it does not
// take (a leading '+', hexadecimal, out-of-range values), so every line reads
// exactly as with strtoul / strtod.
inline const char* skip_blanks(const char* p, const char* e) {
  while (p < e && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\v' || *p == '\f')) ++p;
  return p;
}
inline const char* token_end(const char* p, const char* e) {
  while (p < e && !std::isspace((unsigned char)*p)) ++p;
  return p;
}
bool field_u64(const char*& p, const char* e, unsigned long& v) {
  p = skip_blanks(p, e);
  const auto r = std::from_chars(p, e, v);
  if (r.ec == std::errc() && r.ptr != p && (r.ptr == e || std::isspace((unsigned char)*r.ptr))) {
    p = r.ptr;
    return true;
  }
  const char* te = token_end(p, e);
  if (te == p) return false;
  const std::string tok(p, te);
  char* q = nullptr;
  v = std::strtoul(tok.c_str(), &q, 10);
  if (q == tok.c_str()) return false;
  p += q - tok.c_str();
  return true;
}
bool field_f64(const char*& p, const char* e, double& x) {
  p = skip_blanks(p, e);
  const auto r = std::from_chars(p, e, x, std::chars_format::general);
  if (r.ec == std::errc() && r.ptr != p && (r.ptr == e || std::isspace((unsigned char)*r.ptr))) {
    p = r.ptr;
    return true;
  }
  const char* te = token_end(p, e);
  if (te == p) return false;
  const std::string tok(p, te);
  char* q = nullptr;
  x = std::strtod(tok.c_str(), &q);
  if (q == tok.c_str()) return false;
  p += q - tok.c_str();
  return true;
}

// Starts of the first `count` lines from byte `pos` on, found by several
// threads (each scans one byte range that begins right after a newline);
// *end gets the position after the last of them.  False if the text has
// fewer lines.
bool line_starts(const std::string& s, size_t pos, uint64_t count, std::vector<size_t>& out,
                 size_t* end) {
  out.clear();
  if (count == 0) {
    *end = pos;
    return true;
  }
  const size_t n = s.size() > pos ? s.size() - pos : 0;
  unsigned T = std::max(1u, std::thread::hardware_concurrency());
  if (n < (1u << 22)) T = 1;
  std::vector<size_t> cut(T + 1);
  cut[0] = pos;
  cut[T] = s.size();
  for (unsigned t = 1; t < T; ++t) {
    size_t c = pos + n * t / T;
    const void* nl = c < s.size() ? std::memchr(s.data() + c, '\n', s.size() - c) : nullptr;
    c = nl ? (size_t)(static_cast<const char*>(nl) - s.data()) + 1 : s.size();
    cut[t] = std::max(c, cut[t - 1]);
  }
  std::vector<std::vector<size_t>> parts(T);
  auto work = [&](unsigned t) {
    for (size_t p = cut[t]; p < cut[t + 1];) {
      parts[t].push_back(p);
      const void* nl = std::memchr(s.data() + p, '\n', cut[t + 1] - p);
      p = nl ? (size_t)(static_cast<const char*>(nl) - s.data()) + 1 : cut[t + 1];
    }
  };
  if (T == 1) {
    work(0);
  } else {
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < T; ++t) pool.emplace_back(work, t);
    for (auto& th : pool) th.join();
  }
  size_t total = 0;
  for (auto& p : parts) total += p.size();
  if (total < count) return false;
  out.reserve(count);
  for (auto& p : parts)
    for (size_t v : p) {
      if (out.size() == count) break;
      out.push_back(v);
    }
  if (total > count) {  // the start of the line after the last one taken
    uint64_t k = 0;
    for (auto& p : parts) {
      if (k + p.size() > count) {
        *end = p[count - k];
        return true;
      }
      k += p.size();
    }
  }
  *end = s.size();
  return true;
}

// Cursor over the lines of a text buffer.
struct Lines {
  const std::string& s;
  size_t pos = 0;
  uint64_t number = 0;
  explicit Lines(const std::string& s) : s(s) {}
  bool next(const char*& a, const char*& b) {
    if (pos >= s.size()) return false;
    size_t e = s.find('\n', pos);
    if (e == std::string::npos) e = s.size();
    a = s.data() + pos;
    b = s.data() + e;
    if (b > a && b[-1] == '\r') --b;
    pos = e + 1;
    ++number;
    return true;
  }
};

// Banner, comments and the size line (read_impl.h:53-80).
void read_header(Lines& L, const std::string& path, const char* banner, const char*& a,
                 const char*& b) {
  if (!L.next(a, b)) throw MmError("Unexpected EOF in file " + path);
  std::string line(a, b);
  if (rtrim(line) != banner) throw MmError("Wrong matrix-market banner in file " + path + ": " + line);
  for (;;) {
    if (!L.next(a, b)) throw MmError("Unexpected EOF in file " + path);
    if (a == b || *a != '%') break;
  }
}

}  // namespace

Coo read_mm_coord(const std::string& path, unsigned threads) {
  const std::string s = read_file(path);
  Lines L(s);
  const char *a, *b;
  read_header(L, path, "%%MatrixMarket matrix coordinate real general", a, b);
  std::string dims(a, b);
  long long s1 = 0, s2 = 0, nnz = 0;
  char junk[2] = {0, 0};
  int got = std::sscanf(dims.c_str(), "%lld %lld %lld %1s", &s1, &s2, &nnz, junk);
  if (got != 3 || s1 < 0 || s2 < 0 || nnz < 0)
    throw MmError("Invalid matrix dimensions in file " + path + ": " + dims);
  Coo m;
  m.size1 = (uint64_t)s1;
  m.size2 = (uint64_t)s2;
  m.rows.resize((size_t)nnz);
  m.cols.resize((size_t)nnz);
  m.vals.resize((size_t)nnz);
  // entry lines: find the start of each of the nnz lines, then parse in parallel
  std::vector<size_t> starts;
  size_t pos = 0;
  const uint64_t first_line = L.number + 1;
  if (!line_starts(s, L.pos, (uint64_t)nnz, starts, &pos))
    throw MmError("Unexpected EOF in file " + path);
  if (!blank(s.data() + std::min(pos, s.size()), s.data() + s.size())) {
    // locate the offending line for the message (read_impl.h:106-111)
    Lines R(s);
    R.pos = pos;
    R.number = first_line + nnz - 1;
    while (R.next(a, b))
      if (!blank(a, b))
        throw MmError("Unexpected input at at line " + std::to_string(R.number) + " of " + path +
                      ": " + std::string(a, b));
  }
  unsigned T = threads ? threads : std::max(1u, std::thread::hardware_concurrency());
  T = (unsigned)std::min<long long>(T, std::max<long long>(1, nnz / 100000));
  std::vector<std::string> errors(T);
  auto work = [&](unsigned t) {
    const size_t lo = (size_t)nnz * t / T, hi = (size_t)nnz * (t + 1) / T;
    for (size_t k = lo; k < hi; ++k) {
      const char* p = s.data() + starts[k];
      const char* end = s.data() + (k + 1 < starts.size() ? starts[k + 1] : pos);
      if (end > p && end[-1] == '\n') --end;
      if (end > p && end[-1] == '\r') --end;
      const char* q = p;
      unsigned long i = 0, j = 0;
      double x = 0;
      const bool bad = !field_u64(q, end, i) || !field_u64(q, end, j) || !field_f64(q, end, x) ||
                       !blank(q, end);
      if (bad || i == 0 || j == 0 || i > m.size1 || j > m.size2) {
        if (errors[t].empty())
          errors[t] = "Parse error at line " + std::to_string(first_line + k) + " of " + path +
                      ": " + std::string(p, end);
        continue;
      }
      m.rows[k] = (uint32_t)(i - 1);
      m.cols[k] = (uint32_t)(j - 1);
      m.vals[k] = x;
    }
  };
  if (T > 1) {
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < T; ++t) pool.emplace_back(work, t);
    for (auto& th : pool) th.join();
  } else {
    work(0);
  }
  for (auto& e : errors)
    if (!e.empty()) throw MmError(e);
  return m;
}

Dense read_mm_array(const std::string& path) {
  const std::string s = read_file(path);
  Lines L(s);
  const char *a, *b;
  read_header(L, path, "%%MatrixMarket matrix array real general", a, b);
  std::string dims(a, b);
  long long s1 = 0, s2 = 0;
  char junk[2] = {0, 0};
  if (std::sscanf(dims.c_str(), "%lld %lld %1s", &s1, &s2, junk) != 2 || s1 < 0 || s2 < 0)
    throw MmError("Invalid matrix dimensions in file " + path + ": " + dims);
  Dense m;
  m.size1 = (uint64_t)s1;
  m.size2 = (uint64_t)s2;
  const uint64_t count = m.size1 * m.size2;
  m.colmajor.resize(count);
  // line starts first, then the values in parallel (as read_mm_coord)
  std::vector<size_t> starts;
  const uint64_t first_line = L.number + 1;
  size_t after = 0;
  if (!line_starts(s, L.pos, count, starts, &after))
    throw MmError("Unexpected EOF in file " + path);
  starts.push_back(after);
  L.pos = after;
  L.number += count;
  unsigned T = std::max(1u, std::thread::hardware_concurrency());
  T = (unsigned)std::min<uint64_t>(T, std::max<uint64_t>(1, count / 100000));
  std::vector<std::string> errors(T);
  auto work = [&](unsigned t) {
    const size_t lo = (size_t)(count * t / T), hi = (size_t)(count * (t + 1) / T);
    for (size_t k = lo; k < hi; ++k) {
      const char* p = s.data() + starts[k];
      const char* end = s.data() + std::min(starts[k + 1], s.size());
      if (end > p && end[-1] == '\n') --end;
      if (end > p && end[-1] == '\r') --end;
      const char* q = p;
      double x = 0;
      if (!field_f64(q, end, x) || !blank(q, end)) {
        if (errors[t].empty())
          errors[t] = "Parse error at line " + std::to_string(first_line + k) + " of " + path +
                      ": " + std::string(p, end);
        continue;
      }
      m.colmajor[k] = x;
    }
  };
  if (T > 1) {
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < T; ++t) pool.emplace_back(work, t);
    for (auto& th : pool) th.join();
  } else {
    work(0);
  }
  for (auto& e : errors)
    if (!e.empty()) throw MmError(e);
  while (L.next(a, b))
    if (!blank(a, b))
      throw MmError("Unexpected input at at line " + std::to_string(L.number) + " of " + path +
                    ": " + std::string(a, b));
  return m;
}

namespace {
// %.16g: std::numeric_limits<double>::digits10 + 1 significant digits, as the
// reference's ostream precision (write_impl.h:51,98); std::to_chars with a
// precision formats exactly as printf's %.16g does
void put_double(std::string& out, double x) {
  char buf[40];
  const auto r = std::to_chars(buf, buf + sizeof(buf), x, std::chars_format::general, 16);
  out.append(buf, (size_t)(r.ptr - buf));
}
void put_u64(std::string& out, uint64_t v) {
  char buf[24];
  const auto r = std::to_chars(buf, buf + sizeof(buf), v);
  out.append(buf, (size_t)(r.ptr - buf));
}

// Writes `header` and then lines 0..n-1, each made by line(out, k); the lines
// are formatted by several threads, one contiguous range each, and written in
// order.
template <typename F>
void write_lines(const std::string& path, const std::string& header, size_t n, size_t bytes_per,
                 F line) {
  unsigned T = std::max(1u, std::thread::hardware_concurrency());
  if (n < (1u << 16)) T = 1;
  std::vector<std::string> parts(T);
  auto work = [&](unsigned t) {
    const size_t a = n * t / T, b = n * (t + 1) / T;
    parts[t].reserve((b - a) * bytes_per);
    for (size_t k = a; k < b; ++k) line(parts[t], k);
  };
  if (T == 1) {
    work(0);
  } else {
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < T; ++t) pool.emplace_back(work, t);
    for (auto& th : pool) th.join();
  }
  std::ofstream f(path, std::ios::binary);
  if (!f.is_open()) throw MmError("Cannot open file " + path);
  f.write(header.data(), (std::streamsize)header.size());
  for (const auto& part : parts) f.write(part.data(), (std::streamsize)part.size());
  if (!f) throw MmError("Cannot write file " + path);
}
}  // namespace

void write_mm_coord(const std::string& path, const Coo& m) {
  std::string head;
  head += "%%MatrixMarket matrix coordinate real general\n";
  head += "%=================================================================================\n";
  head += "%\n% Indices are 1-based, i.e. A(1,1) is the first element.\n%\n";
  head += "%=================================================================================\n";
  head += std::to_string(m.size1) + " " + std::to_string(m.size2) + " " +
          std::to_string(m.vals.size()) + "\n";
  write_lines(path, head, m.vals.size(), 40, [&](std::string& out, size_t k) {
    put_u64(out, (uint64_t)m.rows[k] + 1);
    out += ' ';
    put_u64(out, (uint64_t)m.cols[k] + 1);
    out += ' ';
    put_double(out, m.vals[k]);
    out += '\n';
  });
}

void write_mm_array(const std::string& path, const Dense& m) {
  std::string head;
  head += "%%MatrixMarket matrix array real general\n";
  head += "% First line: ROWS COLUMNS\n";
  head += "% Subsequent lines: entries in column-major order\n";
  head += std::to_string(m.size1) + " " + std::to_string(m.size2) + "\n";
  write_lines(path, head, m.colmajor.size(), 24, [&](std::string& out, size_t k) {
    put_double(out, m.colmajor[k]);
    out += '\n';
  });
}

// ---- minimal XML for the descriptor -------------------------------------------------
namespace {

struct XParser {
  const std::string& s;
  size_t p = 0;
  explicit XParser(const std::string& s) : s(s) {}
  void skip_misc() {
    for (;;) {
      while (p < s.size() && std::isspace((unsigned char)s[p])) ++p;
      if (s.compare(p, 4, "<!--") == 0) {
        size_t e = s.find("-->", p);
        p = e == std::string::npos ? s.size() : e + 3;
      } else if (s.compare(p, 2, "<?") == 0) {
        size_t e = s.find("?>", p);
        p = e == std::string::npos ? s.size() : e + 2;
      } else {
        return;
      }
    }
  }
  static std::string unescape(const std::string& t) {
    std::string o;
    for (size_t i = 0; i < t.size(); ++i) {
      if (t[i] == '&') {
        size_t e = t.find(';', i);
        std::string ent = t.substr(i + 1, e - i - 1);
        if (ent == "lt") o += '<';
        else if (ent == "gt") o += '>';
        else if (ent == "amp") o += '&';
        else if (ent == "quot") o += '"';
        else if (ent == "apos") o += '\'';
        i = e;
      } else {
        o += t[i];
      }
    }
    return o;
  }
  XmlNode element() {
    skip_misc();
    if (p >= s.size() || s[p] != '<') throw MmError("malformed XML descriptor");
    size_t e = s.find_first_of(" \t\r\n/>", p + 1);
    XmlNode n;
    n.name = s.substr(p + 1, e - p - 1);
    size_t close = s.find('>', p);
    if (close == std::string::npos) throw MmError("malformed XML descriptor");
    const bool empty = s[close - 1] == '/';
    p = close + 1;
    if (empty) return n;
    for (;;) {
      size_t lt = s.find('<', p);
      if (lt == std::string::npos) throw MmError("malformed XML descriptor");
      n.text += s.substr(p, lt - p);
      p = lt;
      if (s.compare(p, 4, "<!--") == 0) {
        skip_misc();
        continue;
      }
      if (s.compare(p, 2, "</") == 0) {
        size_t gt = s.find('>', p);
        p = gt + 1;
        break;
      }
      n.kids.push_back(element());
    }
    n.text = unescape(n.text);
    size_t a = n.text.find_first_not_of(" \t\r\n"), b = n.text.find_last_not_of(" \t\r\n");
    n.text = a == std::string::npos ? "" : n.text.substr(a, b - a + 1);
    return n;
  }
};

const XmlNode& need(const XmlNode& n, const std::string& name) {
  const XmlNode* c = n.child(name);
  if (!c) throw MmError("XML descriptor lacks matrix." + name);
  return *c;
}

uint64_t to_u64(const std::string& t) {
  char* q = nullptr;
  errno = 0;
  unsigned long long v = std::strtoull(t.c_str(), &q, 10);
  if (q == t.c_str() || *q || errno) throw MmError("bad number in XML descriptor: " + t);
  return v;
}

std::string xml_escape(const std::string& t) {
  std::string o;
  for (char c : t) {
    if (c == '<') o += "&lt;";
    else if (c == '>') o += "&gt;";
    else if (c == '&') o += "&amp;";
    else o += c;
  }
  return o;
}

}  // namespace

const XmlNode* XmlNode::child(const std::string& n) const {
  for (auto& k : kids)
    if (k.name == n) return &k;
  return nullptr;
}

std::vector<XmlNode> parse_xml(const std::string& text) {
  XParser P(text);
  std::vector<XmlNode> out;
  for (;;) {
    P.skip_misc();
    if (P.p >= text.size()) break;
    out.push_back(P.element());
  }
  return out;
}

BlockedDescriptor read_descriptor(const std::string& path) {
  const std::string s = read_file(path);
  XParser P(s);
  XmlNode root = P.element();
  if (root.name != "matrix") throw MmError("XML descriptor root is not <matrix>: " + path);
  BlockedDescriptor d;
  d.size1 = to_u64(need(root, "size1").text);
  d.size2 = to_u64(need(root, "size2").text);
  d.blocks1 = to_u64(need(root, "blocks1").text);
  d.blocks2 = to_u64(need(root, "blocks2").text);
  d.path = need(root, "path").text;
  for (auto& k : need(root, "blockOffsets1").kids) d.offsets1.push_back(to_u64(k.text));
  for (auto& k : need(root, "blockOffsets2").kids) d.offsets2.push_back(to_u64(k.text));
  for (auto& k : need(root, "filenames").kids) d.filenames.push_back(k.text);
  d.format = need(root, "format").text;
  if (d.offsets1.size() != d.blocks1 || d.offsets2.size() != d.blocks2 ||
      d.filenames.size() != d.blocks1 * d.blocks2)
    throw MmError("inconsistent XML descriptor " + path);
  return d;
}

void write_descriptor(const std::string& path, const BlockedDescriptor& d) {
  std::ostringstream o;
  o << "<?xml version=\"1.0\" encoding=\"utf-8\"?>\n<matrix>\n";
  o << "    <size1>" << d.size1 << "</size1>\n    <size2>" << d.size2 << "</size2>\n";
  o << "    <blocks1>" << d.blocks1 << "</blocks1>\n    <blocks2>" << d.blocks2 << "</blocks2>\n";
  o << "    <blockOffsets1>\n";
  for (auto v : d.offsets1) o << "        <offset>" << v << "</offset>\n";
  o << "    </blockOffsets1>\n    <blockOffsets2>\n";
  for (auto v : d.offsets2) o << "        <offset>" << v << "</offset>\n";
  o << "    </blockOffsets2>\n    <path>" << xml_escape(d.path) << "</path>\n    <filenames>\n";
  for (auto& f : d.filenames) o << "        <filename>" << xml_escape(f) << "</filename>\n";
  o << "    </filenames>\n    <format>" << xml_escape(d.format) << "</format>\n</matrix>\n";
  std::ofstream f(path);
  if (!f.is_open()) throw MmError("Cannot open file " + path);
  f << o.str();
}

Coo read_sparse(const std::string& path, BlockedDescriptor* desc_out) {
  if (!ends_with(path, ".xml")) return read_mm_coord(path);
  BlockedDescriptor d = read_descriptor(path);
  if (d.format != "mmc") throw MmError("blocked sparse files must be in mmc format: " + path);
  Coo all;
  all.size1 = d.size1;
  all.size2 = d.size2;
  for (uint64_t b1 = 0; b1 < d.blocks1; ++b1)
    for (uint64_t b2 = 0; b2 < d.blocks2; ++b2) {
      Coo blk = read_mm_coord(d.path + d.filenames[b1 * d.blocks2 + b2]);
      for (size_t k = 0; k < blk.vals.size(); ++k) {
        all.rows.push_back((uint32_t)(blk.rows[k] + d.offsets1[b1]));
        all.cols.push_back((uint32_t)(blk.cols[k] + d.offsets2[b2]));
        all.vals.push_back(blk.vals[k]);
      }
    }
  if (desc_out) *desc_out = d;
  return all;
}

Dense read_dense(const std::string& path) {
  if (!ends_with(path, ".xml")) return read_mm_array(path);
  const BlockedDescriptor d = read_descriptor(path);
  if (d.format != "mma") throw MmError("blocked dense files must be in mma format: " + path);
  Dense all;
  all.size1 = d.size1;
  all.size2 = d.size2;
  all.colmajor.assign(d.size1 * d.size2, 0.0);
  for (uint64_t b1 = 0; b1 < d.blocks1; ++b1)
    for (uint64_t b2 = 0; b2 < d.blocks2; ++b2) {
      const std::string f = d.path + d.filenames[b1 * d.blocks2 + b2];
      const Dense blk = read_mm_array(f);
      const uint64_t r0 = d.offsets1[b1], c0 = d.offsets2[b2];
      const uint64_t r1 = b1 + 1 < d.blocks1 ? d.offsets1[b1 + 1] : d.size1;
      const uint64_t c1 = b2 + 1 < d.blocks2 ? d.offsets2[b2 + 1] : d.size2;
      if (blk.size1 != r1 - r0 || blk.size2 != c1 - c0)
        throw MmError("block " + f + " is " + std::to_string(blk.size1) + " x " +
                      std::to_string(blk.size2) + ", the descriptor says " +
                      std::to_string(r1 - r0) + " x " + std::to_string(c1 - c0));
      for (uint64_t j = 0; j < blk.size2; ++j)
        for (uint64_t i = 0; i < blk.size1; ++i)
          all.colmajor[(c0 + j) * d.size1 + r0 + i] = blk.colmajor[j * blk.size1 + i];
    }
  return all;
}

}  // namespace dsgdpp

// ---- C ABI of the file I/O (include/dsgdpp.h) ----------------------------------------
namespace {
thread_local std::string g_io_error;

template <typename T>
T* copy_out(const std::vector<T>& v) {
  T* p = static_cast<T*>(std::malloc(std::max<size_t>(1, v.size()) * sizeof(T)));
  if (p && !v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
  return p;
}

template <typename F>
int io_guard(F&& f) {
  try {
    g_io_error.clear();
    f();
    return 0;
  } catch (const std::exception& e) {
    g_io_error = e.what();
    return -3;  // DSGDPP_E_IO
  }
}
}  // namespace

extern "C" {

const char* dsgdpp_io_error(void) { return g_io_error.c_str(); }

void dsgdpp_free(void* p) { std::free(p); }

int dsgdpp_read_sparse(const char* path, uint64_t* m, uint64_t* n, uint64_t* nnz,
                       uint32_t** rows, uint32_t** cols, double** vals) {
  return io_guard([&]() {
    dsgdpp::Coo c = dsgdpp::read_sparse(path);
    *m = c.size1;
    *n = c.size2;
    *nnz = c.vals.size();
    *rows = copy_out(c.rows);
    *cols = copy_out(c.cols);
    *vals = copy_out(c.vals);
  });
}

int dsgdpp_write_mm_coord(const char* path, uint64_t m, uint64_t n, uint64_t nnz,
                          const uint32_t* rows, const uint32_t* cols, const double* vals) {
  return io_guard([&]() {
    dsgdpp::Coo c;
    c.size1 = m;
    c.size2 = n;
    c.rows.assign(rows, rows + nnz);
    c.cols.assign(cols, cols + nnz);
    c.vals.assign(vals, vals + nnz);
    dsgdpp::write_mm_coord(path, c);
  });
}

int dsgdpp_read_mm_array(const char* path, uint64_t* m, uint64_t* n, double** colmajor) {
  return io_guard([&]() {
    dsgdpp::Dense d = dsgdpp::read_dense(path);
    *m = d.size1;
    *n = d.size2;
    *colmajor = copy_out(d.colmajor);
  });
}

int dsgdpp_write_mm_array(const char* path, uint64_t m, uint64_t n, const double* colmajor) {
  return io_guard([&]() {
    dsgdpp::Dense d;
    d.size1 = m;
    d.size2 = n;
    d.colmajor.assign(colmajor, colmajor + m * n);
    dsgdpp::write_mm_array(path, d);
  });
}

int dsgdpp_write_blocked(const char* xml_path, const char* dir, const char* base, uint64_t m,
                         uint64_t n, uint32_t blocks1, uint32_t blocks2, uint64_t nnz,
                         const uint32_t* rows, const uint32_t* cols, const double* vals) {
  return io_guard([&]() {
    // the tools/mfdblock.cc output: one .mmc per block with block-local
    // coordinates and an .xml descriptor (descriptor_impl.h:28-50)
    dsgdpp::BlockedDescriptor d;
    d.size1 = m;
    d.size2 = n;
    d.blocks1 = blocks1;
    d.blocks2 = blocks2;
    d.offsets1.resize(blocks1);
    d.offsets2.resize(blocks2);
    dsgdpp_block_offsets(m, blocks1, d.offsets1.data());
    dsgdpp_block_offsets(n, blocks2, d.offsets2.data());
    d.path = std::string(dir);
    if (!d.path.empty() && d.path.back() != '/') d.path += '/';
    d.format = "mmc";
    std::vector<dsgdpp::Coo> blk((size_t)blocks1 * blocks2);
    auto find = [](const std::vector<uint64_t>& off, uint64_t x) {
      return (size_t)(std::upper_bound(off.begin(), off.end(), x) - off.begin() - 1);
    };
    for (size_t b1 = 0; b1 < blocks1; ++b1)
      for (size_t b2 = 0; b2 < blocks2; ++b2) {
        auto& c = blk[b1 * blocks2 + b2];
        c.size1 = (b1 + 1 < blocks1 ? d.offsets1[b1 + 1] : m) - d.offsets1[b1];
        c.size2 = (b2 + 1 < blocks2 ? d.offsets2[b2 + 1] : n) - d.offsets2[b2];
      }
    for (uint64_t k = 0; k < nnz; ++k) {
      const size_t b1 = find(d.offsets1, rows[k]), b2 = find(d.offsets2, cols[k]);
      auto& c = blk[b1 * blocks2 + b2];
      c.rows.push_back((uint32_t)(rows[k] - d.offsets1[b1]));
      c.cols.push_back((uint32_t)(cols[k] - d.offsets2[b2]));
      c.vals.push_back(vals[k]);
    }
    for (size_t b1 = 0; b1 < blocks1; ++b1)
      for (size_t b2 = 0; b2 < blocks2; ++b2) {
        std::string f = std::string(base) + "-" + std::to_string(b1) + "-" + std::to_string(b2) + ".mmc";
        d.filenames.push_back(f);
        dsgdpp::write_mm_coord(d.path + f, blk[b1 * blocks2 + b2]);
      }
    dsgdpp::write_descriptor(xml_path, d);
  });
}

}  // extern "C"
