// meshio.h — io::load_mesh for PLY (io/mod.rs:114-137, io/ply.rs, mesh/clean.rs):
// host code that feeds scans to the device path.
//
// The reader takes ASCII, binary little-endian and binary big-endian PLY
// with any integer or floating property types; the vertex coordinates are the
// `x`, `y`, `z` properties widened to f64, the faces the `vertex_indices` (or
// `vertex_index`) list, a polygon of n corners becoming the fan
// (i0, i_{k-1}, i_k), k = 2..n-1, and a face of fewer than three corners being
// dropped (io/ply.rs:1-16, 86-100). Every other element and property is read
// past. The mesh is then cleaned as mesh/clean.rs:138-142 does: duplicate
// vertices merge onto their first occurrence (equal coordinates, +0 = -0, a
// NaN never equal), faces with a repeated corner are dropped, unreferenced
// vertices are removed, indices renumbered in order.
#pragma once

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

namespace sherd {
namespace meshio {

enum class PlyType { I8, U8, I16, U16, I32, U32, F32, F64, BAD };

inline PlyType ply_type(const std::string &s) {
  if (s == "char" || s == "int8") return PlyType::I8;
  if (s == "uchar" || s == "uint8") return PlyType::U8;
  if (s == "short" || s == "int16") return PlyType::I16;
  if (s == "ushort" || s == "uint16") return PlyType::U16;
  if (s == "int" || s == "int32") return PlyType::I32;
  if (s == "uint" || s == "uint32") return PlyType::U32;
  if (s == "float" || s == "float32") return PlyType::F32;
  if (s == "double" || s == "float64") return PlyType::F64;
  return PlyType::BAD;
}

inline size_t ply_size(PlyType t) {
  switch (t) {
    case PlyType::I8: case PlyType::U8: return 1;
    case PlyType::I16: case PlyType::U16: return 2;
    case PlyType::I32: case PlyType::U32: case PlyType::F32: return 4;
    case PlyType::F64: return 8;
    default: return 0;
  }
}

struct PlyProperty {
  std::string name;
  bool list = false;
  PlyType count = PlyType::BAD, item = PlyType::BAD;
};

struct PlyElement {
  std::string name;
  uint64_t n = 0;
  std::vector<PlyProperty> props;
};

struct HostMesh {
  std::vector<double> v;    // xyz per vertex
  std::vector<uint32_t> f;  // three per face
};

// A cursor over the payload: binary (either endianness) or ASCII tokens.
class PlyCursor {
 public:
  PlyCursor(const std::vector<char> &buf, size_t at, int format)
      : b_(buf), at_(at), format_(format) {}

  // The next value of type t as a double (integers are exact below 2^53).
  bool next(PlyType t, double &out) {
    if (format_ == 0) return next_ascii(out);
    size_t n = ply_size(t);
    if (n == 0 || at_ + n > b_.size()) return false;
    unsigned char raw[8];
    std::memcpy(raw, b_.data() + at_, n);
    at_ += n;
    bool little = format_ == 1;
    bool host_little = true;
    {
      uint16_t probe = 1;
      unsigned char c;
      std::memcpy(&c, &probe, 1);
      host_little = c == 1;
    }
    if (little != host_little)
      for (size_t i = 0; i < n / 2; ++i) std::swap(raw[i], raw[n - 1 - i]);
    switch (t) {
      case PlyType::I8: { int8_t x; std::memcpy(&x, raw, 1); out = x; break; }
      case PlyType::U8: { uint8_t x; std::memcpy(&x, raw, 1); out = x; break; }
      case PlyType::I16: { int16_t x; std::memcpy(&x, raw, 2); out = x; break; }
      case PlyType::U16: { uint16_t x; std::memcpy(&x, raw, 2); out = x; break; }
      case PlyType::I32: { int32_t x; std::memcpy(&x, raw, 4); out = x; break; }
      case PlyType::U32: { uint32_t x; std::memcpy(&x, raw, 4); out = x; break; }
      case PlyType::F32: { float x; std::memcpy(&x, raw, 4); out = x; break; }
      case PlyType::F64: { double x; std::memcpy(&x, raw, 8); out = x; break; }
      default: return false;
    }
    return true;
  }

 private:
  bool next_ascii(double &out) {
    while (at_ < b_.size() && std::isspace(static_cast<unsigned char>(b_[at_]))) ++at_;
    if (at_ >= b_.size()) return false;
    size_t end = at_;
    while (end < b_.size() && !std::isspace(static_cast<unsigned char>(b_[end]))) ++end;
    std::string tok(b_.data() + at_, end - at_);
    at_ = end;
    char *stop = nullptr;
    out = std::strtod(tok.c_str(), &stop);
    return stop && *stop == '\0';
  }

  const std::vector<char> &b_;
  size_t at_;
  int format_;  // 0 ascii, 1 binary little-endian, 2 binary big-endian
};

// Reads `path` into m; returns "" or a message.
inline std::string read_ply(const char *path, HostMesh &m) {
  std::FILE *fp = std::fopen(path, "rb");
  if (!fp) return "cannot open the file";
  std::vector<char> buf;
  char chunk[1 << 16];
  size_t got;
  while ((got = std::fread(chunk, 1, sizeof chunk, fp)) > 0) buf.insert(buf.end(), chunk, chunk + got);
  std::fclose(fp);
  // The header, line by line.
  size_t at = 0;
  auto line = [&](std::string &out) {
    if (at >= buf.size()) return false;
    size_t end = at;
    while (end < buf.size() && buf[end] != '\n') ++end;
    out.assign(buf.data() + at, end - at);
    if (!out.empty() && out.back() == '\r') out.pop_back();
    at = end < buf.size() ? end + 1 : end;
    return true;
  };
  std::string l;
  if (!line(l) || l != "ply") return "not a PLY file";
  int format = -1;
  std::vector<PlyElement> elements;
  bool ended = false;
  while (line(l)) {
    std::vector<std::string> w;
    size_t i = 0;
    while (i < l.size()) {
      while (i < l.size() && std::isspace(static_cast<unsigned char>(l[i]))) ++i;
      size_t j = i;
      while (j < l.size() && !std::isspace(static_cast<unsigned char>(l[j]))) ++j;
      if (j > i) w.emplace_back(l.substr(i, j - i));
      i = j;
    }
    if (w.empty() || w[0] == "comment" || w[0] == "obj_info") continue;
    if (w[0] == "end_header") {
      ended = true;
      break;
    }
    if (w[0] == "format" && w.size() >= 2) {
      format = w[1] == "ascii" ? 0 : w[1] == "binary_little_endian" ? 1
             : w[1] == "binary_big_endian" ? 2 : -1;
      if (format < 0) return "unknown PLY format " + w[1];
    } else if (w[0] == "element" && w.size() >= 3) {
      PlyElement e;
      e.name = w[1];
      e.n = std::strtoull(w[2].c_str(), nullptr, 10);
      elements.push_back(e);
    } else if (w[0] == "property" && !elements.empty()) {
      PlyProperty p;
      if (w.size() >= 5 && w[1] == "list") {
        p.list = true;
        p.count = ply_type(w[2]);
        p.item = ply_type(w[3]);
        p.name = w[4];
        if (p.count == PlyType::BAD || p.item == PlyType::BAD) return "unknown PLY list type";
      } else if (w.size() >= 3) {
        p.item = ply_type(w[1]);
        p.name = w[2];
        if (p.item == PlyType::BAD) return "unknown PLY property type " + w[1];
      } else {
        return "malformed PLY property";
      }
      elements.back().props.push_back(p);
    } else {
      return "malformed PLY header line: " + l;
    }
  }
  if (!ended || format < 0) return "incomplete PLY header";
  PlyCursor cur(buf, at, format);
  std::vector<double> fan;
  for (const PlyElement &e : elements) {
    const bool is_vertex = e.name == "vertex", is_face = e.name == "face";
    // Every instance takes at least one byte of payload.
    if (e.n > buf.size() - std::min(at, buf.size())) return "truncated PLY payload";
    if (is_vertex) m.v.assign(3 * e.n, 0.0);
    for (uint64_t r = 0; r < e.n; ++r) {
      for (const PlyProperty &p : e.props) {
        double x;
        if (p.list) {
          if (!cur.next(p.count, x) || !(x >= 0.0)) return "truncated PLY list";
          uint64_t k = uint64_t(x);
          const bool corners = is_face && (p.name == "vertex_indices" || p.name == "vertex_index");
          fan.clear();
          for (uint64_t c = 0; c < k; ++c) {
            if (!cur.next(p.item, x)) return "truncated PLY list";
            if (corners) fan.push_back(x);
          }
          if (corners && fan.size() >= 3) {
            for (size_t c = 2; c < fan.size(); ++c) {
              for (double idx : {fan[0], fan[c - 1], fan[c]}) {
                if (!(idx >= 0.0) || idx >= 4294967296.0) return "PLY face index out of range";
                m.f.push_back(uint32_t(idx));
              }
            }
          }
        } else {
          if (!cur.next(p.item, x)) return "truncated PLY payload";
          if (is_vertex) {
            if (p.name == "x") m.v[3 * r] = x;
            else if (p.name == "y") m.v[3 * r + 1] = x;
            else if (p.name == "z") m.v[3 * r + 2] = x;
          }
        }
      }
    }
  }
  const size_t nv = m.v.size() / 3;
  for (uint32_t idx : m.f)
    if (idx >= nv) return "a face names a vertex the file does not have";
  return "";
}

// mesh/clean.rs:138-142 in place.
inline void clean(HostMesh &m) {
  const size_t nv = m.v.size() / 3;
  auto bits = [](double x) {
    if (x == 0.0) x = 0.0;  // +0 and -0 are one key
    uint64_t b;
    std::memcpy(&b, &x, 8);
    return b;
  };
  struct Key {
    uint64_t a, b, c;
    bool operator==(const Key &o) const { return a == o.a && b == o.b && c == o.c; }
  };
  struct Hash {
    size_t operator()(const Key &k) const {
      return size_t(k.a * 0x9E3779B97F4A7C15ull ^ (k.b + 0x632BE59BD9B4E019ull) * 31 ^ k.c);
    }
  };
  // Duplicate vertices onto their first occurrence.
  std::unordered_map<Key, uint32_t, Hash> first;
  first.reserve(nv * 2);
  std::vector<uint32_t> to(nv);
  size_t k = 0;
  for (size_t i = 0; i < nv; ++i) {
    const double *p = &m.v[3 * i];
    bool nan = std::isnan(p[0]) || std::isnan(p[1]) || std::isnan(p[2]);
    if (!nan) {
      Key key{bits(p[0]), bits(p[1]), bits(p[2])};
      auto it = first.find(key);
      if (it != first.end()) {
        to[i] = it->second;
        continue;
      }
      first.emplace(key, uint32_t(k));
    }
    for (int c = 0; c < 3; ++c) m.v[3 * k + c] = p[c];
    to[i] = uint32_t(k++);
  }
  m.v.resize(3 * k);
  for (uint32_t &idx : m.f) idx = to[idx];
  // Faces with a repeated corner.
  size_t w = 0;
  for (size_t t = 0; t < m.f.size() / 3; ++t) {
    uint32_t a = m.f[3 * t], b = m.f[3 * t + 1], c = m.f[3 * t + 2];
    if (a == b || b == c || c == a) continue;
    m.f[3 * w] = a;
    m.f[3 * w + 1] = b;
    m.f[3 * w + 2] = c;
    ++w;
  }
  m.f.resize(3 * w);
  // Unreferenced vertices.
  const size_t nv2 = m.v.size() / 3;
  std::vector<uint8_t> used(nv2, 0);
  for (uint32_t idx : m.f) used[idx] = 1;
  std::vector<uint32_t> to2(nv2, 0);
  size_t n = 0;
  for (size_t i = 0; i < nv2; ++i) {
    if (!used[i]) continue;
    for (int c = 0; c < 3; ++c) m.v[3 * n + c] = m.v[3 * i + c];
    to2[i] = uint32_t(n++);
  }
  m.v.resize(3 * n);
  for (uint32_t &idx : m.f) idx = to2[idx];
}

}  // namespace meshio
}  // namespace sherd
