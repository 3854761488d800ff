// ply.cc -- PLY mesh reader with the reference's acceptance rules
// (load/mesh/load-ply.cc:41-214, which drives the vendored RPly library):
//
//   * vertex x, y, z (any PLY scalar type) become a vertex when z is read,
//     taking x and y from the most recent x and y values;
//   * vertex nx, ny, nz become that vertex's normal when nz is read, but
//     only if some component exceeds Eps = 1e-15 (a normal whose components
//     are all <= 1e-15 is skipped); a normal for a vertex whose predecessors
//     do not all have normals is "Normal consistency error" (Mesh::add_normal
//     surface/mesh.cc:121-137 returns another index then);
//   * face vertex_indices lists: entries 0, 1, 2 make one triangle when the
//     third is read; a fourth entry is "Invalid number of indices in face";
//     shorter lists add nothing;
//   * every value passes through single precision (the reader's value
//     buffer is coord_t), face indices included.
//
// The parser itself is written here from the PLY format (header of element
// and property declarations, then the data in ASCII or binary little- or
// big-endian).  Files the reference would accept but then render with
// undefined behaviour are refused with an error instead: normals for only a
// leading part of the vertices, normals without vertices, face indices
// beyond the vertex count.

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "ply.h"

namespace snog {

namespace {

enum PlyType { T_I8, T_U8, T_I16, T_U16, T_I32, T_U32, T_F32, T_F64, T_BAD };

PlyType type_of(const std::string &s) {
  if (s == "char" || s == "int8") return T_I8;
  if (s == "uchar" || s == "uint8") return T_U8;
  if (s == "short" || s == "int16") return T_I16;
  if (s == "ushort" || s == "uint16") return T_U16;
  if (s == "int" || s == "int32") return T_I32;
  if (s == "uint" || s == "uint32") return T_U32;
  if (s == "float" || s == "float32") return T_F32;
  if (s == "double" || s == "float64") return T_F64;
  return T_BAD;
}

int size_of(PlyType t) {
  switch (t) {
    case T_I8: case T_U8: return 1;
    case T_I16: case T_U16: return 2;
    case T_I32: case T_U32: case T_F32: return 4;
    case T_F64: return 8;
    default: return 0;
  }
}

struct Property {
  std::string name;
  bool is_list = false;
  PlyType count_type = T_BAD, value_type = T_BAD;
};

struct Element {
  std::string name;
  uint64_t count = 0;
  std::vector<Property> props;
};

enum Format { ASCII, BIN_LE, BIN_BE };

[[noreturn]] void fail(const std::string &m) { throw std::runtime_error("PLY: " + m); }

// Reads values one at a time from the data section.
struct Reader {
  const std::vector<char> &buf;
  size_t pos;
  Format fmt;

  double ascii_value() {
    while (pos < buf.size() && (buf[pos] == ' ' || buf[pos] == '\t' || buf[pos] == '\n' || buf[pos] == '\r')) pos++;
    if (pos >= buf.size()) fail("unexpected end of file");
    size_t end = pos;
    while (end < buf.size() && !(buf[end] == ' ' || buf[end] == '\t' || buf[end] == '\n' || buf[end] == '\r')) end++;
    std::string tok(buf.data() + pos, end - pos);
    pos = end;
    char *stop = nullptr;
    double v = std::strtod(tok.c_str(), &stop);
    if (stop == tok.c_str() || *stop != '\0') fail("bad number '" + tok + "'");
    return v;
  }

  double value(PlyType t) {
    if (fmt == ASCII) return ascii_value();
    const int n = size_of(t);
    if (pos + size_t(n) > buf.size()) fail("unexpected end of file");
    unsigned char b[8];
    std::memcpy(b, buf.data() + pos, size_t(n));
    pos += size_t(n);
    if (fmt == BIN_BE)
      for (int i = 0; i < n / 2; i++) std::swap(b[i], b[n - 1 - i]);   // to little-endian
    switch (t) {
      case T_I8: { int8_t v; std::memcpy(&v, b, 1); return v; }
      case T_U8: return b[0];
      case T_I16: { int16_t v; std::memcpy(&v, b, 2); return v; }
      case T_U16: { uint16_t v; std::memcpy(&v, b, 2); return v; }
      case T_I32: { int32_t v; std::memcpy(&v, b, 4); return v; }
      case T_U32: { uint32_t v; std::memcpy(&v, b, 4); return v; }
      case T_F32: { float v; std::memcpy(&v, b, 4); return v; }
      case T_F64: { double v; std::memcpy(&v, b, 8); return v; }
      default: fail("bad property type");
    }
  }
};

std::vector<std::string> words(const std::string &line) {
  std::vector<std::string> w;
  size_t i = 0;
  while (i < line.size()) {
    while (i < line.size() && (line[i] == ' ' || line[i] == '\t' || line[i] == '\r')) i++;
    size_t j = i;
    while (j < line.size() && !(line[j] == ' ' || line[j] == '\t' || line[j] == '\r')) j++;
    if (j > i) w.push_back(line.substr(i, j - i));
    i = j;
  }
  return w;
}

}  // namespace

PlyMeshHost read_ply(const std::string &path) {
  std::vector<char> buf;
  {
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) fail("unable to open " + path);
    char tmp[1 << 16];
    size_t n;
    while ((n = std::fread(tmp, 1, sizeof tmp, f)) > 0) buf.insert(buf.end(), tmp, tmp + n);
    std::fclose(f);
  }
  // ---- header --------------------------------------------------------------
  size_t pos = 0;
  auto next_line = [&](std::string &line) {
    if (pos >= buf.size()) return false;
    size_t e = pos;
    while (e < buf.size() && buf[e] != '\n') e++;
    line.assign(buf.data() + pos, e - pos);
    pos = e < buf.size() ? e + 1 : e;
    return true;
  };
  std::string line;
  if (!next_line(line) || words(line) != std::vector<std::string>{"ply"}) fail("not a PLY file");
  Format fmt = ASCII;
  bool have_format = false;
  std::vector<Element> elems;
  for (;;) {
    if (!next_line(line)) fail("header has no end_header");
    std::vector<std::string> w = words(line);
    if (w.empty()) continue;
    if (w[0] == "end_header") break;
    if (w[0] == "comment" || w[0] == "obj_info") continue;
    if (w[0] == "format") {
      if (w.size() < 3 || w[2] != "1.0") fail("unsupported format line");
      if (w[1] == "ascii") fmt = ASCII;
      else if (w[1] == "binary_little_endian") fmt = BIN_LE;
      else if (w[1] == "binary_big_endian") fmt = BIN_BE;
      else fail("unknown format " + w[1]);
      have_format = true;
    } else if (w[0] == "element") {
      if (w.size() != 3) fail("bad element line");
      Element e;
      e.name = w[1];
      e.count = std::strtoull(w[2].c_str(), nullptr, 10);
      elems.push_back(e);
    } else if (w[0] == "property") {
      if (elems.empty()) fail("property before any element");
      Property p;
      if (w.size() == 5 && w[1] == "list") {
        p.is_list = true;
        p.count_type = type_of(w[2]);
        p.value_type = type_of(w[3]);
        p.name = w[4];
        if (p.count_type == T_BAD || p.value_type == T_BAD) fail("bad list property types");
      } else if (w.size() == 3) {
        p.value_type = type_of(w[1]);
        p.name = w[2];
        if (p.value_type == T_BAD) fail("bad property type " + w[1]);
      } else {
        fail("bad property line");
      }
      elems.back().props.push_back(p);
    } else {
      fail("unknown header line '" + w[0] + "'");
    }
  }
  if (!have_format) fail("header has no format line");

  // ---- data, with the reference loader's callbacks ----------------------------
  PlyMeshHost m;
  std::vector<float> normals;
  float vals[3] = {0.f, 0.f, 0.f};   // shared by every callback, as coord_t values
  uint32_t last_vert = 0;
  Reader rd{buf, pos, fmt};
  for (const Element &e : elems) {
    const bool is_vertex = e.name == "vertex", is_face = e.name == "face";
    for (uint64_t i = 0; i < e.count; i++) {
      for (const Property &p : e.props) {
        if (p.is_list) {
          const double cnt = rd.value(p.count_type);
          if (cnt < 0) fail("negative list length");
          const uint64_t n = uint64_t(cnt);
          const bool faces = is_face && p.name == "vertex_indices";
          for (uint64_t k = 0; k < n; k++) {
            const double v = rd.value(p.value_type);
            if (!faces) continue;
            if (k >= 3) fail("Invalid number of indices in face");
            vals[k] = float(v);
            if (k == 2)
              for (int c = 0; c < 3; c++) m.triangles.push_back(uint32_t(vals[c]));
          }
          continue;
        }
        const double v = rd.value(p.value_type);
        if (!is_vertex) continue;
        int axis = -1;
        bool normal = false;
        if (p.name == "x") axis = 0;
        else if (p.name == "y") axis = 1;
        else if (p.name == "z") axis = 2;
        else if (p.name == "nx") axis = 0, normal = true;
        else if (p.name == "ny") axis = 1, normal = true;
        else if (p.name == "nz") axis = 2, normal = true;
        if (axis < 0) continue;
        vals[axis] = float(v);
        if (axis != 2) continue;
        if (!normal) {
          last_vert = uint32_t(m.vertices.size() / 3);
          m.vertices.insert(m.vertices.end(), {vals[0], vals[1], vals[2]});
        } else if (vals[0] > 1e-15f || vals[1] > 1e-15f || vals[2] > 1e-15f) {
          if (normals.size() / 3 < last_vert) fail("Normal consistency error");
          normals.insert(normals.end(), {vals[0], vals[1], vals[2]});
        }
      }
    }
  }
  const size_t nv = m.vertices.size() / 3;
  if (!normals.empty()) {
    if (normals.size() / 3 != nv)
      fail("vertex normals given for " + std::to_string(normals.size() / 3) + " of " + std::to_string(nv) +
           " vertices");
    m.normals = std::move(normals);
  }
  for (uint32_t v : m.triangles)
    if (v >= nv) fail("face index " + std::to_string(v) + " out of range");
  return m;
}

}  // namespace snog
