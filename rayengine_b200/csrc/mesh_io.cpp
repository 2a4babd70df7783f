// Mesh ingestion on the host: PLY (ascii, binary little / big endian) and
// Wavefront OBJ into the (vertices, triangles) arrays re_scene_create takes.
//
// Replaces, in the reference (hadalhw17/RayEngine):
//   RStaticMesh::LoadFromFile   RayEngine/src/Objects/RStaticMesh.cpp:68-128
//                               (through the vendored rply reader): vertex
//                               x, y, z; per face the first three entries of
//                               vertex_indices
//   WavefrontOBJ::loadObjFromFile
//                               RayEngine/includes/ObjFileReader.h:65-180:
//                               v / vt / vn / f, corners "p", "p/t", "p//n",
//                               "p/t/n"; a vertex per distinct (p, t, n) in
//                               order of first use; a quad (a b c d) becomes
//                               (a b c) and (d a c)
// Behaviour beyond the reference: PLY faces with more than three corners are
// fan-triangulated (RE_MESH_FIRST_TRIANGLE keeps the reference's first
// triangle only); OBJ faces with more than four corners are fan-triangulated
// (the reference reads four); negative (relative) OBJ indices and missing
// normals are accepted; malformed input is an error status, not exit().
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <new>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "re_common.hpp"

struct re_mesh {
  std::vector<float> verts;     // 3 per vertex
  std::vector<uint32_t> faces;  // 3 per triangle
};

namespace re {
namespace {

enum class PlyFormat { Ascii, BinLE, BinBE };

struct PlyProp {
  std::string name;
  bool list = false;
  std::string count_type, type;
};

struct PlyElement {
  std::string name;
  uint64_t count = 0;
  std::vector<PlyProp> props;
};

int type_size(const std::string& t) {
  if (t == "char" || t == "uchar" || t == "int8" || t == "uint8") return 1;
  if (t == "short" || t == "ushort" || t == "int16" || t == "uint16") return 2;
  if (t == "int" || t == "uint" || t == "int32" || t == "uint32" || t == "float" || t == "float32")
    return 4;
  if (t == "double" || t == "float64") return 8;
  return 0;
}

bool host_little_endian() {
  uint16_t x = 1;
  unsigned char c;
  std::memcpy(&c, &x, 1);
  return c == 1;
}

// Reads one binary scalar of type t as double.
bool read_bin(std::istream& is, const std::string& t, bool swap, double& out) {
  unsigned char b[8];
  int n = type_size(t);
  if (n == 0 || !is.read(reinterpret_cast<char*>(b), n)) return false;
  if (swap)
    for (int i = 0; i < n / 2; ++i) std::swap(b[i], b[n - 1 - i]);
  if (t == "char" || t == "int8") out = (double)(int8_t)b[0];
  else if (t == "uchar" || t == "uint8") out = (double)b[0];
  else if (t == "short" || t == "int16") { int16_t v; std::memcpy(&v, b, 2); out = v; }
  else if (t == "ushort" || t == "uint16") { uint16_t v; std::memcpy(&v, b, 2); out = v; }
  else if (t == "int" || t == "int32") { int32_t v; std::memcpy(&v, b, 4); out = v; }
  else if (t == "uint" || t == "uint32") { uint32_t v; std::memcpy(&v, b, 4); out = v; }
  else if (t == "float" || t == "float32") { float v; std::memcpy(&v, b, 4); out = v; }
  else { double v; std::memcpy(&v, b, 8); out = v; }
  return true;
}

// Scalar reader over either encoding.
struct PlyReader {
  std::istream& is;
  PlyFormat fmt;
  bool swap;
  bool next(const std::string& t, double& v) {
    if (fmt == PlyFormat::Ascii) {
      std::string tok;
      if (!(is >> tok)) return false;
      char* end = nullptr;
      v = std::strtod(tok.c_str(), &end);
      return end && *end == '\0';
    }
    return read_bin(is, t, swap, v);
  }
};

void add_face(re_mesh& m, const std::vector<uint32_t>& idx, bool first_only) {
  if (idx.size() < 3) return;
  size_t last = first_only ? 3 : idx.size();
  for (size_t k = 1; k + 1 < last; ++k) {
    m.faces.push_back(idx[0]);
    m.faces.push_back(idx[k]);
    m.faces.push_back(idx[k + 1]);
  }
}

re_status load_ply(const char* path, uint32_t flags, re_mesh& m) {
  std::ifstream is(path, std::ios::binary);
  if (!is) return fail(RE_ERR_INVALID_ARG, "re_mesh_load: cannot open %s", path);
  std::string line;
  if (!std::getline(is, line) || line.rfind("ply", 0) != 0)
    return fail(RE_ERR_INVALID_ARG, "re_mesh_load: %s is not a PLY file", path);
  PlyFormat fmt = PlyFormat::Ascii;
  std::vector<PlyElement> elems;
  bool have_format = false;
  for (;;) {
    if (!std::getline(is, line)) return fail(RE_ERR_INVALID_ARG, "re_mesh_load: %s: header not terminated", path);
    if (!line.empty() && line.back() == '\r') line.pop_back();
    std::istringstream ls(line);
    std::string kw;
    ls >> kw;
    if (kw == "end_header") break;
    if (kw == "format") {
      std::string f;
      ls >> f;
      if (f == "ascii") fmt = PlyFormat::Ascii;
      else if (f == "binary_little_endian") fmt = PlyFormat::BinLE;
      else if (f == "binary_big_endian") fmt = PlyFormat::BinBE;
      else return fail(RE_ERR_INVALID_ARG, "re_mesh_load: %s: unknown format %s", path, f.c_str());
      have_format = true;
    } else if (kw == "element") {
      PlyElement e;
      ls >> e.name >> e.count;
      elems.push_back(e);
    } else if (kw == "property") {
      if (elems.empty()) return fail(RE_ERR_INVALID_ARG, "re_mesh_load: %s: property before element", path);
      PlyProp p;
      std::string t;
      ls >> t;
      if (t == "list") {
        p.list = true;
        ls >> p.count_type >> p.type >> p.name;
        if (!type_size(p.count_type) || !type_size(p.type))
          return fail(RE_ERR_INVALID_ARG, "re_mesh_load: %s: bad list property", path);
      } else {
        p.type = t;
        ls >> p.name;
        if (!type_size(p.type)) return fail(RE_ERR_INVALID_ARG, "re_mesh_load: %s: bad type %s", path, t.c_str());
      }
      elems.back().props.push_back(p);
    }
    // comment / obj_info lines are skipped
  }
  if (!have_format) return fail(RE_ERR_INVALID_ARG, "re_mesh_load: %s: no format line", path);
  bool swap = (fmt == PlyFormat::BinLE) != host_little_endian() && fmt != PlyFormat::Ascii;
  PlyReader rd{is, fmt, swap};
  const bool first_only = (flags & RE_MESH_FIRST_TRIANGLE) != 0u;
  uint64_t nverts = 0;
  for (const PlyElement& e : elems) {
    int ix = -1, iy = -1, iz = -1, ifc = -1;
    for (size_t k = 0; k < e.props.size(); ++k) {
      const PlyProp& p = e.props[k];
      if (!p.list && p.name == "x") ix = (int)k;
      if (!p.list && p.name == "y") iy = (int)k;
      if (!p.list && p.name == "z") iz = (int)k;
      if (p.list && (p.name == "vertex_indices" || p.name == "vertex_index")) ifc = (int)k;
    }
    const bool is_vertex = e.name == "vertex", is_face = e.name == "face";
    if (is_vertex && (ix < 0 || iy < 0 || iz < 0))
      return fail(RE_ERR_INVALID_ARG, "re_mesh_load: %s: vertex without x, y, z", path);
    if (is_vertex) {
      nverts = e.count;
      if (nverts > 0xFFFFFFFFull / 3) return fail(RE_ERR_LIMIT, "re_mesh_load: %s: too many vertices", path);
      m.verts.reserve(3 * nverts);
    }
    std::vector<uint32_t> idx;
    for (uint64_t r = 0; r < e.count; ++r) {
      float xyz[3] = {0.f, 0.f, 0.f};
      for (size_t k = 0; k < e.props.size(); ++k) {
        const PlyProp& p = e.props[k];
        double v = 0.0;
        if (!p.list) {
          if (!rd.next(p.type, v)) return fail(RE_ERR_INVALID_ARG, "re_mesh_load: %s: truncated data", path);
          if ((int)k == ix) xyz[0] = (float)v;
          if ((int)k == iy) xyz[1] = (float)v;
          if ((int)k == iz) xyz[2] = (float)v;
          continue;
        }
        double cnt = 0.0;
        if (!rd.next(p.count_type, cnt) || cnt < 0 || cnt > 1e6)
          return fail(RE_ERR_INVALID_ARG, "re_mesh_load: %s: bad list length", path);
        idx.clear();
        for (uint32_t j = 0; j < (uint32_t)cnt; ++j) {
          if (!rd.next(p.type, v)) return fail(RE_ERR_INVALID_ARG, "re_mesh_load: %s: truncated data", path);
          if (is_face && (int)k == ifc) {
            if (v < 0 || v >= (double)nverts)
              return fail(RE_ERR_INVALID_ARG, "re_mesh_load: %s: face index %.0f out of range", path, v);
            idx.push_back((uint32_t)v);
          }
        }
        if (is_face && (int)k == ifc) add_face(m, idx, first_only);
      }
      if (is_vertex) {
        m.verts.push_back(xyz[0]);
        m.verts.push_back(xyz[1]);
        m.verts.push_back(xyz[2]);
      }
    }
  }
  return RE_OK;
}

// OBJ corner "p", "p/t", "p//n" or "p/t/n" (1-based, negative = relative).
bool obj_corner(const std::string& tok, long np, long nt, long nn, long& p, long& t, long& n) {
  p = t = n = 0;
  long* dst[3] = {&p, &t, &n};
  long sizes[3] = {np, nt, nn};
  size_t start = 0;
  for (int f = 0; f < 3; ++f) {
    size_t slash = tok.find('/', start);
    std::string part = tok.substr(start, slash == std::string::npos ? std::string::npos : slash - start);
    if (!part.empty()) {
      char* end = nullptr;
      long v = std::strtol(part.c_str(), &end, 10);
      if (!end || *end != '\0' || v == 0) return false;
      if (v < 0) v = sizes[f] + 1 + v;
      if (v < 1 || v > sizes[f]) return false;
      *dst[f] = v;
    } else if (f == 0) {
      return false;
    }
    if (slash == std::string::npos) break;
    start = slash + 1;
  }
  return true;
}

re_status load_obj(const char* path, re_mesh& m) {
  std::ifstream is(path);
  if (!is) return fail(RE_ERR_INVALID_ARG, "re_mesh_load: cannot open %s", path);
  std::vector<float> pos;
  long nt = 0, nn = 0;
  std::map<std::tuple<long, long, long>, uint32_t> vmap;
  std::string line;
  uint64_t lineno = 0;
  while (std::getline(is, line)) {
    ++lineno;
    std::istringstream ls(line);
    std::string kw;
    if (!(ls >> kw)) continue;
    if (kw == "v") {
      float x, y, z;
      if (!(ls >> x >> y >> z)) return fail(RE_ERR_INVALID_ARG, "re_mesh_load: %s:%llu: bad vertex", path, (unsigned long long)lineno);
      pos.push_back(x);
      pos.push_back(y);
      pos.push_back(z);
    } else if (kw == "vt") {
      ++nt;
    } else if (kw == "vn") {
      ++nn;
    } else if (kw == "f") {
      std::vector<uint32_t> idx;
      std::string tok;
      while (ls >> tok) {
        long p, t, n;
        if (!obj_corner(tok, (long)(pos.size() / 3), nt, nn, p, t, n))
          return fail(RE_ERR_INVALID_ARG, "re_mesh_load: %s:%llu: bad face corner %s", path,
                      (unsigned long long)lineno, tok.c_str());
        auto key = std::make_tuple(p, t, n);
        auto it = vmap.find(key);
        uint32_t id;
        if (it == vmap.end()) {
          id = (uint32_t)(m.verts.size() / 3);
          vmap.emplace(key, id);
          m.verts.push_back(pos[3 * (p - 1)]);
          m.verts.push_back(pos[3 * (p - 1) + 1]);
          m.verts.push_back(pos[3 * (p - 1) + 2]);
        } else {
          id = it->second;
        }
        idx.push_back(id);
      }
      if (idx.size() == 4) {
        // the reference's quad split: (a b c) and (d a c)
        uint32_t q[6] = {idx[0], idx[1], idx[2], idx[3], idx[0], idx[2]};
        m.faces.insert(m.faces.end(), q, q + 6);
      } else {
        add_face(m, idx, false);
      }
    }
  }
  return RE_OK;
}

}  // namespace
}  // namespace re

extern "C" {

RE_API re_status re_mesh_load(const char* path, uint32_t flags, re_mesh** out) {
  if (!path || !out) return re::fail(RE_ERR_INVALID_ARG, "re_mesh_load: bad arguments");
  *out = nullptr;
  std::string p(path);
  std::string ext = p.size() >= 4 ? p.substr(p.size() - 4) : "";
  for (char& c : ext) c = (char)std::tolower((unsigned char)c);
  re_mesh* m = new (std::nothrow) re_mesh();
  if (!m) return re::fail(RE_ERR_OUT_OF_MEMORY, "re_mesh_load: host allocation");
  re_status s;
  try {
    if (ext == ".ply") s = re::load_ply(path, flags, *m);
    else if (ext == ".obj") s = re::load_obj(path, *m);
    else s = re::fail(RE_ERR_INVALID_ARG, "re_mesh_load: %s: expected .ply or .obj", path);
  } catch (const std::bad_alloc&) {
    s = re::fail(RE_ERR_OUT_OF_MEMORY, "re_mesh_load: host allocation");
  }
  if (s == RE_OK && (m->faces.size() / 3 > 0xFFFFFFFFull || m->verts.size() / 3 > 0xFFFFFFFFull))
    s = re::fail(RE_ERR_LIMIT, "re_mesh_load: %s: mesh too large", path);
  if (s != RE_OK) {
    delete m;
    return s;
  }
  *out = m;
  return RE_OK;
}

RE_API re_status re_mesh_info(const re_mesh* m, uint32_t* num_verts, uint32_t* num_faces) {
  if (!m || !num_verts || !num_faces) return re::fail(RE_ERR_INVALID_ARG, "re_mesh_info: bad arguments");
  *num_verts = (uint32_t)(m->verts.size() / 3);
  *num_faces = (uint32_t)(m->faces.size() / 3);
  return RE_OK;
}

RE_API re_status re_mesh_copy(const re_mesh* m, float* verts, uint32_t* faces) {
  if (!m || !verts || !faces) return re::fail(RE_ERR_INVALID_ARG, "re_mesh_copy: bad arguments");
  std::memcpy(verts, m->verts.data(), m->verts.size() * sizeof(float));
  std::memcpy(faces, m->faces.data(), m->faces.size() * sizeof(uint32_t));
  return RE_OK;
}

RE_API re_status re_mesh_destroy(re_mesh* m) {
  delete m;
  return RE_OK;
}

}  // extern "C"
