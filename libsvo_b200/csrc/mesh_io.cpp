// mesh_io.cpp -- PLY meshes, the input format of the reference's octree
// builder (projects/octree_builder/src/octree_builder.cpp:85-157 loads
// "*.ply files with per vertex color and normals" through gloost's PlyLoader,
// which is not part of the reference).
//
// Reads ascii and binary_little_endian PLY: the vertex element's x, y, z and,
// when present, nx, ny, nz and red, green, blue (integer colours divided by
// 255, float colours as they are); the face element's vertex index list,
// polygons split into triangle fans.  Other elements and properties are
// skipped.  svo_mesh_fit_unit_cube restates the builder's placement: an
// optional rotation about x, the bounding box centred at the origin and its
// largest side scaled to 1 (so the mesh fits the octree's [-0.5, 0.5]^3),
// normals rotated and normalised.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/libsvo_b200.h"

struct svo_mesh {
  std::vector<float> v, n, c;
  std::vector<uint32_t> t;
};

namespace {

enum class PType { I8, U8, I16, U16, I32, U32, F32, F64, Bad };

PType ptype(const std::string& s) {
  if (s == "char" || s == "int8") return PType::I8;
  if (s == "uchar" || s == "uint8") return PType::U8;
  if (s == "short" || s == "int16") return PType::I16;
  if (s == "ushort" || s == "uint16") return PType::U16;
  if (s == "int" || s == "int32") return PType::I32;
  if (s == "uint" || s == "uint32") return PType::U32;
  if (s == "float" || s == "float32") return PType::F32;
  if (s == "double" || s == "float64") return PType::F64;
  return PType::Bad;
}

size_t psize(PType t) {
  switch (t) {
    case PType::I8:
    case PType::U8:
      return 1;
    case PType::I16:
    case PType::U16:
      return 2;
    case PType::I32:
    case PType::U32:
    case PType::F32:
      return 4;
    case PType::F64:
      return 8;
    default:
      return 0;
  }
}

bool is_int(PType t) { return t != PType::F32 && t != PType::F64; }

struct Property {
  std::string name;
  PType type = PType::Bad;
  bool list = false;
  PType count_type = PType::Bad;
};

struct Element {
  std::string name;
  uint64_t count = 0;
  std::vector<Property> props;
};

// One scalar in either encoding, as double.
struct Reader {
  std::istream& in;
  bool binary;
  bool ok = true;
  double get(PType t) {
    if (!binary) {
      double v = 0.0;
      if (!(in >> v)) ok = false;
      return v;
    }
    unsigned char b[8];
    const size_t n = psize(t);
    if (!in.read((char*)b, (std::streamsize)n)) {
      ok = false;
      return 0.0;
    }
    switch (t) {  // little endian host and file
      case PType::I8: return (double)(int8_t)b[0];
      case PType::U8: return (double)b[0];
      case PType::I16: { int16_t x; std::memcpy(&x, b, 2); return x; }
      case PType::U16: { uint16_t x; std::memcpy(&x, b, 2); return x; }
      case PType::I32: { int32_t x; std::memcpy(&x, b, 4); return x; }
      case PType::U32: { uint32_t x; std::memcpy(&x, b, 4); return x; }
      case PType::F32: { float x; std::memcpy(&x, b, 4); return x; }
      case PType::F64: { double x; std::memcpy(&x, b, 8); return x; }
      default: ok = false; return 0.0;
    }
  }
};

int load_ply(const char* path, svo_mesh& m) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return SVO_ERR_NOENT;
  std::string line;
  if (!std::getline(f, line) || line.rfind("ply", 0) != 0) return SVO_ERR_INVALID;
  bool binary = false, have_format = false;
  std::vector<Element> elems;
  while (std::getline(f, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    std::istringstream ls(line);
    std::string kw;
    ls >> kw;
    if (kw == "format") {
      std::string fmt;
      ls >> fmt;
      if (fmt == "ascii") binary = false;
      else if (fmt == "binary_little_endian") binary = true;
      else return SVO_ERR_NOTSUP;  // big-endian files
      have_format = true;
    } else if (kw == "element") {
      Element e;
      ls >> e.name >> e.count;
      if (!ls) return SVO_ERR_INVALID;
      elems.push_back(e);
    } else if (kw == "property") {
      if (elems.empty()) return SVO_ERR_INVALID;
      Property p;
      std::string t;
      ls >> t;
      if (t == "list") {
        std::string ct, it;
        ls >> ct >> it >> p.name;
        p.list = true;
        p.count_type = ptype(ct);
        p.type = ptype(it);
        if (p.count_type == PType::Bad || !is_int(p.count_type)) return SVO_ERR_INVALID;
      } else {
        p.type = ptype(t);
        ls >> p.name;
      }
      if (p.type == PType::Bad || !ls) return SVO_ERR_INVALID;
      elems.back().props.push_back(p);
    } else if (kw == "end_header") {
      break;
    }
  }
  if (!have_format) return SVO_ERR_INVALID;
  Reader r{f, binary};
  bool have_normals = false, have_colors = false;
  bool seen_vertex = false, seen_face = false;
  for (const Element& e : elems) {
    const bool is_vertex = e.name == "vertex", is_face = e.name == "face";
    int ix = -1, iy = -1, iz = -1, inx = -1, iny = -1, inz = -1, ir = -1, ig = -1, ib = -1, il = -1;
    for (int k = 0; k < (int)e.props.size(); ++k) {
      const std::string& nm = e.props[k].name;
      if (is_vertex && !e.props[k].list) {
        if (nm == "x") ix = k;
        else if (nm == "y") iy = k;
        else if (nm == "z") iz = k;
        else if (nm == "nx") inx = k;
        else if (nm == "ny") iny = k;
        else if (nm == "nz") inz = k;
        else if (nm == "red" || nm == "r") ir = k;
        else if (nm == "green" || nm == "g") ig = k;
        else if (nm == "blue" || nm == "b") ib = k;
      }
      if (is_face && e.props[k].list && (nm == "vertex_indices" || nm == "vertex_index")) il = k;
    }
    if (is_vertex) {
      if (ix < 0 || iy < 0 || iz < 0) return SVO_ERR_INVALID;
      have_normals = inx >= 0 && iny >= 0 && inz >= 0;
      have_colors = ir >= 0 && ig >= 0 && ib >= 0;
      m.v.resize(3 * e.count);
      if (have_normals) m.n.resize(3 * e.count);
      if (have_colors) m.c.resize(3 * e.count);
      seen_vertex = true;
    }
    if (is_face) {
      if (il < 0) return SVO_ERR_INVALID;
      seen_face = true;
    }
    std::vector<double> vals(e.props.size());
    std::vector<uint32_t> poly;
    for (uint64_t i = 0; i < e.count; ++i) {
      for (size_t k = 0; k < e.props.size(); ++k) {
        const Property& p = e.props[k];
        if (!p.list) {
          vals[k] = r.get(p.type);
          continue;
        }
        const double cnt = r.get(p.count_type);
        if (!r.ok || cnt < 0 || cnt > 1e6) return SVO_ERR_INVALID;
        poly.clear();
        for (uint32_t q = 0; q < (uint32_t)cnt; ++q) {
          const double idx = r.get(p.type);
          if ((int)k == il) {
            if (idx < 0) return SVO_ERR_INVALID;
            poly.push_back((uint32_t)idx);
          }
        }
        if ((int)k == il)
          for (size_t q = 2; q < poly.size(); ++q) {  // fan
            m.t.push_back(poly[0]);
            m.t.push_back(poly[q - 1]);
            m.t.push_back(poly[q]);
          }
      }
      if (!r.ok) return SVO_ERR_IO;
      if (is_vertex) {
        m.v[3 * i] = (float)vals[ix];
        m.v[3 * i + 1] = (float)vals[iy];
        m.v[3 * i + 2] = (float)vals[iz];
        if (have_normals) {
          m.n[3 * i] = (float)vals[inx];
          m.n[3 * i + 1] = (float)vals[iny];
          m.n[3 * i + 2] = (float)vals[inz];
        }
        if (have_colors) {
          const int cs[3] = {ir, ig, ib};
          for (int q = 0; q < 3; ++q)
            m.c[3 * i + q] = is_int(e.props[cs[q]].type) ? (float)(vals[cs[q]] / 255.0)
                                                         : (float)vals[cs[q]];
        }
      }
    }
  }
  if (!seen_vertex || !seen_face || m.t.empty()) return SVO_ERR_INVALID;
  const uint64_t nv = m.v.size() / 3;
  for (uint32_t idx : m.t)
    if (idx >= nv) return SVO_ERR_INVALID;
  return SVO_OK;
}

}  // namespace

extern "C" {

int svo_mesh_load_ply(const char* path, svo_mesh** out) {
  if (!path || !out) return SVO_ERR_INVALID;
  *out = nullptr;
  try {
    std::unique_ptr<svo_mesh> m(new svo_mesh);
    const int rc = load_ply(path, *m);
    if (rc != SVO_OK) return rc;
    *out = m.release();
    return SVO_OK;
  } catch (...) {
    return SVO_ERR_NOMEM;
  }
}

int svo_mesh_info(const svo_mesh* mesh, uint64_t* num_vertices, uint64_t* num_triangles,
                  uint32_t* flags) {
  if (!mesh) return SVO_ERR_INVALID;
  if (num_vertices) *num_vertices = mesh->v.size() / 3;
  if (num_triangles) *num_triangles = mesh->t.size() / 3;
  if (flags)
    *flags = (mesh->n.empty() ? 0u : SVO_MESH_HAS_NORMALS) | (mesh->c.empty() ? 0u : SVO_MESH_HAS_COLORS);
  return SVO_OK;
}

int svo_mesh_copy(const svo_mesh* mesh, float* h_vertices, float* h_normals, float* h_colors,
                  uint32_t* h_triangles) {
  if (!mesh) return SVO_ERR_INVALID;
  if ((h_normals && mesh->n.empty()) || (h_colors && mesh->c.empty())) return SVO_ERR_INVALID;
  if (h_vertices) std::memcpy(h_vertices, mesh->v.data(), mesh->v.size() * sizeof(float));
  if (h_normals) std::memcpy(h_normals, mesh->n.data(), mesh->n.size() * sizeof(float));
  if (h_colors) std::memcpy(h_colors, mesh->c.data(), mesh->c.size() * sizeof(float));
  if (h_triangles) std::memcpy(h_triangles, mesh->t.data(), mesh->t.size() * sizeof(uint32_t));
  return SVO_OK;
}

void svo_mesh_destroy(svo_mesh* mesh) { delete mesh; }

int svo_mesh_fit_unit_cube(float* h_vertices, float* h_normals, uint64_t num_vertices,
                           float rotate_x_deg) {
  if (!h_vertices || num_vertices == 0) return SVO_ERR_INVALID;
  const double a = (double)rotate_x_deg * 3.14159265358979323846 / 180.0;
  const double ca = std::cos(a), sa = std::sin(a);
  auto rot = [&](float* p) {  // about x: y' = c y - s z, z' = s y + c z
    const double y = p[1], z = p[2];
    p[1] = (float)(ca * y - sa * z);
    p[2] = (float)(sa * y + ca * z);
  };
  if (rotate_x_deg != 0.0f)
    for (uint64_t i = 0; i < num_vertices; ++i) rot(h_vertices + 3 * i);
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (uint64_t i = 0; i < num_vertices; ++i)
    for (int k = 0; k < 3; ++k) {
      const double v = h_vertices[3 * i + k];
      if (!std::isfinite(v)) return SVO_ERR_INVALID;
      lo[k] = std::fmin(lo[k], v);
      hi[k] = std::fmax(hi[k], v);
    }
  const double ext = std::fmax(hi[0] - lo[0], std::fmax(hi[1] - lo[1], hi[2] - lo[2]));
  const double s = ext > 0.0 ? 1.0 / ext : 1.0;
  for (uint64_t i = 0; i < num_vertices; ++i)
    for (int k = 0; k < 3; ++k) {
      const double c = 0.5 * (lo[k] + hi[k]);
      h_vertices[3 * i + k] = (float)((h_vertices[3 * i + k] - c) * s);
    }
  if (h_normals)
    for (uint64_t i = 0; i < num_vertices; ++i) {
      float* n = h_normals + 3 * i;
      if (rotate_x_deg != 0.0f) rot(n);
      const double l = std::sqrt((double)n[0] * n[0] + (double)n[1] * n[1] + (double)n[2] * n[2]);
      if (l > 0.0)
        for (int k = 0; k < 3; ++k) n[k] = (float)(n[k] / l);
    }
  return SVO_OK;
}

}  // extern "C"
