// Mesh file readers (host code): PLY into the arrays rq_scene_create takes.
//
// rq_mesh_read_ply follows Manta::readPlyFile (Model/Readers/PlyReader.cc:
// 135-269) on top of a PLY parser of our own (ascii, binary_little_endian,
// binary_big_endian; every PLY scalar type; list properties), with the same
// observable results:
//   * vertex x/y/z values are read as doubles and stored as floats, then
//     moved by the 3x4 transform in float, one row at a time in the order
//     m0*x, +m1*y, +m2*z, +m3 (AffineTransform::multiply_point,
//     Core/Geometry/AffineTransform.cc:357-366);
//   * a vertex is appended when the next vertex's first value arrives, and
//     the last one when the first face is read, so a file whose face
//     element is missing, empty or has no `vertex_indices` list loses its
//     last vertex, as the reference does (PlyReader.cc:30-66, 88-96);
//   * every polygon of `vertex_indices` becomes a fan (first, previous,
//     current) for its third and later vertices, each with the file's
//     material index (PlyReader.cc:98-123);
//   * degenerate triangles (Cross(a-b, c-b) == 0 in float) are removed by
//     moving the last triangle into their slot and re-testing it
//     (Mesh::removeDegenerateTriangles, Model/Groups/Mesh.cc:315-359).
// Values outside their declared type's range, truncated data and malformed
// headers are errors (the reference's reader returns false for them).
#include <cerrno>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/rfmanta_b200.h"
#include "rq_mesh.h"

namespace rq {
void set_error(const std::string& msg);
}


namespace {

enum PlyType { kInt8, kUInt8, kInt16, kUInt16, kInt32, kUInt32, kFloat32, kFloat64, kBad };

PlyType ply_type(const std::string& s) {
  if (s == "char" || s == "int8") return kInt8;
  if (s == "uchar" || s == "uint8") return kUInt8;
  if (s == "short" || s == "int16") return kInt16;
  if (s == "ushort" || s == "uint16") return kUInt16;
  if (s == "int" || s == "int32") return kInt32;
  if (s == "uint" || s == "uint32") return kUInt32;
  if (s == "float" || s == "float32") return kFloat32;
  if (s == "double" || s == "float64") return kFloat64;
  return kBad;
}

int type_size(PlyType t) {
  switch (t) {
    case kInt8: case kUInt8: return 1;
    case kInt16: case kUInt16: return 2;
    case kInt32: case kUInt32: case kFloat32: return 4;
    case kFloat64: return 8;
    default: return 0;
  }
}

struct Property {
  std::string name;
  bool list = false;
  PlyType count_type = kBad, type = kBad;
};

struct Element {
  std::string name;
  long count = 0;
  std::vector<Property> props;
};

enum Format { kAscii, kBinLE, kBinBE };

// Value source over the file's body.
class Reader {
 public:
  Reader(const std::vector<char>& buf, size_t pos, Format f) : b_(buf), p_(pos), f_(f) {}

  bool value(PlyType t, double* out) {
    return f_ == kAscii ? ascii(t, out) : binary(t, out);
  }

 private:
  bool word(std::string& w) {
    while (p_ < b_.size() && std::isspace((unsigned char)b_[p_])) ++p_;
    const size_t s = p_;
    while (p_ < b_.size() && !std::isspace((unsigned char)b_[p_])) ++p_;
    if (p_ == s) return false;
    w.assign(&b_[s], p_ - s);
    return true;
  }

  bool ascii(PlyType t, double* out) {
    std::string w;
    if (!word(w)) return false;
    char* end = nullptr;
    if (t == kFloat32 || t == kFloat64) {
      const double v = std::strtod(w.c_str(), &end);
      if (*end) return false;
      const double lim = t == kFloat32 ? FLT_MAX : DBL_MAX;
      if (v < -lim || v > lim) return false;
      *out = v;
      return true;
    }
    const long v = std::strtol(w.c_str(), &end, 10);
    if (*end) return false;
    const double d = (double)v;
    switch (t) {
      case kInt8: if (d > CHAR_MAX || d < CHAR_MIN) return false; break;
      case kUInt8: if (d > UCHAR_MAX || d < 0) return false; break;
      case kInt16: if (d > SHRT_MAX || d < SHRT_MIN) return false; break;
      case kUInt16: if (d > USHRT_MAX || d < 0) return false; break;
      case kInt32: break;
      case kUInt32: if (d < 0) return false; break;
      default: return false;
    }
    *out = d;
    return true;
  }

  bool binary(PlyType t, double* out) {
    const int n = type_size(t);
    if (n == 0 || p_ + n > b_.size()) return false;
    unsigned char raw[8];
    std::memcpy(raw, &b_[p_], n);
    p_ += n;
    const bool little = f_ == kBinLE;
    if (!little)
      for (int i = 0; i < n / 2; ++i) std::swap(raw[i], raw[n - 1 - i]);
    switch (t) {
      case kInt8: { int8_t v; std::memcpy(&v, raw, 1); *out = v; break; }
      case kUInt8: { uint8_t v; std::memcpy(&v, raw, 1); *out = v; break; }
      case kInt16: { int16_t v; std::memcpy(&v, raw, 2); *out = v; break; }
      case kUInt16: { uint16_t v; std::memcpy(&v, raw, 2); *out = v; break; }
      case kInt32: { int32_t v; std::memcpy(&v, raw, 4); *out = v; break; }
      case kUInt32: { uint32_t v; std::memcpy(&v, raw, 4); *out = v; break; }
      case kFloat32: { float v; std::memcpy(&v, raw, 4); *out = v; break; }
      case kFloat64: { double v; std::memcpy(&v, raw, 8); *out = v; break; }
      default: return false;
    }
    return true;
  }

  const std::vector<char>& b_;
  size_t p_;
  Format f_;
};

int fail(int code, const std::string& m) {
  rq::set_error(m);
  return code;
}

// Parses the header; returns the offset of the body.
int parse_header(const std::vector<char>& buf, Format& fmt, std::vector<Element>& elems,
                 size_t& body) {
  size_t p = 0;
  auto line = [&](std::string& out) -> bool {
    if (p >= buf.size()) return false;
    const size_t s = p;
    while (p < buf.size() && buf[p] != '\n') ++p;
    out.assign(&buf[s], p - s);
    if (p < buf.size()) ++p;  // the newline
    if (!out.empty() && out.back() == '\r') out.pop_back();
    return true;
  };
  std::string l;
  if (!line(l) || l != "ply") return fail(RQ_ERR_FORMAT, "not a PLY file");
  bool have_format = false;
  for (;;) {
    if (!line(l)) return fail(RQ_ERR_FORMAT, "PLY header without end_header");
    std::istringstream ss(l);
    std::string kw;
    if (!(ss >> kw)) continue;
    if (kw == "end_header") break;
    if (kw == "comment" || kw == "obj_info") continue;
    if (kw == "format") {
      std::string f, ver;
      ss >> f >> ver;
      if (f == "ascii") fmt = kAscii;
      else if (f == "binary_little_endian") fmt = kBinLE;
      else if (f == "binary_big_endian") fmt = kBinBE;
      else return fail(RQ_ERR_FORMAT, "unknown PLY format '" + f + "'");
      have_format = true;
    } else if (kw == "element") {
      Element e;
      if (!(ss >> e.name >> e.count) || e.count < 0)
        return fail(RQ_ERR_FORMAT, "bad PLY element line: " + l);
      elems.push_back(e);
    } else if (kw == "property") {
      if (elems.empty()) return fail(RQ_ERR_FORMAT, "PLY property before any element");
      Property pr;
      std::string t;
      if (!(ss >> t)) return fail(RQ_ERR_FORMAT, "bad PLY property line: " + l);
      if (t == "list") {
        std::string ct, it;
        if (!(ss >> ct >> it >> pr.name)) return fail(RQ_ERR_FORMAT, "bad PLY list property: " + l);
        pr.list = true;
        pr.count_type = ply_type(ct);
        pr.type = ply_type(it);
        if (pr.count_type == kBad || pr.type == kBad)
          return fail(RQ_ERR_FORMAT, "unknown PLY type in: " + l);
      } else {
        pr.type = ply_type(t);
        if (pr.type == kBad || !(ss >> pr.name))
          return fail(RQ_ERR_FORMAT, "bad PLY property line: " + l);
      }
      elems.back().props.push_back(pr);
    } else {
      return fail(RQ_ERR_FORMAT, "unknown PLY header line: " + l);
    }
  }
  if (!have_format) return fail(RQ_ERR_FORMAT, "PLY header has no format line");
  body = p;
  return RQ_OK;
}

// State of the reference reader's vertex / face callbacks.
struct PlyBuild {
  const float* m;  // 3x4 row-major transform
  uint32_t material;
  float point[3] = {0.f, 0.f, 0.f};
  long first = 0, prev = 0;
  rq_mesh* mesh;

  void add_vertex() {
    float r[3];
    for (int i = 0; i < 3; ++i) {
      float acc = m[4 * i + 0] * point[0];
      acc += m[4 * i + 1] * point[1];
      acc += m[4 * i + 2] * point[2];
      acc += m[4 * i + 3];
      r[i] = acc;
    }
    for (int i = 0; i < 3; ++i) {
      point[i] = r[i];
      mesh->vertices.push_back(r[i]);
    }
  }
};

}  // namespace

// Mesh::removeDegenerateTriangles.
void rq_mesh_remove_degenerate(rq_mesh* m) {
  std::vector<uint32_t>& vi = m->indices;
  const float* v = m->vertices.data();
  for (size_t i = 0; i < vi.size(); i += 3) {
    const float* a = v + 3 * (size_t)vi[i + 0];
    const float* b = v + 3 * (size_t)vi[i + 1];
    const float* c = v + 3 * (size_t)vi[i + 2];
    const float ab[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
    const float cb[3] = {c[0] - b[0], c[1] - b[1], c[2] - b[2]};
    const float x = ab[1] * cb[2] - ab[2] * cb[1];
    const float y = ab[2] * cb[0] - ab[0] * cb[2];
    const float z = ab[0] * cb[1] - ab[1] * cb[0];
    if (x == 0.f && y == 0.f && z == 0.f) {
      const size_t n = vi.size();
      vi[i + 0] = vi[n - 3];
      vi[i + 1] = vi[n - 2];
      vi[i + 2] = vi[n - 1];
      vi.resize(n - 3);
      m->face_material[i / 3] = m->face_material.back();
      m->face_material.pop_back();
      i -= 3;  // re-test the triangle moved into this slot (wraps at 0)
    }
  }
}

extern "C" {

int rq_mesh_read_ply(const char* path, const float* transform, uint32_t material,
                     rq_mesh** out) {
  if (!out || !path) return fail(RQ_ERR_ARG, "NULL argument");
  *out = nullptr;
  std::ifstream in(path, std::ios::binary);
  if (!in) return fail(RQ_ERR_NOTFOUND, std::string("cannot open ") + path);
  std::vector<char> buf((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  Format fmt = kAscii;
  std::vector<Element> elems;
  size_t body = 0;
  int rc = parse_header(buf, fmt, elems, body);
  if (rc != RQ_OK) return rc;
  static const float kIdentity[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
  std::unique_ptr<rq_mesh> mesh(new rq_mesh());
  PlyBuild st;
  st.m = transform ? transform : kIdentity;
  st.material = material;
  st.mesh = mesh.get();
  Reader rd(buf, body, fmt);
  for (const Element& e : elems) {
    const bool is_vertex = e.name == "vertex";
    const bool is_face = e.name == "face";
    for (long k = 0; k < e.count; ++k) {
      for (const Property& pr : e.props) {
        if (!pr.list) {
          double v;
          if (!rd.value(pr.type, &v)) return fail(RQ_ERR_FORMAT, "PLY data ends early or is malformed");
          if (!is_vertex) continue;
          const int axis = pr.name == "x" ? 0 : pr.name == "y" ? 1 : pr.name == "z" ? 2 : -1;
          const bool watched = axis >= 0 || pr.name == "diffuse_red" ||
                               pr.name == "diffuse_green" || pr.name == "diffuse_blue";
          if (!watched) continue;
          // PlyReader's vertex_cb: the previous vertex is complete once the
          // next one's first watched value arrives
          if ((size_t)k == mesh->vertices.size() / 3 + 1) st.add_vertex();
          if (axis >= 0) st.point[axis] = (float)v;
          continue;
        }
        double cnt;
        if (!rd.value(pr.count_type, &cnt)) return fail(RQ_ERR_FORMAT, "PLY list count missing");
        const bool watched = is_face && pr.name == "vertex_indices";
        if (watched && k == 0) st.add_vertex();  // face_cb, first face, length value
        const long n = (long)cnt;
        for (long j = 0; j < n; ++j) {
          double v;
          if (!rd.value(pr.type, &v)) return fail(RQ_ERR_FORMAT, "PLY list data ends early");
          if (!watched) continue;
          const long cur = (long)v;
          if (j == 0) {
            st.first = cur;
          } else if (j == 1) {
            st.prev = cur;
          } else {
            mesh->indices.push_back((uint32_t)st.first);
            mesh->indices.push_back((uint32_t)st.prev);
            mesh->indices.push_back((uint32_t)cur);
            mesh->face_material.push_back(material);
            st.prev = cur;
          }
        }
      }
    }
  }
  const size_t nv = mesh->vertices.size() / 3;
  for (uint32_t i : mesh->indices)
    if (i >= nv) return fail(RQ_ERR_FORMAT, "PLY face refers to a missing vertex");
  rq_mesh_remove_degenerate(mesh.get());
  *out = mesh.release();
  return RQ_OK;
}

int rq_mesh_info(const rq_mesh* m, int* n_vertices, int* n_tris) {
  if (!m) return fail(RQ_ERR_ARG, "NULL mesh");
  if (n_vertices) *n_vertices = (int)(m->vertices.size() / 3);
  if (n_tris) *n_tris = (int)(m->indices.size() / 3);
  return RQ_OK;
}

int rq_mesh_copy(const rq_mesh* m, float* vertices, uint32_t* indices, uint32_t* face_material) {
  if (!m) return fail(RQ_ERR_ARG, "NULL mesh");
  if (vertices) std::memcpy(vertices, m->vertices.data(), m->vertices.size() * sizeof(float));
  if (indices) std::memcpy(indices, m->indices.data(), m->indices.size() * sizeof(uint32_t));
  if (face_material)
    std::memcpy(face_material, m->face_material.data(),
                m->face_material.size() * sizeof(uint32_t));
  return RQ_OK;
}

int rq_mesh_material_count(const rq_mesh* m, int* n) {
  if (!m || !n) return fail(RQ_ERR_ARG, "NULL argument");
  *n = (int)m->materials.size();
  return RQ_OK;
}

int rq_mesh_materials(const rq_mesh* m, int32_t* kind, float* diffuse, float* specular,
                      int32_t* exponent, float* reflectivity, float* refraction, float* alpha,
                      float* filter) {
  if (!m) return fail(RQ_ERR_ARG, "NULL mesh");
  for (size_t i = 0; i < m->materials.size(); ++i) {
    const rq_mesh_material& q = m->materials[i];
    if (kind) kind[i] = q.kind;
    for (int c = 0; c < 3; ++c) {
      if (diffuse) diffuse[3 * i + c] = q.diffuse[c];
      if (specular) specular[3 * i + c] = q.specular[c];
      if (filter) filter[3 * i + c] = q.filter[c];
    }
    if (exponent) exponent[i] = q.exponent;
    if (reflectivity) reflectivity[i] = q.reflectivity;
    if (refraction) refraction[i] = q.refraction;
    if (alpha) alpha[i] = q.alpha;
  }
  return RQ_OK;
}

int rq_mesh_destroy(rq_mesh* m) {
  delete m;
  return RQ_OK;
}

}  // extern "C"
