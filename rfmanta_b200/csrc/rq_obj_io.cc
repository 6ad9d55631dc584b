// Wavefront OBJ + MTL reading (host code) into the arrays rq_scene_create
// takes, with the observable results of Manta::ObjGroup
// (Model/Groups/ObjGroup.cc:176-320) over the glm reader it uses
// (Model/Readers/glm/glm.cc: _glmFirstPass 574-750, _glmSecondPass
// 755-1010, _glmReadMTL 275-512):
//   * statements are read token by token; a statement is chosen by the
//     token's first character ('v' vertex data, 'f' face, 'g'/'o' group,
//     'u' usemtl, 'm' mtllib, '#' comment; anything else skips its line),
//     so e.g. any token starting with 'm' names a material library;
//   * a name taken from the rest of a line is its second word when it has
//     two or more, else its first (the reference's sscanf("%s %s", buf,
//     buf)); a group name is the first word;
//   * faces go to the group named "<group>_MAT_<material>" (initially
//     "No Group" / "No Material"); groups are emitted newest first (glm
//     prepends each new group to its list) and each group's faces in file
//     order; polygons become fans (first, previous last, current); a
//     negative vertex index counts back from the vertices read so far;
//   * each face's material is its group's glm material + 1 (0 when the
//     model has no material library), a group's glm material being the
//     one current at the last g/o/usemtl statement naming it (a usemtl of
//     an unknown name selects glm material 0, "NO_ASSIGNED_MATERIAL");
//   * degenerate triangles are removed as Mesh::removeDegenerateTriangles
//     does (shared with the PLY reader);
//   * the material table is the one ObjGroup::create_materials builds
//     (ObjGroup.cc:70-172): index 0 is ObjGroup's default material,
//     index i + 1 glm material i, classified Dielectric (Ni not 0 or 1),
//     Transparent (Tf/Tr not white, or d < 1), Phong (Ns != 0, exponent
//     int(Ns)) or Lambertian, with glm's defaults (Kd 0.8, Ks 0, Ns 0,
//     Ni 1, d 1, Tf 1, reflectivity 0).  Texture maps are not loaded: the
//     constant colours stand, as ObjGroup does when an image fails to load.
// Deliberate differences, where the reference's behaviour is undefined:
// a vertex line with more than three values (glm takes a fourth integer
// as the start of per-vertex colours and misreads the rest of the file),
// a vertex index that is 0 or past the vertices read, and faces that come
// before the first group or material statement in a file that has such
// statements later (glm writes those past the end of a group's triangle
// array) are errors here, or in the last case belong to the default group.
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include "../../include/rfmanta_b200.h"
#include "rq_mesh.h"

namespace rq {
void set_error(const std::string& msg);
}

namespace {

int fail(int code, const std::string& m) {
  rq::set_error(m);
  return code;
}

bool is_space(char c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f';
}

// A character stream read the way glm reads it with fscanf / fgets.
struct Scan {
  const std::string& s;
  size_t p = 0;
  explicit Scan(const std::string& text) : s(text) {}

  void skip_space() {
    while (p < s.size() && is_space(s[p])) ++p;
  }
  // fscanf("%s")
  bool token(std::string& out) {
    skip_space();
    if (p >= s.size()) return false;
    const size_t a = p;
    while (p < s.size() && !is_space(s[p])) ++p;
    out.assign(s, a, p - a);
    return true;
  }
  // fgets: the rest of the line, newline included
  std::string rest_of_line() {
    const size_t a = p;
    while (p < s.size() && s[p] != '\n') ++p;
    if (p < s.size()) ++p;
    return s.substr(a, p - a);
  }
  // fscanf("%d"); false (nothing consumed past the blanks) when no digits
  bool read_int(long& v) {
    skip_space();
    if (p >= s.size()) return false;
    const char* b = s.c_str() + p;
    char* e = nullptr;
    v = std::strtol(b, &e, 10);
    if (e == b) return false;
    p += (size_t)(e - b);
    return true;
  }
  // fscanf("%f")
  bool read_float(float& v) {
    skip_space();
    if (p >= s.size()) return false;
    const char* b = s.c_str() + p;
    char* e = nullptr;
    v = std::strtof(b, &e);
    if (e == b) return false;
    p += (size_t)(e - b);
    return true;
  }
  bool literal(char c) {
    if (p < s.size() && s[p] == c) {
      ++p;
      return true;
    }
    return false;
  }
};

std::vector<std::string> words(const std::string& line) {
  std::vector<std::string> w;
  size_t i = 0;
  while (i < line.size()) {
    while (i < line.size() && is_space(line[i])) ++i;
    const size_t a = i;
    while (i < line.size() && !is_space(line[i])) ++i;
    if (i > a) w.push_back(line.substr(a, i - a));
  }
  return w;
}

// sscanf(buf, "%s %s", buf, buf) on the rest of a line
std::string second_or_first_word(const std::string& rest) {
  const std::vector<std::string> w = words(rest);
  if (w.size() >= 2) return w[1];
  if (w.size() == 1) return w[0];
  return rest;
}

// sscanf(buf, "%s", buf)
std::string first_word(const std::string& rest) {
  const std::vector<std::string> w = words(rest);
  return w.empty() ? rest : w[0];
}

bool read_file(const std::string& path, std::string& out) {
  std::ifstream in(path, std::ios::binary);
  if (!in) return false;
  out.assign(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
  return true;
}

struct GlmMaterial {
  std::string name;
  float diffuse[3] = {0.8f, 0.8f, 0.8f};
  float specular[3] = {0.f, 0.f, 0.f};
  float filter[3] = {1.f, 1.f, 1.f};
  float shininess = 0.f, refraction = 1.f, alpha = 1.f, reflectivity = 0.f;
};

// _glmReadMTL: material 0 is "NO_ASSIGNED_MATERIAL", then one per newmtl.
int read_mtl(const std::string& path, std::vector<GlmMaterial>& mats) {
  std::string text;
  if (!read_file(path, text))
    return fail(RQ_ERR_NOTFOUND, "cannot open material library " + path);
  mats.assign(1, GlmMaterial());
  mats[0].name = "NO_ASSIGNED_MATERIAL";
  Scan sc(text);
  std::string tok;
  size_t cur = 0;
  auto floats = [&](float* dst, int n) {
    for (int i = 0; i < n; ++i)
      if (!sc.read_float(dst[i])) return;
  };
  while (sc.token(tok)) {
    GlmMaterial& m = mats[cur];
    switch (tok[0]) {
      case 'n':
        mats.push_back(GlmMaterial());
        cur = mats.size() - 1;
        mats[cur].name = second_or_first_word(sc.rest_of_line());
        break;
      case 'N':
        if (tok.size() > 1 && tok[1] == 's') floats(&m.shininess, 1);
        else if (tok.size() > 1 && tok[1] == 'i') floats(&m.refraction, 1);
        else sc.rest_of_line();
        break;
      case 'T':
        if (tok.size() > 1 && tok[1] == 'r') {
          floats(&m.filter[0], 1);
          m.filter[2] = m.filter[1] = m.filter[0];
        } else if (tok.size() > 1 && tok[1] == 'f') {
          floats(m.filter, 3);
        } else {
          sc.rest_of_line();
        }
        break;
      case 'd':
        floats(&m.alpha, 1);
        break;
      case 'i': {
        long shader;
        sc.read_int(shader);
        break;
      }
      case 'r':
        floats(&m.reflectivity, 1);
        break;
      case 'm':
        if (tok == "map_Ka" || tok == "map_Kd" || tok == "map_Ks" || tok == "map_D") {
          std::string name;
          sc.token(name);
          if (name == "-s") {
            float s[2];
            floats(s, 2);
            sc.token(name);
          }
        }
        break;  // an unknown map keeps the rest of its line, as glm does
      case 'K':
        if (tok.size() > 1 && tok[1] == 'd') floats(m.diffuse, 3);
        else if (tok.size() > 1 && tok[1] == 's') floats(m.specular, 3);
        else if (tok.size() > 1 && tok[1] == 'a') {
          float a[3];
          floats(a, 3);
        } else {
          sc.rest_of_line();
        }
        break;
      default:
        sc.rest_of_line();
        break;
    }
  }
  return RQ_OK;
}

struct Group {
  std::string name;
  // the material name current at the last g/o/usemtl naming this group
  // (none before the first usemtl: glm material 0), resolved against the
  // material library once the whole file is read, as glm's second pass does
  bool has_material = false;
  std::string material;
  std::vector<uint32_t> tris;  // 3 vertex indices (1-based, resolved) per triangle
};

}  // namespace

extern "C" int rq_mesh_read_obj(const char* path, rq_mesh** out) {
  if (!out || !path) return fail(RQ_ERR_ARG, "NULL argument");
  *out = nullptr;
  std::string text;
  if (!read_file(path, text)) return fail(RQ_ERR_NOTFOUND, std::string("cannot open ") + path);
  std::string dir(path);
  const size_t slash = dir.rfind('/');
  dir = slash == std::string::npos ? std::string() : dir.substr(0, slash + 1);

  std::unique_ptr<rq_mesh> mesh(new rq_mesh());
  std::vector<GlmMaterial> mats;
  bool have_mtl = false;
  std::vector<Group> groups;  // in creation order
  auto find_group = [&](const std::string& name) -> int {
    for (size_t i = 0; i < groups.size(); ++i)
      if (groups[i].name == name) return (int)i;
    groups.push_back(Group());
    groups.back().name = name;
    return (int)groups.size() - 1;
  };
  find_group("No Group");
  std::string grpname = "No Group", mtlname = "No Material";
  bool have_usemtl = false;
  int group = 0;
  long nverts = 0;
  Scan sc(text);
  std::string tok;
  auto vindex = [&](long v, uint32_t* o) -> bool {
    const long r = v >= 0 ? v : nverts + 1 + v;  // glm: numvertices counts from 1
    if (r < 1 || r > nverts) return false;
    *o = (uint32_t)r;
    return true;
  };
  while (sc.token(tok)) {
    switch (tok[0]) {
      case '#':
        sc.rest_of_line();
        break;
      case 'v':
        if (tok.size() == 1) {
          // x y z; a fourth value glm would read as an integer starts its
          // per-vertex colours (and w), which it then misreads
          const std::string rest = sc.rest_of_line();
          const char* q = rest.c_str();
          for (int c = 0; c < 3; ++c) {
            char* e = nullptr;
            const float x = std::strtof(q, &e);
            if (e == q) return fail(RQ_ERR_FORMAT, "OBJ vertex needs three numbers");
            mesh->vertices.push_back(x);
            q = e;
          }
          char* e = nullptr;
          std::strtol(q, &e, 10);
          if (e != q)
            return fail(RQ_ERR_FORMAT, "OBJ vertex with a fourth value (w or colours)");
          ++nverts;
        } else if (tok == "vn" || tok == "vt") {
          sc.rest_of_line();
        }
        break;
      case 'm': {
        const std::string name = second_or_first_word(sc.rest_of_line());
        const int rc = read_mtl(dir + name, mats);
        if (rc != RQ_OK) return rc;
        have_mtl = true;
        break;
      }
      case 'u':
        mtlname = second_or_first_word(sc.rest_of_line());
        have_usemtl = true;
        group = find_group(grpname + "_MAT_" + mtlname);
        groups[group].has_material = true;
        groups[group].material = mtlname;
        break;
      case 'o':
      case 'g':
        grpname = first_word(sc.rest_of_line());
        group = find_group(grpname + "_MAT_" + mtlname);
        groups[group].has_material = have_usemtl;
        groups[group].material = mtlname;
        break;
      case 'f': {
        // the first vertex's form fixes the face's: v//n, v/t/n, v/t or v
        std::string first;
        if (!sc.token(first)) break;
        int form = 0;
        long a = 0, b = 0, c = 0;
        char* e = nullptr;
        if (first.find("//") != std::string::npos) form = 1;
        else if (std::sscanf(first.c_str(), "%ld/%ld/%ld", &a, &b, &c) == 3) form = 2;
        else if (std::sscanf(first.c_str(), "%ld/%ld", &a, &b) == 2) form = 3;
        a = std::strtol(first.c_str(), &e, 10);
        if (e == first.c_str()) return fail(RQ_ERR_FORMAT, "OBJ face vertex is not a number");
        // reads one vertex of the face's form; false when none follows
        auto next = [&](long& v) -> bool {
          long x;
          if (!sc.read_int(v)) return false;
          if (form == 1) {
            if (sc.literal('/') && sc.literal('/')) sc.read_int(x);
          } else if (form == 2) {
            if (sc.literal('/') && sc.read_int(x) && sc.literal('/')) sc.read_int(x);
          } else if (form == 3) {
            if (sc.literal('/')) sc.read_int(x);
          }
          return true;
        };
        long v1, v2;
        if (!next(v1) || !next(v2)) return fail(RQ_ERR_FORMAT, "OBJ face with fewer than three vertices");
        uint32_t f0, fprev, fcur;
        if (!vindex(a, &f0) || !vindex(v1, &fprev) || !vindex(v2, &fcur))
          return fail(RQ_ERR_FORMAT, "OBJ face refers to a missing vertex");
        std::vector<uint32_t>& t = groups[group].tris;
        t.insert(t.end(), {f0, fprev, fcur});
        long v;
        while (next(v)) {
          fprev = fcur;
          if (!vindex(v, &fcur)) return fail(RQ_ERR_FORMAT, "OBJ face refers to a missing vertex");
          t.insert(t.end(), {f0, fprev, fcur});
        }
        break;
      }
      default:
        sc.rest_of_line();
        break;
    }
  }
  // ObjGroup walks glm's list, newest group first
  const unsigned nmat = have_mtl ? (unsigned)mats.size() : 0u;
  for (size_t gi = groups.size(); gi-- > 0;) {
    const Group& g = groups[gi];
    unsigned gm = 0;  // _glmFindMaterial: unknown names select material 0
    if (g.has_material)
      for (size_t i = 0; i < mats.size(); ++i)
        if (mats[i].name == g.material) {
          gm = (unsigned)i;
          break;
        }
    const uint32_t fm = gm < nmat ? gm + 1 : 0;
    for (size_t k = 0; k < g.tris.size(); k += 3) {
      for (int j = 0; j < 3; ++j) mesh->indices.push_back(g.tris[k + j] - 1);
      mesh->face_material.push_back(fm);
    }
  }
  // ObjGroup::create_materials
  mesh->materials.assign(1 + nmat, rq_mesh_material());
  rq_mesh_material& d = mesh->materials[0];
  d.kind = RQ_MAT_DEFAULT;
  for (unsigned i = 0; i < nmat; ++i) {
    const GlmMaterial& g = mats[i];
    rq_mesh_material& m = mesh->materials[i + 1];
    for (int c = 0; c < 3; ++c) {
      m.diffuse[c] = g.diffuse[c];
      m.specular[c] = g.specular[c];
      m.filter[c] = g.filter[c];
    }
    m.refraction = g.refraction;
    m.alpha = g.alpha;
    m.reflectivity = g.reflectivity;
    m.exponent = (int32_t)g.shininess;
    const bool white = g.filter[0] == 1.f && g.filter[1] == 1.f && g.filter[2] == 1.f;
    if (g.refraction != 1.f && g.refraction != 0.f) m.kind = RQ_MAT_DIELECTRIC;
    else if (!white || g.alpha < 1.f) m.kind = RQ_MAT_TRANSPARENT;
    else if (g.shininess != 0.f) m.kind = RQ_MAT_PHONG;
    else m.kind = RQ_MAT_LAMBERTIAN;
  }
  rq_mesh_remove_degenerate(mesh.get());
  *out = mesh.release();
  return RQ_OK;
}
