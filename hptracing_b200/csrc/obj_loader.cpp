// Wavefront OBJ/MTL reader, material probabilities and light table.
//
// Parser semantics follow the tinyobjloader copy vendored by the reference
// (src/objloader/tiny_obj_loader.cpp), including its quirks, because they
// decide which triangles, vertices and materials the renderer sees:
//  - faces are fan-triangulated (:249-266) and vertices are re-indexed per
//    exported face group by their (v, vt, vn) triple (:165-203);
//  - 'usemtl' clears the pending face group without exporting it (:629);
//  - 'g' / 'o' / end of file export the pending group as one shape;
//  - 'Tr' and the patched 'Tf' both set dissolve directly (:419-429);
//  - 'Ke' is the emission (:388-396).
// The arrays are then assembled as hp::Scene::Scene does
// (src/hp/scene/base.cpp:37-158).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>

#include "host.h"

namespace hpt {

namespace {

thread_local std::string g_error;

struct VIdx {
  int v, vt, vn;
};
bool operator<(const VIdx& a, const VIdx& b) {  // tiny_obj_loader.cpp:43-50
  if (a.v != b.v) return a.v < b.v;
  if (a.vn != b.vn) return a.vn < b.vn;
  if (a.vt != b.vt) return a.vt < b.vt;
  return false;
}

struct ObjMaterial {
  std::string name;
  float ambient[3], diffuse[3], specular[3], transmittance[3], emission[3];
  float shininess, ior, dissolve;
  int illum;
  std::string ambient_texname, diffuse_texname;
};

void init_material(ObjMaterial& m) {  // tiny_obj_loader.cpp:205-223
  m.name.clear();
  m.ambient_texname.clear();
  m.diffuse_texname.clear();
  for (int i = 0; i < 3; ++i)
    m.ambient[i] = m.diffuse[i] = m.specular[i] = m.transmittance[i] =
        m.emission[i] = 0.f;
  m.illum = 0;
  m.dissolve = 1.f;
  m.shininess = 1.f;
  m.ior = 1.f;
}

struct Shape {
  std::vector<float> positions, normals, texcoords;
  std::vector<int> indices, material_ids;
};

bool is_space(char c) { return c == ' ' || c == '\t'; }
bool is_newline(char c) { return c == '\r' || c == '\n' || c == '\0'; }

int fix_index(int idx, int n) {  // tiny_obj_loader.cpp:67-79
  if (idx > 0) return idx - 1;
  if (idx == 0) return 0;
  return n + idx;
}

float parse_float(const char*& t) {
  t += strspn(t, " \t");
  float f = (float)atof(t);
  t += strcspn(t, " \t\r");
  return f;
}

int parse_int(const char*& t) {
  t += strspn(t, " \t");
  int i = atoi(t);
  t += strcspn(t, " \t\r");
  return i;
}

VIdx parse_triple(const char*& t, int vsize, int vnsize, int vtsize) {
  VIdx vi{-1, -1, -1};  // tiny_obj_loader.cpp:127-162
  vi.v = fix_index(atoi(t), vsize);
  t += strcspn(t, "/ \t\r");
  if (t[0] != '/') return vi;
  t++;
  if (t[0] == '/') {
    t++;
    vi.vn = fix_index(atoi(t), vnsize);
    t += strcspn(t, "/ \t\r");
    return vi;
  }
  vi.vt = fix_index(atoi(t), vtsize);
  t += strcspn(t, "/ \t\r");
  if (t[0] != '/') return vi;
  t++;
  vi.vn = fix_index(atoi(t), vnsize);
  t += strcspn(t, "/ \t\r");
  return vi;
}

// Reads lines the way the reference does: getline, strip one trailing
// '\n' then one trailing '\r'.
bool next_line(std::istream& in, std::string& line) {
  if (in.peek() == EOF) return false;
  std::getline(in, line);
  if (!line.empty() && line.back() == '\n') line.pop_back();
  if (!line.empty() && line.back() == '\r') line.pop_back();
  return true;
}

void load_mtl(std::istream& in, std::map<std::string, int>& material_map,
              std::vector<ObjMaterial>& materials) {
  // tiny_obj_loader.cpp:278-476. The reference leaves the first material
  // uninitialised when the file has no 'newmtl'; it is initialised here.
  material_map.clear();
  ObjMaterial m;
  init_material(m);
  std::string line;
  while (next_line(in, line)) {
    if (line.empty()) continue;
    const char* t = line.c_str();
    t += strspn(t, " \t");
    if (t[0] == '\0' || t[0] == '#') continue;
    if (!strncmp(t, "newmtl", 6) && is_space(t[6])) {
      if (!m.name.empty()) {
        material_map.insert({m.name, (int)materials.size()});
        materials.push_back(m);
      }
      init_material(m);
      char name[4096] = {0};
      sscanf(t + 7, "%4095s", name);
      m.name = name;
      continue;
    }
    auto f3 = [&](float* dst) {
      t += 2;
      dst[0] = parse_float(t);
      dst[1] = parse_float(t);
      dst[2] = parse_float(t);
    };
    if (t[0] == 'K' && t[1] == 'a' && is_space(t[2])) { f3(m.ambient); continue; }
    if (t[0] == 'K' && t[1] == 'd' && is_space(t[2])) { f3(m.diffuse); continue; }
    if (t[0] == 'K' && t[1] == 's' && is_space(t[2])) { f3(m.specular); continue; }
    if (t[0] == 'K' && t[1] == 't' && is_space(t[2])) { f3(m.transmittance); continue; }
    if (t[0] == 'N' && t[1] == 'i' && is_space(t[2])) { t += 2; m.ior = parse_float(t); continue; }
    if (t[0] == 'K' && t[1] == 'e' && is_space(t[2])) { f3(m.emission); continue; }
    if (t[0] == 'N' && t[1] == 's' && is_space(t[2])) { t += 2; m.shininess = parse_float(t); continue; }
    if (!strncmp(t, "illum", 5) && is_space(t[5])) { t += 6; m.illum = parse_int(t); continue; }
    if (t[0] == 'd' && is_space(t[1])) { t += 1; m.dissolve = parse_float(t); continue; }
    if (t[0] == 'T' && (t[1] == 'r' || t[1] == 'f') && is_space(t[2])) {
      t += 2;
      m.dissolve = parse_float(t);
      continue;
    }
    if (!strncmp(t, "map_Ka", 6) && is_space(t[6])) { m.ambient_texname = t + 7; continue; }
    if (!strncmp(t, "map_Kd", 6) && is_space(t[6])) { m.diffuse_texname = t + 7; continue; }
    // map_Ks, map_Ns and unknown keys do not reach the renderer.
  }
  material_map.insert({m.name, (int)materials.size()});
  materials.push_back(m);
}

// tiny_obj_loader.cpp:226-276. The vertex cache starts empty for every
// exported group (the reference passes it by value).
bool export_group(Shape& shape, const std::vector<float>& v,
                  const std::vector<float>& vn, const std::vector<float>& vt,
                  const std::vector<std::vector<VIdx>>& group, int material,
                  std::string& err) {
  if (group.empty()) return false;
  std::map<VIdx, int> cache;
  auto update = [&](const VIdx& i) -> int {
    auto it = cache.find(i);
    if (it != cache.end()) return it->second;
    if (i.v < 0 || 3 * (size_t)i.v + 2 >= v.size() ||
        (i.vn >= 0 && 3 * (size_t)i.vn + 2 >= vn.size()) ||
        (i.vt >= 0 && 2 * (size_t)i.vt + 1 >= vt.size())) {
      err = "face references a missing vertex/normal/texcoord";
      return 0;
    }
    shape.positions.insert(shape.positions.end(), &v[3 * i.v], &v[3 * i.v] + 3);
    if (i.vn >= 0)
      shape.normals.insert(shape.normals.end(), &vn[3 * i.vn], &vn[3 * i.vn] + 3);
    if (i.vt >= 0)
      shape.texcoords.insert(shape.texcoords.end(), &vt[2 * i.vt], &vt[2 * i.vt] + 2);
    int idx = (int)(shape.positions.size() / 3) - 1;
    cache[i] = idx;
    return idx;
  };
  for (const auto& face : group) {
    if (face.size() < 2) continue;
    VIdx i0 = face[0], i1{-1, -1, -1}, i2 = face[1];
    for (size_t k = 2; k < face.size(); ++k) {  // fan triangulation
      i1 = i2;
      i2 = face[k];
      int a = update(i0), b = update(i1), c = update(i2);
      shape.indices.push_back(a);
      shape.indices.push_back(b);
      shape.indices.push_back(c);
      shape.material_ids.push_back(material);
    }
  }
  return true;
}

std::string parse_obj(std::istream& in, const std::string& basepath,
                      std::vector<Shape>& shapes,
                      std::vector<ObjMaterial>& materials) {
  std::vector<float> v, vn, vt;
  std::vector<std::vector<VIdx>> group;
  std::map<std::string, int> material_map;
  int material = -1;
  Shape shape;
  std::string line, err;
  auto flush = [&]() {
    if (export_group(shape, v, vn, vt, group, material, err))
      shapes.push_back(shape);
    shape = Shape();
    group.clear();
  };
  while (next_line(in, line)) {
    if (line.empty()) continue;
    const char* t = line.c_str();
    t += strspn(t, " \t");
    if (t[0] == '\0' || t[0] == '#') continue;
    if (t[0] == 'v' && is_space(t[1])) {
      t += 2;
      for (int k = 0; k < 3; ++k) v.push_back(parse_float(t));
      continue;
    }
    if (t[0] == 'v' && t[1] == 'n' && is_space(t[2])) {
      t += 3;
      for (int k = 0; k < 3; ++k) vn.push_back(parse_float(t));
      continue;
    }
    if (t[0] == 'v' && t[1] == 't' && is_space(t[2])) {
      t += 3;
      for (int k = 0; k < 2; ++k) vt.push_back(parse_float(t));
      continue;
    }
    if (t[0] == 'f' && is_space(t[1])) {
      t += 2;
      t += strspn(t, " \t");
      std::vector<VIdx> face;
      while (!is_newline(t[0])) {
        face.push_back(parse_triple(t, (int)v.size() / 3, (int)vn.size() / 3,
                                    (int)vt.size() / 2));
        t += strspn(t, " \t\r");
      }
      group.push_back(face);
      continue;
    }
    if (!strncmp(t, "usemtl", 6) && is_space(t[6])) {
      char name[4096] = {0};
      sscanf(t + 7, "%4095s", name);
      group.clear();  // the pending faces are dropped, as in the reference
      auto it = material_map.find(name);
      material = it == material_map.end() ? -1 : it->second;
      continue;
    }
    if (!strncmp(t, "mtllib", 6) && is_space(t[6])) {
      char name[4096] = {0};
      sscanf(t + 7, "%4095s", name);
      std::ifstream mf(basepath + name);
      load_mtl(mf, material_map, materials);
      continue;
    }
    if ((t[0] == 'g' || t[0] == 'o') && is_space(t[1])) {
      flush();
      continue;
    }
  }
  flush();
  return err;
}

// Minimal PPM (P6 binary / P3 ascii) decoder for textures.
bool read_ppm(const std::string& path, int& w, int& h, std::vector<float>& rgb) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return false;
  char magic[3] = {0};
  if (fscanf(f, "%2s", magic) != 1) { fclose(f); return false; }
  auto read_int = [&](int& x) -> bool {
    int c;
    while ((c = fgetc(f)) != EOF) {
      if (c == '#') { while ((c = fgetc(f)) != EOF && c != '\n') {} continue; }
      if (!isspace(c)) { ungetc(c, f); break; }
    }
    return fscanf(f, "%d", &x) == 1;
  };
  int maxv = 0;
  if (!read_int(w) || !read_int(h) || !read_int(maxv) || w <= 0 || h <= 0 ||
      maxv <= 0 || maxv > 255) { fclose(f); return false; }
  rgb.resize((size_t)w * h * 3);
  if (!strcmp(magic, "P6")) {
    fgetc(f);
    std::vector<uint8_t> raw(rgb.size());
    if (fread(raw.data(), 1, raw.size(), f) != raw.size()) { fclose(f); return false; }
    for (size_t i = 0; i < raw.size(); ++i) rgb[i] = raw[i];
  } else if (!strcmp(magic, "P3")) {
    for (size_t i = 0; i < rgb.size(); ++i) {
      int x;
      if (!read_int(x)) { fclose(f); return false; }
      rgb[i] = (float)x;
    }
  } else {
    fclose(f);
    return false;
  }
  fclose(f);
  return true;
}

}  // namespace

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_error = buf;
}

hpt_status fail(hpt_status s, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_error = buf;
  return s;
}

const char* last_error_cstr() { return g_error.c_str(); }

// Eigen's norm()/dot() on a fixed-size 3-vector reduce with complete
// unrolling, which associates as x0 + (x1 + x2); the reference's scene
// code (hp::Vec = Eigen::Matrix<float,3,1>, src/hp/common.h:39-40) inherits
// that order, so it is kept here.
static inline float eigen_sum3(float a, float b, float c) { return a + (b + c); }

// src/hp/scene/base.cpp:85-93; the arithmetic keeps the reference's types
// (float, with the 1e-4 added in double before rounding back to float).
void material_probabilities(hpt_ref_material& m) {
  auto norm = [](const float* v) {
    return std::sqrt(eigen_sum3(v[0] * v[0], v[1] * v[1], v[2] * v[2]));
  };
  float specular_length = norm(m.specular);
  float diffuse_length = norm(m.diffuse);
  float refract_length = 1.0f - m.dissolve;
  float sum = (float)((double)(specular_length + diffuse_length + refract_length) + 1e-4);
  m.specular_possibility = specular_length / sum;
  m.refract_possibility = refract_length / sum + m.specular_possibility;
  m.diffuse_possibility = diffuse_length * 0.9f / sum + m.refract_possibility;
}

// src/hp/scene/base.cpp:160-198. The std::map keyed by the running total is
// restated as an ordered list with insert-or-assign semantics.
bool build_light_table(const std::vector<F4>& points,
                       const std::vector<I4>& triangles,
                       const std::vector<hpt_ref_material>& materials,
                       std::vector<I4>& lights) {
  std::map<float, int> lights_map;
  float total = 0;
  auto norm3 = [](float x, float y, float z) {
    return std::sqrt(eigen_sum3(x * x, y * y, z * z));
  };
  for (size_t i = 0; i < triangles.size(); ++i) {
    const I4& tri = triangles[i];
    if (tri.w < 0 || tri.w >= (int)materials.size()) return false;
    const hpt_ref_material& mat = materials[tri.w];
    float emission_norm = norm3(mat.emission[0], mat.emission[1], mat.emission[2]);
    if (emission_norm > 0) {
      const F4 &pa = points[tri.x], &pb = points[tri.y], &pc = points[tri.z];
      float dx[3] = {pb.x - pa.x, pb.y - pa.y, pb.z - pa.z};
      float dy[3] = {pc.x - pa.x, pc.y - pa.y, pc.z - pa.z};
      float dot = eigen_sum3(dx[0] * dy[0], dx[1] * dy[1], dx[2] * dy[2]);
      float nx = norm3(dx[0], dx[1], dx[2]), ny = norm3(dy[0], dy[1], dy[2]);
      float ux[3] = {dx[0] / nx, dx[1] / nx, dx[2] / nx};
      float uy[3] = {dy[0] / ny, dy[1] / ny, dy[2] / ny};
      float cosine = eigen_sum3(ux[0] * uy[0], ux[1] * uy[1], ux[2] * uy[2]);
      float area = dot / cosine * std::sqrt(1 - cosine * cosine);
      float val = area * emission_norm;
      total += val;
      lights_map[total] = (int)i;
    }
  }
  lights.clear();
  if (lights_map.empty()) return true;
  for (int i = 0; i < 256; ++i) {
    float val = float(i) / float(256) * total;
    auto it = lights_map.upper_bound(val);
    if (it == lights_map.end()) it = lights_map.begin();
    lights.push_back(triangles[it->second]);
  }
  return true;
}

hpt_status load_obj(const std::string& filename, const std::string& basepath,
                    int texture_size, bool ignore_textures, Mesh& out) {
  std::ifstream in(filename);
  if (!in) return fail(HPT_ERR_IO, "cannot open %s", filename.c_str());
  std::vector<Shape> shapes;
  std::vector<ObjMaterial> mats;
  std::string err = parse_obj(in, basepath, shapes, mats);
  if (!err.empty()) return fail(HPT_ERR_IO, "%s: %s", filename.c_str(), err.c_str());
  out = Mesh();
  for (const ObjMaterial& mat : mats) {  // base.cpp:47-96
    hpt_ref_material x;
    memset(&x, 0, sizeof x);
    for (int k = 0; k < 3; ++k) {
      x.emission[k] = mat.emission[k];
      x.ambient[k] = mat.ambient[k];
      x.diffuse[k] = mat.diffuse[k];
      x.specular[k] = mat.specular[k];
    }
    x.optical_density = mat.ior;
    x.dissolve = mat.dissolve;
    x.shininess = mat.shininess;
    x.diffuse_texture_id = -1;
    x.ambient_texture_id = -1;
    auto tex_id = [&](const std::string& name) {
      auto f = std::find(out.texture_names.begin(), out.texture_names.end(), name);
      if (f != out.texture_names.end()) return (int)(f - out.texture_names.begin());
      out.texture_names.push_back(name);
      return (int)out.texture_names.size() - 1;
    };
    if (!mat.diffuse_texname.empty()) x.diffuse_texture_id = tex_id(mat.diffuse_texname);
    if (!mat.ambient_texname.empty()) x.ambient_texture_id = tex_id(mat.ambient_texname);
    material_probabilities(x);
    out.materials.push_back(x);
  }
  // base.cpp:31-32 resizes every texture to 512 x 512; texture_size > 0 does
  // the same at that size, 0 keeps each texture at its own size.
  if (texture_size < 0) return fail(HPT_ERR_INVALID_ARGUMENT, "texture_size must be >= 0");
  for (const std::string& name : out.texture_names) {  // base.cpp:98-110
    int w = 0, h = 0;
    std::vector<float> rgb;
    bool ok = read_ppm(basepath + name, w, h, rgb);
    if (!ok && !ignore_textures)
      return fail(HPT_ERR_UNSUPPORTED, "texture %s%s: only PPM textures are decoded",
                  basepath.c_str(), name.c_str());
    if (!ok) {
      out.texture_dims.push_back(1);
      out.texture_dims.push_back(1);
      const uint8_t grey[4] = {128, 128, 128, 0};
      out.texture_data.insert(out.texture_data.end(), grey, grey + 4);
      continue;
    }
    // normalize(0, 255) then nearest resample to tw x th, RGB + 0.
    float lo = *std::min_element(rgb.begin(), rgb.end());
    float hi = *std::max_element(rgb.begin(), rgb.end());
    float scale = hi > lo ? 255.f / (hi - lo) : 0.f;
    const int tw = texture_size > 0 ? texture_size : w;
    const int th = texture_size > 0 ? texture_size : h;
    out.texture_dims.push_back(tw);
    out.texture_dims.push_back(th);
    for (int i = 0; i < th; ++i) {
      int sy = (int)((int64_t)i * h / th);
      for (int j = 0; j < tw; ++j) {
        int sx = (int)((int64_t)j * w / tw);
        for (int k = 0; k < 3; ++k)
          out.texture_data.push_back((uint8_t)((rgb[((size_t)sy * w + sx) * 3 + k] - lo) * scale));
        out.texture_data.push_back(0);
      }
    }
  }
  for (const Shape& s : shapes) {  // base.cpp:112-151
    int base = (int)out.points.size();
    for (size_t i = 0; i + 2 < s.positions.size(); i += 3)
      out.points.push_back({s.positions[i], s.positions[i + 1], s.positions[i + 2], 0.f});
    for (size_t i = 0; i + 2 < s.normals.size(); i += 3)
      out.normals.push_back({s.normals[i], s.normals[i + 1], s.normals[i + 2], 0.f});
    for (size_t i = 0; i + 1 < s.texcoords.size(); i += 2)
      out.texcoords.push_back({s.texcoords[i], s.texcoords[i + 1]});
    for (size_t i = 0; i + 2 < s.indices.size(); i += 3)
      out.triangles.push_back({s.indices[i] + base, s.indices[i + 1] + base,
                               s.indices[i + 2] + base, s.material_ids[i / 3]});
  }
  for (const I4& t : out.triangles)
    if (t.w < 0 || t.w >= (int)out.materials.size())
      return fail(HPT_ERR_INVALID_SCENE,
                  "%s: a face has no valid material (usemtl missing or unknown)",
                  filename.c_str());
  if (!build_light_table(out.points, out.triangles, out.materials, out.lights))
    return fail(HPT_ERR_INVALID_SCENE, "light table: bad material index");
  return HPT_OK;
}

}  // namespace hpt
