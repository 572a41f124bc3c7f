// hptracing - headless command line renderer with the flags of the
// reference's src/hptracing.cpp:213-298 (its GLUT window needs a graphics
// stack; here -o is required and the image is written as binary PPM, rows
// mirrored in y as the reference does before saving, :287-296). It is built
// on the hp::TraceRunner drop-in header, i.e. it makes the same calls a
// reference host makes.
//
//   hptracing -i scene.obj [--mtl DIR] [--width 500] [--height 500]
//             [--view 0,0,-500] [--up 0,1,0] [--right 1,0,0] [--angle 1.0]
//             [-x] [-s 10] [-d 6] [--brightness 1] [--no-diffuse]
//             [--background 0,0,0] [--seed N] [--keys SEQ] -o out.ppm
//   -i generated:K renders synthetic scene K (0 room, 1 spheres, 2 terrain).
//   --keys SEQ replays the reference GUI's camera keys (hptracing.cpp:
//   167-211) without a window: the first frame and one frame per key that
//   makes the GUI re-render are written as out_000.ppm, out_001.ppm, ...
//   Keys: a/d, w/s, q/e rotate -/+15 degrees about up, right, front; k/j move
//   forward/back and U/D/R/L (the arrow keys) along up/right by the step;
//   [ and ] halve and double the step; z/x and -/+ change the angle.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "hpt_trace_runner.hpp"

namespace {

struct F3 {
  float s[4];
};
struct F2 {
  float s[2];
};
struct I4 {
  int32_t s[4];
};

// The members of hp::KDTree that hp::TraceRunner reads (base.h:30-40).
struct Scene {
  std::vector<F3> points, normals;
  std::vector<F2> texcoords;
  std::vector<I4> geometries, lights;
  std::vector<hpt_ref_material> materials;
  std::vector<uint8_t> texture_data;
  std::vector<std::string> texture_names;
  std::vector<int32_t> texture_dims;
  std::pair<std::vector<hpt_ref_node>, std::vector<int32_t>> data;
  std::pair<std::vector<hpt_ref_node>, std::vector<int32_t>> getData() const { return data; }
};

// str2float3, hptracing.cpp:31-39
F3 parse3(const char* s) {
  F3 r = {{0, 0, 0, 0}};
  std::string str(s);
  for (int i = 0; i < 3; ++i) {
    r.s[i] = (float)atof(str.c_str());
    if (i < 2) str = str.substr(str.find(',') + 1);
  }
  return r;
}

template <class T>
void copy_view(std::vector<T>& dst, const void* p, int n) {
  dst.resize(n);
  if (n) memcpy(dst.data(), p, (size_t)n * sizeof(T));
}

int usage() {
  fprintf(stderr,
          "usage: hptracing -i scene.obj|generated:K -o out.ppm [--mtl DIR] [--width W]\n"
          "       [--height H] [--view x,y,z] [--up x,y,z] [--right x,y,z] [--angle A]\n"
          "       [-x] [-s SAMPLES] [-d DEPTH] [--brightness B] [--no-diffuse]\n"
          "       [--background r,g,b] [--seed N] [--device D] [--keys SEQ]\n"
          "       [--texture-size N]   (N > 0: every texture resized to N x N, as the\n"
          "                             reference does with 512; 0: native sizes)\n");
  return 2;
}

struct V3 {
  float x, y, z;
};
V3 v3(const F3& f) { return V3{f.s[0], f.s[1], f.s[2]}; }
F3 f3(const V3& v) { return F3{{v.x, v.y, v.z, 0.f}}; }
V3 cross(const V3& a, const V3& b) {
  return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// rotateView (hptracing.cpp:131-153): Rodrigues' formula with the matrix L
// built from the axis as the reference builds it; ax 1 = right, 2 = up,
// 3 = front (= up x right). Only up and right are kept.
void rotate_view(float alpha, int ax, F3& up_f, F3& right_f) {
  const double kPi = 3.141592653589;  // PI, src/hp/common.h:20
  V3 up = v3(up_f), right = v3(right_f), front = cross(up, right);
  const V3 a = ax == 2 ? up : ax == 3 ? front : right;
  const float L[3][3] = {{0.f, a.z, -a.y}, {-a.z, 0.f, a.x}, {a.y, -a.x, 0.f}};
  const float sn = (float)std::sin(alpha / 180.0 * kPi);
  const float cs = (float)(1.0 - std::cos(alpha / 180.0 * kPi));
  float m[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      float l2 = 0.f;
      for (int k = 0; k < 3; ++k) l2 += L[i][k] * L[k][j];
      m[i][j] = (i == j ? 1.f : 0.f) + sn * L[i][j] + cs * l2;
    }
  auto apply = [&](const V3& v) {
    return V3{m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z,
              m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
              m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
  };
  if (ax != 2) up = apply(up);
  if (ax != 1) right = apply(right);
  up_f = f3(up);
  right_f = f3(right);
}

// translateView (hptracing.cpp:155-167): move along right, up or front.
void translate_view(float step, int ax, F3& view, const F3& up_f, const F3& right_f) {
  const V3 up = v3(up_f), right = v3(right_f), front = cross(up, right);
  const V3 a = ax == 2 ? up : ax == 3 ? front : right;
  view.s[0] += step * a.x;
  view.s[1] += step * a.y;
  view.s[2] += step * a.z;
}

// keyFunc / specKeyFunc (hptracing.cpp:169-211). Returns true when the key
// makes the GUI render again.
bool apply_key(char key, F3& view, F3& up, F3& right, float& angle, float& step) {
  switch (key) {
    case 'z': if (angle > 0.1f) angle -= 0.1f; return true;
    case 'x': angle += 0.1f; return true;
    case 'a': rotate_view(-15, 2, up, right); return true;
    case 'd': rotate_view(15, 2, up, right); return true;
    case 'w': rotate_view(-15, 1, up, right); return true;
    case 's': rotate_view(15, 1, up, right); return true;
    case 'q': rotate_view(-15, 3, up, right); return true;
    case 'e': rotate_view(15, 3, up, right); return true;
    case 'k': translate_view(step, 3, view, up, right); return true;
    case 'j': translate_view(-step, 3, view, up, right); return true;
    case '[': step /= 2.f; return false;
    case ']': step *= 2.f; return false;
    case '+': angle += 0.1f; return true;
    case '-': angle -= 0.1f; return true;
    case 'U': translate_view(step, 2, view, up, right); return true;
    case 'D': translate_view(-step, 2, view, up, right); return true;
    case 'R': translate_view(step, 1, view, up, right); return true;
    case 'L': translate_view(-step, 1, view, up, right); return true;
    default: return false;
  }
}

bool write_ppm(const std::string& path, const std::vector<unsigned char>& pixels, int width,
               int height) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) return false;
  fprintf(f, "P6\n%d %d\n255\n", width, height);
  for (int y = height - 1; y >= 0; --y)  // image.mirror('y'), hptracing.cpp:287-296
    for (int x = 0; x < width; ++x) fwrite(&pixels[((size_t)y * width + x) * 4], 1, 3, f);
  return fclose(f) == 0;
}

std::string frame_name(const std::string& out, int k) {
  const size_t dot = out.rfind('.');
  const std::string stem = dot == std::string::npos ? out : out.substr(0, dot);
  const std::string ext = dot == std::string::npos ? ".ppm" : out.substr(dot);
  char buf[16];
  snprintf(buf, sizeof buf, "_%03d", k);
  return stem + buf + ext;
}

}  // namespace

int main(int argc, char** argv) {
  std::string input, mtl, output, keys;
  int width = 500, height = 500, sample = 10, depth = 6, device = 0, texture_size = 512;
  float angle = 1.0f, brightness = 1.0f;
  bool supersample = false, no_diffuse = false;
  uint64_t seed = 0;
  F3 view = parse3("0,0,-500"), up = parse3("0,1,0"), right = parse3("1,0,0");
  F3 background = parse3("0,0,0");
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    auto next = [&]() -> const char* {
      if (i + 1 >= argc) {
        usage();
        exit(2);
      }
      return argv[++i];
    };
    if (a == "-i" || a == "--input") input = next();
    else if (a == "--mtl") mtl = next();
    else if (a == "--width") width = atoi(next());
    else if (a == "--height") height = atoi(next());
    else if (a == "--view") view = parse3(next());
    else if (a == "--up") up = parse3(next());
    else if (a == "--right") right = parse3(next());
    else if (a == "--angle") angle = (float)atof(next());
    else if (a == "-x" || a == "--supersample") supersample = true;
    else if (a == "-s" || a == "--sample") sample = atoi(next());
    else if (a == "-d" || a == "--depth") depth = atoi(next());
    else if (a == "--brightness") brightness = (float)atof(next());
    else if (a == "--no-diffuse") no_diffuse = true;
    else if (a == "--background") background = parse3(next());
    else if (a == "-o" || a == "--output") output = next();
    else if (a == "--seed") seed = strtoull(next(), nullptr, 10);
    else if (a == "--device") device = atoi(next());
    else if (a == "--keys") keys = next();
    else if (a == "--texture-size") texture_size = atoi(next());
    else return usage();
  }
  if (input.empty() || output.empty()) return usage();

  hpt_mesh* mesh = nullptr;
  hpt_status st;
  if (input.rfind("generated:", 0) == 0) {
    st = hpt_mesh_generate(atoi(input.c_str() + 10), seed, nullptr, &mesh);
  } else {
    if (mtl.empty()) {  // hptracing.cpp:236-244
      size_t pos = input.rfind('/');
      if (pos != std::string::npos && pos > 0) mtl = input.substr(0, pos + 1);
    }
    st = hpt_mesh_load_obj(input.c_str(), mtl.c_str(), texture_size, 0, &mesh);
  }
  if (st != HPT_OK) {
    fprintf(stderr, "hptracing: %s: %s\n", hpt_status_string(st), hpt_last_error());
    return 1;
  }
  Scene scene;
  hpt_mesh_arrays v;
  hpt_mesh_view(mesh, &v);
  copy_view(scene.points, v.points, v.num_points);
  copy_view(scene.normals, v.normals, v.num_normals);
  copy_view(scene.texcoords, v.texcoords, v.num_texcoords);
  copy_view(scene.geometries, v.triangles, v.num_triangles);
  copy_view(scene.lights, v.lights, v.num_lights);
  copy_view(scene.materials, v.materials, v.num_materials);
  scene.texture_data.assign(v.texture_data, v.texture_data + v.texture_bytes);
  scene.texture_names.resize(v.num_textures);
  if (v.num_textures > 0)
    scene.texture_dims.assign(v.texture_dims, v.texture_dims + 2 * (size_t)v.num_textures);
  hpt_kdtree* tree = nullptr;
  st = hpt_kdtree_build(v.points, v.num_points, v.triangles, v.num_triangles, 0, &tree);
  if (st != HPT_OK) {
    fprintf(stderr, "hptracing: %s: %s\n", hpt_status_string(st), hpt_last_error());
    return 1;
  }
  const hpt_ref_node* nodes;
  const int32_t* leaf;
  int32_t nn, nl;
  hpt_kdtree_view(tree, &nodes, &nn, &leaf, &nl);
  scene.data.first.assign(nodes, nodes + nn);
  scene.data.second.assign(leaf, leaf + nl);
  hpt_kdtree_destroy(tree);
  hpt_mesh_destroy(mesh);

  std::vector<unsigned char> pixels((size_t)width * height * 4);
  try {
    Scene* sp = &scene;
    hp::TraceRunner runner(sp, device);
    float step = 1.f;  // translate_step, hptracing.cpp:58
    int frame = 0;
    auto render = [&](const std::string& path) -> bool {
      // runit(), hptracing.cpp:60-84: width = aspect * angle, height = angle.
      runner.run(pixels.data(), view, up, right, (float)width / (float)height * angle, angle,
                 width, height, supersample ? 2 : 1, supersample ? 2 : 1, background, sample,
                 depth, no_diffuse ? 1 : 0, brightness, seed + (uint64_t)frame);
      hpt_render_stats rs;
      hpt_render_stats_get(runner.handle(), &rs);
      fprintf(stderr, "hptracing: %s: %lld intersect queries in %.2f ms (%.1f Mrays/s)\n",
              path.c_str(), (long long)rs.intersect_queries, rs.ms_total,
              rs.ms_total > 0 ? rs.intersect_queries / (rs.ms_total * 1e3) : 0.0);
      if (!write_ppm(path, pixels, width, height)) {
        fprintf(stderr, "hptracing: cannot write %s\n", path.c_str());
        return false;
      }
      return true;
    };
    if (keys.empty()) {
      if (!render(output)) return 1;
    } else {
      if (!render(frame_name(output, frame++))) return 1;
      for (char k : keys)
        if (apply_key(k, view, up, right, angle, step) && !render(frame_name(output, frame++)))
          return 1;
    }
  } catch (const hpt::Error& e) {
    fprintf(stderr, "hptracing: %s\n", e.what());
    return 1;
  }
  return 0;
}
