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
//             [--background 0,0,0] [--seed N] -o out.ppm
//   -i generated:K renders synthetic scene K (0 room, 1 spheres, 2 terrain).
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
          "       [--background r,g,b] [--seed N] [--device D]\n");
  return 2;
}

}  // namespace

int main(int argc, char** argv) {
  std::string input, mtl, output;
  int width = 500, height = 500, sample = 10, depth = 6, device = 0;
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
    st = hpt_mesh_load_obj(input.c_str(), mtl.c_str(), 512, 0, &mesh);
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
  int tex_w = 512, tex_h = 512;
  if (v.num_textures > 0) {
    tex_w = v.texture_dims[0];
    tex_h = v.texture_dims[1];
  }
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
    hp::TraceRunner runner(sp, device, tex_w, tex_h);
    // runit(), hptracing.cpp:60-84: width = aspect * angle, height = angle.
    runner.run(pixels.data(), view, up, right, (float)width / (float)height * angle, angle,
               width, height, supersample ? 2 : 1, supersample ? 2 : 1, background, sample,
               depth, no_diffuse ? 1 : 0, brightness, seed);
    hpt_render_stats rs;
    hpt_render_stats_get(runner.handle(), &rs);
    fprintf(stderr, "hptracing: %lld intersect queries in %.2f ms (%.1f Mrays/s)\n",
            (long long)rs.intersect_queries, rs.ms_total,
            rs.ms_total > 0 ? rs.intersect_queries / (rs.ms_total * 1e3) : 0.0);
  } catch (const hpt::Error& e) {
    fprintf(stderr, "hptracing: %s\n", e.what());
    return 1;
  }
  FILE* f = fopen(output.c_str(), "wb");
  if (!f) {
    fprintf(stderr, "hptracing: cannot write %s\n", output.c_str());
    return 1;
  }
  fprintf(f, "P6\n%d %d\n255\n", width, height);
  for (int y = height - 1; y >= 0; --y)  // image.mirror('y')
    for (int x = 0; x < width; ++x) fwrite(&pixels[((size_t)y * width + x) * 4], 1, 3, f);
  fclose(f);
  return 0;
}
