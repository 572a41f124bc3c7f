// hpt_trace_runner.hpp - header-only C++ drop-in for hp::TraceRunner
// (src/hp/trace_runner.h:21-66) over the C ABI of libhpt.so.
//
// A host that renders with hpTracing swaps
//     #include "hp/trace_runner.h"
// for
//     #include "hpt_trace_runner.hpp"
// and links -lhpt. The constructor and run() keep the reference's
// signatures; the constructor reads the same public members of the scene
// (points, normals, texcoords, geometries, lights, materials, texture_data,
// texture_names) and KDTree::getData(), and, like the reference, leaves the
// caller's scene untouched (it holds device copies). Differences:
//   - errors throw hpt::Error (a std::runtime_error carrying the
//     hpt_status) instead of cl::Error;
//   - run() accepts an optional RNG seed after `brightness` (the reference
//     seeds from time(0)); omitted, it uses a per-runner call counter.
// Scene / value types are templates, so the header compiles against the
// reference's own hp::KDTree and cl_float3 or against any look-alike.
#pragma once

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "hpt.h"

namespace hpt {

class Error : public std::runtime_error {
 public:
  Error(hpt_status s, const std::string& where)
      : std::runtime_error(where + ": " + hpt_status_string(s) + ": " + hpt_last_error()),
        status(s) {}
  hpt_status status;
};

inline void check(hpt_status s, const char* where) {
  if (s != HPT_OK) throw Error(s, where);
}

namespace detail {
template <class...>
struct voider {
  using type = void;
};
// The reference's hp::Scene resizes every texture to its static
// texture_width x texture_height (src/hp/scene/base.h:28, base.cpp:31-32).
template <class S, class = void>
struct has_layer_size : std::false_type {};
template <class S>
struct has_layer_size<S, typename voider<decltype(S::texture_width),
                                         decltype(S::texture_height)>::type> : std::true_type {};
// A scene that keeps its textures at their own sizes lists (w, h) per
// texture in texture_dims.
template <class S, class = void>
struct has_texture_dims : std::false_type {};
template <class S>
struct has_texture_dims<S, typename voider<decltype(std::declval<S&>().texture_dims)>::type>
    : std::true_type {};

// Tags: (has_layer_size, has_texture_dims).
template <class S, class D>
void layer_dims(const S&, int ntex, int w, int h, std::vector<int32_t>& dims,
                std::true_type /*static size*/, D) {
  dims.assign(2 * (size_t)ntex, 0);
  for (int t = 0; t < ntex; ++t) {
    dims[2 * t] = w > 0 ? w : (int)S::texture_width;
    dims[2 * t + 1] = h > 0 ? h : (int)S::texture_height;
  }
}
template <class S>
void layer_dims(const S& s, int ntex, int, int, std::vector<int32_t>& dims, std::false_type,
                std::true_type /*texture_dims*/) {
  dims.assign(s.texture_dims.begin(), s.texture_dims.end());
  dims.resize(2 * (size_t)ntex, 0);
}
template <class S>
void layer_dims(const S&, int ntex, int w, int h, std::vector<int32_t>& dims, std::false_type,
                std::false_type) {
  dims.assign(2 * (size_t)ntex, 0);
  for (int t = 0; t < ntex; ++t) {
    dims[2 * t] = w > 0 ? w : 512;
    dims[2 * t + 1] = h > 0 ? h : 512;
  }
}
}  // namespace detail

}  // namespace hpt

namespace hp {

class TraceRunner {
 public:
  // TraceRunner(std::unique_ptr<hp::KDTree> & scene), trace_runner.h:51.
  // The size of each texture layer in scene->texture_data comes from the
  // scene type: the reference's static Scene::texture_width x
  // texture_height (every texture resized to it), or a per-texture
  // `texture_dims` list (w, h, ...) where the scene keeps native sizes.
  // texture_width/height > 0 override the static size; a scene type with
  // neither member uses them, or 512 x 512 (the reference's size).
  template <class ScenePtr>
  explicit TraceRunner(ScenePtr& scene, int device = 0, int texture_width = 0,
                       int texture_height = 0) {
    auto data = scene->getData();
    const auto& nodes = data.first;
    const auto& leaf = data.second;
    static_assert(sizeof(nodes[0]) == sizeof(hpt_ref_node), "KDTreeNodeHeader is 48 bytes");
    static_assert(sizeof(scene->materials[0]) == sizeof(hpt_ref_material),
                  "Material is 96 bytes");
    using S = typename std::remove_cv<typename std::remove_reference<decltype(*scene)>::type>::type;
    const int ntex = (int)scene->texture_names.size();
    std::vector<int32_t> dims;
    hpt::detail::layer_dims(*scene, ntex, texture_width, texture_height, dims,
                            hpt::detail::has_layer_size<S>(),
                            hpt::detail::has_texture_dims<S>());
    hpt_scene_desc d;
    std::memset(&d, 0, sizeof d);
    d.points = reinterpret_cast<const float*>(scene->points.data());
    d.num_points = (int32_t)scene->points.size();
    d.normals = reinterpret_cast<const float*>(scene->normals.data());
    d.num_normals = (int32_t)scene->normals.size();
    d.texcoords = reinterpret_cast<const float*>(scene->texcoords.data());
    d.num_texcoords = (int32_t)scene->texcoords.size();
    d.triangles = reinterpret_cast<const int32_t*>(scene->geometries.data());
    d.num_triangles = (int32_t)scene->geometries.size();
    d.nodes = reinterpret_cast<const hpt_ref_node*>(nodes.data());
    d.num_nodes = (int32_t)nodes.size();
    d.leaf_data = reinterpret_cast<const int32_t*>(leaf.data());
    d.num_leaf_data = (int32_t)leaf.size();
    d.materials = reinterpret_cast<const hpt_ref_material*>(scene->materials.data());
    d.num_materials = (int32_t)scene->materials.size();
    d.lights = reinterpret_cast<const int32_t*>(scene->lights.data());
    d.num_lights = (int32_t)scene->lights.size();
    d.texture_data = reinterpret_cast<const uint8_t*>(scene->texture_data.data());
    d.num_textures = ntex;
    d.texture_dims = ntex ? dims.data() : nullptr;
    d.device = device;
    hpt::check(hpt_scene_create(&d, &scene_), "hp::TraceRunner");
  }

  TraceRunner(const TraceRunner&) = delete;
  TraceRunner& operator=(const TraceRunner&) = delete;
  ~TraceRunner() { hpt_scene_destroy(scene_); }

  // TraceRunner::run, trace_runner.h:53-65. result_data receives
  // sample_x * sample_y RGBA8 pixels (alpha 0), rows as the reference.
  template <class F3>
  void run(unsigned char* result_data, F3 view_p, F3 top_dir, F3 right_dir, float width,
           float height, int sample_x, int sample_y, int supersample_x, int supersample_y,
           F3 background_color, int sample = 10, int depth = 6, int disable_diffuse = 0,
           float brightness = 1.0f, uint64_t seed = ~0ull) {
    hpt_camera cam;
    hpt_render_params p;
    std::memset(&cam, 0, sizeof cam);
    std::memset(&p, 0, sizeof p);
    for (int k = 0; k < 3; ++k) {
      cam.view_p[k] = view_p.s[k];
      cam.top_dir[k] = top_dir.s[k];
      cam.right_dir[k] = right_dir.s[k];
      p.background[k] = background_color.s[k];
    }
    cam.width = width;
    cam.height = height;
    p.sample_x = sample_x;
    p.sample_y = sample_y;
    p.supersample_x = supersample_x;
    p.supersample_y = supersample_y;
    p.sample = sample;
    p.depth = depth;
    p.disable_diffuse = disable_diffuse;
    p.brightness = brightness;
    p.seed = seed == ~0ull ? calls_++ : seed;
    hpt::check(hpt_render(scene_, &cam, &p, result_data, nullptr), "hp::TraceRunner::run");
  }

  hpt_scene* handle() const { return scene_; }

 private:
  hpt_scene* scene_ = nullptr;
  uint64_t calls_ = 0;
};

}  // namespace hp
