// Host-side data structures shared by the loader, the SAH builder, the
// synthetic scene generators and the device repacker.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/hpt.h"

namespace hpt {

struct F4 {  // cl_float3 / cl_float4 as laid out by the reference (16 B)
  float x, y, z, w;
};
struct F2 {
  float x, y;
};
struct I4 {
  int32_t x, y, z, w;
};
static_assert(sizeof(F4) == 16 && sizeof(I4) == 16 && sizeof(F2) == 8, "layout");
static_assert(sizeof(hpt_ref_node) == 48, "KDTreeNodeHeader is 48 bytes");
static_assert(sizeof(hpt_ref_material) == 96, "Material is 96 bytes");

// The arrays hp::Scene exposes (src/hp/scene/base.h:30-40), with per-texture
// dimensions instead of the reference's fixed 512 x 512.
struct Mesh {
  std::vector<F4> points;
  std::vector<F4> normals;
  std::vector<F2> texcoords;
  std::vector<I4> triangles;
  std::vector<hpt_ref_material> materials;
  std::vector<I4> lights;
  std::vector<std::string> texture_names;
  std::vector<uint8_t> texture_data;
  std::vector<int32_t> texture_dims;  // (w, h) per texture
};

struct KdTree {
  std::vector<hpt_ref_node> nodes;
  std::vector<int32_t> leaf_data;
};

// Thread-local error message for hpt_last_error().
void set_error(const char* fmt, ...) __attribute__((format(printf, 1, 2)));
hpt_status fail(hpt_status s, const char* fmt, ...)
    __attribute__((format(printf, 2, 3)));

// Material probabilities (src/hp/scene/base.cpp:85-93).
void material_probabilities(hpt_ref_material& m);
// Light table (src/hp/scene/base.cpp:160-198). Returns false on an invalid
// material index.
bool build_light_table(const std::vector<F4>& points,
                       const std::vector<I4>& triangles,
                       const std::vector<hpt_ref_material>& materials,
                       std::vector<I4>& lights);

hpt_status load_obj(const std::string& filename, const std::string& basepath,
                    int texture_size, bool ignore_textures, Mesh& out);
hpt_status generate_scene(int config, uint64_t seed, const hpt_gen_params& p,
                          Mesh& out);

// SAH KD-tree (src/hp/scene/kdtree.cpp). points/tris as in the reference.
hpt_status build_kdtree(const F4* points, int num_points, const I4* tris,
                        int num_tris, int num_threads, KdTree& out);

// Structural check of a flattened tree; returns an empty string when valid.
std::string validate_ref_tree(const hpt_ref_node* nodes, int num_nodes,
                              const int32_t* leaf_data, int num_leaf,
                              int num_triangles);

}  // namespace hpt
