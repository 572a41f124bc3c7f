// C ABI: host-only entry points (errors, meshes, SAH KD-tree, light table).
#include <cstring>
#include <memory>
#include <new>

#include "../../include/hpt.h"
#include "host.h"

namespace hpt {
const char* last_error_cstr();
}

using namespace hpt;

struct hpt_mesh {
  Mesh m;
};

struct hpt_kdtree {
  KdTree t;
};

namespace {

template <typename F>
hpt_status guarded(F&& f) {
  try {
    return f();
  } catch (const std::bad_alloc&) {
    return fail(HPT_ERR_OUT_OF_MEMORY, "host allocation failed");
  } catch (...) {
    return fail(HPT_ERR_INVALID_ARGUMENT, "unexpected exception");
  }
}

}  // namespace

extern "C" {

const char* hpt_status_string(hpt_status s) {
  switch (s) {
    case HPT_OK: return "ok";
    case HPT_ERR_INVALID_ARGUMENT: return "invalid argument";
    case HPT_ERR_INVALID_SCENE: return "invalid scene";
    case HPT_ERR_CUDA: return "CUDA error";
    case HPT_ERR_OUT_OF_MEMORY: return "out of memory";
    case HPT_ERR_TRAVERSAL_LIMIT: return "traversal step limit reached";
    case HPT_ERR_NOT_FOUND: return "not found";
    case HPT_ERR_IO: return "I/O error";
    case HPT_ERR_CANCELLED: return "cancelled";
    case HPT_ERR_BUSY: return "busy";
    case HPT_ERR_UNSUPPORTED: return "unsupported";
  }
  return "unknown status";
}

const char* hpt_last_error(void) { return last_error_cstr(); }

int hpt_version(void) { return HPT_VERSION; }

hpt_status hpt_mesh_load_obj(const char* filename, const char* mtl_basepath, int32_t texture_size,
                             int32_t ignore_textures, hpt_mesh** out) {
  if (!filename || !out) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  *out = nullptr;
  return guarded([&]() -> hpt_status {
    std::unique_ptr<hpt_mesh> m(new hpt_mesh());
    std::string base = mtl_basepath ? mtl_basepath : "";
    if (base.empty()) {  // hptracing.cpp:236-244: directory of the input
      std::string in(filename);
      size_t pos = in.rfind('/');
      if (pos != std::string::npos && pos > 0) base = in.substr(0, pos + 1);
    }
    hpt_status s = load_obj(filename, base, texture_size, ignore_textures != 0, m->m);
    if (s != HPT_OK) return s;
    *out = m.release();
    return HPT_OK;
  });
}

hpt_status hpt_mesh_generate(int32_t config, uint64_t seed, const hpt_gen_params* params,
                             hpt_mesh** out) {
  if (!out) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  *out = nullptr;
  return guarded([&]() -> hpt_status {
    hpt_gen_params p;
    memset(&p, 0, sizeof p);
    if (params) p = *params;
    std::unique_ptr<hpt_mesh> m(new hpt_mesh());
    hpt_status s = generate_scene(config, seed, p, m->m);
    if (s != HPT_OK) return s;
    *out = m.release();
    return HPT_OK;
  });
}

hpt_status hpt_mesh_create(const hpt_mesh_arrays* a, int32_t recompute, hpt_mesh** out) {
  if (!a || !out) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  *out = nullptr;
  if (a->num_points < 0 || a->num_triangles < 0 || a->num_materials < 0 || a->num_normals < 0 ||
      a->num_texcoords < 0 || a->num_textures < 0)
    return fail(HPT_ERR_INVALID_ARGUMENT, "negative count");
  return guarded([&]() -> hpt_status {
    std::unique_ptr<hpt_mesh> m(new hpt_mesh());
    Mesh& M = m->m;
    const F4* p = reinterpret_cast<const F4*>(a->points);
    M.points.assign(p, p + a->num_points);
    const F4* n = reinterpret_cast<const F4*>(a->normals);
    if (n) M.normals.assign(n, n + a->num_normals);
    const F2* t = reinterpret_cast<const F2*>(a->texcoords);
    if (t) M.texcoords.assign(t, t + a->num_texcoords);
    const I4* tr = reinterpret_cast<const I4*>(a->triangles);
    M.triangles.assign(tr, tr + a->num_triangles);
    M.materials.assign(a->materials, a->materials + a->num_materials);
    if (recompute)
      for (auto& mat : M.materials) material_probabilities(mat);
    for (const I4& tri : M.triangles)
      if (tri.x < 0 || tri.y < 0 || tri.z < 0 || tri.x >= a->num_points || tri.y >= a->num_points ||
          tri.z >= a->num_points || tri.w < 0 || tri.w >= a->num_materials)
        return fail(HPT_ERR_INVALID_SCENE, "mesh: triangle index out of range");
    if (a->num_textures > 0) {
      if (!a->texture_dims || !a->texture_data)
        return fail(HPT_ERR_INVALID_ARGUMENT, "mesh: texture dims/data missing");
      M.texture_dims.assign(a->texture_dims, a->texture_dims + 2 * a->num_textures);
      int64_t texels = 0;
      for (int i = 0; i < a->num_textures; ++i)
        texels += (int64_t)a->texture_dims[2 * i] * a->texture_dims[2 * i + 1];
      M.texture_data.assign(a->texture_data, a->texture_data + 4 * texels);
      for (int i = 0; i < a->num_textures; ++i) M.texture_names.push_back("tex" + std::to_string(i));
    }
    if (!build_light_table(M.points, M.triangles, M.materials, M.lights))
      return fail(HPT_ERR_INVALID_SCENE, "light table: bad material index");
    *out = m.release();
    return HPT_OK;
  });
}

hpt_status hpt_mesh_view(const hpt_mesh* mesh, hpt_mesh_arrays* out) {
  if (!mesh || !out) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  const Mesh& m = mesh->m;
  memset(out, 0, sizeof *out);
  out->points = reinterpret_cast<const float*>(m.points.data());
  out->num_points = (int32_t)m.points.size();
  out->normals = m.normals.empty() ? nullptr : reinterpret_cast<const float*>(m.normals.data());
  out->num_normals = (int32_t)m.normals.size();
  out->texcoords = m.texcoords.empty() ? nullptr : reinterpret_cast<const float*>(m.texcoords.data());
  out->num_texcoords = (int32_t)m.texcoords.size();
  out->triangles = reinterpret_cast<const int32_t*>(m.triangles.data());
  out->num_triangles = (int32_t)m.triangles.size();
  out->materials = m.materials.data();
  out->num_materials = (int32_t)m.materials.size();
  out->lights = m.lights.empty() ? nullptr : reinterpret_cast<const int32_t*>(m.lights.data());
  out->num_lights = (int32_t)m.lights.size();
  out->texture_data = m.texture_data.empty() ? nullptr : m.texture_data.data();
  out->num_textures = (int32_t)(m.texture_dims.size() / 2);
  out->texture_dims = m.texture_dims.empty() ? nullptr : m.texture_dims.data();
  out->texture_bytes = (int64_t)m.texture_data.size();
  return HPT_OK;
}

void hpt_mesh_destroy(hpt_mesh* mesh) { delete mesh; }

hpt_status hpt_material_probabilities(hpt_ref_material* material) {
  if (!material) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  material_probabilities(*material);
  return HPT_OK;
}

hpt_status hpt_light_table(const float* points4, int32_t num_points, const int32_t* triangles4,
                           int32_t num_triangles, const hpt_ref_material* materials,
                           int32_t num_materials, int32_t* lights_out, int32_t* num_lights) {
  if (!num_lights || !lights_out || num_points < 0 || num_triangles < 0 || num_materials < 0 ||
      (num_points && !points4) || (num_triangles && !triangles4) || (num_materials && !materials))
    return fail(HPT_ERR_INVALID_ARGUMENT, "bad light table arguments");
  return guarded([&]() -> hpt_status {
    std::vector<F4> pts(reinterpret_cast<const F4*>(points4),
                        reinterpret_cast<const F4*>(points4) + num_points);
    std::vector<I4> tris(reinterpret_cast<const I4*>(triangles4),
                         reinterpret_cast<const I4*>(triangles4) + num_triangles);
    for (const I4& t : tris)
      if (t.x < 0 || t.y < 0 || t.z < 0 || t.x >= num_points || t.y >= num_points || t.z >= num_points)
        return fail(HPT_ERR_INVALID_SCENE, "light table: vertex index out of range");
    std::vector<hpt_ref_material> mats(materials, materials + num_materials);
    std::vector<I4> lights;
    if (!build_light_table(pts, tris, mats, lights))
      return fail(HPT_ERR_INVALID_SCENE, "light table: bad material index");
    memcpy(lights_out, lights.data(), lights.size() * sizeof(I4));
    *num_lights = (int32_t)lights.size();
    return HPT_OK;
  });
}

hpt_status hpt_kdtree_build(const float* points4, int32_t num_points, const int32_t* triangles4,
                            int32_t num_triangles, int32_t num_threads, hpt_kdtree** out) {
  if (!out) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  *out = nullptr;
  return guarded([&]() -> hpt_status {
    std::unique_ptr<hpt_kdtree> t(new hpt_kdtree());
    hpt_status s = build_kdtree(reinterpret_cast<const F4*>(points4), num_points,
                                reinterpret_cast<const I4*>(triangles4), num_triangles, num_threads,
                                t->t);
    if (s != HPT_OK) return s;
    *out = t.release();
    return HPT_OK;
  });
}

hpt_status hpt_kdtree_view(const hpt_kdtree* tree, const hpt_ref_node** nodes, int32_t* num_nodes,
                           const int32_t** leaf_data, int32_t* num_leaf_data) {
  if (!tree || !nodes || !num_nodes || !leaf_data || !num_leaf_data)
    return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  *nodes = tree->t.nodes.data();
  *num_nodes = (int32_t)tree->t.nodes.size();
  *leaf_data = tree->t.leaf_data.data();
  *num_leaf_data = (int32_t)tree->t.leaf_data.size();
  return HPT_OK;
}

void hpt_kdtree_destroy(hpt_kdtree* tree) { delete tree; }

}  // extern "C"
