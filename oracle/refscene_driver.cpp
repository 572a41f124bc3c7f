// refscene_driver.cpp - C entry points around the reference's own scene
// loader and SAH KD-tree (hp::KDTree, src/hp/scene/{base,kdtree}.cpp),
// compiled from the reference sources with the header stand-ins in
// refshim/ (Eigen 3-vector, OpenCL value types). Test infrastructure: it
// pins the product's OBJ reader, light table and KD builder bit for bit.
// Built by oracle/build.py into oracle/_ref/ only.
#include <cstring>
#include <memory>
#include <string>

#include "hp/scene/kdtree.h"

extern "C" {

struct RefSceneView {
  const float* points; int num_points;
  const float* normals; int num_normals;
  const float* texcoords; int num_texcoords;
  const int* triangles; int num_triangles;
  const void* materials; int num_materials;
  const int* lights; int num_lights;
  const void* nodes; int num_nodes;
  const int* leaf_data; int num_leaf_data;
};

struct RefSceneHandle {
  std::unique_ptr<hp::KDTree> tree;
  std::vector<hp::KDTreeNodeHeader> nodes;
  std::vector<cl_int> leaf;
};

void* refscene_load(const char* filename, const char* mtl_basepath) {
  try {
    auto* h = new RefSceneHandle();
    h->tree.reset(new hp::KDTree(filename, mtl_basepath ? mtl_basepath : ""));
    auto d = h->tree->getData();
    h->nodes = d.first;
    h->leaf = d.second;
    return h;
  } catch (...) {
    return nullptr;
  }
}

void refscene_view(void* handle, RefSceneView* v) {
  auto* h = static_cast<RefSceneHandle*>(handle);
  hp::KDTree& s = *h->tree;
  memset(v, 0, sizeof *v);
  v->points = reinterpret_cast<const float*>(s.points.data());
  v->num_points = (int)s.points.size();
  v->normals = reinterpret_cast<const float*>(s.normals.data());
  v->num_normals = (int)s.normals.size();
  v->texcoords = reinterpret_cast<const float*>(s.texcoords.data());
  v->num_texcoords = (int)s.texcoords.size();
  v->triangles = reinterpret_cast<const int*>(s.geometries.data());
  v->num_triangles = (int)s.geometries.size();
  v->materials = s.materials.data();
  v->num_materials = (int)s.materials.size();
  v->lights = reinterpret_cast<const int*>(s.lights.data());
  v->num_lights = (int)s.lights.size();
  v->nodes = h->nodes.data();
  v->num_nodes = (int)h->nodes.size();
  v->leaf_data = h->leaf.data();
  v->num_leaf_data = (int)h->leaf.size();
}

void refscene_free(void* handle) { delete static_cast<RefSceneHandle*>(handle); }

int refscene_sizeof_node(void) { return (int)sizeof(hp::KDTreeNodeHeader); }
int refscene_sizeof_material(void) { return (int)sizeof(hp::Material); }

void refscene_log(int enable) { hp::g_log_enable = enable != 0; }

}  // extern "C"
