// Host build of the GPU per-ray code (test infrastructure): the traversal
// (traverse.cuh) and shading (shading.cuh) functions are __host__
// __device__; compiled here for the CPU over the same packed scene the
// kernels read, so CPU tests can check the device logic (packer, ropes,
// leaf hints, mailbox, tie ranks, shading) against the oracle bit for bit.
// Nothing in the product uses this library.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../hptracing_b200/csrc/scene_pack.h"
#include "../../hptracing_b200/csrc/shading.cuh"
#include "../../hptracing_b200/csrc/traverse.cuh"

using namespace hpt;

namespace {

struct EmuScene {
  PackedScene pk;
  DevScene dev;
  std::vector<DevTexInfo> tex;
  std::vector<uint32_t> nodes_u2;
};

}  // namespace

extern "C" {

// Packs the scene exactly as hpt_scene_create does (without uploading).
void* emu_scene_create(const hpt_scene_desc* d, int* status) {
  EmuScene* e = new EmuScene();
  hpt_status s = pack_scene(*d, 8192, e->pk);
  *status = (int)s;
  if (s != HPT_OK) {
    delete e;
    return nullptr;
  }
  DevScene& ds = e->dev;
  memset(&ds, 0, sizeof ds);
  ds.nodes = e->pk.nodes.data();
  ds.leaves = e->pk.leaves.data();
  if (e->pk.refs.empty()) e->pk.refs.push_back(0);
  ds.leaf_refs = e->pk.refs.data();
  ds.tris = e->pk.tris.data();
  ds.points = d->points;
  ds.normals = d->normals;
  ds.texcoords = d->texcoords;
  ds.geometry = d->triangles;
  ds.materials = d->materials;
  ds.lights = d->lights;
  ds.texels = reinterpret_cast<const uint32_t*>(d->texture_data);
  int64_t off = 0;
  for (int t = 0; t < d->num_textures; ++t) {
    DevTexInfo ti;
    ti.offset = off;
    ti.w = d->texture_dims ? d->texture_dims[2 * t] : 512;
    ti.h = d->texture_dims ? d->texture_dims[2 * t + 1] : 512;
    off += (int64_t)ti.w * ti.h;
    e->tex.push_back(ti);
  }
  ds.tex_info = e->tex.data();
  ds.num_nodes = (int32_t)e->pk.nodes.size();
  ds.num_leaves = (int32_t)e->pk.leaves.size();
  ds.num_leaf_tris = (int32_t)e->pk.refs.size();
  ds.num_triangles = d->num_triangles;
  ds.num_points = d->num_points;
  ds.num_normals = d->num_normals;
  ds.num_texcoords = d->num_texcoords;
  ds.num_materials = d->num_materials;
  ds.num_lights = d->num_lights;
  ds.num_textures = d->num_textures;
  float scale = 0.f;
  for (int a = 0; a < 3; ++a) {
    ds.root_lo[a] = e->pk.root_lo[a];
    ds.root_hi[a] = e->pk.root_hi[a];
    scale = std::max(scale, std::max(std::fabs(e->pk.root_lo[a]), std::fabs(e->pk.root_hi[a])));
    scale = std::max(scale, e->pk.root_hi[a] - e->pk.root_lo[a]);
  }
  ds.scene_eps = 2e-5f * scale;
  const int64_t cap = 8 * ((int64_t)e->pk.nodes.size() + (int64_t)e->pk.refs.size()) + 100000;
  ds.max_steps = (int32_t)std::min<int64_t>(cap, 1 << 30);
  return e;
}

void emu_scene_destroy(void* h) { delete static_cast<EmuScene*>(h); }

// counts: num_nodes, num_leaves, num_refs, max_depth
void emu_scene_counts(void* h, int* counts) {
  EmuScene* e = static_cast<EmuScene*>(h);
  counts[0] = e->dev.num_nodes;
  counts[1] = e->dev.num_leaves;
  counts[2] = e->dev.num_leaf_tris;
  counts[3] = e->pk.max_depth;
}

// Closest hit per ray with the device traversal. hints (nullable): start
// leaf node per ray. smem_nodes: emulate the shared-memory node prefix.
// best_node (nullable) receives the leaf node of each hit. err receives
// the error word (flags, site, value).
void emu_intersect(void* h, int n, const float* o, const float* d, const int* hints,
                   int smem_nodes, int32_t* tri, float* t, float* u, float* v, int* best_node,
                   long long* counters, long long* err) {
  EmuScene* e = static_cast<EmuScene*>(h);
  const DevScene& s = e->dev;
  std::vector<uint2> smem((size_t)std::max(0, std::min(smem_nodes, s.num_nodes)));
  for (size_t i = 0; i < smem.size(); ++i) {
    smem[i].x = s.nodes[i].meta;
    std::memcpy(&smem[i].y, &s.nodes[i].split, 4);
  }
  DevErr de;
  memset(&de, 0, sizeof de);
  TravCount cnt{};
  for (int i = 0; i < n; ++i) {
    TravState st;
    TravCold tc;
    trav_init(s, Ray{mk(o[3 * i], o[3 * i + 1], o[3 * i + 2]), mk(d[3 * i], d[3 * i + 1], d[3 * i + 2])},
              st, tc, hints ? hints[i] : -1);
    while (!trav_leaf<true>(s, st, tc, smem.data(), (int)smem.size(), &de, cnt)) {
    }
    tri[i] = st.best.tri;
    t[i] = st.best.rec >= 0 ? st.best.t : 0.f;
    u[i] = st.best.rec >= 0 ? st.best.u : 0.f;
    v[i] = st.best.rec >= 0 ? st.best.v : 0.f;
    if (best_node) best_node[i] = tc.best_node;
  }
  counters[0] = (long long)cnt.nodes;
  counters[1] = (long long)cnt.leaves;
  counters[2] = (long long)cnt.tris;
  counters[3] = (long long)cnt.repeats;
  err[0] = de.flags;
  err[1] = de.site;
  err[2] = de.value;
}

// emu_intersect with the step-at-a-time traversal (trav_step).
void emu_intersect_step(void* h, int n, const float* o, const float* d, const int* hints,
                        int smem_nodes, int32_t* tri, float* t, float* u, float* v,
                        int* best_node, long long* counters, long long* err) {
  EmuScene* e = static_cast<EmuScene*>(h);
  const DevScene& s = e->dev;
  std::vector<uint2> smem((size_t)std::max(0, std::min(smem_nodes, s.num_nodes)));
  for (size_t i = 0; i < smem.size(); ++i) {
    smem[i].x = s.nodes[i].meta;
    std::memcpy(&smem[i].y, &s.nodes[i].split, 4);
  }
  DevErr de;
  memset(&de, 0, sizeof de);
  TravCount cnt{};
  for (int i = 0; i < n; ++i) {
    TravState st;
    TravCold tc;
    trav_init(s, Ray{mk(o[3 * i], o[3 * i + 1], o[3 * i + 2]), mk(d[3 * i], d[3 * i + 1], d[3 * i + 2])},
              st, tc, hints ? hints[i] : -1);
    while (!trav_step<true>(s, st, tc, smem.data(), (int)smem.size(), &de, cnt)) {
    }
    tri[i] = st.best.tri;
    t[i] = st.best.rec >= 0 ? st.best.t : 0.f;
    u[i] = st.best.rec >= 0 ? st.best.u : 0.f;
    v[i] = st.best.rec >= 0 ? st.best.v : 0.f;
    if (best_node) best_node[i] = tc.best_node;
  }
  counters[0] = (long long)cnt.nodes;
  counters[1] = (long long)cnt.leaves;
  counters[2] = (long long)cnt.tris;
  counters[3] = (long long)cnt.repeats;
  err[0] = de.flags;
  err[1] = de.site;
  err[2] = de.value;
}

void emu_shade(void* h, int n, const float* o, const float* d, const float* strength,
               const int32_t* tri, const float* t, uint64_t* seeds, int disable_diffuse,
               float* contrib, int32_t* branch, float* hit_p, float* normal, float* strength_out,
               float* param) {
  const DevScene& s = static_cast<EmuScene*>(h)->dev;
  for (int i = 0; i < n; ++i) {
    uint64_t seed = seeds[i];
    const Ray r{mk(o[3 * i], o[3 * i + 1], o[3 * i + 2]), mk(d[3 * i], d[3 * i + 1], d[3 * i + 2])};
    const ShadeOut so = shade_hit(s, r, mk(strength[3 * i], strength[3 * i + 1], strength[3 * i + 2]),
                                  tri[i], t[i], disable_diffuse, seed);
    seeds[i] = seed;
    const float* c = &so.contrib.x;
    for (int k = 0; k < 3; ++k) {
      contrib[3 * i + k] = (&so.contrib.x)[k];
      hit_p[3 * i + k] = (&so.hit_p.x)[k];
      normal[3 * i + k] = (&so.normal.x)[k];
      strength_out[3 * i + k] = (&so.strength.x)[k];
    }
    (void)c;
    param[i] = so.param;
    branch[i] = so.branch;
  }
}

void emu_next_dir(void* h, int n, const int32_t* branch, const float* d, const float* hit_p,
                  const float* normal, const float* strength, const float* param, uint64_t* seeds,
                  float* o_out, float* d_out, float* s_out, int32_t* alive) {
  const DevScene& s = static_cast<EmuScene*>(h)->dev;
  for (int i = 0; i < n; ++i) {
    uint64_t seed = seeds[i];
    const NextOut no = next_direction(s, branch[i], mk(d[3 * i], d[3 * i + 1], d[3 * i + 2]),
                                      mk(hit_p[3 * i], hit_p[3 * i + 1], hit_p[3 * i + 2]),
                                      mk(normal[3 * i], normal[3 * i + 1], normal[3 * i + 2]),
                                      mk(strength[3 * i], strength[3 * i + 1], strength[3 * i + 2]),
                                      param[i], seed);
    seeds[i] = seed;
    for (int k = 0; k < 3; ++k) {
      o_out[3 * i + k] = (&no.o.x)[k];
      d_out[3 * i + k] = (&no.d.x)[k];
      s_out[3 * i + k] = (&no.strength.x)[k];
    }
    alive[i] = no.alive ? 1 : 0;
  }
}

// Packed tree dump for structural tests: meta/split per node, leaf records.
void emu_tree(void* h, uint32_t* meta, float* split, int* leaf_ints /* 16 per leaf */) {
  EmuScene* e = static_cast<EmuScene*>(h);
  for (size_t i = 0; i < e->pk.nodes.size(); ++i) {
    meta[i] = e->pk.nodes[i].meta;
    split[i] = e->pk.nodes[i].split;
  }
  std::memcpy(leaf_ints, e->pk.leaves.data(), e->pk.leaves.size() * sizeof(DevLeaf));
}

}  // extern "C"
