// refcl_driver.cpp - drives the reference's own OpenCL kernels
// (src/hp/cl_src/kernel.cl, compiled as C++ through refshim/opencl_c.h) on
// host threads. Test infrastructure: the checker that pins the oracle
// restatement and the timed "reference" CPU arm of bench.py. It is built
// by oracle/build.py into oracle/_ref/ only where the reference sources are
// available; the kernel source itself is never copied into the repository.
//
// refcl_render restates the host loop of TraceRunner::run
// (src/hp/trace_runner.cpp:116-356) with one work-item per loop index; the
// per-lane seeds come from a seeded generator instead of srand(time(0)),
// and the result buffer is zeroed (the reference never initialises it).
#include "refshim/opencl_c.h"
// clang-format off
#include "_ref/types_h_cl.inc"
#include "_ref/kernel_cl.inc"
// clang-format on

#include <algorithm>
#include <cstring>
#include <functional>
#include <random>
#include <thread>
#include <vector>

thread_local size_t hpt_cl_gid[2];

namespace {

// Runs fn(gid) for gid in [0, n) over `threads` host threads.
void ndrange(int64_t n, int threads, const std::function<void()>& fn) {
  auto run = [&](int64_t b, int64_t e) {
    for (int64_t g = b; g < e; ++g) {
      hpt_cl_gid[0] = (size_t)g;
      hpt_cl_gid[1] = 0;
      fn();
    }
  };
  if (threads <= 1 || n < 512) {
    run(0, n);
    return;
  }
  std::vector<std::thread> ts;
  int64_t chunk = (n + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    int64_t b = t * chunk, e = std::min(n, b + chunk);
    if (b >= e) break;
    ts.emplace_back(run, b, e);
  }
  for (auto& t : ts) t.join();
}

void ndrange2(int nx, int ny, const std::function<void()>& fn) {
  for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x) {
      hpt_cl_gid[0] = (size_t)x;
      hpt_cl_gid[1] = (size_t)y;
      fn();
    }
}

}  // namespace

extern "C" {

struct RefclScene {
  const float* points;   // cl_float3 (16 B)
  const float* normals;
  int32_t num_normals;
  const float* texcoords;
  int32_t num_texcoords;
  const int32_t* triangles;
  int32_t num_triangles;
  const void* nodes;
  int32_t num_nodes;
  const int32_t* leaf_data;
  const void* materials;
  const int32_t* lights;
  int32_t num_lights;
  const uint8_t* texture_data;
  int32_t num_textures;
  const int32_t* texture_dims;
};

struct RefclCamera {
  float view_p[3], top_dir[3], right_dir[3];
  float width, height;
};

}  // extern "C"

namespace {

struct Images {
  hpt_cl_image img;
  std::vector<long long> offsets;
  std::vector<int> dims;
  unsigned char dummy[4] = {0, 0, 0, 0};
  explicit Images(const RefclScene& s) {
    memset(&img, 0, sizeof img);
    if (s.num_textures <= 0) {  // trace_runner.cpp:79-86: a 1x1x1 image
      img.width = img.height = img.depth = 1;
      img.data = dummy;
      return;
    }
    long long off = 0;
    for (int t = 0; t < s.num_textures; ++t) {
      offsets.push_back(off);
      dims.push_back(s.texture_dims[2 * t]);
      dims.push_back(s.texture_dims[2 * t + 1]);
      off += (long long)s.texture_dims[2 * t] * s.texture_dims[2 * t + 1];
    }
    img.width = dims[0];
    img.height = dims[1];
    img.depth = s.num_textures;
    img.dims = dims.data();
    img.offsets = offsets.data();
    img.data = s.texture_data;
  }
};

float3 f3(const float* p) { return make_float3(p[0], p[1], p[2]); }

}  // namespace

extern "C" {

int refcl_sizeof_unit_data(void) { return (int)sizeof(unit_data); }

// kdtree_intersect over n rays (sample_n = 1, background 0). geometry_out:
// int4 per ray (zero on a miss); hit: 1/0.
void refcl_intersect(const RefclScene* s, int n, const float* o, const float* d,
                     int32_t* geometry_out, float* t_out, int32_t* hit, int threads) {
  std::vector<unit_data> data(n);
  memset(data.data(), 0, n * sizeof(unit_data));
  std::vector<int> s0(n), s1(n, -1);
  for (int i = 0; i < n; ++i) {
    data[i].orig_id = i;
    data[i].strength = make_float3(1, 1, 1);
    data[i].start_p = f3(o + 3 * i);
    data[i].in_dir = f3(d + 3 * i);
    s0[i] = i;
  }
  std::vector<float> result(3 * (size_t)n, 0.f);
  int sizes[10] = {0};
  sizes[0] = n;
  float3 bg = make_float3(0, 0, 0);
  ndrange(n, threads, [&]() {
    kdtree_intersect(sizes, data.data(), s0.data(), s1.data(), (float3*)s->points,
                     (int4*)s->triangles, (int*)s->leaf_data, (KDTreeNodeHeader*)s->nodes,
                     s->num_nodes, result.data(), bg, 1);
  });
  std::vector<uint8_t> is_hit(n, 0);
  for (int k = 0; k < sizes[1]; ++k) is_hit[s1[k]] = 1;
  for (int i = 0; i < n; ++i) {
    hit[i] = is_hit[i];
    const int4& g = data[i].geometry;
    geometry_out[4 * i] = is_hit[i] ? g.x : 0;
    geometry_out[4 * i + 1] = is_hit[i] ? g.y : 0;
    geometry_out[4 * i + 2] = is_hit[i] ? g.z : 0;
    geometry_out[4 * i + 3] = is_hit[i] ? g.w : 0;
    t_out[i] = is_hit[i] ? data[i].intersect_number : 0.f;
  }
}

// s1_run over n hits with S1 = [0, n): element i draws from seeds[i]
// (v_seed[i] is set to seeds[i] - i, the kernel adds global_id back).
void refcl_shade(const RefclScene* s, int n, const float* o, const float* d, const float* strength,
                 const int32_t* tri, const float* t, int64_t* seeds, int disable_diffuse,
                 float* contrib, int32_t* branch, float* hit_p, float* normal, float* strength_out,
                 float* param) {
  Images im(*s);
  std::vector<unit_data> data(n);
  memset(data.data(), 0, n * sizeof(unit_data));
  std::vector<int> s1(n), l[4];
  for (int k = 0; k < 4; ++k) l[k].assign(n, -1);
  std::vector<long> v_seed(n);
  for (int i = 0; i < n; ++i) {
    unit_data& u = data[i];
    u.orig_id = i;
    u.start_p = f3(o + 3 * i);
    u.in_dir = f3(d + 3 * i);
    u.strength = f3(strength + 3 * i);
    const int32_t* g = s->triangles + 4 * tri[i];
    u.geometry.x = g[0]; u.geometry.y = g[1]; u.geometry.z = g[2]; u.geometry.w = g[3];
    u.intersect_number = t[i];
    s1[i] = i;
    v_seed[i] = (long)(seeds[i] - i);
  }
  std::vector<float> result(3 * (size_t)n, 0.f);
  int sizes[10] = {0};
  sizes[1] = n;
  ndrange(n, 1, [&]() {
    s1_run(sizes, data.data(), s1.data(), result.data(), l[0].data(), l[1].data(), l[2].data(),
           l[3].data(), (float3*)s->points, (float3*)s->normals, s->num_normals,
           (float2*)s->texcoords, s->num_texcoords, (Material*)s->materials, &im.img,
           disable_diffuse, v_seed.data());
  });
  std::vector<int> br(n, -1);
  for (int k = 0; k < 4; ++k)
    for (int j = 0; j < sizes[2 + k]; ++j) br[l[k][j]] = k;
  for (int i = 0; i < n; ++i) {
    const unit_data& u = data[i];
    branch[i] = br[i];
    seeds[i] = (int64_t)v_seed[i];
    for (int c = 0; c < 3; ++c) contrib[3 * i + c] = result[3 * i + c];
    hit_p[3 * i] = u.intersect_p.x; hit_p[3 * i + 1] = u.intersect_p.y; hit_p[3 * i + 2] = u.intersect_p.z;
    normal[3 * i] = u.normal.x; normal[3 * i + 1] = u.normal.y; normal[3 * i + 2] = u.normal.z;
    strength_out[3 * i] = u.strength.x;
    strength_out[3 * i + 1] = u.strength.y;
    strength_out[3 * i + 2] = u.strength.z;
    param[i] = br[i] == 1 ? u.shininess : (br[i] == 0 ? u.optical_density : 0.f);
  }
}

// One s2_*_run kernel over n records of the given branch, S2 list = [0, n).
void refcl_next(const RefclScene* s, int branch, int n, const float* d, const float* hit_p,
                const float* normal, const float* strength, const float* param, int64_t* seeds,
                float* o_out, float* d_out, float* s_out, int32_t* alive) {
  std::vector<unit_data> data(n);
  memset(data.data(), 0, n * sizeof(unit_data));
  std::vector<int> list(n), s0(n, -1);
  std::vector<long> v_seed(n);
  for (int i = 0; i < n; ++i) {
    unit_data& u = data[i];
    u.orig_id = i;
    u.in_dir = f3(d + 3 * i);
    u.intersect_p = f3(hit_p + 3 * i);
    u.start_p = u.intersect_p;
    u.normal = f3(normal + 3 * i);
    u.strength = f3(strength + 3 * i);
    u.shininess = param[i];
    u.optical_density = param[i];
    list[i] = i;
    v_seed[i] = (long)(seeds[i] - i);
  }
  int sizes[10] = {0};
  sizes[2 + branch] = n;
  ndrange(n, 1, [&]() {
    switch (branch) {
      case 0: s2_refract_run(sizes, data.data(), list.data(), s0.data()); break;
      case 1: s2_specular_run(sizes, data.data(), list.data(), s0.data(), v_seed.data()); break;
      case 2: s2_diffuse_run(sizes, data.data(), list.data(), s0.data(), v_seed.data()); break;
      default:
        s2_light_run(sizes, data.data(), list.data(), s0.data(), (int4*)s->lights, s->num_lights,
                     (float3*)s->points, v_seed.data());
    }
  });
  std::vector<uint8_t> al(n, 0);
  for (int j = 0; j < sizes[0]; ++j) al[s0[j]] = 1;
  for (int i = 0; i < n; ++i) {
    const unit_data& u = data[i];
    alive[i] = al[i];
    if (branch == 0) seeds[i] = seeds[i];
    else if (branch == 3 && s->num_lights == 0) seeds[i] = seeds[i];
    else seeds[i] = (int64_t)v_seed[i];
    o_out[3 * i] = u.start_p.x; o_out[3 * i + 1] = u.start_p.y; o_out[3 * i + 2] = u.start_p.z;
    d_out[3 * i] = u.in_dir.x; d_out[3 * i + 1] = u.in_dir.y; d_out[3 * i + 2] = u.in_dir.z;
    s_out[3 * i] = u.strength.x; s_out[3 * i + 1] = u.strength.y; s_out[3 * i + 2] = u.strength.z;
  }
}

// set_viewdirs / set_viewdirs_vr with the host arguments of
// trace_runner.cpp:131-150.
void refcl_raygen(const RefclCamera* c, int sample_x, int sample_y, int ssx, int ssy, float* o,
                  float* d) {
  const int nx = sample_x * ssx, ny = sample_y * ssy;
  std::vector<unit_data> data((size_t)nx * ny);
  memset(data.data(), 0, data.size() * sizeof(unit_data));
  float3 vp = f3(c->view_p), top = f3(c->top_dir), right = f3(c->right_dir);
  if (c->height < 0) {
    int shift = (int)c->right_dir[0];
    ndrange2(nx, ny, [&]() {
      set_viewdirs_vr(vp, shift * ssx, sample_x * ssy, sample_y * ssy, data.data());
    });
  } else {
    ndrange2(nx, ny, [&]() {
      set_viewdirs(vp, top, right, c->width, c->height, nx, ny, data.data());
    });
  }
  for (size_t i = 0; i < data.size(); ++i) {
    o[3 * i] = data[i].start_p.x; o[3 * i + 1] = data[i].start_p.y; o[3 * i + 2] = data[i].start_p.z;
    d[3 * i] = data[i].in_dir.x; d[3 * i + 1] = data[i].in_dir.y; d[3 * i + 2] = data[i].in_dir.z;
  }
}

void refcl_get_image(const float* accum, int W, int H, int ssx, int ssy, int sample,
                     float brightness, uint8_t* rgba) {
  hpt_cl_image img;
  memset(&img, 0, sizeof img);
  img.width = W;
  img.height = H;
  img.depth = 1;
  img.wdata = rgba;
  ndrange2(W, H, [&]() { get_image((float*)accum, ssx, ssy, sample, brightness, &img); });
}

// TraceRunner::run (trace_runner.cpp:116-356). counts[0] = intersect
// queries, counts[1] = shade calls.
void refcl_render(const RefclScene* s, const RefclCamera* c, int sample_x, int sample_y, int ssx,
                  int ssy, const float* bg, int sample, int depth, int disable_diffuse,
                  float brightness, uint64_t seed, int threads, uint8_t* rgba, float* accum_out,
                  int64_t* counts) {
  Images im(*s);
  const int64_t ray_count = (int64_t)sample_x * ssx * sample_y * ssy;
  std::vector<unit_data> data_initial(ray_count);
  memset(data_initial.data(), 0, ray_count * sizeof(unit_data));
  float3 vp = f3(c->view_p), top = f3(c->top_dir), right = f3(c->right_dir);
  if (c->height < 0) {
    int shift = (int)c->right_dir[0];
    ndrange2(sample_x * ssx, sample_y * ssy, [&]() {
      set_viewdirs_vr(vp, shift * ssx, sample_x * ssy, sample_y * ssy, data_initial.data());
    });
  } else {
    ndrange2(sample_x * ssx, sample_y * ssy, [&]() {
      set_viewdirs(vp, top, right, c->width, c->height, sample_x * ssx, sample_y * ssy,
                   data_initial.data());
    });
  }
  std::vector<float> results(3 * ray_count, 0.f);
  int sizes[10] = {0};
  std::vector<int> stage_cache(ray_count);
  for (int64_t i = 0; i < ray_count; ++i) stage_cache[i] = (int)i;
  std::vector<int> stage[6];
  for (auto& st : stage) st.assign(ray_count, 0);
  std::vector<long> seeds(ray_count);
  std::mt19937 gen((uint32_t)seed);
  for (auto& x : seeds) x = (long)(gen() & 0x7FFFFFFF);
  float3 bgc = make_float3(bg[0], bg[1], bg[2]);
  sizes[0] = (int)ray_count;
  int64_t queries = ray_count, shades = 0;
  ndrange(ray_count, threads, [&]() {
    kdtree_intersect(sizes, data_initial.data(), stage_cache.data(), stage[1].data(),
                     (float3*)s->points, (int4*)s->triangles, (int*)s->leaf_data,
                     (KDTreeNodeHeader*)s->nodes, s->num_nodes, results.data(), bgc, sample);
  });
  stage_cache = stage[1];
  const int initial_s1 = sizes[1];
  std::vector<unit_data> data;
  for (int ii = 0; ii < sample; ++ii) {
    memset(sizes, 0, sizeof sizes);
    sizes[1] = initial_s1;
    data = data_initial;
    stage[1] = stage_cache;
    for (int i = 0; i < depth; ++i) {
      if (sizes[0]) {
        queries += sizes[0];
        ndrange(sizes[0], threads, [&]() {
          kdtree_intersect(sizes, data.data(), stage[0].data(), stage[1].data(),
                           (float3*)s->points, (int4*)s->triangles, (int*)s->leaf_data,
                           (KDTreeNodeHeader*)s->nodes, s->num_nodes, results.data(), bgc, 1);
        });
      }
      if (sizes[1]) {
        shades += sizes[1];
        ndrange(sizes[1], threads, [&]() {
          s1_run(sizes, data.data(), stage[1].data(), results.data(), stage[2].data(),
                 stage[3].data(), stage[4].data(), stage[5].data(), (float3*)s->points,
                 (float3*)s->normals, s->num_normals, (float2*)s->texcoords, s->num_texcoords,
                 (Material*)s->materials, &im.img, disable_diffuse, seeds.data());
        });
      }
      sizes[0] = sizes[1] = 0;
      if (i == depth - 1) break;
      for (int k = 0; k < 4; ++k) {
        const int nk = sizes[k + 2];
        if (!nk) continue;
        ndrange(nk, threads, [&]() {
          switch (k) {
            case 0: s2_refract_run(sizes, data.data(), stage[2].data(), stage[0].data()); break;
            case 1:
              s2_specular_run(sizes, data.data(), stage[3].data(), stage[0].data(), seeds.data());
              break;
            case 2:
              s2_diffuse_run(sizes, data.data(), stage[4].data(), stage[0].data(), seeds.data());
              break;
            default:
              s2_light_run(sizes, data.data(), stage[5].data(), stage[0].data(), (int4*)s->lights,
                           s->num_lights, (float3*)s->points, seeds.data());
          }
        });
      }
      sizes[2] = sizes[3] = sizes[4] = sizes[5] = 0;
    }
  }
  if (accum_out) memcpy(accum_out, results.data(), results.size() * sizeof(float));
  if (rgba) refcl_get_image(results.data(), sample_x, sample_y, ssx, ssy, sample, brightness, rgba);
  if (counts) {
    counts[0] = queries;
    counts[1] = shades;
  }
}

}  // extern "C"
