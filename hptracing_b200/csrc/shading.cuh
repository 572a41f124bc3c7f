// Shading and next-direction device functions, one per reference kernel
// stage. Same FP32 operation order as src/hp/cl_src/kernel.cl; the
// transcendental calls (acos, sin, cos, asin, pow, exp) are CUDA's
// accurate-path functions and agree with the host's within a few ulp.
#pragma once

#include "checks.cuh"
#include "device_types.h"
#include "dmath.cuh"

namespace hpt {

// Material record, byte-compatible with the reference Material
// (src/hp/cl_src/types.h.cl:19-34), read as six float4.
struct DMat {
  f3 emission, ambient, diffuse, specular;
  float optical_density, dissolve, shininess;
  int diffuse_tex, ambient_tex;
  float p_spec, p_refr, p_diff;
};

HPT_HD DMat load_material(const DevScene& s, int m) {
  const float4* p = reinterpret_cast<const float4*>(s.materials) + 6 * (size_t)m;
  float4 a = ldg(p), b = ldg(p + 1), c = ldg(p + 2), d = ldg(p + 3);
  float4 e = ldg(p + 4), f = ldg(p + 5);
  DMat x;
  x.emission = mk(a.x, a.y, a.z);
  x.ambient = mk(b.x, b.y, b.z);
  x.diffuse = mk(c.x, c.y, c.z);
  x.specular = mk(d.x, d.y, d.z);
  x.optical_density = e.x;
  x.dissolve = e.y;
  x.shininess = e.z;
  x.diffuse_tex = as_int(e.w);
  x.ambient_tex = as_int(f.x);
  x.p_spec = f.y;
  x.p_refr = f.z;
  x.p_diff = f.w;
  return x;
}

HPT_HD f3 load_f4(const float* base, int i) {
  float4 v = ldg(reinterpret_cast<const float4*>(base) + i);
  return mk(v.x, v.y, v.z);
}

// read_imagef on an RGBA UNORM_INT8 image array with
// CLK_NORMALIZED_COORDS_TRUE | CLK_ADDRESS_REPEAT | CLK_FILTER_LINEAR
// (kernel.cl:247-251), evaluated with the OpenCL 1.2 specification's
// formulas in FP32: u = (s - floor(s)) * w, i0 = floor(u - 0.5), i1 = i0 + 1
// (wrapped), a = frac(u - 0.5), and the bilinear sum in the spec's order.
// Non-finite coordinates are treated as 0 (the reference leaves them to
// the sampler hardware).
HPT_HD f3 sample_texture(const DevScene& s, int tex, float su, float sv,
                         DevErr* err = nullptr) {
  if (tex < 0 || tex >= s.num_textures) return mk(0.f, 0.f, 0.f);
  const DevTexInfo ti = s.tex_info[tex];
  if (!hpt_isfinite(su)) su = 0.f;
  if (!hpt_isfinite(sv)) sv = 0.f;
  const float u = rn_mul(rn_sub(su, floorf(su)), (float)ti.w);
  const float v = rn_mul(rn_sub(sv, floorf(sv)), (float)ti.h);
  const float x = rn_sub(u, 0.5f), y = rn_sub(v, 0.5f);
  const float fx = floorf(x), fy = floorf(y);
  int i0 = (int)fx, j0 = (int)fy;
  const float a = rn_sub(x, fx), b = rn_sub(y, fy);
  int i1 = i0 + 1, j1 = j0 + 1;
  if (i0 < 0) i0 += ti.w;
  if (j0 < 0) j0 += ti.h;
  if (i1 > ti.w - 1) i1 -= ti.w;
  if (j1 > ti.h - 1) j1 -= ti.h;
  HPT_DCHECK(err, i0 >= 0 && i0 < ti.w && i1 >= 0 && i1 < ti.w, 306, i0, return mk(0.f, 0.f, 0.f));
  HPT_DCHECK(err, j0 >= 0 && j0 < ti.h && j1 >= 0 && j1 < ti.h, 306, j0, return mk(0.f, 0.f, 0.f));
  const uint32_t* base = s.texels + ti.offset;
  auto texel = [&](int i, int j) {
    uint32_t p = ldg(base + (size_t)j * ti.w + i);
    return mk(rn_div((float)(p & 0xFF), 255.f), rn_div((float)((p >> 8) & 0xFF), 255.f),
              rn_div((float)((p >> 16) & 0xFF), 255.f));
  };
  const float ia = rn_sub(1.f, a), ib = rn_sub(1.f, b);
  f3 r = scale(rn_mul(ia, ib), texel(i0, j0));
  r = add(r, scale(rn_mul(a, ib), texel(i1, j0)));
  r = add(r, scale(rn_mul(ia, b), texel(i0, j1)));
  r = add(r, scale(rn_mul(a, b), texel(i1, j1)));
  return r;
}

enum Branch : int { kDead = -1, kRefract = 0, kSpecular = 1, kDiffuse = 2, kLight = 3 };

struct ShadeOut {
  f3 contrib;    // added to the ray's accumulator
  f3 hit_p, normal, strength;
  float param;   // shininess (specular) / optical density (refract)
  int branch;
};

// s1_run (kernel.cl:258-409) for one hit: hit point, area barycentrics,
// interpolated (unnormalised) or flat normal, UV with V flipped, ambient /
// diffuse textures, self-emission, termination below 1e-4 and the
// one-draw branch choice.
HPT_HD ShadeOut shade_hit(const DevScene& s, const Ray& r, f3 strength,
                                              int tri, float t, int disable_diffuse,
                                              uint64_t& seed, DevErr* err = nullptr) {
  ShadeOut out;
#define HPT_SHADE_FAIL              \
  {                                 \
    out.contrib = mk(0.f, 0.f, 0.f); \
    out.hit_p = out.contrib;        \
    out.normal = out.contrib;       \
    out.strength = out.contrib;     \
    out.param = 0.f;                \
    out.branch = kDead;             \
    return out;                     \
  }
  HPT_DCHECK(err, tri >= 0 && tri < s.num_triangles, 301, tri, HPT_SHADE_FAIL);
  const int4 g = ldg(reinterpret_cast<const int4*>(s.geometry) + tri);
  HPT_DCHECK(err, g.x >= 0 && g.x < s.num_points && g.y >= 0 && g.y < s.num_points && g.z >= 0 &&
                      g.z < s.num_points, 302, tri, HPT_SHADE_FAIL);
  HPT_DCHECK(err, g.w >= 0 && g.w < s.num_materials, 303, g.w, HPT_SHADE_FAIL);
  HPT_DCHECK(err, s.num_normals == 0 || (g.x < s.num_normals && g.y < s.num_normals &&
                                         g.z < s.num_normals), 304, tri, HPT_SHADE_FAIL);
  HPT_DCHECK(err, s.num_texcoords == 0 || (g.x < s.num_texcoords && g.y < s.num_texcoords &&
                                           g.z < s.num_texcoords), 305, tri, HPT_SHADE_FAIL);
#undef HPT_SHADE_FAIL
  const f3 ga = load_f4(s.points, g.x), gb = load_f4(s.points, g.y), gc = load_f4(s.points, g.z);
  const DMat mat = load_material(s, g.w);
  const f3 ip = add(r.o, scale(t, r.d));
  const f3 f1 = sub(ga, ip), f2 = sub(gb, ip), f3v = sub(gc, ip);
  const f3 ab = sub(gb, ga), ac = sub(gc, ga);
  const float area_all = length(cross(ab, ac));
  const float area1 = rn_div(length(cross(f2, f3v)), area_all);
  const float area2 = rn_div(length(cross(f1, f3v)), area_all);
  const float area3 = rn_div(length(cross(f1, f2)), area_all);
  f3 normal;
  if (s.num_normals == 0) {
    normal = normalize(cross(ab, ac));
  } else {
    normal = add(add(scale(area1, load_f4(s.normals, g.x)), scale(area2, load_f4(s.normals, g.y))),
                 scale(area3, load_f4(s.normals, g.z)));
  }
  float uvx = 0.f, uvy = 0.f;
  const bool textured = mat.ambient_tex >= 0 || mat.diffuse_tex >= 0;
  if (textured) {
    if (s.num_texcoords == 0) {
      const float len = rn_sqrt(rn_add(rn_mul(ip.x, ip.x), rn_mul(ip.y, ip.y)));
      uvx = rn_div(ip.x, len);
      uvy = rn_div(ip.y, len);
    } else {
      const float2 ta = ldg(reinterpret_cast<const float2*>(s.texcoords) + g.x);
      const float2 tb = ldg(reinterpret_cast<const float2*>(s.texcoords) + g.y);
      const float2 tc = ldg(reinterpret_cast<const float2*>(s.texcoords) + g.z);
      uvx = rn_add(rn_add(rn_mul(area1, ta.x), rn_mul(area2, tb.x)), rn_mul(area3, tc.x));
      uvy = rn_add(rn_add(rn_mul(area1, ta.y), rn_mul(area2, tb.y)), rn_mul(area3, tc.y));
    }
    uvy = rn_sub(1.f, uvy);
  }
  f3 ambient = mat.ambient;
  if (mat.ambient_tex >= 0) ambient = sample_texture(s, mat.ambient_tex, uvx, uvy, err);
  f3 res = mul(strength, add(ambient, mat.emission));
  res = scale(fabsf(dot(normal, r.d)), res);
  out.contrib = res;
  out.hit_p = ip;
  out.normal = normal;
  out.strength = strength;
  out.param = 0.f;
  out.branch = kDead;
  if (length(strength) < 1e-4f) return out;
  const float rn = lcg_randf(seed);
  if (rn < mat.p_spec) {
    out.branch = kSpecular;
    out.strength = mul(strength, mat.specular);
    out.param = mat.shininess;
    return out;
  }
  if (rn < mat.p_refr) {
    out.branch = kRefract;
    out.strength = scale(rn_sub(1.0f, mat.dissolve), strength);
    out.param = mat.optical_density;
    return out;
  }
  f3 diffuse = mat.diffuse;
  if (mat.diffuse_tex >= 0) diffuse = sample_texture(s, mat.diffuse_tex, uvx, uvy, err);
  out.branch = (rn < mat.p_diff && disable_diffuse == 0) ? kDiffuse : kLight;
  out.strength = mul(strength, diffuse);
  return out;
}

// randf3 (kernel.cl:38-47): alpha, beta in [0, pi] (not a uniform sphere).
HPT_HD f3 randf3(uint64_t& seed) {
  const float alpha = rn_mul(lcg_randf(seed), 3.1415926535f);
  const float beta = rn_mul(lcg_randf(seed), 3.1415926535f);
  const float cb = cosf(beta);
  return mk(rn_mul(cb, cosf(alpha)), rn_mul(cb, sinf(alpha)), sinf(beta));
}

struct NextOut {
  f3 o, d, strength;
  bool alive;
};

// s2_refract_run / s2_specular_run / s2_diffuse_run / s2_light_run
// (kernel.cl:413-557): the next ray leaves hit_p + 1e-5 * dir.
HPT_HD NextOut next_direction(const DevScene& s, int branch, f3 in_dir,
                                                  f3 hit_p, f3 normal, f3 strength,
                                                  float param, uint64_t& seed,
                                                  DevErr* err = nullptr) {
  NextOut out;
  out.strength = strength;
  out.alive = false;
  out.o = hit_p;
  out.d = in_dir;
  f3 dir;
  if (branch == kRefract) {
    const float cos_alpha = dot(in_dir, neg(normal));
    const float reverse = cos_alpha < 0.f ? -1.f : 1.0f;
    const float alpha = acosf(cos_alpha);
    const f3 p = scale(cos_alpha, normal);
    const f3 q = normalize(add(in_dir, p));
    const float sin_beta = rn_mul(sinf(alpha), powf(param, -reverse));
    if (sin_beta <= 1.f) {
      const float beta = asinf(sin_beta);
      dir = add(scale(rn_mul(-reverse, cosf(beta)), normal), scale(sin_beta, q));
    } else {
      dir = add(add(in_dir, p), p);
    }
  } else if (branch == kSpecular) {
    f3 rv = randf3(seed);
    rv = divs(divs(rv, 2.0f), param);
    const float d_ = dot(in_dir, normal);
    const f3 projection = scale(d_, normal);
    dir = sub(in_dir, scale(2.0f, projection));
    dir = add(dir, rv);
  } else if (branch == kDiffuse) {
    const bool front = dot(in_dir, normal) < 0.f;
    f3 p = randf3(seed);
    float dn = dot(p, normal);
    if (dn < 0.f) {
      dn = -dn;
      if (front) p = neg(p);
    }
    out.strength = scale(dn, strength);
    dir = p;
  } else if (branch == kLight) {
    if (s.num_lights == 0) return out;
    const bool front = dot(in_dir, normal) < 0.f;
    const uint32_t ri = lcg_next(seed);
    const int li = (int)((int64_t)ri % (int64_t)s.num_lights);
    HPT_DCHECK(err, li >= 0 && li < s.num_lights, 307, li, return out);
    const int4 light = ldg(reinterpret_cast<const int4*>(s.lights) + li);
    HPT_DCHECK(err, light.x >= 0 && light.x < s.num_points && light.y >= 0 &&
                        light.y < s.num_points && light.z >= 0 && light.z < s.num_points,
               308, li, return out);
    const f3 pa = load_f4(s.points, light.x), pb = load_f4(s.points, light.y),
             pc = load_f4(s.points, light.z);
    float rx = lcg_randf(seed), ry = lcg_randf(seed);
    if (rn_add(rx, ry) > 1.f) {
      rx = rn_sub(1.f, rx);
      ry = rn_sub(1.f, ry);
    }
    const f3 point = add(add(pa, scale(rx, sub(pb, pa))), scale(ry, sub(pc, pa)));
    const f3 p = normalize(sub(point, hit_p));
    const float d_ = dot(p, normal);
    if ((d_ > 0.f) != front) return out;
    out.strength = scale(fabsf(d_), strength);
    dir = p;
  } else {
    return out;
  }
  out.alive = true;
  out.d = dir;
  out.o = add(hit_p, scale(1e-5f, dir));
  return out;
}

// set_viewdirs (kernel.cl:559-585) for ray (x, y) of an nx x ny frame.
HPT_HD f3 pinhole_dir(const float view_top[3], const float view_right[3],
                                          float width, float height, int x, int y, int nx,
                                          int ny) {
  const f3 top = mk(view_top[0], view_top[1], view_top[2]);
  const f3 right = mk(view_right[0], view_right[1], view_right[2]);
  f3 nd = cross(top, right);
  const float fy = rn_sub(rn_mul(rn_div((float)y, (float)ny), height), rn_mul(height, 0.5f));
  nd = add(nd, scale(fy, top));
  const float fx = rn_sub(rn_mul(rn_div((float)x, (float)nx), width), rn_mul(width, 0.5f));
  nd = add(nd, scale(fx, right));
  return normalize(nd);
}

// set_viewdirs_vr (kernel.cl:587-613); sample_y is the panorama height in
// rays. In the source `... * PI - PI / 2.0` subtracts a double (PI is a
// float literal, 2.0 a double), so that step is done in double and rounded.
HPT_HD f3 pano_dir(int x, int y, int x_shift, int sample_y) {
  const float PI = 3.1415926535f;
  const float lon = rn_sub(rn_mul(rn_mul(rn_div((float)(x + x_shift), (float)(sample_y * 2)), PI), 2.f), PI);
  const float lat = d2f_rn(
      dsub_rn((double)rn_mul(rn_div((float)y, (float)sample_y), PI), (double)PI / 2.0));
  const float cl = cosf(lat);
  return normalize(mk(rn_mul(cl, cosf(lon)), sinf(lat), rn_mul(cl, sinf(lon))));
}

}  // namespace hpt
