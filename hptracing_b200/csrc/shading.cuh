// Shading and next-direction device functions, one per reference kernel
// stage. Same FP32 operation order as src/hp/cl_src/kernel.cl; the
// transcendental calls (acos, sin, cos, asin, pow, exp) are CUDA's
// accurate-path functions and agree with the host's within a few ulp.
#pragma once

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

__device__ __forceinline__ DMat load_material(const DevScene& s, int m) {
  const float4* p = reinterpret_cast<const float4*>(s.materials) + 6 * (size_t)m;
  float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
  float4 e = __ldg(p + 4), f = __ldg(p + 5);
  DMat x;
  x.emission = mk(a.x, a.y, a.z);
  x.ambient = mk(b.x, b.y, b.z);
  x.diffuse = mk(c.x, c.y, c.z);
  x.specular = mk(d.x, d.y, d.z);
  x.optical_density = e.x;
  x.dissolve = e.y;
  x.shininess = e.z;
  x.diffuse_tex = __float_as_int(e.w);
  x.ambient_tex = __float_as_int(f.x);
  x.p_spec = f.y;
  x.p_refr = f.z;
  x.p_diff = f.w;
  return x;
}

__device__ __forceinline__ f3 load_f4(const float* base, int i) {
  float4 v = __ldg(reinterpret_cast<const float4*>(base) + i);
  return mk(v.x, v.y, v.z);
}

// read_imagef on an RGBA UNORM_INT8 image array with
// CLK_NORMALIZED_COORDS_TRUE | CLK_ADDRESS_REPEAT | CLK_FILTER_LINEAR
// (kernel.cl:247-251), evaluated with the OpenCL 1.2 specification's
// formulas in FP32: u = (s - floor(s)) * w, i0 = floor(u - 0.5), i1 = i0 + 1
// (wrapped), a = frac(u - 0.5), and the bilinear sum in the spec's order.
// Non-finite coordinates are treated as 0 (the reference leaves them to
// the sampler hardware).
__device__ __forceinline__ f3 sample_texture(const DevScene& s, int tex, float su, float sv) {
  if (tex < 0 || tex >= s.num_textures) return mk(0.f, 0.f, 0.f);
  const DevTexInfo ti = s.tex_info[tex];
  if (!isfinite(su)) su = 0.f;
  if (!isfinite(sv)) sv = 0.f;
  const float u = __fmul_rn(__fsub_rn(su, floorf(su)), (float)ti.w);
  const float v = __fmul_rn(__fsub_rn(sv, floorf(sv)), (float)ti.h);
  const float x = __fsub_rn(u, 0.5f), y = __fsub_rn(v, 0.5f);
  const float fx = floorf(x), fy = floorf(y);
  int i0 = (int)fx, j0 = (int)fy;
  const float a = __fsub_rn(x, fx), b = __fsub_rn(y, fy);
  int i1 = i0 + 1, j1 = j0 + 1;
  if (i0 < 0) i0 += ti.w;
  if (j0 < 0) j0 += ti.h;
  if (i1 > ti.w - 1) i1 -= ti.w;
  if (j1 > ti.h - 1) j1 -= ti.h;
  const uint32_t* base = s.texels + ti.offset;
  auto texel = [&](int i, int j) {
    uint32_t p = __ldg(base + (size_t)j * ti.w + i);
    return mk(__fdiv_rn((float)(p & 0xFF), 255.f), __fdiv_rn((float)((p >> 8) & 0xFF), 255.f),
              __fdiv_rn((float)((p >> 16) & 0xFF), 255.f));
  };
  const float ia = __fsub_rn(1.f, a), ib = __fsub_rn(1.f, b);
  f3 r = scale(__fmul_rn(ia, ib), texel(i0, j0));
  r = add(r, scale(__fmul_rn(a, ib), texel(i1, j0)));
  r = add(r, scale(__fmul_rn(ia, b), texel(i0, j1)));
  r = add(r, scale(__fmul_rn(a, b), texel(i1, j1)));
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
__device__ __forceinline__ ShadeOut shade_hit(const DevScene& s, const Ray& r, f3 strength,
                                              int tri, float t, int disable_diffuse,
                                              uint64_t& seed) {
  ShadeOut out;
  const int4 g = __ldg(reinterpret_cast<const int4*>(s.geometry) + tri);
  const f3 ga = load_f4(s.points, g.x), gb = load_f4(s.points, g.y), gc = load_f4(s.points, g.z);
  const DMat mat = load_material(s, g.w);
  const f3 ip = add(r.o, scale(t, r.d));
  const f3 f1 = sub(ga, ip), f2 = sub(gb, ip), f3v = sub(gc, ip);
  const f3 ab = sub(gb, ga), ac = sub(gc, ga);
  const float area_all = length(cross(ab, ac));
  const float area1 = __fdiv_rn(length(cross(f2, f3v)), area_all);
  const float area2 = __fdiv_rn(length(cross(f1, f3v)), area_all);
  const float area3 = __fdiv_rn(length(cross(f1, f2)), area_all);
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
      const float len = __fsqrt_rn(__fadd_rn(__fmul_rn(ip.x, ip.x), __fmul_rn(ip.y, ip.y)));
      uvx = __fdiv_rn(ip.x, len);
      uvy = __fdiv_rn(ip.y, len);
    } else {
      const float2 ta = __ldg(reinterpret_cast<const float2*>(s.texcoords) + g.x);
      const float2 tb = __ldg(reinterpret_cast<const float2*>(s.texcoords) + g.y);
      const float2 tc = __ldg(reinterpret_cast<const float2*>(s.texcoords) + g.z);
      uvx = __fadd_rn(__fadd_rn(__fmul_rn(area1, ta.x), __fmul_rn(area2, tb.x)), __fmul_rn(area3, tc.x));
      uvy = __fadd_rn(__fadd_rn(__fmul_rn(area1, ta.y), __fmul_rn(area2, tb.y)), __fmul_rn(area3, tc.y));
    }
    uvy = __fsub_rn(1.f, uvy);
  }
  f3 ambient = mat.ambient;
  if (mat.ambient_tex >= 0) ambient = sample_texture(s, mat.ambient_tex, uvx, uvy);
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
    out.strength = scale(__fsub_rn(1.0f, mat.dissolve), strength);
    out.param = mat.optical_density;
    return out;
  }
  f3 diffuse = mat.diffuse;
  if (mat.diffuse_tex >= 0) diffuse = sample_texture(s, mat.diffuse_tex, uvx, uvy);
  out.branch = (rn < mat.p_diff && disable_diffuse == 0) ? kDiffuse : kLight;
  out.strength = mul(strength, diffuse);
  return out;
}

// randf3 (kernel.cl:38-47): alpha, beta in [0, pi] (not a uniform sphere).
__device__ __forceinline__ f3 randf3(uint64_t& seed) {
  const float alpha = __fmul_rn(lcg_randf(seed), 3.1415926535f);
  const float beta = __fmul_rn(lcg_randf(seed), 3.1415926535f);
  const float cb = cosf(beta);
  return mk(__fmul_rn(cb, cosf(alpha)), __fmul_rn(cb, sinf(alpha)), sinf(beta));
}

struct NextOut {
  f3 o, d, strength;
  bool alive;
};

// s2_refract_run / s2_specular_run / s2_diffuse_run / s2_light_run
// (kernel.cl:413-557): the next ray leaves hit_p + 1e-5 * dir.
__device__ __forceinline__ NextOut next_direction(const DevScene& s, int branch, f3 in_dir,
                                                  f3 hit_p, f3 normal, f3 strength,
                                                  float param, uint64_t& seed) {
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
    const float sin_beta = __fmul_rn(sinf(alpha), powf(param, -reverse));
    if (sin_beta <= 1.f) {
      const float beta = asinf(sin_beta);
      dir = add(scale(__fmul_rn(-reverse, cosf(beta)), normal), scale(sin_beta, q));
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
    const int4 light = __ldg(reinterpret_cast<const int4*>(s.lights) + li);
    const f3 pa = load_f4(s.points, light.x), pb = load_f4(s.points, light.y),
             pc = load_f4(s.points, light.z);
    float rx = lcg_randf(seed), ry = lcg_randf(seed);
    if (__fadd_rn(rx, ry) > 1.f) {
      rx = __fsub_rn(1.f, rx);
      ry = __fsub_rn(1.f, ry);
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
__device__ __forceinline__ f3 pinhole_dir(const float view_top[3], const float view_right[3],
                                          float width, float height, int x, int y, int nx,
                                          int ny) {
  const f3 top = mk(view_top[0], view_top[1], view_top[2]);
  const f3 right = mk(view_right[0], view_right[1], view_right[2]);
  f3 nd = cross(top, right);
  const float fy = __fsub_rn(__fmul_rn(__fdiv_rn((float)y, (float)ny), height), __fmul_rn(height, 0.5f));
  nd = add(nd, scale(fy, top));
  const float fx = __fsub_rn(__fmul_rn(__fdiv_rn((float)x, (float)nx), width), __fmul_rn(width, 0.5f));
  nd = add(nd, scale(fx, right));
  return normalize(nd);
}

// set_viewdirs_vr (kernel.cl:587-613); sample_y is the panorama height in
// rays. In the source `... * PI - PI / 2.0` subtracts a double (PI is a
// float literal, 2.0 a double), so that step is done in double and rounded.
__device__ __forceinline__ f3 pano_dir(int x, int y, int x_shift, int sample_y) {
  const float PI = 3.1415926535f;
  const float lon = __fsub_rn(__fmul_rn(__fmul_rn(__fdiv_rn((float)(x + x_shift), (float)(sample_y * 2)), PI), 2.f), PI);
  const float lat = __double2float_rn(
      __dsub_rn((double)__fmul_rn(__fdiv_rn((float)y, (float)sample_y), PI), (double)PI / 2.0));
  const float cl = cosf(lat);
  return normalize(mk(__fmul_rn(cl, cosf(lon)), sinf(lat), __fmul_rn(cl, sinf(lon))));
}

}  // namespace hpt
