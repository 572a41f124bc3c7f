// opencl_c.h - just enough of OpenCL C 1.2 to compile the reference's
// src/hp/cl_src/kernel.cl (and types.h.cl) as C++ on the host.
// Test infrastructure: it exists so the checker can run the reference's own
// kernel source; nothing in the product uses it.
//
// Vector built-ins are defined by their scalar expansion in left-to-right
// order (dot(a,b) = a.x*b.x + a.y*b.y + a.z*b.z, normalize(v) = v/length(v));
// compile with -ffp-contract=off. read_imagef / write_imagef follow the
// OpenCL 1.2 specification for RGBA UNORM_INT8 images with normalized
// coordinates, CLK_ADDRESS_REPEAT and CLK_FILTER_LINEAR.
#pragma once

#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <type_traits>

using std::acos;
using std::asin;
using std::cos;
using std::exp;
using std::fabs;
using std::fmax;
using std::fmin;
using std::pow;
using std::sin;
using std::sqrt;

#undef RAND_MAX

struct float2 {
  union {
    struct {
      float x, y;
    };
    struct {
      float s0, s1;
    };
  };
};
struct alignas(16) float3 {
  union {
    struct {
      float x, y, z, w;
    };
    struct {
      float s0, s1, s2, s3;
    };
    float2 xy;
  };
};
struct alignas(16) float4 {
  union {
    struct {
      float x, y, z, w;
    };
    struct {
      float s0, s1, s2, s3;
    };
    float3 xyz;
    float2 xy;
  };
};
struct int2 {
  int x, y;
};
struct alignas(16) int4 {
  union {
    struct {
      int x, y, z, w;
    };
    struct {
      int s0, s1, s2, s3;
    };
  };
};
static_assert(sizeof(float3) == 16 && sizeof(float4) == 16 && sizeof(int4) == 16, "cl sizes");

inline float2 make_float2(float x, float y) { float2 r; r.x = x; r.y = y; return r; }
inline float3 make_float3(float x, float y, float z) { float3 r; r.x = x; r.y = y; r.z = z; r.w = 0; return r; }
inline float4 make_float4(float x, float y, float z, float w) {
  float4 r; r.x = x; r.y = y; r.z = z; r.w = w; return r;
}
inline int2 make_int2(int x, int y) { int2 r; r.x = x; r.y = y; return r; }

template <typename S>
using if_scalar = typename std::enable_if<std::is_arithmetic<S>::value, int>::type;

// float3
inline float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
template <typename S, if_scalar<S> = 0>
inline float3 operator*(float3 a, S s) { float f = (float)s; return make_float3(a.x * f, a.y * f, a.z * f); }
template <typename S, if_scalar<S> = 0>
inline float3 operator*(S s, float3 a) { float f = (float)s; return make_float3(f * a.x, f * a.y, f * a.z); }
template <typename S, if_scalar<S> = 0>
inline float3 operator/(float3 a, S s) { float f = (float)s; return make_float3(a.x / f, a.y / f, a.z / f); }
inline float3& operator+=(float3& a, float3 b) { a = a + b; return a; }
template <typename S, if_scalar<S> = 0>
inline float3& operator*=(float3& a, S s) { a = a * s; return a; }

// float2
inline float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
template <typename S, if_scalar<S> = 0>
inline float2 operator*(S s, float2 a) { float f = (float)s; return make_float2(f * a.x, f * a.y); }

// float4
template <typename S, if_scalar<S> = 0>
inline float4& operator/=(float4& a, S s) {
  float f = (float)s; a.x /= f; a.y /= f; a.z /= f; a.w /= f; return a;
}
template <typename S, if_scalar<S> = 0>
inline float4& operator*=(float4& a, S s) {
  float f = (float)s; a.x *= f; a.y *= f; a.z *= f; a.w *= f; return a;
}

inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
inline float3 cross(float3 a, float3 b) {
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float length(float3 a) { return std::sqrt(dot(a, a)); }
inline float length(float2 a) { return std::sqrt(dot(a, a)); }
inline float3 normalize(float3 a) { float l = length(a); return make_float3(a.x / l, a.y / l, a.z / l); }
inline float2 normalize(float2 a) { float l = length(a); return make_float2(a.x / l, a.y / l); }

template <typename T>
inline float convert_float(T v) { return (float)v; }

// Work-item ids, set by the driver before each call.
extern thread_local size_t hpt_cl_gid[2];
inline size_t get_global_id(int d) { return hpt_cl_gid[d]; }

inline int atomic_inc(int* p) { return __atomic_fetch_add(p, 1, __ATOMIC_RELAXED); }
inline unsigned atomic_cmpxchg(volatile unsigned* p, unsigned cmp, unsigned val) {
  unsigned expected = cmp;
  __atomic_compare_exchange_n((unsigned*)p, &expected, val, false, __ATOMIC_RELAXED,
                              __ATOMIC_RELAXED);
  return expected;
}

// Images: RGBA UNORM_INT8.
struct hpt_cl_image {
  int width, height, depth;
  const int* dims;  // (w, h) per layer when layers differ; may be null
  const long long* offsets;  // texel offset per layer; may be null
  const unsigned char* data;
  unsigned char* wdata;
};
typedef hpt_cl_image* image2d_array_t;
typedef hpt_cl_image* image3d_t;
typedef hpt_cl_image* image2d_t;
typedef int sampler_t;
#define CLK_NORMALIZED_COORDS_TRUE 1
#define CLK_NORMALIZED_COORDS_FALSE 0
#define CLK_ADDRESS_REPEAT 2
#define CLK_FILTER_LINEAR 4
#define CLK_FILTER_NEAREST 0

inline float4 read_imagef(image2d_array_t img, sampler_t, float4 c) {
  int layer = (int)std::nearbyint(c.z);
  if (layer < 0) layer = 0;
  if (layer > img->depth - 1) layer = img->depth - 1;
  const int w = img->dims ? img->dims[2 * layer] : img->width;
  const int h = img->dims ? img->dims[2 * layer + 1] : img->height;
  const long long off = img->offsets ? img->offsets[layer] : (long long)layer * w * h;
  float su = c.x, sv = c.y;
  if (!std::isfinite(su)) su = 0.f;
  if (!std::isfinite(sv)) sv = 0.f;
  float u = (su - std::floor(su)) * (float)w;
  float v = (sv - std::floor(sv)) * (float)h;
  float x = u - 0.5f, y = v - 0.5f;
  float fx = std::floor(x), fy = std::floor(y);
  int i0 = (int)fx, j0 = (int)fy;
  float a = x - fx, b = y - fy;
  int i1 = i0 + 1, j1 = j0 + 1;
  if (i0 < 0) i0 += w;
  if (j0 < 0) j0 += h;
  if (i1 > w - 1) i1 -= w;
  if (j1 > h - 1) j1 -= h;
  auto T = [&](int i, int j, int ch) {
    return (float)img->data[4 * (off + (long long)j * w + i) + ch] / 255.f;
  };
  float4 r;
  r.w = 0.f;
  float* out[3] = {&r.x, &r.y, &r.z};
  for (int ch = 0; ch < 3; ++ch) {
    float s = (1.f - a) * (1.f - b) * T(i0, j0, ch);
    s = s + a * (1.f - b) * T(i1, j0, ch);
    s = s + (1.f - a) * b * T(i0, j1, ch);
    s = s + a * b * T(i1, j1, ch);
    *out[ch] = s;
  }
  return r;
}

inline int get_image_width(image2d_t img) { return img->width; }
inline int get_image_height(image2d_t img) { return img->height; }

inline unsigned char hpt_cl_unorm8(float x) {
  float v = x * 255.0f;
  if (!(v >= 0.f)) return 0;
  if (v >= 255.f) return 255;
  return (unsigned char)std::nearbyint(v);
}
inline void write_imagef(image2d_t img, int2 c, float4 p) {
  unsigned char* o = img->wdata + 4 * ((long long)c.y * img->width + c.x);
  o[0] = hpt_cl_unorm8(p.x);
  o[1] = hpt_cl_unorm8(p.y);
  o[2] = hpt_cl_unorm8(p.z);
  o[3] = hpt_cl_unorm8(p.w);
}

#define __kernel
#define __global
#define global
#define __constant
#define __read_only
#define __write_only
#define CL_VERSION_1_2 1
