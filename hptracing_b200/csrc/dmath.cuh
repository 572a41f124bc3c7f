// Device vector math with the reference's operation order.
//
// The OpenCL kernels (src/hp/cl_src/kernel.cl) are specified here by the
// scalar expansion of their vector built-ins:
//   dot(a, b)     = (a.x*b.x + a.y*b.y) + a.z*b.z
//   cross(a, b)   = (a.y*b.z - a.z*b.y, a.z*b.x - a.x*b.z, a.x*b.y - a.y*b.x)
//   length(a)     = sqrt(dot(a, a))
//   normalize(a)  = a / length(a)   (component-wise IEEE division)
// Every operation below is an explicit round-to-nearest intrinsic, which the
// compiler never contracts into an FMA, so results are bit-identical to the
// same expressions evaluated in IEEE single precision on the host.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstring>

// The per-ray functions are host+device: the same source also compiles for
// the host (test builds), where plain IEEE operations with contraction off
// give the same bits as the device's round-to-nearest intrinsics.
#define HPT_HD __host__ __device__ __forceinline__

namespace hpt {

HPT_HD float rn_add(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fadd_rn(a, b);
#else
  return a + b;
#endif
}
HPT_HD float rn_sub(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fsub_rn(a, b);
#else
  return a - b;
#endif
}
HPT_HD float rn_mul(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fmul_rn(a, b);
#else
  return a * b;
#endif
}
HPT_HD float rn_div(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fdiv_rn(a, b);
#else
  return a / b;
#endif
}
HPT_HD float rn_sqrt(float a) {
#ifdef __CUDA_ARCH__
  return __fsqrt_rn(a);
#else
  return std::sqrt(a);
#endif
}
HPT_HD float rn_rcp(float a) {
#ifdef __CUDA_ARCH__
  return __frcp_rn(a);
#else
  return 1.0f / a;
#endif
}
HPT_HD float u2f_rn(uint32_t u) {
#ifdef __CUDA_ARCH__
  return __uint2float_rn(u);
#else
  return (float)u;
#endif
}
HPT_HD float d2f_rn(double d) {
#ifdef __CUDA_ARCH__
  return __double2float_rn(d);
#else
  return (float)d;
#endif
}
HPT_HD double dsub_rn(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
template <typename T>
HPT_HD T ldg(const T* p) {
#ifdef __CUDA_ARCH__
  return __ldg(p);
#else
  return *p;
#endif
}
HPT_HD float as_float(int i) {
#ifdef __CUDA_ARCH__
  return __int_as_float(i);
#else
  float f;
  std::memcpy(&f, &i, 4);
  return f;
#endif
}
HPT_HD float as_float_u(uint32_t i) {
#ifdef __CUDA_ARCH__
  return __uint_as_float(i);
#else
  float f;
  std::memcpy(&f, &i, 4);
  return f;
#endif
}
HPT_HD int as_int(float f) {
#ifdef __CUDA_ARCH__
  return __float_as_int(f);
#else
  int i;
  std::memcpy(&i, &f, 4);
  return i;
#endif
}
HPT_HD bool hpt_isfinite(float x) {
#ifdef __CUDA_ARCH__
  return isfinite(x);
#else
  return std::isfinite(x);
#endif
}
HPT_HD void hpt_atomic_or(uint32_t* p, uint32_t v) {
#ifdef __CUDA_ARCH__
  atomicOr(p, v);
#else
  *p |= v;
#endif
}

struct f3 {
  float x, y, z;
};

struct Ray {
  f3 o, d;
};

HPT_HD f3 mk(float x, float y, float z) { return f3{x, y, z}; }
HPT_HD f3 add(f3 a, f3 b) {
  return f3{rn_add(a.x, b.x), rn_add(a.y, b.y), rn_add(a.z, b.z)};
}
HPT_HD f3 sub(f3 a, f3 b) {
  return f3{rn_sub(a.x, b.x), rn_sub(a.y, b.y), rn_sub(a.z, b.z)};
}
HPT_HD f3 mul(f3 a, f3 b) {
  return f3{rn_mul(a.x, b.x), rn_mul(a.y, b.y), rn_mul(a.z, b.z)};
}
HPT_HD f3 scale(float s, f3 a) {
  return f3{rn_mul(s, a.x), rn_mul(s, a.y), rn_mul(s, a.z)};
}
HPT_HD f3 divs(f3 a, float s) {
  return f3{rn_div(a.x, s), rn_div(a.y, s), rn_div(a.z, s)};
}
HPT_HD f3 neg(f3 a) { return f3{-a.x, -a.y, -a.z}; }
HPT_HD float dot(f3 a, f3 b) {
  return rn_add(rn_add(rn_mul(a.x, b.x), rn_mul(a.y, b.y)), rn_mul(a.z, b.z));
}
HPT_HD f3 cross(f3 a, f3 b) {
  return f3{rn_sub(rn_mul(a.y, b.z), rn_mul(a.z, b.y)),
            rn_sub(rn_mul(a.z, b.x), rn_mul(a.x, b.z)),
            rn_sub(rn_mul(a.x, b.y), rn_mul(a.y, b.x))};
}
HPT_HD float length(f3 a) { return rn_sqrt(dot(a, a)); }
HPT_HD f3 normalize(f3 a) { return divs(a, length(a)); }
HPT_HD bool finite3(f3 a) {
  return hpt_isfinite(a.x) && hpt_isfinite(a.y) && hpt_isfinite(a.z);
}

// --- RNG -------------------------------------------------------------------
// The reference's 48-bit LCG (kernel.cl:26-47): s = (s * 0x5DEECE66D + 0xB)
// mod 2^48, output bits 16..47, randf = output / 0xFFFFFFFF in float.
constexpr uint64_t kLcgMask = (1ull << 48) - 1;
HPT_HD uint32_t lcg_next(uint64_t& s) {
  s = (s * 0x5DEECE66Dull + 0xBull) & kLcgMask;
  return (uint32_t)((s >> 16) & 0xFFFFFFFFull);
}
HPT_HD float lcg_randf(uint64_t& s) {
  return rn_div(u2f_rn(lcg_next(s)), 4294967296.0f);
}

// Counter-based stream key for one (job, ray, sample, bounce): the same
// numbers come out however paths are scheduled, batched or interleaved.
__host__ HPT_HD uint64_t path_seed(uint64_t key, uint32_t ray,
                                                       uint32_t sample, uint32_t bounce) {
  uint64_t z = key ^ (((uint64_t)ray << 32) | sample) * 0x9E3779B97F4A7C15ull;
  z ^= (uint64_t)(bounce + 1) * 0xD1B54A32D192ED03ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return z & kLcgMask;
}

}  // namespace hpt
