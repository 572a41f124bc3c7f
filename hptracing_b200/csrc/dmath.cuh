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

namespace hpt {

struct f3 {
  float x, y, z;
};

struct Ray {
  f3 o, d;
};

__device__ __forceinline__ f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 add(f3 a, f3 b) {
  return f3{__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)};
}
__device__ __forceinline__ f3 sub(f3 a, f3 b) {
  return f3{__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)};
}
__device__ __forceinline__ f3 mul(f3 a, f3 b) {
  return f3{__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y), __fmul_rn(a.z, b.z)};
}
__device__ __forceinline__ f3 scale(float s, f3 a) {
  return f3{__fmul_rn(s, a.x), __fmul_rn(s, a.y), __fmul_rn(s, a.z)};
}
__device__ __forceinline__ f3 divs(f3 a, float s) {
  return f3{__fdiv_rn(a.x, s), __fdiv_rn(a.y, s), __fdiv_rn(a.z, s)};
}
__device__ __forceinline__ f3 neg(f3 a) { return f3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ float dot(f3 a, f3 b) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
  return f3{__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
            __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}
__device__ __forceinline__ float length(f3 a) { return __fsqrt_rn(dot(a, a)); }
__device__ __forceinline__ f3 normalize(f3 a) { return divs(a, length(a)); }
__device__ __forceinline__ bool finite3(f3 a) {
  return isfinite(a.x) && isfinite(a.y) && isfinite(a.z);
}

// --- RNG -------------------------------------------------------------------
// The reference's 48-bit LCG (kernel.cl:26-47): s = (s * 0x5DEECE66D + 0xB)
// mod 2^48, output bits 16..47, randf = output / 0xFFFFFFFF in float.
constexpr uint64_t kLcgMask = (1ull << 48) - 1;
__device__ __forceinline__ uint32_t lcg_next(uint64_t& s) {
  s = (s * 0x5DEECE66Dull + 0xBull) & kLcgMask;
  return (uint32_t)((s >> 16) & 0xFFFFFFFFull);
}
__device__ __forceinline__ float lcg_randf(uint64_t& s) {
  return __fdiv_rn(__uint2float_rn(lcg_next(s)), 4294967296.0f);
}

// Counter-based stream key for one (job, ray, sample, bounce): the same
// numbers come out however paths are scheduled, batched or interleaved.
__host__ __device__ __forceinline__ uint64_t path_seed(uint64_t key, uint32_t ray,
                                                       uint32_t sample, uint32_t bounce) {
  uint64_t z = key ^ (((uint64_t)ray << 32) | sample) * 0x9E3779B97F4A7C15ull;
  z ^= (uint64_t)(bounce + 1) * 0xD1B54A32D192ED03ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return z & kLcgMask;
}

}  // namespace hpt
