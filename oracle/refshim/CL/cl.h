/* Minimal stand-in for the OpenCL host header, enough for the reference's
 * scene loader and KD-tree builder (which only use the cl_* value types).
 * Test infrastructure: used only to compile the reference checker. */
#ifndef HPT_REFSHIM_CL_H
#define HPT_REFSHIM_CL_H
#include <cstdint>
#include <cfloat>
typedef int32_t cl_int;
typedef uint32_t cl_uint;
typedef int64_t cl_long;
typedef float cl_float;
typedef union { cl_float s[2]; struct { cl_float x, y; }; } cl_float2;
typedef union alignas(16) { cl_float s[4]; struct { cl_float x, y, z, w; }; } cl_float4;
typedef cl_float4 cl_float3;
typedef union alignas(16) { cl_int s[4]; struct { cl_int x, y, z, w; }; } cl_int4;
#define CL_FLT_MAX FLT_MAX
#endif
