// Closest-hit query against the rope KD-tree.
//
// Result contract (src/hp/cl_src/kernel.cl:111-208): the hit is the
// minimum-t triangle over the leaves whose reference box passes
// _box_intersect (kernel.cl:56-83), tested with the reference's
// Moller-Trumbore (kernel.cl:85-109) in the same FP32 operation order; on an
// exact tie in t the triangle the reference meets first wins (leaf lists
// are stored in the reference's gather order, so the lower position wins).
//
// The reference gathers every leaf the ray's line pierces and tests them
// all. Here the leaves are walked front to back with ropes (stackless) and
// the walk stops once the next leaf starts beyond the best hit plus a small
// slack (so ties and rounding at leaf faces are still visited). Leaves are
// still filtered with the reference's own box test on the reference box, so
// every triangle considered is one the reference would consider.
// The one reference behaviour not reproduced is its 512-leaf gather cap
// (kernel.cl:133, 146): a ray whose line pierces more than 512 leaves may
// lose its true closest hit in the reference, never here.
#pragma once

#include "device_types.h"
#include "dmath.cuh"

namespace hpt {

struct Hit {
  int32_t rec;   // position in the leaf lists (reference rank), -1 = none
  int32_t tri;   // triangle id
  float t, u, v;
};

// _box_intersect (kernel.cl:56-83) with the slab distances kept for the
// exit computation: returns the reference's verdict; t_exit is the
// smallest far-slab distance over axes with a non-zero direction and
// exit_face its face (2*axis + 1 if leaving through the high side).
__device__ __forceinline__ bool leaf_slabs(const Ray& r, const float lo[3], const float hi[3],
                                           float& t_exit, int& exit_face) {
  const float o[3] = {r.o.x, r.o.y, r.o.z};
  const float d[3] = {r.d.x, r.d.y, r.d.z};
  bool inside = true;
  float max_of_mins = 0.f, min_of_maxs = 0.f;
  t_exit = __int_as_float(0x7f800000);  // +inf
  exit_face = -1;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    inside = inside && o[a] >= lo[a] && o[a] <= hi[a];
    float t0 = __fdiv_rn(__fsub_rn(lo[a], o[a]), d[a]);
    float t1 = __fdiv_rn(__fsub_rn(hi[a], o[a]), d[a]);
    float mn = fminf(t0, t1), mx = fmaxf(t0, t1);
    max_of_mins = a == 0 ? mn : fmaxf(max_of_mins, mn);
    min_of_maxs = a == 0 ? mx : fminf(min_of_maxs, mx);
    if (d[a] != 0.f) {
      float tf = d[a] > 0.f ? t1 : t0;
      if (tf < t_exit) {
        t_exit = tf;
        exit_face = 2 * a + (d[a] > 0.f ? 1 : 0);
      }
    }
  }
  if (inside) return true;
  if (min_of_maxs <= 0.f) return false;
  return max_of_mins <= min_of_maxs;
}

// _single_intersect (kernel.cl:85-109) on a pre-subtracted record. The
// epsilon test at kernel.cl:93 can never be true and is omitted.
__device__ __forceinline__ bool mt_test(const Ray& r, const float4 A, const float4 E1,
                                        const float4 E2, float& t, float& u, float& v) {
  f3 a = mk(A.x, A.y, A.z), e1 = mk(E1.x, E1.y, E1.z), e2 = mk(E2.x, E2.y, E2.z);
  f3 P = cross(r.d, e2);
  float det = dot(e1, P);
  float inv_det = __fdiv_rn(1.f, det);
  f3 T = sub(r.o, a);
  u = __fmul_rn(dot(T, P), inv_det);
  if (u < 0.f || u > 1.f) return false;
  f3 Q = cross(T, e1);
  v = __fmul_rn(dot(r.d, Q), inv_det);
  if (v < 0.f || __fadd_rn(u, v) > 1.f) return false;
  t = __fmul_rn(dot(e2, Q), inv_det);
  return t > 0.f;
}

// Traversal state of one ray; lives in registers so a lane can be
// refilled with a new ray between leaves.
struct TravState {
  Ray ray;
  float t_entry, t_end;  // current entry distance, scene exit distance
  float slack;           // world-space rounding slack in t units
  int32_t node;          // node to descend from, -1 = finished
  int32_t steps;
  Hit best;
};

// Work counters of one lane (summed over the rays it traced).
struct TravCount {
  unsigned long long nodes = 0, leaves = 0, tris = 0;
};

__device__ __forceinline__ void trav_init(const DevScene& s, const Ray& r, TravState& st) {
  st.ray = r;
  st.best.rec = -1;
  st.best.tri = -1;
  st.best.t = 0.f;
  st.best.u = st.best.v = 0.f;
  st.steps = 0;
  st.node = -1;
  if (!finite3(r.o) || !finite3(r.d)) return;
  const float o[3] = {r.o.x, r.o.y, r.o.z};
  const float d[3] = {r.d.x, r.d.y, r.d.z};
  float t0 = 0.f, t1 = __int_as_float(0x7f800000);
  float dmax = 0.f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    dmax = fmaxf(dmax, fabsf(d[a]));
    if (d[a] != 0.f) {
      float ta = __fdiv_rn(__fsub_rn(s.root_lo[a], o[a]), d[a]);
      float tb = __fdiv_rn(__fsub_rn(s.root_hi[a], o[a]), d[a]);
      t0 = fmaxf(t0, fminf(ta, tb));
      t1 = fminf(t1, fmaxf(ta, tb));
    } else if (o[a] < s.root_lo[a] || o[a] > s.root_hi[a]) {
      return;
    }
  }
  if (!(dmax > 0.f) || !(t0 <= t1)) return;
  st.t_entry = t0;
  st.t_end = t1;
  st.slack = __fdiv_rn(s.scene_eps, dmax);
  st.node = 0;
}

// Node fetch with an optional shared-memory copy of the first n_smem nodes.
__device__ __forceinline__ uint2 fetch_node(const DevScene& s, const uint2* smem, int n_smem,
                                            int i) {
  if (i < n_smem) return smem[i];
  return __ldg(reinterpret_cast<const uint2*>(s.nodes) + i);
}

// Processes one leaf: descends from st.node to the leaf containing the
// entry point, tests its triangles, then follows the exit rope.
// Returns true when the ray is finished.
__device__ __forceinline__ bool trav_leaf(const DevScene& s, TravState& st, const uint2* smem,
                                          int n_smem, uint32_t* err, TravCount& cnt) {
  if (st.node < 0) return true;
  const Ray& r = st.ray;
  // Entry point p = o + t_entry * d (kernel.cl:291 style, no FMA).
  const float px = __fadd_rn(r.o.x, __fmul_rn(st.t_entry, r.d.x));
  const float py = __fadd_rn(r.o.y, __fmul_rn(st.t_entry, r.d.y));
  const float pz = __fadd_rn(r.o.z, __fmul_rn(st.t_entry, r.d.z));
  int node = st.node;
  uint2 nd = fetch_node(s, smem, n_smem, node);
  while ((nd.x >> 30) != kLeafKind) {
    const uint32_t axis = nd.x >> 30;
    const float split = __uint_as_float(nd.y);
    const float p = axis == 0 ? px : (axis == 1 ? py : pz);
    const float dd = axis == 0 ? r.d.x : (axis == 1 ? r.d.y : r.d.z);
    const bool right = p > split || (p == split && dd > 0.f);
    node = (int)(nd.x & kIndexMask) + (right ? 1 : 0);
    nd = fetch_node(s, smem, n_smem, node);
    ++cnt.nodes;
    if (++st.steps > s.max_steps) {
      atomicOr(err, 1u);
      st.node = -1;
      return true;
    }
  }
  const DevLeaf* L = s.leaves + (nd.x & kIndexMask);
  const float4 L0 = __ldg(reinterpret_cast<const float4*>(L));
  const float4 L1 = __ldg(reinterpret_cast<const float4*>(L) + 1);
  const float lo[3] = {L0.x, L0.y, L0.z};
  const float hi[3] = {L1.x, L1.y, L1.z};
  float t_exit;
  int face;
  const bool pierced = leaf_slabs(r, lo, hi, t_exit, face);
  const int begin = __float_as_int(L0.w), count = __float_as_int(L1.w);
  ++cnt.leaves;
  if (pierced && count > 0) {
    cnt.tris += (unsigned)count;
    const int32_t* ids = s.leaf_refs + begin;
    const float4* recs = reinterpret_cast<const float4*>(s.tris);
    for (int k = 0; k < count; ++k) {
      const float4* rec = recs + 3 * (size_t)__ldg(ids + k);
      const float4 A = __ldg(rec), E1 = __ldg(rec + 1), E2 = __ldg(rec + 2);
      float t, u, v;
      if (mt_test(r, A, E1, E2, t, u, v)) {
        const int j = begin + k;
        if (st.best.rec < 0 || t < st.best.t || (t == st.best.t && j < st.best.rec)) {
          st.best.rec = j;
          st.best.tri = __float_as_int(A.w);
          st.best.t = t;
          st.best.u = u;
          st.best.v = v;
        }
      }
    }
  }
  st.steps += 1 + count;
  // Stop once the rest of the ray starts beyond the best hit (+ slack).
  if (face < 0 || !(t_exit < st.t_end)) { st.node = -1; return true; }
  if (st.best.rec >= 0 &&
      t_exit > __fadd_rn(st.best.t, __fadd_rn(__fmul_rn(st.best.t, 1e-4f), st.slack))) {
    st.node = -1;
    return true;
  }
  const int rope = __ldg(reinterpret_cast<const int*>(L) + 8 + face);
  if (rope < 0 || st.steps > s.max_steps) {
    if (rope >= 0) atomicOr(err, 1u);
    st.node = -1;
    return true;
  }
  st.node = rope;
  st.t_entry = fmaxf(st.t_entry, t_exit);
  return false;
}

}  // namespace hpt
