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
// A ray lying exactly in a split plane is walked on both sides of it (see
// trav_finish). Not reproduced: the reference's 512-leaf gather cap
// (kernel.cl:133, 146; a ray whose line pierces more than 512 leaves may
// lose its true closest hit there, never here); exact ties where a ray
// passes exactly through a leaf's edge or corner (a vertex or edge hit may
// report another triangle meeting there, at the same t); a zero direction
// vector, which misses here (the reference reports t = +inf hits).
#pragma once

#include "checks.cuh"
#include "device_types.h"
#include "dmath.cuh"

namespace hpt {

struct Hit {
  int32_t rec;   // position in the leaf lists (reference rank), -1 = none
  int32_t tri;   // triangle id
  float t, u, v;
};

// _box_intersect (kernel.cl:56-83), exactly: origin-inside shortcut, then
// slabs (s - p0) / p with IEEE division, fmin/fmax, min_of_maxs <= 0 -> miss.
HPT_HD bool ref_box_test(const Ray& r, const float4 lo, const float4 hi) {
  const float o[3] = {r.o.x, r.o.y, r.o.z};
  const float d[3] = {r.d.x, r.d.y, r.d.z};
  const float l[3] = {lo.x, lo.y, lo.z};
  const float h[3] = {hi.x, hi.y, hi.z};
  bool inside = true;
  float max_of_mins = 0.f, min_of_maxs = 0.f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    inside = inside && o[a] >= l[a] && o[a] <= h[a];
    const float t0 = rn_div(rn_sub(l[a], o[a]), d[a]);
    const float t1 = rn_div(rn_sub(h[a], o[a]), d[a]);
    const float mn = fminf(t0, t1), mx = fmaxf(t0, t1);
    max_of_mins = a == 0 ? mn : fmaxf(max_of_mins, mn);
    min_of_maxs = a == 0 ? mx : fminf(min_of_maxs, mx);
  }
  if (inside) return true;
  if (min_of_maxs <= 0.f) return false;
  return max_of_mins <= min_of_maxs;
}

// _single_intersect (kernel.cl:85-109) on a pre-subtracted record. The
// epsilon test at kernel.cl:93 can never be true and is omitted.
HPT_HD bool mt_test(const Ray& r, const float4 A, const float4 E1,
                                        const float4 E2, float& t, float& u, float& v) {
  f3 a = mk(A.x, A.y, A.z), e1 = mk(E1.x, E1.y, E1.z), e2 = mk(E2.x, E2.y, E2.z);
  f3 P = cross(r.d, e2);
  float det = dot(e1, P);
  float inv_det = rn_div(1.f, det);
  f3 T = sub(r.o, a);
  u = rn_mul(dot(T, P), inv_det);
  if (u < 0.f || u > 1.f) return false;
  f3 Q = cross(T, e1);
  v = rn_mul(dot(r.d, Q), inv_det);
  if (v < 0.f || rn_add(u, v) > 1.f) return false;
  t = rn_mul(dot(e2, Q), inv_det);
  return t > 0.f;
}

// Entries of the per-ray triangle mailbox (a performance knob only: a
// repeated triangle that misses the mailbox is simply tested again).
#ifndef HPT_MAILBOX
#define HPT_MAILBOX 1
#endif
constexpr int kMailbox = HPT_MAILBOX;

// Phases of the step-at-a-time walk (trav_step).
constexpr int32_t kStepDescend = 0;
constexpr int32_t kStepTest = 1;

// Traversal state of one ray that most units touch; lives in registers so
// a lane can be refilled with a new ray between leaves.
struct TravState {
  Ray ray;
  float t_entry;         // current entry distance
  int32_t node;          // node to descend from, -1 = finished
  int32_t steps;
  Hit best;
  // The last kMailbox triangles tested and their Moller-Trumbore t (-1 =
  // miss): the reference tree repeats a triangle in every leaf it straddles.
  int32_t mb_id[kMailbox];
  float mb_t[kMailbox];
  // trav_step only: kStepDescend / kStepTest, and in a leaf the next
  // position in leaf_refs and the end of its list.
  int32_t phase;
  int32_t k, end;
};

// The rest of a ray's traversal state: written when the query starts or a
// leaf is set up, read at a leaf's exit or when a candidate would win -
// at most a few times per leaf. The kernels keep it in shared memory
// (eleven words per lane: an odd stride, free of bank conflicts) so that
// the registers go to the state every unit touches.
struct TravCold {
  f3 inv_d;           // 1 / d (exit distances only; the filter divides)
  float t_end;        // scene exit distance
  float slack;        // world-space rounding slack in t units
  int32_t best_node;  // leaf node where the best hit was found
  // trav_step's current leaf:
  int32_t leaf;       // leaf record
  int32_t leaf_node;  // its node index (reported as best_node)
  int32_t rope;       // node behind the exit face, -1 when there is none
  int32_t pierced;    // reference box test of the leaf: -1 not evaluated yet
  float t_exit;
  // Rays that lie exactly in a split plane (see trav_finish):
  float t_start;      // scene entry distance, where every walk starts
  int32_t ties;       // bits 0-2: axes with a zero direction component;
                      // 3-5: axes on which a descent met such a plane;
                      // 6-8: axes whose planes this walk passes on the right
};
static_assert(sizeof(TravCold) == 52, "odd word stride in shared memory");

// A ray with a zero direction component whose coordinate equals a node's
// split on that axis lies in the plane between the two children, and a
// single stackless walk can only take one side. In the reference a box
// with that plane as a face gives its slab test 0/0 = NaN and is rejected
// (_box_intersect, kernel.cl:56-83) unless its inside test holds, i.e. the
// box contains the ray's origin: so beyond the leaves that contain the
// origin, both sides of the plane are rejected alike, and only those leaves
// differ between the sides. The first walk takes the left side of every
// such plane and records the axes where it met one; if the origin lies in
// the scene, trav_finish then walks again from the origin once per
// remaining left/right combination of the zero axes (at most 3 more walks),
// each only through the leaves that contain the origin, keeping the best
// hit over all walks. Rays off every split plane walk once.
HPT_HD bool tie_goes_right(TravCold& tc, uint32_t axis) {
  tc.ties |= 8 << axis;
  return (tc.ties >> (6 + axis)) & 1;
}

// End of a walk: starts the next one if the ray lay in a split plane and a
// side combination is left (returns false, walk on), else finishes the ray.
HPT_HD bool trav_finish(TravState& st, TravCold& tc) {
  const int z = tc.ties & 7, seen = (tc.ties >> 3) & 7, cur = (tc.ties >> 6) & 7;
  const int next = ((cur | ~z) + 1) & z;  // next subset of z
  if (seen && next && tc.t_start == 0.f) {
    tc.ties = z | (seen << 3) | (next << 6);
    st.node = 0;
    st.t_entry = 0.f;
    st.phase = kStepDescend;
    // Only leaves that contain the origin count on this side: the walk
    // leaves at the first exit beyond t = 0.
    tc.t_end = as_float(1);
    return false;
  }
  st.node = -1;
  return true;
}

// Work counters of one lane over one kernel launch (summed per warp in 64
// bits when the launch ends; they feed statistics only).
// (Plain data: declare with `TravCount cnt{}` to start from zero.)
struct TravCount {
  uint32_t nodes, leaves, tris, repeats;
};

// The work counters of a run of traversal units in one register: four
// 8-bit fields (nodes, leaves, triangle tests, mailbox repeats), added into
// a TravCount by count_flush before any field can pass 255.
struct PackedCount {
  uint32_t v;
};
HPT_HD void count_node(TravCount& c) { ++c.nodes; }
HPT_HD void count_leaf(TravCount& c) { ++c.leaves; }
HPT_HD void count_test(TravCount& c) { ++c.tris; }
HPT_HD void count_repeat(TravCount& c) { ++c.repeats; }
HPT_HD void count_node(PackedCount& c) { c.v += 1u; }
HPT_HD void count_leaf(PackedCount& c) { c.v += 1u << 8; }
HPT_HD void count_test(PackedCount& c) { c.v += 1u << 16; }
HPT_HD void count_repeat(PackedCount& c) { c.v += 1u << 24; }
HPT_HD void count_flush(PackedCount& p, TravCount& c) {
  c.nodes += p.v & 255u;
  c.leaves += (p.v >> 8) & 255u;
  c.tris += (p.v >> 16) & 255u;
  c.repeats += p.v >> 24;
  p.v = 0;
}

// Starts a query. start_node (>= 0) names a leaf node the origin is
// expected to lie in (the leaf of the previous hit): if its box contains the
// origin the walk starts there instead of descending from the root.
template <class Sc>
HPT_HD void trav_init(const Sc& s, const Ray& r, TravState& st, TravCold& tc,
                      int start_node = -1) {
  st.ray = r;
  st.best.rec = -1;
  st.best.tri = -1;
  st.best.t = 0.f;
  st.best.u = st.best.v = 0.f;
  tc.best_node = -1;
  tc.leaf = tc.leaf_node = 0;
  tc.rope = -1;
  tc.pierced = -1;
  tc.t_exit = 0.f;
  tc.t_start = 0.f;
  tc.ties = 0;
  st.steps = 0;
  st.node = -1;
  st.phase = kStepDescend;
  st.k = st.end = 0;
#pragma unroll
  for (int k = 0; k < kMailbox; ++k) {
    st.mb_id[k] = -1;
    st.mb_t[k] = -1.f;
  }
  if (!finite3(r.o) || !finite3(r.d)) return;
  const float o[3] = {r.o.x, r.o.y, r.o.z};
  const float d[3] = {r.d.x, r.d.y, r.d.z};
  float t0 = 0.f, t1 = as_float(0x7f800000);
  float dmax = 0.f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    dmax = fmaxf(dmax, fabsf(d[a]));
    if (d[a] != 0.f) {
      float ta = rn_div(rn_sub(s.root_lo[a], o[a]), d[a]);
      float tb = rn_div(rn_sub(s.root_hi[a], o[a]), d[a]);
      t0 = fmaxf(t0, fminf(ta, tb));
      t1 = fminf(t1, fmaxf(ta, tb));
    } else if (o[a] < s.root_lo[a] || o[a] > s.root_hi[a]) {
      return;
    }
  }
  if (!(dmax > 0.f) || !(t0 <= t1)) return;
  tc.inv_d = mk(rn_rcp(r.d.x), rn_rcp(r.d.y), rn_rcp(r.d.z));
  st.t_entry = t0;
  tc.t_end = t1;
  tc.slack = rn_div(s.scene_eps, dmax);
  tc.t_start = t0;
  tc.ties = (d[0] == 0.f ? 1 : 0) | (d[1] == 0.f ? 2 : 0) | (d[2] == 0.f ? 4 : 0);
  st.node = 0;
  if (start_node > 0 && start_node < s.num_nodes) {
    const uint2 nd = ldg(reinterpret_cast<const uint2*>(s.nodes) + start_node);
    if ((nd.x >> 30) == kLeafKind) {
      const float4* L = reinterpret_cast<const float4*>(s.leaves + (nd.x & kIndexMask));
      const float4 lo = ldg(L), hi = ldg(L + 1);
      // A hinted start skips the descents from the root, and with them any
      // split plane the ray lies in; such a plane bounds the leaf, so along a
      // zero direction component the origin must lie strictly inside.
      const int z = tc.ties;
      const bool off_planes = (!(z & 1) || (o[0] > lo.x && o[0] < hi.x)) &&
                              (!(z & 2) || (o[1] > lo.y && o[1] < hi.y)) &&
                              (!(z & 4) || (o[2] > lo.z && o[2] < hi.z));
      if (o[0] >= lo.x && o[0] <= hi.x && o[1] >= lo.y && o[1] <= hi.y && o[2] >= lo.z &&
          o[2] <= hi.z && off_planes) {
        st.node = start_node;
        st.t_entry = 0.f;
      }
    }
  }
}

// The traversal's view of a scene (the fields trav_* read).
HPT_HD TravScene trav_scene(const DevScene& s) {
  TravScene t;
  t.nodes = s.nodes;
  t.leaves = s.leaves;
  t.leaf_refs = s.leaf_refs;
  t.tris = s.tris;
  t.num_nodes = s.num_nodes;
  t.num_leaves = s.num_leaves;
  t.num_leaf_tris = s.num_leaf_tris;
  t.num_triangles = s.num_triangles;
  for (int a = 0; a < 3; ++a) {
    t.root_lo[a] = s.root_lo[a];
    t.root_hi[a] = s.root_hi[a];
  }
  t.scene_eps = s.scene_eps;
  t.max_steps = s.max_steps;
  return t;
}

// Node fetch with an optional shared-memory copy of the first n_smem nodes.
template <class Sc>
HPT_HD uint2 fetch_node(const Sc& s, const uint2* smem, int n_smem,
                                            int i) {
  if (i < n_smem) return smem[i];
  return ldg(reinterpret_cast<const uint2*>(s.nodes) + i);
}

// A node that ends the walk (used when a self-check rejects an index).
constexpr uint32_t kDeadLeafMeta = 0xFFFFFFFFu;

// Processes one leaf: descends from st.node to the leaf containing the
// entry point, tests its triangles, then follows the exit rope.
// Returns true when the ray is finished.
// kUV: also report the winning test's Moller-Trumbore u, v (stage entry).
template <bool kUV = false, class Sc = DevScene>
HPT_HD bool trav_leaf(const Sc& s, TravState& st, TravCold& tc, const uint2* smem,
                      int n_smem, DevErr* err, TravCount& cnt) {
  if (st.node < 0) return true;
  HPT_DCHECK(err, st.node < s.num_nodes, 101, st.node, { st.node = -1; return true; });
  const Ray& r = st.ray;
  // Entry point p = o + t_entry * d (kernel.cl:291 style, no FMA).
  const float px = rn_add(r.o.x, rn_mul(st.t_entry, r.d.x));
  const float py = rn_add(r.o.y, rn_mul(st.t_entry, r.d.y));
  const float pz = rn_add(r.o.z, rn_mul(st.t_entry, r.d.z));
  int node = st.node;
  uint2 nd = fetch_node(s, smem, n_smem, node);
  while ((nd.x >> 30) != kLeafKind) {
    const uint32_t axis = nd.x >> 30;
    const float split = as_float_u(nd.y);
    const float p = axis == 0 ? px : (axis == 1 ? py : pz);
    const float dd = axis == 0 ? r.d.x : (axis == 1 ? r.d.y : r.d.z);
    const bool right =
        p > split || (p == split && (dd > 0.f || (dd == 0.f && tie_goes_right(tc, axis))));
    HPT_DCHECK(err, (int)(nd.x & kIndexMask) + 1 < s.num_nodes, 106, nd.x & kIndexMask,
               { st.node = -1; return true; });
    node = (int)(nd.x & kIndexMask) + (right ? 1 : 0);
    nd = fetch_node(s, smem, n_smem, node);
    ++cnt.nodes;
    if (++st.steps > s.max_steps) {
      hpt_atomic_or(&err->flags, 1u);
      st.node = -1;
      return true;
    }
  }
  HPT_DCHECK(err, (int)(nd.x & kIndexMask) < s.num_leaves, 102, nd.x & kIndexMask,
             { st.node = -1; return true; });
  const DevLeaf* L = s.leaves + (nd.x & kIndexMask);
  const float4 L0 = ldg(reinterpret_cast<const float4*>(L));
  const float4 L1 = ldg(reinterpret_cast<const float4*>(L) + 1);
  // Exit distance and face (reciprocal multiplies; only the reference's box
  // filter below needs the division form).
  float t_exit = as_float(0x7f800000);
  int face = -1;
  {
    const float d[3] = {r.d.x, r.d.y, r.d.z};
    const float o[3] = {r.o.x, r.o.y, r.o.z};
    const float iv[3] = {tc.inv_d.x, tc.inv_d.y, tc.inv_d.z};
    const float lo[3] = {L0.x, L0.y, L0.z};
    const float hi[3] = {L1.x, L1.y, L1.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (d[a] != 0.f) {
        const float tf = rn_mul(rn_sub(d[a] > 0.f ? hi[a] : lo[a], o[a]), iv[a]);
        if (tf < t_exit) {
          t_exit = tf;
          face = 2 * a + (d[a] > 0.f ? 1 : 0);
        }
      }
    }
  }
  const int begin = as_int(L0.w), count = as_int(L1.w);
  ++cnt.leaves;
  HPT_DCHECK(err, begin >= 0 && count >= 0 && (long long)begin + count <= s.num_leaf_tris, 103,
             begin, { st.node = -1; return true; });
  if (count > 0) {
    // The reference only considers triangles of leaves whose box passes
    // _box_intersect; evaluated once, when a candidate would win.
    int pierced = -1;
    const int32_t* ids = s.leaf_refs + begin;
    const float4* recs = reinterpret_cast<const float4*>(s.tris);
    for (int k = 0; k < count; ++k) {
      const int id = ldg(ids + k);
      const int j = begin + k;
      HPT_DCHECK(err, id >= 0 && id < s.num_triangles, 104, id, continue);
      float t = -1.f, u = 0.f, v = 0.f;
      bool tested = false;
      int slot = -1;
#pragma unroll
      for (int m = 0; m < kMailbox; ++m)
        if (st.mb_id[m] == id) slot = m;
      if (slot >= 0) {
        ++cnt.repeats;
#pragma unroll
        for (int m = 0; m < kMailbox; ++m)
          if (m == slot) t = st.mb_t[m];
      } else {
        ++cnt.tris;
        const float4* rec = recs + 3 * (size_t)id;
        const float4 A = ldg(rec), E1 = ldg(rec + 1), E2 = ldg(rec + 2);
        if (!mt_test(r, A, E1, E2, t, u, v)) t = -1.f;
        tested = true;
#pragma unroll
        for (int m = kMailbox - 1; m > 0; --m) {
          st.mb_id[m] = st.mb_id[m - 1];
          st.mb_t[m] = st.mb_t[m - 1];
        }
        st.mb_id[0] = id;
        st.mb_t[0] = t;
      }
      if (t > 0.f &&
          (st.best.rec < 0 || t < st.best.t || (t == st.best.t && j < st.best.rec))) {
        if (pierced < 0) pierced = ref_box_test(r, L0, L1) ? 1 : 0;
        if (pierced) {
          if (kUV && !tested) {  // a repeat that now wins: recover its u, v
            const float4* rec = recs + 3 * (size_t)id;
            float t2;
            mt_test(r, ldg(rec), ldg(rec + 1), ldg(rec + 2), t2, u, v);
          }
          st.best.rec = j;
          st.best.tri = id;
          st.best.t = t;
          if (kUV) {
            st.best.u = u;
            st.best.v = v;
          }
          tc.best_node = node;
        }
      }
    }
  }
  st.steps += 1 + count;
  // Stop once the rest of the ray starts beyond the best hit (+ slack).
  const int rope = face < 0 ? -1 : ldg(reinterpret_cast<const int*>(L) + 8 + face);
  if (!(t_exit < tc.t_end) || rope < 0 ||
      (st.best.rec >= 0 &&
       t_exit > rn_add(st.best.t, rn_add(rn_mul(st.best.t, 1e-4f), tc.slack))))
    return trav_finish(st, tc);
  if (st.steps > s.max_steps) {
    hpt_atomic_or(&err->flags, 1u);
    st.node = -1;
    return true;
  }
  HPT_DCHECK(err, rope < s.num_nodes, 105, rope, { st.node = -1; return true; });
  st.node = rope;
  st.t_entry = fmaxf(st.t_entry, t_exit);
  return false;
}

// Leaf exit of the step-at-a-time walk, once every triangle of the current
// leaf was tested: stop once the rest of the ray starts beyond the best hit
// (+ slack), else follow the exit rope. A leaf without an exit face has
// t_exit = +inf and stops here. Returns true when the ray is finished.
template <class Sc>
HPT_HD bool trav_exit(const Sc& s, TravState& st, TravCold& tc, DevErr* err) {
  st.phase = kStepDescend;
  const int rope = tc.rope;
  if (!(tc.t_exit < tc.t_end) || rope < 0 ||
      (st.best.rec >= 0 &&
       tc.t_exit > rn_add(st.best.t, rn_add(rn_mul(st.best.t, 1e-4f), tc.slack))))
    return trav_finish(st, tc);
  if (st.steps > s.max_steps) {
    hpt_atomic_or(&err->flags, 1u);
    st.node = -1;
    return true;
  }
  HPT_DCHECK(err, rope < s.num_nodes, 105, rope, { st.node = -1; return true; });
  st.node = rope;
  st.t_entry = fmaxf(st.t_entry, tc.t_exit);
  return false;
}

// Leaf set-up of the step-at-a-time walk for the leaf record st.k, reached
// at node st.node: exit distance and face, triangle range; the walk then
// tests the leaf's triangles (phase kStepTest). Returns true when the ray is
// finished (a failed self-check).
template <class Sc, class Cnt>
HPT_HD bool trav_setup(const Sc& s, TravState& st, TravCold& tc, DevErr* err, Cnt& cnt) {
  const Ray& r = st.ray;
  const int leaf = st.k;
  const float4* L = reinterpret_cast<const float4*>(s.leaves + leaf);
  // The six ropes are read with the box (independent loads) so that the
  // exit needs no dependent load of its own.
  const float4 L0 = ldg(L), L1 = ldg(L + 1);
  const int4 R03 = ldg(reinterpret_cast<const int4*>(L + 2));
  const int2 R45 = ldg(reinterpret_cast<const int2*>(L + 3));
  float t_exit = as_float(0x7f800000);
  int face = -1;
  {
    const float d[3] = {r.d.x, r.d.y, r.d.z};
    const float o[3] = {r.o.x, r.o.y, r.o.z};
    const float iv[3] = {tc.inv_d.x, tc.inv_d.y, tc.inv_d.z};
    const float lo[3] = {L0.x, L0.y, L0.z};
    const float hi[3] = {L1.x, L1.y, L1.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (d[a] != 0.f) {
        const float tf = rn_mul(rn_sub(d[a] > 0.f ? hi[a] : lo[a], o[a]), iv[a]);
        if (tf < t_exit) {
          t_exit = tf;
          face = 2 * a + (d[a] > 0.f ? 1 : 0);
        }
      }
    }
  }
  const int begin = as_int(L0.w), count = as_int(L1.w);
  count_leaf(cnt);
  HPT_DCHECK(err, begin >= 0 && count >= 0 && (long long)begin + count <= s.num_leaf_tris, 103,
             begin, { st.node = -1; return true; });
  // trav_leaf adds the leaf's cost when it leaves it; every comparison with
  // max_steps comes later in both orders, so adding it here is equivalent.
  st.steps += 1 + count;
  st.k = begin;
  st.end = begin + count;
  tc.leaf = leaf;
  tc.leaf_node = st.node;
  tc.rope = face == 0 ? R03.x : face == 1 ? R03.y : face == 2 ? R03.z
          : face == 3 ? R03.w : face == 4 ? R45.x : face == 5 ? R45.y : -1;
  tc.t_exit = t_exit;
  tc.pierced = -1;
  st.phase = kStepTest;
  return false;
}

// --- Step-at-a-time traversal ----------------------------------------------
// The same walk as trav_leaf, cut into units of similar cost: one descent
// step, the set-up of a newly reached leaf, one triangle test, or the exit
// of a finished leaf through its rope. A warp that calls trav_step in a loop
// lets every lane move on to its next leaf as soon as its own leaf is done,
// instead of waiting for the lane with the deepest descent and then for the
// one with the longest triangle list; results are identical to trav_leaf's
// (same tests in the same order, same termination).
// A call runs one unit, except that a leaf's last triangle test falls
// through to the leaf's exit in the same call: the exit needs no load of
// its own (the ropes are read at set-up), so this saves a call per leaf for
// a few instructions. Falling through from set-up to the first test as
// well measured slower (the set-up's loads and the test's loads then
// chain within one call).

// Returns true when the ray is finished.
// kSmem: nodes below n_smem are read from the shared-memory prefix (false:
// every node from global memory, and smem / n_smem are ignored).
// kTests = false: the caller only calls it in the descent phase (its
// triangle tests run elsewhere), so the test unit is left out.
template <bool kUV = false, bool kSmem = true, class Sc = DevScene, bool kTests = true,
          class Cnt = TravCount>
HPT_HD bool trav_step(const Sc& s, TravState& st, TravCold& tc, const uint2* smem,
                      int n_smem, DevErr* err, Cnt& cnt) {
  if (st.node < 0) return true;
  const Ray& r = st.ray;
  if (st.phase == kStepDescend) {
    // st.node is in range: every value it takes is checked where it is made
    // (the root, a hint in trav_init, a child at check 106, a rope at check
    // 105, the root again in trav_finish).
    const uint2 nd = fetch_node(s, smem, kSmem ? n_smem : 0, st.node);
    if ((nd.x >> 30) != kLeafKind) {
      // One descent step; the entry point p = o + t_entry * d on the split
      // axis (kernel.cl:291 style, no FMA), as trav_leaf computes it.
      const uint32_t axis = nd.x >> 30;
      const float split = as_float_u(nd.y);
      const float o = axis == 0 ? r.o.x : (axis == 1 ? r.o.y : r.o.z);
      const float dd = axis == 0 ? r.d.x : (axis == 1 ? r.d.y : r.d.z);
      const float p = rn_add(o, rn_mul(st.t_entry, dd));
      const bool right =
        p > split || (p == split && (dd > 0.f || (dd == 0.f && tie_goes_right(tc, axis))));
      HPT_DCHECK(err, (int)(nd.x & kIndexMask) + 1 < s.num_nodes, 106, nd.x & kIndexMask,
                 { st.node = -1; return true; });
      st.node = (int)(nd.x & kIndexMask) + (right ? 1 : 0);
      count_node(cnt);
      if (++st.steps > s.max_steps) {
        hpt_atomic_or(&err->flags, 1u);
        st.node = -1;
        return true;
      }
      return false;
    }
    HPT_DCHECK(err, (int)(nd.x & kIndexMask) < s.num_leaves, 102, nd.x & kIndexMask,
               { st.node = -1; return true; });
    st.k = (int)(nd.x & kIndexMask);
    return trav_setup(s, st, tc, err, cnt);
  }
  if constexpr (!kTests) return false;
  if (st.k < st.end) {
    // One triangle test (the body of trav_leaf's triangle loop).
    const int j = st.k++;
    const int id = ldg(s.leaf_refs + j);
    HPT_DCHECK(err, id >= 0 && id < s.num_triangles, 104, id, return false);
    const float4* recs = reinterpret_cast<const float4*>(s.tris);
    float t = -1.f, u = 0.f, v = 0.f;
    bool tested = false;
    int slot = -1;
#pragma unroll
    for (int m = 0; m < kMailbox; ++m)
      if (st.mb_id[m] == id) slot = m;
    if (slot >= 0) {
      count_repeat(cnt);
#pragma unroll
      for (int m = 0; m < kMailbox; ++m)
        if (m == slot) t = st.mb_t[m];
    } else {
      count_test(cnt);
      const float4* rec = recs + 3 * (size_t)id;
      const float4 A = ldg(rec), E1 = ldg(rec + 1), E2 = ldg(rec + 2);
      if (!mt_test(r, A, E1, E2, t, u, v)) t = -1.f;
      tested = true;
#pragma unroll
      for (int m = kMailbox - 1; m > 0; --m) {
        st.mb_id[m] = st.mb_id[m - 1];
        st.mb_t[m] = st.mb_t[m - 1];
      }
      st.mb_id[0] = id;
      st.mb_t[0] = t;
    }
    if (t > 0.f && (st.best.rec < 0 || t < st.best.t || (t == st.best.t && j < st.best.rec))) {
      if (tc.pierced < 0) {
        const float4* L = reinterpret_cast<const float4*>(s.leaves + tc.leaf);
        tc.pierced = ref_box_test(r, ldg(L), ldg(L + 1)) ? 1 : 0;
      }
      if (tc.pierced) {
        if (kUV && !tested) {  // a repeat that now wins: recover its u, v
          const float4* rec = recs + 3 * (size_t)id;
          float t2;
          mt_test(r, ldg(rec), ldg(rec + 1), ldg(rec + 2), t2, u, v);
        }
        st.best.rec = j;
        st.best.tri = id;
        st.best.t = t;
        if (kUV) {
          st.best.u = u;
          st.best.v = v;
        }
        tc.best_node = tc.leaf_node;
      }
    }
    if (st.k < st.end) return false;
    // The leaf's last test falls through to its exit.
  }
  return trav_exit(s, st, tc, err);
}

}  // namespace hpt
