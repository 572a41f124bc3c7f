// Repacks the reference's flattened KD-tree (48-byte KDTreeNodeHeader
// array + [count, ids...] leaf list, src/hp/scene/kdtree.cpp:248-292) into
// the traversal layout of the CUDA kernels:
//
//  * 8-byte nodes (axis + child index, split position) whose children are
//    stored side by side; the top levels are laid out breadth-first so a
//    kernel can stage a prefix of the array in shared memory, the rest is
//    depth-first by sibling pairs.
//  * Every reference node box is nested in its parent's box. Where
//    removeEmptyNode (kdtree.cpp:171-206) shrank a box, the missing slab is
//    re-inserted as a split with an empty leaf, so each cell of the new tree
//    is exactly the reference box of the node it stands for.
//  * Leaf records with the reference box (used both for the exit distance
//    and, unchanged, for the reference's _box_intersect filter) and six
//    ropes (Popov et al., "Stackless KD-Tree Traversal for High Performance
//    GPU Ray Tracing", 2007) pointing to the smallest node that covers the
//    neighbouring face.
//  * Leaf triangle lists concatenated in the order the reference gathers
//    leaves (pre-order of its node array), so a list position is the rank of
//    that test in the reference's first-hit-wins tie rule (kernel.cl:180),
//    and one record (a, b - a, c - a) per triangle.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>
#include <string>

#include "device_types.h"
#include "host.h"
#include "scene_pack.h"

namespace hpt {

namespace {

struct TmpNode {
  int axis = -1;  // -1 = leaf
  float split = 0;
  int left = -1, right = -1;
  int leaf = -1;
};

struct Packer {
  const hpt_ref_node* ref;
  int num_ref;
  const int32_t* leaf_data;
  const I4* tris;
  const F4* points;
  std::vector<TmpNode> nodes;
  std::vector<DevLeaf> leaves;
  std::vector<int32_t> refs;
  std::string err;
  int max_depth = 0;

  int new_leaf(const float lo[3], const float hi[3], int ref_node, int ref_data) {
    DevLeaf L;
    memset(&L, 0, sizeof L);
    for (int a = 0; a < 3; ++a) {
      L.lo[a] = lo[a];
      L.hi[a] = hi[a];
    }
    for (int f = 0; f < 6; ++f) L.rope[f] = -1;
    L.ref_node = ref_node;
    L.tri_begin = (int32_t)refs.size();
    L.tri_count = 0;
    if (ref_data >= 0) {
      int cnt = leaf_data[ref_data];
      for (int k = 0; k < cnt; ++k) refs.push_back(leaf_data[ref_data + 1 + k]);
      L.tri_count = cnt;
    }
    leaves.push_back(L);
    TmpNode n;
    n.leaf = (int)leaves.size() - 1;
    nodes.push_back(n);
    return (int)nodes.size() - 1;
  }

  int new_inner(int axis, float split) {
    TmpNode n;
    n.axis = axis;
    n.split = split;
    nodes.push_back(n);
    return (int)nodes.size() - 1;
  }

  // Emits reference node i into the cell [lo, hi].
  int emit(int i, const float lo_in[3], const float hi_in[3], int depth) {
    if (!err.empty()) return -1;
    if (depth > 4096) {
      err = "tree deeper than 4096 levels";
      return -1;
    }
    max_depth = std::max(max_depth, depth);
    float lo[3], hi[3];
    memcpy(lo, lo_in, sizeof lo);
    memcpy(hi, hi_in, sizeof hi);
    const hpt_ref_node& n = ref[i];
    for (int a = 0; a < 3; ++a) {
      if (n.box_start[a] < lo[a] || n.box_end[a] > hi[a]) {
        err = "node " + std::to_string(i) + " box is not inside its parent box";
        return -1;
      }
    }
    // Clip the cell down to the node's box, one face at a time.
    for (int a = 0; a < 3; ++a) {
      if (n.box_start[a] > lo[a]) {
        int id = new_inner(a, n.box_start[a]);
        float elo[3], ehi[3];
        memcpy(elo, lo, sizeof elo);
        memcpy(ehi, hi, sizeof ehi);
        ehi[a] = n.box_start[a];
        int e = new_leaf(elo, ehi, -1, -1);
        lo[a] = n.box_start[a];
        int r = emit(i, lo, hi, depth + 1);
        nodes[id].left = e;
        nodes[id].right = r;
        return id;
      }
      if (n.box_end[a] < hi[a]) {
        int id = new_inner(a, n.box_end[a]);
        float elo[3], ehi[3];
        memcpy(elo, lo, sizeof elo);
        memcpy(ehi, hi, sizeof ehi);
        elo[a] = n.box_end[a];
        hi[a] = n.box_end[a];
        int l = emit(i, lo, hi, depth + 1);
        int e = new_leaf(elo, ehi, -1, -1);
        nodes[id].left = l;
        nodes[id].right = e;
        return id;
      }
    }
    if (n.child < 0) return new_leaf(lo, hi, i, n.data);
    int L = n.child, R = ref[L].sibling;
    // Split axis: the one on which the left child ends where the right
    // child begins (a gap left by removeEmptyNode is clipped inside R).
    int axis = -1;
    for (int a = 0; a < 3 && axis < 0; ++a)
      if (ref[L].box_end[a] == ref[R].box_start[a]) axis = a;
    for (int a = 0; a < 3 && axis < 0; ++a)
      if (ref[L].box_end[a] < ref[R].box_start[a]) axis = a;
    if (axis < 0) {
      err = "children of node " + std::to_string(i) + " overlap on every axis";
      return -1;
    }
    float s = ref[L].box_end[axis];
    int id = new_inner(axis, s);
    float llo[3], lhi[3], rlo[3], rhi[3];
    memcpy(llo, lo, sizeof llo); memcpy(lhi, hi, sizeof lhi);
    memcpy(rlo, lo, sizeof rlo); memcpy(rhi, hi, sizeof rhi);
    lhi[axis] = s;
    rlo[axis] = s;
    int l = emit(L, llo, lhi, depth + 1);
    int r = emit(R, rlo, rhi, depth + 1);
    nodes[id].left = l;
    nodes[id].right = r;
    return id;
  }

  // Pushes a rope down to the smallest node covering the face (Popov 2007).
  int optimize(int r, int face, const float lo[3], const float hi[3]) const {
    int fa = face >> 1, side = face & 1;
    while (r >= 0 && nodes[r].axis >= 0) {
      const TmpNode& n = nodes[r];
      if (n.axis == fa) {
        r = side == 0 ? n.right : n.left;
      } else if (n.split <= lo[n.axis]) {
        r = n.right;
      } else if (n.split >= hi[n.axis]) {
        r = n.left;
      } else {
        break;
      }
    }
    return r;
  }

  void ropes(int root, const float rlo[3], const float rhi[3]) {
    struct Item {
      int node;
      int rope[6];
      float lo[3], hi[3];
    };
    std::vector<Item> stack;
    Item it;
    it.node = root;
    for (int f = 0; f < 6; ++f) it.rope[f] = -1;
    memcpy(it.lo, rlo, sizeof it.lo);
    memcpy(it.hi, rhi, sizeof it.hi);
    stack.push_back(it);
    while (!stack.empty()) {
      Item c = stack.back();
      stack.pop_back();
      const TmpNode& n = nodes[c.node];
      if (n.axis < 0) {
        DevLeaf& L = leaves[n.leaf];
        for (int f = 0; f < 6; ++f) L.rope[f] = c.rope[f];
        continue;
      }
      for (int f = 0; f < 6; ++f) c.rope[f] = optimize(c.rope[f], f, c.lo, c.hi);
      Item l = c, r = c;
      l.node = n.left;
      r.node = n.right;
      l.rope[2 * n.axis + 1] = n.right;
      r.rope[2 * n.axis] = n.left;
      l.hi[n.axis] = n.split;
      r.lo[n.axis] = n.split;
      stack.push_back(r);
      stack.push_back(l);
    }
  }
};

}  // namespace

hpt_status pack_scene(const hpt_scene_desc& d, int bfs_nodes, PackedScene& out) {
  std::string verr = validate_ref_tree(d.nodes, d.num_nodes, d.leaf_data,
                                       d.num_leaf_data, d.num_triangles);
  if (!verr.empty()) return fail(HPT_ERR_INVALID_SCENE, "kd-tree: %s", verr.c_str());
  Packer p;
  p.ref = d.nodes;
  p.num_ref = d.num_nodes;
  p.leaf_data = d.leaf_data;
  p.tris = reinterpret_cast<const I4*>(d.triangles);
  p.points = reinterpret_cast<const F4*>(d.points);
  p.nodes.reserve((size_t)d.num_nodes * 5 / 4 + 16);
  const hpt_ref_node& r0 = d.nodes[0];
  float lo[3] = {r0.box_start[0], r0.box_start[1], r0.box_start[2]};
  float hi[3] = {r0.box_end[0], r0.box_end[1], r0.box_end[2]};
  int root = p.emit(0, lo, hi, 0);
  if (!p.err.empty()) return fail(HPT_ERR_INVALID_SCENE, "kd-tree: %s", p.err.c_str());
  p.ropes(root, lo, hi);

  // Final layout: breadth-first for the first bfs_nodes slots, then
  // depth-first by sibling pairs.
  size_t nn = p.nodes.size();
  if (nn >= (size_t)kIndexMask || p.leaves.size() >= (size_t)kIndexMask)
    return fail(HPT_ERR_INVALID_SCENE, "tree too large for 30-bit node indices");
  std::vector<int32_t> idx(nn, -1);
  idx[root] = 0;
  int next = 1;
  std::deque<int> q{root};
  while (!q.empty() && next < bfs_nodes) {
    int n = q.front();
    q.pop_front();
    const TmpNode& t = p.nodes[n];
    if (t.axis < 0) continue;
    idx[t.left] = next;
    idx[t.right] = next + 1;
    next += 2;
    q.push_back(t.left);
    q.push_back(t.right);
  }
  std::vector<int> stack;
  for (int n : q) stack.push_back(n);
  std::reverse(stack.begin(), stack.end());
  while (!stack.empty()) {
    int n = stack.back();
    stack.pop_back();
    const TmpNode& t = p.nodes[n];
    if (t.axis < 0) continue;
    idx[t.left] = next;
    idx[t.right] = next + 1;
    next += 2;
    stack.push_back(t.right);
    stack.push_back(t.left);
  }
  out.nodes.assign(nn, DevNode{0, 0.f});
  for (size_t n = 0; n < nn; ++n) {
    const TmpNode& t = p.nodes[n];
    DevNode& o = out.nodes[idx[n]];
    if (t.axis < 0) {
      o.meta = (kLeafKind << 30) | (uint32_t)t.leaf;
      o.split = 0.f;
    } else {
      o.meta = ((uint32_t)t.axis << 30) | (uint32_t)idx[t.left];
      o.split = t.split;
    }
  }
  for (DevLeaf& L : p.leaves)
    for (int f = 0; f < 6; ++f)
      if (L.rope[f] >= 0) L.rope[f] = idx[L.rope[f]];
  out.leaves = std::move(p.leaves);
  out.refs = std::move(p.refs);
  out.tris.resize(d.num_triangles);
  for (int id = 0; id < d.num_triangles; ++id) {
    const I4& t = p.tris[id];
    const F4 &pa = p.points[t.x], &pb = p.points[t.y], &pc = p.points[t.z];
    DevTri& r = out.tris[id];
    r.a[0] = pa.x; r.a[1] = pa.y; r.a[2] = pa.z;
    // kernel.cl:89-90: e1 = pb - pa, e2 = pc - pa, in FP32.
    r.e1[0] = pb.x - pa.x; r.e1[1] = pb.y - pa.y; r.e1[2] = pb.z - pa.z;
    r.e2[0] = pc.x - pa.x; r.e2[1] = pc.y - pa.y; r.e2[2] = pc.z - pa.z;
    r.tri_id = id;
    r.material = t.w;
    r.pad = 0;
  }
  for (int a = 0; a < 3; ++a) {
    out.root_lo[a] = lo[a];
    out.root_hi[a] = hi[a];
  }
  out.max_depth = p.max_depth;
  return HPT_OK;
}

}  // namespace hpt
