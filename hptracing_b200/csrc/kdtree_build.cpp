// SAH KD-tree builder and flattener with the exact output of the
// reference's hp::KDTree (src/hp/scene/kdtree.cpp):
//  - per node, per dimension, sorted triangle min/max values (:23-34);
//  - root box = value range +- 1e-3 (:36-41); children inherit the parent
//    box cut at the split, boxes are never tightened (:129-135);
//  - 1-D "length" SAH with C_t = 1, C_i = 3 over the sorted candidate
//    values strictly inside the box (:47-89), first minimum over x, y, z;
//  - leaves below 5 triangles, no depth limit (:91-99);
//  - a triangle goes left unless all its vertices are > split and right
//    unless all are < split (:145-154);
//  - removeEmptyNode folds an empty leaf child into its parent (:171-206);
//  - getData: pre-order nodes, leaf list [count, ids...], sibling on left
//    children only (:248-292).
// Differences that do not change the output: the candidate list is a merge
// of the two sorted arrays instead of a re-sort, min/max arrays are freed
// after a node is split, and large subtrees are built on worker threads.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <functional>
#include <memory>
#include <string>
#include <thread>
#include <unordered_map>

#include "host.h"

namespace hpt {

namespace {

struct Node {
  std::unique_ptr<Node> left, right;
  Node* parent = nullptr;
  float box_start[3], box_end[3];
  std::vector<int32_t> geo;
};

struct Builder {
  const F4* points;
  const I4* tris;
  std::atomic<int> threads_left{0};

  float coord(int vertex, int d) const {
    const F4& p = points[vertex];
    return d == 0 ? p.x : d == 1 ? p.y : p.z;
  }

  void min_max(const std::vector<int32_t>& geo, int d, std::vector<float>& mins,
               std::vector<float>& maxs) const {
    mins.resize(geo.size());
    maxs.resize(geo.size());
    for (size_t i = 0; i < geo.size(); ++i) {
      const I4& t = tris[geo[i]];
      float v[3] = {coord(t.x, d), coord(t.y, d), coord(t.z, d)};
      mins[i] = *std::min_element(v, v + 3);
      maxs[i] = *std::max_element(v, v + 3);
    }
    std::sort(mins.begin(), mins.end());
    std::sort(maxs.begin(), maxs.end());
  }

  // kdtree.cpp:47-89
  static void best_split(const std::vector<float>& mins,
                         const std::vector<float>& maxs, float box_start,
                         float box_end, float& best_pos, float& best_cost) {
    std::vector<float> all(mins.size() + maxs.size());
    // +0.0 and -0.0 compare equal, so their order in the sorted candidate
    // list (and with it the bits of a chosen split at zero) is whatever the
    // reference's std::sort of the concatenation produces. Sort the same way
    // when both zeros occur; otherwise all equal values are bit-identical and
    // a merge gives the same list.
    bool pos_zero = false, neg_zero = false;
    for (const std::vector<float>* v : {&mins, &maxs})
      for (float x : *v)
        if (x == 0.f) (std::signbit(x) ? neg_zero : pos_zero) = true;
    if (pos_zero && neg_zero) {
      std::copy(mins.begin(), mins.end(), all.begin());
      std::copy(maxs.begin(), maxs.end(), all.begin() + mins.size());
      std::sort(all.begin(), all.end());
    } else {
      std::merge(mins.begin(), mins.end(), maxs.begin(), maxs.end(), all.begin());
    }
    best_cost = FLT_MAX;
    best_pos = 0;
    size_t mi = 0, ma = 0;
    int leftT = 0, rightT = (int)mins.size();
    for (float val : all) {
      if (val <= box_start || val >= box_end) continue;
      while (mi < mins.size() && mins[mi] <= val) { ++mi; ++leftT; }
      while (ma < maxs.size() && maxs[ma] < val) { ++ma; --rightT; }
      float area_length = box_end - box_start;
      float left_length = val - box_start;
      float cost = 1.f + 3.f * (leftT * left_length / area_length +
                                rightT * (1.f - left_length / area_length));
      if (cost < best_cost) {
        best_cost = cost;
        best_pos = val;
      }
    }
  }

  // kdtree.cpp:93-169
  void split(Node* node) {
    if (node->geo.size() < 5) return;
    float no_split_cost = 3.f * node->geo.size();
    float best_pos[3], best_val[3];
    {
      std::vector<float> mins, maxs;
      for (int d = 0; d < 3; ++d) {
        min_max(node->geo, d, mins, maxs);
        best_split(mins, maxs, node->box_start[d], node->box_end[d], best_pos[d],
                   best_val[d]);
      }
    }
    int bd = (int)(std::min_element(best_val, best_val + 3) - best_val);
    if (best_val[bd] > no_split_cost) return;
    float pos = best_pos[bd];
    if (pos <= node->box_start[bd] || pos >= node->box_end[bd]) return;

    node->left.reset(new Node());
    node->right.reset(new Node());
    Node* l = node->left.get();
    Node* r = node->right.get();
    l->parent = r->parent = node;
    for (int d = 0; d < 3; ++d) {
      l->box_start[d] = r->box_start[d] = node->box_start[d];
      l->box_end[d] = r->box_end[d] = node->box_end[d];
    }
    l->box_end[bd] = pos;
    r->box_start[bd] = pos;
    for (int32_t g : node->geo) {
      const I4& t = tris[g];
      float v[3] = {coord(t.x, bd), coord(t.y, bd), coord(t.z, bd)};
      if (!(v[0] > pos && v[1] > pos && v[2] > pos)) l->geo.push_back(g);
      if (!(v[0] < pos && v[1] < pos && v[2] < pos)) r->geo.push_back(g);
    }
    std::vector<int32_t>().swap(node->geo);

    // The two subtrees are independent; big ones go to a worker thread.
    bool spawn = false;
    if (l->geo.size() > 20000 && r->geo.size() > 20000) {
      if (threads_left.fetch_sub(1) > 0)
        spawn = true;
      else
        threads_left.fetch_add(1);
    }
    if (spawn) {
      std::thread th([this, l] { split(l); });
      split(r);
      th.join();
      threads_left.fetch_add(1);
    } else {
      split(l);
      split(r);
    }
  }

  // kdtree.cpp:171-206
  static void remove_empty(Node* n) {
    if (!n->left && !n->right) return;
    remove_empty(n->left.get());
    remove_empty(n->right.get());
    Node* l = n->left.get();
    Node* r = n->right.get();
    if (l && l->geo.empty() && !l->left && !l->right) {
      for (int d = 0; d < 3; ++d) {
        n->box_start[d] = r->box_start[d];
        n->box_end[d] = r->box_end[d];
      }
      n->geo = r->geo;
      std::unique_ptr<Node> rl = std::move(r->left);
      std::unique_ptr<Node> rr = std::move(r->right);
      n->left = std::move(rl);
      n->right = std::move(rr);
      if (n->right) n->right->parent = n;
      if (n->left) n->left->parent = n;
      return;
    }
    if (r && r->geo.empty() && !r->left && !r->right) {
      for (int d = 0; d < 3; ++d) {
        n->box_start[d] = l->box_start[d];
        n->box_end[d] = l->box_end[d];
      }
      n->geo = l->geo;
      std::unique_ptr<Node> lr = std::move(l->right);
      std::unique_ptr<Node> ll = std::move(l->left);
      n->right = std::move(lr);
      n->left = std::move(ll);
      if (n->right) n->right->parent = n;
      if (n->left) n->left->parent = n;
      return;
    }
  }
};

}  // namespace

hpt_status build_kdtree(const F4* points, int num_points, const I4* tris,
                        int num_tris, int num_threads, KdTree& out) {
  if (num_tris < 0 || num_points < 0 || (num_tris > 0 && (!points || !tris)))
    return fail(HPT_ERR_INVALID_ARGUMENT, "kdtree: bad arguments");
  if (num_tris == 0)
    return fail(HPT_ERR_INVALID_SCENE, "kdtree: scene has no triangles");
  for (int i = 0; i < num_tris; ++i) {
    const I4& t = tris[i];
    if (t.x < 0 || t.y < 0 || t.z < 0 || t.x >= num_points ||
        t.y >= num_points || t.z >= num_points)
      return fail(HPT_ERR_INVALID_SCENE, "kdtree: triangle %d has a vertex index out of range", i);
  }
  for (int i = 0; i < num_points; ++i)
    if (!std::isfinite(points[i].x) || !std::isfinite(points[i].y) ||
        !std::isfinite(points[i].z))
      return fail(HPT_ERR_INVALID_SCENE, "kdtree: vertex %d is not finite", i);

  Builder b;
  b.points = points;
  b.tris = tris;
  if (num_threads <= 0) num_threads = (int)std::max(1u, std::thread::hardware_concurrency());
  b.threads_left = num_threads - 1;

  std::unique_ptr<Node> root(new Node());
  root->geo.resize(num_tris);
  for (int i = 0; i < num_tris; ++i) root->geo[i] = i;
  {  // setBoxSize on the root only (kdtree.cpp:36-41, 235-246)
    std::vector<float> mins, maxs;
    for (int d = 0; d < 3; ++d) {
      b.min_max(root->geo, d, mins, maxs);
      root->box_start[d] = mins.front() - 1e-3f;
      root->box_end[d] = maxs.back() + 1e-3f;
    }
  }
  b.split(root.get());
  Builder::remove_empty(root.get());

  // getData (kdtree.cpp:248-292): pre-order numbering.
  std::vector<Node*> order;
  std::vector<Node*> stack{root.get()};
  while (!stack.empty()) {
    Node* n = stack.back();
    stack.pop_back();
    order.push_back(n);
    if (n->right) stack.push_back(n->right.get());
    if (n->left) stack.push_back(n->left.get());
  }
  std::unordered_map<const Node*, int> index;
  index.reserve(order.size() * 2);
  for (size_t i = 0; i < order.size(); ++i) index[order[i]] = (int)i;

  out.nodes.assign(order.size(), hpt_ref_node());
  out.leaf_data.clear();
  for (size_t i = 0; i < order.size(); ++i) {
    Node* n = order[i];
    hpt_ref_node& h = out.nodes[i];
    h.data = -1;
    if (!n->geo.empty()) {
      h.data = (int32_t)out.leaf_data.size();
      out.leaf_data.push_back((int32_t)n->geo.size());
      out.leaf_data.insert(out.leaf_data.end(), n->geo.begin(), n->geo.end());
    }
    for (int d = 0; d < 3; ++d) {
      h.box_start[d] = n->box_start[d];
      h.box_end[d] = n->box_end[d];
    }
    h.box_start[3] = h.box_end[3] = 0.f;
    h.child = n->left ? index[n->left.get()] : -1;
    h.parent = n->parent ? index[n->parent] : -1;
    h.sibling = -1;
    if (n->parent && n->parent->right && n->parent->right.get() != n)
      h.sibling = index[n->parent->right.get()];
  }
  // Free the pointer tree iteratively (deep trees would overflow the stack
  // through recursive unique_ptr destructors).
  std::vector<std::unique_ptr<Node>> kill;
  kill.push_back(std::move(root));
  while (!kill.empty()) {
    std::unique_ptr<Node> n = std::move(kill.back());
    kill.pop_back();
    if (n->left) kill.push_back(std::move(n->left));
    if (n->right) kill.push_back(std::move(n->right));
  }
  return HPT_OK;
}

std::string validate_ref_tree(const hpt_ref_node* nodes, int num_nodes,
                              const int32_t* leaf_data, int num_leaf,
                              int num_triangles) {
  char buf[256];
  if (num_nodes <= 0 || !nodes) return "tree has no nodes";
  if (nodes[0].parent != -1) return "root has a parent";
  std::vector<uint8_t> seen(num_nodes, 0);
  // Walk the pre-order structure with an explicit stack.
  std::vector<int> stack{0};
  int visited = 0;
  int expect_next = 0;
  while (!stack.empty()) {
    int i = stack.back();
    stack.pop_back();
    if (i < 0 || i >= num_nodes) return "node index out of range";
    if (seen[i]) return "node reached twice (cycle)";
    seen[i] = 1;
    ++visited;
    if (i != expect_next) {
      snprintf(buf, sizeof buf, "node %d is not in pre-order position %d", i, expect_next);
      return buf;
    }
    ++expect_next;
    const hpt_ref_node& n = nodes[i];
    for (int d = 0; d < 3; ++d) {
      if (!std::isfinite(n.box_start[d]) || !std::isfinite(n.box_end[d]) ||
          n.box_start[d] > n.box_end[d]) {
        snprintf(buf, sizeof buf, "node %d has an invalid box", i);
        return buf;
      }
    }
    if (n.child >= 0) {
      if (n.child != i + 1) {
        snprintf(buf, sizeof buf, "node %d: child is not the next node", i);
        return buf;
      }
      if (n.child >= num_nodes) return "child out of range";
      int right = nodes[n.child].sibling;
      if (right <= n.child || right >= num_nodes) {
        snprintf(buf, sizeof buf, "node %d has no right child", i);
        return buf;
      }
      if (nodes[n.child].parent != i || nodes[right].parent != i) {
        snprintf(buf, sizeof buf, "node %d: children disagree on parent", i);
        return buf;
      }
      if (nodes[right].sibling != -1) return "right child has a sibling";
      if (n.data >= 0) {
        snprintf(buf, sizeof buf, "inner node %d carries leaf data", i);
        return buf;
      }
      stack.push_back(right);
      stack.push_back(n.child);
    } else {
      if (n.data < 0) continue;  // empty leaf (only a root can be empty)
      if (n.data >= num_leaf) return "leaf data offset out of range";
      int cnt = leaf_data[n.data];
      if (cnt < 0 || (int64_t)n.data + 1 + cnt > num_leaf) return "leaf list out of range";
      for (int k = 0; k < cnt; ++k) {
        int t = leaf_data[n.data + 1 + k];
        if (t < 0 || t >= num_triangles) {
          snprintf(buf, sizeof buf, "leaf of node %d references triangle %d", i, t);
          return buf;
        }
      }
    }
  }
  if (visited != num_nodes) return "nodes unreachable from the root";
  return std::string();
}

}  // namespace hpt
