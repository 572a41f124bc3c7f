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
// Differences that do not change the output:
//  - a triangle's min / max along an axis does not depend on the node, so a
//    child's sorted arrays are its parent's sorted (value, triangle) arrays
//    filtered to the child's triangles (linear per node) instead of being
//    recomputed and re-sorted (the reference sorts 6 arrays per node). The
//    filtered arrays hold the same values in the same order; the one case
//    where the order of equal values shows in the output (+0.0 and -0.0 in
//    one candidate list, see best_split) recomputes that axis the
//    reference's way. Small nodes keep their arrays on a per-thread stack;
//  - the candidate list is a merge of the two sorted arrays instead of a
//    re-sort;
//  - nodes come from per-thread arenas, subtrees are built by a pool of
//    worker threads, and the largest nodes scan their three axes in
//    parallel; getData numbers nodes through an index kept in each node.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <climits>
#include <cmath>
#include <functional>
#include <memory>
#include <string>
#include <thread>
#include <condition_variable>
#include <deque>
#include <mutex>

#include "host.h"

namespace hpt {

namespace {

struct Node {
  Node* left = nullptr;
  Node* right = nullptr;
  Node* parent = nullptr;
  float box_start[3], box_end[3];
  std::vector<int32_t> geo;
  int32_t index = -1;  // pre-order position (getData)
};

// Nodes come from per-thread arenas owned by the builder: no allocation per
// node on the hot path and no per-node delete (tens of millions of nodes on
// the large scenes); chunks grow geometrically.
struct NodeArena {
  std::vector<std::unique_ptr<Node[]>> chunks;
  size_t used = 0, size = 0;
  Node* make() {
    if (used == size) {
      size = size ? std::min<size_t>(2 * size, 1 << 16) : 256;
      chunks.emplace_back(new Node[size]);
      used = 0;
    }
    return &chunks.back()[used++];
  }
};

// Sorted (value, triangle) arrays of a node: per axis, the triangles' minima
// and maxima in ascending value order.
struct Keyed {
  float v;
  int32_t id;
};
struct NodeLists {
  std::vector<Keyed> mins[3], maxs[3];
};

// A node's sorted arrays wherever they live: n entries per axis and side,
// in a node's own vectors (large nodes) or in its thread's list stack.
struct ListView {
  const Keyed* mins[3];
  const Keyed* maxs[3];
  size_t n;
};

ListView view_of(const NodeLists& L) {
  ListView v;
  for (int d = 0; d < 3; ++d) {
    v.mins[d] = L.mins[d].data();
    v.maxs[d] = L.maxs[d].data();
  }
  v.n = L.mins[0].size();
  return v;
}

// Per-thread stack of the small nodes' arrays: a node's children take their
// arrays from it and give them back once both subtrees are built, so the
// arrays of a depth-first build live in a few reused chunks instead of
// being allocated per node. Chunks never move, so pointers stay valid.
struct ListStack {
  static constexpr size_t kChunk = size_t(1) << 20;  // Keyed entries
  std::vector<std::unique_ptr<Keyed[]>> chunks;
  std::vector<size_t> caps;
  size_t chunk = 0, used = 0;
  struct Mark {
    size_t chunk, used;
  };
  Mark mark() const { return {chunk, used}; }
  void release(Mark m) {
    chunk = m.chunk;
    used = m.used;
  }
  Keyed* alloc(size_t n) {
    if (chunks.empty()) {
      chunks.emplace_back(new Keyed[std::max(n, kChunk)]);
      caps.push_back(std::max(n, kChunk));
    } else if (used + n > caps[chunk]) {
      // The chunks past the current one are free (last in, first out).
      ++chunk;
      used = 0;
      if (chunk == chunks.size()) {
        chunks.emplace_back(new Keyed[std::max(n, kChunk)]);
        caps.push_back(std::max(n, kChunk));
      } else if (caps[chunk] < n) {
        chunks[chunk].reset(new Keyed[n]);
        caps[chunk] = n;
      }
    }
    Keyed* p = chunks[chunk].get() + used;
    used += n;
    return p;
  }
};

// A child subtree of more than this many triangles is handed to the worker
// pool when a worker is idle; smaller ones are built by the thread that
// split their parent.
constexpr size_t kTaskMin = 1024;
// Nodes above this many triangles scan their three axes on three threads.
constexpr size_t kParallelAxes = 1 << 15;
// Nodes up to this many triangles keep their filtered arrays on their
// thread's list stack; larger ones own vectors (they may move to another
// thread with their subtree).
constexpr size_t kSmallNode = 256;

std::atomic<uint64_t> g_builder_generation{0};

struct Builder {
  const F4* points;
  const I4* tris;
  int num_tris = 0;
  const uint64_t generation = ++g_builder_generation;
  std::mutex arenas_mu;
  std::vector<std::unique_ptr<NodeArena>> arenas;
  // Worker pool: subtrees waiting to be built, and how many are queued or
  // being built (the build is done when none are).
  struct Task {
    Node* node;
    NodeLists lists;
  };
  std::mutex q_mu;
  std::condition_variable q_cv;
  std::deque<Task> queue;
  int outstanding = 0;
  std::atomic<int> idle{0};

  // This thread's arena for this build.
  Node* make_node() {
    thread_local uint64_t tl_generation = 0;
    thread_local NodeArena* tl_arena = nullptr;
    if (tl_generation != generation) {
      std::lock_guard<std::mutex> lk(arenas_mu);
      arenas.emplace_back(new NodeArena());
      tl_arena = arenas.back().get();
      tl_generation = generation;
    }
    return tl_arena->make();
  }

  // Builds the subtree of `n` here, or queues it for an idle worker.
  void build_subtree(Node* n, NodeLists&& L) {
    if (n->geo.size() > kTaskMin && idle.load(std::memory_order_relaxed) > 0) {
      std::lock_guard<std::mutex> lk(q_mu);
      queue.push_back(Task{n, std::move(L)});
      ++outstanding;
      q_cv.notify_one();
      return;
    }
    split(n, std::move(L));
  }

  void worker() {
    std::unique_lock<std::mutex> lk(q_mu);
    while (true) {
      idle.fetch_add(1);
      q_cv.wait(lk, [&] { return !queue.empty() || outstanding == 0; });
      idle.fetch_sub(1);
      if (queue.empty()) return;  // nothing queued or running: done
      Task t = std::move(queue.front());
      queue.pop_front();
      lk.unlock();
      split(t.node, std::move(t.lists));
      lk.lock();
      if (--outstanding == 0) q_cv.notify_all();
    }
  }

  void run(Node* root, NodeLists&& L, int threads) {
    {
      std::lock_guard<std::mutex> lk(q_mu);
      queue.push_back(Task{root, std::move(L)});
      outstanding = 1;
    }
    std::vector<std::thread> th;
    for (int i = 1; i < threads; ++i) th.emplace_back([this] { worker(); });
    worker();
    for (std::thread& t : th) t.join();
  }

  float coord(int vertex, int d) const {
    const F4& p = points[vertex];
    return d == 0 ? p.x : d == 1 ? p.y : p.z;
  }

  // kdtree.cpp:23-34: the node's triangle minima and maxima along d, each
  // sorted with std::sort from the node's triangle order.
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

  // The root's sorted arrays: computed and sorted once.
  void root_lists(const std::vector<int32_t>& geo, int d, NodeLists& L) const {
    std::vector<Keyed>& mn = L.mins[d];
    std::vector<Keyed>& mx = L.maxs[d];
    mn.resize(geo.size());
    mx.resize(geo.size());
    for (size_t i = 0; i < geo.size(); ++i) {
      const I4& t = tris[geo[i]];
      float v[3] = {coord(t.x, d), coord(t.y, d), coord(t.z, d)};
      mn[i] = {*std::min_element(v, v + 3), geo[i]};
      mx[i] = {*std::max_element(v, v + 3), geo[i]};
    }
    auto by_value = [](const Keyed& a, const Keyed& b) { return a.v < b.v; };
    std::sort(mn.begin(), mn.end(), by_value);
    std::sort(mx.begin(), mx.end(), by_value);
  }

  static bool mixed_zeros(const Keyed* a, const Keyed* b, size_t n) {
    bool pos_zero = false, neg_zero = false;
    for (const Keyed* v : {a, b})
      for (size_t i = 0; i < n; ++i)
        if (v[i].v == 0.f) (std::signbit(v[i].v) ? neg_zero : pos_zero) = true;
    return pos_zero && neg_zero;
  }

  // Best split along axis d (kdtree.cpp:47-89), from the node's filtered
  // arrays when it has them (L != nullptr), else from its own sort.
  void axis_split(const Node* node, const ListView* L, int d, float& best_pos,
                  float& best_cost) const {
    thread_local std::vector<float> mins, maxs;
    if (!L || mixed_zeros(L->mins[d], L->maxs[d], L->n)) {
      // The order of +0.0 and -0.0 among themselves is the reference's sort
      // order of this node's own arrays: small nodes, and this rare case,
      // compute them its way.
      min_max(node->geo, d, mins, maxs);
    } else {
      const Keyed* mn = L->mins[d];
      const Keyed* mx = L->maxs[d];
      mins.resize(L->n);
      maxs.resize(L->n);
      for (size_t i = 0; i < L->n; ++i) mins[i] = mn[i].v;
      for (size_t i = 0; i < L->n; ++i) maxs[i] = mx[i].v;
    }
    best_split(mins, maxs, node->box_start[d], node->box_end[d], best_pos, best_cost);
  }

  // kdtree.cpp:47-89
  static void best_split(const std::vector<float>& mins,
                         const std::vector<float>& maxs, float box_start,
                         float box_end, float& best_pos, float& best_cost) {
    thread_local std::vector<float> all;
    all.resize(mins.size() + maxs.size());
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

  // kdtree.cpp:93-169. The node's filtered sorted arrays: `small` (on this
  // thread's list stack) when given, else L (consumed).
  void split(Node* node, NodeLists L, const ListView* small = nullptr) {
    const size_t n = node->geo.size();
    if (n < 5) return;
    const ListView own = small ? *small : view_of(L);
    const ListView* lists = &own;
    float no_split_cost = 3.f * n;
    float best_pos[3], best_val[3];
    if (n > kParallelAxes) {
      std::thread t1([&] { axis_split(node, lists, 1, best_pos[1], best_val[1]); });
      std::thread t2([&] { axis_split(node, lists, 2, best_pos[2], best_val[2]); });
      axis_split(node, lists, 0, best_pos[0], best_val[0]);
      t1.join();
      t2.join();
    } else {
      for (int d = 0; d < 3; ++d) axis_split(node, lists, d, best_pos[d], best_val[d]);
    }
    int bd = (int)(std::min_element(best_val, best_val + 3) - best_val);
    if (best_val[bd] > no_split_cost) return;
    float pos = best_pos[bd];
    if (pos <= node->box_start[bd] || pos >= node->box_end[bd]) return;

    Node* l = make_node();
    Node* r = make_node();
    node->left = l;
    node->right = r;
    l->parent = r->parent = node;
    for (int d = 0; d < 3; ++d) {
      l->box_start[d] = r->box_start[d] = node->box_start[d];
      l->box_end[d] = r->box_end[d] = node->box_end[d];
    }
    l->box_end[bd] = pos;
    r->box_start[bd] = pos;
    // Side of every triangle of the node (bit 0 left, bit 1 right), in this
    // thread's own table (subtrees on other threads share triangles).
    thread_local std::vector<uint8_t> side;
    if ((int)side.size() < num_tris) side.assign(num_tris, 0);
    size_t nl = 0, nr = 0;
    for (int32_t g : node->geo) {
      const I4& t = tris[g];
      float v[3] = {coord(t.x, bd), coord(t.y, bd), coord(t.z, bd)};
      const bool to_l = !(v[0] > pos && v[1] > pos && v[2] > pos);
      const bool to_r = !(v[0] < pos && v[1] < pos && v[2] < pos);
      nl += to_l;
      nr += to_r;
      side[g] = (uint8_t)((to_l ? 1 : 0) | (to_r ? 2 : 0));
    }
    l->geo.resize(nl);
    r->geo.resize(nr);
    {
      size_t il = 0, ir = 0;
      for (int32_t g : node->geo) {
        if (side[g] & 1) l->geo[il++] = g;
        if (side[g] & 2) r->geo[ir++] = g;
      }
    }
    std::vector<int32_t>().swap(node->geo);
    // The children's sorted arrays: the node's, filtered (order kept) - a
    // large child's into its own vectors, a small child's onto this
    // thread's list stack, given back once both subtrees are built (small
    // subtrees are always built here, depth first).
    thread_local ListStack stack;
    const ListStack::Mark mark = stack.mark();
    const bool big_l = nl > kSmallNode, big_r = nr > kSmallNode;
    NodeLists LL, RL;
    ListView SL{}, SR{};
    SL.n = nl;
    SR.n = nr;
    const uint8_t* sides = side.data();
    auto filter = [&](const Keyed* src, Keyed* dl, Keyed* dr) {
      size_t il = 0, ir = 0;
      for (size_t i = 0; i < n; ++i) {
        const Keyed k = src[i];
        const uint8_t sd = sides[k.id];
        if (sd & 1) dl[il++] = k;
        if (sd & 2) dr[ir++] = k;
      }
    };
    Keyed* dst[3][2][2];  // [axis][min/max][left/right]
    for (int d = 0; d < 3; ++d) {
      for (int m = 0; m < 2; ++m) {
        std::vector<Keyed>& vl = m ? LL.maxs[d] : LL.mins[d];
        std::vector<Keyed>& vr = m ? RL.maxs[d] : RL.mins[d];
        if (big_l) vl.resize(nl);
        if (big_r) vr.resize(nr);
        dst[d][m][0] = big_l ? vl.data() : stack.alloc(nl);
        dst[d][m][1] = big_r ? vr.data() : stack.alloc(nr);
        (m ? SL.maxs[d] : SL.mins[d]) = dst[d][m][0];
        (m ? SR.maxs[d] : SR.mins[d]) = dst[d][m][1];
      }
    }
    auto filter_axis = [&](int d) {
      filter(lists->mins[d], dst[d][0][0], dst[d][0][1]);
      filter(lists->maxs[d], dst[d][1][0], dst[d][1][1]);
    };
    if (n > kParallelAxes) {
      // The six arrays of a large node are independent: one axis per thread
      // (the side table is only read here).
      std::thread t1([&] { filter_axis(1); });
      std::thread t2([&] { filter_axis(2); });
      filter_axis(0);
      t1.join();
      t2.join();
    } else {
      for (int d = 0; d < 3; ++d) filter_axis(d);
    }
    if (!small) L = NodeLists();  // the node's own vectors are spent
    // The two subtrees are independent.
    if (big_r) build_subtree(r, std::move(RL));
    else split(r, NodeLists(), &SR);
    if (big_l) build_subtree(l, std::move(LL));
    else split(l, NodeLists(), &SL);
    stack.release(mark);
  }

  // kdtree.cpp:171-206
  static void remove_empty(Node* n) {
    if (!n->left && !n->right) return;
    remove_empty(n->left);
    remove_empty(n->right);
    Node* l = n->left;
    Node* r = n->right;
    if (l && l->geo.empty() && !l->left && !l->right) {
      for (int d = 0; d < 3; ++d) {
        n->box_start[d] = r->box_start[d];
        n->box_end[d] = r->box_end[d];
      }
      n->geo = std::move(r->geo);
      n->left = r->left;
      n->right = r->right;
      if (n->right) n->right->parent = n;
      if (n->left) n->left->parent = n;
      return;
    }
    if (r && r->geo.empty() && !r->left && !r->right) {
      for (int d = 0; d < 3; ++d) {
        n->box_start[d] = l->box_start[d];
        n->box_end[d] = l->box_end[d];
      }
      n->geo = std::move(l->geo);
      n->right = l->right;
      n->left = l->left;
      if (n->right) n->right->parent = n;
      if (n->left) n->left->parent = n;
      return;
    }
  }

  // Releases every arena, several at a time.
  void release() {
    std::vector<std::unique_ptr<NodeArena>> all = std::move(arenas);
    const size_t workers =
        std::min<size_t>(all.size(), std::max(1u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    std::atomic<size_t> next{0};
    for (size_t w = 0; w < workers; ++w)
      th.emplace_back([&] {
        for (size_t i = next++; i < all.size(); i = next++) all[i].reset();
      });
    for (std::thread& t : th) t.join();
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
  b.num_tris = num_tris;
  if (num_threads <= 0) num_threads = (int)std::max(1u, std::thread::hardware_concurrency());

  Node* root = b.make_node();
  root->geo.resize(num_tris);
  for (int i = 0; i < num_tris; ++i) root->geo[i] = i;
  // setBoxSize on the root only (kdtree.cpp:36-41, 235-246): the smallest
  // minimum and largest maximum per axis, +- 1e-3. The sorted arrays hold
  // exactly those values at their ends.
  NodeLists lists;
  {
    std::thread t1([&] { b.root_lists(root->geo, 1, lists); });
    std::thread t2([&] { b.root_lists(root->geo, 2, lists); });
    b.root_lists(root->geo, 0, lists);
    t1.join();
    t2.join();
  }
  for (int d = 0; d < 3; ++d) {
    root->box_start[d] = lists.mins[d].front().v - 1e-3f;
    root->box_end[d] = lists.maxs[d].back().v + 1e-3f;
  }
  b.run(root, std::move(lists), num_threads);
  Builder::remove_empty(root);

  // getData (kdtree.cpp:248-292): pre-order numbering, left subtree first.
  std::vector<Node*> order;
  {
    std::vector<Node*> stack{root};
    while (!stack.empty()) {
      Node* n = stack.back();
      stack.pop_back();
      n->index = (int32_t)order.size();
      order.push_back(n);
      if (n->right) stack.push_back(n->right);
      if (n->left) stack.push_back(n->left);
    }
  }
  // Leaf list offsets in pre-order, then the nodes and lists filled in
  // parallel.
  std::vector<int64_t> offset(order.size() + 1, 0);
  for (size_t i = 0; i < order.size(); ++i)
    offset[i + 1] = offset[i] + (order[i]->geo.empty() ? 0 : 1 + (int64_t)order[i]->geo.size());
  if (offset.back() > INT32_MAX) {
    b.release();
    return fail(HPT_ERR_OUT_OF_MEMORY, "kdtree: leaf list too long");
  }
  out.nodes.assign(order.size(), hpt_ref_node());
  out.leaf_data.assign((size_t)offset.back(), 0);
  {
    const size_t workers = (size_t)std::max(1, num_threads);
    std::vector<std::thread> th;
    const size_t per = (order.size() + workers - 1) / workers;
    for (size_t w = 0; w < workers; ++w)
      th.emplace_back([&, w] {
        const size_t lo = w * per, hi = std::min(order.size(), lo + per);
        for (size_t i = lo; i < hi; ++i) {
          const Node* n = order[i];
          hpt_ref_node& h = out.nodes[i];
          h.data = -1;
          if (!n->geo.empty()) {
            h.data = (int32_t)offset[i];
            out.leaf_data[offset[i]] = (int32_t)n->geo.size();
            std::copy(n->geo.begin(), n->geo.end(), out.leaf_data.begin() + offset[i] + 1);
          }
          for (int d = 0; d < 3; ++d) {
            h.box_start[d] = n->box_start[d];
            h.box_end[d] = n->box_end[d];
          }
          h.box_start[3] = h.box_end[3] = 0.f;
          h.child = n->left ? n->left->index : -1;
          h.parent = n->parent ? n->parent->index : -1;
          h.sibling = -1;
          if (n->parent && n->parent->right && n->parent->right != n)
            h.sibling = n->parent->right->index;
        }
      });
    for (std::thread& t : th) t.join();
  }
  b.release();
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
