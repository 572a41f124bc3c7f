// Device-side scene and wavefront layouts, shared by the host packer (C++)
// and the CUDA kernels. Plain structs only: no CUDA headers needed here.
#pragma once

#include <cstddef>
#include <cstdint>

namespace hpt {

// --- Traversal tree ------------------------------------------------------
// 8-byte node. meta bits 31..30: 0/1/2 = split axis of an inner node,
// 3 = leaf. Inner nodes: bits 29..0 = index of the left child; the right
// child is stored right after it. Leaves: bits 29..0 = leaf record index.
// word 1: split position (inner) / unused (leaf).
struct DevNode {
  uint32_t meta;
  float split;
};
static_assert(sizeof(DevNode) == 8, "8-byte traversal node");
constexpr uint32_t kLeafKind = 3u;
constexpr uint32_t kIndexMask = 0x3FFFFFFFu;

// Leaf record, 64 bytes (4 x 16 B):
//  [0] lo.x lo.y lo.z  first entry in leaf_refs (int bits)
//  [1] hi.x hi.y hi.z  number of entries (int bits)
//  [2] rope -x, +x, -y, +y   (node index, -1 = leaves the scene)
//  [3] rope -z, +z, reference node index, 0
// The box is the reference node's own box; ropes point to the smallest
// node on the other side of each face that contains the whole face.
struct DevLeaf {
  float lo[3];
  int32_t tri_begin;
  float hi[3];
  int32_t tri_count;
  int32_t rope[6];
  int32_t ref_node;
  int32_t pad;
};
static_assert(sizeof(DevLeaf) == 64, "64-byte leaf record");
static_assert(offsetof(DevLeaf, rope) == 32, "ropes at bytes 32-55 (read as int4 + int2)");

// Triangle record, one per triangle, 48 bytes (3 x 16 B): vertex a,
// e1 = b - a, e2 = c - a (computed in FP32 exactly as the reference's
// _single_intersect does), triangle id and material in the .w slots.
// Leaves reference triangles through 4-byte ids stored in the reference's
// gather order (the reference duplicates a straddling triangle in every
// leaf it touches - tens of references per triangle on its SAH trees - so
// ids keep the records themselves small enough to stay in L2).
struct DevTri {
  float a[3];
  int32_t tri_id;
  float e1[3];
  int32_t material;
  float e2[3];
  int32_t pad;
};
static_assert(sizeof(DevTri) == 48, "48-byte triangle record");

// Per-texture descriptor: texel offset into the RGBA8 pool, width, height.
struct DevTexInfo {
  int64_t offset;
  int32_t w, h;
};

// Pointers of one device-resident scene (all device addresses).
struct DevScene {
  const DevNode* nodes;
  const DevLeaf* leaves;
  const int32_t* leaf_refs;   // triangle ids in leaf (= reference gather) order
  const DevTri* tris;         // indexed by triangle id
  const float* points;      // float4 per vertex
  const float* normals;     // float4 per vertex or null
  const float* texcoords;   // float2 per vertex or null
  const int32_t* geometry;  // int4 (v0, v1, v2, material) per triangle
  const void* materials;    // hpt_ref_material[]
  const int32_t* lights;    // int4 [num_lights]
  const uint32_t* texels;   // RGBA8 pool
  const DevTexInfo* tex_info;
  int32_t num_nodes, num_leaves, num_leaf_tris, num_triangles;
  int32_t num_points, num_normals, num_texcoords, num_materials;
  int32_t num_lights, num_textures;
  float root_lo[3], root_hi[3];
  float scene_eps;          // termination slack in world units
  int32_t max_steps;        // traversal step cap per ray
};

// The fields of a DevScene the traversal reads (80 bytes): a launch whose
// jobs render several scenes keeps one per job slot in shared memory, so a
// traversal step reads its scene's pointers and sizes from there instead
// of from the job table in global memory.
struct TravScene {
  const DevNode* nodes;
  const DevLeaf* leaves;
  const int32_t* leaf_refs;
  const DevTri* tris;
  int32_t num_nodes, num_leaves, num_leaf_tris, num_triangles;
  float root_lo[3], root_hi[3];
  float scene_eps;
  int32_t max_steps;
};
static_assert(sizeof(TravScene) == 80, "80-byte traversal scene");

// --- Wavefront job table ------------------------------------------------
// One render job (a frame of one scene) in a slot of the engine's table.
// Read-only while the job runs; its mutable scheduling state is DevSlot.
struct DevJob {
  DevScene scene;
  float view_p[3], top[3], right[3];
  float width, height;
  int32_t nx, ny;           // rays per frame along x and y
  int32_t pano;             // 1 = equirectangular (set_viewdirs_vr)
  int32_t vr_x_shift;       // int(right.x) * supersample_x
  float bg[3];
  int32_t spp, depth, disable_diffuse;
  int32_t first_sample;     // the frame's index of this job's sample 0 (RNG key)
  uint64_t seed;
  unsigned long long* accum;  // 3 x fixed-point u64 per ray
  uint32_t* flags;          // per ray: NaN / +inf / -inf markers (4 bits per channel)
  float* prim;              // primary hit cache, 8 floats per entry
  int32_t* prim_count;      // number of primary hits
  int64_t max_inflight;     // cap on started-but-unfinished paths (0 = none)
};

// Scheduling state of a slot. A job's paths are (primary hit k, sample s)
// pairs enumerated as q = s * hits + k; `cursor` is the next q to start.
struct DevSlot {
  int64_t num_paths;        // hits * spp, set after the primary pass
  int64_t cursor;
  unsigned long long done;  // paths finished (flushed)
  unsigned long long queries;  // secondary intersect queries issued
  int64_t max_inflight;     // copied from the job at admission (0 = none)
  int32_t alloc;            // new paths granted for the coming shade pass
  int32_t active;           // admitted and not yet fully issued
};

// Error word shared by the kernels. flags bit 0: a traversal hit its step
// cap; bit 1: a device self-check failed (builds with HPT_DEVICE_CHECKS),
// in which case site / value describe the first failure.
struct DevErr {
  uint32_t flags;
  int32_t site;
  long long value;
};

// Wavefront control block (device memory, updated by the control kernel).
struct DevCtrl {
  int32_t nA;               // paths in the current shade queue
  int32_t nR;               // rays in the intersect queue
  int32_t nA_next;          // hits appended by the intersect kernel
  int32_t parity;           // which shade buffer is current
  int32_t n_new;            // new paths granted to the coming shade pass
  int32_t done;             // no queued path and nothing left to issue
  int32_t n_quota;          // slots with a grant (quota_slot / quota_prefix)
  int32_t n_order;          // slots in priority order (host-written)
  int64_t iterations;
  // Refill cursors of the intersect and primary kernels. 64-bit: one
  // admission's primary rays may exceed 2^31 (several jobs of up to 2^30
  // rays each).
  unsigned long long isect_head;
  unsigned long long prim_head;
  DevErr err;
  unsigned long long isect_queries;
  unsigned long long shades;
  unsigned long long nodes_visited;
  unsigned long long leaves_visited;
  unsigned long long tri_tests;
  unsigned long long tri_repeats;
  // Self-check builds only: items the shade / intersect passes of the
  // current iteration actually processed, compared by the control kernel
  // with the queue sizes.
  int32_t chk_shade_items;
  int32_t chk_shade_done;
  int32_t chk_isect_done;
  int32_t chk_pad;
  // Started-but-unfinished paths all capped slots (max_inflight > 0) may
  // hold together (0 = no shared cap); host-written.
  int64_t capped_budget;
};

// Fixed-point scale of the per-ray accumulators (2^32): integer sums are
// exact and order-independent, so a render is bit-reproducible no matter
// how paths are scheduled.
constexpr double kAccumScale = 4294967296.0;

}  // namespace hpt
