// C ABI: device-resident scenes, render, per-stage entry points, stream
// compaction, batching. (Host-only producers live in capi_host.cpp.)
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/hpt.h"
#include "engine.h"
#include "scene_pack.h"
#include "shading.cuh"
#include "traverse.cuh"

using namespace hpt;

namespace hpt {

namespace {

template <typename T>
hpt_status dev_upload(SceneDev& s, const T* host, size_t count, const T** out) {
  *out = nullptr;
  if (count == 0) return HPT_OK;
  void* p = nullptr;
  HPT_CUDA(cudaMalloc(&p, count * sizeof(T)));
  s.allocations.push_back(p);
  s.bytes += (int64_t)(count * sizeof(T));
  HPT_CUDA(cudaMemcpy(p, host, count * sizeof(T), cudaMemcpyHostToDevice));
  *out = static_cast<const T*>(p);
  return HPT_OK;
}

// Device buffer for stage entry points: upload (optional) and download.
struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~DBuf() {
    if (p) HPT_SOFT(cudaFree(p));
  }
  hpt_status alloc(size_t b) {
    bytes = b;
    if (b == 0) return HPT_OK;
    HPT_CUDA(cudaMalloc(&p, b));
    return HPT_OK;
  }
  hpt_status up(const void* host, size_t b) {
    hpt_status s = alloc(b);
    if (s != HPT_OK || b == 0) return s;
    HPT_CUDA(cudaMemcpy(p, host, b, cudaMemcpyHostToDevice));
    return HPT_OK;
  }
  hpt_status down(void* host) const {
    if (!host || bytes == 0) return HPT_OK;
    HPT_CUDA(cudaMemcpy(host, p, bytes, cudaMemcpyDeviceToHost));
    return HPT_OK;
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// ---------------------------------------------------------------------------
// Stage kernels (one thread per element).
// ---------------------------------------------------------------------------
__global__ void k_stage_intersect(const DevScene* s, int n, const float* o, const float* d,
                                  int32_t* tri, float* t, float* u, float* v, DevErr* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  TravState st;
  TravCold tc;
  trav_init(*s, Ray{mk(o[3 * i], o[3 * i + 1], o[3 * i + 2]), mk(d[3 * i], d[3 * i + 1], d[3 * i + 2])},
            st, tc);
  TravCount cnt{};
  while (!trav_leaf<true>(*s, st, tc, nullptr, 0, err, cnt)) {
  }
  tri[i] = st.best.tri;
  t[i] = st.best.rec >= 0 ? st.best.t : 0.f;
  u[i] = st.best.rec >= 0 ? st.best.u : 0.f;
  v[i] = st.best.rec >= 0 ? st.best.v : 0.f;
}

__global__ void k_stage_shade(const DevScene* s, int n, const float* o, const float* d,
                              const float* strength, const int32_t* tri, const float* t,
                              uint64_t* seeds, int disable_diffuse, float* contrib,
                              int32_t* branch, float* hit_p, float* normal, float* strength_out,
                              float* param) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t seed = seeds[i];
  const Ray r{mk(o[3 * i], o[3 * i + 1], o[3 * i + 2]), mk(d[3 * i], d[3 * i + 1], d[3 * i + 2])};
  const ShadeOut so = shade_hit(*s, r, mk(strength[3 * i], strength[3 * i + 1], strength[3 * i + 2]),
                                tri[i], t[i], disable_diffuse, seed);
  seeds[i] = seed;
  contrib[3 * i] = so.contrib.x; contrib[3 * i + 1] = so.contrib.y; contrib[3 * i + 2] = so.contrib.z;
  hit_p[3 * i] = so.hit_p.x; hit_p[3 * i + 1] = so.hit_p.y; hit_p[3 * i + 2] = so.hit_p.z;
  normal[3 * i] = so.normal.x; normal[3 * i + 1] = so.normal.y; normal[3 * i + 2] = so.normal.z;
  strength_out[3 * i] = so.strength.x;
  strength_out[3 * i + 1] = so.strength.y;
  strength_out[3 * i + 2] = so.strength.z;
  param[i] = so.param;
  branch[i] = so.branch;
}

__global__ void k_stage_next(const DevScene* s, int n, const int32_t* branch, const float* d,
                             const float* hit_p, const float* normal, const float* strength,
                             const float* param, uint64_t* seeds, float* o_out, float* d_out,
                             float* s_out, int32_t* alive) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t seed = seeds[i];
  const NextOut no = next_direction(*s, branch[i], mk(d[3 * i], d[3 * i + 1], d[3 * i + 2]),
                                    mk(hit_p[3 * i], hit_p[3 * i + 1], hit_p[3 * i + 2]),
                                    mk(normal[3 * i], normal[3 * i + 1], normal[3 * i + 2]),
                                    mk(strength[3 * i], strength[3 * i + 1], strength[3 * i + 2]),
                                    param[i], seed);
  seeds[i] = seed;
  o_out[3 * i] = no.o.x; o_out[3 * i + 1] = no.o.y; o_out[3 * i + 2] = no.o.z;
  d_out[3 * i] = no.d.x; d_out[3 * i + 1] = no.d.y; d_out[3 * i + 2] = no.d.z;
  s_out[3 * i] = no.strength.x; s_out[3 * i + 1] = no.strength.y; s_out[3 * i + 2] = no.strength.z;
  alive[i] = no.alive ? 1 : 0;
}

__global__ void k_stage_raygen(hpt_camera cam, int nx, int ny, int pano, int x_shift, float* o,
                               float* d) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= nx || y >= ny) return;
  const f3 dir = pano ? pano_dir(x, y, x_shift, ny)
                      : pinhole_dir(cam.top_dir, cam.right_dir, cam.width, cam.height, x, y, nx, ny);
  const int64_t idx = (int64_t)nx * y + x;
  o[3 * idx] = cam.view_p[0]; o[3 * idx + 1] = cam.view_p[1]; o[3 * idx + 2] = cam.view_p[2];
  d[3 * idx] = dir.x; d[3 * idx + 1] = dir.y; d[3 * idx + 2] = dir.z;
}

__device__ __forceinline__ uint8_t unorm8(float x) {
  const float v = __fmul_rn(x, 255.0f);
  if (!(v >= 0.f)) return 0;
  if (v >= 255.f) return 255;
  return (uint8_t)__float2int_rn(v);
}

__global__ void k_stage_resolve(const float* accum, int W, int H, int ssx, int ssy, int spp,
                                float brightness, uint8_t* rgba) {
  const int gx = blockIdx.x * blockDim.x + threadIdx.x;
  const int gy = blockIdx.y * blockDim.y + threadIdx.y;
  if (gx >= W || gy >= H) return;
  float p[3] = {0.f, 0.f, 0.f};
  for (int i = 0; i < ssx; ++i)
    for (int j = 0; j < ssy; ++j) {
      const int64_t idx = (int64_t)(gy * ssy + j) * W * ssx + gx * ssx + i;
      for (int c = 0; c < 3; ++c) p[c] = __fadd_rn(p[c], accum[3 * idx + c]);
    }
  uint8_t* out = rgba + 4 * ((int64_t)gy * W + gx);
  for (int c = 0; c < 3; ++c) {
    float x = __fmul_rn(__fdiv_rn(__fdiv_rn(p[c], (float)(ssx * ssy)), (float)spp), brightness);
    out[c] = unorm8(__fsub_rn(1.f, expf(-x)));
  }
  out[3] = 0;
}

// --- Stream compaction: per-tile counts, then a stable scatter. ----------
// A tile is 4096 flags: 256 threads x 16 consecutive flags, read as four
// 16-byte loads where the flag array is 16-byte aligned and the tile is
// whole. The flags are read once: the count pass also stores each thread's
// 16 flags as a 16-bit mask (n / 8 bytes in all), which the scatter pass
// reads instead of the flags. Tiles are grouped into superblocks of
// 2^shift tiles with shift = ceil(log2(tiles) / 2); the count pass adds
// each tile's count to its superblock's total, and the scatter pass finds a
// tile's output offset by summing at most 2^shift superblock totals and
// 2^shift tile counts (L2-resident) instead of waiting for a scan. No
// kernel waits on another block: the two passes are ordered by the stream.
constexpr int kCompactThreads = 256;
constexpr int kCompactItems = 16;
constexpr int kCompactTile = kCompactThreads * kCompactItems;

inline int compact_super_shift(int tiles) {
  int s = 0;
  while ((int64_t)1 << (2 * s) < tiles) ++s;
  return s;
}
inline int compact_supers(int tiles, int shift) { return (tiles + (1 << shift) - 1) >> shift; }

// This thread's 16 flags as a bit mask (bit k: flag i0 + k nonzero).
__device__ __forceinline__ uint32_t load_flags16(const uint32_t* flags, int64_t i0, int n,
                                                 bool vec) {
  uint32_t m = 0;
  if (vec && i0 + kCompactItems <= n) {
    const uint4* p = reinterpret_cast<const uint4*>(flags + i0);
    const uint4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
    m = (a.x != 0) | (a.y != 0) << 1 | (a.z != 0) << 2 | (a.w != 0) << 3 | (b.x != 0) << 4 |
        (b.y != 0) << 5 | (b.z != 0) << 6 | (b.w != 0) << 7 | (c.x != 0) << 8 |
        (c.y != 0) << 9 | (c.z != 0) << 10 | (c.w != 0) << 11 | (d.x != 0) << 12 |
        (d.y != 0) << 13 | (d.z != 0) << 14 | (d.w != 0) << 15;
  } else {
    for (int k = 0; k < kCompactItems; ++k)
      if (i0 + k < n && __ldg(flags + i0 + k) != 0) m |= 1u << k;
  }
  return m;
}

// Exclusive scan of one value per thread over a block of BS threads;
// *total receives the block's sum. Two barriers.
template <int BS>
__device__ __forceinline__ int block_exclusive_scan(int v, int* total) {
  __shared__ int warp_tot[BS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int inc = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) warp_tot[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    int t = lane < BS / 32 ? warp_tot[lane] : 0;
    int ti = t;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xFFFFFFFFu, ti, o);
      if (lane >= o) ti += y;
    }
    if (lane < BS / 32) warp_tot[lane] = ti - t;  // exclusive warp offsets
    const int all = __shfl_sync(0xFFFFFFFFu, ti, 31);
    if (lane == 0) *total = all;
  }
  __syncthreads();
  return warp_tot[warp] + inc - v;
}

__global__ void __launch_bounds__(kCompactThreads)
    k_compact_count(const uint32_t* flags, int n, int shift, int* tile_counts, int* super_counts,
                    uint16_t* masks) {
  __shared__ int warp_sum[kCompactThreads / 32];
  const bool vec = (reinterpret_cast<uintptr_t>(flags) & 15) == 0;
  const int64_t i0 = (int64_t)blockIdx.x * kCompactTile + (int64_t)threadIdx.x * kCompactItems;
  const uint32_t m = load_flags16(flags, i0, n, vec);
  masks[(int64_t)blockIdx.x * kCompactThreads + threadIdx.x] = (uint16_t)m;
  const int w = __reduce_add_sync(0xFFFFFFFFu, __popc(m));
  if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = w;
  __syncthreads();
  if (threadIdx.x == 0) {
    int sum = 0;
    for (int k = 0; k < kCompactThreads / 32; ++k) sum += warp_sum[k];
    tile_counts[blockIdx.x] = sum;
    if (sum) atomicAdd(&super_counts[blockIdx.x >> shift], sum);
  }
}

// One tile per block, no staging: the 16-bit masks of lanes 2r and 2r + 1
// of a warp, read as one 32-bit word, are the survivor bits of the 32
// consecutive flags w * 512 + r * 32 + [0, 32) of its tile, lane l's flag
// in bit l. So for each of its 16 rows a warp writes the row's survivors
// to consecutive slots with one coalesced store (position: the popcount of
// the row's bits below the lane). Mask bits of flags at or past n are zero
// (the count pass bounds-checks), so the scatter needs no n. The block of
// the last tile writes the survivor total.
__global__ void __launch_bounds__(kCompactThreads)
    k_compact_scatter(const uint32_t* rows, int tiles, int shift, const int* tile_counts,
                      const int* super_counts, int* out, int* total) {
  constexpr int kWarps = kCompactThreads / 32;
  constexpr int kRows = kCompactItems;  // 32-flag rows per warp
  __shared__ int before[kWarps], warp_count[kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int b = blockIdx.x;
  const uint32_t word = lane < kRows ? rows[((int64_t)b * kWarps + warp) * kRows + lane] : 0u;
  const int wcount = __reduce_add_sync(0xFFFFFFFFu, __popc(word));
  // Survivors of the earlier superblocks, then of this superblock's earlier
  // tiles (each warp sums a share).
  const int sb = b >> shift;
  int acc = 0;
  for (int i = threadIdx.x; i < sb; i += kCompactThreads) acc += super_counts[i];
  for (int i = (sb << shift) + threadIdx.x; i < b; i += kCompactThreads) acc += tile_counts[i];
  acc = __reduce_add_sync(0xFFFFFFFFu, acc);
  if (lane == 0) {
    before[warp] = acc;
    warp_count[warp] = wcount;
  }
  __syncthreads();
  int base = 0, offset = 0, count = 0;
#pragma unroll
  for (int k = 0; k < kWarps; ++k) {
    base += before[k];
    offset += k < warp ? warp_count[k] : 0;
    count += warp_count[k];
  }
  int o = base + offset;
  const int f0 = (int)((int64_t)b * kCompactTile) + warp * (kRows * 32) + lane;
  const uint32_t below = (1u << lane) - 1u;  // lanes below this one
#pragma unroll
  for (int r = 0; r < kRows; ++r) {
    const uint32_t bits = __shfl_sync(0xFFFFFFFFu, word, r);
    if ((bits >> lane) & 1u) out[o + __popc(bits & below)] = f0 + r * 32;
    o += __popc(bits);
  }
  if (b == tiles - 1 && threadIdx.x == 0) *total = base + count;
}

inline int blocks_for(int64_t n, int bs) { return (int)((n + bs - 1) / bs); }

// Enqueues the two compaction passes on `st`. Scratch: tile_counts (tiles
// ints), super_counts (compact_supers(tiles, shift) ints, zeroed here) and
// masks (tiles * 256 16-bit masks); the survivor count goes to *total.
cudaError_t launch_compact(const uint32_t* flags, int n, int* tile_counts, int* super_counts,
                           uint16_t* masks, int* out, int* total, cudaStream_t st) {
  const int tiles = blocks_for(n, kCompactTile);
  const int shift = compact_super_shift(tiles);
  cudaError_t e = cudaMemsetAsync(super_counts, 0,
                                  (size_t)compact_supers(tiles, shift) * sizeof(int), st);
  if (e != cudaSuccess) return e;
  k_compact_count<<<tiles, kCompactThreads, 0, st>>>(flags, n, shift, tile_counts, super_counts,
                                                     masks);
  k_compact_scatter<<<tiles, kCompactThreads, 0, st>>>(reinterpret_cast<const uint32_t*>(masks),
                                                       tiles, shift, tile_counts, super_counts,
                                                       out, total);
  return cudaGetLastError();
}

hpt_status check_scene_desc(const hpt_scene_desc& d) {
  if (d.num_points < 0 || d.num_triangles <= 0 || d.num_nodes <= 0 || d.num_leaf_data < 0 ||
      d.num_materials <= 0 || d.num_lights < 0 || d.num_textures < 0 || d.num_normals < 0 ||
      d.num_texcoords < 0)
    return fail(HPT_ERR_INVALID_ARGUMENT, "scene: negative or empty counts");
  if (!d.points || !d.triangles || !d.nodes || !d.materials || (d.num_leaf_data && !d.leaf_data))
    return fail(HPT_ERR_INVALID_ARGUMENT, "scene: missing buffers");
  if (d.num_normals != 0 && d.num_normals != d.num_points)
    return fail(HPT_ERR_INVALID_SCENE,
                "scene: %d normals for %d vertices (normals are indexed by vertex id)",
                d.num_normals, d.num_points);
  if (d.num_texcoords != 0 && d.num_texcoords != d.num_points)
    return fail(HPT_ERR_INVALID_SCENE, "scene: %d texcoords for %d vertices", d.num_texcoords,
                d.num_points);
  const F4* pts = reinterpret_cast<const F4*>(d.points);
  for (int i = 0; i < d.num_points; ++i)
    if (!std::isfinite(pts[i].x) || !std::isfinite(pts[i].y) || !std::isfinite(pts[i].z))
      return fail(HPT_ERR_INVALID_SCENE, "scene: vertex %d is not finite", i);
  const I4* tris = reinterpret_cast<const I4*>(d.triangles);
  for (int i = 0; i < d.num_triangles; ++i) {
    const I4& t = tris[i];
    if (t.x < 0 || t.y < 0 || t.z < 0 || t.x >= d.num_points || t.y >= d.num_points ||
        t.z >= d.num_points)
      return fail(HPT_ERR_INVALID_SCENE, "scene: triangle %d vertex index out of range", i);
    if (t.w < 0 || t.w >= d.num_materials)
      return fail(HPT_ERR_INVALID_SCENE, "scene: triangle %d material %d out of range", i, t.w);
  }
  if (d.num_lights > 0 && !d.lights) return fail(HPT_ERR_INVALID_ARGUMENT, "scene: lights missing");
  const I4* lights = reinterpret_cast<const I4*>(d.lights);
  for (int i = 0; i < d.num_lights; ++i) {
    const I4& t = lights[i];
    if (t.x < 0 || t.y < 0 || t.z < 0 || t.x >= d.num_points || t.y >= d.num_points ||
        t.z >= d.num_points)
      return fail(HPT_ERR_INVALID_SCENE, "scene: light %d vertex index out of range", i);
  }
  for (int i = 0; i < d.num_materials; ++i) {
    const hpt_ref_material& m = d.materials[i];
    if (m.diffuse_texture_id >= d.num_textures || m.ambient_texture_id >= d.num_textures)
      return fail(HPT_ERR_INVALID_SCENE, "scene: material %d references a missing texture", i);
  }
  if (d.num_textures > 0 && !d.texture_data)
    return fail(HPT_ERR_INVALID_ARGUMENT, "scene: texture data missing");
  if (d.texture_dims)
    for (int i = 0; i < d.num_textures; ++i)
      if (d.texture_dims[2 * i] <= 0 || d.texture_dims[2 * i + 1] <= 0)
        return fail(HPT_ERR_INVALID_SCENE, "scene: texture %d has no texels", i);
  return HPT_OK;
}

}  // namespace

hpt_status upload_scene(const hpt_scene_desc& d, SceneDev& out) {
  hpt_status s = check_scene_desc(d);
  if (s != HPT_OK) return s;
  PackedScene pk;
  s = pack_scene(d, 8192, pk);
  if (s != HPT_OK) return s;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(HPT_ERR_CUDA, "no CUDA device");
  if (d.device < 0 || d.device >= ndev) return fail(HPT_ERR_INVALID_ARGUMENT, "bad device %d", d.device);
  HPT_CUDA(cudaSetDevice(d.device));
  out.device = d.device;
  DevScene& ds = out.dev;
  memset(&ds, 0, sizeof ds);
  const DevNode* nodes;
  const DevLeaf* leaves;
  const DevTri* recs;
  const int32_t* refs;
  if ((s = dev_upload(out, pk.nodes.data(), pk.nodes.size(), &nodes)) != HPT_OK) return s;
  if ((s = dev_upload(out, pk.leaves.data(), pk.leaves.size(), &leaves)) != HPT_OK) return s;
  // At least one entry so the pointer is valid even for an empty tree.
  if (pk.refs.empty()) pk.refs.push_back(0);
  if ((s = dev_upload(out, pk.refs.data(), pk.refs.size(), &refs)) != HPT_OK) return s;
  if ((s = dev_upload(out, pk.tris.data(), pk.tris.size(), &recs)) != HPT_OK) return s;
  ds.nodes = nodes;
  ds.leaves = leaves;
  ds.leaf_refs = refs;
  ds.tris = recs;
  const float* f = nullptr;
  if ((s = dev_upload(out, d.points, 4 * (size_t)d.num_points, &f)) != HPT_OK) return s;
  ds.points = f;
  if ((s = dev_upload(out, d.normals, 4 * (size_t)d.num_normals, &f)) != HPT_OK) return s;
  ds.normals = f;
  if ((s = dev_upload(out, d.texcoords, 2 * (size_t)d.num_texcoords, &f)) != HPT_OK) return s;
  ds.texcoords = f;
  const int32_t* ip = nullptr;
  if ((s = dev_upload(out, d.triangles, 4 * (size_t)d.num_triangles, &ip)) != HPT_OK) return s;
  ds.geometry = ip;
  const hpt_ref_material* mp = nullptr;
  if ((s = dev_upload(out, d.materials, (size_t)d.num_materials, &mp)) != HPT_OK) return s;
  ds.materials = mp;
  if ((s = dev_upload(out, d.lights, 4 * (size_t)d.num_lights, &ip)) != HPT_OK) return s;
  ds.lights = ip;
  std::vector<DevTexInfo> ti(d.num_textures);
  int64_t texels = 0;
  for (int t = 0; t < d.num_textures; ++t) {
    ti[t].offset = texels;
    ti[t].w = d.texture_dims ? d.texture_dims[2 * t] : 512;
    ti[t].h = d.texture_dims ? d.texture_dims[2 * t + 1] : 512;
    texels += (int64_t)ti[t].w * ti[t].h;
  }
  const uint32_t* tx = nullptr;
  if ((s = dev_upload(out, reinterpret_cast<const uint32_t*>(d.texture_data), (size_t)texels, &tx)) != HPT_OK)
    return s;
  ds.texels = tx;
  const DevTexInfo* tip = nullptr;
  if ((s = dev_upload(out, ti.data(), ti.size(), &tip)) != HPT_OK) return s;
  ds.tex_info = tip;
  ds.num_nodes = (int32_t)pk.nodes.size();
  ds.num_leaves = (int32_t)pk.leaves.size();
  ds.num_leaf_tris = (int32_t)pk.refs.size();
  ds.num_triangles = d.num_triangles;
  ds.num_points = d.num_points;
  ds.num_normals = d.num_normals;
  ds.num_texcoords = d.num_texcoords;
  ds.num_materials = d.num_materials;
  ds.num_lights = d.num_lights;
  ds.num_textures = d.num_textures;
  float scale = 0.f;
  for (int a = 0; a < 3; ++a) {
    ds.root_lo[a] = pk.root_lo[a];
    ds.root_hi[a] = pk.root_hi[a];
    scale = std::max({scale, std::fabs(pk.root_lo[a]), std::fabs(pk.root_hi[a]),
                      pk.root_hi[a] - pk.root_lo[a]});
  }
  ds.scene_eps = 2e-5f * scale;
  const int64_t cap = 8 * ((int64_t)pk.nodes.size() + (int64_t)pk.refs.size()) + 100000;
  ds.max_steps = (int32_t)std::min<int64_t>(cap, 1 << 30);
  void* p = nullptr;
  HPT_CUDA(cudaMalloc(&p, sizeof(DevScene)));
  out.allocations.push_back(p);
  HPT_CUDA(cudaMemcpy(p, &ds, sizeof(DevScene), cudaMemcpyHostToDevice));
  // A cudaMemcpy from pageable memory may return before its DMA has landed,
  // and the render engines run on non-blocking streams that are not ordered
  // after the legacy stream: wait here so no kernel can read a partially
  // uploaded scene.
  HPT_CUDA(cudaDeviceSynchronize());
  out.d_scene = static_cast<DevScene*>(p);
  out.info.num_triangles = d.num_triangles;
  out.info.num_ref_nodes = d.num_nodes;
  out.info.num_device_nodes = ds.num_nodes;
  out.info.num_leaves = ds.num_leaves;
  out.info.num_leaf_triangles = (int32_t)pk.refs.size();
  out.info.max_depth = pk.max_depth;
  out.info.device_bytes = out.bytes;
  return HPT_OK;
}

void release_scene(SceneDev& s) {
  HPT_SOFT(cudaSetDevice(s.device));
  for (void* p : s.allocations) HPT_SOFT(cudaFree(p));
  s.allocations.clear();
}

}  // namespace hpt

namespace {

// Ranges the engine supports (capacity: queue entries; smem_nodes: shared
// node prefix; trav_steps: 0 = leaf per round, 1..256 step units per round;
// isect_block / isect_min_blocks: a compiled traversal variant,
// 0 min blocks = the block size's default).
hpt_status check_tuning(const hpt_tuning& t) {
  if (t.capacity < 1024 || t.capacity > (1 << 27) || t.smem_nodes < 0 ||
      t.smem_nodes > kMaxSmemNodes || t.refill_chunk < 1 || t.refill_chunk > 32 ||
      (t.isect_block != 128 && t.isect_block != 256) || t.isect_min_blocks < 0 ||
      t.trav_steps < 0 || t.trav_steps > 256 || t.max_steps < 0 ||
      (t.shade_min_blocks != 0 && t.shade_min_blocks != 3 && t.shade_min_blocks != 4))
    return fail(HPT_ERR_INVALID_ARGUMENT, "tuning out of range");
  return HPT_OK;
}

hpt_status check_params(const hpt_camera* cam, const hpt_render_params* p) {
  return check_render_params(cam, p);
}

template <typename F>
hpt_status guarded(F&& f) {
  try {
    return f();
  } catch (const std::bad_alloc&) {
    return fail(HPT_ERR_OUT_OF_MEMORY, "host allocation failed");
  } catch (...) {
    return fail(HPT_ERR_INVALID_ARGUMENT, "unexpected exception");
  }
}

}  // namespace

extern "C" {

int hpt_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    (void)cudaGetLastError();  // "no device" is an answer here, not an error
    return 0;
  }
  return n;
}

hpt_status hpt_scene_create(const hpt_scene_desc* desc, hpt_scene** out) {
  if (!desc || !out) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  *out = nullptr;
  return guarded([&]() -> hpt_status {
    std::unique_ptr<hpt_scene> s(new hpt_scene());
    hpt_status st = upload_scene(*desc, s->h.scene);
    if (st != HPT_OK) {
      release_scene(s->h.scene);
      return st;
    }
    s->h.tuning = default_tuning();
    *out = s.release();
    return HPT_OK;
  });
}

hpt_status hpt_scene_info_get(const hpt_scene* scene, hpt_scene_info* out) {
  if (!scene || !out) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  *out = scene->h.scene.info;
  return HPT_OK;
}

void hpt_scene_destroy(hpt_scene* scene) {
  if (!scene) return;
  {
    std::lock_guard<std::mutex> lk(scene->h.mu);
    scene->h.engine.reset();
    release_scene(scene->h.scene);
  }
  delete scene;
}

hpt_status hpt_render(hpt_scene* scene, const hpt_camera* camera, const hpt_render_params* params,
                      uint8_t* rgba_out, float* accum_out) {
  if (!scene) return fail(HPT_ERR_INVALID_ARGUMENT, "scene is NULL");
  hpt_status s = check_params(camera, params);
  if (s != HPT_OK) return s;
  return guarded([&]() -> hpt_status {
    std::lock_guard<std::mutex> lk(scene->h.mu);
    if (!scene->h.engine) scene->h.engine.reset(new Engine(scene->h.scene.device));
    scene->h.engine->tuning = scene->h.tuning;
    JobSpec js;
    js.scene = &scene->h.scene;
    js.camera = *camera;
    js.params = *params;
    js.rgba_out = rgba_out;
    js.accum_out = accum_out;
    return scene->h.engine->run({js}, &scene->h.last_stats);
  });
}

hpt_status hpt_render_stats_get(const hpt_scene* scene, hpt_render_stats* out) {
  if (!scene || !out) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  *out = scene->h.last_stats;
  return HPT_OK;
}

hpt_status hpt_tuning_get(const hpt_scene* scene, hpt_tuning* out) {
  if (!scene || !out) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  *out = scene->h.tuning;
  return HPT_OK;
}

hpt_status hpt_tuning_set(hpt_scene* scene, const hpt_tuning* in) {
  if (!scene || !in) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  hpt_status st = check_tuning(*in);
  if (st != HPT_OK) return st;
  std::lock_guard<std::mutex> lk(scene->h.mu);
  scene->h.tuning = *in;
  scene->h.tuning.shade_block = 256;
  scene->h.engine.reset();
  return HPT_OK;
}

hpt_status hpt_raygen(const hpt_camera* camera, int32_t sample_x, int32_t sample_y,
                      int32_t supersample_x, int32_t supersample_y, float* origins,
                      float* directions) {
  if (!camera || !origins || !directions || sample_x <= 0 || sample_y <= 0 || supersample_x <= 0 ||
      supersample_y <= 0)
    return fail(HPT_ERR_INVALID_ARGUMENT, "bad raygen arguments");
  if (camera->height < 0 && supersample_x != supersample_y)
    return fail(HPT_ERR_INVALID_ARGUMENT, "panorama needs supersample_x == supersample_y");
  return guarded([&]() -> hpt_status {
    const int nx = sample_x * supersample_x, ny = sample_y * supersample_y;
    const size_t bytes = (size_t)nx * ny * 3 * sizeof(float);
    DBuf o, d;
    hpt_status s;
    if ((s = o.alloc(bytes)) != HPT_OK || (s = d.alloc(bytes)) != HPT_OK) return s;
    const int pano = camera->height < 0;
    const int shift = (int)camera->right_dir[0] * supersample_x;
    dim3 blk(16, 16), grd((nx + 15) / 16, (ny + 15) / 16);
    k_stage_raygen<<<grd, blk>>>(*camera, nx, ny, pano, shift, o.as<float>(), d.as<float>());
    HPT_CUDA(cudaGetLastError());
    if ((s = o.down(origins)) != HPT_OK) return s;
    return d.down(directions);
  });
}

hpt_status hpt_intersect(hpt_scene* scene, int32_t n, const float* origins,
                         const float* directions, int32_t* tri_out, float* t_out, float* u_out,
                         float* v_out) {
  if (!scene || n < 0 || (n > 0 && (!origins || !directions || !tri_out || !t_out || !u_out || !v_out)))
    return fail(HPT_ERR_INVALID_ARGUMENT, "bad intersect arguments");
  if (n == 0) return HPT_OK;
  return guarded([&]() -> hpt_status {
    std::lock_guard<std::mutex> lk(scene->h.mu);
    HPT_CUDA(cudaSetDevice(scene->h.scene.device));
    DBuf o, d, tri, t, u, v, err;
    hpt_status s;
    const size_t b3 = (size_t)n * 3 * sizeof(float), b1 = (size_t)n * 4;
    if ((s = o.up(origins, b3)) || (s = d.up(directions, b3)) || (s = tri.alloc(b1)) ||
        (s = t.alloc(b1)) || (s = u.alloc(b1)) || (s = v.alloc(b1)) ||
        (s = err.alloc(sizeof(DevErr))))
      return s;
    HPT_CUDA(cudaMemset(err.p, 0, sizeof(DevErr)));
    k_stage_intersect<<<blocks_for(n, 128), 128>>>(scene->h.scene.d_scene, n, o.as<float>(),
                                                   d.as<float>(), tri.as<int32_t>(), t.as<float>(),
                                                   u.as<float>(), v.as<float>(), err.as<DevErr>());
    HPT_CUDA(cudaGetLastError());
    DevErr e;
    if ((s = tri.down(tri_out)) || (s = t.down(t_out)) || (s = u.down(u_out)) || (s = v.down(v_out)) ||
        (s = err.down(&e)))
      return s;
    if (e.flags & 2u)
      return fail(HPT_ERR_INVALID_SCENE, "device self-check %d failed (value %lld)", e.site,
                  (long long)e.value);
    if (e.flags) return fail(HPT_ERR_TRAVERSAL_LIMIT, "a traversal hit its step cap");
    return HPT_OK;
  });
}

hpt_status hpt_shade(hpt_scene* scene, int32_t n, const float* origins, const float* directions,
                     const float* strengths, const int32_t* tris, const float* ts, uint64_t* seeds,
                     int32_t disable_diffuse, float* contrib, int32_t* branch, float* hit_p,
                     float* normal, float* strength_out, float* param) {
  if (!scene || n < 0 ||
      (n > 0 && (!origins || !directions || !strengths || !tris || !ts || !seeds || !contrib ||
                 !branch || !hit_p || !normal || !strength_out || !param)))
    return fail(HPT_ERR_INVALID_ARGUMENT, "bad shade arguments");
  if (n == 0) return HPT_OK;
  for (int i = 0; i < n; ++i)
    if (tris[i] < 0 || tris[i] >= scene->h.scene.info.num_triangles)
      return fail(HPT_ERR_INVALID_ARGUMENT, "shade: triangle id %d out of range", tris[i]);
  return guarded([&]() -> hpt_status {
    std::lock_guard<std::mutex> lk(scene->h.mu);
    HPT_CUDA(cudaSetDevice(scene->h.scene.device));
    const size_t b3 = (size_t)n * 3 * sizeof(float), b1 = (size_t)n * 4, b8 = (size_t)n * 8;
    DBuf o, d, st, tri, t, sd, co, br, hp, nm, so, pa;
    hpt_status s;
    if ((s = o.up(origins, b3)) || (s = d.up(directions, b3)) || (s = st.up(strengths, b3)) ||
        (s = tri.up(tris, b1)) || (s = t.up(ts, b1)) || (s = sd.up(seeds, b8)) ||
        (s = co.alloc(b3)) || (s = br.alloc(b1)) || (s = hp.alloc(b3)) || (s = nm.alloc(b3)) ||
        (s = so.alloc(b3)) || (s = pa.alloc(b1)))
      return s;
    k_stage_shade<<<blocks_for(n, 128), 128>>>(
        scene->h.scene.d_scene, n, o.as<float>(), d.as<float>(), st.as<float>(), tri.as<int32_t>(),
        t.as<float>(), sd.as<uint64_t>(), disable_diffuse, co.as<float>(), br.as<int32_t>(),
        hp.as<float>(), nm.as<float>(), so.as<float>(), pa.as<float>());
    HPT_CUDA(cudaGetLastError());
    if ((s = sd.down(seeds)) || (s = co.down(contrib)) || (s = br.down(branch)) ||
        (s = hp.down(hit_p)) || (s = nm.down(normal)) || (s = so.down(strength_out)) ||
        (s = pa.down(param)))
      return s;
    return HPT_OK;
  });
}

hpt_status hpt_next_dir(hpt_scene* scene, int32_t n, const int32_t* branch,
                        const float* directions, const float* hit_p, const float* normal,
                        const float* strengths, const float* param, uint64_t* seeds,
                        float* origins_out, float* directions_out, float* strength_out,
                        int32_t* alive_out) {
  if (!scene || n < 0 ||
      (n > 0 && (!branch || !directions || !hit_p || !normal || !strengths || !param || !seeds ||
                 !origins_out || !directions_out || !strength_out || !alive_out)))
    return fail(HPT_ERR_INVALID_ARGUMENT, "bad next_dir arguments");
  if (n == 0) return HPT_OK;
  return guarded([&]() -> hpt_status {
    std::lock_guard<std::mutex> lk(scene->h.mu);
    HPT_CUDA(cudaSetDevice(scene->h.scene.device));
    const size_t b3 = (size_t)n * 3 * sizeof(float), b1 = (size_t)n * 4, b8 = (size_t)n * 8;
    DBuf br, d, hp, nm, st, pa, sd, oo, dd, so, al;
    hpt_status s;
    if ((s = br.up(branch, b1)) || (s = d.up(directions, b3)) || (s = hp.up(hit_p, b3)) ||
        (s = nm.up(normal, b3)) || (s = st.up(strengths, b3)) || (s = pa.up(param, b1)) ||
        (s = sd.up(seeds, b8)) || (s = oo.alloc(b3)) || (s = dd.alloc(b3)) || (s = so.alloc(b3)) ||
        (s = al.alloc(b1)))
      return s;
    k_stage_next<<<blocks_for(n, 128), 128>>>(scene->h.scene.d_scene, n, br.as<int32_t>(),
                                              d.as<float>(), hp.as<float>(), nm.as<float>(),
                                              st.as<float>(), pa.as<float>(), sd.as<uint64_t>(),
                                              oo.as<float>(), dd.as<float>(), so.as<float>(),
                                              al.as<int32_t>());
    HPT_CUDA(cudaGetLastError());
    if ((s = sd.down(seeds)) || (s = oo.down(origins_out)) || (s = dd.down(directions_out)) ||
        (s = so.down(strength_out)) || (s = al.down(alive_out)))
      return s;
    return HPT_OK;
  });
}

hpt_status hpt_compact(const uint32_t* flags, int32_t n, int32_t* out, int32_t* count) {
  if (n < 0 || !count || (n > 0 && (!flags || !out)))
    return fail(HPT_ERR_INVALID_ARGUMENT, "bad compact arguments");
  *count = 0;
  if (n == 0) return HPT_OK;
  if (hpt_device_count() == 0) return fail(HPT_ERR_CUDA, "no CUDA device");
  return guarded([&]() -> hpt_status {
    const int nb = blocks_for(n, kCompactTile);
    const int ns = compact_supers(nb, compact_super_shift(nb));
    DBuf f, o, bc, sc, tot, mk;
    hpt_status s;
    if ((s = f.up(flags, (size_t)n * 4)) || (s = o.alloc((size_t)n * 4)) ||
        (s = bc.alloc((size_t)nb * 4)) || (s = sc.alloc((size_t)ns * 4)) ||
        (s = tot.alloc(4)) || (s = mk.alloc((size_t)nb * kCompactThreads * 2)))
      return s;
    HPT_CUDA(launch_compact(f.as<uint32_t>(), n, bc.as<int>(), sc.as<int>(), mk.as<uint16_t>(),
                            o.as<int>(), tot.as<int>(), 0));
    int total = 0;
    if ((s = tot.down(&total))) return s;
    if (total > 0) HPT_CUDA(cudaMemcpy(out, o.p, (size_t)total * 4, cudaMemcpyDeviceToHost));
    *count = total;
    return HPT_OK;
  });
}

hpt_status hpt_resolve(const float* accum, int32_t sample_x, int32_t sample_y, int32_t supersample_x,
                       int32_t supersample_y, int32_t sample, float brightness, uint8_t* rgba_out) {
  if (!accum || !rgba_out || sample_x <= 0 || sample_y <= 0 || supersample_x <= 0 ||
      supersample_y <= 0 || sample <= 0)
    return fail(HPT_ERR_INVALID_ARGUMENT, "bad resolve arguments");
  if (hpt_device_count() == 0) return fail(HPT_ERR_CUDA, "no CUDA device");
  return guarded([&]() -> hpt_status {
    const size_t rays = (size_t)sample_x * supersample_x * sample_y * supersample_y;
    DBuf a, o;
    hpt_status s;
    if ((s = a.up(accum, rays * 3 * sizeof(float))) || (s = o.alloc((size_t)sample_x * sample_y * 4)))
      return s;
    dim3 blk(16, 16), grd((sample_x + 15) / 16, (sample_y + 15) / 16);
    k_stage_resolve<<<grd, blk>>>(a.as<float>(), sample_x, sample_y, supersample_x, supersample_y,
                                  sample, brightness, o.as<uint8_t>());
    HPT_CUDA(cudaGetLastError());
    return o.down(rgba_out);
  });
}

// --- Batching ---------------------------------------------------------------

struct hpt_batch {
  int device;
  std::unique_ptr<Engine> engine;
  std::vector<JobSpec> jobs;
  hpt_render_stats stats{};
  hpt_tuning tuning = default_tuning();
};

hpt_status hpt_batch_create(int32_t device, hpt_batch** out) {
  if (!out) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  *out = nullptr;
  if (device < 0 || device >= hpt_device_count()) return fail(HPT_ERR_CUDA, "no CUDA device %d", device);
  return guarded([&]() -> hpt_status {
    hpt_batch* b = new hpt_batch();
    b->device = device;
    *out = b;
    return HPT_OK;
  });
}

hpt_status hpt_batch_add(hpt_batch* batch, hpt_scene* scene, const hpt_camera* camera,
                         const hpt_render_params* params, uint8_t* rgba_out, float* accum_out,
                         int32_t* job_id) {
  if (!batch || !scene) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  hpt_status s = check_params(camera, params);
  if (s != HPT_OK) return s;
  if (scene->h.scene.device != batch->device)
    return fail(HPT_ERR_INVALID_ARGUMENT, "scene lives on another device");
  JobSpec js;
  js.scene = &scene->h.scene;
  js.camera = *camera;
  js.params = *params;
  js.rgba_out = rgba_out;
  js.accum_out = accum_out;
  batch->jobs.push_back(js);
  if (job_id) *job_id = (int32_t)batch->jobs.size() - 1;
  return HPT_OK;
}

hpt_status hpt_batch_run(hpt_batch* batch) {
  if (!batch) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  return guarded([&]() -> hpt_status {
    if (!batch->engine) batch->engine.reset(new Engine(batch->device));
    batch->engine->tuning = batch->tuning;
    hpt_status s = batch->engine->run(batch->jobs, &batch->stats);
    batch->jobs.clear();
    return s;
  });
}

hpt_status hpt_batch_stats_get(const hpt_batch* batch, hpt_render_stats* out) {
  if (!batch || !out) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  *out = batch->stats;
  return HPT_OK;
}

hpt_status hpt_batch_tuning_set(hpt_batch* batch, const hpt_tuning* in) {
  if (!batch || !in) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  hpt_status st = check_tuning(*in);
  if (st != HPT_OK) return st;
  batch->tuning = *in;
  batch->tuning.shade_block = 256;
  batch->engine.reset();
  return HPT_OK;
}

void hpt_batch_destroy(hpt_batch* batch) { delete batch; }

}  // extern "C"

// ---------------------------------------------------------------------------
// hpt_compact_noalloc: the compaction kernels over caller-owned device
// buffers, with the per-block counts and the mask bytes in static device
// arrays instead of cudaMalloc'd ones. For callers that cannot allocate device memory where
// they call it (allocation synchronises the device and would stall their
// stream; a fixed memory budget leaves nothing to allocate).
// ---------------------------------------------------------------------------
namespace {

// One count per 4096-flag tile (32 KB per device), one total per
// superblock of at most 128 tiles (8,192 tiles need 64), and 16-bit masks,
// one per 16 flags (4 MiB per device).
constexpr int kNoallocMaxBlocks = HPT_COMPACT_NOALLOC_MAX_N / kCompactTile;
static_assert(kNoallocMaxBlocks * kCompactTile == HPT_COMPACT_NOALLOC_MAX_N,
              "the limit is a whole number of tiles");
constexpr int kNoallocMaxSupers = 128;
static_assert(kNoallocMaxBlocks <= kNoallocMaxSupers * kNoallocMaxSupers,
              "superblocks of at most 128 tiles cover the limit");
static __device__ __align__(256) int g_noalloc_block_counts[kNoallocMaxBlocks];
static __device__ __align__(256) int g_noalloc_super_counts[kNoallocMaxSupers];
static __device__ __align__(256) uint16_t g_noalloc_masks[kNoallocMaxBlocks * kCompactThreads];

struct NoallocScratch {
  int* counts = nullptr;
  int* supers = nullptr;
  uint16_t* masks = nullptr;
};

// Device addresses of the static scratch arrays, looked up once per device
// with that device current (the first call on a device does this set-up).
// The cached addresses belong to the device's current context: after a
// cudaDeviceReset the caller must not use this entry point again in the
// same process.
hpt_status noalloc_scratch(int device, NoallocScratch* out) {
  static std::mutex mu;
  static std::vector<NoallocScratch> addr;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)addr.size() <= device) addr.resize(device + 1);
  if (!addr[device].counts) {
    void* c = nullptr;
    void* sc = nullptr;
    void* m = nullptr;
    HPT_CUDA(cudaGetSymbolAddress(&c, g_noalloc_block_counts));
    HPT_CUDA(cudaGetSymbolAddress(&sc, g_noalloc_super_counts));
    HPT_CUDA(cudaGetSymbolAddress(&m, g_noalloc_masks));
    addr[device].counts = static_cast<int*>(c);
    addr[device].supers = static_cast<int*>(sc);
    addr[device].masks = static_cast<uint16_t*>(m);
  }
  *out = addr[device];
  return HPT_OK;
}

}  // namespace

extern "C" hpt_status hpt_compact_noalloc(const uint32_t* flags, int32_t n, int32_t* out,
                                          int32_t* count, void* stream) {
  if (n < 0 || !count || (n > 0 && (!flags || !out)))
    return fail(HPT_ERR_INVALID_ARGUMENT, "bad compact arguments");
  if (n > HPT_COMPACT_NOALLOC_MAX_N)
    return fail(HPT_ERR_INVALID_ARGUMENT,
                "hpt_compact_noalloc: n = %d exceeds the limit of %d flags (static scratch)", n,
                HPT_COMPACT_NOALLOC_MAX_N);
  int device = 0;
  HPT_CUDA(cudaGetDevice(&device));
  NoallocScratch scratch;
  // The lookup table may grow (host memory): no exception leaves the ABI.
  hpt_status s = guarded([&]() -> hpt_status { return noalloc_scratch(device, &scratch); });
  if (s != HPT_OK) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n == 0) {
    HPT_CUDA(cudaMemsetAsync(count, 0, sizeof(int32_t), st));
    return HPT_OK;
  }
  // Every tile count is written by the count pass before the scatter reads
  // it; the total goes straight to the caller's counter.
  HPT_CUDA(launch_compact(flags, n, scratch.counts, scratch.supers, scratch.masks, out, count,
                          st));
  return HPT_OK;
}
