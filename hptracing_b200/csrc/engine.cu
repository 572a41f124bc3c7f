// Wavefront path-tracing engine for sm_100a.
//
// Reference control flow (src/hp/trace_runner.cpp:116-356): primary rays are
// generated and intersected once per frame (misses write background *
// sample); then, per sample, every primary hit is shaded, branched and
// re-intersected up to `depth` shading passes, with blocking host reads of
// the stage sizes after every stage.
//
// Here the same per-path arithmetic runs as a regenerating wavefront:
//   k_primary  - ray generation + closest hit for every primary ray of every
//                job; hits go to a per-job cache, misses write background.
//   k_shade    - for each pending hit: self-emission, normal / UV / texture,
//                branch choice and next direction (s1_run + s2_*_run fused);
//                new (primary hit, sample) paths are started in the same
//                pass until the wavefront is full. Survivors are compacted
//                (warp ballot + block scan, one atomic per block) into the
//                intersect queue; finished paths flush their radiance.
//   k_isect    - closest hit for the intersect queue with persistent warps
//                that refill idle lanes from the queue (ballot + one atomic
//                per warp); hits are appended to the next shade queue.
//   k_ctrl     - advances the queue counters (device-resident; the host
//                never reads stage sizes).
//   k_resolve  - fixed-point accumulators -> get_image's tone map.
// Every random number is drawn from a stream keyed by (job, ray, sample,
// bounce) and radiance is summed in 2^-32 fixed point, so the image does not
// depend on how paths are scheduled or batched.
#include <algorithm>
#include <cstdio>
#include <cstring>

#include "engine.h"
#include "shading.cuh"
#include "traverse.cuh"

namespace hpt {

namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;

struct EngineParams {
  DevJob* jobs;
  int num_jobs;
  DevCtrl* ctrl;
  float4* A_o[2];
  float4* A_d[2];
  float4* A_s[2];
  float4* A_r[2];
  int32_t* A_tri[2];
  float4* R_o;
  float4* R_d;
  float4* R_s;
  float4* R_r;
  int capacity;
  int smem_nodes;   // > 0 only when every job uses shared_nodes' scene
  int refill;
  const DevNode* shared_nodes;
  int64_t total_primary;
};

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ int find_job_prim(const DevJob* jobs, int n, int64_t g) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].prim_base <= g) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int find_job_path(const DevJob* jobs, int n, int64_t q) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].path_base <= q) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Adds a path's radiance to its ray's fixed-point accumulator. Non-finite
// or out-of-range values set a marker so the resolve reproduces the float
// semantics (NaN stays NaN, +-inf saturates).
__device__ __forceinline__ void flush_radiance(const DevJob& J, int64_t ray, f3 rad) {
  const float v[3] = {rad.x, rad.y, rad.z};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (v[c] == 0.f) continue;
    if (isnan(v[c])) {
      atomicOr(J.flags + ray, 1u << (4 * c));
    } else if (!(fabsf(v[c]) < 1073741824.0f)) {
      atomicOr(J.flags + ray, 1u << (4 * c + (v[c] > 0.f ? 1 : 2)));
    } else {
      long long q = __double2ll_rn((double)v[c] * kAccumScale);
      atomicAdd(J.accum + 3 * ray + c, (unsigned long long)q);
    }
  }
}

// Warp-level reduction of the per-lane query and work counters.
__device__ __forceinline__ void flush_counts(DevCtrl* c, unsigned long long q, TravCount n) {
  for (int o = 16; o > 0; o >>= 1) {
    q += __shfl_down_sync(kFull, q, o);
    n.nodes += __shfl_down_sync(kFull, n.nodes, o);
    n.leaves += __shfl_down_sync(kFull, n.leaves, o);
    n.tris += __shfl_down_sync(kFull, n.tris, o);
  }
  if ((threadIdx.x & 31) == 0 && q) {
    atomicAdd(&c->isect_queries, q);
    atomicAdd(&c->nodes_visited, n.nodes);
    atomicAdd(&c->leaves_visited, n.leaves);
    atomicAdd(&c->tri_tests, n.tris);
  }
}

__device__ __forceinline__ int stage_nodes(const EngineParams& P, uint2* snodes) {
  if (P.smem_nodes <= 0) return 0;
  const uint2* src = reinterpret_cast<const uint2*>(P.shared_nodes);
  for (int i = threadIdx.x; i < P.smem_nodes; i += blockDim.x) snodes[i] = __ldg(src + i);
  __syncthreads();
  return P.smem_nodes;
}

// ---------------------------------------------------------------------------
// Primary pass: raygen + closest hit, lanes refilled from a global counter.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_primary(EngineParams P) {
  extern __shared__ uint2 snodes[];
  const int n_smem = stage_nodes(P, snodes);
  DevCtrl* c = P.ctrl;
  const int lane = threadIdx.x & 31;
  bool active = false;
  TravState st;
  int job = 0;
  int64_t ray = 0;
  unsigned long long queries = 0;
  TravCount cnt;
  while (true) {
    const unsigned idle = __ballot_sync(kFull, !active);
    if (__popc(idle) >= P.refill) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(reinterpret_cast<unsigned long long*>(&c->cursor), (unsigned long long)__popc(idle));
      base = __shfl_sync(kFull, base, 0);
      if (!active) {
        const int64_t g = (int64_t)base + __popc(idle & lanemask_lt());
        if (g < P.total_primary) {
          job = find_job_prim(P.jobs, P.num_jobs, g);
          const DevJob& J = P.jobs[job];
          ray = g - J.prim_base;
          const int x = (int)(ray % J.nx), y = (int)(ray / J.nx);
          const f3 d = J.pano ? pano_dir(x, y, J.vr_x_shift, J.ny)
                              : pinhole_dir(J.top, J.right, J.width, J.height, x, y, J.nx, J.ny);
          Ray r{mk(J.view_p[0], J.view_p[1], J.view_p[2]), d};
          trav_init(J.scene, r, st);
          active = true;
          ++queries;
        }
      }
    }
    if (__ballot_sync(kFull, active) == 0) break;
    bool finished = false;
    if (active) finished = trav_leaf(P.jobs[job].scene, st, snodes, n_smem, &c->error, cnt);
    if (finished) {
      const DevJob& J = P.jobs[job];
      if (st.best.rec >= 0) {
        const int k = atomicAdd(J.prim_count, 1);
        float4* dst = reinterpret_cast<float4*>(J.prim) + 2 * (size_t)k;
        dst[0] = make_float4(st.ray.d.x, st.ray.d.y, st.ray.d.z, __int_as_float((int)ray));
        dst[1] = make_float4(__int_as_float(st.best.tri), st.best.t, 0.f, 0.f);
      } else {
        // kernel.cl:193-206: the first pass assigns background * strength *
        // sample_n with strength (1,1,1).
        const float spp = (float)J.spp;
        const f3 val = scale(spp, mul(mk(J.bg[0], J.bg[1], J.bg[2]), mk(1.f, 1.f, 1.f)));
        flush_radiance(J, ray, val);
      }
      active = false;
    }
  }
  flush_counts(c, queries, cnt);
}

// Sets path ranges after the primary pass (one thread).
__global__ void k_setup(DevJob* jobs, int n, DevCtrl* c) {
  int64_t base = 0;
  for (int j = 0; j < n; ++j) {
    const int64_t np = (int64_t)(*jobs[j].prim_count) * jobs[j].spp;
    jobs[j].path_base = base;
    jobs[j].num_paths = np;
    base += np;
  }
  c->total_paths = base;
  c->cursor = 0;
  c->nA = 0;
  c->nA_next = 0;
  c->nR = 0;
  c->isect_head = 0;
  c->n_new = 0;
  c->parity = 0;
  c->done = base == 0 ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Shade + next direction (+ new paths), compacting survivors into R.
// ---------------------------------------------------------------------------
template <int BS>
__global__ void __launch_bounds__(BS) k_shade(EngineParams P) {
  __shared__ int warp_counts[BS / 32];
  __shared__ int block_base;
  DevCtrl* c = P.ctrl;
  const int par = c->parity;
  const int nA = c->nA;
  const int64_t cursor = c->cursor, total = c->total_paths;
  const int64_t room = (int64_t)P.capacity - nA;
  const int n_new = (int)max((int64_t)0, min(room, total - cursor));
  if (blockIdx.x == 0 && threadIdx.x == 0) c->n_new = n_new;
  const int n_items = nA + n_new;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long shades = 0;
  for (int base = blockIdx.x * BS; base < n_items; base += gridDim.x * BS) {
    const int i = base + threadIdx.x;
    bool alive = false;
    float4 oo, dd, ss, rr;
    if (i < n_items) {
      int job, sample, bounce, tri;
      int64_t ray;
      f3 o, d, strength, rad;
      float t;
      if (i < nA) {
        const float4 ao = P.A_o[par][i], ad = P.A_d[par][i], as = P.A_s[par][i], ar = P.A_r[par][i];
        tri = P.A_tri[par][i];
        o = mk(ao.x, ao.y, ao.z);
        ray = __float_as_int(ao.w);
        d = mk(ad.x, ad.y, ad.z);
        const uint32_t meta = __float_as_uint(ad.w);
        sample = (int)(meta >> 8);
        bounce = (int)(meta & 0xFF);
        strength = mk(as.x, as.y, as.z);
        job = __float_as_int(as.w);
        rad = mk(ar.x, ar.y, ar.z);
        t = ar.w;
      } else {
        const int64_t q = cursor + (i - nA);
        job = find_job_path(P.jobs, P.num_jobs, q);
        const DevJob& J = P.jobs[job];
        const int64_t local = q - J.path_base;
        const int nh = *J.prim_count;
        const int64_t k = local % nh;
        sample = (int)(local / nh);
        bounce = 0;
        const float4* src = reinterpret_cast<const float4*>(J.prim) + 2 * k;
        const float4 p0 = src[0], p1 = src[1];
        o = mk(J.view_p[0], J.view_p[1], J.view_p[2]);
        d = mk(p0.x, p0.y, p0.z);
        ray = __float_as_int(p0.w);
        tri = __float_as_int(p1.x);
        t = p1.y;
        strength = mk(1.f, 1.f, 1.f);
        rad = mk(0.f, 0.f, 0.f);
      }
      const DevJob& J = P.jobs[job];
      uint64_t seed = path_seed(J.seed, (uint32_t)ray, (uint32_t)sample, (uint32_t)bounce);
      const Ray r{o, d};
      const ShadeOut so = shade_hit(J.scene, r, strength, tri, t, J.disable_diffuse, seed);
      ++shades;
      rad = add(rad, so.contrib);
      if (so.branch != kDead && bounce + 1 < J.depth) {
        const NextOut no = next_direction(J.scene, so.branch, d, so.hit_p, so.normal,
                                          so.strength, so.param, seed);
        if (no.alive) {
          alive = true;
          oo = make_float4(no.o.x, no.o.y, no.o.z, __int_as_float((int)ray));
          dd = make_float4(no.d.x, no.d.y, no.d.z,
                           __uint_as_float(((uint32_t)sample << 8) | (uint32_t)(bounce + 1)));
          ss = make_float4(no.strength.x, no.strength.y, no.strength.z, __int_as_float(job));
          rr = make_float4(rad.x, rad.y, rad.z, 0.f);
        }
      }
      if (!alive) flush_radiance(J, ray, rad);
    }
    // Block-level stable compaction: ballot per warp, scan over warps.
    const unsigned m = __ballot_sync(kFull, alive);
    if (lane == 0) warp_counts[warp] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
      int sum = 0;
      for (int w = 0; w < BS / 32; ++w) {
        const int v = warp_counts[w];
        warp_counts[w] = sum;
        sum += v;
      }
      block_base = sum ? atomicAdd(&c->nR, sum) : 0;
    }
    __syncthreads();
    if (alive) {
      const int pos = block_base + warp_counts[warp] + __popc(m & lanemask_lt());
      P.R_o[pos] = oo;
      P.R_d[pos] = dd;
      P.R_s[pos] = ss;
      P.R_r[pos] = rr;
    }
    __syncthreads();
  }
  for (int o = 16; o > 0; o >>= 1) shades += __shfl_down_sync(kFull, shades, o);
  if (lane == 0 && shades) atomicAdd(&c->shades, shades);
}

// ---------------------------------------------------------------------------
// Intersect queue -> next shade queue, persistent warps with lane refill.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_isect(EngineParams P) {
  extern __shared__ uint2 snodes[];
  const int n_smem = stage_nodes(P, snodes);
  DevCtrl* c = P.ctrl;
  const int n = c->nR;
  const int out_par = c->parity ^ 1;
  const int lane = threadIdx.x & 31;
  bool active = false;
  TravState st;
  float4 s4 = make_float4(0, 0, 0, 0), r4 = make_float4(0, 0, 0, 0);
  float ow = 0.f, dw = 0.f;
  int job = 0;
  unsigned long long queries = 0;
  TravCount cnt;
  while (true) {
    const unsigned idle = __ballot_sync(kFull, !active);
    if (__popc(idle) >= P.refill) {
      int base = 0;
      if (lane == 0) base = atomicAdd(&c->isect_head, __popc(idle));
      base = __shfl_sync(kFull, base, 0);
      if (!active) {
        const int i = base + __popc(idle & lanemask_lt());
        if (i < n) {
          const float4 o4 = P.R_o[i], d4 = P.R_d[i];
          s4 = P.R_s[i];
          r4 = P.R_r[i];
          ow = o4.w;
          dw = d4.w;
          job = __float_as_int(s4.w);
          trav_init(P.jobs[job].scene, Ray{mk(o4.x, o4.y, o4.z), mk(d4.x, d4.y, d4.z)}, st);
          active = true;
          ++queries;
        }
      }
    }
    if (__ballot_sync(kFull, active) == 0) break;
    bool finished = false;
    if (active) finished = trav_leaf(P.jobs[job].scene, st, snodes, n_smem, &c->error, cnt);
    const bool hit = finished && st.best.rec >= 0;
    const unsigned hm = __ballot_sync(kFull, hit);
    if (hm) {
      const int leader = __ffs(hm) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(&c->nA_next, __popc(hm));
      base = __shfl_sync(kFull, base, leader);
      if (hit) {
        const int pos = base + __popc(hm & lanemask_lt());
        P.A_o[out_par][pos] = make_float4(st.ray.o.x, st.ray.o.y, st.ray.o.z, ow);
        P.A_d[out_par][pos] = make_float4(st.ray.d.x, st.ray.d.y, st.ray.d.z, dw);
        P.A_s[out_par][pos] = s4;
        P.A_r[out_par][pos] = make_float4(r4.x, r4.y, r4.z, st.best.t);
        P.A_tri[out_par][pos] = st.best.tri;
      }
    }
    if (finished && !hit) {
      // kernel.cl:195-200: miss adds background * strength (sample_n = 1).
      const DevJob& J = P.jobs[job];
      f3 rad = mk(r4.x, r4.y, r4.z);
      rad = add(rad, mul(mk(J.bg[0], J.bg[1], J.bg[2]), mk(s4.x, s4.y, s4.z)));
      flush_radiance(J, __float_as_int(ow), rad);
    }
    if (finished) active = false;
  }
  flush_counts(c, queries, cnt);
}

__global__ void k_ctrl(DevCtrl* c) {
  c->nA = c->nA_next;
  c->nA_next = 0;
  c->nR = 0;
  c->isect_head = 0;
  c->cursor += c->n_new;
  c->n_new = 0;
  c->parity ^= 1;
  c->iterations += 1;
  c->done = (c->nA == 0 && c->cursor >= c->total_paths) ? 1 : 0;
}

__device__ __forceinline__ float ray_value(const unsigned long long* acc, const uint32_t* flags,
                                           int64_t ray, int ch) {
  const uint32_t f = (flags[ray] >> (4 * ch)) & 0xF;
  if (f & 1u) return __int_as_float(0x7fc00000);
  if ((f & 6u) == 6u) return __int_as_float(0x7fc00000);
  if (f & 2u) return __int_as_float(0x7f800000);
  if (f & 4u) return __int_as_float(0xff800000);
  const long long v = (long long)acc[3 * ray + ch];
  return __double2float_rn(__ll2double_rn(v) * (1.0 / kAccumScale));
}

// write_imagef to an RGBA UNORM_INT8 image: convert_uchar_sat_rte(x * 255).
__device__ __forceinline__ uint8_t to_unorm8(float x) {
  const float v = __fmul_rn(x, 255.0f);
  if (!(v >= 0.f)) return 0;
  if (v >= 255.f) return 255;
  return (uint8_t)__float2int_rn(v);
}

// get_image (kernel.cl:615-652) from the fixed-point accumulators.
__global__ void k_resolve(const DevJob* jp, int W, int H, int ssx, int ssy, float brightness,
                          uint8_t* rgba, float* accum_f) {
  const int gx = blockIdx.x * blockDim.x + threadIdx.x;
  const int gy = blockIdx.y * blockDim.y + threadIdx.y;
  if (gx >= W || gy >= H) return;
  const DevJob& J = *jp;
  float px = 0.f, py = 0.f, pz = 0.f;
  for (int i = 0; i < ssx; ++i)
    for (int j = 0; j < ssy; ++j) {
      const int row = gy * ssy + j, col = gx * ssx + i;
      const int64_t idx = (int64_t)row * W * ssx + col;
      const float vx = ray_value(J.accum, J.flags, idx, 0);
      const float vy = ray_value(J.accum, J.flags, idx, 1);
      const float vz = ray_value(J.accum, J.flags, idx, 2);
      if (accum_f) {
        accum_f[3 * idx] = vx;
        accum_f[3 * idx + 1] = vy;
        accum_f[3 * idx + 2] = vz;
      }
      px = __fadd_rn(px, vx);
      py = __fadd_rn(py, vy);
      pz = __fadd_rn(pz, vz);
    }
  const float nss = (float)(ssx * ssy), ns = (float)J.spp;
  px = __fmul_rn(__fdiv_rn(__fdiv_rn(px, nss), ns), brightness);
  py = __fmul_rn(__fdiv_rn(__fdiv_rn(py, nss), ns), brightness);
  pz = __fmul_rn(__fdiv_rn(__fdiv_rn(pz, nss), ns), brightness);
  uint8_t* o = rgba + 4 * ((int64_t)gy * W + gx);
  o[0] = to_unorm8(__fsub_rn(1.f, expf(-px)));
  o[1] = to_unorm8(__fsub_rn(1.f, expf(-py)));
  o[2] = to_unorm8(__fsub_rn(1.f, expf(-pz)));
  o[3] = 0;
}

}  // namespace

// ===========================================================================
// Host side
// ===========================================================================

hpt_status cuda_fail(cudaError_t e, const char* what) {
  return fail(e == cudaErrorMemoryAllocation ? HPT_ERR_OUT_OF_MEMORY : HPT_ERR_CUDA, "%s: %s",
              what, cudaGetErrorString(e));
}

hpt_tuning default_tuning() {
  hpt_tuning t;
  memset(&t, 0, sizeof t);
  t.capacity = 1 << 21;
  t.isect_block = 256;
  t.shade_block = 256;
  t.refill_chunk = 16;
  t.smem_nodes = 2048;
  t.use_graph = 0;
  return t;
}

Engine::Engine(int dev) : device(dev) {
  tuning = default_tuning();
  cudaSetDevice(device);
  cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
  cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device);
  cudaMalloc(&ctrl_, sizeof(DevCtrl));
  cudaMallocHost(&ctrl_host_, sizeof(DevCtrl));
  for (auto& e : ev_) cudaEventCreate(&e);
}

Engine::~Engine() {
  cudaSetDevice(device);
  if (stream) cudaStreamSynchronize(stream);
  for (int p = 0; p < 2; ++p) {
    cudaFree(A_o_[p]); cudaFree(A_d_[p]); cudaFree(A_s_[p]); cudaFree(A_r_[p]); cudaFree(A_tri_[p]);
  }
  cudaFree(R_o_); cudaFree(R_d_); cudaFree(R_s_); cudaFree(R_r_);
  cudaFree(ctrl_);
  cudaFree(jobs_);
  cudaFreeHost(ctrl_host_);
  for (auto& e : ev_) cudaEventDestroy(e);
  if (stream) cudaStreamDestroy(stream);
}

hpt_status Engine::ensure_capacity(int capacity) {
  if (capacity <= capacity_) return HPT_OK;
  cudaStreamSynchronize(stream);
  for (int p = 0; p < 2; ++p) {
    cudaFree(A_o_[p]); cudaFree(A_d_[p]); cudaFree(A_s_[p]); cudaFree(A_r_[p]); cudaFree(A_tri_[p]);
    A_o_[p] = A_d_[p] = A_s_[p] = A_r_[p] = nullptr;
    A_tri_[p] = nullptr;
  }
  cudaFree(R_o_); cudaFree(R_d_); cudaFree(R_s_); cudaFree(R_r_);
  R_o_ = R_d_ = R_s_ = R_r_ = nullptr;
  capacity_ = 0;
  const size_t n = (size_t)capacity;
  for (int p = 0; p < 2; ++p) {
    HPT_CUDA(cudaMalloc(&A_o_[p], n * sizeof(float4)));
    HPT_CUDA(cudaMalloc(&A_d_[p], n * sizeof(float4)));
    HPT_CUDA(cudaMalloc(&A_s_[p], n * sizeof(float4)));
    HPT_CUDA(cudaMalloc(&A_r_[p], n * sizeof(float4)));
    HPT_CUDA(cudaMalloc(&A_tri_[p], n * sizeof(int32_t)));
  }
  HPT_CUDA(cudaMalloc(&R_o_, n * sizeof(float4)));
  HPT_CUDA(cudaMalloc(&R_d_, n * sizeof(float4)));
  HPT_CUDA(cudaMalloc(&R_s_, n * sizeof(float4)));
  HPT_CUDA(cudaMalloc(&R_r_, n * sizeof(float4)));
  capacity_ = capacity;
  return HPT_OK;
}

void Engine::query_occupancy() {
  if (occ_done_) return;
  const size_t smem = (size_t)std::max(0, tuning.smem_nodes) * sizeof(uint2);
  int b = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_isect, 256, smem);
  occ_isect_ = std::max(1, b);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_shade<256>, 256, 0);
  occ_shade_ = std::max(1, b);
  occ_done_ = true;
}

hpt_status Engine::alloc_job(const JobSpec& js, bool want_accum, JobBuffers& b) {
  const hpt_render_params& p = js.params;
  const int64_t nx = (int64_t)p.sample_x * p.supersample_x, ny = (int64_t)p.sample_y * p.supersample_y;
  b.rays = nx * ny;
  HPT_CUDA(cudaMallocAsync(&b.accum, (size_t)b.rays * 3 * sizeof(unsigned long long), stream));
  HPT_CUDA(cudaMallocAsync(&b.flags, (size_t)b.rays * sizeof(uint32_t), stream));
  HPT_CUDA(cudaMallocAsync(&b.prim, (size_t)b.rays * 8 * sizeof(float), stream));
  HPT_CUDA(cudaMallocAsync(&b.prim_count, sizeof(int32_t), stream));
  HPT_CUDA(cudaMallocAsync(&b.counters, 4 * sizeof(unsigned long long), stream));
  HPT_CUDA(cudaMallocAsync(&b.rgba, (size_t)p.sample_x * p.sample_y * 4, stream));
  if (want_accum) HPT_CUDA(cudaMallocAsync(&b.accum_f, (size_t)b.rays * 3 * sizeof(float), stream));
  HPT_CUDA(cudaMemsetAsync(b.accum, 0, (size_t)b.rays * 3 * sizeof(unsigned long long), stream));
  HPT_CUDA(cudaMemsetAsync(b.flags, 0, (size_t)b.rays * sizeof(uint32_t), stream));
  HPT_CUDA(cudaMemsetAsync(b.prim_count, 0, sizeof(int32_t), stream));
  HPT_CUDA(cudaMemsetAsync(b.counters, 0, 4 * sizeof(unsigned long long), stream));
  b.bytes = b.rays * (24 + 4 + 32 + (want_accum ? 12 : 0)) + (int64_t)p.sample_x * p.sample_y * 4;
  return HPT_OK;
}

void Engine::free_job(JobBuffers& b) {
  cudaFreeAsync(b.accum, stream);
  cudaFreeAsync(b.flags, stream);
  cudaFreeAsync(b.prim, stream);
  cudaFreeAsync(b.prim_count, stream);
  cudaFreeAsync(b.counters, stream);
  cudaFreeAsync(b.rgba, stream);
  if (b.accum_f) cudaFreeAsync(b.accum_f, stream);
  b = JobBuffers();
}

DevJob Engine::make_job(const JobSpec& js, const JobBuffers& b, int64_t prim_base) const {
  DevJob j;
  memset(&j, 0, sizeof j);
  const hpt_camera& cam = js.camera;
  const hpt_render_params& p = js.params;
  j.scene = js.scene->dev;
  for (int k = 0; k < 3; ++k) {
    j.view_p[k] = cam.view_p[k];
    j.top[k] = cam.top_dir[k];
    j.right[k] = cam.right_dir[k];
    j.bg[k] = p.background[k];
  }
  j.width = cam.width;
  j.height = cam.height;
  j.nx = p.sample_x * p.supersample_x;
  j.ny = p.sample_y * p.supersample_y;
  j.pano = cam.height < 0 ? 1 : 0;
  // trace_runner.cpp:131-140: shift = int(right_dir.x), times supersample_x.
  j.vr_x_shift = (int)cam.right_dir[0] * p.supersample_x;
  j.vr_sample_x = p.sample_x * p.supersample_y;
  j.vr_sample_y = p.sample_y * p.supersample_y;
  j.spp = p.sample;
  j.depth = p.depth;
  j.disable_diffuse = p.disable_diffuse;
  j.seed = p.seed;
  j.accum = b.accum;
  j.flags = b.flags;
  j.prim = b.prim;
  j.prim_count = b.prim_count;
  j.prim_base = prim_base;
  j.counters = b.counters;
  return j;
}

hpt_status Engine::upload_jobs(const std::vector<DevJob>& jobs) {
  if ((int)jobs.size() > jobs_cap_) {
    cudaStreamSynchronize(stream);
    cudaFree(jobs_);
    jobs_ = nullptr;
    jobs_cap_ = 0;
    HPT_CUDA(cudaMalloc(&jobs_, jobs.size() * sizeof(DevJob)));
    jobs_cap_ = (int)jobs.size();
  }
  HPT_CUDA(cudaMemcpyAsync(jobs_, jobs.data(), jobs.size() * sizeof(DevJob), cudaMemcpyHostToDevice,
                           stream));
  num_jobs_ = (int)jobs.size();
  return HPT_OK;
}

static EngineParams make_params(Engine& e, DevCtrl* ctrl, DevJob* jobs, int num_jobs, int capacity,
                                float4* const* A, int32_t* const* Atri, float4* const* R,
                                const DevScene* shared, int64_t total_primary) {
  EngineParams P;
  memset(&P, 0, sizeof P);
  P.jobs = jobs;
  P.num_jobs = num_jobs;
  P.ctrl = ctrl;
  for (int p = 0; p < 2; ++p) {
    P.A_o[p] = A[4 * p + 0];
    P.A_d[p] = A[4 * p + 1];
    P.A_s[p] = A[4 * p + 2];
    P.A_r[p] = A[4 * p + 3];
    P.A_tri[p] = Atri[p];
  }
  P.R_o = R[0];
  P.R_d = R[1];
  P.R_s = R[2];
  P.R_r = R[3];
  P.capacity = capacity;
  P.refill = std::max(1, std::min(32, e.tuning.refill_chunk));
  if (shared && e.tuning.smem_nodes > 0) {
    P.smem_nodes = std::min(e.tuning.smem_nodes, shared->num_nodes);
    P.shared_nodes = shared->nodes;
  }
  P.total_primary = total_primary;
  return P;
}

void Engine::launch_primary(int64_t total_primary, const DevScene* shared_scene) {
  query_occupancy();
  float4* A[8] = {A_o_[0], A_d_[0], A_s_[0], A_r_[0], A_o_[1], A_d_[1], A_s_[1], A_r_[1]};
  float4* R[4] = {R_o_, R_d_, R_s_, R_r_};
  EngineParams P = make_params(*this, ctrl_, jobs_, num_jobs_, capacity_, A, A_tri_, R,
                               shared_scene, total_primary);
  const size_t smem = (size_t)P.smem_nodes * sizeof(uint2);
  k_primary<<<num_sms * occ_isect_, 256, smem, stream>>>(P);
}

void Engine::launch_setup(int num_jobs, bool) {
  k_setup<<<1, 1, 0, stream>>>(jobs_, num_jobs, ctrl_);
}

void Engine::launch_iteration(const DevScene* shared_scene, cudaEvent_t* ev) {
  query_occupancy();
  float4* A[8] = {A_o_[0], A_d_[0], A_s_[0], A_r_[0], A_o_[1], A_d_[1], A_s_[1], A_r_[1]};
  float4* R[4] = {R_o_, R_d_, R_s_, R_r_};
  EngineParams P = make_params(*this, ctrl_, jobs_, num_jobs_, capacity_, A, A_tri_, R,
                               shared_scene, 0);
  if (ev) cudaEventRecord(ev[0], stream);
  k_shade<256><<<num_sms * occ_shade_, 256, 0, stream>>>(P);
  if (ev) cudaEventRecord(ev[1], stream);
  const size_t smem = (size_t)P.smem_nodes * sizeof(uint2);
  k_isect<<<num_sms * occ_isect_, 256, smem, stream>>>(P);
  if (ev) cudaEventRecord(ev[2], stream);
  k_ctrl<<<1, 1, 0, stream>>>(ctrl_);
}

hpt_status Engine::run(const std::vector<JobSpec>& jobs, hpt_render_stats* stats) {
  HPT_CUDA(cudaSetDevice(device));
  if (jobs.empty()) return HPT_OK;
  hpt_status s = ensure_capacity(std::max(1024, tuning.capacity));
  if (s != HPT_OK) return s;
  {  // smem staging must fit in the opt-in shared memory limit
    const size_t smem = (size_t)std::max(0, tuning.smem_nodes) * sizeof(uint2);
    cudaFuncSetAttribute(k_primary, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_isect, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  }
  std::vector<JobBuffers> bufs(jobs.size());
  std::vector<DevJob> djobs;
  int64_t prim_base = 0;
  const SceneDev* shared = jobs[0].scene;
  for (size_t j = 0; j < jobs.size(); ++j) {
    s = alloc_job(jobs[j], jobs[j].accum_out != nullptr, bufs[j]);
    if (s != HPT_OK) {
      for (size_t k = 0; k <= j; ++k) free_job(bufs[k]);
      return s;
    }
    djobs.push_back(make_job(jobs[j], bufs[j], prim_base));
    prim_base += bufs[j].rays;
    if (jobs[j].scene != shared) shared = nullptr;
  }
  s = upload_jobs(djobs);
  if (s != HPT_OK) return s;
  HPT_CUDA(cudaMemsetAsync(ctrl_, 0, sizeof(DevCtrl), stream));
  const DevScene* shared_dev = shared ? &shared->dev : nullptr;

  cudaEventRecord(ev_[0], stream);
  launch_primary(prim_base, shared_dev);
  cudaEventRecord(ev_[1], stream);
  launch_setup((int)jobs.size(), true);
  // Iterate until the device says the wavefront is drained. Batches of
  // iterations are queued ahead; the done flag of batch k is checked while
  // batch k+1 runs (extra iterations after completion are empty launches).
  const int kBatch = 4;
  const bool prof = tuning.profile != 0;
  int32_t* done_host = nullptr;
  HPT_CUDA(cudaMallocHost(&done_host, 2 * sizeof(int32_t)));
  done_host[0] = done_host[1] = 0;
  cudaEvent_t ev_done[2];
  cudaEventCreateWithFlags(&ev_done[0], cudaEventDisableTiming);
  cudaEventCreateWithFlags(&ev_done[1], cudaEventDisableTiming);
  // Profile mode: three events per iteration, two batches in flight.
  std::vector<cudaEvent_t> pev;
  if (prof) {
    pev.resize(2 * kBatch * 3);
    for (auto& e : pev) cudaEventCreate(&e);
  }
  float ms_shade = 0.f, ms_isect = 0.f;
  auto harvest = [&](int sl) {
    for (int k = 0; k < kBatch; ++k) {
      cudaEvent_t* e = &pev[(sl * kBatch + k) * 3];
      float a = 0.f, b = 0.f;
      cudaEventElapsedTime(&a, e[0], e[1]);
      cudaEventElapsedTime(&b, e[1], e[2]);
      ms_shade += a;
      ms_isect += b;
    }
  };
  // Upper bound on iterations: every live path advances one bounce per
  // iteration, so the wavefront drains within paths * depth / capacity
  // iterations plus one path lifetime; 2x that plus slack is the cap.
  int64_t work = 0;
  int max_depth = 1;
  for (const JobSpec& js : jobs) {
    const hpt_render_params& p = js.params;
    work += (int64_t)p.sample_x * p.supersample_x * p.sample_y * p.supersample_y * p.sample *
            p.depth;
    max_depth = std::max(max_depth, p.depth);
  }
  const int64_t max_batches = (2 * (work / std::max(1, capacity_) + max_depth) + 64) / kBatch + 4;
  int64_t guard = 0;
  bool drained = false;
  int slot = 0;
  bool pending = false;
  while (true) {
    for (int k = 0; k < kBatch; ++k)
      launch_iteration(shared_dev, prof ? &pev[(slot * kBatch + k) * 3] : nullptr);
    cudaMemcpyAsync(&done_host[slot], &ctrl_->done, sizeof(int32_t), cudaMemcpyDeviceToHost, stream);
    cudaEventRecord(ev_done[slot], stream);
    if (pending) {
      cudaEventSynchronize(ev_done[slot ^ 1]);
      if (prof) harvest(slot ^ 1);
      if (done_host[slot ^ 1]) {
        drained = true;
        break;
      }
    }
    pending = true;
    slot ^= 1;
    if (++guard > max_batches) break;
  }
  cudaEventRecord(ev_[2], stream);
  for (size_t j = 0; j < jobs.size(); ++j) {
    const hpt_render_params& p = jobs[j].params;
    dim3 blk(16, 16), grd((p.sample_x + 15) / 16, (p.sample_y + 15) / 16);
    k_resolve<<<grd, blk, 0, stream>>>(jobs_ + j, p.sample_x, p.sample_y, p.supersample_x,
                                        p.supersample_y, p.brightness, bufs[j].rgba,
                                        bufs[j].accum_f);
  }
  cudaEventRecord(ev_[3], stream);
  for (size_t j = 0; j < jobs.size(); ++j) {
    const hpt_render_params& p = jobs[j].params;
    if (jobs[j].rgba_out)
      cudaMemcpyAsync(jobs[j].rgba_out, bufs[j].rgba, (size_t)p.sample_x * p.sample_y * 4,
                      cudaMemcpyDeviceToHost, stream);
    if (jobs[j].accum_out)
      cudaMemcpyAsync(jobs[j].accum_out, bufs[j].accum_f, (size_t)bufs[j].rays * 3 * sizeof(float),
                      cudaMemcpyDeviceToHost, stream);
  }
  cudaMemcpyAsync(ctrl_host_, ctrl_, sizeof(DevCtrl), cudaMemcpyDeviceToHost, stream);
  for (auto& b : bufs) free_job(b);
  cudaError_t e = cudaStreamSynchronize(stream);
  if (prof) harvest(slot);
  for (auto& ev : pev) cudaEventDestroy(ev);
  cudaEventDestroy(ev_done[0]);
  cudaEventDestroy(ev_done[1]);
  cudaFreeHost(done_host);
  if (e != cudaSuccess) return cuda_fail(e, "render");
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "render launch");
  if (stats) {
    memset(stats, 0, sizeof *stats);
    stats->primary_rays = prim_base;
    stats->intersect_queries = (int64_t)ctrl_host_->isect_queries;
    stats->shade_calls = (int64_t)ctrl_host_->shades;
    stats->paths = ctrl_host_->total_paths;
    stats->iterations = (int32_t)ctrl_host_->iterations;
    stats->error_flags = (int32_t)ctrl_host_->error;
    cudaEventElapsedTime(&stats->ms_total, ev_[0], ev_[3]);
    cudaEventElapsedTime(&stats->ms_primary, ev_[0], ev_[1]);
    cudaEventElapsedTime(&stats->ms_loop, ev_[1], ev_[2]);
    stats->ms_shade = prof ? ms_shade : -1.f;
    stats->ms_intersect = prof ? ms_isect : -1.f;
    cudaEventElapsedTime(&stats->ms_resolve, ev_[2], ev_[3]);
    stats->nodes_visited = (int64_t)ctrl_host_->nodes_visited;
    stats->leaves_visited = (int64_t)ctrl_host_->leaves_visited;
    stats->triangle_tests = (int64_t)ctrl_host_->tri_tests;
  }
  if (ctrl_host_->error) return fail(HPT_ERR_TRAVERSAL_LIMIT, "a traversal hit its step cap");
  if (!drained && !ctrl_host_->done)
    return fail(HPT_ERR_TRAVERSAL_LIMIT, "the wavefront did not drain within %lld iterations",
                (long long)(max_batches * kBatch));
  return HPT_OK;
}

// ---------------------------------------------------------------------------
// Scene upload
// ---------------------------------------------------------------------------
}  // namespace hpt
