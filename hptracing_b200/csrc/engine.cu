// Wavefront path-tracing engine for sm_100a.
//
// Reference control flow (src/hp/trace_runner.cpp:116-356): primary rays are
// generated and intersected once per frame (misses write background *
// sample); then, per sample, every primary hit is shaded, branched and
// re-intersected up to `depth` shading passes, with blocking host reads of
// the stage sizes after every stage.
//
// Here the same per-path arithmetic runs as a regenerating wavefront over
// job slots (one job = one frame of one scene):
//   k_primary  - ray generation + closest hit for the primary rays of newly
//                admitted jobs; hits go to a per-job cache, misses write
//                background * sample.
//   k_admit    - sets each new job's path count and grants paths.
//   k_shade    - for each pending hit: self-emission, normal / UV / texture,
//                branch choice and next direction (s1_run + s2_*_run fused);
//                new (primary hit, sample) paths are started in the same
//                pass from the grants. Survivors are compacted (warp ballot
//                + block scan, one atomic per block) into the intersect
//                queue; finished paths flush their radiance.
//   k_isect    - closest hit for the intersect queue with persistent warps
//                that refill idle lanes from the queue (ballot + one atomic
//                per warp); hits are appended to the next shade queue.
//   k_ctrl     - advances queue counters and path cursors and grants the
//                free wavefront capacity to the active jobs in priority
//                order (the host never reads stage sizes).
//   k_resolve  - fixed-point accumulators -> get_image's tone map.
// Every random number is drawn from a stream keyed by (job, ray, sample,
// bounce) and radiance is summed in 2^-32 fixed point, so a job's image does
// not depend on how its paths are scheduled, batched or interleaved.
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <type_traits>

#include "engine.h"
#include "shading.cuh"
#include "traverse.cuh"

namespace hpt {

namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;

struct EngineParams {
  DevJob* jobs;
  DevSlot* slots;
  int num_slots;
  DevCtrl* ctrl;
  const int32_t* order;
  int32_t* quota_slot;
  int32_t* quota_prefix;
  const int32_t* prim_slot;
  const int64_t* prim_prefix;
  // Primary passes over part of a job's rays (null: every entry covers its
  // job from ray 0 and completes its primary pass): entry e covers rays
  // [prim_first[e], prim_first[e] + its count); prim_final[e] != 0 marks
  // the part that completes the job's primary pass.
  const int64_t* prim_first;
  const int32_t* prim_final;
  int prim_n;
  float4* A_o[2];
  float4* A_d[2];
  float4* A_s[2];
  float4* A_r[2];
  int32_t* A_tri[2];
  int32_t* A_leaf[2];   // leaf node of the hit (start hint for the next ray)
  float4* R_o;
  float4* R_d;
  float4* R_s;
  float4* R_r;
  int capacity;
  int smem_nodes;       // > 0 only when every job uses shared_nodes' scene
  int refill;
  int trav_steps;       // > 0: step-at-a-time traversal, units per round
  const DevNode* shared_nodes;
  // When every job of the launch renders the same scene (a frame, or a
  // batch over one scene): a copy of its DevScene in the kernel's parameter
  // space. The step loop then reads the scene's pointers and sizes as
  // constant operands instead of loading them from the job table on every
  // traversal unit (one dependent load less per unit).
  int uniform_scene;
  DevScene uscene;
  // Several scenes, and their per-slot TravScene table fits the dynamic
  // shared memory: the traversal reads its scene from there.
  int scene_table;
};

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Index of the last prefix entry <= g (prefix[0] = 0, n entries).
template <typename T>
__device__ __forceinline__ int find_prefix(const T* prefix, int n, int64_t g) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if ((int64_t)prefix[mid] <= g) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int64_t job_rays(const DevJob& J) { return (int64_t)J.nx * J.ny; }

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
      const long long q = __double2ll_rn((double)v[c] * kAccumScale);
      atomicAdd(J.accum + 3 * ray + c, (unsigned long long)q);
    }
  }
}

// Counts finished paths per slot with one atomic per (warp, slot).
__device__ __forceinline__ void count_done(DevSlot* slots, bool done, int slot) {
  const unsigned m = __ballot_sync(kFull, done);
  if (!m) return;
  const unsigned same = __match_any_sync(kFull, done ? slot : -1);
  if (done && (__ffs(same & m) - 1) == (int)(threadIdx.x & 31))
    atomicAdd(&slots[slot].done, (unsigned long long)__popc(same & m));
}

// Counts the paths each slot sends to the intersect queue (one atomic per
// (warp, slot)).
__device__ __forceinline__ void count_queries(DevSlot* slots, bool alive, int slot) {
  const unsigned m = __ballot_sync(kFull, alive);
  if (!m) return;
  const unsigned same = __match_any_sync(kFull, alive ? slot : -1);
  if (alive && (__ffs(same & m) - 1) == (int)(threadIdx.x & 31))
    atomicAdd(&slots[slot].queries, (unsigned long long)__popc(same & m));
}

// A lane's work counters in shared memory (five words: an odd stride, so
// the lanes of a warp hit distinct banks); they are touched once per
// traversal unit and would otherwise hold four registers.
struct CountSlot {
  TravCount c;
  uint32_t queries;  // the lane's queries in this launch
};

// Warp-level reduction of the per-lane query and work counters.
__device__ __forceinline__ void flush_counts(DevCtrl* c, unsigned long long q, TravCount lane) {
  unsigned long long nodes = lane.nodes, leaves = lane.leaves, tris = lane.tris,
                     repeats = lane.repeats;
  for (int o = 16; o > 0; o >>= 1) {
    q += __shfl_down_sync(kFull, q, o);
    nodes += __shfl_down_sync(kFull, nodes, o);
    leaves += __shfl_down_sync(kFull, leaves, o);
    tris += __shfl_down_sync(kFull, tris, o);
    repeats += __shfl_down_sync(kFull, repeats, o);
  }
  if ((threadIdx.x & 31) == 0 && q) {
#ifdef HPT_DEVICE_CHECKS
    atomicAdd(&c->chk_isect_done, (int)q);
#endif
    atomicAdd(&c->isect_queries, q);
    atomicAdd(&c->nodes_visited, nodes);
    atomicAdd(&c->leaves_visited, leaves);
    atomicAdd(&c->tri_tests, tris);
    atomicAdd(&c->tri_repeats, repeats);
  }
}

__device__ __forceinline__ int stage_nodes(const EngineParams& P, uint2* snodes) {
  if (P.smem_nodes <= 0) return 0;
  const uint2* src = reinterpret_cast<const uint2*>(P.shared_nodes);
  for (int i = threadIdx.x; i < P.smem_nodes; i += blockDim.x) snodes[i] = __ldg(src + i);
  __syncthreads();
  return P.smem_nodes;
}

// A launch over several scenes copies each job slot's TravScene into the
// dynamic shared memory (the node prefix is only used by one-scene
// launches, so the table starts at offset 0): the traversal steps then read
// their scene's pointers and sizes from shared memory.
__device__ __forceinline__ const TravScene* stage_scenes(const EngineParams& P, uint2* smem) {
  if (!P.scene_table) return nullptr;
  TravScene* tab = reinterpret_cast<TravScene*>(smem);
  for (int i = threadIdx.x; i < P.num_slots; i += blockDim.x) tab[i] = trav_scene(P.jobs[i].scene);
  __syncthreads();
  return tab;
}

// Grants the free wavefront capacity to active slots in priority order
// (one thread). A slot with nothing left to issue no longer needs grants.
__device__ void schedule(const EngineParams& P) {
  DevCtrl* c = P.ctrl;
  const int budget = P.capacity - c->nA;
  int n_new = 0, nq = 0;
  bool remaining = false;
  // Paths the capped slots hold now, against their shared budget.
  int64_t capped = 0;
  if (c->capped_budget > 0)
    for (int k = 0; k < c->n_order; ++k) {
      const int s = P.order[k];
      if (s < 0 || s >= P.num_slots) continue;
      const DevSlot& S = P.slots[s];
      if (S.active && S.max_inflight > 0) capped += S.cursor - (int64_t)S.done;
    }
  for (int k = 0; k < c->n_order; ++k) {
    const int s = P.order[k];
    HPT_DCHECK(&c->err, s >= 0 && s < P.num_slots, 231, s, continue);
    DevSlot& S = P.slots[s];
    S.alloc = 0;
    if (!S.active) continue;
    const int64_t rem = S.num_paths - S.cursor;
    if (rem <= 0) continue;
    remaining = true;
    int64_t grant = min(rem, (int64_t)(budget - n_new));
    // A capped job (e.g. a large request that must not crowd out the
    // latency-sensitive ones behind it) keeps at most max_inflight paths
    // started and unfinished.
    if (S.max_inflight > 0) {
      grant = min(grant, S.max_inflight - (S.cursor - (int64_t)S.done));
      if (c->capped_budget > 0) grant = min(grant, c->capped_budget - capped);
    }
    const int a = (int)grant;
    if (a <= 0) continue;
    if (S.max_inflight > 0) capped += a;
    S.alloc = a;
    P.quota_slot[nq] = s;
    P.quota_prefix[nq] = n_new;
    n_new += a;
    ++nq;
  }
  P.quota_prefix[nq] = n_new;
  c->n_quota = nq;
  c->n_new = n_new;
  c->done = (c->nA == 0 && !remaining) ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Primary pass: raygen + closest hit, lanes refilled from a global counter.
// Traversal modes of k_primary / k_isect.
constexpr int kTravLeaf = 0;      // trav_leaf, one leaf per lane per round
constexpr int kTravStep = 1;      // trav_step, nodes from global memory
constexpr int kTravStepSmem = 2;  // trav_step with the shared-memory node prefix

// Phase vote (default; -DHPT_PHASE_VOTE=0 builds the per-lane loop for
// comparison): in each warp round of the step-at-a-time walk only the lanes
// of the more common phase (descent / leaf set-up, or triangle test) run a
// unit, so that a round executes one phase's code instead of both. Measured
// on the spheres frame 107.9 -> 105.7 ms and on the terrain frame 85.1 ->
// 79.0 ms per frame (4 spp), images unchanged (each lane still runs its own
// units in order).
#ifndef HPT_PHASE_VOTE
#define HPT_PHASE_VOTE 1
#endif
// The tests' phase runs when it holds at least this many sixths of the
// warp's live lanes: with one test per testing lane a round (3, the
// majority), and with cooperative tests (1; a cooperative round tests up to
// 32 references whatever the number of testing lanes).
#ifndef HPT_VOTE_TEST_SIXTHS
#define HPT_VOTE_TEST_SIXTHS 3
#endif
#ifndef HPT_COOP_TEST_SIXTHS
#define HPT_COOP_TEST_SIXTHS 1
#endif

// k_primary tests one reference per testing lane a round unless built with
// -DHPT_COOP_PRIMARY=1: camera rays are coherent, neighbouring lanes test
// the same triangles and share their loads, and the terrain frame's
// primary pass measured 9.6 ms with per-lane tests against 11.3 ms with
// cooperative ones (the spheres frame's 1.16 against 0.87 ms).
#ifndef HPT_COOP_PRIMARY
#define HPT_COOP_PRIMARY 0
#endif
constexpr bool kCoopPrimary = HPT_COOP_PRIMARY != 0;

// Scene accessors of the traversal loops: scene_of(slot) is the scene of a
// job slot's rays - the launch's one scene (kernel parameters), the
// per-block table of a several-scene launch, or the job table.
struct OneScene {
  const DevScene& s;
  __device__ __forceinline__ const DevScene& operator()(int) const { return s; }
};
struct TableScene {
  const TravScene* tab;
  __device__ __forceinline__ const TravScene& operator()(int slot) const { return tab[slot]; }
};
struct JobScene {
  const DevJob* jobs;
  __device__ __forceinline__ const DevScene& operator()(int slot) const {
    return jobs[slot].scene;
  }
};

// Warp-cooperative triangle tests (default with the phase vote;
// -DHPT_COOP_TESTS=0 builds the one-test-per-lane rounds): in a test round
// the untested references of every testing lane's current leaf are dealt
// out over the warp's 32 lanes, one test per lane, and a segmented minimum
// over (t, rank) hands each ray the best of its candidates. The reference's
// rule - the smallest t wins, the lower rank on an exact tie - is a
// lexicographic minimum, so the order in which the tests run does not
// change any result.
#ifndef HPT_COOP_TESTS
#define HPT_COOP_TESTS 1
#endif

#if HPT_PHASE_VOTE
#if HPT_COOP_TESTS
// One cooperative test round; every lane of the warp calls it. `testing`:
// this lane's ray is in the test phase; `slot`: its job slot, whose scene
// scene_of(slot) gives (a lane may test for a ray of another job, so it
// reads that ray's scene). Returns true when this lane's ray finished (its
// leaf's last reference was tested and the exit ended it).
template <class SceneOf, class Cnt>
__device__ __forceinline__ bool coop_tests(const SceneOf& scene_of, int slot, bool testing,
                                           TravState& st, TravCold& tc, DevErr* err, Cnt& cnt) {
  const int lane = threadIdx.x & 31;
  const int rem = testing ? st.end - st.k : 0;
  // This lane's references take slots [excl, incl) of the round.
  int incl = rem;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += v;
  }
  const int excl = incl - rem;
  const int total = __shfl_sync(kFull, incl, 31);
  // Slot `lane` belongs to the first lane whose inclusive end exceeds it.
  int owner = 0;
#pragma unroll
  for (int step = 16; step > 0; step >>= 1) {
    const int v = __shfl_sync(kFull, incl, owner + step - 1);
    if (v <= lane) owner += step;
  }
  const bool valid = lane < total;
  const int o_k = __shfl_sync(kFull, st.k, owner);
  const int o_excl = __shfl_sync(kFull, excl, owner);
  const int o_mb = __shfl_sync(kFull, st.mb_id[0], owner);
  const int o_slot = __shfl_sync(kFull, slot, owner);
  Ray r;
  r.o.x = __shfl_sync(kFull, st.ray.o.x, owner);
  r.o.y = __shfl_sync(kFull, st.ray.o.y, owner);
  r.o.z = __shfl_sync(kFull, st.ray.o.z, owner);
  r.d.x = __shfl_sync(kFull, st.ray.d.x, owner);
  r.d.y = __shfl_sync(kFull, st.ray.d.y, owner);
  r.d.z = __shfl_sync(kFull, st.ray.d.z, owner);
  int id = -1;
  uint32_t key = ~0u;  // t's bits for a hit (t > 0: ordered like t), else the maximum
  if (valid) {
    const auto& so = scene_of(o_slot);
    const int j = o_k + (lane - o_excl);
    bool ok = true;
    HPT_DCHECK(err, j >= 0 && j < so.num_leaf_tris, 107, j, ok = false);
    if (ok) {
      id = ldg(so.leaf_refs + j);
      HPT_DCHECK(err, id >= 0 && id < so.num_triangles, 104, id, ok = false);
    }
    if (ok) {
      const float4* rec = reinterpret_cast<const float4*>(so.tris) + 3 * (size_t)id;
      float t, u, v;
      if (mt_test(r, ldg(rec), ldg(rec + 1), ldg(rec + 2), t, u, v)) key = __float_as_uint(t);
    }
  }
  // Work counters as the one-test-per-lane walk counts them: a reference
  // equal to the one before it in its ray's sequence is a mailbox repeat.
  const int up = __shfl_up_sync(kFull, id, 1);
  if (valid) {
    if (id == (lane == o_excl ? o_mb : up)) count_repeat(cnt);
    else count_test(cnt);
  }
  // Segmented minimum of t: the first slot of each ray's range ends with
  // its range's minimum. Bit s of `starts`: slot s begins a range.
  const unsigned starts = __ballot_sync(kFull, valid && lane == o_excl);
  const uint32_t mine = key;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t other = __shfl_down_sync(kFull, key, o);
    const bool same =
        lane + o < 32 &&
        ((unsigned)((unsigned long long)starts >> (lane + 1)) & ((1u << o) - 1)) == 0;
    if (same && other < key) key = other;
  }
  // Of the slots that hold their range's minimum the lowest one - the
  // lowest rank - wins, as the reference's strict comparison in list order
  // keeps the first of equal t.
  const uint32_t seg_min = __shfl_sync(kFull, key, o_excl);
  const unsigned wins = __ballot_sync(kFull, valid && mine != ~0u && mine == seg_min);
  const int first = excl < 32 ? excl : 31;
  const int last = incl < 32 ? incl - 1 : 31;
  const unsigned my_wins = (unsigned)(((unsigned long long)wins >> first) << first);
  const int w = my_wins ? __ffs(my_wins) - 1 : 0;
  const int last_id = __shfl_sync(kFull, id, last < 0 ? 0 : last);
  const int win_id = __shfl_sync(kFull, id, w);
  const uint32_t best = __shfl_sync(kFull, key, first);
  if (!testing) return false;
  if (rem > 0 && excl < 32) {
    const int k0 = st.k;
    st.k += last + 1 - excl;
    st.mb_id[0] = last_id;
    // When the range holds a hit, w is its lowest slot at the range's
    // minimum (the slots past the range belong to other rays).
    if (best != ~0u && w <= last) {
      const float t = __uint_as_float(best);
      const int jb = k0 + (w - excl);
      if (st.best.rec < 0 || t < st.best.t || (t == st.best.t && jb < st.best.rec)) {
        const auto& s = scene_of(slot);
        if (tc.pierced < 0) {
          const float4* L = reinterpret_cast<const float4*>(s.leaves + tc.leaf);
          tc.pierced = ref_box_test(st.ray, ldg(L), ldg(L + 1)) ? 1 : 0;
        }
        if (tc.pierced) {
          st.best.rec = jb;
          st.best.tri = win_id;
          st.best.t = t;
          tc.best_node = tc.leaf_node;
        }
      }
    }
  }
  if (st.k < st.end) return false;
  return trav_exit(scene_of(slot), st, tc, err);
}
#endif

// Up to `units` warp rounds. Every lane of the warp calls it; `live` is
// false for a lane without a ray; scene_of(slot) is the scene of this
// lane's job. kCoop: test rounds are cooperative (coop_tests). Returns true
// when this lane's ray finished.
template <int kMode, bool kCoop, class SceneOf>
__device__ __forceinline__ bool vote_units(const SceneOf& scene_of, int slot, bool live,
                                           TravState& st, TravCold& tc, const uint2* snodes,
                                           int n_smem, DevErr* err, TravCount& cnt, int units) {
  bool finished = false;
  // The cooperative loop's work counts stay in one register and are added
  // to the shared-memory counters at most 128 rounds apart and on return
  // (a shared-memory update per unit measured 1-2 % slower).
  PackedCount ucnt{0};
  for (int u = 0; u < units; ++u) {
    const bool go = live && !finished;
    const unsigned lm = __ballot_sync(kFull, go);
    if (lm == 0) break;
    const bool testing = go && st.phase == kStepTest;
    const unsigned tm = __ballot_sync(kFull, testing);
#if HPT_COOP_TESTS
    if constexpr (kCoop) {
      using SceneT = std::decay_t<decltype(scene_of(slot))>;
      // Every round moves a lane on: a test round needs a testing lane
      // (whatever the threshold), else the descending lanes run.
      if (tm != 0 && 6 * __popc(tm) >= HPT_COOP_TEST_SIXTHS * __popc(lm)) {
        if (coop_tests(scene_of, slot, testing, st, tc, err, ucnt)) finished = true;
      } else if (go && !testing) {
        finished = trav_step<false, kMode == kTravStepSmem, SceneT, false>(
            scene_of(slot), st, tc, snodes, n_smem, err, ucnt);
      }
      if ((u & 127) == 127) count_flush(ucnt, cnt);
      continue;
    }
#endif
    const bool pick_test = 6 * __popc(tm) >= HPT_VOTE_TEST_SIXTHS * __popc(lm);
    if (go && testing == pick_test)
      finished = trav_step<false, kMode == kTravStepSmem>(scene_of(slot), st, tc, snodes, n_smem,
                                                          err, cnt);
  }
  count_flush(ucnt, cnt);
  return finished;
}
#endif

// --- Camera rays of a launch's primary-pass entries (P.prim_*), shared by
// k_primary and the k_isect launches that carry them.
// Entry g: its slot and ray index within the job.
__device__ __forceinline__ bool prim_locate(const EngineParams& P, int64_t g, int& slot,
                                            int64_t& ray) {
  const int e = find_prefix(P.prim_prefix, P.prim_n, g);
  slot = P.prim_slot[e];
  ray = g - P.prim_prefix[e] + (P.prim_first ? P.prim_first[e] : 0);
  bool ok = true;
  HPT_DCHECK(&P.ctrl->err, slot >= 0 && slot < P.num_slots, 201, slot, ok = false);
  HPT_DCHECK(&P.ctrl->err, !ok || (ray >= 0 && ray < job_rays(P.jobs[slot])), 202, ray,
             ok = false);
  return ok;
}

// Starts the walk of the job's camera ray (set_viewdirs / set_viewdirs_vr,
// kernel.cl:559-613).
__device__ __forceinline__ void prim_init(const DevJob& J, int64_t ray, TravState& st,
                                          TravCold& tc) {
  const int x = (int)(ray % J.nx), y = (int)(ray / J.nx);
  const f3 d = J.pano ? pano_dir(x, y, J.vr_x_shift, J.ny)
                      : pinhole_dir(J.top, J.right, J.width, J.height, x, y, J.nx, J.ny);
  trav_init(J.scene, Ray{mk(J.view_p[0], J.view_p[1], J.view_p[2]), d}, st, tc);
}

// A finished camera ray: its hit goes to the job's primary-hit cache; a
// miss adds the background (kernel.cl:193-206: the first pass assigns
// background * strength * sample_n with strength (1,1,1)).
__device__ __forceinline__ void prim_finish(const EngineParams& P, int slot, int64_t ray,
                                            const TravState& st, const TravCold& tc) {
  const DevJob& J = P.jobs[slot];
  if (st.best.rec >= 0) {
    int k = atomicAdd(J.prim_count, 1);
    HPT_DCHECK(&P.ctrl->err, k < job_rays(J), 203, k, k = -1);
    if (k >= 0) {
      float4* dst = reinterpret_cast<float4*>(J.prim) + 2 * (size_t)k;
      dst[0] = make_float4(st.ray.d.x, st.ray.d.y, st.ray.d.z, __int_as_float((int)ray));
      dst[1] = make_float4(__int_as_float(st.best.tri), st.best.t, __int_as_float(tc.best_node),
                           0.f);
    }
  } else {
    const f3 val = scale((float)J.spp, mul(mk(J.bg[0], J.bg[1], J.bg[2]), mk(1.f, 1.f, 1.f)));
    flush_radiance(J, ray, val);
  }
}

// ---------------------------------------------------------------------------
// kMode: traversal as in k_isect.
template <int BS, int MINB, int kMode>
__global__ void __launch_bounds__(BS, MINB) k_primary(EngineParams P) {
  constexpr bool kStep = kMode != kTravLeaf;
  extern __shared__ uint2 snodes[];
  const int n_smem = kMode == kTravStep ? 0 : stage_nodes(P, snodes);
  const TravScene* scene_tab = stage_scenes(P, snodes);
  DevCtrl* c = P.ctrl;
  const int lane = threadIdx.x & 31;
  const int64_t total = P.prim_prefix[P.prim_n];
  bool active = false;
  TravState st;
  __shared__ TravCold cold_sh[BS];
  __shared__ CountSlot count_sh[BS];
  TravCold& tc = cold_sh[threadIdx.x];
  TravCount& cnt = count_sh[threadIdx.x].c;
  cnt = TravCount{};
  uint32_t& queries = count_sh[threadIdx.x].queries;
  queries = 0;
  int slot = 0;
  // The lane's camera ray (read when it finishes; shared memory keeps the
  // registers for the traversal).
  __shared__ int64_t ray_sh[BS];
  int64_t& ray = ray_sh[threadIdx.x];
  ray = 0;
  // Once a refill finds the rays exhausted the warp stops asking (the value
  // is warp-uniform), so the cursor overshoots by at most one grab per warp.
  bool drained = false;
  while (true) {
    const unsigned idle = __ballot_sync(kFull, !active);
    if (!drained && __popc(idle) >= P.refill) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(&c->prim_head, (unsigned long long)__popc(idle));
      base = __shfl_sync(kFull, base, 0);
      drained = (int64_t)base + __popc(idle) >= total;
      if (!active) {
        const int64_t g = (int64_t)base + __popc(idle & lanemask_lt());
        if (g < total && prim_locate(P, g, slot, ray)) {
          prim_init(P.jobs[slot], ray, st, tc);
          active = true;
          ++queries;
        }
      }
    }
    if (__ballot_sync(kFull, active) == 0) break;
    bool finished = false;
#if HPT_PHASE_VOTE
    if constexpr (kStep) {
      if (P.uniform_scene)
        finished = vote_units<kMode, kCoopPrimary>(OneScene{P.uscene}, slot, active, st, tc,
                                         snodes, n_smem, &c->err, cnt, P.trav_steps);
      else if (P.scene_table)
        finished = vote_units<kMode, kCoopPrimary>(TableScene{scene_tab}, slot, active, st, tc,
                                         snodes, n_smem, &c->err, cnt, P.trav_steps);
      else
        finished = vote_units<kMode, kCoopPrimary>(JobScene{P.jobs}, slot, active, st, tc,
                                         snodes, n_smem, &c->err, cnt, P.trav_steps);
    } else if (active) {
      finished = trav_leaf(P.jobs[slot].scene, st, tc, snodes, n_smem, &c->err, cnt);
    }
#else
    if (active) {
      if constexpr (kStep) {
        if (P.uniform_scene) {
          for (int u = 0; u < P.trav_steps; ++u)
            if (trav_step<false, kMode == kTravStepSmem>(P.uscene, st, tc, snodes, n_smem,
                                                         &c->err, cnt)) {
              finished = true;
              break;
            }
        } else if (P.scene_table) {
          const TravScene& sc = scene_tab[slot];
          for (int u = 0; u < P.trav_steps; ++u)
            if (trav_step<false, kMode == kTravStepSmem>(sc, st, tc, snodes, n_smem, &c->err,
                                                         cnt)) {
              finished = true;
              break;
            }
        } else {
          const DevScene& sc = P.jobs[slot].scene;
          for (int u = 0; u < P.trav_steps; ++u)
            if (trav_step<false, kMode == kTravStepSmem>(sc, st, tc, snodes, n_smem, &c->err,
                                                         cnt)) {
              finished = true;
              break;
            }
        }
      } else {
        finished = trav_leaf(P.jobs[slot].scene, st, tc, snodes, n_smem, &c->err, cnt);
      }
    }
#endif
    if (finished) {
      prim_finish(P, slot, ray, st, tc);
      active = false;
    }
  }
  flush_counts(c, queries, cnt);
}

// Sets the path count of primary-pass entry e's slot when the entry
// completes its job's primary pass. A slot whose primary pass is still
// partial stays as it was: inactive, or finished with nothing left to issue.
__device__ void activate_slot(const EngineParams& P, int e) {
  const int s = P.prim_slot[e];
  HPT_DCHECK(&P.ctrl->err, s >= 0 && s < P.num_slots, 232, s, return);
  if (P.prim_final && !P.prim_final[e]) return;
  DevSlot& S = P.slots[s];
  S.num_paths = (int64_t)(*P.jobs[s].prim_count) * P.jobs[s].spp;
  S.cursor = 0;
  S.done = 0;
  S.queries = 0;
  S.max_inflight = P.jobs[s].max_inflight;
  S.alloc = 0;
  S.active = 1;
}

// After k_primary: starts the paths of the slots whose primary pass
// completed and grants paths (one thread).
__global__ void k_admit(EngineParams P) {
#ifdef HPT_DEVICE_CHECKS
  HPT_DCHECK(&P.ctrl->err, P.ctrl->chk_isect_done == P.prim_prefix[P.prim_n], 243,
             P.ctrl->chk_isect_done, (void)0);
  P.ctrl->chk_isect_done = 0;
#endif
  for (int e = 0; e < P.prim_n; ++e) activate_slot(P, e);
  P.ctrl->prim_head = 0;
  schedule(P);
}

// ---------------------------------------------------------------------------
// Shade + next direction (+ new paths), compacting survivors into R.
// ---------------------------------------------------------------------------
// MINB: blocks of BS threads per SM the register budget must fit (1 leaves
// the compiler's natural allocation, ~106 registers = 2 blocks of 256). The
// kernel is bound by gather latency, so resident warps can pay for a few
// spills; the tuning chooses.
template <int BS, int MINB>
__global__ void __launch_bounds__(BS, MINB) k_shade(EngineParams P) {
  __shared__ int warp_counts[BS / 32];
  __shared__ int block_base;
  DevCtrl* c = P.ctrl;
  const int par = c->parity;
  const int nA = c->nA;
  const int n_new = c->n_new, n_quota = c->n_quota;
  const int n_items = nA + n_new;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long shades = 0;
#ifdef HPT_DEVICE_CHECKS
  if (blockIdx.x == 0 && threadIdx.x == 0) c->chk_shade_items = n_items;
  int chk_items = 0;
#endif
  for (int base = blockIdx.x * BS; base < n_items; base += gridDim.x * BS) {
    const int i = base + threadIdx.x;
#ifdef HPT_DEVICE_CHECKS
    if (i < n_items) ++chk_items;
#endif
    bool alive = false, ended = false;
    int slot = 0;
    float4 oo, dd, ss, rr;
    if (i < n_items) {
      int sample = 0, bounce = 0, tri = -1, hint = -1;
      int64_t ray = -1;
      f3 o, d, strength, rad;
      float t = 0.f;
      bool ok = true;
      if (i < nA) {
        HPT_DCHECK(&c->err, i < P.capacity, 211, i, ok = false);
        if (ok) {
          const float4 ao = P.A_o[par][i], ad = P.A_d[par][i], as = P.A_s[par][i],
                       ar = P.A_r[par][i];
          tri = P.A_tri[par][i];
          hint = P.A_leaf[par][i];
          o = mk(ao.x, ao.y, ao.z);
          ray = __float_as_int(ao.w);
          d = mk(ad.x, ad.y, ad.z);
          const uint32_t meta = __float_as_uint(ad.w);
          sample = (int)(meta >> 8);
          bounce = (int)(meta & 0xFF);
          strength = mk(as.x, as.y, as.z);
          slot = __float_as_int(as.w);
          rad = mk(ar.x, ar.y, ar.z);
          t = ar.w;
        }
      } else {
        const int off = i - nA;
        const int e = find_prefix(P.quota_prefix, n_quota, off);
        slot = P.quota_slot[e];
        HPT_DCHECK(&c->err, slot >= 0 && slot < P.num_slots, 212, slot, ok = false);
        if (ok) {
          const DevJob& J = P.jobs[slot];
          const int64_t q = P.slots[slot].cursor + (off - P.quota_prefix[e]);
          const int nh = *J.prim_count;
          HPT_DCHECK(&c->err, nh > 0 && q < (int64_t)nh * J.spp, 213, q, ok = false);
          HPT_DCHECK(&c->err, !ok || nh <= job_rays(J), 217, nh, ok = false);
          if (ok) {
            const int64_t k = q % nh;
            sample = (int)(q / nh);
            bounce = 0;
            const float4* src = reinterpret_cast<const float4*>(J.prim) + 2 * k;
            const float4 p0 = src[0], p1 = src[1];
            o = mk(J.view_p[0], J.view_p[1], J.view_p[2]);
            d = mk(p0.x, p0.y, p0.z);
            ray = __float_as_int(p0.w);
            tri = __float_as_int(p1.x);
            t = p1.y;
            hint = __float_as_int(p1.z);
            strength = mk(1.f, 1.f, 1.f);
            rad = mk(0.f, 0.f, 0.f);
          }
        }
      }
      HPT_DCHECK(&c->err, !ok || (slot >= 0 && slot < P.num_slots), 212, slot, ok = false);
      HPT_DCHECK(&c->err, !ok || (tri >= 0 && tri < P.jobs[slot].scene.num_triangles), 214, tri,
                 ok = false);
      HPT_DCHECK(&c->err, !ok || (ray >= 0 && ray < job_rays(P.jobs[slot])), 215, ray, ok = false);
      if (ok) {
        const DevJob& J = P.jobs[slot];
        // The frame's sample index keys the random stream, so a render of
        // samples [first_sample, first_sample + spp) traces the same paths
        // as those samples of one whole-frame render.
        uint64_t seed = path_seed(J.seed, (uint32_t)ray, (uint32_t)(J.first_sample + sample),
                                  (uint32_t)bounce);
        const Ray r{o, d};
        const ShadeOut so = shade_hit(J.scene, r, strength, tri, t, J.disable_diffuse, seed,
                                      &c->err);
        ++shades;
        rad = add(rad, so.contrib);
        if (so.branch != kDead && bounce + 1 < J.depth) {
          const NextOut no = next_direction(J.scene, so.branch, d, so.hit_p, so.normal,
                                            so.strength, so.param, seed, &c->err);
          if (no.alive) {
            alive = true;
            oo = make_float4(no.o.x, no.o.y, no.o.z, __int_as_float((int)ray));
            dd = make_float4(no.d.x, no.d.y, no.d.z,
                             __uint_as_float(((uint32_t)sample << 8) | (uint32_t)(bounce + 1)));
            ss = make_float4(no.strength.x, no.strength.y, no.strength.z, __int_as_float(slot));
            rr = make_float4(rad.x, rad.y, rad.z, __int_as_float(hint));
          }
        }
        if (!alive) {
          flush_radiance(J, ray, rad);
          ended = true;
        }
      }
    }
    count_done(P.slots, ended, slot);
    count_queries(P.slots, alive, slot);
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
      bool ok = true;
      HPT_DCHECK(&c->err, pos < P.capacity, 216, pos, ok = false);
      if (ok) {
        P.R_o[pos] = oo;
        P.R_d[pos] = dd;
        P.R_s[pos] = ss;
        P.R_r[pos] = rr;
      }
    }
    __syncthreads();
  }
  for (int o = 16; o > 0; o >>= 1) shades += __shfl_down_sync(kFull, shades, o);
  if (lane == 0 && shades) atomicAdd(&c->shades, shades);
#ifdef HPT_DEVICE_CHECKS
  for (int o = 16; o > 0; o >>= 1) chk_items += __shfl_down_sync(kFull, chk_items, o);
  if (lane == 0 && chk_items) atomicAdd(&c->chk_shade_done, chk_items);
#endif
}

// ---------------------------------------------------------------------------
// Intersect queue -> next shade queue, persistent warps with lane refill.
// ---------------------------------------------------------------------------
// kMode: kTravStep / kTravStepSmem traverse with trav_step, P.trav_steps
// calls per lane between refill checks (lanes move to their next leaf
// independently), reading nodes from global memory only / also from the
// shared-memory prefix; kTravLeaf: one leaf per lane per round with
// trav_leaf.
// kPrim: the launch also traces the camera rays of its primary-pass entries
// (P.prim_*), after the queue's rays, and records them as k_primary does;
// k_ctrl then starts the paths of the jobs whose primary pass completed.
// A serving loop admits requests this way, with no launch of its own.
template <int BS, int MINB, int kMode, bool kPrim = false>
__global__ void __launch_bounds__(BS, MINB) k_isect(EngineParams P) {
  constexpr bool kStep = kMode != kTravLeaf;
  extern __shared__ uint2 snodes[];
  const int n_smem = kMode == kTravStep ? 0 : stage_nodes(P, snodes);
  const TravScene* scene_tab = stage_scenes(P, snodes);
  DevCtrl* c = P.ctrl;
  const int n = c->nR;
  const int64_t total = kPrim ? (int64_t)n + P.prim_prefix[P.prim_n] : (int64_t)n;
  const int out_par = c->parity ^ 1;
  const int lane = threadIdx.x & 31;
  bool active = false;
  TravState st;
  __shared__ TravCold cold_sh[BS];
  __shared__ CountSlot count_sh[BS];
  TravCold& tc = cold_sh[threadIdx.x];
  TravCount& cnt = count_sh[threadIdx.x].c;
  cnt = TravCount{};
  uint32_t& queries = count_sh[threadIdx.x].queries;
  queries = 0;
  // Index in the intersect queue (the payload is reloaded at the end); with
  // kPrim, -1 - ray for a camera ray. Read when the ray finishes, so it
  // stays in shared memory.
  __shared__ int item_sh[BS];
  int& item = item_sh[threadIdx.x];
  item = 0;
  int slot = 0;
  // As in k_primary: a warp that finds the queue exhausted stops refilling.
  bool drained = false;
  while (true) {
    const unsigned idle = __ballot_sync(kFull, !active);
    if (!drained && __popc(idle) >= P.refill) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(&c->isect_head, (unsigned long long)__popc(idle));
      base = __shfl_sync(kFull, base, 0);
      drained = (int64_t)base + __popc(idle) >= total;
      if (!active) {
        const int64_t i = (int64_t)base + __popc(idle & lanemask_lt());
        if constexpr (kPrim) {
          int64_t ray = 0;
          if (i >= n && i < total && prim_locate(P, i - n, slot, ray)) {
            prim_init(P.jobs[slot], ray, st, tc);
            item = -1 - (int)ray;
            active = true;
            ++queries;
          }
        }
        if (i < n) {
          bool ok = true;
          HPT_DCHECK(&c->err, i < P.capacity, 221, i, ok = false);
          if (ok) {
            const float4 o4 = P.R_o[i], d4 = P.R_d[i];
            item = (int)i;
            slot = __float_as_int(P.R_s[i].w);
            HPT_DCHECK(&c->err, slot >= 0 && slot < P.num_slots, 222, slot, ok = false);
            if (ok) {
              trav_init(P.jobs[slot].scene, Ray{mk(o4.x, o4.y, o4.z), mk(d4.x, d4.y, d4.z)}, st,
                        tc, __float_as_int(P.R_r[i].w));
              active = true;
              ++queries;
            }
          }
        }
      }
    }
    if (__ballot_sync(kFull, active) == 0) break;
    bool finished = false;
#if HPT_PHASE_VOTE
    if constexpr (kStep) {
      if (P.uniform_scene)
        finished = vote_units<kMode, true>(OneScene{P.uscene}, slot, active, st, tc,
                                         snodes, n_smem, &c->err, cnt, P.trav_steps);
      else if (P.scene_table)
        finished = vote_units<kMode, true>(TableScene{scene_tab}, slot, active, st, tc,
                                         snodes, n_smem, &c->err, cnt, P.trav_steps);
      else
        finished = vote_units<kMode, true>(JobScene{P.jobs}, slot, active, st, tc,
                                         snodes, n_smem, &c->err, cnt, P.trav_steps);
    } else if (active) {
      finished = trav_leaf(P.jobs[slot].scene, st, tc, snodes, n_smem, &c->err, cnt);
    }
#else
    if (active) {
      if constexpr (kStep) {
        if (P.uniform_scene) {
          for (int u = 0; u < P.trav_steps; ++u)
            if (trav_step<false, kMode == kTravStepSmem>(P.uscene, st, tc, snodes, n_smem,
                                                         &c->err, cnt)) {
              finished = true;
              break;
            }
        } else if (P.scene_table) {
          const TravScene& sc = scene_tab[slot];
          for (int u = 0; u < P.trav_steps; ++u)
            if (trav_step<false, kMode == kTravStepSmem>(sc, st, tc, snodes, n_smem, &c->err,
                                                         cnt)) {
              finished = true;
              break;
            }
        } else {
          const DevScene& sc = P.jobs[slot].scene;
          for (int u = 0; u < P.trav_steps; ++u)
            if (trav_step<false, kMode == kTravStepSmem>(sc, st, tc, snodes, n_smem, &c->err,
                                                         cnt)) {
              finished = true;
              break;
            }
        }
      } else {
        finished = trav_leaf(P.jobs[slot].scene, st, tc, snodes, n_smem, &c->err, cnt);
      }
    }
#endif
    // A camera ray (kPrim) goes to its job's primary-hit cache instead.
    const bool queued = !kPrim || item >= 0;
    if constexpr (kPrim) {
      if (finished && !queued) prim_finish(P, slot, -1 - (int64_t)item, st, tc);
    }
    const bool hit = finished && queued && st.best.rec >= 0;
    const unsigned hm = __ballot_sync(kFull, hit);
    if (hm) {
      const int leader = __ffs(hm) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(&c->nA_next, __popc(hm));
      base = __shfl_sync(kFull, base, leader);
      if (hit) {
        const int pos = base + __popc(hm & lanemask_lt());
        bool ok = true;
        HPT_DCHECK(&c->err, pos < P.capacity, 223, pos, ok = false);
        if (ok) {
          const float4 r4 = P.R_r[item];
          P.A_o[out_par][pos] = P.R_o[item];
          P.A_d[out_par][pos] = P.R_d[item];
          P.A_s[out_par][pos] = P.R_s[item];
          P.A_r[out_par][pos] = make_float4(r4.x, r4.y, r4.z, st.best.t);
          P.A_tri[out_par][pos] = st.best.tri;
          P.A_leaf[out_par][pos] = tc.best_node;
        }
      }
    }
    const bool missed = finished && queued && !hit;
    if (missed) {
      // kernel.cl:195-200: miss adds background * strength (sample_n = 1).
      const DevJob& J = P.jobs[slot];
      const float4 s4 = P.R_s[item], r4 = P.R_r[item];
      const int64_t ray = __float_as_int(P.R_o[item].w);
      bool ok = true;
      HPT_DCHECK(&c->err, ray >= 0 && ray < job_rays(J), 224, ray, ok = false);
      if (ok) {
        f3 rad = mk(r4.x, r4.y, r4.z);
        rad = add(rad, mul(mk(J.bg[0], J.bg[1], J.bg[2]), mk(s4.x, s4.y, s4.z)));
        flush_radiance(J, ray, rad);
      }
    }
    count_done(P.slots, missed, slot);
    if (finished) active = false;
  }
  flush_counts(c, queries, cnt);
}

// Advances the queues and the path cursors, then grants paths (one thread).
__global__ void k_ctrl(EngineParams P) {
  DevCtrl* c = P.ctrl;
#ifdef HPT_DEVICE_CHECKS
  HPT_DCHECK(&c->err, c->chk_shade_done == c->chk_shade_items, 241,
             (long long)c->chk_shade_items * 1000000 + c->chk_shade_done, (void)0);
  HPT_DCHECK(&c->err, c->chk_isect_done == c->nR + (P.prim_n ? P.prim_prefix[P.prim_n] : 0),
             242, (long long)c->nR * 1000000 + c->chk_isect_done, (void)0);
  c->chk_shade_items = 0;
  c->chk_shade_done = 0;
  c->chk_isect_done = 0;
#endif
  for (int k = 0; k < c->n_quota; ++k) {
    DevSlot& S = P.slots[P.quota_slot[k]];
    S.cursor += S.alloc;
    S.alloc = 0;
  }
  c->nA = c->nA_next;
  c->nA_next = 0;
  c->nR = 0;
  c->isect_head = 0;
  c->parity ^= 1;
  c->iterations += 1;
  // Jobs whose primary pass the iteration's k_isect completed (kPrim).
  for (int e = 0; e < P.prim_n; ++e) activate_slot(P, e);
  schedule(P);
}

// Register budgets for the traversal kernels: (threads per block, blocks
// per SM the compiler must fit). The natural allocation is ~97 registers;
// tighter budgets trade spills for resident warps. Chosen by the tuning.
struct IsectVariant {
  int block, min_blocks;
  void (*isect)(EngineParams);            // one leaf per round
  void (*isect_step)(EngineParams);       // step-at-a-time, nodes from global memory
  void (*isect_step_smem)(EngineParams);  // step-at-a-time, shared-memory node prefix
  void (*primary)(EngineParams);
  void (*primary_step)(EngineParams);
  void (*primary_step_smem)(EngineParams);
  void (*isect_step_prim)(EngineParams);  // step-at-a-time with primary-pass entries
  // The kernel a launch with these tuning values uses (shared-node prefix
  // only when smem_nodes > 0).
  void (*isect_kernel(int trav_steps, int smem_nodes) const)(EngineParams) {
    return trav_steps <= 0 ? isect : (smem_nodes > 0 ? isect_step_smem : isect_step);
  }
  void (*primary_kernel(int trav_steps, int smem_nodes) const)(EngineParams) {
    return trav_steps <= 0 ? primary : (smem_nodes > 0 ? primary_step_smem : primary_step);
  }
};
#define HPT_ISECT_VARIANT(B, M)                                                       \
  {B, M, k_isect<B, M, kTravLeaf>, k_isect<B, M, kTravStep>,                          \
   k_isect<B, M, kTravStepSmem>, k_primary<B, M, kTravLeaf>, k_primary<B, M, kTravStep>, \
   k_primary<B, M, kTravStepSmem>, k_isect<B, M, kTravStep, true>}
const IsectVariant kIsectVariants[] = {
    HPT_ISECT_VARIANT(128, 5), HPT_ISECT_VARIANT(128, 6), HPT_ISECT_VARIANT(128, 7),
    HPT_ISECT_VARIANT(128, 8), HPT_ISECT_VARIANT(128, 9), HPT_ISECT_VARIANT(128, 10),
    HPT_ISECT_VARIANT(256, 2), HPT_ISECT_VARIANT(256, 3),
};
#undef HPT_ISECT_VARIANT
constexpr int kNumIsectVariants = sizeof(kIsectVariants) / sizeof(kIsectVariants[0]);

// The shading kernel for a tuning's register budget (shade_min_blocks 3 or
// 4 blocks of 256 per SM; anything else: the natural allocation).
void (*shade_kernel(const hpt_tuning& t))(EngineParams) {
  if (t.shade_min_blocks == 3) return k_shade<256, 3>;
  if (t.shade_min_blocks == 4) return k_shade<256, 4>;
  return k_shade<256, 1>;
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
// samples is the divisor: the full sample count for the final image, or the
// samples completed so far for a progressive preview.
__global__ void k_resolve(const DevJob* jp, int W, int H, int ssx, int ssy, float samples,
                          float brightness, uint8_t* rgba, float* accum_f) {
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
  const float nss = (float)(ssx * ssy), ns = samples;
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

void cuda_soft_fail(cudaError_t e, const char* what) {
  (void)cudaGetLastError();
#ifdef HPT_DEVICE_CHECKS
  fprintf(stderr, "hpt: best-effort call failed: %s: %s\n", what, cudaGetErrorString(e));
#else
  (void)e;
  (void)what;
#endif
}

hpt_tuning default_tuning() {
  hpt_tuning t;
  memset(&t, 0, sizeof t);
  // From the tuning sweeps on the 61k-triangle spheres frame (512x512,
  // 64 spp) and the 2.4M-triangle terrain frame: step-at-a-time traversal
  // with the phase vote, 48 warp rounds per refill check (16 / 24 / 32 /
  // 48: spheres 107.0 / 105.7 / 105.0 / 105.0 ms, terrain at 4 spp 79.6 /
  // 79.0 / 78.7 / 77.7 ms; with cooperative tests 32 / 48 / 64: 92.5 /
  // 92.3 / 93.0 ms), 9 blocks of 128 per SM (56 registers; with
  // cooperative tests 8 / 9 / 10 blocks: spheres 94.8 / 92.3 / 101.4 ms,
  // terrain 74.3 / 70.7 / 81.5 ms - at 10 the 48-register budget spills),
  // no shared-node prefix, a wavefront of 2^24 paths (2^22 / 2^23 / 2^24 /
  // 2^25: spheres 92.2 / 88.7 / 87.0 / 87.1 ms, terrain at 16 spp 227.5 /
  // 223.0 / 220.3 / 218.4 ms; 3.5 GB of queues, allocated only up to the
  // paths a run has).
  t.capacity = 1 << 24;
  t.isect_block = 128;
  t.isect_min_blocks = 9;
  t.shade_block = 256;
  t.refill_chunk = 4;
  t.smem_nodes = 0;
  t.use_graph = 0;
  t.trav_steps = 48;
  // Shading at 4 blocks of 256 per SM (64 registers): 7.0 instead of 8.4 ms
  // per spheres frame at the natural 106-register allocation (2 blocks).
  t.shade_min_blocks = 4;
  return t;
}

// The scene as a job sees it: the tuning's step cap, when set, replaces the
// scene's own (only ever lowering it).
DevScene capped_scene(const DevScene& s, const hpt_tuning& t) {
  DevScene out = s;
  if (t.max_steps > 0) out.max_steps = std::min(out.max_steps, t.max_steps);
  return out;
}

hpt_status check_render_params(const hpt_camera* cam, const hpt_render_params* p) {
  if (!cam || !p) return fail(HPT_ERR_INVALID_ARGUMENT, "camera/params is NULL");
  if (p->sample_x <= 0 || p->sample_y <= 0 || p->supersample_x <= 0 || p->supersample_y <= 0 ||
      p->sample <= 0 || p->depth <= 0)
    return fail(HPT_ERR_INVALID_ARGUMENT, "sizes, sample and depth must be positive");
  const int64_t rays = (int64_t)p->sample_x * p->supersample_x * p->sample_y * p->supersample_y;
  if (rays > (1ll << 30)) return fail(HPT_ERR_INVALID_ARGUMENT, "too many rays per frame");
  if (p->sample >= (1 << 24)) return fail(HPT_ERR_INVALID_ARGUMENT, "sample must be < 2^24");
  if (p->first_sample < 0 || p->first_sample > INT32_MAX - p->sample)
    return fail(HPT_ERR_INVALID_ARGUMENT, "first_sample must be >= 0 and first_sample + sample < 2^31");
  if (p->depth > 255) return fail(HPT_ERR_INVALID_ARGUMENT, "depth must be <= 255");
  if (cam->height < 0 && p->supersample_x != p->supersample_y)
    return fail(HPT_ERR_INVALID_ARGUMENT,
                "panorama needs supersample_x == supersample_y (the reference indexes rays with "
                "sample_x * supersample_y)");
  return HPT_OK;
}

int64_t job_footprint(const hpt_render_params& p, bool want_accum) {
  const int64_t rays = (int64_t)p.sample_x * p.supersample_x * p.sample_y * p.supersample_y;
  return rays * (24 + 4 + 32 + (want_accum ? 12 : 0)) + (int64_t)p.sample_x * p.sample_y * 4 + 64;
}

Engine::Engine(int dev) : device(dev) {
  tuning = default_tuning();
  for (auto& e : ev_) e = nullptr;
  init_status_ = init();
}

// Device resources every run needs; a failure is reported by run().
hpt_status Engine::init() {
  HPT_CUDA(cudaSetDevice(device));
  HPT_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  HPT_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
  HPT_CUDA(cudaMalloc(&ctrl_, sizeof(DevCtrl)));
  HPT_CUDA(cudaMallocHost(&ctrl_host_, sizeof(DevCtrl)));
  for (auto& e : ev_) HPT_CUDA(cudaEventCreate(&e));
  for (auto& e : ev_done_) HPT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  HPT_CUDA(cudaMallocHost(&done_host_, 2 * sizeof(int32_t)));
  // Per-job buffers come from the engine's own stream-ordered pool, which
  // keeps up to 4 GiB of freed memory mapped between renders instead of
  // returning it to the driver at every synchronisation.
  cudaMemPoolProps props;
  memset(&props, 0, sizeof props);
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  HPT_CUDA(cudaMemPoolCreate(&pool_, &props));
  uint64_t keep = 4ull << 30;
  HPT_CUDA(cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep));
  return HPT_OK;
}

Engine::~Engine() {
  HPT_SOFT(cudaSetDevice(device));
  if (stream) HPT_SOFT(cudaStreamSynchronize(stream));
  for (int p = 0; p < 2; ++p) {
    HPT_SOFT(cudaFree(A_o_[p]));
    HPT_SOFT(cudaFree(A_d_[p]));
    HPT_SOFT(cudaFree(A_s_[p]));
    HPT_SOFT(cudaFree(A_r_[p]));
    HPT_SOFT(cudaFree(A_tri_[p]));
    HPT_SOFT(cudaFree(A_leaf_[p]));
  }
  HPT_SOFT(cudaFree(R_o_));
  HPT_SOFT(cudaFree(R_d_));
  HPT_SOFT(cudaFree(R_s_));
  HPT_SOFT(cudaFree(R_r_));
  HPT_SOFT(cudaFree(ctrl_));
  HPT_SOFT(cudaFree(jobs_));
  HPT_SOFT(cudaFree(slot_state_));
  HPT_SOFT(cudaFree(order_));
  HPT_SOFT(cudaFree(quota_slot_));
  HPT_SOFT(cudaFree(quota_prefix_));
  HPT_SOFT(cudaFree(prim_slot_));
  HPT_SOFT(cudaFree(prim_prefix_));
  HPT_SOFT(cudaFree(prim_first_));
  HPT_SOFT(cudaFree(prim_final_));
  HPT_SOFT(cudaFreeHost(ctrl_host_));
  HPT_SOFT(cudaFreeHost(host_i32_));
  HPT_SOFT(cudaFreeHost(host_i64_));
  HPT_SOFT(cudaFreeHost(host_jobs_));
  HPT_SOFT(cudaFreeHost(slots_host_));
  for (auto& e : ev_)
    if (e) HPT_SOFT(cudaEventDestroy(e));
  for (auto& e : ev_done_)
    if (e) HPT_SOFT(cudaEventDestroy(e));
  for (auto& e : pev_) HPT_SOFT(cudaEventDestroy(e));
  if (done_host_) HPT_SOFT(cudaFreeHost(done_host_));
  if (pool_) HPT_SOFT(cudaMemPoolDestroy(pool_));
  if (graph_exec_) HPT_SOFT(cudaGraphExecDestroy(graph_exec_));
  for (StagingSet& st : staging_) {
    HPT_SOFT(cudaFreeHost(st.jobs));
    HPT_SOFT(cudaFreeHost(st.i32));
    HPT_SOFT(cudaFreeHost(st.i64));
    if (st.ev) HPT_SOFT(cudaEventDestroy(st.ev));
  }
  if (stream) HPT_SOFT(cudaStreamDestroy(stream));
}

hpt_status Engine::ensure_capacity(int capacity) {
  if (capacity <= capacity_) return HPT_OK;
  HPT_SOFT(cudaStreamSynchronize(stream));
  for (int p = 0; p < 2; ++p) {
    HPT_SOFT(cudaFree(A_o_[p]));
    HPT_SOFT(cudaFree(A_d_[p]));
    HPT_SOFT(cudaFree(A_s_[p]));
    HPT_SOFT(cudaFree(A_r_[p]));
    HPT_SOFT(cudaFree(A_tri_[p]));
    HPT_SOFT(cudaFree(A_leaf_[p]));
    A_o_[p] = A_d_[p] = A_s_[p] = A_r_[p] = nullptr;
    A_tri_[p] = A_leaf_[p] = nullptr;
  }
  HPT_SOFT(cudaFree(R_o_));
  HPT_SOFT(cudaFree(R_d_));
  HPT_SOFT(cudaFree(R_s_));
  HPT_SOFT(cudaFree(R_r_));
  R_o_ = R_d_ = R_s_ = R_r_ = nullptr;
  capacity_ = 0;
  const size_t n = (size_t)capacity;
  for (int p = 0; p < 2; ++p) {
    HPT_CUDA(cudaMalloc(&A_o_[p], n * sizeof(float4)));
    HPT_CUDA(cudaMalloc(&A_d_[p], n * sizeof(float4)));
    HPT_CUDA(cudaMalloc(&A_s_[p], n * sizeof(float4)));
    HPT_CUDA(cudaMalloc(&A_r_[p], n * sizeof(float4)));
    HPT_CUDA(cudaMalloc(&A_tri_[p], n * sizeof(int32_t)));
    HPT_CUDA(cudaMalloc(&A_leaf_[p], n * sizeof(int32_t)));
  }
  HPT_CUDA(cudaMalloc(&R_o_, n * sizeof(float4)));
  HPT_CUDA(cudaMalloc(&R_d_, n * sizeof(float4)));
  HPT_CUDA(cudaMalloc(&R_s_, n * sizeof(float4)));
  HPT_CUDA(cudaMalloc(&R_r_, n * sizeof(float4)));
  capacity_ = capacity;
  return HPT_OK;
}

hpt_status Engine::ensure_slots(int slots) {
  if (slots <= slots_) return HPT_OK;
  HPT_SOFT(cudaStreamSynchronize(stream));
  HPT_SOFT(cudaFree(jobs_));
  HPT_SOFT(cudaFree(slot_state_));
  HPT_SOFT(cudaFree(order_));
  HPT_SOFT(cudaFree(quota_slot_));
  HPT_SOFT(cudaFree(quota_prefix_));
  HPT_SOFT(cudaFree(prim_slot_));
  HPT_SOFT(cudaFree(prim_prefix_));
  HPT_SOFT(cudaFree(prim_first_));
  HPT_SOFT(cudaFree(prim_final_));
  HPT_SOFT(cudaFreeHost(host_i32_));
  HPT_SOFT(cudaFreeHost(host_i64_));
  HPT_SOFT(cudaFreeHost(host_jobs_));
  HPT_SOFT(cudaFreeHost(slots_host_));
  slots_host_ = nullptr;
  jobs_ = nullptr;
  slot_state_ = nullptr;
  order_ = quota_slot_ = quota_prefix_ = prim_slot_ = prim_final_ = nullptr;
  prim_prefix_ = prim_first_ = nullptr;
  host_i32_ = nullptr;
  host_i64_ = nullptr;
  host_jobs_ = nullptr;
  slots_ = 0;
  const size_t n = (size_t)slots;
  HPT_CUDA(cudaMalloc(&jobs_, n * sizeof(DevJob)));
  HPT_CUDA(cudaMalloc(&slot_state_, n * sizeof(DevSlot)));
  HPT_CUDA(cudaMalloc(&order_, n * sizeof(int32_t)));
  HPT_CUDA(cudaMalloc(&quota_slot_, n * sizeof(int32_t)));
  HPT_CUDA(cudaMalloc(&quota_prefix_, (n + 1) * sizeof(int32_t)));
  HPT_CUDA(cudaMalloc(&prim_slot_, n * sizeof(int32_t)));
  HPT_CUDA(cudaMalloc(&prim_prefix_, (n + 1) * sizeof(int64_t)));
  HPT_CUDA(cudaMalloc(&prim_first_, n * sizeof(int64_t)));
  HPT_CUDA(cudaMalloc(&prim_final_, n * sizeof(int32_t)));
  HPT_CUDA(cudaMallocHost(&host_i32_, (2 * n + 3) * sizeof(int32_t)));
  HPT_CUDA(cudaMallocHost(&host_i64_, (n + 1) * sizeof(int64_t)));
  HPT_CUDA(cudaMallocHost(&host_jobs_, n * sizeof(DevJob)));
  HPT_CUDA(cudaMallocHost(&slots_host_, n * sizeof(DevSlot)));
  HPT_CUDA(cudaMemsetAsync(jobs_, 0, n * sizeof(DevJob), stream));
  HPT_CUDA(cudaMemsetAsync(slot_state_, 0, n * sizeof(DevSlot), stream));
  HPT_CUDA(cudaMemsetAsync(quota_prefix_, 0, (n + 1) * sizeof(int32_t), stream));
  HPT_CUDA(cudaMemsetAsync(prim_prefix_, 0, (n + 1) * sizeof(int64_t), stream));
  slots_ = slots;
  return HPT_OK;
}

// The compiled variant with the tuning's block size and blocks-per-SM
// budget; without an exact match, the first one with that block size.
int Engine::isect_variant() const {
  for (int i = 0; i < kNumIsectVariants; ++i)
    if (kIsectVariants[i].block == tuning.isect_block &&
        kIsectVariants[i].min_blocks == tuning.isect_min_blocks)
      return i;
  for (int i = 0; i < kNumIsectVariants; ++i)
    if (kIsectVariants[i].block == tuning.isect_block) return i;
  return 0;
}

// The dynamic shared-memory limit is an attribute of the kernel function
// (per device, shared by every engine of the process), so it is raised once
// to the largest node prefix a tuning may ask for and never lowered.
static hpt_status raise_smem_limits(int device) {
  static std::mutex mu;
  static std::vector<char> done;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)done.size() <= device) done.resize(device + 1, 0);
  if (done[device]) return HPT_OK;
  const int bytes = kMaxSmemNodes * (int)sizeof(uint2);
  for (const IsectVariant& v : kIsectVariants) {
    HPT_CUDA(cudaFuncSetAttribute(v.primary, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    HPT_CUDA(cudaFuncSetAttribute(v.primary_step, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  bytes));
    HPT_CUDA(cudaFuncSetAttribute(v.isect, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    HPT_CUDA(cudaFuncSetAttribute(v.isect_step, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  bytes));
    HPT_CUDA(cudaFuncSetAttribute(v.primary_step_smem,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    HPT_CUDA(cudaFuncSetAttribute(v.isect_step_smem,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  }
  done[device] = 1;
  return HPT_OK;
}

hpt_status Engine::query_occupancy() {
  if (occ_done_) return HPT_OK;
  hpt_status s = raise_smem_limits(device);
  if (s != HPT_OK) return s;
  const IsectVariant& v = kIsectVariants[isect_variant()];
  const size_t smem = (size_t)std::max(0, tuning.smem_nodes) * sizeof(uint2);
  int b = 0;
  HPT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &b, v.isect_kernel(tuning.trav_steps, tuning.smem_nodes), v.block, smem));
  occ_isect_ = std::max(1, b);
  HPT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, shade_kernel(tuning), 256, 0));
  occ_shade_ = std::max(1, b);
  occ_done_ = true;
  return HPT_OK;
}

hpt_status Engine::alloc_job(const JobSpec& js, bool want_accum, JobBuffers& b) {
  const hpt_render_params& p = js.params;
  const int64_t nx = (int64_t)p.sample_x * p.supersample_x, ny = (int64_t)p.sample_y * p.supersample_y;
  b.rays = nx * ny;
  auto take = [&](auto** ptr, size_t bytes) {
    return cudaMallocFromPoolAsync(reinterpret_cast<void**>(ptr), bytes, pool_, stream);
  };
  HPT_CUDA(take(&b.accum, (size_t)b.rays * 3 * sizeof(unsigned long long)));
  HPT_CUDA(take(&b.flags, (size_t)b.rays * sizeof(uint32_t)));
  HPT_CUDA(take(&b.prim, (size_t)b.rays * 8 * sizeof(float)));
  HPT_CUDA(take(&b.prim_count, sizeof(int32_t)));
  HPT_CUDA(take(&b.rgba, (size_t)p.sample_x * p.sample_y * 4));
  if (want_accum) HPT_CUDA(take(&b.accum_f, (size_t)b.rays * 3 * sizeof(float)));
  HPT_CUDA(cudaMemsetAsync(b.accum, 0, (size_t)b.rays * 3 * sizeof(unsigned long long), stream));
  HPT_CUDA(cudaMemsetAsync(b.flags, 0, (size_t)b.rays * sizeof(uint32_t), stream));
  HPT_CUDA(cudaMemsetAsync(b.prim_count, 0, sizeof(int32_t), stream));
  b.bytes = job_footprint(p, want_accum);
  return HPT_OK;
}

void Engine::free_job(JobBuffers& b) {
  HPT_SOFT(cudaFreeAsync(b.accum, stream));
  HPT_SOFT(cudaFreeAsync(b.flags, stream));
  HPT_SOFT(cudaFreeAsync(b.prim, stream));
  HPT_SOFT(cudaFreeAsync(b.prim_count, stream));
  HPT_SOFT(cudaFreeAsync(b.rgba, stream));
  if (b.accum_f) HPT_SOFT(cudaFreeAsync(b.accum_f, stream));
  b = JobBuffers();
}

DevJob Engine::make_job(const JobSpec& js, const JobBuffers& b) const {
  DevJob j;
  memset(&j, 0, sizeof j);
  const hpt_camera& cam = js.camera;
  const hpt_render_params& p = js.params;
  j.scene = capped_scene(js.scene->dev, tuning);
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
  j.spp = p.sample;
  j.depth = p.depth;
  j.disable_diffuse = p.disable_diffuse;
  j.first_sample = p.first_sample;
  j.seed = p.seed;
  j.accum = b.accum;
  j.flags = b.flags;
  j.prim = b.prim;
  j.prim_count = b.prim_count;
  return j;
}

// Largest per-slot scene table kept in shared memory (102 slots): 10
// blocks of 128 per SM then still fit beside their static shared memory.
constexpr size_t kSceneTableBytes = 8192;

static EngineParams make_params(const Engine& e, DevCtrl* ctrl, DevJob* jobs, DevSlot* slots,
                                int num_slots, const int32_t* order, int32_t* quota_slot,
                                int32_t* quota_prefix, const int32_t* prim_slot,
                                const int64_t* prim_prefix, int prim_n, int capacity,
                                float4* const* A, int32_t* const* Atri, int32_t* const* Aleaf,
                                float4* const* R, const DevScene* shared) {
  EngineParams P;
  memset(&P, 0, sizeof P);
  P.jobs = jobs;
  P.slots = slots;
  P.num_slots = num_slots;
  P.ctrl = ctrl;
  P.order = order;
  P.quota_slot = quota_slot;
  P.quota_prefix = quota_prefix;
  P.prim_slot = prim_slot;
  P.prim_prefix = prim_prefix;
  P.prim_n = prim_n;
  for (int p = 0; p < 2; ++p) {
    P.A_o[p] = A[4 * p + 0];
    P.A_d[p] = A[4 * p + 1];
    P.A_s[p] = A[4 * p + 2];
    P.A_r[p] = A[4 * p + 3];
    P.A_tri[p] = Atri[p];
    P.A_leaf[p] = Aleaf[p];
  }
  P.R_o = R[0];
  P.R_d = R[1];
  P.R_s = R[2];
  P.R_r = R[3];
  P.capacity = capacity;
  P.refill = std::max(1, std::min(32, e.tuning.refill_chunk));
  P.trav_steps = std::max(0, e.tuning.trav_steps);
  if (shared) {
    P.uniform_scene = 1;
    P.uscene = capped_scene(*shared, e.tuning);
  }
  if (shared && e.tuning.smem_nodes > 0) {
    P.smem_nodes = std::min(e.tuning.smem_nodes, shared->num_nodes);
    P.shared_nodes = shared->nodes;
  }
  if (!shared && (size_t)num_slots * sizeof(TravScene) <= kSceneTableBytes) P.scene_table = 1;
  return P;
}

// Dynamic shared memory of a traversal launch: the node prefix of a
// one-scene launch, or the per-slot scene table of a several-scene one.
static size_t launch_smem(const EngineParams& P) {
  return P.scene_table ? (size_t)P.num_slots * sizeof(TravScene)
                       : (size_t)P.smem_nodes * sizeof(uint2);
}

void Engine::reset_ctrl() {
  HPT_SOFT(cudaMemsetAsync(ctrl_, 0, sizeof(DevCtrl), stream));
  if (slots_ > 0) HPT_SOFT(cudaMemsetAsync(slot_state_, 0, (size_t)slots_ * sizeof(DevSlot), stream));
}

hpt_status Engine::set_order(const std::vector<int>& order) {
  if ((int)order.size() > slots_) return fail(HPT_ERR_INVALID_ARGUMENT, "order larger than slots");
  // Pinned staging: [0, slots] prim_slot (admit), [slots + 1, 2 slots + 1]
  // order, [2 slots + 2] n_order. Regions never overlap, so a copy still
  // queued behind a kernel reads what was written for it.
  int32_t* stage = host_i32_ + (slots_ + 1);
  for (size_t k = 0; k < order.size(); ++k) stage[k] = order[k];
  if (!order.empty())
    HPT_CUDA(cudaMemcpyAsync(order_, stage, order.size() * sizeof(int32_t),
                             cudaMemcpyHostToDevice, stream));
  stage[slots_ + 1] = (int32_t)order.size();
  HPT_CUDA(cudaMemcpyAsync(&ctrl_->n_order, &stage[slots_ + 1], sizeof(int32_t),
                           cudaMemcpyHostToDevice, stream));
  // The pinned staging is reused by the next call: wait for these copies.
  HPT_CUDA(cudaStreamSynchronize(stream));
  return HPT_OK;
}

hpt_status Engine::admit(const std::vector<int>& slot_ids, const std::vector<DevJob>& jobs,
                         const std::vector<int64_t>& rays, const std::vector<int>& order,
                         const DevScene* shared_scene) {
  const int n = (int)slot_ids.size();
  if (n == 0) return set_order(order);
  {
    hpt_status qs = query_occupancy();
    if (qs != HPT_OK) return qs;
  }
  for (int k = 0; k < n; ++k) {
    if (slot_ids[k] < 0 || slot_ids[k] >= slots_)
      return fail(HPT_ERR_INVALID_ARGUMENT, "slot %d out of range", slot_ids[k]);
    host_jobs_[slot_ids[k]] = jobs[k];
    HPT_CUDA(cudaMemcpyAsync(jobs_ + slot_ids[k], host_jobs_ + slot_ids[k], sizeof(DevJob),
                             cudaMemcpyHostToDevice, stream));
  }
  host_i64_[0] = 0;
  for (int k = 0; k < n; ++k) {
    host_i32_[k] = slot_ids[k];
    host_i64_[k + 1] = host_i64_[k] + rays[k];
  }
  HPT_CUDA(cudaMemcpyAsync(prim_slot_, host_i32_, n * sizeof(int32_t), cudaMemcpyHostToDevice,
                           stream));
  HPT_CUDA(cudaMemcpyAsync(prim_prefix_, host_i64_, (n + 1) * sizeof(int64_t),
                           cudaMemcpyHostToDevice, stream));
  float4* A[8] = {A_o_[0], A_d_[0], A_s_[0], A_r_[0], A_o_[1], A_d_[1], A_s_[1], A_r_[1]};
  float4* R[4] = {R_o_, R_d_, R_s_, R_r_};
  EngineParams P = make_params(*this, ctrl_, jobs_, slot_state_, slots_, order_, quota_slot_,
                               quota_prefix_, prim_slot_, prim_prefix_, n, capacity_, A, A_tri_,
                               A_leaf_, R, shared_scene);
  const size_t smem = launch_smem(P);
  const IsectVariant& v = kIsectVariants[isect_variant()];
  v.primary_kernel(P.trav_steps, P.smem_nodes)<<<num_sms * occ_isect_, v.block, smem, stream>>>(P);
  HPT_CUDA(cudaGetLastError());
  hpt_status s = set_order(order);  // synchronises: the staging is free again
  if (s != HPT_OK) return s;
  k_admit<<<1, 1, 0, stream>>>(P);
  HPT_CUDA(cudaGetLastError());
  return HPT_OK;
}

// --- Asynchronous uploads (serving loop) ------------------------------------
hpt_status Engine::next_staging(StagingSet** out) {
  if (staging_slots_ != slots_) {
    for (StagingSet& st : staging_) {
      if (st.ev) HPT_CUDA(cudaEventSynchronize(st.ev));
      HPT_SOFT(cudaFreeHost(st.jobs));
      HPT_SOFT(cudaFreeHost(st.i32));
      HPT_SOFT(cudaFreeHost(st.i64));
      st.jobs = nullptr;
      st.i32 = nullptr;
      st.i64 = nullptr;
    }
    staging_slots_ = 0;
    const size_t n = (size_t)slots_;
    for (StagingSet& st : staging_) {
      HPT_CUDA(cudaMallocHost(&st.jobs, n * sizeof(DevJob)));
      HPT_CUDA(cudaMallocHost(&st.i32, (3 * n + 3) * sizeof(int32_t)));
      HPT_CUDA(cudaMallocHost(&st.i64, (2 * n + 1) * sizeof(int64_t)));
      if (!st.ev) HPT_CUDA(cudaEventCreateWithFlags(&st.ev, cudaEventDisableTiming));
    }
    staging_slots_ = slots_;
  }
  StagingSet& st = staging_[staging_next_];
  staging_next_ = (staging_next_ + 1) % kStagingRing;
  // The set's previous copies were enqueued kStagingRing uploads ago; wait
  // until they have run before overwriting their source.
  HPT_CUDA(cudaEventSynchronize(st.ev));
  *out = &st;
  return HPT_OK;
}

hpt_status Engine::upload_order(const std::vector<int>& order, StagingSet& st) {
  if ((int)order.size() > slots_) return fail(HPT_ERR_INVALID_ARGUMENT, "order larger than slots");
  int32_t* stage = st.i32 + (slots_ + 1);
  for (size_t k = 0; k < order.size(); ++k) stage[k] = order[k];
  if (!order.empty())
    HPT_CUDA(cudaMemcpyAsync(order_, stage, order.size() * sizeof(int32_t),
                             cudaMemcpyHostToDevice, stream));
  stage[slots_ + 1] = (int32_t)order.size();
  HPT_CUDA(cudaMemcpyAsync(&ctrl_->n_order, &stage[slots_ + 1], sizeof(int32_t),
                           cudaMemcpyHostToDevice, stream));
  return HPT_OK;
}

hpt_status Engine::set_order_async(const std::vector<int>& order) {
  StagingSet* st = nullptr;
  hpt_status s = next_staging(&st);
  if (s != HPT_OK) return s;
  s = upload_order(order, *st);
  if (s != HPT_OK) return s;
  HPT_CUDA(cudaEventRecord(st->ev, stream));
  return HPT_OK;
}

// Uploads n primary-pass entries through a staging set: each entry's job
// into its slot, then the slot list, the ray-count prefix and, with
// `first` / `fin`, the first rays and final flags.
hpt_status Engine::stage_primary(StagingSet& st, int n, const int* slot_ids, const DevJob* jobs,
                                 const int64_t* rays, const int64_t* first, const int* fin) {
  if (n > slots_)
    return fail(HPT_ERR_INVALID_ARGUMENT, "%d primary entries for %d slots", n, slots_);
  for (int k = 0; k < n; ++k) {
    if (slot_ids[k] < 0 || slot_ids[k] >= slots_)
      return fail(HPT_ERR_INVALID_ARGUMENT, "slot %d out of range", slot_ids[k]);
    st.jobs[k] = jobs[k];
    HPT_CUDA(cudaMemcpyAsync(jobs_ + slot_ids[k], st.jobs + k, sizeof(DevJob),
                             cudaMemcpyHostToDevice, stream));
  }
  st.i64[0] = 0;
  // Staging layout: i32 [0, n) slots, [slots + 1, 2 slots + 2] order (see
  // upload_order), [2 slots + 3, + n) final flags; i64 [0, n] prefix,
  // [slots + 1, + n) first rays.
  int32_t* sfin = st.i32 + 2 * slots_ + 3;
  int64_t* sfst = st.i64 + slots_ + 1;
  for (int k = 0; k < n; ++k) {
    st.i32[k] = slot_ids[k];
    st.i64[k + 1] = st.i64[k] + rays[k];
    if (first) {
      sfst[k] = first[k];
      sfin[k] = fin[k];
    }
  }
  HPT_CUDA(cudaMemcpyAsync(prim_slot_, st.i32, n * sizeof(int32_t), cudaMemcpyHostToDevice,
                           stream));
  HPT_CUDA(cudaMemcpyAsync(prim_prefix_, st.i64, (n + 1) * sizeof(int64_t),
                           cudaMemcpyHostToDevice, stream));
  if (first) {
    HPT_CUDA(cudaMemcpyAsync(prim_first_, sfst, n * sizeof(int64_t), cudaMemcpyHostToDevice,
                             stream));
    HPT_CUDA(cudaMemcpyAsync(prim_final_, sfin, n * sizeof(int32_t), cudaMemcpyHostToDevice,
                             stream));
  }
  return HPT_OK;
}

bool Engine::fused_primary() const { return tuning.trav_steps > 0; }

hpt_status Engine::queue_primary(int slot, const DevJob& job, int64_t rays, int64_t first,
                                 bool final_part) {
  if (slot < 0 || slot >= slots_ || rays <= 0 || first < 0)
    return fail(HPT_ERR_INVALID_ARGUMENT, "primary entry: slot %d, %lld rays from %lld", slot,
                (long long)rays, (long long)first);
  for (size_t k = 0; k < pend_slot_.size(); ++k) {
    if (pend_slot_[k] != slot) continue;
    // A later part of the same job, queued before an iteration carried the
    // earlier one: extend that entry.
    if (pend_final_[k] || first != pend_first_[k] + pend_rays_[k])
      return fail(HPT_ERR_INVALID_ARGUMENT, "primary parts of slot %d out of order", slot);
    pend_rays_[k] += rays;
    pend_final_[k] = final_part ? 1 : 0;
    pend_job_[k] = job;
    return HPT_OK;
  }
  pend_slot_.push_back(slot);
  pend_job_.push_back(job);
  pend_rays_.push_back(rays);
  pend_first_.push_back(first);
  pend_final_.push_back(final_part ? 1 : 0);
  return HPT_OK;
}

hpt_status Engine::launch_iteration_async() {
  const int n = (int)pend_slot_.size();
  if (n == 0) {
    launch_iteration(nullptr);
    return HPT_OK;
  }
  if (!fused_primary())
    return fail(HPT_ERR_INVALID_ARGUMENT, "queued primary rays need step-at-a-time traversal");
  hpt_status s = query_occupancy();
  if (s != HPT_OK) return s;
  StagingSet* st = nullptr;
  s = next_staging(&st);
  if (s != HPT_OK) return s;
  s = stage_primary(*st, n, pend_slot_.data(), pend_job_.data(), pend_rays_.data(),
                    pend_first_.data(), pend_final_.data());
  if (s != HPT_OK) return s;
  HPT_CUDA(cudaEventRecord(st->ev, stream));
  pend_slot_.clear();
  pend_job_.clear();
  pend_rays_.clear();
  pend_first_.clear();
  pend_final_.clear();
  float4* A[8] = {A_o_[0], A_d_[0], A_s_[0], A_r_[0], A_o_[1], A_d_[1], A_s_[1], A_r_[1]};
  float4* R[4] = {R_o_, R_d_, R_s_, R_r_};
  EngineParams P = make_params(*this, ctrl_, jobs_, slot_state_, slots_, order_, quota_slot_,
                               quota_prefix_, prim_slot_, prim_prefix_, n, capacity_, A, A_tri_,
                               A_leaf_, R, nullptr);
  P.prim_first = prim_first_;
  P.prim_final = prim_final_;
  shade_kernel(tuning)<<<num_sms * occ_shade_, 256, 0, stream>>>(P);
  const IsectVariant& v = kIsectVariants[isect_variant()];
  v.isect_step_prim<<<num_sms * occ_isect_, v.block, launch_smem(P), stream>>>(P);
  k_ctrl<<<1, 1, 0, stream>>>(P);
  HPT_CUDA(cudaGetLastError());
  return HPT_OK;
}

hpt_status Engine::admit_async(const std::vector<int>& slot_ids, const std::vector<DevJob>& jobs,
                               const std::vector<int64_t>& rays, const std::vector<int>& order,
                               const DevScene* shared_scene, const std::vector<int64_t>& first,
                               const std::vector<int>& final_part) {
  const int n = (int)slot_ids.size();
  if (n == 0) return set_order_async(order);
  hpt_status s = query_occupancy();
  if (s != HPT_OK) return s;
  const bool parts = !first.empty();
  if (parts && ((int)first.size() != n || (int)final_part.size() != n))
    return fail(HPT_ERR_INVALID_ARGUMENT, "primary parts: %d entries, %d firsts, %d flags", n,
                (int)first.size(), (int)final_part.size());
  StagingSet* st = nullptr;
  s = next_staging(&st);
  if (s != HPT_OK) return s;
  s = stage_primary(*st, n, slot_ids.data(), jobs.data(), rays.data(),
                    parts ? first.data() : nullptr, parts ? final_part.data() : nullptr);
  if (s != HPT_OK) return s;
  s = upload_order(order, *st);
  if (s != HPT_OK) return s;
  HPT_CUDA(cudaEventRecord(st->ev, stream));
  float4* A[8] = {A_o_[0], A_d_[0], A_s_[0], A_r_[0], A_o_[1], A_d_[1], A_s_[1], A_r_[1]};
  float4* R[4] = {R_o_, R_d_, R_s_, R_r_};
  EngineParams P = make_params(*this, ctrl_, jobs_, slot_state_, slots_, order_, quota_slot_,
                               quota_prefix_, prim_slot_, prim_prefix_, n, capacity_, A, A_tri_,
                               A_leaf_, R, shared_scene);
  if (parts) {
    P.prim_first = prim_first_;
    P.prim_final = prim_final_;
  }
  const size_t smem = launch_smem(P);
  const IsectVariant& v = kIsectVariants[isect_variant()];
  v.primary_kernel(P.trav_steps, P.smem_nodes)<<<num_sms * occ_isect_, v.block, smem, stream>>>(P);
  k_admit<<<1, 1, 0, stream>>>(P);
  HPT_CUDA(cudaGetLastError());
  return HPT_OK;
}

hpt_status Engine::read_state_async(DevSlot* slots, DevCtrl* ctrl, cudaEvent_t ev) {
  if (slots_ > 0)
    HPT_CUDA(cudaMemcpyAsync(slots, slot_state_, (size_t)slots_ * sizeof(DevSlot),
                             cudaMemcpyDeviceToHost, stream));
  HPT_CUDA(cudaMemcpyAsync(ctrl, ctrl_, sizeof(DevCtrl), cudaMemcpyDeviceToHost, stream));
  HPT_CUDA(cudaEventRecord(ev, stream));
  return HPT_OK;
}

hpt_status Engine::ensure_graph(const DevScene* shared_scene, int iterations) {
  // The key covers the whole shared scene, not just its node array: a scene
  // freed and replaced by one whose nodes land at the same address must not
  // reuse a graph that holds the old scene's other pointers.
  const bool shared = shared_scene != nullptr;
  const bool same_scene =
      graph_shared_ == shared &&
      (!shared || memcmp(&graph_scene_, shared_scene, sizeof(DevScene)) == 0);
  if (graph_exec_ && same_scene && graph_capacity_ == capacity_ &&
      graph_slots_ == slots_ && graph_iters_ == iterations && graph_tuning_ == isect_variant() &&
      graph_smem_ == tuning.smem_nodes && graph_refill_ == tuning.refill_chunk &&
      graph_steps_ == tuning.trav_steps && graph_max_steps_ == tuning.max_steps &&
      graph_shade_ == tuning.shade_min_blocks)
    return HPT_OK;
  if (graph_exec_) {
    HPT_SOFT(cudaGraphExecDestroy(graph_exec_));
    graph_exec_ = nullptr;
  }
  cudaGraph_t g = nullptr;
  HPT_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
  for (int k = 0; k < iterations; ++k) launch_iteration(shared_scene, nullptr);
  const cudaError_t launch = cudaGetLastError();
  const cudaError_t end = cudaStreamEndCapture(stream, &g);
  if (launch != cudaSuccess) {
    if (g) HPT_SOFT(cudaGraphDestroy(g));
    return cuda_fail(launch, "graph capture");
  }
  HPT_CUDA(end);
  const cudaError_t inst = cudaGraphInstantiate(&graph_exec_, g, 0);
  HPT_SOFT(cudaGraphDestroy(g));
  HPT_CUDA(inst);
  graph_shared_ = shared;
  if (shared) graph_scene_ = *shared_scene;
  graph_capacity_ = capacity_;
  graph_slots_ = slots_;
  graph_iters_ = iterations;
  graph_tuning_ = isect_variant();
  graph_smem_ = tuning.smem_nodes;
  graph_refill_ = tuning.refill_chunk;
  graph_steps_ = tuning.trav_steps;
  graph_max_steps_ = tuning.max_steps;
  graph_shade_ = tuning.shade_min_blocks;
  return HPT_OK;
}

void Engine::launch_iteration(const DevScene* shared_scene, cudaEvent_t* ev) {
  float4* A[8] = {A_o_[0], A_d_[0], A_s_[0], A_r_[0], A_o_[1], A_d_[1], A_s_[1], A_r_[1]};
  float4* R[4] = {R_o_, R_d_, R_s_, R_r_};
  EngineParams P = make_params(*this, ctrl_, jobs_, slot_state_, slots_, order_, quota_slot_,
                               quota_prefix_, prim_slot_, prim_prefix_, 0, capacity_, A, A_tri_,
                               A_leaf_, R, shared_scene);
  if (ev) HPT_SOFT(cudaEventRecord(ev[0], stream));
  shade_kernel(tuning)<<<num_sms * occ_shade_, 256, 0, stream>>>(P);
  if (ev) HPT_SOFT(cudaEventRecord(ev[1], stream));
  const size_t smem = launch_smem(P);
  const IsectVariant& v = kIsectVariants[isect_variant()];
  v.isect_kernel(P.trav_steps, P.smem_nodes)<<<num_sms * occ_isect_, v.block, smem, stream>>>(P);
  if (ev) HPT_SOFT(cudaEventRecord(ev[2], stream));
  k_ctrl<<<1, 1, 0, stream>>>(P);
}

void Engine::launch_resolve(int slot, const JobSpec& js, const JobBuffers& b, float samples) {
  const hpt_render_params& p = js.params;
  dim3 blk(16, 16), grd((p.sample_x + 15) / 16, (p.sample_y + 15) / 16);
  k_resolve<<<grd, blk, 0, stream>>>(jobs_ + slot, p.sample_x, p.sample_y, p.supersample_x,
                                      p.supersample_y, samples > 0.f ? samples : (float)p.sample,
                                      p.brightness, b.rgba, b.accum_f);
}

hpt_status Engine::read_slots(std::vector<DevSlot>& out) {
  out.resize(slots_);
  if (slots_ == 0) return HPT_OK;
  HPT_CUDA(cudaMemcpyAsync(slots_host_, slot_state_, (size_t)slots_ * sizeof(DevSlot),
                           cudaMemcpyDeviceToHost, stream));
  HPT_CUDA(cudaStreamSynchronize(stream));
  std::copy(slots_host_, slots_host_ + slots_, out.begin());
  return HPT_OK;
}

hpt_status Engine::read_state(std::vector<DevSlot>& slots, DevCtrl* ctrl) {
  slots.resize(slots_);
  if (slots_ > 0)
    HPT_CUDA(cudaMemcpyAsync(slots_host_, slot_state_, (size_t)slots_ * sizeof(DevSlot),
                             cudaMemcpyDeviceToHost, stream));
  HPT_CUDA(cudaMemcpyAsync(ctrl_host_, ctrl_, sizeof(DevCtrl), cudaMemcpyDeviceToHost, stream));
  HPT_CUDA(cudaStreamSynchronize(stream));
  std::copy(slots_host_, slots_host_ + slots_, slots.begin());
  *ctrl = *ctrl_host_;
  return HPT_OK;
}

hpt_status Engine::reserve_pool(size_t bytes) {
  if (bytes == 0) return HPT_OK;
  uint64_t keep = 0;
  HPT_CUDA(cudaMemPoolGetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep));
  if (keep < bytes) {
    keep = bytes;
    HPT_CUDA(cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  void* p = nullptr;
  HPT_CUDA(cudaMallocFromPoolAsync(&p, bytes, pool_, stream));
  HPT_CUDA(cudaFreeAsync(p, stream));
  HPT_CUDA(cudaStreamSynchronize(stream));
  return HPT_OK;
}

hpt_status Engine::set_capped_budget(int64_t paths) {
  ctrl_host_->capped_budget = paths;
  HPT_CUDA(cudaMemcpyAsync(&ctrl_->capped_budget, &ctrl_host_->capped_budget, sizeof(int64_t),
                           cudaMemcpyHostToDevice, stream));
  HPT_CUDA(cudaStreamSynchronize(stream));
  return HPT_OK;
}

hpt_status Engine::read_ctrl(DevCtrl* out) {
  HPT_CUDA(cudaMemcpyAsync(ctrl_host_, ctrl_, sizeof(DevCtrl), cudaMemcpyDeviceToHost, stream));
  HPT_CUDA(cudaStreamSynchronize(stream));
  *out = *ctrl_host_;
  return HPT_OK;
}

hpt_status Engine::run(const std::vector<JobSpec>& jobs, hpt_render_stats* stats) {
  if (init_status_ != HPT_OK) return fail(init_status_, "engine set-up failed");
  HPT_CUDA(cudaSetDevice(device));
  if (jobs.empty()) return HPT_OK;
  // The wavefront never holds more paths than the run has, so the queues
  // are sized to the smaller of the tuning's capacity and the run's paths
  // (results do not depend on the capacity: fixed-point sums, counter RNG).
  int64_t paths = 0;
  for (const JobSpec& js : jobs) {
    const hpt_render_params& p = js.params;
    paths += (int64_t)p.sample_x * p.supersample_x * p.sample_y * p.supersample_y * p.sample;
  }
  hpt_status s = ensure_capacity(
      (int)std::max<int64_t>(1024, std::min<int64_t>(tuning.capacity, paths)));
  if (s != HPT_OK) return s;
  s = ensure_slots((int)jobs.size());
  if (s != HPT_OK) return s;
  const int n = (int)jobs.size();
  std::vector<JobBuffers> bufs(n);
  std::vector<DevJob> djobs;
  std::vector<int> slot_ids(n);
  std::vector<int64_t> rays(n);
  const SceneDev* shared = jobs[0].scene;
  for (int j = 0; j < n; ++j) {
    s = alloc_job(jobs[j], jobs[j].accum_out != nullptr, bufs[j]);
    if (s != HPT_OK) {
      for (int k = 0; k <= j; ++k) free_job(bufs[k]);
      return s;
    }
    djobs.push_back(make_job(jobs[j], bufs[j]));
    slot_ids[j] = j;
    rays[j] = bufs[j].rays;
    if (jobs[j].scene != shared) shared = nullptr;
  }
  // Smallest jobs first.
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return rays[a] * jobs[a].params.sample < rays[b] * jobs[b].params.sample;
  });
  const DevScene* shared_dev = shared ? &shared->dev : nullptr;
  reset_ctrl();
  HPT_SOFT(cudaEventRecord(ev_[0], stream));
  s = admit(slot_ids, djobs, rays, order, shared_dev);
  if (s != HPT_OK) {
    for (auto& b : bufs) free_job(b);
    HPT_SOFT(cudaStreamSynchronize(stream));
    return s;
  }
  HPT_SOFT(cudaEventRecord(ev_[1], stream));
  // Iterate until the device says the wavefront is drained. Batches of
  // iterations are queued ahead; the done flag of batch k is checked while
  // batch k+1 runs (extra iterations after completion are empty launches).
  const int kBatch = 4;
  const bool prof = tuning.profile != 0;
  int32_t* done_host = done_host_;
  done_host[0] = done_host[1] = 0;
  cudaEvent_t* ev_done = ev_done_;
  std::vector<cudaEvent_t>& pev = pev_;
  if (prof && pev.empty()) {
    pev.resize(2 * kBatch * 3);
    for (auto& e : pev) HPT_CUDA(cudaEventCreate(&e));
  }
  float ms_shade = 0.f, ms_isect = 0.f;
  auto harvest = [&](int sl) {
    for (int k = 0; k < kBatch; ++k) {
      cudaEvent_t* e = &pev[(sl * kBatch + k) * 3];
      float a = 0.f, b = 0.f;
      HPT_SOFT(cudaEventElapsedTime(&a, e[0], e[1]));
      HPT_SOFT(cudaEventElapsedTime(&b, e[1], e[2]));
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
  // With use_graph, the kBatch iterations are replayed from one CUDA graph
  // (their parameters live in device memory, so one capture serves every
  // batch); it is captured again when the queues, the slot table or the
  // shared-scene prefix change. Profiling needs per-kernel events: eager.
  const bool use_graph = tuning.use_graph != 0 && !prof;
  if (use_graph) {
    s = ensure_graph(shared_dev, kBatch);
    if (s != HPT_OK) {
      for (auto& b : bufs) free_job(b);
      HPT_SOFT(cudaStreamSynchronize(stream));
      return s;
    }
  }
  int64_t guard = 0;
  bool drained = false;
  int slot = 0;
  bool pending = false;
  while (true) {
    if (use_graph) {
      HPT_CUDA(cudaGraphLaunch(graph_exec_, stream));
    } else {
      for (int k = 0; k < kBatch; ++k)
        launch_iteration(shared_dev, prof ? &pev[(slot * kBatch + k) * 3] : nullptr);
    }
    HPT_SOFT(cudaMemcpyAsync(&done_host[slot], &ctrl_->done, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
    HPT_SOFT(cudaEventRecord(ev_done[slot], stream));
    if (pending) {
      HPT_SOFT(cudaEventSynchronize(ev_done[slot ^ 1]));
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
  HPT_SOFT(cudaEventRecord(ev_[2], stream));
  for (int j = 0; j < n; ++j) launch_resolve(j, jobs[j], bufs[j]);
  HPT_SOFT(cudaEventRecord(ev_[3], stream));
  for (int j = 0; j < n; ++j) {
    const hpt_render_params& p = jobs[j].params;
    if (jobs[j].rgba_out)
      HPT_SOFT(cudaMemcpyAsync(jobs[j].rgba_out, bufs[j].rgba, (size_t)p.sample_x * p.sample_y * 4, cudaMemcpyDeviceToHost, stream));
    if (jobs[j].accum_out)
      HPT_SOFT(cudaMemcpyAsync(jobs[j].accum_out, bufs[j].accum_f, (size_t)bufs[j].rays * 3 * sizeof(float), cudaMemcpyDeviceToHost, stream));
  }
  HPT_SOFT(cudaMemcpyAsync(ctrl_host_, ctrl_, sizeof(DevCtrl), cudaMemcpyDeviceToHost, stream));
  for (auto& b : bufs) free_job(b);
  cudaError_t e = cudaStreamSynchronize(stream);
  if (prof) harvest(slot);
  if (e != cudaSuccess) return cuda_fail(e, "render");
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "render launch");
  int64_t prim = 0;
  for (int64_t r : rays) prim += r;
  if (stats) {
    memset(stats, 0, sizeof *stats);
    stats->primary_rays = prim;
    stats->intersect_queries = (int64_t)ctrl_host_->isect_queries;
    stats->shade_calls = (int64_t)ctrl_host_->shades;
    stats->iterations = (int32_t)ctrl_host_->iterations;
    stats->error_flags = (int32_t)ctrl_host_->err.flags;
    HPT_SOFT(cudaEventElapsedTime(&stats->ms_total, ev_[0], ev_[3]));
    HPT_SOFT(cudaEventElapsedTime(&stats->ms_primary, ev_[0], ev_[1]));
    HPT_SOFT(cudaEventElapsedTime(&stats->ms_loop, ev_[1], ev_[2]));
    stats->ms_shade = prof ? ms_shade : -1.f;
    stats->ms_intersect = prof ? ms_isect : -1.f;
    HPT_SOFT(cudaEventElapsedTime(&stats->ms_resolve, ev_[2], ev_[3]));
    stats->nodes_visited = (int64_t)ctrl_host_->nodes_visited;
    stats->leaves_visited = (int64_t)ctrl_host_->leaves_visited;
    stats->triangle_tests = (int64_t)ctrl_host_->tri_tests;
    stats->triangle_repeats = (int64_t)ctrl_host_->tri_repeats;
    std::vector<DevSlot> st(n);
    const cudaError_t ce =
        cudaMemcpy(st.data(), slot_state_, n * sizeof(DevSlot), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) cuda_soft_fail(ce, "slot state read-back");
    if (ce == cudaSuccess) {
      int64_t paths = 0;
      for (const DevSlot& x : st) paths += x.num_paths;
      stats->paths = paths;
    }
  }
  if (ctrl_host_->err.flags & 2u)
    return fail(HPT_ERR_INVALID_SCENE, "device self-check %d failed (value %lld)",
                ctrl_host_->err.site, (long long)ctrl_host_->err.value);
  if (ctrl_host_->err.flags & 1u)
    return fail(HPT_ERR_TRAVERSAL_LIMIT, "a traversal hit its step cap");
  if (!drained && !ctrl_host_->done)
    return fail(HPT_ERR_TRAVERSAL_LIMIT, "the wavefront did not drain within %lld iterations",
                (long long)(max_batches * kBatch));
  return HPT_OK;
}

}  // namespace hpt
