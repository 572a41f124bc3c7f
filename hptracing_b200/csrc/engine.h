// Host-side objects behind the C ABI: device-resident scenes and the
// wavefront engine that renders one or many jobs.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <mutex>
#include <vector>

#include "device_types.h"
#include "host.h"

namespace hpt {

// Largest shared-memory node prefix a tuning may ask for (64 KB).
constexpr int kMaxSmemNodes = 8192;

struct SceneDev {
  int device = 0;
  DevScene dev;              // device pointers (host copy)
  DevScene* d_scene = nullptr;  // device copy (for stage kernels)
  std::vector<void*> allocations;
  hpt_scene_info info{};
  int64_t bytes = 0;
};

// One render request.
struct JobSpec {
  const SceneDev* scene = nullptr;
  hpt_camera camera{};
  hpt_render_params params{};
  uint8_t* rgba_out = nullptr;   // host, may be null
  float* accum_out = nullptr;    // host, may be null
};

// Per-job device buffers (owned by the engine while the job runs).
struct JobBuffers {
  unsigned long long* accum = nullptr;  // 3 per ray, fixed point
  uint32_t* flags = nullptr;            // non-finite markers per ray
  float* prim = nullptr;                // primary hit cache
  int32_t* prim_count = nullptr;
  uint8_t* rgba = nullptr;
  float* accum_f = nullptr;
  int64_t rays = 0;
  int64_t bytes = 0;
};

// Device bytes a job needs besides the shared wavefront (admission control).
int64_t job_footprint(const hpt_render_params& p, bool want_accum);

class Engine {
 public:
  explicit Engine(int device);
  ~Engine();

  // Renders all jobs in one wavefront: primary pass for every job, then the
  // paths of all jobs share the queues (smallest job first).
  hpt_status run(const std::vector<JobSpec>& jobs, hpt_render_stats* stats);

  hpt_tuning tuning;
  int device;
  cudaStream_t stream = nullptr;
  int num_sms = 0;

  // --- building blocks (also used by the server) --------------------------
  hpt_status ensure_capacity(int capacity);
  hpt_status ensure_slots(int slots);
  int slots() const { return slots_; }
  hpt_status alloc_job(const JobSpec& js, bool want_accum, JobBuffers& b);
  void free_job(JobBuffers& b);
  DevJob make_job(const JobSpec& js, const JobBuffers& b) const;
  // Stream-ordered: writes the jobs into their slots, runs their primary
  // pass and grants them paths. `order` lists every active slot, highest
  // priority first.
  hpt_status admit(const std::vector<int>& slot_ids, const std::vector<DevJob>& jobs,
                   const std::vector<int64_t>& rays, const std::vector<int>& order,
                   const DevScene* shared_scene);
  hpt_status set_order(const std::vector<int>& order);
  // Asynchronous forms for a serving loop: the uploads go through a ring of
  // pinned staging sets and nothing waits for the stream (only, rarely, for
  // a staging set's previous copies to have run).
  // With `first` and `final_part` (one entry per slot), entry k traces rays
  // [first[k], first[k] + rays[k]) of its job, and only an entry with
  // final_part[k] != 0 starts the job's paths: a large job's primary pass
  // can be split over several calls (same slot, same job, consecutive
  // ranges, the last one final) so that no single launch stalls the
  // iterations of the others for long.
  hpt_status admit_async(const std::vector<int>& slot_ids, const std::vector<DevJob>& jobs,
                         const std::vector<int64_t>& rays, const std::vector<int>& order,
                         const DevScene* shared_scene, const std::vector<int64_t>& first = {},
                         const std::vector<int>& final_part = {});
  hpt_status set_order_async(const std::vector<int>& order);
  // Serving loop: a newly admitted job's camera rays can instead be traced
  // inside the next iteration's traversal launch (fused_primary(): the
  // tuning traverses step at a time), so that admissions add no launch of
  // their own. queue_primary() records rays [first, first + rays) of the
  // job in `slot` (parts of one job in order; final_part on the last, which
  // starts its paths); launch_iteration_async() uploads what was queued and
  // launches one iteration that carries it.
  bool fused_primary() const;
  hpt_status queue_primary(int slot, const DevJob& job, int64_t rays, int64_t first,
                           bool final_part);
  hpt_status launch_iteration_async();
  // Enqueues a copy of the slot table and control block into pinned host
  // memory and records ev after it.
  hpt_status read_state_async(DevSlot* slots, DevCtrl* ctrl, cudaEvent_t ev);
  void launch_iteration(const DevScene* shared_scene, cudaEvent_t* ev3 = nullptr);
  // Captures `iterations` consecutive iterations into graph_exec_ (kept
  // until the queues, slots, shared scene or tuning change).
  hpt_status ensure_graph(const DevScene* shared_scene, int iterations);
  // samples: the divisor of the accumulated radiance (<= 0: params.sample).
  void launch_resolve(int slot, const JobSpec& js, const JobBuffers& b, float samples = 0.f);
  // Synchronous read-back of the slot table / control block.
  hpt_status read_slots(std::vector<DevSlot>& out);
  hpt_status read_ctrl(DevCtrl* out);
  // Maps `bytes` of device memory into the job-buffer pool now and keeps
  // it there, so later job allocations do not map memory (which blocks the
  // host) on their way.
  hpt_status reserve_pool(size_t bytes);
  // Shared in-flight budget of the capped slots (reset_ctrl clears it).
  hpt_status set_capped_budget(int64_t paths);
  hpt_status read_state(std::vector<DevSlot>& slots, DevCtrl* ctrl);  // one sync
  void reset_ctrl();
  DevCtrl* ctrl_dev() const { return ctrl_; }
  DevSlot* slots_dev() const { return slot_state_; }
  int isect_variant() const;  // index into the traversal kernel variants

 private:
  int capacity_ = 0;
  int slots_ = 0;
  DevCtrl* ctrl_ = nullptr;
  DevCtrl* ctrl_host_ = nullptr;  // pinned
  DevJob* jobs_ = nullptr;
  DevSlot* slot_state_ = nullptr;
  int32_t* order_ = nullptr;
  int32_t* quota_slot_ = nullptr;
  int32_t* quota_prefix_ = nullptr;
  int32_t* prim_slot_ = nullptr;
  int64_t* prim_prefix_ = nullptr;
  int64_t* prim_first_ = nullptr;
  int32_t* prim_final_ = nullptr;
  int32_t* host_i32_ = nullptr;   // pinned staging for small uploads
  int64_t* host_i64_ = nullptr;
  DevJob* host_jobs_ = nullptr;
  DevSlot* slots_host_ = nullptr;  // pinned mirror for read_slots
  // Shade queues (double-buffered) and the intersect queue.
  float4* A_o_[2] = {nullptr, nullptr};
  float4* A_d_[2] = {nullptr, nullptr};
  float4* A_s_[2] = {nullptr, nullptr};
  float4* A_r_[2] = {nullptr, nullptr};
  int32_t* A_tri_[2] = {nullptr, nullptr};
  int32_t* A_leaf_[2] = {nullptr, nullptr};
  float4* R_o_ = nullptr;
  float4* R_d_ = nullptr;
  float4* R_s_ = nullptr;
  float4* R_r_ = nullptr;
  cudaEvent_t ev_[6];
  cudaEvent_t ev_done_[2] = {nullptr, nullptr};
  std::vector<cudaEvent_t> pev_;  // profiling events, created on first use
  int32_t* done_host_ = nullptr;  // pinned drain flags (double-buffered)
  cudaMemPool_t pool_ = nullptr;  // per-job buffers
  struct StagingSet {
    DevJob* jobs = nullptr;
    int32_t* i32 = nullptr;
    int64_t* i64 = nullptr;
    cudaEvent_t ev = nullptr;
  };
  static constexpr int kStagingRing = 8;
  StagingSet staging_[kStagingRing];
  int staging_next_ = 0, staging_slots_ = 0;
  hpt_status next_staging(StagingSet** out);
  hpt_status upload_order(const std::vector<int>& order, StagingSet& st);
  hpt_status stage_primary(StagingSet& st, int n, const int* slot_ids, const DevJob* jobs,
                           const int64_t* rays, const int64_t* first, const int* fin);
  std::vector<int> pend_slot_, pend_final_;
  std::vector<DevJob> pend_job_;
  std::vector<int64_t> pend_rays_, pend_first_;
  cudaGraphExec_t graph_exec_ = nullptr;
  // The one scene the captured iterations were launched with (its pointers
  // and sizes are baked into the graph's kernel parameters), if any.
  bool graph_shared_ = false;
  DevScene graph_scene_{};
  int graph_capacity_ = 0, graph_slots_ = 0, graph_iters_ = 0, graph_tuning_ = -1;
  int graph_smem_ = -1, graph_refill_ = -1, graph_steps_ = -1, graph_max_steps_ = -1;
  int graph_shade_ = -1;
  hpt_status init_status_ = HPT_OK;
  hpt_status init();
  int occ_isect_ = 1, occ_shade_ = 1;
  bool occ_done_ = false;
  hpt_status query_occupancy();
};

struct SceneHandle {
  SceneDev scene;
  std::mutex mu;
  std::unique_ptr<Engine> engine;
  hpt_render_stats last_stats{};
  hpt_tuning tuning{};
};

hpt_status upload_scene(const hpt_scene_desc& desc, SceneDev& out);
void release_scene(SceneDev& s);
hpt_tuning default_tuning();
DevScene capped_scene(const DevScene& s, const hpt_tuning& t);
hpt_status check_render_params(const hpt_camera* cam, const hpt_render_params* p);

// CUDA error -> hpt_status with message.
hpt_status cuda_fail(cudaError_t e, const char* what);
#define HPT_CUDA(call)                                      \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return ::hpt::cuda_fail(e_, #call); \
  } while (0)

// Best-effort call (teardown, timing, stream-ordered frees): its error is
// not returned, but it is cleared from the runtime's per-thread error state
// so that a later launch check does not report it as its own. Self-check
// builds print it.
void cuda_soft_fail(cudaError_t e, const char* what);
#define HPT_SOFT(call)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) ::hpt::cuda_soft_fail(e_, #call); \
  } while (0)

}  // namespace hpt

// The opaque scene handle of the C ABI.
struct hpt_scene {
  hpt::SceneHandle h;
};
