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

struct SceneDev {
  int device = 0;
  DevScene dev;              // device pointers (host copy)
  DevScene* d_scene = nullptr;  // device copy (for stage kernels)
  std::vector<void*> allocations;
  hpt_scene_info info{};
  int64_t bytes = 0;
};

// One render request inside a wavefront run.
struct JobSpec {
  const SceneDev* scene = nullptr;
  hpt_camera camera{};
  hpt_render_params params{};
  uint8_t* rgba_out = nullptr;   // host, may be null
  float* accum_out = nullptr;    // host, may be null
};

// Per-job device buffers, owned by the engine for the duration of a run
// (or of a request in the server).
struct JobBuffers {
  unsigned long long* accum = nullptr;  // 3 per ray, fixed point
  uint32_t* flags = nullptr;            // non-finite markers per ray
  float* prim = nullptr;                // primary hit cache
  int32_t* prim_count = nullptr;
  unsigned long long* counters = nullptr;
  uint8_t* rgba = nullptr;
  float* accum_f = nullptr;
  int64_t rays = 0;
  int64_t bytes = 0;
};

class Engine {
 public:
  explicit Engine(int device);
  ~Engine();

  // Renders all jobs in one wavefront (primary pass for all jobs, then
  // paths of every job interleaved in the same queues).
  hpt_status run(const std::vector<JobSpec>& jobs, hpt_render_stats* stats);

  hpt_tuning tuning;
  int device;
  cudaStream_t stream = nullptr;
  int num_sms = 0;

  // --- pieces shared with the server ------------------------------------
  hpt_status ensure_capacity(int capacity);
  hpt_status alloc_job(const JobSpec& js, bool want_accum, JobBuffers& b);
  void free_job(JobBuffers& b);
  DevJob make_job(const JobSpec& js, const JobBuffers& b, int64_t prim_base) const;
  // Enqueue helpers (stream-ordered, no sync).
  hpt_status upload_jobs(const std::vector<DevJob>& jobs);
  void launch_primary(int64_t total_primary, const DevScene* shared_scene);
  void launch_setup(int num_jobs, bool reset_cursor);
  void launch_iteration(const DevScene* shared_scene, cudaEvent_t* ev3 = nullptr);
  DevCtrl* ctrl_dev() const { return ctrl_; }
  DevJob* jobs_dev() const { return jobs_; }
  int num_jobs_dev() const { return num_jobs_; }

 private:
  int capacity_ = 0;
  DevCtrl* ctrl_ = nullptr;
  DevCtrl* ctrl_host_ = nullptr;  // pinned
  DevJob* jobs_ = nullptr;
  int jobs_cap_ = 0;
  int num_jobs_ = 0;
  // Shade queues (double-buffered) and the intersect queue.
  float4* A_o_[2] = {nullptr, nullptr};
  float4* A_d_[2] = {nullptr, nullptr};
  float4* A_s_[2] = {nullptr, nullptr};
  float4* A_r_[2] = {nullptr, nullptr};
  int32_t* A_tri_[2] = {nullptr, nullptr};
  float4* R_o_ = nullptr;
  float4* R_d_ = nullptr;
  float4* R_s_ = nullptr;
  float4* R_r_ = nullptr;
  cudaEvent_t ev_[6];
  int occ_isect_ = 1, occ_shade_ = 1;
  bool occ_done_ = false;
  void query_occupancy();
};

struct SceneHandle {
  SceneDev scene;
  std::mutex mu;
  std::unique_ptr<Engine> engine;
  hpt_render_stats last_stats{};
  hpt_tuning tuning{};
  bool tuning_set = false;
};

hpt_status upload_scene(const hpt_scene_desc& desc, SceneDev& out);
void release_scene(SceneDev& s);
hpt_tuning default_tuning();

// CUDA error -> hpt_status with message.
hpt_status cuda_fail(cudaError_t e, const char* what);
#define HPT_CUDA(call)                                      \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return ::hpt::cuda_fail(e_, #call); \
  } while (0)

}  // namespace hpt
