// Serving loop and autotuner. Neither has a reference counterpart: the
// reference re-runs TraceRunner::run for every camera move of its GLUT loop
// (src/hptracing.cpp:124-211), one frame at a time.
//
// Serving is continuous batching over the engine's job slots: requests
// against device-resident scenes wait in a queue, are admitted as soon as a
// slot and their device footprint (ray state, accumulators, image) fit,
// share one wavefront with every request already running (smallest
// remaining work first), and are resolved and copied back when their last
// path finishes. Random streams are keyed by (request seed, ray, sample,
// bounce) and radiance is summed in fixed point, so a request's image is
// bit-identical whether it runs alone or in any mix.
//
// The pump never waits for the GPU in the steady state: it keeps up to
// `pipeline_depth` wavefront iterations queued, each followed by an
// asynchronous copy of the slot table into a ring of pinned buffers; it
// admits requests and updates the priority order through pinned staging
// on the same stream; finished requests are resolved into pinned output
// buffers and marked done when that copy's event has completed. A read-back
// is only applied to requests admitted before it was recorded.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <deque>
#include <fstream>
#include <iterator>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/hpt.h"
#include "engine.h"

using namespace hpt;

// Diagnostic build only (-DHPT_SERVER_TRACE): report pump phases that take
// longer than 20 ms on stderr.
#ifdef HPT_SERVER_TRACE
#define HPT_TRACE_BEGIN(name) const auto trace_t0_##name = std::chrono::steady_clock::now()
#define HPT_TRACE_END(name)                                                                  \
  do {                                                                                       \
    const double ms = std::chrono::duration<double, std::milli>(                             \
                          std::chrono::steady_clock::now() - trace_t0_##name)                \
                          .count();                                                          \
    if (ms > 20.0) fprintf(stderr, "hpt server: %s took %.1f ms\n", #name, ms);             \
  } while (0)
#else
#define HPT_TRACE_BEGIN(name) (void)0
#define HPT_TRACE_END(name) (void)0
#endif

namespace {

enum RequestState { kQueued = 0, kRunning = 1, kDone = 2, kFailed = 3, kCancelled = 4 };

struct Request {
  uint64_t id = 0;
  JobSpec js;
  int scene_slot = 0;
  bool small = true;        // rays x spp <= capacity: latency-bound
  bool shed = false;        // dropped by the overload policy
  int state = kQueued;
  int slot = -1;
  bool want_accum = true;
  bool cancel = false;
  bool finishing = false;   // resolve and copy-back enqueued
  cudaEvent_t fin_ev = nullptr;
  uint64_t admit_seq = 0;   // iterations launched before its primary pass completed
  int64_t prim_next = 0;    // rays whose primary pass has been enqueued
  DevJob dj{};              // the job as admitted (for the later parts of its primary pass)
  JobBuffers buf;
  int64_t footprint = 0;
  int64_t rays = 0;
  int64_t paths = -1;       // hits * spp, known after the primary pass
  int64_t done_paths = 0;
  int64_t queries = 0;
  double submit_ms = 0, admit_ms = 0, done_ms = 0;
  double due_ms = -1;       // completion the overload policy predicted at admission
  bool alone = false;       // admitted while no other latency-bound request ran
  double drift_ms = 0;      // the server's prediction drift when it was admitted
  hpt_status error = HPT_OK;
  uint8_t* rgba = nullptr;  // pinned, from the server's pool
  float* accum = nullptr;
  size_t rgba_bytes = 0, accum_bytes = 0;
};

// One asynchronous read-back of the slot table and control block.
struct Readback {
  DevSlot* slots = nullptr;  // pinned
  DevCtrl* ctrl = nullptr;   // pinned
  cudaEvent_t ev = nullptr;
  uint64_t seq = 0;          // iterations launched before it was recorded
  bool pending = false;
};

constexpr int kReadbacks = 8;

}  // namespace

struct hpt_server {
  hpt_server_config cfg{};
  std::unique_ptr<Engine> engine;
  std::vector<hpt_scene*> scenes;
  std::mutex mu;
  std::map<uint64_t, std::unique_ptr<Request>> reqs;
  std::deque<uint64_t> queue;
  std::vector<uint64_t> slot_req;  // slot -> request id holding it, 0 = free
  int64_t used_bytes = 0;
  uint64_t next_id = 1;
  std::chrono::steady_clock::time_point t0;
  Readback rb[kReadbacks];
  int rb_fill = 0, rb_drain = 0, rb_pending = 0;
  uint64_t launched = 0;
  int depth = 2;
  DevCtrl ctrl_view{};
  std::vector<uint64_t> finished_ids;  // since the last hpt_server_drain_completed
  std::multimap<size_t, void*> pinned_pool;  // free pinned output buffers by size
  // Pinned host memory for results, pinned at creation (cudaMallocHost in
  // the middle of a stream stalls the pump for milliseconds): a first-fit
  // arena in 4 KB units; cudaMallocHost only once it is full.
  uint8_t* arena = nullptr;
  size_t arena_bytes = 0;
  std::map<size_t, size_t> arena_free;  // offset -> length of each free range
  std::vector<cudaEvent_t> event_pool;
  int64_t completed = 0;
  int64_t pumps = 0;
  // Overload policy (cfg.deadline_ms > 0). Per scene and request size, two
  // service times of a latency-bound request, each an upper quantile of
  // recent observations:
  // `alone` = completion minus admission for one admitted while no other
  // latency-bound request was running, `gap` = completion minus the previous
  // latency-bound completion for one admitted behind others. -1 = not
  // measured yet.
  struct ServiceEstimate {
    double alone = -1, gap = -1;
    bool probing = false;  // the first request of this scene and size is running
  };
  std::vector<ServiceEstimate> est;
  double last_small_done_ms = 0;
  double tail_ms = 0;  // predicted completion of the latest admitted latency-bound request
  double drift_ms = 0;  // sum of the corrections applied to the predictions so far
  // Fraction of the deadline that admissions aim at: cut by 15 % whenever a
  // served latency-bound request finishes late, raised by 0.001 when one
  // finishes in time, so that about one in a hundred finishes late.
  double slack = 1.0;
  int64_t shed = 0;
  // Camera rays of large requests queued since the last iteration launch.
  int64_t large_queued = 0;

  double now_ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
        .count();
  }
  Request* find(uint64_t id) {
    auto it = reqs.find(id);
    return it == reqs.end() ? nullptr : it->second.get();
  }
  bool running() const {
    for (size_t k = 0; k < slot_req.size(); ++k)
      if (slot_req[k] && !reqs.at(slot_req[k])->finishing) return true;
    return false;
  }
  // Slots still computing in grant order: smallest remaining work first;
  // under the overload policy, latency-bound requests first-come
  // first-served ahead of all larger ones.
  std::vector<int> order() const {
    std::vector<std::pair<std::pair<int64_t, int64_t>, int>> v;
    for (size_t k = 0; k < slot_req.size(); ++k) {
      if (!slot_req[k]) continue;
      const Request* r = reqs.at(slot_req[k]).get();
      if (r->finishing) continue;
      const int64_t total = r->paths >= 0 ? r->paths : r->rays * r->js.params.sample;
      if (cfg.deadline_ms > 0)
        v.push_back({{r->small ? 0 : 1, r->small ? (int64_t)r->id : total - r->done_paths},
                     (int)k});
      else
        v.push_back({{0, total - r->done_paths}, (int)k});
    }
    std::stable_sort(v.begin(), v.end());
    std::vector<int> o;
    for (auto& p : v) o.push_back(p.second);
    return o;
  }
  // Estimates are kept per scene and per request size (paths = rays x
  // spp, by power of two): a 128x128 1-spp request says little about a
  // 512x512 4-spp one on the same scene.
  ServiceEstimate& estimate(const Request* r) {
    const int64_t paths = std::max<int64_t>(1, r->rays * r->js.params.sample);
    int bucket = 0;
    while (bucket < 62 && ((int64_t)1 << (bucket + 1)) <= paths) ++bucket;
    const size_t key = (size_t)r->scene_slot * 64 + bucket;
    if (est.size() <= key) est.resize(key + 1);
    return est[key];
  }
  // Latency-bound requests admitted and not yet retired.
  bool small_running() const {
    for (size_t k = 0; k < slot_req.size(); ++k)
      if (slot_req[k] && reqs.at(slot_req[k])->small) return true;
    return false;
  }
  static size_t arena_units(size_t bytes) { return (bytes + 4095) & ~(size_t)4095; }
  bool in_arena(const void* p) const {
    return arena && p >= arena && static_cast<const uint8_t*>(p) < arena + arena_bytes;
  }
  hpt_status take_pinned(size_t bytes, void** out) {
    const size_t len = arena_units(bytes);
    for (auto it = arena_free.begin(); it != arena_free.end(); ++it) {
      if (it->second < len) continue;
      const size_t off = it->first, rest = it->second - len;
      arena_free.erase(it);
      if (rest) arena_free[off + len] = rest;
      *out = arena + off;
      return HPT_OK;
    }
    auto it = pinned_pool.find(bytes);
    if (it != pinned_pool.end()) {
      *out = it->second;
      pinned_pool.erase(it);
      return HPT_OK;
    }
    HPT_CUDA(cudaMallocHost(out, bytes));
    return HPT_OK;
  }
  void give_pinned(void* p, size_t bytes) {
    if (!p) return;
    if (!in_arena(p)) {
      pinned_pool.insert({bytes, p});
      return;
    }
    size_t off = static_cast<uint8_t*>(p) - arena, len = arena_units(bytes);
    auto next = arena_free.lower_bound(off);
    if (next != arena_free.end() && next->first == off + len) {  // merge with the range after
      len += next->second;
      next = arena_free.erase(next);
    }
    if (next != arena_free.begin()) {  // and with the range before
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        prev->second += len;
        return;
      }
    }
    arena_free[off] = len;
  }
  void free_pinned(void* p) {
    if (p && !in_arena(p)) HPT_SOFT(cudaFreeHost(p));
  }
  hpt_status take_event(cudaEvent_t* ev) {
    if (!event_pool.empty()) {
      *ev = event_pool.back();
      event_pool.pop_back();
      return HPT_OK;
    }
    HPT_CUDA(cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
    return HPT_OK;
  }
  hpt_status admit_pending();
  hpt_status apply_readback(Readback& b);
  hpt_status finish(Request* r);
  hpt_status retire_finished();
};

// Moves queued requests into free slots while the memory budget allows
// (first fit in arrival order) and enqueues their primary pass.
hpt_status hpt_server::admit_pending() {
  std::vector<int> ids;
  std::vector<DevJob> jobs;
  std::vector<int64_t> rays, first;
  std::vector<int> final_part;
  const double now = now_ms();
  // A latency-bound request's camera rays are traced whole at admission. A
  // large request's are traced in parts, at most its in-flight share of the
  // wavefront (large_inflight_pct, else a quarter) of rays per iteration for
  // all large requests together: one panorama's 2M camera rays traced at
  // once would stall every request in flight for milliseconds. With
  // step-at-a-time traversal the camera rays ride in the next iteration's
  // traversal launch (no launch, and no launch tail, of their own).
  const int pct = cfg.large_inflight_pct;
  const int64_t share = pct > 0 && pct < 100 ? (int64_t)cfg.capacity * pct / 100
                                             : (int64_t)cfg.capacity / 4;
  int64_t large_budget = std::max<int64_t>(1024, share) - large_queued;
  auto enqueue_part = [&](Request* r) {
    const int64_t left = r->rays - r->prim_next;
    const int64_t n = r->small ? left : std::min(left, std::max<int64_t>(1024, large_budget));
    ids.push_back(r->slot);
    jobs.push_back(r->dj);
    rays.push_back(n);
    first.push_back(r->prim_next);
    r->prim_next += n;
    const bool last = r->prim_next == r->rays;
    final_part.push_back(last ? 1 : 0);
    // Read-backs count the request only once its paths exist.
    r->admit_seq = last ? launched : std::numeric_limits<uint64_t>::max();
    if (!r->small) {
      large_budget -= n;
      large_queued += n;
    }
  };
  {
    // Requests part-way through their primary pass, oldest first.
    std::vector<Request*> priming;
    for (size_t k = 0; k < slot_req.size(); ++k)
      if (slot_req[k]) {
        Request* r = reqs.at(slot_req[k]).get();
        if (r->prim_next < r->rays) priming.push_back(r);
      }
    std::sort(priming.begin(), priming.end(),
              [](const Request* a, const Request* b) { return a->id < b->id; });
    for (Request* r : priming)
      if (r->small || large_budget > 0) enqueue_part(r);
  }
  bool busy = cfg.deadline_ms > 0 && small_running();
  for (auto it = queue.begin(); it != queue.end();) {
    Request* r = find(*it);
    if (!r || r->cancel) {
      if (r) {
        r->state = kCancelled;
        finished_ids.push_back(r->id);
      }
      it = queue.erase(it);
      continue;
    }
    double due = -1;
    if (cfg.deadline_ms > 0 && r->small) {
      // Overload policy. A request that cannot finish within the deadline
      // even on an idle wavefront is shed now; one that would finish in time
      // behind the latency-bound work already admitted is admitted; the rest
      // wait (without holding back younger requests that fit) until they
      // fit or are shed.
      const double waited = now - r->submit_ms;
      const double target = slack * cfg.deadline_ms;
      ServiceEstimate& e = estimate(r);
      if (waited > cfg.deadline_ms || (e.alone >= 0 && waited + e.alone > target)) {
        // A stale estimate would shed this scene's requests for good:
        // every shed lowers it a little so that one is measured again.
        if (e.alone >= 0) e.alone *= 0.98;
        r->state = kCancelled;
        r->shed = true;
        ++shed;
        finished_ids.push_back(r->id);
        it = queue.erase(it);
        continue;
      }
      if (e.alone >= 0) {
        due = now + e.alone;
        if (busy) due = std::max(due, tail_ms + (e.gap >= 0 ? e.gap : e.alone));
        if (due - r->submit_ms > target) {
          ++it;
          continue;
        }
      } else if (e.probing) {
        ++it;  // one request measures a new scene before more are admitted
        continue;
      }
    }
    if (!r->small && large_budget <= 0) {
      ++it;  // this pump's primary rays of large requests are spent
      continue;
    }
    int slot = -1;
    for (size_t k = 0; k < slot_req.size(); ++k)
      if (!slot_req[k]) {
        slot = (int)k;
        break;
      }
    if (slot < 0) break;
    if (used_bytes + r->footprint > cfg.memory_budget) {
      ++it;
      continue;
    }
    HPT_TRACE_BEGIN(alloc_job);
    hpt_status s = engine->alloc_job(r->js, r->want_accum, r->buf);
    HPT_TRACE_END(alloc_job);
    if (s == HPT_ERR_OUT_OF_MEMORY) {
      engine->free_job(r->buf);
      break;  // retry after something finishes
    }
    if (s != HPT_OK) return s;
    r->slot = slot;
    r->state = kRunning;
    r->admit_ms = now_ms();
    if (cfg.deadline_ms > 0 && r->small) {
      r->due_ms = due;
      r->drift_ms = drift_ms;
      r->alone = !busy;
      if (due >= 0) tail_ms = busy ? std::max(tail_ms, due) : due;
      if (due < 0) estimate(r).probing = true;
      busy = true;
    }
    slot_req[slot] = r->id;
    used_bytes += r->footprint;
    r->dj = engine->make_job(r->js, r->buf);
    if (pct > 0 && pct < 100 && r->rays * r->js.params.sample > (int64_t)cfg.capacity)
      r->dj.max_inflight = std::max<int64_t>(1024, (int64_t)cfg.capacity * pct / 100);
    r->prim_next = 0;
    enqueue_part(r);
    it = queue.erase(it);
  }
  if (ids.empty()) return HPT_OK;
  if (engine->fused_primary()) {
    for (size_t k = 0; k < ids.size(); ++k) {
      const hpt_status s = engine->queue_primary(ids[k], jobs[k], rays[k], first[k],
                                                 final_part[k] != 0);
      if (s != HPT_OK) return s;
    }
    return engine->set_order_async(order());
  }
  large_queued = 0;  // traced right now by their own launch
  HPT_TRACE_BEGIN(admit_async);
  const hpt_status s = engine->admit_async(ids, jobs, rays, order(), nullptr, first, final_part);
  HPT_TRACE_END(admit_async);
  return s;
}

// Enqueues the resolve and copy-back of a request whose paths all finished.
hpt_status hpt_server::finish(Request* r) {
  const hpt_render_params& p = r->js.params;
  engine->launch_resolve(r->slot, r->js, r->buf);
  r->rgba_bytes = (size_t)p.sample_x * p.sample_y * 4;
  void* mem = nullptr;
  HPT_TRACE_BEGIN(take_pinned);
  hpt_status s = take_pinned(r->rgba_bytes, &mem);
  HPT_TRACE_END(take_pinned);
  if (s != HPT_OK) return s;
  r->rgba = static_cast<uint8_t*>(mem);
  HPT_CUDA(cudaMemcpyAsync(r->rgba, r->buf.rgba, r->rgba_bytes, cudaMemcpyDeviceToHost,
                           engine->stream));
  if (r->want_accum) {
    r->accum_bytes = (size_t)r->rays * 3 * sizeof(float);
    s = take_pinned(r->accum_bytes, &mem);
    if (s != HPT_OK) return s;
    r->accum = static_cast<float*>(mem);
    HPT_CUDA(cudaMemcpyAsync(r->accum, r->buf.accum_f, r->accum_bytes, cudaMemcpyDeviceToHost,
                             engine->stream));
  }
  s = take_event(&r->fin_ev);
  if (s != HPT_OK) return s;
  HPT_CUDA(cudaEventRecord(r->fin_ev, engine->stream));
  r->finishing = true;
  return HPT_OK;
}

// Applies a completed read-back: progress of the requests admitted before
// it, and the resolve of those whose paths all finished.
hpt_status hpt_server::apply_readback(Readback& b) {
  ctrl_view = *b.ctrl;
  bool any = false;
  for (size_t k = 0; k < slot_req.size(); ++k) {
    if (!slot_req[k]) continue;
    Request* r = reqs.at(slot_req[k]).get();
    if (r->finishing || b.seq <= r->admit_seq) continue;
    const DevSlot& S = b.slots[k];
    r->paths = S.num_paths;
    r->done_paths = (int64_t)S.done;
    r->queries = r->rays + (int64_t)S.queries;
    if ((int64_t)S.done >= S.num_paths && S.cursor >= S.num_paths) {
      hpt_status s = finish(r);
      if (s != HPT_OK) return s;
      any = true;
    }
  }
  if (ctrl_view.err.flags & 2u)
    return fail(HPT_ERR_INVALID_SCENE, "device self-check %d failed (value %lld)",
                ctrl_view.err.site, (long long)ctrl_view.err.value);
  if (ctrl_view.err.flags & 1u) return fail(HPT_ERR_TRAVERSAL_LIMIT, "a traversal hit its step cap");
  return any ? engine->set_order_async(order()) : HPT_OK;
}

// Marks done the finishing requests whose copy-back has completed and
// releases their slot and device buffers.
hpt_status hpt_server::retire_finished() {
  for (size_t k = 0; k < slot_req.size(); ++k) {
    if (!slot_req[k]) continue;
    Request* r = reqs.at(slot_req[k]).get();
    if (!r->finishing) continue;
    const cudaError_t e = cudaEventQuery(r->fin_ev);
    if (e == cudaErrorNotReady) continue;
    if (e != cudaSuccess) return cuda_fail(e, "copy-back");
    event_pool.push_back(r->fin_ev);
    r->fin_ev = nullptr;
    r->finishing = false;
    engine->free_job(r->buf);
    slot_req[k] = 0;
    used_bytes -= r->footprint;
    r->slot = -1;
    r->state = r->cancel ? kCancelled : kDone;
    r->done_ms = now_ms();
    finished_ids.push_back(r->id);
    ++completed;
    if (r->small && cfg.deadline_ms > 0) estimate(r).probing = false;
    if (r->small && !r->cancel && cfg.deadline_ms > 0) {
      // Upper-quantile running estimates: quick to rise, slow to fall.
      auto track = [](double& q, double x) {
        q = q < 0 ? x : q + (x > q ? 0.25 : 0.05) * (x - q);
      };
      ServiceEstimate& e = estimate(r);
      if (r->alone || e.alone < 0)
        track(e.alone, r->done_ms - r->admit_ms);
      else
        track(e.gap, r->done_ms - std::max(r->admit_ms, last_small_done_ms));
      last_small_done_ms = r->done_ms;
      if (r->done_ms - r->submit_ms > cfg.deadline_ms)
        slack = std::max(0.25, slack * 0.85);
      else
        slack = std::min(1.0, slack + 0.001);
      // Requests admitted behind this one finish as much earlier or later
      // than predicted as it did (its prediction already moved by the
      // corrections made since its admission).
      if (r->due_ms >= 0) {
        const double delta = r->done_ms - (r->due_ms + drift_ms - r->drift_ms);
        drift_ms += delta;
        tail_ms = std::max(r->done_ms, tail_ms + delta);
      }
    }
  }
  return HPT_OK;
}

extern "C" {

hpt_status hpt_server_create(const hpt_server_config* config, hpt_server** out) {
  if (!config || !out) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  *out = nullptr;
  if (config->max_jobs < 1 || config->max_jobs > 4096 || config->memory_budget <= 0 ||
      config->capacity < 1024 || config->capacity > (1 << 27) ||
      config->large_inflight_pct < 0 || config->large_inflight_pct > 100 ||
      config->pipeline_depth < 0 || config->pipeline_depth > kReadbacks - 1)
    return fail(HPT_ERR_INVALID_ARGUMENT, "server config out of range");
  if (config->device < 0 || config->device >= hpt_device_count())
    return fail(HPT_ERR_CUDA, "no CUDA device %d", config->device);
  try {
    std::unique_ptr<hpt_server> s(new hpt_server());
    s->cfg = *config;
    s->depth = config->pipeline_depth > 0 ? config->pipeline_depth : 1;
    s->t0 = std::chrono::steady_clock::now();
    s->engine.reset(new Engine(config->device));
    s->engine->tuning.capacity = config->capacity;
    s->engine->tuning.smem_nodes = 0;  // requests mix scenes
    HPT_CUDA(cudaSetDevice(config->device));
    hpt_status st = s->engine->ensure_capacity(config->capacity);
    if (st == HPT_OK) st = s->engine->ensure_slots(config->max_jobs);
    if (st != HPT_OK) return st;
    s->engine->reset_ctrl();
    HPT_CUDA(cudaStreamSynchronize(s->engine->stream));
    // All large requests together keep at most large_inflight_pct of the
    // wavefront in flight, however many of them are running.
    const int pct = config->large_inflight_pct;
    if (pct > 0 && pct < 100) {
      st = s->engine->set_capped_budget(
          std::max<int64_t>(1024, (int64_t)config->capacity * pct / 100));
      if (st != HPT_OK) return st;
    }
    // The admission budget is the per-request device memory the server may
    // use: map it into the job pool now, so admitting a request never waits
    // for the driver to map memory.
    st = s->engine->reserve_pool((size_t)config->memory_budget);
    if (st != HPT_OK) return st;
    s->arena_bytes = std::min<size_t>(512u << 20, std::max<size_t>(16u << 20,
                                      (size_t)config->memory_budget / 16));
    void* arena = nullptr;
    HPT_CUDA(cudaMallocHost(&arena, s->arena_bytes));
    s->arena = static_cast<uint8_t*>(arena);
    s->arena_free[0] = s->arena_bytes;
    for (Readback& b : s->rb) {
      HPT_CUDA(cudaMallocHost(&b.slots, (size_t)config->max_jobs * sizeof(DevSlot)));
      HPT_CUDA(cudaMallocHost(&b.ctrl, sizeof(DevCtrl)));
      HPT_CUDA(cudaEventCreateWithFlags(&b.ev, cudaEventDisableTiming));
    }
    s->slot_req.assign(config->max_jobs, 0);
    *out = s.release();
    return HPT_OK;
  } catch (const std::bad_alloc&) {
    return fail(HPT_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

hpt_status hpt_server_add_scene(hpt_server* server, hpt_scene* scene, int32_t* scene_slot) {
  if (!server || !scene || !scene_slot) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  std::lock_guard<std::mutex> lk(server->mu);
  if (scene->h.scene.device != server->cfg.device)
    return fail(HPT_ERR_INVALID_ARGUMENT, "scene lives on another device");
  server->scenes.push_back(scene);
  *scene_slot = (int32_t)server->scenes.size() - 1;
  return HPT_OK;
}

hpt_status hpt_server_submit(hpt_server* server, int32_t scene_slot, const hpt_camera* camera,
                             const hpt_render_params* params, uint64_t* request_id) {
  if (!server || !request_id) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  hpt_status s = check_render_params(camera, params);
  if (s != HPT_OK) return s;
  std::lock_guard<std::mutex> lk(server->mu);
  if (scene_slot < 0 || scene_slot >= (int32_t)server->scenes.size())
    return fail(HPT_ERR_NOT_FOUND, "scene slot %d not registered", scene_slot);
  std::unique_ptr<Request> r(new Request());
  r->id = server->next_id++;
  r->js.scene = &server->scenes[scene_slot]->h.scene;
  r->scene_slot = scene_slot;
  r->js.camera = *camera;
  r->js.params = *params;
  r->want_accum = server->cfg.keep_accum != 0;
  r->rays = (int64_t)params->sample_x * params->supersample_x * params->sample_y *
            params->supersample_y;
  r->footprint = job_footprint(*params, r->want_accum);
  r->small = r->rays * params->sample <= (int64_t)server->cfg.capacity;
  if (r->footprint > server->cfg.memory_budget)
    return fail(HPT_ERR_OUT_OF_MEMORY, "request needs %lld bytes, budget is %lld",
                (long long)r->footprint, (long long)server->cfg.memory_budget);
  r->submit_ms = server->now_ms();
  *request_id = r->id;
  server->queue.push_back(r->id);
  server->reqs[r->id] = std::move(r);
  return HPT_OK;
}

hpt_status hpt_server_pump(hpt_server* server, int32_t max_iterations) {
  if (!server) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  std::lock_guard<std::mutex> lk(server->mu);
  hpt_server& S = *server;
  HPT_CUDA(cudaSetDevice(S.cfg.device));
  ++S.pumps;
  // 1. Completed read-backs, oldest first, and finished copy-backs.
  auto drain_ready = [&]() -> hpt_status {
    while (S.rb_pending > 0) {
      Readback& b = S.rb[S.rb_drain];
      const cudaError_t e = cudaEventQuery(b.ev);
      if (e == cudaErrorNotReady) break;
      if (e != cudaSuccess) return cuda_fail(e, "slot read-back");
      b.pending = false;
      S.rb_drain = (S.rb_drain + 1) % kReadbacks;
      --S.rb_pending;
      hpt_status s = S.apply_readback(b);
      if (s != HPT_OK) return s;
    }
    return S.retire_finished();
  };
  HPT_TRACE_BEGIN(drain);
  hpt_status s = drain_ready();
  HPT_TRACE_END(drain);
  if (s != HPT_OK) return s;
  // 2. Admission.
  HPT_TRACE_BEGIN(admit);
  s = S.admit_pending();
  HPT_TRACE_END(admit);
  if (s != HPT_OK) return s;
  HPT_TRACE_BEGIN(launch);
  // 3. Keep up to `depth` iterations queued, each followed by a read-back.
  int n = 0;
  while (n < std::max(1, max_iterations) && S.rb_pending < S.depth && S.running()) {
    s = S.engine->launch_iteration_async();
    if (s != HPT_OK) return s;
    S.large_queued = 0;
    ++S.launched;
    ++n;
    Readback& b = S.rb[S.rb_fill];
    b.seq = S.launched;
    b.pending = true;
    s = S.engine->read_state_async(b.slots, b.ctrl, b.ev);
    if (s != HPT_OK) return s;
    S.rb_fill = (S.rb_fill + 1) % kReadbacks;
    ++S.rb_pending;
  }
  HPT_CUDA(cudaGetLastError());
  HPT_TRACE_END(launch);
  // 4. Nothing new to launch: wait for the oldest read-back (or copy-back)
  // instead of returning to a caller that would spin.
  if (n == 0) {
    HPT_TRACE_BEGIN(wait);
    if (S.rb_pending > 0) {
      HPT_CUDA(cudaEventSynchronize(S.rb[S.rb_drain].ev));
    } else {
      for (size_t k = 0; k < S.slot_req.size(); ++k)
        if (S.slot_req[k] && S.reqs.at(S.slot_req[k])->finishing) {
          HPT_CUDA(cudaEventSynchronize(S.reqs.at(S.slot_req[k])->fin_ev));
          break;
        }
    }
    HPT_TRACE_END(wait);
    s = drain_ready();
    if (s != HPT_OK) return s;
  }
  return HPT_OK;
}

hpt_status hpt_server_poll(hpt_server* server, uint64_t request_id, hpt_request_info* info,
                           uint8_t* rgba_out, float* accum_out) {
  if (!server) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  std::lock_guard<std::mutex> lk(server->mu);
  Request* r = server->find(request_id);
  if (!r) return fail(HPT_ERR_NOT_FOUND, "unknown request %llu", (unsigned long long)request_id);
  const hpt_render_params& p = r->js.params;
  const int64_t per_sample = r->paths > 0 ? r->paths / std::max(1, p.sample) : 0;
  if (info) {
    info->state = r->state;
    info->samples_done = r->state == kDone ? p.sample
                         : per_sample > 0  ? (int32_t)(r->done_paths / per_sample)
                                           : 0;
    info->submit_ms = r->submit_ms;
    info->admit_ms = r->admit_ms;
    info->done_ms = r->done_ms;
    info->intersect_queries = r->queries;
    info->due_ms = r->due_ms;
  }
  if (r->state == kDone) {
    if (rgba_out) std::memcpy(rgba_out, r->rgba, r->rgba_bytes);
    if (accum_out && r->accum) std::memcpy(accum_out, r->accum, r->accum_bytes);
    server->give_pinned(r->rgba, r->rgba_bytes);
    server->give_pinned(r->accum, r->accum_bytes);
    server->reqs.erase(request_id);
    return HPT_OK;
  }
  if (r->state == kCancelled || r->state == kFailed) {
    const hpt_status e = r->state == kCancelled ? HPT_ERR_CANCELLED : r->error;
    server->give_pinned(r->rgba, r->rgba_bytes);
    server->give_pinned(r->accum, r->accum_bytes);
    const bool shed = r->shed;
    server->reqs.erase(request_id);
    return fail(e, "request %llu %s", (unsigned long long)request_id,
                shed ? "was shed by the overload policy (deadline)"
                     : e == HPT_ERR_CANCELLED ? "was cancelled" : "failed");
  }
  // Running: a progressive preview divides by the samples completed so far
  // (paths finish out of order, so this is the fraction of finished paths).
  if (r->state == kRunning && !r->finishing && server->cfg.progressive && rgba_out &&
      per_sample > 0 && r->done_paths > 0) {
    const float samples = (float)((double)r->done_paths / (double)per_sample);
    server->engine->launch_resolve(r->slot, r->js, r->buf, samples);
    HPT_CUDA(cudaMemcpyAsync(rgba_out, r->buf.rgba, (size_t)p.sample_x * p.sample_y * 4,
                             cudaMemcpyDeviceToHost, server->engine->stream));
    HPT_CUDA(cudaStreamSynchronize(server->engine->stream));
  }
  return HPT_ERR_BUSY;
}

hpt_status hpt_server_cancel(hpt_server* server, uint64_t request_id) {
  if (!server) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  std::lock_guard<std::mutex> lk(server->mu);
  Request* r = server->find(request_id);
  if (!r) return fail(HPT_ERR_NOT_FOUND, "unknown request %llu", (unsigned long long)request_id);
  r->cancel = true;  // queued: dropped at the next admission; running: discarded when done
  if (r->state == kQueued) r->state = kCancelled;
  return HPT_OK;
}

hpt_status hpt_server_drain_completed(hpt_server* server, uint64_t* ids, int32_t max_ids,
                                      int32_t* count) {
  if (!server || !count || max_ids < 0 || (max_ids > 0 && !ids))
    return fail(HPT_ERR_INVALID_ARGUMENT, "bad drain arguments");
  std::lock_guard<std::mutex> lk(server->mu);
  const int32_t n = std::min<int32_t>(max_ids, (int32_t)server->finished_ids.size());
  std::copy(server->finished_ids.begin(), server->finished_ids.begin() + n, ids);
  server->finished_ids.erase(server->finished_ids.begin(), server->finished_ids.begin() + n);
  *count = n;
  return HPT_OK;
}

int64_t hpt_server_shed(const hpt_server* server) {
  if (!server) return 0;
  hpt_server* s = const_cast<hpt_server*>(server);
  std::lock_guard<std::mutex> lk(s->mu);
  return s->shed;
}

int32_t hpt_server_pending(const hpt_server* server) {
  if (!server) return 0;
  hpt_server* s = const_cast<hpt_server*>(server);
  std::lock_guard<std::mutex> lk(s->mu);
  int32_t n = 0;
  for (auto& kv : s->reqs) n += kv.second->state == kQueued || kv.second->state == kRunning;
  return n;
}

hpt_status hpt_server_stats_get(hpt_server* server, hpt_render_stats* out) {
  if (!server || !out) return fail(HPT_ERR_INVALID_ARGUMENT, "NULL argument");
  std::lock_guard<std::mutex> lk(server->mu);
  DevCtrl c;
  hpt_status s = server->engine->read_ctrl(&c);
  if (s != HPT_OK) return s;
  memset(out, 0, sizeof *out);
  out->intersect_queries = (int64_t)c.isect_queries;
  out->shade_calls = (int64_t)c.shades;
  out->iterations = (int32_t)c.iterations;
  out->error_flags = (int32_t)c.err.flags;
  out->nodes_visited = (int64_t)c.nodes_visited;
  out->leaves_visited = (int64_t)c.leaves_visited;
  out->triangle_tests = (int64_t)c.tri_tests;
  out->triangle_repeats = (int64_t)c.tri_repeats;
  out->paths = server->completed;
  return HPT_OK;
}

void hpt_server_destroy(hpt_server* server) {
  if (!server) return;
  {
    std::lock_guard<std::mutex> lk(server->mu);
    if (server->engine) {
      HPT_SOFT(cudaStreamSynchronize(server->engine->stream));
      for (auto& kv : server->reqs) {
        Request* r = kv.second.get();
        if (r->slot >= 0) server->engine->free_job(r->buf);
        if (r->fin_ev) HPT_SOFT(cudaEventDestroy(r->fin_ev));
        server->free_pinned(r->rgba);
        server->free_pinned(r->accum);
      }
      HPT_SOFT(cudaStreamSynchronize(server->engine->stream));
    }
    for (Readback& b : server->rb) {
      if (b.slots) HPT_SOFT(cudaFreeHost(b.slots));
      if (b.ctrl) HPT_SOFT(cudaFreeHost(b.ctrl));
      if (b.ev) HPT_SOFT(cudaEventDestroy(b.ev));
    }
    for (auto& kv : server->pinned_pool) HPT_SOFT(cudaFreeHost(kv.second));
    if (server->arena) HPT_SOFT(cudaFreeHost(server->arena));
    for (cudaEvent_t e : server->event_pool) HPT_SOFT(cudaEventDestroy(e));
  }
  delete server;
}

}  // extern "C"

// ===========================================================================
// Autotuner
// ===========================================================================
namespace {

std::string tune_key(const hpt_scene* scene, const hpt_render_params* p) {
  cudaDeviceProp prop;
  memset(&prop, 0, sizeof prop);
  if (cudaGetDeviceProperties(&prop, scene->h.scene.device) != cudaSuccess) {
    (void)cudaGetLastError();
    snprintf(prop.name, sizeof prop.name, "unknown");
  }
  std::string dev(prop.name);
  for (char& ch : dev)
    if (ch == ' ' || ch == '|') ch = '_';
  std::ostringstream k;
  const hpt_scene_info& in = scene->h.scene.info;
  k << dev << "|tris=" << in.num_triangles << "|nodes=" << in.num_device_nodes
    << "|rays=" << (int64_t)p->sample_x * p->supersample_x * p->sample_y * p->supersample_y
    << "|spp=" << p->sample << "|depth=" << p->depth;
  return k.str();
}

bool cache_lookup(const char* path, const std::string& key, hpt_tuning* t) {
  if (!path) return false;
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream is(line);
    std::string k;
    hpt_tuning x = default_tuning();
    if (!(is >> k >> x.capacity >> x.isect_block >> x.isect_min_blocks >> x.refill_chunk >>
          x.smem_nodes >> x.use_graph >> x.trav_steps))
      continue;
    if (!(is >> x.shade_min_blocks)) x.shade_min_blocks = default_tuning().shade_min_blocks;
    if (k == key) {
      *t = x;
      return true;
    }
  }
  return false;
}

void cache_store(const char* path, const std::string& key, const hpt_tuning& t) {
  if (!path) return;
  std::ofstream f(path, std::ios::app);
  f << key << " " << t.capacity << " " << t.isect_block << " " << t.isect_min_blocks << " "
    << t.refill_chunk << " " << t.smem_nodes << " " << t.use_graph << " " << t.trav_steps
    << " " << t.shade_min_blocks << "\n";
}

}  // namespace

extern "C" hpt_status hpt_autotune(hpt_scene* scene, const hpt_camera* camera,
                                   const hpt_render_params* params, const char* cache_path,
                                   hpt_tuning* best) {
  if (!scene) return fail(HPT_ERR_INVALID_ARGUMENT, "scene is NULL");
  hpt_status s = check_render_params(camera, params);
  if (s != HPT_OK) return s;
  const std::string key = tune_key(scene, params);
  hpt_tuning cur;
  {
    std::lock_guard<std::mutex> lk(scene->h.mu);
    cur = scene->h.tuning;
  }
  if (cache_lookup(cache_path, key, &cur)) {
    std::lock_guard<std::mutex> lk(scene->h.mu);
    cur.profile = scene->h.tuning.profile;
    cur.shade_block = 256;
    scene->h.tuning = cur;
    scene->h.engine.reset();
    if (best) *best = cur;
    return HPT_OK;
  }
  // Device time of one render with tuning t (best of two after a warm-up).
  auto time_of = [&](const hpt_tuning& t, float* ms) -> hpt_status {
    std::lock_guard<std::mutex> lk(scene->h.mu);
    Engine e(scene->h.scene.device);
    e.tuning = t;
    JobSpec js;
    js.scene = &scene->h.scene;
    js.camera = *camera;
    js.params = *params;
    float bestms = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
      hpt_render_stats st;
      hpt_status r = e.run({js}, &st);
      if (r != HPT_OK) return r;
      if (rep > 0) bestms = std::min(bestms, st.ms_total);
    }
    *ms = bestms;
    return HPT_OK;
  };
  float cur_ms = 0.f;
  s = time_of(cur, &cur_ms);
  if (s != HPT_OK) return s;
  // Coordinate search: one knob at a time, keeping the best value.
  struct Knob {
    std::vector<std::pair<int, int>> values;  // (a, b); b used by the variant knob
    void (*apply)(hpt_tuning&, int, int);
  };
  const Knob knobs[] = {
      {{{128, 5}, {128, 6}, {128, 7}, {128, 8}, {128, 9}, {128, 10}, {256, 2}, {256, 3}},
       [](hpt_tuning& t, int a, int b) {
         t.isect_block = a;
         t.isect_min_blocks = b;
       }},
      {{{0, 0}, {16, 0}, {32, 0}, {48, 0}},
       [](hpt_tuning& t, int a, int) { t.trav_steps = a; }},
      {{{2, 0}, {4, 0}, {8, 0}, {16, 0}},
       [](hpt_tuning& t, int a, int) { t.refill_chunk = a; }},
      {{{0, 0}, {1024, 0}, {2048, 0}, {4096, 0}},
       [](hpt_tuning& t, int a, int) { t.smem_nodes = a; }},
      {{{1 << 20, 0}, {1 << 21, 0}, {1 << 22, 0}, {1 << 23, 0}, {1 << 24, 0}},
       [](hpt_tuning& t, int a, int) { t.capacity = a; }},
      {{{0, 0}, {1, 0}}, [](hpt_tuning& t, int a, int) { t.use_graph = a; }},
      {{{0, 0}, {3, 0}, {4, 0}}, [](hpt_tuning& t, int a, int) { t.shade_min_blocks = a; }},
  };
  for (const Knob& k : knobs) {
    for (const auto& v : k.values) {
      hpt_tuning t = cur;
      k.apply(t, v.first, v.second);
      if (memcmp(&t, &cur, sizeof t) == 0) continue;
      float ms = 0.f;
      s = time_of(t, &ms);
      if (s != HPT_OK) return s;
      if (ms < cur_ms * 0.99f) {
        cur = t;
        cur_ms = ms;
      }
    }
  }
  cache_store(cache_path, key, cur);
  {
    std::lock_guard<std::mutex> lk(scene->h.mu);
    cur.profile = scene->h.tuning.profile;
    cur.shade_block = 256;
    scene->h.tuning = cur;
    scene->h.engine.reset();
  }
  if (best) *best = cur;
  return HPT_OK;
}
