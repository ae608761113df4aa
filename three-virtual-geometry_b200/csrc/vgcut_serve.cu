// Serving loop of the cut engine (vgc_server_* in include/vgcut.h). The reference cuts once per rendered frame of
// one camera (VirtualGeometry.update, VirtualGeometry.ts:392-484); a server instead takes cut requests against
// several resident scenes as they arrive:
//
//  * admission: a request waits until an output slot of its scene is free and the output-slot bytes of all
//    admitted, unreleased requests plus its own stay within the HBM budget;
//  * batching: the worker launches up to max_batch of the oldest admissible requests as one launch sequence (the
//    plain path's kernels, one view per request). With cross_scene they may belong to different scenes: each view
//    then reads its own context's scene through a scene table (the multi-scene kernel variants); otherwise a
//    batch takes the requests of the oldest admissible request's scene;
//  * continuous batching: each of `streams` lanes owns a CUDA stream and launch scratch; a lane that finishes is
//    refilled from whatever is pending, while the other lanes' batches keep running;
//  * completion: the lane's stream gathers every view's counters into pinned memory and then runs a host callback,
//    which stamps the completion time and wakes the worker; no CUDA call that can wait on a stream is made under
//    the server lock (the callbacks take it).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <thread>
#include <unordered_map>

#include "vgcut_host.h"
#include "vgcut_kernels.h"

namespace {

double now_us() {
  return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
  uint32_t scene = 0;
  vgc_view view{};
  bool done = false;
  vgc_serve_result result{};
};

struct SceneState {
  vgc_context *ctx = nullptr;
  std::vector<uint32_t> free_slots;
  size_t slot_bytes = 0;
};

struct Lane {
  cudaStream_t stream = nullptr;
  LaunchScratch scratch;
  cudaEvent_t start = nullptr, end = nullptr;
  uint32_t *d_words = nullptr;  // 32 words per view (launch_gather_stats)
  uint32_t *h_words = nullptr;  // pinned copy
  bool busy = false;
  bool complete = false;  // set by the stream callback
  double done_us = 0;
  uint32_t scenes = 0;  // distinct scenes in the batch
  double start_us = 0;
  std::vector<uint64_t> tickets;
  int status = VGC_OK;
};

}  // namespace

struct vgc_server {
  vgc_server_options opts{};
  std::vector<SceneState> scenes;
  std::vector<vgc_context *> ctxs;  // the scene table of multi-scene launches (index = scene)
  std::deque<uint64_t> pending;     // tickets in arrival order, all scenes
  uint32_t multi_grid[2] = {0, 0};  // persistent grids of the multi-scene k_instances / k_chunks
  std::vector<Lane> lanes;
  std::vector<std::pair<vgc_server *, Lane *>> callbacks;  // host-callback arguments, one per lane
  std::mutex mu;
  std::condition_variable wake;  // worker: new request, release or completion
  std::condition_variable done;  // waiters: a request completed
  std::unordered_map<uint64_t, Request> requests;
  uint64_t next_ticket = 1;
  uint64_t bytes_in_use = 0;
  vgc_server_stats stats{};
  uint32_t in_flight = 0;
  bool stop = false;
  std::thread worker;
  std::string error;  // last launch error (worker thread)
};

namespace {

void CUDART_CB lane_done(void *arg) {
  auto *pair = static_cast<std::pair<vgc_server *, Lane *> *>(arg);
  vgc_server *s = pair->first;
  Lane *lane = pair->second;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    lane->done_us = now_us();
    lane->complete = true;
  }
  s->wake.notify_all();
}

// The next batch for an idle lane, chosen under the lock: the oldest admissible requests in arrival order (a request
// is admissible while its scene has a free output slot and its slot bytes fit the HBM budget), from any scene with
// cross_scene, else from the oldest one's scene. Returns false when nothing can start now.
bool pick_batch(vgc_server *s, Lane &lane, std::vector<uint32_t> &slots, std::vector<vgc_view> &views,
                std::vector<uint32_t> &scene_ids) {
  auto admissible = [&](const SceneState &sc) {
    return !sc.free_slots.empty() &&
           !(s->opts.hbm_budget_bytes && s->bytes_in_use + sc.slot_bytes > s->opts.hbm_budget_bytes);
  };
  auto first = s->pending.end();
  size_t ready = 0;
  for (auto it = s->pending.begin(); it != s->pending.end(); ++it)
    if (admissible(s->scenes[s->requests[*it].scene])) {
      if (first == s->pending.end()) first = it;
      if (++ready >= s->opts.max_batch) break;
    }
  if (first == s->pending.end()) return false;
  const double oldest = s->requests[*first].result.submit_us;
  // linger: while another batch runs, a short batch waits (up to linger_us from its oldest request) for more
  // requests; with every lane idle it starts at once
  if (s->opts.linger_us && ready < s->opts.max_batch && s->in_flight > 0 && now_us() - oldest < s->opts.linger_us)
    return false;
  const uint32_t lead = s->requests[*first].scene;
  lane.tickets.clear();
  slots.clear();
  views.clear();
  scene_ids.clear();
  // views x scene instances of the batch: large scenes go in smaller batches, which bounds latency and queued work
  uint64_t work = 0;
  std::vector<bool> seen(s->scenes.size(), false);
  uint32_t distinct = 0;
  for (auto it = first; it != s->pending.end() && lane.tickets.size() < s->opts.max_batch;) {
    Request &r = s->requests[*it];
    SceneState &sc = s->scenes[r.scene];
    if ((!s->opts.cross_scene && r.scene != lead) || !admissible(sc)) {
      ++it;
      continue;
    }
    const uint64_t inst = std::max<uint64_t>(1, sc.ctx->inst_slot.size());
    if (s->opts.max_batch_instances && !lane.tickets.empty() && work + inst > s->opts.max_batch_instances) break;
    work += inst;
    const uint64_t t = *it;
    it = s->pending.erase(it);
    const uint32_t slot = sc.free_slots.back();
    sc.free_slots.pop_back();
    s->bytes_in_use += sc.slot_bytes;
    r.result.slot = slot;
    vgc_view v = r.view;
    v.state_slot = slot;
    v.flags |= VGC_VIEW_FRESH_STATE;
    lane.tickets.push_back(t);
    slots.push_back(slot);
    views.push_back(v);
    scene_ids.push_back(r.scene);
    if (!seen[r.scene]) seen[r.scene] = true, distinct++;
  }
  s->stats.max_bytes_in_use = std::max<uint64_t>(s->stats.max_bytes_in_use, s->bytes_in_use);
  lane.scenes = distinct;
  lane.busy = true;
  lane.complete = false;
  return true;
}

// Launches a picked batch on its lane (no server lock held: prepare may synchronise the device). A batch of one
// scene takes that context's plain launch sequence; a mixed batch the multi-scene variant over the server's scene
// table.
int launch_batch(vgc_server *s, Lane &lane, const std::vector<uint32_t> &slots, const std::vector<vgc_view> &views,
                 const std::vector<uint32_t> &scene_ids, std::pair<vgc_server *, Lane *> *cb) {
  vgc_context *ctx = s->scenes[scene_ids[0]].ctx;
  cudaSetDevice(ctx->device);
  const uint32_t n = (uint32_t)views.size();
  int rc;
  if (lane.scenes <= 1) {
    lane.scratch.grid_instances = lane.scratch.grid_chunks = 0;  // the context's single-scene grids
    rc = prepare(ctx, lane.scratch, views.data(), n, 0, slots.data());
  } else {
    lane.scratch.grid_instances = s->multi_grid[0];
    lane.scratch.grid_chunks = s->multi_grid[1];
    ctx = s->ctxs[0];
    rc = prepare_multi(s->ctxs.data(), (uint32_t)s->ctxs.size(), lane.scratch, views.data(), scene_ids.data(), n,
                       slots.data());
  }
  if (rc) return rc;
  CUDA_TRY(cudaEventRecord(lane.start, lane.stream));
  if ((rc = enqueue(ctx, lane.scratch, n, lane.stream, false))) return rc;
  CUDA_TRY(launch_gather_stats(lane.scratch.d_views, n, lane.d_words, lane.stream));
  CUDA_TRY(cudaMemcpyAsync(lane.h_words, lane.d_words, (size_t)n * 32 * 4, cudaMemcpyDeviceToHost, lane.stream));
  CUDA_TRY(cudaEventRecord(lane.end, lane.stream));
  CUDA_TRY(cudaLaunchHostFunc(lane.stream, lane_done, cb));
  return VGC_OK;
}

// Results of a completed lane (under the lock).
void finish_lane(vgc_server *s, Lane &lane) {
  float gpu_ms = 0;
  if (lane.status == VGC_OK) cudaEventElapsedTime(&gpu_ms, lane.start, lane.end);
  for (size_t i = 0; i < lane.tickets.size(); i++) {
    Request &r = s->requests[lane.tickets[i]];
    vgc_context *ctx = s->scenes[r.scene].ctx;
    r.result.status = lane.status;
    r.result.batch_views = (uint32_t)lane.tickets.size();
    r.result.batch_scenes = lane.scenes;
    r.result.start_us = lane.start_us;
    r.result.done_us = lane.status == VGC_OK ? lane.done_us : now_us();
    r.result.batch_gpu_ms = gpu_ms;
    if (lane.status == VGC_OK) {
      const uint32_t *w = lane.h_words + i * 32;
      float threshold;
      std::memcpy(&threshold, &w[VGC_COUNTER_HEADER], 4);
      decode_stats(ctx, w, threshold, &r.result.stats);
    }
    r.done = true;
    s->stats.completed++;
  }
  lane.busy = false;
  lane.complete = false;
  lane.tickets.clear();
  s->in_flight--;
}

void worker_main(vgc_server *s) {
  std::vector<uint32_t> slots, scene_ids;
  std::vector<vgc_view> views;
  std::unique_lock<std::mutex> lock(s->mu);
  while (!s->stop) {
    bool progress = false;
    for (Lane &lane : s->lanes)
      if (lane.busy && lane.complete) {
        finish_lane(s, lane);
        progress = true;
      }
    if (progress) s->done.notify_all();
    for (size_t i = 0; i < s->lanes.size(); i++) {
      Lane &lane = s->lanes[i];
      if (lane.busy || !pick_batch(s, lane, slots, views, scene_ids)) continue;
      lane.start_us = now_us();
      s->in_flight++;
      s->stats.batches++;
      if (lane.scenes > 1) s->stats.multi_scene_batches++;
      s->stats.views_launched += views.size();
      s->stats.max_in_flight = std::max(s->stats.max_in_flight, s->in_flight);
      lock.unlock();
      const int rc = launch_batch(s, lane, slots, views, scene_ids, &s->callbacks[i]);
      std::string why;
      if (rc) {  // the batch's callback was not queued: wait out what was, then complete it with the error
        why = vgc_last_error();
        cudaStreamSynchronize(lane.stream);
      }
      lock.lock();
      if (rc) {
        lane.status = rc;
        s->error = why;
        finish_lane(s, lane);
        lane.status = VGC_OK;
        s->done.notify_all();
      }
      progress = true;
    }
    if (!progress) {
      const bool lingering = s->opts.linger_us != 0;
      s->wake.wait_for(lock, std::chrono::microseconds(lingering ? std::max(1u, s->opts.linger_us / 4) : 2000));
    }
  }
}

}  // namespace

extern "C" {

void vgc_server_default_options(vgc_server_options *o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->streams = 2;
  o->max_batch = 64;
  o->max_batch_instances = 32u << 20;
  o->cross_scene = 1;
}

int vgc_server_create(vgc_context *const *scenes, uint32_t scene_count, const vgc_server_options *opts,
                      vgc_server **out) {
  if (!scenes || scene_count == 0 || !out) return fail(VGC_INVALID_ARG, "no scenes");
  vgc_server_options o;
  vgc_server_default_options(&o);
  if (opts) o = *opts;
  if (o.streams == 0) o.streams = 2;
  if (o.max_batch == 0) o.max_batch = 64;
  if (o.slots_per_scene == 0) o.slots_per_scene = o.streams * o.max_batch;
  for (uint32_t i = 0; i < scene_count; i++)
    if (!scenes[i]) return fail(VGC_INVALID_ARG, "null scene context");
  auto *s = new vgc_server();
  s->opts = o;
  s->scenes.resize(scene_count);
  s->lanes.resize(o.streams);
  for (Lane &lane : s->lanes) s->callbacks.push_back({s, &lane});
  auto cleanup = [&](int rc) {
    vgc_server_destroy(s);
    return rc;
  };
  // output and state slots up front: nothing reallocates while batches run
  vgc_context *largest = scenes[0];
  for (uint32_t i = 0; i < scene_count; i++) {
    vgc_context *ctx = scenes[i];
    cudaSetDevice(ctx->device);
    int rc = sync_scene(ctx);
    if (!rc) rc = ensure_outputs(ctx, o.slots_per_scene);
    if (!rc) rc = ensure_state(ctx, o.slots_per_scene - 1);
    if (rc) return cleanup(rc);
    SceneState &sc = s->scenes[i];
    sc.ctx = ctx;
    s->ctxs.push_back(ctx);
    if (ctx->device != scenes[0]->device) s->opts.cross_scene = 0;  // a multi-scene launch runs on one device
    sc.slot_bytes = output_slot_bytes(ctx);
    for (uint32_t k = o.slots_per_scene; k-- > 0;) sc.free_slots.push_back(k);
    if (ctx->cells.size() > largest->cells.size()) largest = ctx;
  }
  if (o.hbm_budget_bytes)
    for (const SceneState &sc : s->scenes)
      if (sc.slot_bytes > o.hbm_budget_bytes) return cleanup(fail(VGC_OVER_BUDGET, "one output slot exceeds the budget"));
  cudaSetDevice(largest->device);
  int mi = 0, mc = 0;
  if (configure_select(true, &mi, &mc) != cudaSuccess) {
    cudaGetLastError();
    mi = mc = 1;
  }
  s->multi_grid[0] = (uint32_t)std::max(1, mi) * largest->sm_count;
  s->multi_grid[1] = (uint32_t)std::max(1, mc) * largest->sm_count;
  const size_t units = (size_t)o.max_batch * pad32((uint32_t)largest->cells.size());
  for (Lane &lane : s->lanes) {
    int rc = ensure_scratch(largest, lane.scratch, o.max_batch, units);
    if (rc) return cleanup(rc);
    if (cudaStreamCreateWithFlags(&lane.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&lane.start) != cudaSuccess || cudaEventCreate(&lane.end) != cudaSuccess ||
        cudaMalloc(&lane.d_words, (size_t)o.max_batch * 32 * 4) != cudaSuccess ||
        cudaMallocHost(&lane.h_words, (size_t)o.max_batch * 32 * 4) != cudaSuccess)
      return cleanup(fail(VGC_DEVICE_ERROR, "server lane setup failed"));
  }
  s->worker = std::thread(worker_main, s);
  *out = s;
  return VGC_OK;
}

int vgc_server_submit(vgc_server *s, uint32_t scene, const vgc_view *view, uint64_t *ticket) {
  if (!s || !view || !ticket) return fail(VGC_INVALID_ARG, "null argument");
  if (scene >= s->scenes.size()) return fail(VGC_INVALID_ARG, "scene index out of range");
  if (view->depth) return fail(VGC_INVALID_ARG, "served views take a built HZB slot, not a depth image");
  {
    std::lock_guard<std::mutex> lock(s->mu);
    const uint64_t t = s->next_ticket++;
    Request &r = s->requests[t];
    r.scene = scene;
    r.view = *view;
    r.result.ticket = t;
    r.result.scene = scene;
    r.result.submit_us = now_us();
    s->pending.push_back(t);
    s->stats.submitted++;
    *ticket = t;
  }
  s->wake.notify_all();
  return VGC_OK;
}

int vgc_server_wait(vgc_server *s, uint64_t ticket, uint32_t timeout_ms, vgc_serve_result *out) {
  if (!s || !out) return fail(VGC_INVALID_ARG, "null argument");
  std::unique_lock<std::mutex> lock(s->mu);
  auto it = s->requests.find(ticket);
  if (it == s->requests.end()) return fail(VGC_NOT_FOUND, "unknown or released ticket");
  const bool ok = s->done.wait_for(lock, std::chrono::milliseconds(timeout_ms), [&] {
    auto jt = s->requests.find(ticket);
    return jt == s->requests.end() || jt->second.done;
  });
  it = s->requests.find(ticket);
  if (it == s->requests.end()) return fail(VGC_NOT_FOUND, "request released while waiting");
  if (!ok) return fail(VGC_TIMEOUT, "request not completed within the timeout");
  *out = it->second.result;
  if (it->second.result.status != VGC_OK) return fail(it->second.result.status, "launch failed: " + s->error);
  return VGC_OK;
}

int vgc_server_release(vgc_server *s, uint64_t ticket) {
  if (!s) return fail(VGC_INVALID_ARG, "null server");
  {
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return fail(VGC_NOT_FOUND, "unknown or released ticket");
    if (!it->second.done) return fail(VGC_INVALID_ARG, "request still queued or running");
    SceneState &sc = s->scenes[it->second.scene];
    sc.free_slots.push_back(it->second.result.slot);
    s->bytes_in_use -= sc.slot_bytes;
    s->requests.erase(it);
  }
  s->wake.notify_all();
  return VGC_OK;
}

int vgc_server_drain(vgc_server *s, uint32_t timeout_ms) {
  if (!s) return fail(VGC_INVALID_ARG, "null server");
  std::unique_lock<std::mutex> lock(s->mu);
  const bool ok = s->done.wait_for(lock, std::chrono::milliseconds(timeout_ms),
                                   [&] { return s->stats.completed == s->stats.submitted; });
  return ok ? VGC_OK : fail(VGC_TIMEOUT, "requests still pending after the timeout");
}

int vgc_server_stats_get(vgc_server *s, vgc_server_stats *out) {
  if (!s || !out) return fail(VGC_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lock(s->mu);
  *out = s->stats;
  out->bytes_in_use = s->bytes_in_use;
  return VGC_OK;
}

int vgc_server_destroy(vgc_server *s) {
  if (!s) return VGC_OK;
  // stop launching, then let the lanes' streams (and their callbacks, which take the lock) finish
  if (s->worker.joinable()) {
    {
      std::lock_guard<std::mutex> lock(s->mu);
      s->stop = true;
    }
    s->wake.notify_all();
    s->worker.join();
  }
  for (Lane &lane : s->lanes) {
    if (lane.stream) cudaStreamSynchronize(lane.stream);
    free_scratch(lane.scratch);
    if (lane.start) cudaEventDestroy(lane.start);
    if (lane.end) cudaEventDestroy(lane.end);
    if (lane.d_words) cudaFree(lane.d_words);
    if (lane.h_words) cudaFreeHost(lane.h_words);
    if (lane.stream) cudaStreamDestroy(lane.stream);
  }
  delete s;
  return VGC_OK;
}

}  // extern "C"
