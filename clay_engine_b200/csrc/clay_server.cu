// clay_server.cu - the continuous-batching server behind clay_server_* (include/clay_fluid.h).
//
// Host code only, written against the library's own C ABI: scenes are FluidSims created and
// destroyed through clay_fluid_*, each frame is one clay_batch_step_subset over the scenes
// that have a request in progress, and completion is tracked with CUDA events on the
// server's stream. There is no reference counterpart: the reference steps the scenes of one
// game; this is the serving loop of many independent scenes on one GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <string>
#include <thread>
#include <vector>

#include "../../include/clay_fluid.h"

// clay_last_error is set through the library's own error paths; the server's own refusals
// go through the fluid API's validation where possible, else are reported here.
namespace clay {
int set_error(int code, const char* fmt, ...);
}

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  int32_t scene = 0;
  int32_t frames = 0;
  int32_t remaining = 0;
  double t_arrival = 0;  // seconds since the server's time origin
  double t_done = -1;
  bool done = false;
};

struct Scene {
  const clay_field* world = nullptr;
  clay_fluid_opts opts{};
  std::vector<clay_fluid_particle> state;  // host copy while not resident
  int64_t live = 0;
  clay_fluid* sim = nullptr;
  uint64_t bytes = 0;       // device bytes while resident
  uint64_t estimate = 0;    // clay_fluid_estimate_bytes
  uint64_t last_use = 0;    // LRU stamp
  int32_t inflight = 0;     // frames in flight that step this scene
  int64_t active = -1;      // ticket in progress
  std::deque<int64_t> waiting;
};

struct Frame {
  cudaEvent_t ev = nullptr;
  std::vector<int32_t> scenes;
  std::vector<int64_t> finished;
};

}  // namespace

struct clay_server {
  clay_ctx* ctx = nullptr;
  cudaStream_t stream = nullptr;
  clay_server_opts opts{};
  std::vector<Scene> scenes;
  std::vector<Request> reqs;
  std::deque<Frame> inflight;
  std::vector<cudaEvent_t> event_pool;
  clay_batch* batch = nullptr;
  std::vector<int32_t> batch_scene;  // batch slot -> scene
  std::vector<int32_t> slot_of;      // scene -> batch slot, -1 when not in the batch
  bool dirty = true;
  uint64_t clock = 0;
  uint64_t resident_bytes = 0;
  int32_t resident = 0;
  clay_server_stats stats{};
  Clock::time_point t0;
  cudaEvent_t ev0 = nullptr;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

int cuda_fail(cudaError_t e, const char* what) {
  return clay::set_error(CLAY_ECUDA, "clay_server: %s: %s", what, cudaGetErrorString(e));
}
#define SCK(call, what)                              \
  do {                                               \
    cudaError_t e_ = (call);                         \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

int take_event(clay_server* s, cudaEvent_t* out) {
  if (!s->event_pool.empty()) {
    *out = s->event_pool.back();
    s->event_pool.pop_back();
    return CLAY_OK;
  }
  SCK(cudaEventCreate(out), "cudaEventCreate");
  return CLAY_OK;
}

// Completion time of a frame's event on the server's clock (seconds).
double event_time(const clay_server* s, cudaEvent_t ev) {
  float ms = 0;
  cudaEventElapsedTime(&ms, s->ev0, ev);
  return ms / 1000.0;
}

void retire_front(clay_server* s) {
  Frame f = std::move(s->inflight.front());
  s->inflight.pop_front();
  const double t = event_time(s, f.ev);
  for (int64_t id : f.finished) {
    Request& r = s->reqs[static_cast<size_t>(id)];
    r.t_done = t;
    r.done = true;
    s->stats.completed++;
  }
  for (int32_t sc : f.scenes) s->scenes[static_cast<size_t>(sc)].inflight--;
  s->event_pool.push_back(f.ev);
}

int retire(clay_server* s) {
  while (!s->inflight.empty()) {
    cudaError_t q = cudaEventQuery(s->inflight.front().ev);
    if (q == cudaErrorNotReady) break;
    if (q != cudaSuccess) return cuda_fail(q, "cudaEventQuery");
    retire_front(s);
  }
  return CLAY_OK;
}

int wait_all(clay_server* s) {
  SCK(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize");
  while (!s->inflight.empty()) retire_front(s);
  return CLAY_OK;
}

void drop_batch(clay_server* s) {
  if (s->batch) clay_batch_destroy(s->batch);
  s->batch = nullptr;
  std::fill(s->slot_of.begin(), s->slot_of.end(), -1);
  s->batch_scene.clear();
}

// Evicts an idle resident scene: its particle state goes to the host, its sim is freed.
// Served scenes never emit (the server has no spawn request), so the particle records and
// their count are the whole state: a re-admitted sim starts its emission ring at the count
// (clay_fluid_upload), which is where it stood.
int evict(clay_server* s, int32_t id) {
  Scene& sc = s->scenes[static_cast<size_t>(id)];
  // the batch references the sim: it is rebuilt before the next launch
  int rc = wait_all(s);
  if (rc) return rc;
  drop_batch(s);
  sc.live = clay_fluid_particle_count(sc.sim);
  sc.state.resize(static_cast<size_t>(std::max<int64_t>(sc.live, 0)));
  if (sc.live > 0 && (rc = clay_fluid_download(sc.sim, sc.state.data(), sc.live, s->stream))) return rc;
  SCK(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize");
  clay_fluid_destroy(sc.sim);
  sc.sim = nullptr;
  s->resident_bytes -= sc.bytes;
  sc.bytes = 0;
  s->resident--;
  s->stats.evictions++;
  s->dirty = true;
  return CLAY_OK;
}

// Makes a scene resident within the budget. *ok = false when it has to wait for room.
int admit(clay_server* s, int32_t id, bool* ok) {
  Scene& sc = s->scenes[static_cast<size_t>(id)];
  *ok = true;
  if (sc.sim) return CLAY_OK;
  const uint64_t budget = s->opts.budget_bytes;
  if (budget) {
    if (sc.estimate > budget)
      return clay::set_error(CLAY_ENOMEM, "clay_server: scene %d needs %llu bytes, over the %llu-byte budget", id,
                             static_cast<unsigned long long>(sc.estimate), static_cast<unsigned long long>(budget));
    while (s->resident_bytes + sc.estimate > budget) {
      int32_t victim = -1;
      for (size_t k = 0; k < s->scenes.size(); k++) {
        const Scene& o = s->scenes[k];
        if (!o.sim || o.active >= 0 || o.inflight > 0 || !o.waiting.empty()) continue;
        if (victim < 0 || o.last_use < s->scenes[static_cast<size_t>(victim)].last_use) victim = static_cast<int32_t>(k);
      }
      if (victim < 0) {
        *ok = false;
        return CLAY_OK;
      }
      int rc = evict(s, victim);
      if (rc) return rc;
    }
  }
  uint64_t before = 0, after = 0;
  clay_ctx_bytes_in_use(s->ctx, &before);
  int rc = clay_fluid_create(s->ctx, sc.world, &sc.opts, &sc.sim);
  if (rc) return rc;
  clay_fluid_set_mode(sc.sim, s->opts.mode);
  if (sc.live > 0 && (rc = clay_fluid_upload(sc.sim, sc.state.data(), sc.live, s->stream))) return rc;
  SCK(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize");
  std::vector<clay_fluid_particle>().swap(sc.state);
  clay_ctx_bytes_in_use(s->ctx, &after);
  sc.bytes = after - before;
  s->resident_bytes += sc.bytes;
  s->resident++;
  s->stats.admissions++;
  s->dirty = true;
  return CLAY_OK;
}

int rebuild(clay_server* s) {
  int rc = wait_all(s);
  if (rc) return rc;
  drop_batch(s);
  std::vector<clay_fluid*> sims;
  for (size_t k = 0; k < s->scenes.size(); k++) {
    if (!s->scenes[k].sim) continue;
    s->slot_of[k] = static_cast<int32_t>(s->batch_scene.size());
    s->batch_scene.push_back(static_cast<int32_t>(k));
    sims.push_back(s->scenes[k].sim);
  }
  if ((rc = clay_batch_create(s->ctx, sims.data(), static_cast<int>(sims.size()), &s->batch))) return rc;
  clay_batch_tuning t{};
  clay_batch_get_tuning(s->batch, &t);
  t.use_graph = 0;
  if (s->opts.sph_block) t.sph_block = s->opts.sph_block;
  if ((rc = clay_batch_set_tuning(s->batch, &t))) return rc;
  s->dirty = false;
  return CLAY_OK;
}

int pump(clay_server* s, int32_t* launched) {
  if (launched) *launched = 0;
  int rc = retire(s);
  if (rc) return rc;
  // the head request of every scene that waits and is idle, when the scene can be resident
  for (size_t k = 0; k < s->scenes.size(); k++) {
    Scene& sc = s->scenes[k];
    if (sc.active >= 0 || sc.waiting.empty()) continue;
    bool ok = false;
    if ((rc = admit(s, static_cast<int32_t>(k), &ok))) return rc;
    if (!ok) continue;
    sc.active = sc.waiting.front();
    sc.waiting.pop_front();
  }
  if (static_cast<int32_t>(s->inflight.size()) >= s->opts.depth) return CLAY_OK;
  std::vector<int32_t> step;
  for (size_t k = 0; k < s->scenes.size(); k++)
    if (s->scenes[k].active >= 0) step.push_back(static_cast<int32_t>(k));
  if (step.empty()) return CLAY_OK;
  // least recently stepped first when the frame is capped
  if (s->opts.max_batch > 0 && static_cast<int32_t>(step.size()) > s->opts.max_batch) {
    std::stable_sort(step.begin(), step.end(), [&](int32_t a, int32_t b) {
      return s->scenes[static_cast<size_t>(a)].last_use < s->scenes[static_cast<size_t>(b)].last_use;
    });
    step.resize(static_cast<size_t>(s->opts.max_batch));
  }
  if (s->dirty && (rc = rebuild(s))) return rc;
  std::vector<int32_t> slots;
  slots.reserve(step.size());
  for (int32_t k : step) slots.push_back(s->slot_of[static_cast<size_t>(k)]);
  if ((rc = clay_batch_step_subset(s->batch, slots.data(), static_cast<int>(slots.size()), s->stream))) return rc;
  Frame f;
  if ((rc = take_event(s, &f.ev))) return rc;
  SCK(cudaEventRecord(f.ev, s->stream), "cudaEventRecord");
  s->clock++;
  for (int32_t k : step) {
    Scene& sc = s->scenes[static_cast<size_t>(k)];
    Request& r = s->reqs[static_cast<size_t>(sc.active)];
    s->stats.particle_steps += clay_fluid_particle_count(sc.sim);
    sc.last_use = s->clock;
    sc.inflight++;
    if (--r.remaining == 0) {
      f.finished.push_back(sc.active);
      sc.active = -1;
    }
  }
  f.scenes = std::move(step);
  s->stats.frames++;
  s->stats.scene_frames += static_cast<int64_t>(f.scenes.size());
  s->inflight.push_back(std::move(f));
  if (launched) *launched = 1;
  return CLAY_OK;
}

}  // namespace

extern "C" {

int clay_server_create(clay_ctx* ctx, const clay_server_opts* opts, void* stream, clay_server** out) {
  if (!ctx || !out) return clay::set_error(CLAY_EINVAL, "clay_server_create: NULL argument");
  clay_server_opts o{};
  if (opts) o = *opts;
  if (o.depth == 0) o.depth = 2;
  if (o.depth < 1 || o.depth > 8) return clay::set_error(CLAY_EINVAL, "clay_server_create: depth %d outside 1..8", o.depth);
  if (o.max_batch < 0) return clay::set_error(CLAY_EINVAL, "clay_server_create: max_batch %d < 0", o.max_batch);
  if (o.mode != CLAY_MODE_FAST && o.mode != CLAY_MODE_REFERENCE)
    return clay::set_error(CLAY_EINVAL, "clay_server_create: unknown mode %d", o.mode);
  if (o.sph_block && (o.sph_block < 64 || o.sph_block > 256 || (o.sph_block & 31)))
    return clay::set_error(CLAY_EINVAL, "clay_server_create: sph_block %d must be a multiple of 32 in 64..256", o.sph_block);
  clay_server* s = new clay_server();
  s->ctx = ctx;
  s->opts = o;
  s->stream = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaEventCreate(&s->ev0);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e == cudaSuccess) e = cudaEventRecord(s->ev0, s->stream);
  if (e == cudaSuccess) e = cudaEventSynchronize(s->ev0);
  if (e != cudaSuccess) {
    if (s->ev0) cudaEventDestroy(s->ev0);
    delete s;
    return cuda_fail(e, "clay_server_create");
  }
  s->t0 = Clock::now();
  *out = s;
  return CLAY_OK;
}

void clay_server_destroy(clay_server* s) {
  if (!s) return;
  cudaStreamSynchronize(s->stream);
  while (!s->inflight.empty()) retire_front(s);
  drop_batch(s);
  for (auto& sc : s->scenes)
    if (sc.sim) clay_fluid_destroy(sc.sim);
  for (cudaEvent_t ev : s->event_pool) cudaEventDestroy(ev);
  if (s->ev0) cudaEventDestroy(s->ev0);
  delete s;
}

int clay_server_add_scene(clay_server* s, const clay_field* world, const clay_fluid_opts* opts,
                          const clay_fluid_particle* particles, int64_t count, int32_t* scene_out) {
  if (!s || !scene_out || (count > 0 && !particles)) return clay::set_error(CLAY_EINVAL, "clay_server_add_scene: NULL argument");
  Scene sc;
  sc.world = world;
  if (opts) sc.opts = *opts;
  int rc = clay_fluid_estimate_bytes(&sc.opts, &sc.estimate);
  if (rc) return rc;
  const int64_t cap = (sc.opts.set & CLAY_FLUID_CAPACITY) ? sc.opts.capacity : 8192;
  if (count < 0 || count > cap)
    return clay::set_error(CLAY_EINVAL, "clay_server_add_scene: count %lld outside 0..capacity %lld",
                           static_cast<long long>(count), static_cast<long long>(cap));
  sc.state.assign(particles, particles + count);
  sc.live = count;
  s->scenes.push_back(std::move(sc));
  s->slot_of.push_back(-1);
  *scene_out = static_cast<int32_t>(s->scenes.size() - 1);
  return CLAY_OK;
}

int clay_server_submit(clay_server* s, int32_t scene, int32_t frames, int64_t* ticket_out) {
  if (!s || !ticket_out) return clay::set_error(CLAY_EINVAL, "clay_server_submit: NULL argument");
  if (scene < 0 || scene >= static_cast<int32_t>(s->scenes.size()))
    return clay::set_error(CLAY_EINVAL, "clay_server_submit: scene %d outside 0..%d", scene,
                           static_cast<int>(s->scenes.size()) - 1);
  if (frames < 1) return clay::set_error(CLAY_EINVAL, "clay_server_submit: frames %d < 1", frames);
  Request r;
  r.scene = scene;
  r.frames = r.remaining = frames;
  r.t_arrival = s->now();
  s->reqs.push_back(r);
  const int64_t id = static_cast<int64_t>(s->reqs.size() - 1);
  s->scenes[static_cast<size_t>(scene)].waiting.push_back(id);
  s->stats.submitted++;
  *ticket_out = id;
  return CLAY_OK;
}

int clay_server_pump(clay_server* s, int32_t* launched) {
  if (!s) return clay::set_error(CLAY_EINVAL, "clay_server_pump: NULL server");
  return pump(s, launched);
}

int clay_server_wait(clay_server* s, double timeout_ms) {
  if (!s) return clay::set_error(CLAY_EINVAL, "clay_server_wait: NULL server");
  if (s->inflight.empty()) return CLAY_OK;
  cudaEvent_t ev = s->inflight.front().ev;
  if (timeout_ms < 0) {
    SCK(cudaEventSynchronize(ev), "cudaEventSynchronize");
  } else {
    const auto until = Clock::now() + std::chrono::duration<double, std::milli>(timeout_ms);
    for (;;) {
      cudaError_t q = cudaEventQuery(ev);
      if (q == cudaSuccess) break;
      if (q != cudaErrorNotReady) return cuda_fail(q, "cudaEventQuery");
      if (Clock::now() >= until) return CLAY_OK;
      std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
  }
  return retire(s);
}

int clay_server_drain(clay_server* s) {
  if (!s) return clay::set_error(CLAY_EINVAL, "clay_server_drain: NULL server");
  while (s->stats.completed < s->stats.submitted) {
    int32_t launched = 0;
    int rc = pump(s, &launched);
    if (rc) return rc;
    if (launched) continue;
    if (!s->inflight.empty()) {
      SCK(cudaEventSynchronize(s->inflight.front().ev), "cudaEventSynchronize");
      continue;
    }
    // nothing in flight and nothing launched: the waiting scenes cannot be admitted
    return clay::set_error(CLAY_ENOMEM, "clay_server_drain: %lld request(s) wait for scenes that do not fit the budget",
                           static_cast<long long>(s->stats.submitted - s->stats.completed));
  }
  return CLAY_OK;
}

int clay_server_poll(const clay_server* s, int64_t ticket, int32_t* done, double* latency_ms) {
  if (!s || !done) return clay::set_error(CLAY_EINVAL, "clay_server_poll: NULL argument");
  if (ticket < 0 || ticket >= static_cast<int64_t>(s->reqs.size()))
    return clay::set_error(CLAY_EINVAL, "clay_server_poll: unknown ticket %lld", static_cast<long long>(ticket));
  const Request& r = s->reqs[static_cast<size_t>(ticket)];
  *done = r.done ? 1 : 0;
  if (latency_ms) *latency_ms = r.done ? (r.t_done - r.t_arrival) * 1000.0 : -1.0;
  return CLAY_OK;
}

int clay_server_get_stats(const clay_server* s, clay_server_stats* out) {
  if (!s || !out) return clay::set_error(CLAY_EINVAL, "clay_server_get_stats: NULL argument");
  *out = s->stats;
  out->resident_bytes = s->resident_bytes;
  out->resident_scenes = s->resident;
  out->inflight = static_cast<int32_t>(s->inflight.size());
  return CLAY_OK;
}

int clay_server_scene_sim(clay_server* s, int32_t scene, clay_fluid** sim_out) {
  if (!s || !sim_out) return clay::set_error(CLAY_EINVAL, "clay_server_scene_sim: NULL argument");
  if (scene < 0 || scene >= static_cast<int32_t>(s->scenes.size()))
    return clay::set_error(CLAY_EINVAL, "clay_server_scene_sim: scene %d unknown", scene);
  *sim_out = s->scenes[static_cast<size_t>(scene)].sim;
  return CLAY_OK;
}

int clay_server_download(clay_server* s, int32_t scene, clay_fluid_particle* host, int64_t cap, int64_t* n_out) {
  if (!s || !n_out || (cap > 0 && !host)) return clay::set_error(CLAY_EINVAL, "clay_server_download: NULL argument");
  if (scene < 0 || scene >= static_cast<int32_t>(s->scenes.size()))
    return clay::set_error(CLAY_EINVAL, "clay_server_download: scene %d unknown", scene);
  Scene& sc = s->scenes[static_cast<size_t>(scene)];
  if (sc.active >= 0 || !sc.waiting.empty())
    return clay::set_error(CLAY_ESTATE, "clay_server_download: scene %d has requests not yet launched", scene);
  int rc = wait_all(s);
  if (rc) return rc;
  const int64_t n = sc.sim ? clay_fluid_particle_count(sc.sim) : sc.live;
  *n_out = n;
  const int64_t c = std::min(n, cap);
  if (c <= 0) return CLAY_OK;
  if (sc.sim) {
    if ((rc = clay_fluid_download(sc.sim, host, c, s->stream))) return rc;
    SCK(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize");
  } else {
    std::memcpy(host, sc.state.data(), sizeof(clay_fluid_particle) * static_cast<size_t>(c));
  }
  return CLAY_OK;
}

}  // extern "C"
