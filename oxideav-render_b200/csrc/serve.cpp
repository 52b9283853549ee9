// Serving layer (include/pt_b200_serve.h): continuous batching of render
// requests over scenes resident in HBM.
//
// One worker thread owns a private engine (stream, wave buffers, counters).
// Its loop:
//   1. admit pending requests while accumulator slots are free: make the
//      request's scene resident (evicting least-recently-used scenes that no
//      admitted request needs, within the HBM budget), allocate and clear its
//      accumulator, build its refine job;
//   2. pack one wave from every admitted request, earliest expected finish
//      first (submit time + remaining samples at the measured throughput:
//      short requests overtake long ones only by about their own length, so
//      nothing starves), upload the wave's request table and segments
//      from pinned staging, launch it; requests whose last samples are in the
//      wave get a resolve kernel + a copy of the HDR image into pinned host
//      memory behind it, on the same stream;
//   3. keep up to `pipeline_depth` waves in flight; when the oldest finishes,
//      its finished requests become visible to pt_server_wait.
// Each request's job is exactly the job pt_tracer_refine would run (same
// request, first sample, sample count), and waves keep every pixel's samples
// in index order, so images do not depend on the mix.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pt_b200.h"
#include "../../include/pt_b200_debug.h"
#include "../../include/pt_b200_serve.h"
#include "context.h"
#include "host_scene.h"
#include "kernels.h"

using namespace ptd;
using Clock = std::chrono::steady_clock;

namespace {

thread_local std::string t_err;

pt_status sfail(pt_status st, const std::string &msg) {
  t_err = msg;
  return st;
}

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct SceneEntry {
  uint32_t key = 0;
  SceneImage img;
  bool has_env = false;
  pt_environment env{};
  std::vector<float> env_pixels;
  std::unique_ptr<SceneHost> dev;     // non-null while resident
  std::unique_ptr<EnvHost> env_dev;
  uint64_t est_bytes = 0;             // device bytes when resident
  uint64_t dev_bytes = 0;
  uint64_t last_use = 0;
  uint32_t pins = 0;                  // admitted requests drawing on it
  uint32_t queued = 0;                // pending requests naming it
  bool registered = true;
};

// One progressive accumulation: created with its first request, given device
// memory when that request is admitted, continued by later requests.
struct Accum {
  pt_tracer t;                        // accumulator, camera, options, sample count
  std::shared_ptr<SceneEntry> scene;
  uint32_t refs = 0;                  // tickets on it that are not released
  bool busy = false;                  // a request on it is admitted
  bool failed = false;                // its first request failed: continuations fail too
  pt_status fail_status = PT_OK;
  std::string fail_msg;
};

enum class RState { Pending, Active, Done, Failed };

struct Request {
  uint64_t ticket = 0;
  pt_server_request in{};
  std::shared_ptr<SceneEntry> scene;
  std::shared_ptr<Accum> acc;
  RState state = RState::Pending;
  pt_status status = PT_OK;
  std::string error;
  Clock::time_point t_submit, t_admit, t_done;
  Job job{};
  uint32_t waves = 0;
  uint32_t samples_after = 0;
  uint32_t w = 0, h = 0;
  float *hdr = nullptr;               // pinned host image, w * h * 4 floats
  size_t hdr_bytes = 0;
  uint32_t readers = 0;               // waits copying `hdr` out (outside the lock)
  bool has_deadline = false;
  Clock::time_point deadline;
  // Cancelled (or timed out) while its last wave was on the GPU: it ends
  // with this status when that wave completes.
  pt_status end_status = PT_OK;
  std::string end_msg;
};

// Pinned host buffers, recycled by power-of-two size class.
struct PinnedPool {
  std::map<size_t, std::vector<void *>> free;
  static size_t cls(size_t bytes) {
    size_t c = 1 << 16;
    while (c < bytes) c <<= 1;
    return c;
  }
  void *get(size_t bytes) {
    size_t c = cls(bytes);
    auto &v = free[c];
    if (!v.empty()) {
      void *p = v.back();
      v.pop_back();
      return p;
    }
    void *p = nullptr;
    if (cudaMallocHost(&p, c) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return p;
  }
  void put(void *p, size_t bytes) {
    if (p) free[cls(bytes)].push_back(p);
  }
  void clear() {
    for (auto &kv : free)
      for (void *p : kv.second) cudaFreeHost(p);
    free.clear();
  }
};

// One wave on the stream: its staging, device tables, events and the
// requests that finish in it.
struct Flight {
  cudaEvent_t ev_start = nullptr, ev_end = nullptr;
  DevRequest *d_reqs = nullptr, *h_reqs = nullptr;
  size_t req_cap = 0;
  WaveSegment *d_segs = nullptr, *h_segs = nullptr;
  size_t seg_cap = 0;
  DevCounters *h_ctr = nullptr;
  std::vector<std::shared_ptr<Request>> finishing;
  uint64_t samples = 0;
};

}  // namespace

struct pt_server {
  pt_context *eng = nullptr;
  uint64_t budget = 0;
  uint32_t wave_slots = 1u << 22, max_active = 256, depth = 3;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::thread worker;
  bool stop = false;
  bool broken = false;
  std::string broken_msg;
  std::map<uint32_t, std::shared_ptr<SceneEntry>> scenes;
  std::vector<std::shared_ptr<SceneEntry>> dead_scenes;  // unregistered, device copy still to free
  uint32_t next_scene = 1;
  std::map<uint64_t, std::shared_ptr<Request>> reqs;
  uint64_t next_ticket = 1;
  std::deque<std::shared_ptr<Request>> pending;
  std::vector<std::shared_ptr<Request>> active;
  std::vector<std::shared_ptr<Accum>> dead_accums;
  std::vector<Flight> flights;
  std::deque<size_t> inflight;
  uint64_t wave_no = 0;
  float4 *d_resolve = nullptr;
  size_t resolve_cap = 0;
  PinnedPool pinned;
  pt_server_stats st{};
  uint64_t tick = 0;
  uint32_t accum_count = 0;
  bool autotune = false;
  bool spatial_bvh = true;    // registered scenes get the spatial-split tree
  bool tune_pending = false;  // a request waits for an idle stream to tune its class
  uint64_t rays_base = 0;     // rays counted before the device counters were last cleared
  // Overlapped waves (wavefront engine): consecutive waves are traced in the
  // engine's two arenas on its two wave streams; the accumulates, resolves
  // and accumulator allocations stay on the engine stream. Scene and
  // environment uploads then run on `upload` (the host waits for each, so a
  // trace never waits on the engine stream), and an eviction's frees wait
  // on the engine stream's position first (every trace already launched).
  bool overlap = false;
  cudaStream_t upload = nullptr;
  cudaEvent_t ev_free = nullptr;
  // Packing key: expected samples per ms of the served waves (measured; the
  // first waves use a nominal 100 M samples/s).
  double samples_per_ms = 1e5;
  std::atomic<uint32_t> fail_allocs{0};  // host-side allocation-failure injection
};

namespace {

uint64_t env_bytes_estimate(const pt_environment &e) {
  uint64_t w = std::max(e.width, 1u), h = std::max(e.height, 1u);
  return w * h * 24 + (h + 1) * 4 + h * (w + 1) * 4 + 5 * 256;
}

void evict(pt_server *s, SceneEntry &e) {
  if (!e.dev) return;
  if (s->overlap) {
    // The arenas are freed on the upload stream: after the engine stream's
    // accumulates, which wait for their waves' traces.
    cudaEventRecord(s->ev_free, s->eng->stream);
    cudaStreamWaitEvent(s->upload, s->ev_free, 0);
  }
  release_scene(*e.dev);  // stream-ordered free: after every wave already queued
  e.dev.reset();
  if (e.env_dev) {
    release_env(*e.env_dev);
    e.env_dev.reset();
  }
  s->st.resident_bytes -= e.dev_bytes;
  e.dev_bytes = 0;
  s->st.scene_evictions++;
}

enum class Admit { Yes, Wait, Failed };

// Consumes one injected allocation failure, if armed.
bool injected_oom(pt_server *s) {
  uint32_t n = s->fail_allocs.load();
  while (n > 0)
    if (s->fail_allocs.compare_exchange_weak(n, n - 1)) return true;
  return false;
}

void fail_request(pt_server *s, const std::shared_ptr<Request> &r, pt_status st, const std::string &msg) {
  r->state = RState::Failed;
  r->status = st;
  r->error = msg;
  r->t_done = Clock::now();
  s->st.failed++;
  s->cv_done.notify_all();
}

// Makes `e` resident. Called with the lock held; drops it around the copy.
Admit make_resident(pt_server *s, const std::shared_ptr<SceneEntry> &e, std::unique_lock<std::mutex> &lk,
                    std::string &err) {
  if (e->dev) return Admit::Yes;
  const uint64_t need = e->est_bytes;
  if (s->budget) {
    while (s->st.resident_bytes + need > s->budget) {
      SceneEntry *victim = nullptr;
      for (auto &kv : s->scenes) {
        SceneEntry &c = *kv.second;
        if (c.dev && c.pins == 0 && &c != e.get() && (!victim || c.last_use < victim->last_use)) victim = &c;
      }
      if (!victim) {
        if (s->active.empty() && s->inflight.empty()) {
          err = "scene " + std::to_string(e->key) + " needs " + std::to_string(need) +
                " device bytes; the HBM budget is " + std::to_string(s->budget) + " and nothing can be evicted";
          return Admit::Failed;
        }
        return Admit::Wait;
      }
      evict(s, *victim);
    }
  }
  if (injected_oom(s)) {
    err = "scene " + std::to_string(e->key) + ": device allocation failed (injected)";
    return Admit::Failed;
  }
  cudaStream_t stream = s->overlap ? s->upload : s->eng->stream;
  e->pins++;  // keeps it from eviction / unregistration while unlocked
  lk.unlock();
  auto dev = std::make_unique<SceneHost>();
  std::unique_ptr<EnvHost> env_dev;
  bool oom = false;
  std::string msg = commit_scene(e->img, *dev, oom, stream);
  if (msg.empty() && e->has_env) {
    env_dev = std::make_unique<EnvHost>();
    msg = upload_env(e->env, *env_dev, oom, stream);
    if (!msg.empty()) {
      release_scene(*dev);
      env_dev.reset();
    }
  }
  if (msg.empty() && s->overlap) {
    // Resident before any wave that reads it is launched, on any stream.
    cudaError_t se = cudaStreamSynchronize(stream);
    if (se != cudaSuccess) {
      msg = std::string("scene upload failed: ") + cudaGetErrorString(se);
      release_scene(*dev);
      if (env_dev) release_env(*env_dev);
      env_dev.reset();
    }
  }
  lk.lock();
  e->pins--;
  if (!msg.empty()) {
    err = msg;
    return Admit::Failed;
  }
  e->dev_bytes = dev->device_bytes() + (env_dev ? env_dev->arena.bytes : 0);
  e->est_bytes = e->dev_bytes;
  e->dev = std::move(dev);
  e->env_dev = std::move(env_dev);
  s->st.resident_bytes += e->dev_bytes;
  s->st.peak_resident_bytes = std::max(s->st.peak_resident_bytes, s->st.resident_bytes);
  s->st.scene_uploads++;
  return Admit::Yes;
}

// Fails request `r`; when it was the first request of its accumulation, the
// accumulation fails too (its continuations inherit the error).
void fail_admission(pt_server *s, const std::shared_ptr<Request> &r, pt_status st, const std::string &msg) {
  if (!r->in.continues) {
    r->scene->queued--;
    r->acc->failed = true;
    r->acc->fail_status = st;
    r->acc->fail_msg = msg;
  }
  fail_request(s, r, st, msg);
}

Admit try_admit(pt_server *s, const std::shared_ptr<Request> &r, std::unique_lock<std::mutex> &lk) {
  Accum &acc = *r->acc;
  if (acc.failed) {
    fail_request(s, r, acc.fail_status, "the continued request failed: " + acc.fail_msg);
    return Admit::Failed;
  }
  if (acc.busy) return Admit::Wait;                       // behind a running request on it
  if (r->in.continues && !acc.t.d_accum) return Admit::Wait;  // its first request is not admitted yet
  std::shared_ptr<SceneEntry> sc = acc.scene;
  if (!sc->registered) {
    fail_admission(s, r, PT_ERR_EVICTED, "scene " + std::to_string(sc->key) + " was unregistered");
    return Admit::Failed;
  }
  std::string err;
  Admit a = make_resident(s, sc, lk, err);
  // Cancelled or timed out while the lock was dropped: already ended.
  if (r->state != RState::Pending) return Admit::Failed;
  if (a == Admit::Wait) return a;
  if (a == Admit::Failed) {
    fail_admission(s, r, PT_ERR_OOM, err);
    return a;
  }
  if (s->autotune && !s->eng->tuned.count(scene_class(*sc->dev, sc->env_dev != nullptr))) {
    // A new scene class: tune on an idle stream (no wave launches until the
    // ones in flight finish), then admit.
    if (!s->inflight.empty()) {
      s->tune_pending = true;
      return Admit::Wait;
    }
    sc->pins++;
    lk.unlock();
    TuneChoice best{};
    // Calibrate on one full wave whatever the request's size.
    pt_status tst = autotune(s->eng, &acc.t, *sc->dev, sc->env_dev.get(), 0, best);
    lk.lock();
    sc->pins--;
    // The calibration refines used the engine's counters: restart them.
    s->rays_base = s->st.rays;
    cudaMemsetAsync(s->eng->d_ctr, 0, sizeof(DevCounters), s->eng->stream);
    // No wave is in flight while a class tunes: the wave streams may wait
    // for the engine stream here without serialising anything.
    if (s->overlap) engine_overlap_begin(s->eng);
    if (r->state != RState::Pending) {
      // Ended while tuning; the class is tuned all the same.
      if (tst == PT_OK) s->st.tuned_classes++;
      return Admit::Failed;
    }
    if (tst != PT_OK) {
      fail_admission(s, r, tst, "autotune: " + s->eng->err);
      return Admit::Failed;
    }
    s->st.tuned_classes++;
  }
  cudaStream_t stream = s->eng->stream;
  pt_tracer &t = acc.t;
  if (!t.d_accum) {
    size_t bytes = (size_t)t.w * t.h * 4 * sizeof(double);
    cudaError_t e = injected_oom(s) ? cudaErrorMemoryAllocation : cudaMallocAsync((void **)&t.d_accum, bytes, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(t.d_accum, 0, bytes, stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      if (t.d_accum) cudaFreeAsync(t.d_accum, stream);
      t.d_accum = nullptr;
      fail_admission(s, r, e == cudaErrorMemoryAllocation ? PT_ERR_OOM : PT_ERR_DEVICE,
                     std::string("accumulator allocation failed: ") + cudaGetErrorString(e));
      return Admit::Failed;
    }
    t.accum_cap = (size_t)t.w * t.h * 4;
    t.have_state = true;
    t.dirty = false;
    sc->queued--;
    s->accum_count++;
  }
  uint32_t n = std::min<uint32_t>(r->in.samples, 0xffffffffu - t.samples);
  if (n == 0) {
    fail_request(s, r, PT_ERR_INVALID_ARG, "the accumulation holds the maximum sample count");
    return Admit::Failed;
  }
  r->job = make_job(t, *sc->dev, sc->env_dev.get(), n);
  acc.busy = true;
  sc->pins++;
  sc->last_use = ++s->tick;
  r->state = RState::Active;
  r->t_admit = Clock::now();
  s->active.push_back(r);
  return Admit::Yes;
}

void admit(pt_server *s, std::unique_lock<std::mutex> &lk) {
  s->tune_pending = false;
  for (size_t i = 0; i < s->pending.size() && s->active.size() < s->max_active;) {
    std::shared_ptr<Request> r = s->pending[i];
    Admit a = try_admit(s, r, lk);
    // try_admit may drop the lock: a cancel can have changed the queue.
    auto it = std::find(s->pending.begin(), s->pending.end(), r);
    if (a == Admit::Wait) {
      i = it == s->pending.end() ? i : (size_t)(it - s->pending.begin()) + 1;
    } else if (it != s->pending.end()) {
      i = (size_t)(it - s->pending.begin());
      s->pending.erase(it);
    }
  }
}

template <class T>
cudaError_t grow_pair(T *&d, T *&h, size_t &cap, size_t need) {
  if (need <= cap) return cudaSuccess;
  size_t n = std::max<size_t>(need, 2 * cap);
  if (d) cudaFree(d);
  if (h) cudaFreeHost(h);
  d = nullptr;
  h = nullptr;
  cap = 0;
  cudaError_t e = cudaMalloc((void **)&d, n * sizeof(T));
  if (e == cudaSuccess) e = cudaMallocHost((void **)&h, n * sizeof(T));
  if (e == cudaSuccess) cap = n;
  return e;
}

// A device error ends the server: running and queued requests fail with it.
void break_server(pt_server *s, const std::string &msg) {
  s->broken = true;
  s->broken_msg = msg;
  for (auto &r : s->active) fail_request(s, r, PT_ERR_DEVICE, msg);
  s->active.clear();
  for (auto &r : s->pending) fail_request(s, r, PT_ERR_DEVICE, msg);
  s->pending.clear();
}

// Packs and launches the next wave. Called with the lock held.
void launch_next_wave(pt_server *s) {
  cudaStream_t stream = s->eng->stream;
  const size_t n = s->active.size();
  std::vector<Job> jobs(n);
  for (size_t i = 0; i < n; ++i) jobs[i] = s->active[i]->job;
  std::vector<uint32_t> order(n);
  std::iota(order.begin(), order.end(), 0u);
  // Earliest expected finish first: submit time (ms since the oldest active
  // request's) + remaining samples / measured throughput.
  Clock::time_point t0 = s->active[0]->t_submit;
  for (size_t i = 1; i < n; ++i) t0 = std::min(t0, s->active[i]->t_submit);
  std::vector<double> key(n);
  for (size_t i = 0; i < n; ++i) {
    const Job &j = jobs[i];
    const double remaining = (double)j.npix * (j.target - j.done) - j.pix_done;
    key[i] = ms_between(t0, s->active[i]->t_submit) + remaining / s->samples_per_ms;
  }
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
  std::vector<WaveSegment> segs = pack_wave(jobs, order, s->wave_slots);
  // The priority order chose what goes into the wave; inside it, the
  // segments are laid out scene by scene (a job has at most one segment per
  // wave, so samples stay in order), so the wave's first rays walk one BVH
  // at a time.
  std::stable_sort(segs.begin(), segs.end(), [&](const WaveSegment &a, const WaveSegment &b) {
    return jobs[a.request].scene_key < jobs[b.request].scene_key;
  });
  {
    uint32_t slot = 0;
    for (WaveSegment &sg : segs) {
      sg.slot_begin = slot;
      slot += sg.pixel_count * sg.spp;
    }
  }
  // Compact request table: only the jobs this wave carries.
  std::vector<int> remap(n, -1);
  std::vector<DevRequest> table;
  std::vector<uint32_t> carried;
  uint32_t iters = 1, shadow = 1, wide = WIDE_EXTENSION | WIDE_SHADOW;
  bool area = false;
  uint64_t total = 0;
  for (WaveSegment &sg : segs) {
    if (remap[sg.request] < 0) {
      remap[sg.request] = (int)table.size();
      table.push_back(jobs[sg.request].req);
      carried.push_back(sg.request);
      iters = std::max(iters, jobs[sg.request].iterations);
      shadow = std::max(shadow, jobs[sg.request].shadow_slots);
      area = area || jobs[sg.request].area;
      wide &= jobs[sg.request].wide;
    }
    total += (uint64_t)sg.pixel_count * sg.spp;
    sg.request = (uint32_t)remap[sg.request];
  }
  pt_status pst = engine_reserve(s->eng, s->wave_slots, shadow, iters, s->overlap);
  if (pst != PT_OK) {
    break_server(s, "wave buffers: " + s->eng->err);
    return;
  }
  const size_t fi = s->wave_no % s->flights.size();
  Flight &f = s->flights[fi];
  cudaError_t e = grow_pair(f.d_reqs, f.h_reqs, f.req_cap, table.size());
  if (e == cudaSuccess) e = grow_pair(f.d_segs, f.h_segs, f.seg_cap, segs.size());
  if (e != cudaSuccess) {
    cudaGetLastError();
    break_server(s, std::string("wave tables: ") + cudaGetErrorString(e));
    return;
  }
  std::memcpy(f.h_reqs, table.data(), table.size() * sizeof(DevRequest));
  std::memcpy(f.h_segs, segs.data(), segs.size() * sizeof(WaveSegment));
  // Overlapped: the tables go up on the wave's own stream, so its trace
  // waits for nothing queued on the engine stream.
  const int arena = s->overlap ? (int)(s->wave_no % s->eng->overlap_arenas) : -1;
  cudaStream_t up = arena >= 0 ? s->eng->wave_streams[arena] : stream;
  if (arena >= 0) e = cudaStreamWaitEvent(up, s->eng->ev_accumulated[arena], 0);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(f.d_reqs, f.h_reqs, table.size() * sizeof(DevRequest), cudaMemcpyHostToDevice, up);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(f.d_segs, f.h_segs, segs.size() * sizeof(WaveSegment), cudaMemcpyHostToDevice, up);
  if (e == cudaSuccess) e = cudaEventRecord(f.ev_start, up);
  if (e != cudaSuccess) {
    break_server(s, std::string("wave upload: ") + cudaGetErrorString(e));
    return;
  }
  pst = launch_wave(s->eng, f.d_reqs, f.d_segs, segs, iters, nullptr, arena, area, wide);
  if (pst != PT_OK) {
    break_server(s, "wave launch: " + s->eng->err);
    return;
  }
  f.finishing.clear();
  f.samples = total;
  std::vector<std::shared_ptr<Request>> still;
  std::vector<bool> done_now(n, false);
  for (uint32_t i : carried) {
    std::shared_ptr<Request> &r = s->active[i];
    r->job = jobs[i];
    r->waves++;
    if (!jobs[i].finished()) continue;
    // Last samples of this request: resolve behind the wave.
    Accum &acc = *r->acc;
    acc.t.samples += jobs[i].target;
    r->samples_after = acc.t.samples;
    const size_t npix = (size_t)acc.t.w * acc.t.h;
    if (s->resolve_cap < npix) {
      if (s->d_resolve) cudaFreeAsync(s->d_resolve, stream);
      s->d_resolve = nullptr;
      s->resolve_cap = 0;
      e = cudaMallocAsync((void **)&s->d_resolve, npix * sizeof(float4), stream);
      if (e == cudaSuccess) s->resolve_cap = npix;
    }
    r->hdr_bytes = npix * sizeof(float4);
    r->hdr = (float *)s->pinned.get(r->hdr_bytes);
    if (e == cudaSuccess && !r->hdr) e = cudaErrorMemoryAllocation;
    if (e == cudaSuccess)
      e = launch_resolve_hdr(acc.t.d_accum, (uint32_t)npix, acc.t.samples, bg_linear(acc.t.opts), s->d_resolve,
                             stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(r->hdr, s->d_resolve, r->hdr_bytes, cudaMemcpyDeviceToHost, stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      fail_request(s, r, PT_ERR_DEVICE, std::string("resolve: ") + cudaGetErrorString(e));
    } else {
      f.finishing.push_back(r);
    }
    // Stream order makes the accumulator and the scene safe to reuse or
    // evict from here on.
    acc.busy = false;
    r->acc->scene->pins--;
    done_now[i] = true;
  }
  for (size_t i = 0; i < n; ++i)
    if (!done_now[i]) still.push_back(s->active[i]);
  s->active.swap(still);
  e = cudaMemcpyAsync(f.h_ctr, s->eng->d_ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaEventRecord(f.ev_end, stream);
  if (e != cudaSuccess) {
    break_server(s, std::string("wave record: ") + cudaGetErrorString(e));
    return;
  }
  s->inflight.push_back(fi);
  s->wave_no++;
}

void complete_flight(pt_server *s, size_t fi, cudaError_t e) {
  Flight &f = s->flights[fi];
  s->inflight.pop_front();
  if (e != cudaSuccess) {
    std::string msg = std::string("wave failed: ") + cudaGetErrorString(e);
    for (auto &r : f.finishing) fail_request(s, r, PT_ERR_DEVICE, msg);
    f.finishing.clear();
    break_server(s, msg);
    return;
  }
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, f.ev_start, f.ev_end);
  s->st.gpu_ms += ms;
  if (ms > 0.0f && f.samples >= (1u << 20)) {
    // Throughput of full-ish waves steers the packing key (smoothed).
    s->samples_per_ms = 0.8 * s->samples_per_ms + 0.2 * ((double)f.samples / ms);
  }
  s->st.waves++;
  s->st.samples += f.samples;
  s->st.rays = s->rays_base + f.h_ctr->ext_rays + f.h_ctr->shadow_rays;
  const bool overflow = (f.h_ctr->error_flags & ERR_STACK_OVERFLOW) != 0;
  Clock::time_point now = Clock::now();
  for (auto &r : f.finishing) {
    if (overflow) {
      fail_request(s, r, PT_ERR_DEVICE, "BVH traversal stack overflow");
      continue;
    }
    if (r->end_status != PT_OK) {
      fail_request(s, r, r->end_status, r->end_msg);
      continue;
    }
    r->state = RState::Done;
    r->t_done = now;
    s->st.completed++;
  }
  f.finishing.clear();
  s->cv_done.notify_all();
}

void free_dead(pt_server *s) {
  cudaStream_t stream = s->eng->stream;
  for (auto &a : s->dead_accums) {
    if (!a->t.d_accum) continue;
    cudaFreeAsync(a->t.d_accum, stream);
    a->t.d_accum = nullptr;
    s->accum_count--;
  }
  s->dead_accums.clear();
  for (auto &e : s->dead_scenes) evict(s, *e);
  s->dead_scenes.clear();
}

// Ends request `r` with `st` (PT_ERR_CANCELLED or PT_ERR_TIMEOUT). Called
// with the lock held. A queued request leaves the queue. An admitted one
// gets no further waves: its waves on the GPU still add to its accumulator,
// which is left inconsistent, so the accumulation fails for continuations;
// stream-ordered frees keep its memory alive until those waves are done. A
// request whose last wave was launched ends when that wave completes.
pt_status end_request(pt_server *s, const std::shared_ptr<Request> &r, pt_status st, const std::string &msg) {
  if (r->state == RState::Done || r->state == RState::Failed)
    return sfail(PT_ERR_INVALID_ARG, "request " + std::to_string(r->ticket) + " has already finished");
  (st == PT_ERR_CANCELLED ? s->st.cancelled : s->st.timed_out)++;
  if (r->state == RState::Pending) {
    auto it = std::find(s->pending.begin(), s->pending.end(), r);
    if (it != s->pending.end()) s->pending.erase(it);
    if (!r->in.continues) {
      fail_admission(s, r, st, msg);
    } else {
      fail_request(s, r, st, msg);
    }
  } else {
    auto it = std::find(s->active.begin(), s->active.end(), r);
    if (it != s->active.end()) {
      s->active.erase(it);
      Accum &acc = *r->acc;
      acc.busy = false;
      acc.failed = true;
      acc.fail_status = st;
      acc.fail_msg = msg + " with samples still to add";
      acc.scene->pins--;
      fail_request(s, r, st, msg);
    } else {
      r->end_status = st;  // its last wave is on the GPU
      r->end_msg = msg;
    }
  }
  s->cv_work.notify_all();
  return PT_OK;
}

// Ends every queued or admitted request whose deadline has passed, and
// returns the nearest deadline still ahead (or `far`).
Clock::time_point expire_deadlines(pt_server *s, Clock::time_point far) {
  const Clock::time_point now = Clock::now();
  Clock::time_point next = far;
  std::vector<std::shared_ptr<Request>> due;
  auto check = [&](const std::shared_ptr<Request> &r) {
    if (!r->has_deadline || r->end_status != PT_OK) return;
    if (r->deadline <= now)
      due.push_back(r);
    else
      next = std::min(next, r->deadline);
  };
  for (auto &r : s->pending) check(r);
  for (auto &r : s->active) check(r);
  for (auto &r : due) end_request(s, r, PT_ERR_TIMEOUT, "deadline of " + std::to_string(r->in.deadline_ms) + " ms passed");
  return next;
}

void worker_main(pt_server *s) {
  cudaSetDevice(s->eng->device);
  std::unique_lock<std::mutex> lk(s->mu);
  const Clock::time_point far = Clock::time_point::max();
  for (;;) {
    free_dead(s);
    const Clock::time_point next_deadline = expire_deadlines(s, far);
    if (!s->stop && !s->broken) admit(s, lk);
    if (!s->stop && !s->broken && !s->tune_pending && !s->active.empty() && s->inflight.size() < s->depth) {
      launch_next_wave(s);
      continue;
    }
    if (!s->inflight.empty()) {
      size_t fi = s->inflight.front();
      cudaEvent_t ev = s->flights[fi].ev_end;
      lk.unlock();
      cudaError_t e = cudaEventSynchronize(ev);
      lk.lock();
      complete_flight(s, fi, e);
      continue;
    }
    if (s->stop) break;
    if (next_deadline == far)
      s->cv_work.wait(lk);
    else
      s->cv_work.wait_until(lk, next_deadline);
  }
  for (auto &r : s->active) fail_request(s, r, PT_ERR_CANCELLED, "server stopped");
  s->active.clear();
  for (auto &r : s->pending) fail_request(s, r, PT_ERR_CANCELLED, "server stopped");
  s->pending.clear();
  free_dead(s);
}

template <class F>
pt_status sguard(F &&f) {
  try {
    return f();
  } catch (const std::bad_alloc &) {
    return sfail(PT_ERR_OOM, "host allocation failed");
  } catch (const std::exception &e) {
    return sfail(PT_ERR_DEVICE, e.what());
  } catch (...) {
    return sfail(PT_ERR_DEVICE, "unknown failure");
  }
}

}  // namespace

extern "C" {

pt_status pt_server_create(pt_context *ctx, const pt_server_config *cfg, pt_server **out) {
  if (!ctx || !out) return sfail(PT_ERR_INVALID_ARG, "ctx / out is NULL");
  *out = nullptr;
  return sguard([&]() -> pt_status {
    auto s = std::make_unique<pt_server>();
    pt_status st = engine_create(ctx->device, &s->eng);
    if (st != PT_OK) return sfail(st, pt_last_error(nullptr));
    pt_server_config c{};
    if (cfg) c = *cfg;
    s->budget = c.hbm_budget_bytes;
    if (c.wave_slots) s->wave_slots = std::max<uint32_t>(c.wave_slots, 1024);
    if (c.max_active) s->max_active = c.max_active;
    if (c.pipeline_depth) s->depth = std::min<uint32_t>(c.pipeline_depth, 8);
    s->eng->schedule = c.megakernel ? PT_SCHEDULE_MEGAKERNEL : PT_SCHEDULE_WAVEFRONT;
    s->eng->wave_slots = s->wave_slots;
    s->eng->wide_nodes = (c.node_width_extension == 2 ? 0u : WIDE_EXTENSION) |
                         (c.node_width_shadow == 2 ? 0u : WIDE_SHADOW);
    s->eng->material_sort = c.material_sort_off == 0;
    if (c.wave_overlap_off) {
      s->eng->overlap_waves = false;
      s->eng->overlap_arenas = 0;
    }
    s->autotune = c.autotune != 0;
    {
      // Accumulators and wave tables are stream-ordered allocations from the
      // device's default pool: keep freed memory cached in the pool instead
      // of returning it at every synchronisation (a request's accumulator
      // comes and goes with every request).
      cudaMemPool_t pool = nullptr;
      if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess) {
        uint64_t keep = c.hbm_budget_bytes ? c.hbm_budget_bytes : UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      }
      cudaGetLastError();
    }
    s->spatial_bvh = c.bvh_binned == 0;
    s->flights.resize(s->depth + 1);
    cudaError_t e = cudaSuccess;
    for (Flight &f : s->flights) {
      if (e == cudaSuccess) e = cudaEventCreate(&f.ev_start);
      if (e == cudaSuccess) e = cudaEventCreate(&f.ev_end);
      if (e == cudaSuccess) e = cudaMallocHost((void **)&f.h_ctr, sizeof(DevCounters));
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(s->eng->d_ctr, 0, sizeof(DevCounters), s->eng->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->eng->stream);
    s->overlap = e == cudaSuccess && s->eng->schedule == PT_SCHEDULE_WAVEFRONT && s->eng->overlap_waves;
    if (s->overlap) {
      e = cudaStreamCreateWithFlags(&s->upload, cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_free, cudaEventDisableTiming);
      if (e == cudaSuccess && engine_overlap_begin(s->eng) != PT_OK) e = cudaErrorUnknown;
    }
    if (e != cudaSuccess) {
      pt_server_destroy(s.release());
      return sfail(PT_ERR_DEVICE, std::string("server setup failed: ") + cudaGetErrorString(e));
    }
    pt_server *p = s.get();
    s->worker = std::thread(worker_main, p);
    *out = s.release();
    return PT_OK;
  });
}

void pt_server_destroy(pt_server *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  if (s->eng) {
    cudaSetDevice(s->eng->device);
    for (auto &kv : s->scenes) evict(s, *kv.second);
    for (auto &kv : s->reqs) {
      Request &r = *kv.second;
      s->pinned.put(r.hdr, r.hdr_bytes);
      r.hdr = nullptr;
      if (r.acc && r.acc->t.d_accum) {
        cudaFreeAsync(r.acc->t.d_accum, s->eng->stream);
        r.acc->t.d_accum = nullptr;
      }
    }
    if (s->d_resolve) cudaFreeAsync(s->d_resolve, s->eng->stream);
    cudaStreamSynchronize(s->eng->stream);
    if (s->upload) {
      cudaStreamSynchronize(s->upload);
      cudaStreamDestroy(s->upload);
    }
    if (s->ev_free) cudaEventDestroy(s->ev_free);
    for (Flight &f : s->flights) {
      if (f.ev_start) cudaEventDestroy(f.ev_start);
      if (f.ev_end) cudaEventDestroy(f.ev_end);
      if (f.d_reqs) cudaFree(f.d_reqs);
      if (f.h_reqs) cudaFreeHost(f.h_reqs);
      if (f.d_segs) cudaFree(f.d_segs);
      if (f.h_segs) cudaFreeHost(f.h_segs);
      if (f.h_ctr) cudaFreeHost(f.h_ctr);
    }
    s->pinned.clear();
    pt_destroy(s->eng);
  }
  delete s;
}

const char *pt_server_last_error(const pt_server *) { return t_err.c_str(); }

pt_status pt_server_scene_register(pt_server *s, const pt_scene_desc *desc, const pt_environment *env,
                                   uint32_t *key) {
  if (!s || !desc || !key) return sfail(PT_ERR_INVALID_ARG, "server / desc / scene_key is NULL");
  return sguard([&]() -> pt_status {
    auto e = std::make_shared<SceneEntry>();
    std::string err = build_scene_image(*desc, e->img, true, nullptr, s->spatial_bvh);
    if (!err.empty()) return sfail(PT_ERR_INVALID_ARG, err);
    e->est_bytes = e->img.device_bytes();
    if (env) {
      e->has_env = true;
      e->env = *env;
      if (env->pixels && env->width && env->height) {
        e->env_pixels.assign(env->pixels, env->pixels + (size_t)env->width * env->height * 4);
        e->env.pixels = e->env_pixels.data();
      } else {
        e->env.pixels = nullptr;
      }
      e->est_bytes += env_bytes_estimate(e->env);
    }
    std::lock_guard<std::mutex> g(s->mu);
    e->key = s->next_scene++;
    s->scenes[e->key] = e;
    *key = e->key;
    return PT_OK;
  });
}

pt_status pt_server_scene_unregister(pt_server *s, uint32_t key) {
  if (!s) return sfail(PT_ERR_INVALID_ARG, "server is NULL");
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->scenes.find(key);
  if (it == s->scenes.end()) return sfail(PT_ERR_NOT_FOUND, "unknown scene " + std::to_string(key));
  SceneEntry &e = *it->second;
  if (e.pins || e.queued) return sfail(PT_ERR_INVALID_ARG, "scene " + std::to_string(key) + " has requests");
  for (auto &r : s->pending)
    if (r->acc && r->acc->scene.get() == &e)
      return sfail(PT_ERR_INVALID_ARG, "scene " + std::to_string(key) + " has requests");
  e.registered = false;
  s->dead_scenes.push_back(it->second);
  s->scenes.erase(it);
  s->cv_work.notify_all();
  return PT_OK;
}

pt_status pt_server_scene_info(pt_server *s, uint32_t key, uint64_t *device_bytes, int *resident) {
  if (!s) return sfail(PT_ERR_INVALID_ARG, "server is NULL");
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->scenes.find(key);
  if (it == s->scenes.end()) return sfail(PT_ERR_NOT_FOUND, "unknown scene " + std::to_string(key));
  if (device_bytes) *device_bytes = it->second->est_bytes;
  if (resident) *resident = it->second->dev ? 1 : 0;
  return PT_OK;
}

pt_status pt_server_submit(pt_server *s, const pt_server_request *in, uint64_t *ticket) {
  if (!s || !in || !ticket) return sfail(PT_ERR_INVALID_ARG, "server / request / ticket is NULL");
  return sguard([&]() -> pt_status {
    if (in->samples == 0) return sfail(PT_ERR_INVALID_ARG, "samples must be >= 1");
    if (!in->continues) {
      if (check_options(nullptr, &in->camera, &in->options) != PT_OK)
        return sfail(PT_ERR_INVALID_ARG, pt_last_error(nullptr));
    }
    auto r = std::make_shared<Request>();
    r->in = *in;
    std::lock_guard<std::mutex> g(s->mu);
    if (s->broken) return sfail(PT_ERR_DEVICE, "server stopped after a device error: " + s->broken_msg);
    if (s->stop) return sfail(PT_ERR_CANCELLED, "server is stopping");
    if (in->continues) {
      auto it = s->reqs.find(in->continues);
      if (it == s->reqs.end())
        return sfail(PT_ERR_NOT_FOUND, "ticket " + std::to_string(in->continues) + " is unknown or released");
      r->acc = it->second->acc;
      if (r->acc->failed) return sfail(PT_ERR_INVALID_ARG, "the continued request failed: " + r->acc->fail_msg);
      r->acc->refs++;
    } else {
      auto it = s->scenes.find(in->scene);
      if (it == s->scenes.end()) return sfail(PT_ERR_NOT_FOUND, "unknown scene " + std::to_string(in->scene));
      r->scene = it->second;
      r->scene->queued++;
      auto acc = std::make_shared<Accum>();
      pt_tracer &t = acc->t;
      t.ctx = s->eng;
      t.cam = in->camera;
      t.opts = in->options;
      t.w = std::max(in->options.width, 1u);
      t.h = std::max(in->options.height, 1u);
      t.scene_id = r->scene->key;
      acc->scene = r->scene;
      acc->refs = 1;
      r->acc = acc;
    }
    r->w = r->acc->t.w;
    r->h = r->acc->t.h;
    r->ticket = s->next_ticket++;
    r->t_submit = Clock::now();
    if (in->deadline_ms) {
      r->has_deadline = true;
      r->deadline = r->t_submit + std::chrono::milliseconds(in->deadline_ms);
    }
    s->reqs[r->ticket] = r;
    s->pending.push_back(r);
    s->st.submitted++;
    *ticket = r->ticket;
    s->cv_work.notify_all();
    return PT_OK;
  });
}

pt_status pt_server_wait(pt_server *s, uint64_t ticket, int32_t timeout_ms, float *hdr, size_t hdr_floats,
                         pt_request_stats *stats) {
  if (!s) return sfail(PT_ERR_INVALID_ARG, "server is NULL");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return sfail(PT_ERR_NOT_FOUND, "ticket " + std::to_string(ticket) + " is unknown");
  std::shared_ptr<Request> r = it->second;
  auto ready = [&] { return r->state == RState::Done || r->state == RState::Failed; };
  if (timeout_ms < 0)
    s->cv_done.wait(lk, ready);
  else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
    return sfail(timeout_ms == 0 ? PT_ERR_NOT_READY : PT_ERR_TIMEOUT,
                 "request " + std::to_string(ticket) + " still running");
  if (r->state == RState::Failed) return sfail(r->status, r->error);
  const size_t nf = (size_t)r->w * r->h * 4;
  if (hdr) {
    if (hdr_floats < nf) return sfail(PT_ERR_INVALID_ARG, "output buffer too small");
    // The copy runs without the lock (the worker keeps launching waves);
    // release waits for readers before the pinned buffer is recycled.
    r->readers++;
    lk.unlock();
    std::memcpy(hdr, r->hdr, nf * sizeof(float));
    lk.lock();
    if (--r->readers == 0) s->cv_done.notify_all();
  }
  if (stats) {
    stats->queue_ms = ms_between(r->t_submit, r->t_admit);
    stats->latency_ms = ms_between(r->t_submit, r->t_done);
    stats->width = r->w;
    stats->height = r->h;
    stats->samples = r->samples_after;
    stats->waves = r->waves;
  }
  return PT_OK;
}

pt_status pt_server_poll(pt_server *s, uint64_t ticket, float *hdr, size_t hdr_floats, pt_request_stats *stats) {
  return pt_server_wait(s, ticket, 0, hdr, hdr_floats, stats);
}

pt_status pt_server_cancel(pt_server *s, uint64_t ticket) {
  if (!s) return sfail(PT_ERR_INVALID_ARG, "server is NULL");
  return sguard([&]() -> pt_status {
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return sfail(PT_ERR_NOT_FOUND, "ticket " + std::to_string(ticket) + " is unknown");
    return end_request(s, it->second, PT_ERR_CANCELLED, "request " + std::to_string(ticket) + " was cancelled");
  });
}

pt_status pt_server_debug_fail_allocations(pt_server *s, uint32_t count) {
  if (!s) return sfail(PT_ERR_INVALID_ARG, "server is NULL");
  s->fail_allocs.store(count);
  return PT_OK;
}

pt_status pt_server_release(pt_server *s, uint64_t ticket) {
  if (!s) return sfail(PT_ERR_INVALID_ARG, "server is NULL");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return sfail(PT_ERR_NOT_FOUND, "ticket " + std::to_string(ticket) + " is unknown");
  std::shared_ptr<Request> keep = it->second;
  Request &r = *keep;
  if (r.state != RState::Done && r.state != RState::Failed)
    return sfail(PT_ERR_INVALID_ARG, "request " + std::to_string(ticket) + " is still running");
  // A wait of another thread may still be copying the image out.
  s->cv_done.wait(lk, [&] { return r.readers == 0; });
  it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return sfail(PT_ERR_NOT_FOUND, "ticket " + std::to_string(ticket) + " is unknown");
  s->pinned.put(r.hdr, r.hdr_bytes);
  r.hdr = nullptr;
  if (r.acc && --r.acc->refs == 0) s->dead_accums.push_back(r.acc);
  s->reqs.erase(it);
  s->cv_work.notify_all();
  return PT_OK;
}

pt_status pt_server_stats_get(pt_server *s, pt_server_stats *out) {
  if (!s || !out) return sfail(PT_ERR_INVALID_ARG, "server / out is NULL");
  std::lock_guard<std::mutex> g(s->mu);
  *out = s->st;
  uint32_t res = 0;
  for (auto &kv : s->scenes) res += kv.second->dev ? 1u : 0u;
  out->resident_scenes = res;
  out->active = (uint32_t)s->active.size();
  out->pending = (uint32_t)s->pending.size();
  out->accumulators = s->accum_count;
  return PT_OK;
}

}  // extern "C"
