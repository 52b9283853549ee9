// extern "C" entry points (include/pt_b200.h, include/pt_b200_debug.h).
//
// pt_tracer mirrors PathTracer (src/pathtrace.rs:2369-2735): the same reset
// rule (radiance_key, :2402-2418), sample indices continuing across refine
// calls (:2526-2591) and the same resolve (:2593-2734), with the f64
// accumulator resident on the device. No exception crosses the ABI: every
// entry point catches and maps failures to a pt_status plus a message.
#include <algorithm>
#include <functional>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pt_b200.h"
#include "../../include/pt_b200_debug.h"
#include "context.h"
#include "host_scene.h"
#include "kernels.h"

using namespace ptd;

namespace {

thread_local std::string g_create_error;

pt_status fail(pt_context *ctx, pt_status st, const std::string &msg) {
  if (ctx)
    ctx->err = msg;
  else
    g_create_error = msg;
  return st;
}

#define CK(ctx, call)                                                                            \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      return fail((ctx), e_ == cudaErrorMemoryAllocation ? PT_ERR_OOM : PT_ERR_DEVICE,           \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                           \
  } while (0)

// Consumes one injected allocation failure of `ctx`, if armed.
bool injected_oom(pt_context *ctx) {
  if (!ctx) return false;
  uint32_t n = ctx->fail_allocs.load();
  while (n > 0)
    if (ctx->fail_allocs.compare_exchange_weak(n, n - 1)) return true;
  return false;
}

// cudaMalloc, or the injected out-of-memory failure.
template <class T>
cudaError_t dev_malloc(pt_context *ctx, T **p, size_t bytes) {
  if (injected_oom(ctx)) return cudaErrorMemoryAllocation;
  return cudaMalloc(p, bytes);
}

template <class F>
pt_status guard(pt_context *ctx, F &&f) {
  try {
    return f();
  } catch (const std::bad_alloc &) {
    return fail(ctx, PT_ERR_OOM, "host allocation failed");
  } catch (const std::exception &e) {
    return fail(ctx, PT_ERR_DEVICE, e.what());
  } catch (...) {
    return fail(ctx, PT_ERR_DEVICE, "unknown failure");
  }
}

template <class T>
pt_status ensure(pt_context *ctx, T *&p, size_t &cap, size_t need) {
  if (need <= cap && p) return PT_OK;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  CK(ctx, dev_malloc(ctx, &p, std::max<size_t>(need, 1) * sizeof(T)));
  cap = need;
  return PT_OK;
}

bool same_radiance_key(const pt_tracer &t, const pt_camera &cam, const pt_render_options &o) {
  const pt_render_options &a = t.opts;
  pt_path_trace_options pa = a.path_trace, pb = o.path_trace;
  pa.samples_per_pixel = pb.samples_per_pixel = 0;
  return std::memcmp(&t.cam, &cam, sizeof cam) == 0 && a.width == o.width && a.height == o.height &&
         std::memcmp(&a.ambient, &o.ambient, sizeof(float)) == 0 && std::memcmp(&pa, &pb, sizeof pa) == 0;
}

pt_status validate_opts(pt_context *ctx, const pt_camera *cam, const pt_render_options *o) {
  if (!cam || !o) return fail(ctx, PT_ERR_INVALID_ARG, "camera / options pointer is NULL");
  if (o->path_trace.max_bounces > 1024)
    return fail(ctx, PT_ERR_INVALID_ARG, "path_trace.max_bounces must be <= 1024");
  if (o->path_trace.strategy > PT_BSDF_ONLY) return fail(ctx, PT_ERR_INVALID_ARG, "unknown light strategy");
  if (o->tone_map > PT_TONE_ACES) return fail(ctx, PT_ERR_INVALID_ARG, "unknown tone map");
  if (cam->projection > PT_ORTHOGRAPHIC) return fail(ctx, PT_ERR_INVALID_ARG, "unknown projection");
  uint64_t px = (uint64_t)std::max(o->width, 1u) * std::max(o->height, 1u);
  if (px > (1ull << 28)) return fail(ctx, PT_ERR_INVALID_ARG, "image larger than 268435456 pixels");
  return PT_OK;
}

}  // namespace

namespace ptd {

DevRequest make_request(const pt_tracer &t, const SceneHost &sc, const EnvHost *env) {
  DevRequest rq;
  std::memset(&rq, 0, sizeof rq);
  rq.scene = sc.d_desc;
  rq.env = env ? env->d_desc : nullptr;
  rq.cam = t.cam;
  rq.width = t.w;
  rq.height = t.h;
  rq.ambient = std::isfinite(t.opts.ambient) ? std::fmax(t.opts.ambient, 0.0f) : 0.0f;
  rq.pixel_spread = 2.0f * t.cam.half_h / (float)t.h;
  rq.orthographic = t.cam.projection == PT_ORTHOGRAPHIC ? 1u : 0u;
  rq.max_bounces = t.opts.path_trace.max_bounces;
  rq.rr_start = t.opts.path_trace.rr_start;
  rq.seed = t.opts.path_trace.seed;
  rq.strategy = t.opts.path_trace.strategy;
  rq.clamp = t.opts.path_trace.clamp;
  rq.p_env = env ? (sc.dev.em_count > 0 ? 0.5f : 1.0f) : 0.0f;
  rq.wide_nodes = (uint32_t)(WIDE_EXTENSION | WIDE_SHADOW);
  if (t.ctx) {
    rq.wide_nodes = t.ctx->wide_nodes;
    auto it = t.ctx->tuned.find(scene_class(sc, env != nullptr));
    if (it != t.ctx->tuned.end()) rq.wide_nodes = it->second.wide_nodes;
  }
  rq.accum = t.d_accum;
  return rq;
}

Job make_job(const pt_tracer &t, const SceneHost &sc, const EnvHost *env, uint32_t n) {
  Job j{};
  j.req = make_request(t, sc, env);
  j.target = n;
  j.first = t.samples;
  j.npix = t.w * t.h;
  j.iterations = t.opts.path_trace.max_bounces + 1;
  j.shadow_slots = sc.light_count + 1;
  j.scene_key = t.scene_id;
  j.area = sc.dev.em_count > 0 || env != nullptr;
  j.wide = sc.dev.nodes4 ? j.req.wide_nodes & (uint32_t)(WIDE_EXTENSION | WIDE_SHADOW) : 0u;
  return j;
}

std::vector<WaveSegment> pack_wave(std::vector<Job> &jobs, const std::vector<uint32_t> &order, uint64_t cap) {
  std::vector<WaveSegment> segs;
  uint64_t slot = 0;
  for (uint32_t oj = 0; oj < order.size() && slot < cap; ++oj) {
    const uint32_t j = order[oj];
    Job &jb = jobs[j];
    if (jb.finished()) continue;
    uint64_t left = cap - slot;
    if (jb.pix_done > 0 || jb.npix > left) {
      // One pixel range of one sample (the image is larger than what is
      // left of the wave, or a previous wave ended inside this sample).
      uint32_t m = (uint32_t)std::min<uint64_t>(jb.npix - jb.pix_done, left);
      if (m == 0) continue;
      segs.push_back(WaveSegment{j, (uint32_t)slot, jb.pix_done, m, jb.first + jb.done, 1, 0, 0});
      slot += m;
      jb.pix_done += m;
      if (jb.pix_done == jb.npix) {
        jb.pix_done = 0;
        jb.done += 1;
      }
    } else {
      uint32_t c = (uint32_t)std::min<uint64_t>(jb.target - jb.done, left / jb.npix);
      segs.push_back(WaveSegment{j, (uint32_t)slot, 0, jb.npix, jb.first + jb.done, c, 0, 0});
      slot += (uint64_t)jb.npix * c;
      jb.done += c;
    }
  }
  return segs;
}

pt_status check_options(pt_context *ctx, const pt_camera *cam, const pt_render_options *o) {
  return validate_opts(ctx, cam, o);
}

uint32_t scene_class(const SceneHost &sc, bool env) {
  uint32_t scale = 0;
  for (uint64_t t = std::max<uint64_t>(sc.tri_count, 1); t >= 4; t >>= 2) ++scale;
  return scale | (sc.dev.em_count > 0 ? 1u << 8 : 0u) | (env ? 1u << 9 : 0u) | (sc.light_count > 0 ? 1u << 10 : 0u) |
         (sc.dev.texture_count > 0 ? 1u << 11 : 0u);
}

float4 bg_linear(const pt_render_options &o) {
  return make_float4(host_srgb_to_linear((float)o.background[0] / 255.0f),
                     host_srgb_to_linear((float)o.background[1] / 255.0f),
                     host_srgb_to_linear((float)o.background[2] / 255.0f), (float)o.background[3] / 255.0f);
}

}  // namespace ptd

namespace {

SceneHost *find_scene(pt_context *ctx, uint32_t id) {
  auto it = ctx->scenes.find(id);
  return it == ctx->scenes.end() ? nullptr : it->second.get();
}

// (Re)allocates wavefront arena `which` (0 or 1) for `capacity` slots with
// `shadow_slots` queued shadow rays each and `iterations` bounce rounds.
pt_status ensure_wavefront(pt_context *ctx, uint32_t capacity, uint32_t shadow_slots, uint32_t iterations,
                           int which = 0) {
  WaveBuffers &w = which ? ctx->wf_more[which - 1] : ctx->wf;
  void *&arena = which ? ctx->wf_arena_more[which - 1] : ctx->wf_arena;
  size_t &arena_bytes = which ? ctx->wf_bytes_more[which - 1] : ctx->wf_bytes;
  if (arena && w.capacity >= capacity && w.shadow_slots >= shadow_slots) {
    if (w.iterations >= iterations) return PT_OK;
  }
  if (arena) {
    // Every wave of earlier calls has finished: refines synchronise
    // ctx->stream, whose accumulates wait for the waves traced elsewhere.
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    cudaFree(arena);
    arena = nullptr;
    arena_bytes = 0;
  }
  // Captured waves point into the old arena.
  for (auto &kv : ctx->graphs) cudaGraphExecDestroy(kv.second);
  ctx->graphs.clear();
  capacity = std::max(capacity, w.capacity);
  shadow_slots = std::max(shadow_slots, w.shadow_slots);
  iterations = std::max(iterations, w.iterations);
  size_t P = capacity, S = shadow_slots;
  size_t sizes[] = {16 * P, 16 * P, 16 * P, 16 * P, 16 * P, 16 * P, 16 * P,  // o d beta rad prev sigma seed
                    16 * P, 4 * P,                                           // hit_tb hit_g
                    16 * P * S, 16 * P * S, 16 * P * S, 4 * P,               // sh_o sh_d sh_c sh_n
                    4 * P, 4 * P, 4 * P,                                     // q0 q1 q_shadow
                    4 * (size_t)kWfCounterStride * (iterations + 1),
                    4 * P, 4 * 2 * (size_t)kSortBuckets * (iterations + 1),   // q_sorted sort_counts
                    sizeof(WaveDesc), 4 * P,                                   // desc sort_keys
                    3 * 16 * P,                                                // nee
                    P * S};                                                    // sh_vis
  size_t off[sizeof(sizes) / sizeof(sizes[0])], total = 0;
  for (size_t i = 0; i < sizeof(sizes) / sizeof(sizes[0]); ++i) {
    total = (total + 255) & ~(size_t)255;
    off[i] = total;
    total += sizes[i];
  }
  CK(ctx, dev_malloc(ctx, &arena, total));
  arena_bytes = total;
  char *b = static_cast<char *>(arena);
  int k = 0;
  w.o = (float4 *)(b + off[k++]);
  w.d = (float4 *)(b + off[k++]);
  w.beta = (float4 *)(b + off[k++]);
  w.rad = (float4 *)(b + off[k++]);
  w.prev = (float4 *)(b + off[k++]);
  w.sigma = (float4 *)(b + off[k++]);
  w.seed = (uint4 *)(b + off[k++]);
  w.hit_tb = (float4 *)(b + off[k++]);
  w.hit_g = (uint32_t *)(b + off[k++]);
  w.sh_o = (float4 *)(b + off[k++]);
  w.sh_d = (float4 *)(b + off[k++]);
  w.sh_c = (float4 *)(b + off[k++]);
  w.sh_n = (uint32_t *)(b + off[k++]);
  w.q[0] = (uint32_t *)(b + off[k++]);
  w.q[1] = (uint32_t *)(b + off[k++]);
  w.q_shadow = (uint32_t *)(b + off[k++]);
  w.counters = (uint32_t *)(b + off[k++]);
  w.q_sorted = (uint32_t *)(b + off[k++]);
  w.sort_counts = (uint32_t *)(b + off[k++]);
  w.desc = (WaveDesc *)(b + off[k++]);
  w.sort_keys = (uint32_t *)(b + off[k++]);
  w.nee = (float4 *)(b + off[k++]);
  w.sh_vis = (uint8_t *)(b + off[k++]);
  w.capacity = capacity;
  w.shadow_slots = shadow_slots;
  w.iterations = iterations;
  return PT_OK;
}

// Runs a batch of refine jobs in merged waves: every wave carries path
// slots of several tracers, each path reading its own request (scene,
// camera, options, accumulator). Per-sample radiance is a pure function of
// (request, pixel, sample), and each pixel's samples are accumulated in
// sample order, so every tracer ends bit-identical to refining it alone.
pt_status run_jobs(pt_context *ctx, std::vector<pt_tracer *> &tracers, std::vector<Job> &jobs,
                   pt_tracer *stats_to) {
  if (jobs.empty()) return PT_OK;
  CK(ctx, cudaSetDevice(ctx->device));
  uint32_t max_iter = 1, max_shadow = 1;
  for (const Job &jb : jobs) {
    max_iter = std::max(max_iter, jb.iterations);
    max_shadow = std::max(max_shadow, jb.shadow_slots);
  }
  // Visit jobs grouped by scene (stable within a scene) so a wave mostly
  // traverses one BVH: cache locality only, results do not depend on it.
  std::vector<uint32_t> order(jobs.size());
  for (uint32_t j = 0; j < jobs.size(); ++j) order[j] = j;
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return jobs[a].scene_key < jobs[b].scene_key; });
  const uint64_t cap = std::max<uint32_t>(ctx->wave_slots, 1024);
  std::vector<std::vector<WaveSegment>> waves;
  for (;;) {
    std::vector<WaveSegment> w = pack_wave(jobs, order, cap);
    if (w.empty()) break;
    waves.push_back(std::move(w));
  }
  std::vector<WaveSegment> flat;
  std::vector<size_t> first_seg;
  size_t max_slots = 0;
  for (auto &w : waves) {
    first_seg.push_back(flat.size());
    size_t slots = 0;
    for (WaveSegment &s : w) {
      slots += (size_t)s.pixel_count * s.spp;
      flat.push_back(s);
    }
    max_slots = std::max(max_slots, slots);
  }
  // Overlapped waves need the wavefront, two or more waves, and no per-stage
  // timing (whose events sit on one stream).
  const bool overlap = ctx->overlap_waves && ctx->schedule == PT_SCHEDULE_WAVEFRONT && waves.size() >= 2 &&
                       !ctx->stage_timing;
  pt_status st = engine_reserve(ctx, max_slots, max_shadow, max_iter, overlap);
  if (st != PT_OK) return st;
  if ((st = ensure(ctx, ctx->d_segs, ctx->seg_cap, flat.size())) != PT_OK) return st;
  if ((st = ensure(ctx, ctx->d_reqs, ctx->req_cap, jobs.size())) != PT_OK) return st;
  std::vector<DevRequest> reqs(jobs.size());
  for (size_t j = 0; j < jobs.size(); ++j) reqs[j] = jobs[j].req;
  CK(ctx, cudaMemcpyAsync(ctx->d_reqs, reqs.data(), reqs.size() * sizeof(DevRequest), cudaMemcpyHostToDevice,
                          ctx->stream));
  CK(ctx, cudaMemcpyAsync(ctx->d_segs, flat.data(), flat.size() * sizeof(WaveSegment), cudaMemcpyHostToDevice,
                          ctx->stream));
  CK(ctx, cudaMemsetAsync(ctx->d_ctr, 0, sizeof(DevCounters), ctx->stream));
  StageTimer timer;
  if (ctx->stage_timing) {
    size_t need = waves.size() * (4 * (size_t)max_iter + 3) + 1;
    while (ctx->stage_events.size() < need) {
      cudaEvent_t ev;
      CK(ctx, cudaEventCreate(&ev));
      ctx->stage_events.push_back(ev);
    }
    timer.events = ctx->stage_events.data();
    timer.capacity = ctx->stage_events.size();
  }
  CK(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
  if (overlap && (st = engine_overlap_begin(ctx)) != PT_OK) return st;
  for (size_t i = 0; i < waves.size(); ++i) {
    uint32_t iters = 1, wide = WIDE_EXTENSION | WIDE_SHADOW;
    bool area = false;
    for (const WaveSegment &s : waves[i]) {
      iters = std::max(iters, jobs[s.request].iterations);
      area = area || jobs[s.request].area;
      wide &= jobs[s.request].wide;
    }
    st = launch_wave(ctx, ctx->d_reqs, ctx->d_segs + first_seg[i], waves[i], iters, &timer,
                     overlap ? (int)(i % ctx->overlap_arenas) : -1, area, wide);
    if (st != PT_OK) return st;
  }
  timer.mark(STAGE_END, ctx->stream);
  CK(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
  DevCounters c;
  CK(ctx, cudaMemcpyAsync(&c, ctx->d_ctr, sizeof c, cudaMemcpyDeviceToHost, ctx->stream));
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  float ms = 0.0f;
  CK(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  ctx->last_batch_ms = ms;
  ctx->last_batch_waves = (uint32_t)waves.size();
  {
    uint64_t samples = 0, rounds = 0;
    for (const Job &jb : jobs) samples += (uint64_t)jb.npix * jb.target;
    for (const auto &wv : waves) {
      uint32_t iters = 1;
      for (const WaveSegment &s : wv) iters = std::max(iters, jobs[s.request].iterations);
      rounds += iters;
    }
    const uint64_t v[9] = {c.ext_rays, c.shadow_rays, c.ext_nodes, c.ext_tris, c.sh_nodes, c.sh_tris, samples,
                           (uint64_t)waves.size(), rounds};
    std::memcpy(ctx->last_batch_counts, v, sizeof v);
    for (int k = 0; k < STAGE_COUNT; ++k) ctx->last_batch_stage_ms[k] = 0.0f;
    for (size_t i = 0; i + 1 < timer.count(); ++i) {
      float sm = 0.0f;
      CK(ctx, cudaEventElapsedTime(&sm, ctx->stage_events[i], ctx->stage_events[i + 1]));
      ctx->last_batch_stage_ms[timer.kinds[i]] += sm;
    }
  }
  if (stats_to) {
    pt_tracer *t = stats_to;
    t->last_ms = ms;
    t->ext = c.ext_rays;
    t->sh = c.shadow_rays;
    t->ext_nodes = c.ext_nodes;
    t->ext_tris = c.ext_tris;
    t->sh_nodes = c.sh_nodes;
    t->sh_tris = c.sh_tris;
    for (int k = 0; k < STAGE_COUNT; ++k) t->stage_ms[k] = 0.0f;
    for (size_t i = 0; i + 1 < timer.count(); ++i) {
      float sm = 0.0f;
      CK(ctx, cudaEventElapsedTime(&sm, ctx->stage_events[i], ctx->stage_events[i + 1]));
      t->stage_ms[timer.kinds[i]] += sm;
    }
  }
  ctx->last_batch_rays = c.ext_rays + c.shadow_rays;
  if (c.error_flags & ERR_STACK_OVERFLOW) return fail(ctx, PT_ERR_DEVICE, "BVH traversal stack overflow");
  for (size_t j = 0; j < jobs.size(); ++j) tracers[j]->samples += jobs[j].target;
  return PT_OK;
}

// Appends the job of tracer `t` (n more samples) to a batch.
pt_status add_job(pt_context *ctx, pt_tracer *t, uint32_t n, std::vector<pt_tracer *> &tracers,
                  std::vector<Job> &jobs) {
  SceneHost *sc = find_scene(ctx, t->scene_id);
  if (!sc) return fail(ctx, PT_ERR_EVICTED, "scene " + std::to_string(t->scene_id) + " is no longer resident");
  tracers.push_back(t);
  jobs.push_back(make_job(*t, *sc, t->env.get(), n));
  return PT_OK;
}

// Applies a tuned configuration's wave-level knobs for one call and
// restores the context's own afterwards.
struct KnobScope {
  pt_context *ctx;
  uint32_t schedule, wave_slots, shade_blocks, arenas, trav_threads, claim_chunk;
  bool sort;
  KnobScope(pt_context *c, const TuneChoice *tc)
      : ctx(c), schedule(c->schedule), wave_slots(c->wave_slots), shade_blocks(c->shade_blocks),
        arenas(c->overlap_arenas), trav_threads(c->trav_threads), claim_chunk(c->claim_chunk),
        sort(c->material_sort) {
    if (tc) {
      c->schedule = tc->schedule;
      c->wave_slots = tc->wave_slots;
      c->material_sort = tc->material_sort != 0;
      c->shade_blocks = tc->shade_blocks;
      c->trav_threads = tc->trav_threads;
      c->claim_chunk = tc->claim_chunk;
      // The tuned number of waves in flight, unless overlap is switched off
      // or its count was set explicitly.
      if (c->overlap_waves && !c->overlap_fixed) c->overlap_arenas = tc->arenas;
    }
  }
  ~KnobScope() {
    ctx->schedule = schedule;
    ctx->wave_slots = wave_slots;
    ctx->material_sort = sort;
    ctx->shade_blocks = shade_blocks;
    ctx->overlap_arenas = arenas;
    ctx->trav_threads = trav_threads;
    ctx->claim_chunk = claim_chunk;
  }
};

pt_status refine_impl(pt_tracer *t, uint32_t n) {
  if (!t->have_state || n == 0) return PT_OK;
  n = std::min(n, 0xffffffffu - t->samples);
  if (n == 0) return PT_OK;
  pt_context *ctx = t->ctx;
  const TuneChoice *tc = nullptr;
  if (SceneHost *sc = find_scene(ctx, t->scene_id)) {
    auto it = ctx->tuned.find(scene_class(*sc, t->env != nullptr));
    if (it != ctx->tuned.end()) tc = &it->second;
  }
  KnobScope knobs(ctx, tc);
  std::vector<pt_tracer *> tracers;
  std::vector<Job> jobs;
  pt_status st = add_job(ctx, t, n, tracers, jobs);
  if (st != PT_OK) return st;
  return run_jobs(ctx, tracers, jobs, t);
}

// Calibration refines of `samples` spp of t's scene, camera and options on a
// scratch accumulator under every candidate configuration; the fastest
// (device time, best of two runs) becomes the scene class's configuration.
pt_status autotune_scene(pt_context *ctx, const pt_tracer *t, SceneHost *sc, const EnvHost *env, uint32_t samples,
                         TuneChoice &best) {
  if (samples == 0) {
    // One full wave (8,388,608 paths): the size real refines run at, where
    // per-launch costs weigh as they will in use.
    const uint64_t npix = (uint64_t)std::max(t->w, 1u) * std::max(t->h, 1u);
    samples = (uint32_t)std::min<uint64_t>(std::max<uint64_t>((1ull << 23) / npix, 1), 4096);
  }
  CK(ctx, cudaSetDevice(ctx->device));
  pt_tracer s;
  s.ctx = ctx;
  s.cam = t->cam;
  s.opts = t->opts;
  s.w = t->w;
  s.h = t->h;
  s.scene_id = t->scene_id;
  s.have_state = true;
  s.dirty = false;
  const size_t n = (size_t)s.w * s.h * 4;
  CK(ctx, cudaMalloc(&s.d_accum, n * sizeof(double)));
  s.accum_cap = n;
  struct Free {
    double *p;
    ~Free() { cudaFree(p); }
  } free_accum{s.d_accum};
  const uint32_t cls = scene_class(*sc, env != nullptr);
  std::vector<TuneChoice> cands;
  cands.push_back({PT_SCHEDULE_MEGAKERNEL, WIDE_EXTENSION | WIDE_SHADOW, 0, 1u << 22, 0.0f});
  for (uint32_t wide : {WIDE_EXTENSION | WIDE_SHADOW, (uint32_t)WIDE_SHADOW, 0u, (uint32_t)WIDE_EXTENSION})
    for (uint32_t sort : {1u, 0u})
      for (uint32_t slots : {1u << 23, 1u << 20}) cands.push_back({PT_SCHEDULE_WAVEFRONT, wide, sort, slots, 0.0f});
  KnobScope restore(ctx, nullptr);
  best = cands[0];
  float best_ms = -1.0f;
  auto time_choice = [&](TuneChoice &c, float &ms, uint32_t spp) -> pt_status {
    ctx->schedule = c.schedule;
    ctx->wave_slots = c.wave_slots;
    ctx->material_sort = c.material_sort != 0;
    ctx->shade_blocks = c.shade_blocks;
    ctx->trav_threads = c.trav_threads;
    ctx->claim_chunk = c.claim_chunk;
    if (ctx->overlap_waves) ctx->overlap_arenas = c.arenas;
    ms = -1.0f;
    for (int rep = 0; rep < 2; ++rep) {
      s.samples = 0;
      std::vector<pt_tracer *> tr{&s};
      std::vector<Job> jobs{make_job(s, *sc, env, spp)};
      jobs[0].req.wide_nodes = c.wide_nodes;
      jobs[0].wide = sc->dev.nodes4 ? c.wide_nodes : 0u;
      pt_status st = run_jobs(ctx, tr, jobs, nullptr);
      if (st != PT_OK) return st;
      if (ms < 0.0f || ctx->last_batch_ms < ms) ms = ctx->last_batch_ms;
    }
    c.samples_per_s = ms > 0.0f ? (float)((double)s.w * s.h * spp / (ms * 1e-3)) : 0.0f;
    return PT_OK;
  };
  for (TuneChoice &c : cands) {
    float ms;
    pt_status st = time_choice(c, ms, samples);
    if (st != PT_OK) return st;
    if (best_ms < 0.0f || ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  if (best.schedule == PT_SCHEDULE_WAVEFRONT) {
    // The shade kernel's occupancy on the winning configuration.
    TuneChoice c = best;
    c.shade_blocks = 4;
    float ms;
    pt_status st = time_choice(c, ms, samples);
    if (st != PT_OK) return st;
    if (ms < best_ms) {
      best_ms = ms;
      best = c;
    }
    // The traversal kernels' block size and refill chunk on the winner.
    for (auto tc2 : {std::make_pair(128u, 1u), std::make_pair(256u, 2u), std::make_pair(256u, 4u)}) {
      TuneChoice t = best;
      t.trav_threads = tc2.first;
      t.claim_chunk = tc2.second;
      if ((st = time_choice(t, ms, samples)) != PT_OK) return st;
      if (ms < best_ms) {
        best_ms = ms;
        best = t;
      }
    }
    if (ctx->overlap_waves) {
      // Waves in flight: measured on eight waves (one cannot overlap, and
      // the third arena pays off only over several).
      const uint32_t spp4 = std::min<uint32_t>(samples * 8, 32768);
      TuneChoice c2 = best, c3 = best;
      c2.arenas = 2;
      c3.arenas = 3;
      float ms2, ms3;
      if ((st = time_choice(c2, ms2, spp4)) != PT_OK) return st;
      if ((st = time_choice(c3, ms3, spp4)) != PT_OK) return st;
      best.arenas = ms3 < ms2 ? 3u : 2u;
    }
  }
  ctx->tuned[cls] = best;
  return PT_OK;
}

pt_status autotune_impl(pt_context *ctx, pt_tracer *t, uint32_t samples, TuneChoice &best) {
  if (!t->have_state) return fail(ctx, PT_ERR_INVALID_ARG, "tracer is not synced");
  SceneHost *sc = find_scene(ctx, t->scene_id);
  if (!sc) return fail(ctx, PT_ERR_EVICTED, "scene " + std::to_string(t->scene_id) + " is no longer resident");
  return autotune_scene(ctx, t, sc, t->env.get(), samples, best);
}

pt_status refine_many_impl(pt_context *ctx, pt_tracer *const *tracers, const uint32_t *samples, uint32_t count) {
  std::vector<pt_tracer *> ts;
  std::vector<Job> jobs;
  for (uint32_t i = 0; i < count; ++i) {
    pt_tracer *t = tracers[i];
    if (!t || t->ctx != ctx) return fail(ctx, PT_ERR_INVALID_ARG, "tracer " + std::to_string(i) + " is not of ctx");
    for (uint32_t j = 0; j < i; ++j)
      if (tracers[j] == t) return fail(ctx, PT_ERR_INVALID_ARG, "a tracer appears twice in one batch");
  }
  for (uint32_t i = 0; i < count; ++i) {
    pt_tracer *t = tracers[i];
    if (!t->have_state || samples[i] == 0) continue;
    uint32_t n = std::min(samples[i], 0xffffffffu - t->samples);
    if (!n) continue;
    pt_status st = add_job(ctx, t, n, ts, jobs);
    if (st != PT_OK) return st;
  }
  return run_jobs(ctx, ts, jobs, jobs.size() == 1 ? ts[0] : nullptr);
}

pt_status sync_impl(pt_tracer *t, uint32_t scene_id, const pt_camera *cam, const pt_render_options *opts, int *reset) {
  pt_context *ctx = t->ctx;
  pt_status st = validate_opts(ctx, cam, opts);
  if (st != PT_OK) return st;
  if (!find_scene(ctx, scene_id)) return fail(ctx, PT_ERR_NOT_FOUND, "unknown scene " + std::to_string(scene_id));
  bool need_prepare = t->dirty || !t->have_state || t->scene_id != scene_id;
  bool changed = need_prepare || !same_radiance_key(*t, *cam, *opts);
  t->opts = *opts;
  t->cam = *cam;
  if (reset) *reset = changed ? 1 : 0;
  if (!changed) return PT_OK;
  CK(ctx, cudaSetDevice(ctx->device));
  t->scene_id = scene_id;
  t->w = std::max(opts->width, 1u);
  t->h = std::max(opts->height, 1u);
  size_t n = (size_t)t->w * t->h * 4;
  st = ensure(ctx, t->d_accum, t->accum_cap, n);
  if (st != PT_OK) return st;
  CK(ctx, cudaMemsetAsync(t->d_accum, 0, n * sizeof(double), ctx->stream));
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  t->samples = 0;
  t->have_state = true;
  t->dirty = false;
  return PT_OK;
}

pt_status read_impl(pt_tracer *t, void *out, size_t count, bool image) {
  pt_context *ctx = t->ctx;
  if (!out) return fail(ctx, PT_ERR_INVALID_ARG, "output pointer is NULL");
  uint32_t w = t->have_state ? t->w : std::max(t->opts.width, 1u);
  uint32_t h = t->have_state ? t->h : std::max(t->opts.height, 1u);
  size_t n = (size_t)w * h;
  if (count < n * 4) return fail(ctx, PT_ERR_INVALID_ARG, "output buffer too small");
  float4 bg = bg_linear(t->opts);
  if (!t->have_state) {
    for (size_t i = 0; i < n; ++i) {
      if (image)
        std::memcpy((uint8_t *)out + 4 * i, t->opts.background, 4);
      else
        std::memcpy((float *)out + 4 * i, &bg, sizeof bg);
    }
    return PT_OK;
  }
  CK(ctx, cudaSetDevice(ctx->device));
  size_t elem = image ? 4 : 16;
  if (t->resolve_cap < n * elem) {
    if (t->d_resolve) cudaFree(t->d_resolve);
    t->d_resolve = nullptr;
    t->resolve_cap = 0;
    CK(ctx, dev_malloc(ctx, &t->d_resolve, n * elem));
    t->resolve_cap = n * elem;
  }
  if (image) {
    uchar4 bb = make_uchar4(t->opts.background[0], t->opts.background[1], t->opts.background[2],
                            t->opts.background[3]);
    CK(ctx, launch_resolve_image(t->d_accum, (uint32_t)n, t->samples, bg, bb, t->opts.tone_map, t->opts.exposure,
                                 (uchar4 *)t->d_resolve, ctx->stream));
  } else {
    CK(ctx, launch_resolve_hdr(t->d_accum, (uint32_t)n, t->samples, bg, (float4 *)t->d_resolve, ctx->stream));
  }
  CK(ctx, cudaMemcpyAsync(out, t->d_resolve, n * elem, cudaMemcpyDeviceToHost, ctx->stream));
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  return PT_OK;
}

pt_status set_env_impl(pt_tracer *t, const pt_environment *env) {
  pt_context *ctx = t->ctx;
  CK(ctx, cudaSetDevice(ctx->device));
  if (t->env) {
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    release_env(*t->env);
    t->env.reset();
  }
  if (env) {
    auto e = std::make_unique<EnvHost>();
    bool oom = false;
    std::string err = upload_env(*env, *e, oom);
    if (!err.empty()) return fail(ctx, oom ? PT_ERR_OOM : PT_ERR_DEVICE, err);
    t->env = std::move(e);
  }
  // PathTracer::set_environment resets the accumulation.
  t->samples = 0;
  if (t->have_state && t->d_accum) {
    CK(ctx, cudaMemsetAsync(t->d_accum, 0, (size_t)t->w * t->h * 4 * sizeof(double), ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return PT_OK;
}

}  // namespace

namespace ptd {
pt_status ctx_fail(pt_context *ctx, pt_status st, const std::string &msg) { return fail(ctx, st, msg); }
SceneHost *ctx_find_scene(pt_context *ctx, uint32_t id) { return find_scene(ctx, id); }
pt_status autotune(pt_context *ctx, const pt_tracer *t, SceneHost &sc, const EnvHost *env, uint32_t samples,
                   TuneChoice &best) {
  return autotune_scene(ctx, t, &sc, env, samples, best);
}

pt_status engine_reserve(pt_context *ctx, size_t slots, uint32_t shadow_slots, uint32_t iterations,
                         bool both_arenas) {
  if (ctx->schedule == PT_SCHEDULE_WAVEFRONT) {
    pt_status st = ensure_wavefront(ctx, (uint32_t)slots, shadow_slots, iterations, 0);
    const int n = both_arenas ? (int)ctx->overlap_arenas : 1;
    for (int k = 1; k < n && st == PT_OK; ++k) st = ensure_wavefront(ctx, (uint32_t)slots, shadow_slots, iterations, k);
    return st;
  }
  return ensure(ctx, ctx->d_out, ctx->out_cap, slots);
}

pt_status engine_overlap_begin(pt_context *ctx) {
  if (!ctx->ev_ready) {
    for (int k = 0; k < pt_context::kMaxArenas; ++k) {
      CK(ctx, cudaStreamCreateWithFlags(&ctx->wave_streams[k], cudaStreamNonBlocking));
      CK(ctx, cudaEventCreateWithFlags(&ctx->ev_traced[k], cudaEventDisableTiming));
      CK(ctx, cudaEventCreateWithFlags(&ctx->ev_accumulated[k], cudaEventDisableTiming));
    }
    CK(ctx, cudaEventCreateWithFlags(&ctx->ev_ready, cudaEventDisableTiming));
  }
  CK(ctx, cudaEventRecord(ctx->ev_ready, ctx->stream));
  for (int k = 0; k < pt_context::kMaxArenas; ++k) CK(ctx, cudaStreamWaitEvent(ctx->wave_streams[k], ctx->ev_ready, 0));
  return PT_OK;
}

pt_status launch_wave(pt_context *ctx, const DevRequest *d_reqs, const WaveSegment *d_segs,
                      const std::vector<WaveSegment> &segs, uint32_t iters, StageTimer *timer, int arena,
                      bool area, uint32_t all_wide) {
  uint32_t nseg = (uint32_t)segs.size(), total = 0, max_pix = 0;
  for (const WaveSegment &s : segs) {
    total += s.pixel_count * s.spp;
    max_pix = std::max(max_pix, s.pixel_count);
  }
  if (ctx->schedule == PT_SCHEDULE_WAVEFRONT) {
    if (total == 0) return PT_OK;
    const bool own_stream = arena >= 0;
    WaveBuffers w = arena > 0 ? ctx->wf_more[arena - 1] : ctx->wf;
    w.iterations = iters;
    w.sort_materials = ctx->material_sort ? 1u : 0u;
    w.shade_blocks = ctx->shade_blocks == 4 ? 4u : 3u;
    w.trav_threads = ctx->trav_threads == 128 ? 128u : 256u;
    w.claim_chunk = ctx->claim_chunk == 2 || ctx->claim_chunk == 4 ? ctx->claim_chunk : 1u;
    w.all_wide = all_wide & (uint32_t)(WIDE_EXTENSION | WIDE_SHADOW);
    cudaStream_t ws = own_stream ? ctx->wave_streams[arena] : ctx->stream;
    // The arena's previous wave must be accumulated before this one
    // overwrites its descriptor, queues and per-slot radiance.
    if (own_stream) CK(ctx, cudaStreamWaitEvent(ws, ctx->ev_accumulated[arena], 0));
    // Pageable source: the copy is staged before the call returns and lands
    // in stream order, after the previous wave has read its descriptor.
    WaveDesc wd{d_reqs, d_segs, nseg, total, max_pix, area ? (uint32_t)WAVE_AREA_LIGHTS : 0u};
    CK(ctx, cudaMemcpyAsync(w.desc, &wd, sizeof wd, cudaMemcpyHostToDevice, ws));
    const bool timed = timer && timer->events;
    if (ctx->use_graphs && !timed) {
      // One captured graph per (bounce count, traversal variant, arena /
      // whole wave, shade variant, material sort) replays the wave: one
      // launch instead of ~6 per bounce.
      const uint32_t key = iters << 12 | w.all_wide << 10 | w.claim_chunk << 7 | (w.trav_threads == 128 ? 64u : 0u) |
                           (own_stream ? 4u * (1u + (uint32_t)arena) : 0u) | (w.shade_blocks == 4 ? 2u : 0u) |
                           w.sort_materials;
      auto it = ctx->graphs.find(key);
      if (it == ctx->graphs.end()) {
        cudaGraphExec_t ge = nullptr;
        CK(ctx, capture_wavefront(w, ctx->d_ctr, ctx->num_sms, &ge, !own_stream));
        it = ctx->graphs.emplace(key, ge).first;
      }
      CK(ctx, cudaGraphLaunch(it->second, ws));
    } else {
      CK(ctx, launch_wavefront(w, ctx->d_ctr, ctx->num_sms, ws, timer, !own_stream));
    }
    if (own_stream) {
      // Accumulate in wave order on ctx->stream once the trace is done.
      CK(ctx, cudaEventRecord(ctx->ev_traced[arena], ws));
      CK(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_traced[arena], 0));
      CK(ctx, launch_wave_accumulate(w, ctx->num_sms, ctx->stream));
      CK(ctx, cudaEventRecord(ctx->ev_accumulated[arena], ctx->stream));
    }
  } else {
    if (timer) timer->mark(STAGE_MEGAKERNEL, ctx->stream);
    CK(ctx, launch_megakernel(d_reqs, d_segs, nseg, total, ctx->d_out, ctx->d_ctr, ctx->stream));
    if (timer) timer->mark(STAGE_ACCUMULATE, ctx->stream);
    CK(ctx, launch_accumulate(d_reqs, d_segs, nseg, max_pix, ctx->d_out, ctx->stream));
  }
  return PT_OK;
}

pt_status engine_create(int device, pt_context **out) {
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0)
    return fail(nullptr, PT_ERR_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
  if (device < 0 || device >= count) return fail(nullptr, PT_ERR_INVALID_ARG, "device index out of range");
  auto ctx = std::make_unique<pt_context>();
  ctx->device = device;
  e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  float sheen[512], thr[255];
  host_sheen_lut(sheen);
  host_srgb_thresholds(thr);
  if (e == cudaSuccess) e = set_tables(sheen, thr);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_ctr, sizeof(DevCounters));
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev1);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) {
    pt_destroy(ctx.release());
    return fail(nullptr, PT_ERR_DEVICE, std::string("context setup failed: ") + cudaGetErrorString(e));
  }
  *out = ctx.release();
  return PT_OK;
}
}  // namespace ptd

extern "C" {

uint32_t pt_abi_version(void) { return PT_ABI_VERSION; }

pt_status pt_create(pt_context **out, int device) {
  if (!out) return fail(nullptr, PT_ERR_INVALID_ARG, "out is NULL");
  *out = nullptr;
  return guard(nullptr, [&]() -> pt_status { return engine_create(device, out); });
}

void pt_destroy(pt_context *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (cudaStream_t s : ctx->wave_streams)
    if (s) cudaStreamSynchronize(s);
  for (auto &kv : ctx->scenes) release_scene(*kv.second);
  ctx->scenes.clear();
  if (ctx->d_out) cudaFree(ctx->d_out);
  for (auto &kv : ctx->graphs) cudaGraphExecDestroy(kv.second);
  ctx->graphs.clear();
  if (ctx->wf_arena) cudaFree(ctx->wf_arena);
  for (void *a : ctx->wf_arena_more)
    if (a) cudaFree(a);
  for (int k = 0; k < pt_context::kMaxArenas; ++k) {
    if (ctx->wave_streams[k]) cudaStreamDestroy(ctx->wave_streams[k]);
    if (ctx->ev_traced[k]) cudaEventDestroy(ctx->ev_traced[k]);
    if (ctx->ev_accumulated[k]) cudaEventDestroy(ctx->ev_accumulated[k]);
  }
  if (ctx->ev_ready) cudaEventDestroy(ctx->ev_ready);
  if (ctx->d_segs) cudaFree(ctx->d_segs);
  if (ctx->d_reqs) cudaFree(ctx->d_reqs);
  if (ctx->d_ctr) cudaFree(ctx->d_ctr);
  for (cudaEvent_t ev : ctx->stage_events) cudaEventDestroy(ev);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  ctx->staging.release();
  delete ctx;
}

const char *pt_last_error(const pt_context *ctx) { return ctx ? ctx->err.c_str() : g_create_error.c_str(); }

pt_status pt_scene_upload(pt_context *ctx, const pt_scene_desc *desc, uint32_t *scene_id) {
  if (!ctx) return fail(nullptr, PT_ERR_INVALID_ARG, "context is NULL");
  if (!desc || !scene_id) return fail(ctx, PT_ERR_INVALID_ARG, "desc / scene_id is NULL");
  return guard(ctx, [&]() -> pt_status {
    CK(ctx, cudaSetDevice(ctx->device));
    auto sc = std::make_unique<SceneHost>();
    if (injected_oom(ctx)) return fail(ctx, PT_ERR_OOM, "scene upload: device allocation failed (injected)");
    bool oom = false;
    std::string err = upload_scene(*desc, *sc, oom, ctx->bvh_builder, ctx->stream, &ctx->staging);
    if (!err.empty()) return fail(ctx, oom ? PT_ERR_OOM : PT_ERR_INVALID_ARG, err);
    uint32_t id = ctx->next_id++;
    ctx->scenes[id] = std::move(sc);
    *scene_id = id;
    return PT_OK;
  });
}

pt_status pt_scene_release(pt_context *ctx, uint32_t scene_id) {
  if (!ctx) return fail(nullptr, PT_ERR_INVALID_ARG, "context is NULL");
  return guard(ctx, [&]() -> pt_status {
    auto it = ctx->scenes.find(scene_id);
    if (it == ctx->scenes.end()) return fail(ctx, PT_ERR_NOT_FOUND, "unknown scene");
    CK(ctx, cudaSetDevice(ctx->device));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    release_scene(*it->second);
    ctx->scenes.erase(it);
    return PT_OK;
  });
}

pt_status pt_scene_refit(pt_context *ctx, uint32_t scene_id, const pt_scene_desc *desc) {
  if (!ctx) return fail(nullptr, PT_ERR_INVALID_ARG, "context is NULL");
  if (!desc) return fail(ctx, PT_ERR_INVALID_ARG, "desc is NULL");
  return guard(ctx, [&]() -> pt_status {
    SceneHost *sc = find_scene(ctx, scene_id);
    if (!sc) return fail(ctx, PT_ERR_NOT_FOUND, "unknown scene " + std::to_string(scene_id));
    CK(ctx, cudaSetDevice(ctx->device));
    // Waves already queued read the old arena: let them finish first.
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    if (injected_oom(ctx)) return fail(ctx, PT_ERR_OOM, "scene refit: device allocation failed (injected)");
    bool oom = false;
    std::string err = refit_scene(*desc, *sc, oom, ctx->stream, &ctx->staging);
    if (!err.empty()) return fail(ctx, oom ? PT_ERR_OOM : PT_ERR_INVALID_ARG, err);
    return PT_OK;
  });
}

pt_status pt_scene_device_bytes(pt_context *ctx, uint32_t scene_id, uint64_t *bytes) {
  if (!ctx || !bytes) return fail(ctx, PT_ERR_INVALID_ARG, "NULL argument");
  SceneHost *s = find_scene(ctx, scene_id);
  if (!s) return fail(ctx, PT_ERR_NOT_FOUND, "unknown scene");
  *bytes = s->device_bytes();
  return PT_OK;
}

pt_status pt_scene_triangle_count(pt_context *ctx, uint32_t scene_id, uint64_t *count) {
  if (!ctx || !count) return fail(ctx, PT_ERR_INVALID_ARG, "NULL argument");
  SceneHost *s = find_scene(ctx, scene_id);
  if (!s) return fail(ctx, PT_ERR_NOT_FOUND, "unknown scene");
  *count = s->tri_count;
  return PT_OK;
}

pt_status pt_scene_bvh_stats(pt_context *ctx, uint32_t scene_id, uint32_t *nodes, uint32_t *leaves,
                             uint32_t *max_depth, double *sah_cost, double *build_seconds) {
  if (!ctx) return fail(nullptr, PT_ERR_INVALID_ARG, "context is NULL");
  SceneHost *s = find_scene(ctx, scene_id);
  if (!s) return fail(ctx, PT_ERR_NOT_FOUND, "unknown scene");
  if (nodes) *nodes = s->bvh.nodes;
  if (leaves) *leaves = s->bvh.leaves;
  if (max_depth) *max_depth = s->bvh.max_depth;
  if (sah_cost) *sah_cost = s->bvh.sah_cost;
  if (build_seconds) *build_seconds = s->bvh.seconds;
  return PT_OK;
}

pt_status pt_set_bvh_builder(pt_context *ctx, uint32_t builder) {
  if (!ctx) return fail(nullptr, PT_ERR_INVALID_ARG, "context is NULL");
  if (builder > PT_BVH_BUILD_HOST_SPATIAL) return fail(ctx, PT_ERR_INVALID_ARG, "unknown BVH builder");
  ctx->bvh_builder = (int)builder;
  return PT_OK;
}

pt_status pt_scene_upload_seconds(pt_context *ctx, uint32_t scene_id, double seconds[4]) {
  if (!ctx || !seconds) return fail(ctx, PT_ERR_INVALID_ARG, "NULL argument");
  SceneHost *s = find_scene(ctx, scene_id);
  if (!s) return fail(ctx, PT_ERR_NOT_FOUND, "unknown scene");
  for (int k = 0; k < 4; ++k) seconds[k] = s->upload_seconds[k];
  return PT_OK;
}

pt_status pt_debug_scene_texels(pt_context *ctx, uint32_t scene_id, float *out, uint64_t capacity, uint64_t *total) {
  if (!ctx || !total) return fail(ctx, PT_ERR_INVALID_ARG, "NULL argument");
  return guard(ctx, [&]() -> pt_status {
    SceneHost *s = find_scene(ctx, scene_id);
    if (!s) return fail(ctx, PT_ERR_NOT_FOUND, "unknown scene");
    *total = s->pool_texels;
    const uint64_t n = std::min(capacity, s->pool_texels);
    if (n && out) {
      CK(ctx, cudaSetDevice(ctx->device));
      CK(ctx, cudaStreamSynchronize(ctx->stream));
      CK(ctx, cudaMemcpy(out, s->dev.texels, n * sizeof(float4), cudaMemcpyDeviceToHost));
    }
    return PT_OK;
  });
}

pt_status pt_scene_bvh_on_device(pt_context *ctx, uint32_t scene_id, int *on_device) {
  if (!ctx || !on_device) return fail(ctx, PT_ERR_INVALID_ARG, "NULL argument");
  SceneHost *s = find_scene(ctx, scene_id);
  if (!s) return fail(ctx, PT_ERR_NOT_FOUND, "unknown scene");
  *on_device = s->device_bvh ? 1 : 0;
  return PT_OK;
}

pt_status pt_tracer_create(pt_context *ctx, pt_tracer **out) {
  if (!ctx || !out) return fail(ctx, PT_ERR_INVALID_ARG, "NULL argument");
  return guard(ctx, [&]() -> pt_status {
    auto t = std::make_unique<pt_tracer>();
    t->ctx = ctx;
    CK(ctx, cudaSetDevice(ctx->device));
    CK(ctx, dev_malloc(ctx, &t->d_req, sizeof(DevRequest)));
    *out = t.release();
    return PT_OK;
  });
}

void pt_tracer_destroy(pt_tracer *t) {
  if (!t) return;
  cudaSetDevice(t->ctx->device);
  cudaStreamSynchronize(t->ctx->stream);
  if (t->env) release_env(*t->env);
  if (t->d_accum) cudaFree(t->d_accum);
  if (t->d_req) cudaFree(t->d_req);
  if (t->d_resolve) cudaFree(t->d_resolve);
  delete t;
}

pt_status pt_tracer_sync(pt_tracer *t, uint32_t scene_id, const pt_camera *camera, const pt_render_options *opts,
                         int *reset) {
  if (!t) return fail(nullptr, PT_ERR_INVALID_ARG, "tracer is NULL");
  return guard(t->ctx, [&] { return sync_impl(t, scene_id, camera, opts, reset); });
}

pt_status pt_tracer_refine(pt_tracer *t, uint32_t samples) {
  if (!t) return fail(nullptr, PT_ERR_INVALID_ARG, "tracer is NULL");
  return guard(t->ctx, [&] { return refine_impl(t, samples); });
}

pt_status pt_tracer_refine_many(pt_context *ctx, pt_tracer *const *tracers, const uint32_t *samples,
                                uint32_t count) {
  if (!ctx) return fail(nullptr, PT_ERR_INVALID_ARG, "context is NULL");
  if (count && (!tracers || !samples)) return fail(ctx, PT_ERR_INVALID_ARG, "tracers / samples is NULL");
  return guard(ctx, [&] { return refine_many_impl(ctx, tracers, samples, count); });
}

pt_status pt_batch_stats(const pt_context *ctx, float *ms, uint32_t *waves, uint64_t *rays) {
  if (!ctx) return fail(nullptr, PT_ERR_INVALID_ARG, "context is NULL");
  if (ms) *ms = ctx->last_batch_ms;
  if (waves) *waves = ctx->last_batch_waves;
  if (rays) *rays = ctx->last_batch_rays;
  return PT_OK;
}

pt_status pt_batch_counters(const pt_context *ctx, uint64_t out[9]) {
  if (!ctx || !out) return fail(nullptr, PT_ERR_INVALID_ARG, "NULL argument");
  std::memcpy(out, ctx->last_batch_counts, sizeof ctx->last_batch_counts);
  return PT_OK;
}

pt_status pt_batch_stage_ms(const pt_context *ctx, float *out, uint32_t n) {
  if (!ctx || !out) return fail(nullptr, PT_ERR_INVALID_ARG, "NULL argument");
  for (uint32_t k = 0; k < n && k < (uint32_t)STAGE_COUNT; ++k) out[k] = ctx->last_batch_stage_ms[k];
  return PT_OK;
}

pt_status pt_tracer_samples(const pt_tracer *t, uint32_t *samples) {
  if (!t || !samples) return fail(t ? t->ctx : nullptr, PT_ERR_INVALID_ARG, "NULL argument");
  *samples = t->samples;
  return PT_OK;
}

pt_status pt_tracer_is_converged(const pt_tracer *t, int *converged) {
  if (!t || !converged) return fail(t ? t->ctx : nullptr, PT_ERR_INVALID_ARG, "NULL argument");
  *converged = t->samples >= t->opts.path_trace.samples_per_pixel ? 1 : 0;
  return PT_OK;
}

pt_status pt_tracer_reset(pt_tracer *t) {
  if (!t) return fail(nullptr, PT_ERR_INVALID_ARG, "tracer is NULL");
  return guard(t->ctx, [&]() -> pt_status {
    pt_context *ctx = t->ctx;
    t->samples = 0;
    if (t->have_state && t->d_accum) {
      CK(ctx, cudaSetDevice(ctx->device));
      CK(ctx, cudaMemsetAsync(t->d_accum, 0, (size_t)t->w * t->h * 4 * sizeof(double), ctx->stream));
      CK(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return PT_OK;
  });
}

pt_status pt_tracer_invalidate_scene(pt_tracer *t) {
  if (!t) return fail(nullptr, PT_ERR_INVALID_ARG, "tracer is NULL");
  t->dirty = true;
  return PT_OK;
}

pt_status pt_tracer_set_environment(pt_tracer *t, const pt_environment *env) {
  if (!t) return fail(nullptr, PT_ERR_INVALID_ARG, "tracer is NULL");
  return guard(t->ctx, [&] { return set_env_impl(t, env); });
}

pt_status pt_tracer_read_hdr(pt_tracer *t, float *out, size_t n) {
  if (!t) return fail(nullptr, PT_ERR_INVALID_ARG, "tracer is NULL");
  return guard(t->ctx, [&] { return read_impl(t, out, n, false); });
}

pt_status pt_tracer_read_image(pt_tracer *t, uint8_t *out, size_t n) {
  if (!t) return fail(nullptr, PT_ERR_INVALID_ARG, "tracer is NULL");
  return guard(t->ctx, [&] { return read_impl(t, out, n, true); });
}

pt_status pt_tracer_read_accum(pt_tracer *t, double *out, size_t n) {
  if (!t || !out) return fail(t ? t->ctx : nullptr, PT_ERR_INVALID_ARG, "NULL argument");
  return guard(t->ctx, [&]() -> pt_status {
    pt_context *ctx = t->ctx;
    size_t need = (size_t)t->w * t->h * 4;
    if (n < need) return fail(ctx, PT_ERR_INVALID_ARG, "output buffer too small");
    if (!t->have_state) {
      std::memset(out, 0, need * sizeof(double));
      return PT_OK;
    }
    CK(ctx, cudaSetDevice(ctx->device));
    CK(ctx, cudaMemcpyAsync(out, t->d_accum, need * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return PT_OK;
  });
}

pt_status pt_tracer_ray_counts(const pt_tracer *t, uint64_t *ext, uint64_t *shadow) {
  if (!t) return fail(nullptr, PT_ERR_INVALID_ARG, "tracer is NULL");
  if (ext) *ext = t->ext;
  if (shadow) *shadow = t->sh;
  return PT_OK;
}

pt_status pt_tracer_traversal_counts(const pt_tracer *t, uint64_t *nodes, uint64_t *tris) {
  if (!t) return fail(nullptr, PT_ERR_INVALID_ARG, "tracer is NULL");
  if (nodes) *nodes = t->ext_nodes + t->sh_nodes;
  if (tris) *tris = t->ext_tris + t->sh_tris;
  return PT_OK;
}

pt_status pt_tracer_traversal_split(const pt_tracer *t, uint64_t out[4]) {
  if (!t || !out) return fail(t ? t->ctx : nullptr, PT_ERR_INVALID_ARG, "NULL argument");
  out[0] = t->ext_nodes;
  out[1] = t->ext_tris;
  out[2] = t->sh_nodes;
  out[3] = t->sh_tris;
  return PT_OK;
}

pt_status pt_set_stage_timing(pt_context *ctx, int on) {
  if (!ctx) return fail(nullptr, PT_ERR_INVALID_ARG, "context is NULL");
  ctx->stage_timing = on != 0;
  return PT_OK;
}

pt_status pt_tracer_stage_ms(const pt_tracer *t, float *out, uint32_t n) {
  if (!t || !out) return fail(t ? t->ctx : nullptr, PT_ERR_INVALID_ARG, "NULL argument");
  for (uint32_t k = 0; k < n && k < (uint32_t)STAGE_COUNT; ++k) out[k] = t->stage_ms[k];
  return PT_OK;
}

pt_status pt_tracer_last_kernel_ms(const pt_tracer *t, float *ms) {
  if (!t || !ms) return fail(t ? t->ctx : nullptr, PT_ERR_INVALID_ARG, "NULL argument");
  *ms = t->last_ms;
  return PT_OK;
}

static pt_status render_impl(pt_context *ctx, uint32_t scene_id, const pt_camera *camera,
                             const pt_render_options *opts, const pt_environment *env, void *out, size_t n,
                             bool image) {
  if (!ctx) return fail(nullptr, PT_ERR_INVALID_ARG, "context is NULL");
  pt_tracer *t = nullptr;
  pt_status st = pt_tracer_create(ctx, &t);
  if (st != PT_OK) return st;
  std::unique_ptr<pt_tracer, void (*)(pt_tracer *)> hold(t, pt_tracer_destroy);
  if (env && (st = pt_tracer_set_environment(t, env)) != PT_OK) return st;
  t->dirty = true;
  if ((st = pt_tracer_sync(t, scene_id, camera, opts, nullptr)) != PT_OK) return st;
  if ((st = pt_tracer_refine(t, std::max(opts->path_trace.samples_per_pixel, 1u))) != PT_OK) return st;
  return image ? pt_tracer_read_image(t, (uint8_t *)out, n) : pt_tracer_read_hdr(t, (float *)out, n);
}

pt_status pt_render_hdr(pt_context *ctx, uint32_t scene_id, const pt_camera *camera, const pt_render_options *opts,
                        const pt_environment *env, float *out, size_t n) {
  return guard(ctx, [&] { return render_impl(ctx, scene_id, camera, opts, env, out, n, false); });
}

pt_status pt_render_image(pt_context *ctx, uint32_t scene_id, const pt_camera *camera, const pt_render_options *opts,
                          const pt_environment *env, uint8_t *out, size_t n) {
  return guard(ctx, [&] { return render_impl(ctx, scene_id, camera, opts, env, out, n, true); });
}

// ---------------------------------------------------------------- raycast
namespace {
// build_light, src/shade.rs:26-35: azimuth / elevation in degrees to a unit
// direction toward the light (f32 throughout, as the reference).
void legacy_light(const pt_raycast_options &o, float dir[3]) {
  const float deg = 3.14159265358979323846f / 180.0f;
  float az = o.light_azimuth_deg * deg, el = o.light_elevation_deg * deg;
  float cos_el = std::cos(el);
  float d[3] = {cos_el * std::sin(az), std::sin(el), cos_el * std::cos(az)};
  float len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  for (int k = 0; k < 3; ++k) dir[k] = len < 1.1920929e-7f ? 0.0f : d[k] / len;
}
}  // namespace

pt_status pt_raycast_render(pt_context *ctx, uint32_t scene_id, const pt_camera *camera,
                            const pt_raycast_options *opts, float *out_hdr, size_t hdr_floats, uint8_t *out_rgba,
                            size_t rgba_bytes) {
  if (!ctx) return fail(nullptr, PT_ERR_INVALID_ARG, "context is NULL");
  if (!camera || !opts) return fail(ctx, PT_ERR_INVALID_ARG, "camera / options is NULL");
  const pt_raycast_options &o = *opts;
  if (o.width == 0 || o.height == 0) return fail(ctx, PT_ERR_INVALID_ARG, "width and height must be positive");
  if (o.aa < 1 || o.aa > 8) return fail(ctx, PT_ERR_INVALID_ARG, "aa must be in 1..=8");
  if (o.shading > PT_SHADE_PBR) return fail(ctx, PT_ERR_INVALID_ARG, "unknown shading mode");
  if (o.tone_map > PT_TONE_ACES) return fail(ctx, PT_ERR_INVALID_ARG, "unknown tone map");
  const uint64_t rw = (uint64_t)o.width * o.aa, rh = (uint64_t)o.height * o.aa;
  if (rw * rh > (1ull << 30)) return fail(ctx, PT_ERR_INVALID_ARG, "render resolution too large");
  const uint64_t npx = (uint64_t)o.width * o.height;
  if (out_hdr && hdr_floats < 4 * npx) return fail(ctx, PT_ERR_INVALID_ARG, "HDR buffer too small");
  if (out_rgba && rgba_bytes < 4 * npx) return fail(ctx, PT_ERR_INVALID_ARG, "RGBA buffer too small");
  return guard(ctx, [&]() -> pt_status {
    SceneHost *sc = find_scene(ctx, scene_id);
    if (!sc) return fail(ctx, PT_ERR_NOT_FOUND, "unknown scene " + std::to_string(scene_id));
    CK(ctx, cudaSetDevice(ctx->device));
    static float decode[256];
    static bool init = [] {
      for (int i = 0; i < 256; ++i) decode[i] = host_srgb_to_linear((float)i / 255.0f);
      return true;
    }();
    (void)init;
    float light[3];
    legacy_light(o, light);
    const bool display = o.shading == PT_SHADE_NORMAL_DEBUG || o.shading == PT_SHADE_DEPTH_DEBUG;
    float4 bg = make_float4(decode[o.background[0]], decode[o.background[1]], decode[o.background[2]],
                            (float)o.background[3] / 255.0f);
    const uint64_t ns = rw * rh;
    const bool pbr = o.shading == PT_SHADE_PBR;
    // Samples the Pbr kernel re-traces with deep frame stacks: this many at
    // a time.
    const uint32_t deep_slots = 2048;
    // One stream-ordered allocation: samples, coverage, error word and
    // overflow count, outputs; for Pbr the overflow list and deep stacks.
    auto al = [](uint64_t x) { return (x + 255) & ~uint64_t(255); };
    const uint64_t off_cov = al(ns * sizeof(float4)), off_err = off_cov + al(ns);
    const uint64_t off_hdr = off_err + 256, off_rgba = off_hdr + al(npx * sizeof(float4));
    const uint64_t off_ovf = off_rgba + al(npx * 4);
    const uint64_t off_deep = off_ovf + (pbr ? al(ns * sizeof(uint32_t)) : 0);
    const uint64_t total = off_deep + (pbr ? al((uint64_t)deep_slots * raycast_pbr_frame_bytes()) : 0);
    void *buf = nullptr;
    CK(ctx, cudaMallocAsync(&buf, total, ctx->stream));
    std::unique_ptr<void, std::function<void(void *)>> hold(buf, [ctx](void *q) { cudaFreeAsync(q, ctx->stream); });
    uint8_t *b = static_cast<uint8_t *>(buf);
    uint32_t *d_err = reinterpret_cast<uint32_t *>(b + off_err);
    CK(ctx, cudaMemsetAsync(d_err, 0, 2 * sizeof(uint32_t), ctx->stream));
    if (pbr) {
      const float ambient = std::isfinite(o.ambient) ? std::max(o.ambient, 0.0f) : 0.0f;
      const float cutoff = std::isfinite(o.reflection_roughness_cutoff)
                               ? std::min(std::max(o.reflection_roughness_cutoff, 0.0f), 1.0f)
                               : 0.0f;
      // trace::pixel_spread, src/trace.rs:1139-1146.
      const float spread = camera->projection == PT_PERSPECTIVE ? std::atan(2.0f * camera->half_h / (float)rh) : 0.0f;
      CK(ctx, launch_raycast_pbr(sc->dev, *camera, (uint32_t)rw, (uint32_t)rh, o.max_ray_depth, o.shadows != 0,
                                 ambient, cutoff, spread, bg, reinterpret_cast<float4 *>(b), b + off_cov, d_err,
                                 reinterpret_cast<uint32_t *>(b + off_ovf), d_err + 1, b + off_deep, deep_slots,
                                 ctx->num_sms, ctx->stream));
    } else {
      CK(ctx, launch_raycast(sc->dev, *camera, (uint32_t)rw, (uint32_t)rh, o.shading, o.max_ray_depth, light,
                             o.light_intensity, o.near_plane, o.far_plane, decode, reinterpret_cast<float4 *>(b),
                             b + off_cov, d_err, ctx->num_sms, ctx->stream));
    }
    float4 *d_hdr = out_hdr ? reinterpret_cast<float4 *>(b + off_hdr) : nullptr;
    uchar4 *d_rgba = out_rgba ? reinterpret_cast<uchar4 *>(b + off_rgba) : nullptr;
    CK(ctx, launch_raycast_resolve(reinterpret_cast<float4 *>(b), b + off_cov, o.width, o.height, o.aa, bg,
                                   display ? (uint32_t)PT_TONE_CLAMP : o.tone_map, display ? 1.0f : o.exposure, d_hdr,
                                   d_rgba, ctx->stream));
    uint32_t err = 0;
    CK(ctx, cudaMemcpyAsync(&err, d_err, sizeof err, cudaMemcpyDeviceToHost, ctx->stream));
    if (d_hdr)
      CK(ctx, cudaMemcpyAsync(out_hdr, d_hdr, npx * sizeof(float4), cudaMemcpyDeviceToHost, ctx->stream));
    if (d_rgba) CK(ctx, cudaMemcpyAsync(out_rgba, d_rgba, npx * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    if (err & ERR_STACK_OVERFLOW) return fail(ctx, PT_ERR_DEVICE, "BVH traversal stack overflow");
    return PT_OK;
  });
}

// ---------------------------------------------------------------- debug hooks
pt_status pt_set_schedule(pt_context *ctx, uint32_t schedule) {
  if (!ctx) return fail(nullptr, PT_ERR_INVALID_ARG, "context is NULL");
  if (schedule != PT_SCHEDULE_MEGAKERNEL && schedule != PT_SCHEDULE_WAVEFRONT)
    return fail(ctx, PT_ERR_INVALID_ARG, "unknown schedule");
  ctx->schedule = schedule;
  return PT_OK;
}

pt_status pt_set_wave_slots(pt_context *ctx, uint32_t slots) {
  if (!ctx || slots == 0) return fail(ctx, PT_ERR_INVALID_ARG, "bad argument");
  ctx->wave_slots = slots;
  return PT_OK;
}

namespace {
pt_tune_choice to_c(const TuneChoice &c) {
  pt_tune_choice o;
  o.schedule = c.schedule;
  o.node_width_extension = (c.wide_nodes & WIDE_EXTENSION) ? 4u : 2u;
  o.node_width_shadow = (c.wide_nodes & WIDE_SHADOW) ? 4u : 2u;
  o.material_sort = c.material_sort;
  o.shade_blocks_per_sm = c.shade_blocks;
  o.wave_arenas = c.arenas;
  o.wave_slots = c.wave_slots;
  o.samples_per_s = c.samples_per_s;
  o.traversal_threads = c.trav_threads;
  o.claim_chunk = c.claim_chunk;
  return o;
}
}  // namespace

pt_status pt_debug_prepare_scene(const pt_scene_desc *desc, double seconds[4], uint64_t *device_bytes) {
  if (!desc || !seconds) return fail(nullptr, PT_ERR_INVALID_ARG, "desc / seconds is NULL");
  return guard(nullptr, [&]() -> pt_status {
    SceneImage img;
    std::string err = build_scene_image(*desc, img);
    if (!err.empty()) return fail(nullptr, PT_ERR_INVALID_ARG, err);
    for (int k = 0; k < 4; ++k) seconds[k] = img.seconds[k];
    if (device_bytes) *device_bytes = img.device_bytes();
    return PT_OK;
  });
}

pt_status pt_debug_build_bvh(const float *positions, uint32_t triangles, uint32_t spatial, double stats[6],
                             void *nodes, uint64_t node_capacity, void *records, uint64_t record_capacity) {
  if (!positions || !stats) return fail(nullptr, PT_ERR_INVALID_ARG, "positions / stats is NULL");
  return guard(nullptr, [&]() -> pt_status {
    std::vector<BvhNode> n2;
    std::vector<Bvh4Node> n4;
    std::vector<float4> rec;
    BvhBuildStats st;
    const int threads = (int)std::max(1u, std::thread::hardware_concurrency());
    if (spatial)
      build_bvh_spatial(positions, triangles, nullptr, n2, n4, rec, st, threads);
    else
      build_bvh(positions, triangles, nullptr, n2, n4, rec, st, threads);
    stats[0] = (double)st.nodes;
    stats[1] = (double)st.leaves;
    stats[2] = (double)st.max_depth;
    stats[3] = st.sah_cost;
    stats[4] = st.seconds;
    stats[5] = (double)(rec.size() / 3);
    if (nodes && node_capacity >= n2.size()) std::memcpy(nodes, n2.data(), n2.size() * sizeof(BvhNode));
    if (records && record_capacity >= rec.size() / 3) std::memcpy(records, rec.data(), rec.size() * sizeof(float4));
    return PT_OK;
  });
}

pt_status pt_autotune(pt_context *ctx, pt_tracer *t, uint32_t samples, pt_tune_choice *best) {
  if (!ctx || !t || t->ctx != ctx) return fail(ctx, PT_ERR_INVALID_ARG, "bad context / tracer");
  return guard(ctx, [&]() -> pt_status {
    TuneChoice c{};
    pt_status st = autotune_impl(ctx, t, samples, c);
    if (st == PT_OK && best) *best = to_c(c);
    return st;
  });
}

pt_status pt_tune_lookup(pt_context *ctx, const pt_tracer *t, pt_tune_choice *out) {
  if (!ctx || !t || !out) return fail(ctx, PT_ERR_INVALID_ARG, "NULL argument");
  SceneHost *sc = find_scene(ctx, t->scene_id);
  if (!sc) return fail(ctx, PT_ERR_NOT_FOUND, "tracer has no resident scene");
  auto it = ctx->tuned.find(scene_class(*sc, t->env != nullptr));
  if (it == ctx->tuned.end()) return fail(ctx, PT_ERR_NOT_FOUND, "scene class not tuned");
  *out = to_c(it->second);
  return PT_OK;
}

pt_status pt_tune_reset(pt_context *ctx) {
  if (!ctx) return fail(ctx, PT_ERR_INVALID_ARG, "context is NULL");
  ctx->tuned.clear();
  return PT_OK;
}

pt_status pt_debug_fail_allocations(pt_context *ctx, uint32_t count) {
  if (!ctx) return fail(nullptr, PT_ERR_INVALID_ARG, "context is NULL");
  ctx->fail_allocs.store(count);
  return PT_OK;
}

pt_status pt_set_wave_graphs(pt_context *ctx, int on) {
  if (!ctx) return fail(ctx, PT_ERR_INVALID_ARG, "context is NULL");
  ctx->use_graphs = on != 0;
  return PT_OK;
}

pt_status pt_set_wave_overlap(pt_context *ctx, int on) {
  if (!ctx) return fail(ctx, PT_ERR_INVALID_ARG, "context is NULL");
  if (on < 0 || on > pt_context::kMaxArenas) return fail(ctx, PT_ERR_INVALID_ARG, "overlap must be 0..3");
  ctx->overlap_arenas = on == 0 ? 0u : (on == 1 ? 3u : (uint32_t)on);
  ctx->overlap_waves = ctx->overlap_arenas >= 2;
  ctx->overlap_fixed = on >= 2;
  return PT_OK;
}

pt_status pt_set_shade_blocks(pt_context *ctx, uint32_t blocks_per_sm) {
  if (!ctx || (blocks_per_sm != 3 && blocks_per_sm != 4))
    return fail(ctx, PT_ERR_INVALID_ARG, "shade blocks per SM must be 3 or 4");
  ctx->shade_blocks = blocks_per_sm;
  return PT_OK;
}

pt_status pt_set_traversal(pt_context *ctx, uint32_t threads, uint32_t claim_chunk) {
  if (!ctx || (threads != 128 && threads != 256) || (claim_chunk != 1 && claim_chunk != 2 && claim_chunk != 4))
    return fail(ctx, PT_ERR_INVALID_ARG, "traversal threads must be 128 or 256 and the claim chunk 1, 2 or 4");
  ctx->trav_threads = threads;
  ctx->claim_chunk = claim_chunk;
  return PT_OK;
}

pt_status pt_set_material_sort(pt_context *ctx, int on) {
  if (!ctx) return fail(ctx, PT_ERR_INVALID_ARG, "context is NULL");
  ctx->material_sort = on != 0;
  return PT_OK;
}

pt_status pt_set_node_width(pt_context *ctx, uint32_t extension_width, uint32_t shadow_width) {
  if (!ctx || (extension_width != 2 && extension_width != 4) || (shadow_width != 2 && shadow_width != 4))
    return fail(ctx, PT_ERR_INVALID_ARG, "node widths must be 2 or 4");
  ctx->wide_nodes = (extension_width == 4 ? WIDE_EXTENSION : 0u) | (shadow_width == 4 ? WIDE_SHADOW : 0u);
  return PT_OK;
}

pt_status pt_debug_sobol(pt_context *ctx, uint32_t n, uint32_t seed, float *out) {
  if (!ctx || !out) return fail(ctx, PT_ERR_INVALID_ARG, "NULL argument");
  return guard(ctx, [&]() -> pt_status {
    if (n == 0) return PT_OK;
    CK(ctx, cudaSetDevice(ctx->device));
    float4 *d = nullptr;
    CK(ctx, cudaMalloc(&d, (size_t)n * sizeof(float4)));
    cudaError_t e = launch_debug_sobol(n, seed, d, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, (size_t)n * sizeof(float4), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d);
    CK(ctx, e);
    return PT_OK;
  });
}

pt_status pt_debug_pattern(pt_tracer *t, uint32_t index, uint32_t pattern, float *out) {
  if (!t || !out) return fail(t ? t->ctx : nullptr, PT_ERR_INVALID_ARG, "NULL argument");
  return guard(t->ctx, [&]() -> pt_status {
    pt_context *ctx = t->ctx;
    if (!t->have_state) return fail(ctx, PT_ERR_INVALID_ARG, "tracer not synced");
    SceneHost *sc = find_scene(ctx, t->scene_id);
    if (!sc) return fail(ctx, PT_ERR_EVICTED, "scene not resident");
    CK(ctx, cudaSetDevice(ctx->device));
    DevRequest rq = make_request(*t, *sc, t->env.get());
    CK(ctx, cudaMemcpyAsync(t->d_req, &rq, sizeof rq, cudaMemcpyHostToDevice, ctx->stream));
    uint32_t npix = t->w * t->h;
    float4 *d = nullptr;
    CK(ctx, cudaMalloc(&d, (size_t)npix * sizeof(float4)));
    cudaError_t e = launch_debug_pattern(t->d_req, npix, index, pattern, d, ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(out, d, (size_t)npix * sizeof(float4), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d);
    CK(ctx, e);
    return PT_OK;
  });
}

pt_status pt_debug_primary_hits(pt_tracer *t, uint32_t index, uint32_t *out_g, float *out_tb) {
  if (!t || !out_g || !out_tb) return fail(t ? t->ctx : nullptr, PT_ERR_INVALID_ARG, "NULL argument");
  return guard(t->ctx, [&]() -> pt_status {
    pt_context *ctx = t->ctx;
    if (!t->have_state) return fail(ctx, PT_ERR_INVALID_ARG, "tracer not synced");
    SceneHost *sc = find_scene(ctx, t->scene_id);
    if (!sc) return fail(ctx, PT_ERR_EVICTED, "scene not resident");
    CK(ctx, cudaSetDevice(ctx->device));
    DevRequest rq = make_request(*t, *sc, t->env.get());
    CK(ctx, cudaMemcpyAsync(t->d_req, &rq, sizeof rq, cudaMemcpyHostToDevice, ctx->stream));
    uint32_t npix = t->w * t->h;
    uint32_t *dg = nullptr;
    float4 *dt = nullptr;
    CK(ctx, cudaMalloc(&dg, (size_t)npix * 4));
    cudaError_t e = cudaMalloc(&dt, (size_t)npix * sizeof(float4));
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_ctr, 0, sizeof(DevCounters), ctx->stream);
    if (e == cudaSuccess) e = launch_debug_primary(t->d_req, npix, index, dg, dt, ctx->d_ctr, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_g, dg, (size_t)npix * 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(out_tb, dt, (size_t)npix * sizeof(float4), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(dg);
    if (dt) cudaFree(dt);
    CK(ctx, e);
    return PT_OK;
  });
}

pt_status pt_debug_bsdf(pt_context *ctx, const float *params, const float *dirs, const float *us, uint32_t n,
                        float *out) {
  if (!ctx || !params || !dirs || !us || !out) return fail(ctx, PT_ERR_INVALID_ARG, "NULL argument");
  return guard(ctx, [&]() -> pt_status {
    if (n == 0) return PT_OK;
    CK(ctx, cudaSetDevice(ctx->device));
    float *d = nullptr;
    size_t fl = 43 + 3 * (size_t)n + 3 * (size_t)n + 12 * (size_t)n;
    CK(ctx, cudaMalloc(&d, fl * 4));
    float *dp = d, *dd = d + 43, *du = dd + 3 * (size_t)n, *dout = du + 3 * (size_t)n;
    cudaError_t e = cudaMemcpyAsync(dp, params, 43 * 4, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dd, dirs, 12 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(du, us, 12 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = launch_debug_bsdf(dp, dd, du, n, dout, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, 48 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d);
    CK(ctx, e);
    return PT_OK;
  });
}

}  // extern "C"
