// The context object behind the opaque pt_context handle, shared by the C
// entry points (capi.cpp, noalloc.cu).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/pt_b200.h"
#include "../../include/pt_b200_debug.h"
#include "host_scene.h"
#include "kernels.h"

namespace ptd {
// An autotuned configuration of one scene class (pt_autotune).
struct TuneChoice {
  uint32_t schedule, wide_nodes, material_sort, wave_slots;
  float samples_per_s;
  uint32_t shade_blocks = 3;  // k_wf_shade blocks per SM (3 or 4)
  uint32_t arenas = 2;        // overlapped waves in flight (2 or 3)
  uint32_t trav_threads = 256;  // traversal kernels' block size (128 or 256)
  uint32_t claim_chunk = 1;     // queue entries per traversal refill (1, 2, 4)
};
}  // namespace ptd

struct pt_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  std::map<uint32_t, std::unique_ptr<ptd::SceneHost>> scenes;
  uint32_t next_id = 1;
  // The wavefront is the default schedule (C1: 646 M samples/s against
  // about 200 M for the megakernel); pt_set_schedule / tuned choices change it.
  uint32_t schedule = PT_SCHEDULE_WAVEFRONT;
  // Path slots per wave. 8 M measured best with overlapped waves (C1: 646 M
  // samples/s against 613 M at 4 M and 474 M at 1 M, three in flight).
  uint32_t wave_slots = 1u << 23;
  // WIDE_* bits: rays that walk the four-child node layout in the wavefront
  // (default: both kinds).
  uint32_t wide_nodes = ptd::WIDE_EXTENSION | ptd::WIDE_SHADOW;
  bool material_sort = true;  // bucket each shade queue by material
  uint32_t shade_blocks = 3;   // k_wf_shade instantiation: blocks per SM (3 or 4)
  uint32_t trav_threads = 256;  // traversal kernels' block size (128 or 256; 1,024 threads per SM)
  uint32_t claim_chunk = 1;     // queue entries a traversal lane claims per refill (1, 2 or 4)
  int bvh_builder = ptd::BVH_BUILD_AUTO;  // where pt_scene_upload builds the BVH (ptd::BvhBuilder)
  ptd::HostStaging staging;  // pinned host image buffer of pt_scene_upload
  std::map<uint32_t, ptd::TuneChoice> tuned;  // by scene class (ptd::scene_class)
  // Wavefront waves replayed as CUDA graphs (bounce count << 1 | sort -> exec).
  bool use_graphs = true;
  std::map<uint32_t, cudaGraphExec_t> graphs;
  float4 *d_out = nullptr;
  size_t out_cap = 0;
  ptd::WaveSegment *d_segs = nullptr;
  size_t seg_cap = 0;
  ptd::DevRequest *d_reqs = nullptr;  // requests of the running batch
  size_t req_cap = 0;
  float last_batch_ms = 0.0f;
  uint32_t last_batch_waves = 0;
  uint64_t last_batch_rays = 0;
  // Counters of the last batch: extension / shadow rays, their nodes and
  // triangles, samples, waves (pt_batch_counters); per-stage ms.
  uint64_t last_batch_counts[9] = {};
  float last_batch_stage_ms[ptd::STAGE_COUNT] = {};
  ptd::DevCounters *d_ctr = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int num_sms = 148;
  bool stage_timing = false;
  std::vector<cudaEvent_t> stage_events;
  // Wavefront schedule: an arena holding the SoA path state and queues, and a
  // second one so that consecutive waves of a refine overlap (one wave's
  // last bounces, which leave most of the GPU idle, with the next wave's
  // first), each traced on its own stream while the accumulates stay in
  // order on `stream`.
  static constexpr int kMaxArenas = 3;
  ptd::WaveBuffers wf{};  // the first arena (the only one without overlap)
  void *wf_arena = nullptr;
  size_t wf_bytes = 0;
  ptd::WaveBuffers wf_more[kMaxArenas - 1] = {};  // the others
  void *wf_arena_more[kMaxArenas - 1] = {};
  size_t wf_bytes_more[kMaxArenas - 1] = {};
  // Waves in flight at once (0: one wave at a time). Three by default: C1
  // +4 % over two, the soup and C2 within 1 % either way.
  uint32_t overlap_arenas = 3;
  bool overlap_waves = true;    // overlap_arenas >= 2
  bool overlap_fixed = false;   // the count was set explicitly: tuned choices keep it
  cudaStream_t wave_streams[kMaxArenas] = {};
  cudaEvent_t ev_ready = nullptr, ev_traced[kMaxArenas] = {}, ev_accumulated[kMaxArenas] = {};
  // Host-side fault injection (pt_debug_fail_allocations): this many of the
  // next device allocations fail as out of memory without calling CUDA.
  std::atomic<uint32_t> fail_allocs{0};
};

// The object behind pt_tracer: one progressive accumulation (the
// reference's PathTracer state, src/pathtrace.rs:2369-2400).
struct pt_tracer {
  pt_context *ctx = nullptr;
  bool have_state = false, dirty = true;
  uint32_t scene_id = 0;
  pt_camera cam{};
  pt_render_options opts{};
  std::unique_ptr<ptd::EnvHost> env;
  double *d_accum = nullptr;
  size_t accum_cap = 0;
  ptd::DevRequest *d_req = nullptr;
  void *d_resolve = nullptr;
  size_t resolve_cap = 0;
  uint32_t w = 1, h = 1, samples = 0;
  uint64_t ext = 0, sh = 0, ext_nodes = 0, ext_tris = 0, sh_nodes = 0, sh_tris = 0;
  float last_ms = 0.0f;
  float stage_ms[ptd::STAGE_COUNT] = {};
};

namespace ptd {
// Records `msg` as the context's last error and returns `st`.
pt_status ctx_fail(pt_context *ctx, pt_status st, const std::string &msg);
// The resident scene `id`, or nullptr.
SceneHost *ctx_find_scene(pt_context *ctx, uint32_t id);

// ---- the wave engine shared by refine, refine_many and the server ----

// One refine job: `target` samples added to an accumulation whose device
// request is `req` (scene, environment, camera, options, accumulator).
struct Job {
  DevRequest req;
  uint32_t target;
  uint32_t first;         // sample index of the job's first sample
  uint32_t npix;
  uint32_t done = 0;      // whole samples finished
  uint32_t pix_done = 0;  // pixels of sample `done` finished (partial-pixel waves)
  uint32_t iterations = 1;
  uint32_t shadow_slots = 1;
  uint32_t scene_key = 0;  // only orders the packing (locality)
  bool area = false;       // emissive triangles or an environment: the wave runs k_wf_nee
  uint32_t wide = 0;       // WIDE_* bits of the request that its scene's layouts honour
  bool finished() const { return done >= target; }
};

// The device request of tracer `t` drawing on resident scene `sc` and
// environment `env` (nullptr: constant sky).
DevRequest make_request(const pt_tracer &t, const SceneHost &sc, const EnvHost *env);
// A job adding `n` samples to `t` (whose samples so far are `t.samples`).
Job make_job(const pt_tracer &t, const SceneHost &sc, const EnvHost *env, uint32_t n);

// Packs the next wave of at most `cap` path slots from `jobs`, visiting
// them in `order`, and advances the jobs' progress. WaveSegment.request is
// the index into `jobs`. A job contributes at most one segment per wave;
// within a job, samples (and pixel ranges of one sample) go in order.
std::vector<WaveSegment> pack_wave(std::vector<Job> &jobs, const std::vector<uint32_t> &order, uint64_t cap);

// Sizes the context's wave buffers for waves of `slots` paths with up to
// `shadow_slots` shadow rays per path and `iterations` bounce rounds.
pt_status engine_reserve(pt_context *ctx, size_t slots, uint32_t shadow_slots, uint32_t iterations,
                         bool both_arenas = false);
// Enqueues one wave: path kernels + ordered accumulate. `d_reqs` / `d_segs`
// are device copies of the wave's request table and `segs`; `iters` is the
// largest bounce-round count among the wave's jobs. With `arena` -1 the whole
// wave runs on ctx->stream in the first arena; with 0 or 1 the wave is traced
// in that arena on its own stream (after the arena's previous accumulate)
// and accumulated on ctx->stream after the trace (engine_reserve must have
// been asked for both arenas, and engine_overlap_begin called).
// `area`: some job of the wave has emissive triangles or an environment.
pt_status launch_wave(pt_context *ctx, const DevRequest *d_reqs, const WaveSegment *d_segs,
                      const std::vector<WaveSegment> &segs, uint32_t iters, StageTimer *timer, int arena = -1,
                      bool area = true, uint32_t all_wide = 0);
// Makes both wave streams wait for the work enqueued on ctx->stream so far
// (request / segment uploads, counter reset) before overlapped waves.
pt_status engine_overlap_begin(pt_context *ctx);
// A new context's engine state on `device` (stream, tables, counters).
pt_status engine_create(int device, pt_context **out);
// The background colour in linear light (PathTracer::bg_linear,
// src/pathtrace.rs:2593-2602).
float4 bg_linear(const pt_render_options &o);
// PathTracer::sync's option checks (camera / enum / size limits).
pt_status check_options(pt_context *ctx, const pt_camera *cam, const pt_render_options *o);
// Autotuner key of a scene: triangle-count scale (factors of 4), emissive
// triangles, environment map, punctual lights, textures.
uint32_t scene_class(const SceneHost &sc, bool env);
// Times the candidate configurations on a calibration refine of t's camera
// and options over scene `sc` / environment `env` (own scratch accumulator)
// and records the fastest for the scene's class.
pt_status autotune(pt_context *ctx, const pt_tracer *t, SceneHost &sc, const EnvHost *env, uint32_t samples,
                   TuneChoice &best);
}  // namespace ptd
