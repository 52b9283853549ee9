/*
 * pt_b200_serve.h — serving layer of the B200 path tracer: continuous
 * batching of render requests over scenes kept resident in HBM.
 *
 * The reference renders one request per call (Renderer::render ->
 * PathTracer::{sync, refine, hdr}, src/pathtrace.rs:2745-2782 and
 * 2474-2734) and re-prepares the scene every time; it has no serving layer.
 * This one keeps that per-request contract and changes only where the work
 * runs:
 *
 *   - Scenes are registered once. The server keeps each scene's prepared
 *     host image (BVH, triangle records, attributes, materials, texel pool,
 *     light tables) and makes it resident on the device on demand, within an
 *     HBM budget, evicting the least recently used scene that no running
 *     request needs. A re-admitted scene is one host-to-device copy (no
 *     second BVH build).
 *   - Every request owns a progressive accumulator on the device (the
 *     PathTracer's f64 accumulator). A continuation request adds samples to
 *     the accumulator of an earlier request (PathTracer::refine on a live
 *     tracer) and returns the refined image.
 *   - A worker thread admits requests as accumulator slots and scene memory
 *     allow and runs waves of path slots drawn from every admitted request,
 *     so requests that arrive while others are on the GPU share the next
 *     waves. Waves are packed earliest expected finish first: a request's
 *     key is its submit time plus its remaining samples at the measured
 *     throughput, which favours short requests without starving long ones.
 *   - A request can be cancelled (pt_server_cancel) or given a deadline
 *     (pt_server_request.deadline_ms) after which it fails with
 *     PT_ERR_TIMEOUT; pt_server_poll asks without blocking.
 *
 * Determinism: every sample is a pure function of (request seed, pixel,
 * sample index) and each pixel's samples are accumulated in index order, so
 * the HDR image of a request is bit-identical to rendering it alone with
 * pt_tracer_sync / pt_tracer_refine / pt_tracer_read_hdr and the same scene,
 * camera, options and sample count, however the requests were mixed.
 *
 * Threading: all pt_server_* calls are thread-safe; GPU work runs on the
 * server's own stream and buffers, independent of any pt_context's.
 */
#ifndef PT_B200_SERVE_H
#define PT_B200_SERVE_H

#include "pt_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pt_server pt_server;

typedef struct pt_server_config {
  uint64_t hbm_budget_bytes; /* device bytes for resident scenes and their environments; 0 = no limit */
  uint32_t wave_slots;       /* path slots per wave; 0 = 4194304 */
  uint32_t max_active;       /* requests admitted to the GPU at once; 0 = 256 */
  uint32_t megakernel;       /* nonzero: one-kernel-per-path schedule instead of the wavefront */
  uint32_t pipeline_depth;   /* waves in flight; 0 = 3 (one per path-state arena) */
  uint32_t node_width_extension; /* BVH node layout of extension rays: 2 or 4; 0 = 4 */
  uint32_t node_width_shadow;    /* BVH node layout of shadow rays: 2 or 4; 0 = 4 */
  uint32_t autotune;             /* nonzero: tune each new scene class before its first request runs
                                    (pt_autotune on the request's camera and options; the node
                                    layouts of the class's requests follow the result) */
  uint32_t material_sort_off;    /* nonzero: shade without material sort */
  uint32_t wave_overlap_off;     /* nonzero: trace one wave at a time (default: consecutive waves
                                    overlap in two path-state arenas on two streams) */
  uint32_t bvh_binned;           /* nonzero: registered scenes get the binned-SAH tree; default: the
                                    spatial-split tree (PT_BVH_BUILD_HOST_SPATIAL), built once at
                                    registration since the scene stays resident */
} pt_server_config;

typedef struct pt_server_request {
  uint32_t scene;             /* key from pt_server_scene_register (ignored for continuations) */
  uint32_t samples;           /* samples per pixel to add (>= 1) */
  uint64_t continues;         /* 0: a new accumulation; else the ticket whose accumulator gains `samples` */
  pt_camera camera;           /* Camera::resolve output (ignored for continuations) */
  pt_render_options options;  /* as for pt_tracer_sync (ignored for continuations) */
  uint32_t deadline_ms;       /* 0: none; else the request fails with PT_ERR_TIMEOUT when it has not
                                 finished this many ms after its submit (checked between waves) */
} pt_server_request;

typedef struct pt_request_stats {
  double queue_ms;   /* submit -> admitted to the GPU */
  double latency_ms; /* submit -> HDR image in host memory */
  uint32_t width, height;
  uint32_t samples;  /* samples per pixel in the accumulation after this request */
  uint32_t waves;    /* waves that carried this request's paths */
} pt_request_stats;

typedef struct pt_server_stats {
  uint64_t submitted, completed, failed;
  uint64_t samples;         /* camera paths traced */
  uint64_t waves;
  uint64_t rays;            /* extension + shadow rays traced */
  double gpu_ms;            /* device time of all completed waves */
  uint64_t scene_uploads;   /* device commits of scene images (first admissions and re-admissions) */
  uint64_t scene_evictions;
  uint64_t resident_bytes, peak_resident_bytes;
  uint32_t resident_scenes, active, pending, accumulators;
  uint64_t tuned_classes;   /* scene classes tuned by the server (config.autotune) */
  uint64_t cancelled;       /* requests ended by pt_server_cancel (also counted in `failed`) */
  uint64_t timed_out;       /* requests ended by their deadline (also counted in `failed`) */
} pt_server_stats;

/* A server on `ctx`'s device. `cfg` may be NULL (defaults). The server does
 * not use ctx's stream or buffers; ctx must outlive the server. */
PT_API pt_status pt_server_create(pt_context *ctx, const pt_server_config *cfg, pt_server **out);
/* Cancels pending requests (PT_ERR_CANCELLED), lets waves in flight finish,
 * frees everything. */
PT_API void pt_server_destroy(pt_server *server);
/* Message of the last failed pt_server_* call on the calling thread. */
PT_API const char *pt_server_last_error(const pt_server *server);

/* Prepares `desc` on the host (validation, BVH build, tables) and keeps the
 * image; the device copy is made when a request first needs it. `env` may
 * be NULL (constant sky `ambient`); it is the scene's environment map for
 * every request on it (PathTracer::set_environment). */
PT_API pt_status pt_server_scene_register(pt_server *server, const pt_scene_desc *desc, const pt_environment *env,
                                          uint32_t *scene_key);
/* Forgets a scene. PT_ERR_INVALID_ARG while a pending or running request
 * uses it; continuations of finished requests on it then fail. */
PT_API pt_status pt_server_scene_unregister(pt_server *server, uint32_t scene_key);
PT_API pt_status pt_server_scene_info(pt_server *server, uint32_t scene_key, uint64_t *device_bytes,
                                      int *resident);

/* Queues a request and returns its ticket at once. */
PT_API pt_status pt_server_submit(pt_server *server, const pt_server_request *request, uint64_t *ticket);
/* Waits up to `timeout_ms` (< 0: no limit) for `ticket`. PT_OK: the request
 * finished; its HDR image (width * height * 4 floats, row-major RGBA) is
 * copied to `hdr` when non-NULL (`hdr_floats` is its capacity) and `stats`
 * is filled when non-NULL. PT_ERR_TIMEOUT: still running when `timeout_ms`
 * ran out (the request goes on; wait again or cancel it). Any other status
 * is the request's own failure (PT_ERR_CANCELLED, PT_ERR_TIMEOUT from its
 * deadline, PT_ERR_OOM, ...). */
PT_API pt_status pt_server_wait(pt_server *server, uint64_t ticket, int32_t timeout_ms, float *hdr,
                                size_t hdr_floats, pt_request_stats *stats);
/* pt_server_wait without blocking: PT_ERR_NOT_READY while the request is
 * queued or running, else what pt_server_wait returns. */
PT_API pt_status pt_server_poll(pt_server *server, uint64_t ticket, float *hdr, size_t hdr_floats,
                                pt_request_stats *stats);
/* Cancels `ticket`. A queued request leaves the queue; a running one gets no
 * further waves (waves already on the GPU finish, their samples are
 * discarded with the accumulation). Either way it ends with
 * PT_ERR_CANCELLED, and continuations of a cancelled request fail. A request
 * whose last wave is already on the GPU ends cancelled when that wave
 * completes; its accumulation stays usable. PT_ERR_INVALID_ARG when the
 * request has already finished, PT_ERR_NOT_FOUND for an unknown ticket.
 * The ticket must still be released. */
PT_API pt_status pt_server_cancel(pt_server *server, uint64_t ticket);
/* Drops a finished request's image; the accumulator goes once no ticket on
 * it is left. A released ticket cannot be continued. */
PT_API pt_status pt_server_release(pt_server *server, uint64_t ticket);
PT_API pt_status pt_server_stats_get(pt_server *server, pt_server_stats *out);
/* Fault injection on the host (tests): the next `count` device allocations
 * the server makes for requests and scenes (accumulators, scene and
 * environment images) fail as if the device were out of memory, without
 * calling CUDA. The request that needed one fails with PT_ERR_OOM; the
 * server goes on serving. 0 disarms it. */
PT_API pt_status pt_server_debug_fail_allocations(pt_server *server, uint32_t count);

#ifdef __cplusplus
}
#endif

#endif /* PT_B200_SERVE_H */
