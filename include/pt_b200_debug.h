/*
 * pt_b200_debug.h — test and measurement hooks of the B200 path tracer.
 *
 * These have no counterpart in the reference's Renderer / PathTracer API;
 * they expose intermediate values of the hot path (sampler values, primary
 * hits, BSDF evaluations, traversal counters) so parity tests can compare
 * them one by one with a CPU restatement of the reference, and select the
 * schedule the tracer uses.
 */
#ifndef PT_B200_DEBUG_H
#define PT_B200_DEBUG_H

#include "pt_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* sobol_owen_4d(i, seed) for i in 0..n (src/pathtrace.rs:388-398): 4n floats. */
PT_API pt_status pt_debug_sobol(pt_context *ctx, uint32_t n, uint32_t seed, float *out);
/* Sampler::pattern(pattern) of sample `index` for every pixel of the synced
 * tracer: width*height*4 floats. */
PT_API pt_status pt_debug_pattern(pt_tracer *tr, uint32_t index, uint32_t pattern, float *out);
/* Camera-ray closest hit (k = 0 acceptance filter) of sample `index` for every
 * pixel: global triangle id (0xffffffff on a miss) and (t, b0, b1, b2). */
PT_API pt_status pt_debug_primary_hits(pt_tracer *tr, uint32_t index, uint32_t *out_global, float *out_tbary);
/* Bsdf::new(ms, v, ng, front) then eval(dirs[i]) and sample(us[i]) for i < n.
 * params: 36 MaterialSample floats (layout of the oracle's test hook) then
 * v[3], ng[3], front. out: 12 floats per i = f[3], pdf, ok, l[3], f_s[3], pdf_s. */
PT_API pt_status pt_debug_bsdf(pt_context *ctx, const float *params, const float *dirs, const float *us, uint32_t n,
                        float *out);
/* Traversal work of the last refine: BVH nodes visited, triangles tested. */
PT_API pt_status pt_tracer_traversal_counts(const pt_tracer *tr, uint64_t *nodes, uint64_t *tris);
/* Traversal work of the last refine split by ray kind:
 * out = {closest-hit nodes, closest-hit triangles, any-hit nodes, any-hit triangles}. */
PT_API pt_status pt_tracer_traversal_split(const pt_tracer *tr, uint64_t out[4]);
/* Per-stage device time of refine calls (CUDA events between the kernels of
 * each stage on the context stream), off by default. Stages, in order:
 * ray generation, closest hit, shade, shadow rays, accumulate, megakernel,
 * material sort. */
PT_API pt_status pt_set_stage_timing(pt_context *ctx, int on);
PT_API pt_status pt_tracer_stage_ms(const pt_tracer *tr, float *out, uint32_t n);
/* The same figures for the last refine or batch of the context as a whole
 * (pt_tracer_refine_many included): out = {closest-hit rays, any-hit rays,
 * closest-hit nodes, closest-hit triangles, any-hit nodes, any-hit
 * triangles, samples, waves, bounce rounds summed over the waves (each
 * round is one extension, shade and shadow launch in the wavefront)}, and
 * per-stage device ms (stage timing on). */
PT_API pt_status pt_batch_counters(const pt_context *ctx, uint64_t out[9]);
PT_API pt_status pt_batch_stage_ms(const pt_context *ctx, float *out, uint32_t n);
/* Wavefront shade order: nonzero buckets the active queue by (scene,
 * material) before each shade launch so warps shade one material at a time
 * (three small kernels per bounce; on by default). Images are identical
 * either way. */
PT_API pt_status pt_set_material_sort(pt_context *ctx, int on);
/* Traversal kernels (closest hit and shadow rays): `threads` per block (128
 * or 256; 1,024 threads per SM either way) and `claim_chunk` queue entries
 * a lane claims per refill (1, 2 or 4: fewer atomics, coarser load
 * balance). Defaults 256 and 1. Images are identical whatever the setting;
 * pt_autotune tries both knobs on its winning configuration. */
PT_API pt_status pt_set_traversal(pt_context *ctx, uint32_t threads, uint32_t claim_chunk);
/* Overlapped waves (default on): a refine of two or more waves traces
 * consecutive waves in several path-state arenas on as many streams, so one
 * wave's last bounces (few paths, most of the GPU idle) run beside the next
 * wave's first; the accumulates stay in wave order. `on`: 0 one wave at a
 * time, 1 the default (three arenas, or the scene class's tuned count), 2
 * or 3 that many arenas. Images are identical whatever the setting. */
PT_API pt_status pt_set_wave_overlap(pt_context *ctx, int on);
/* Occupancy of the wavefront shade kernel: 3 (default) or 4 blocks of 128
 * threads per SM. Images are identical either way. */
PT_API pt_status pt_set_shade_blocks(pt_context *ctx, uint32_t blocks_per_sm);
/* Wavefront waves replayed from CUDA graphs (one capture per bounce count
 * and sort setting; on by default, bypassed while stage timing is on). */
PT_API pt_status pt_set_wave_graphs(pt_context *ctx, int on);

/* Builds a scene's device image on the host only (validation, textures,
 * BVH, tables; no GPU needed) and reports its host time in seconds:
 * {total, tables (textures and mips, materials, lights, emissive tables),
 * BVH build, the image fill (corner streams and tables copied into place)},
 * and the device bytes the scene would occupy. */
PT_API pt_status pt_debug_prepare_scene(const pt_scene_desc *desc, double seconds[4], uint64_t *device_bytes);

/* ---- autotuner: one configuration per scene class ----
 * A scene class groups scenes by triangle-count scale (factors of 4),
 * emissive triangles, environment map, punctual lights and textures. */
typedef struct pt_tune_choice {
  uint32_t schedule;             /* pt_schedule */
  uint32_t node_width_extension; /* 2 or 4 */
  uint32_t node_width_shadow;    /* 2 or 4 */
  uint32_t material_sort;        /* 0 / 1 */
  uint32_t wave_slots;
  float samples_per_s;           /* calibration throughput */
  uint32_t shade_blocks_per_sm;  /* 3 or 4: the shade kernel's occupancy */
  uint32_t wave_arenas;          /* 2 or 3: overlapped waves in flight (pt_set_wave_overlap) */
  uint32_t traversal_threads;    /* 128 or 256: block size of the traversal kernels (pt_set_traversal) */
  uint32_t claim_chunk;          /* 1, 2 or 4: queue entries a traversal lane claims per refill */
} pt_tune_choice;
/* Times every candidate (megakernel; wavefront x node widths x material sort
 * x wave size; then the winner with the shade kernel at 4 instead of 3
 * blocks per SM, with 128-thread traversal blocks or 2 / 4 queue entries per
 * lane refill, and with 2 or 3 waves in flight over eight waves) on a
 * calibration refine of `samples` spp (0: one full wave of
 * 8,388,608 paths, capped at 4096 spp) of the tracer's
 * scene, camera and options (a scratch accumulator: the tracer's own is
 * untouched) and records the fastest as the configuration of the scene's
 * class: later refines of tracers in that class use it. Every candidate
 * gives bit-identical images. `best` may be NULL. */
PT_API pt_status pt_autotune(pt_context *ctx, pt_tracer *tr, uint32_t samples, pt_tune_choice *best);
/* The recorded configuration of the tracer's scene class: PT_OK, or
 * PT_ERR_NOT_FOUND when the class has not been tuned. */
PT_API pt_status pt_tune_lookup(pt_context *ctx, const pt_tracer *tr, pt_tune_choice *out);
/* Forgets every recorded configuration. */
PT_API pt_status pt_tune_reset(pt_context *ctx);
/* BVH statistics of a resident scene. */
PT_API pt_status pt_scene_bvh_stats(pt_context *ctx, uint32_t scene_id, uint32_t *nodes, uint32_t *leaves,
                             uint32_t *max_depth, double *sah_cost, double *build_seconds);

/* Where pt_scene_upload builds a scene's BVH: on the host (binned SAH, 16
 * bins per axis), on the device with the same split rule (DEVICE: the
 * host's tree, built level by level on the GPU), on the device by
 * parallel locally-ordered clustering over Morton order with an SAH leaf
 * collapse (DEVICE_PLOC: faster to build, 3-12 % more node visits per ray),
 * or AUTO (the default): DEVICE for scenes of at least 16,384 triangles,
 * the host below. The device builders take scenes of at least 64
 * triangles; a device-built tree deeper than the traversal stacks allow is
 * rebuilt on the host. Images are identical whichever tree a scene has. */
typedef enum pt_bvh_builder {
  PT_BVH_BUILD_AUTO = 0,
  PT_BVH_BUILD_HOST = 1,
  PT_BVH_BUILD_DEVICE = 2,
  PT_BVH_BUILD_DEVICE_PLOC = 3,
  /* Spatial-split BVH on the host (Stich et al. 2009): triangles straddling
   * a split plane are referenced from both sides with clipped bounds, up
   * to 4x the triangle records. On scenes of many small overlapping
   * triangles (the random soups) it cuts node visits by about 38 % and
   * triangle tests by a third; well-shaped meshes barely change. The build
   * takes seconds, so it suits scenes that stay resident. */
  PT_BVH_BUILD_HOST_SPATIAL = 4
} pt_bvh_builder;
PT_API pt_status pt_set_bvh_builder(pt_context *ctx, uint32_t builder);
/* Host-only BVH build of a triangle soup (9 floats per triangle), for tests
 * and tree-quality studies: `spatial` nonzero builds the spatial-split tree.
 * stats = {two-child nodes, leaves, max depth, SAH cost, seconds, triangle
 * records}. When `nodes` / `records` are non-NULL and their capacities
 * (in 64-byte nodes / 48-byte records) suffice, the two-child nodes and the
 * leaf-ordered records are copied out. */
PT_API pt_status pt_debug_build_bvh(const float *positions, uint32_t triangles, uint32_t spatial, double stats[6],
                                    void *nodes, uint64_t node_capacity, void *records, uint64_t record_capacity);
/* 1 when the scene's current BVH was built on the device. */
PT_API pt_status pt_scene_bvh_on_device(pt_context *ctx, uint32_t scene_id, int *on_device);
/* Host wall time in seconds of the scene's pt_scene_upload: [0] the host
 * image (validation, attribute streams, materials, texture mips, tables,
 * and the host BVH when built there), [1] device allocation + copy, [2] the
 * device BVH build (0 when built on the host), [3] total. */
PT_API pt_status pt_scene_upload_seconds(pt_context *ctx, uint32_t scene_id, double seconds[4]);
/* The scene's texel pool as generated on the device: for each texture in
 * order, for each mip level, the sRGB-decoded level then the linear level
 * (RGBA f32). Copies at most `capacity` texels to `out` (may be NULL) and
 * reports the pool's texel count in `total`. */
PT_API pt_status pt_debug_scene_texels(pt_context *ctx, uint32_t scene_id, float *out, uint64_t capacity,
                                       uint64_t *total);

/* Fault injection on the host (tests): the next `count` device allocations
 * the context makes (accumulators, wave arenas and tables, scene uploads)
 * fail with PT_ERR_OOM as if cudaMalloc had run out of memory, without
 * calling CUDA. The context stays usable. 0 disarms it. */
PT_API pt_status pt_debug_fail_allocations(pt_context *ctx, uint32_t count);

/* Schedule of the hot loop: one path per thread (megakernel), or the
 * wavefront (extend / shade / shadow kernels over compacted queues; the
 * default of a new context). Both produce bit-identical accumulators. */
typedef enum pt_schedule { PT_SCHEDULE_MEGAKERNEL = 0, PT_SCHEDULE_WAVEFRONT = 1 } pt_schedule;
PT_API pt_status pt_set_schedule(pt_context *ctx, uint32_t schedule);
/* Maximum path slots per wave (device sample buffer 16 B per slot). */
PT_API pt_status pt_set_wave_slots(pt_context *ctx, uint32_t slots);
/* BVH node layout the wavefront's traversal kernels walk, for extension and
 * for shadow rays: 2 (two-child 64-byte nodes) or 4 (the same tree as
 * four-child 128-byte nodes). Default: 4 for both. Hits are identical
 * either way. */
PT_API pt_status pt_set_node_width(pt_context *ctx, uint32_t extension_width, uint32_t shadow_width);
/* Device time in ms of the last refine's path-tracing kernels (CUDA events
 * on the context stream). */
PT_API pt_status pt_tracer_last_kernel_ms(const pt_tracer *tr, float *ms);

#ifdef __cplusplus
}
#endif

#endif /* PT_B200_DEBUG_H */
