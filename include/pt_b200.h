/*
 * pt_b200.h — C ABI of the B200-native path tracer (RenderBackend::PathTraceCuda).
 *
 * The library is a drop-in for oxideav-render's CPU PathTrace backend. A Rust
 * host binds these entry points through a thin `extern "C"` crate and keeps the
 * reference's own front half unchanged:
 *
 *   Scene3D --PreparedScene::build--> PreparedScene   (src/prepare.rs:1098-1234)
 *           --Camera::resolve-------> Camera           (src/camera.rs:177-188)
 *   RenderOptions / PathTraceOptions                  (src/options.rs:67-146, 325-414)
 *
 * and hands the flattened result to this library, which owns the device copy of
 * the scene (BVH, triangles, attributes, materials, textures, lights), the
 * progressive accumulator, and every kernel of the hot loop
 * (PathTracer::refine -> Integrator::sample, src/pathtrace.rs:2004-2329, 2531-2591).
 *
 * Conventions
 *   - Every call returns a pt_status; PT_OK is 0. On failure pt_last_error()
 *     holds a one-line message. No exception and no abort crosses the ABI.
 *   - Caller-owned host arrays are read during the call only (the library copies
 *     what it keeps to the device).
 *   - A pt_context is single-owner (Renderer: Send, not Sync): calls on one
 *     context must not overlap. Distinct contexts are independent.
 *   - All structs are plain C, fixed-width, naturally aligned, #[repr(C)]
 *     compatible.
 */
#ifndef PT_B200_H
#define PT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PT_ABI_VERSION 2u

#if defined(__GNUC__)
#define PT_API __attribute__((visibility("default")))
#else
#define PT_API
#endif

/* ------------------------------------------------------------------ status */

/* Maps to oxideav_render::Error (src/error.rs:16-43): INVALID_ARG ->
 * Error::InvalidOptions / Error::Scene, everything else -> Error::Backend. */
typedef enum pt_status {
  PT_OK = 0,
  PT_ERR_INVALID_ARG = 1, /* bad pointer, size or enum value */
  PT_ERR_OOM = 2,         /* device allocation failed / over the HBM budget */
  PT_ERR_DEVICE = 3,      /* CUDA runtime error (no device, launch failure) */
  PT_ERR_TIMEOUT = 4,     /* a bounded device wait gave up */
  PT_ERR_EVICTED = 5,     /* the scene was evicted from the resident cache */
  PT_ERR_CANCELLED = 6,   /* the request was cancelled */
  PT_ERR_NOT_FOUND = 7,   /* unknown scene / request / tracer handle */
  PT_ERR_NOT_READY = 8    /* pt_server_poll: request still running */
} pt_status;

/* ------------------------------------------------------------------ scene */

#define PT_MAX_UV_SETS 4

/* TextureBinding (src/prepare.rs:380-432) with the KHR_texture_transform
 * already turned into a 2x3 affine matrix by the host:
 *   u' = m[0]*u + m[1]*v + m[2];  v' = m[3]*u + m[4]*v + m[5].
 * texture < 0 means "no binding" (Option::None, or an unresolved
 * extension texture reference, TraceScene::bind_ref src/trace.rs:624-633). */
typedef struct pt_texture_binding {
  int32_t texture;
  uint32_t uv_set;        /* effective TEXCOORD set (TextureRef::effective_uv_set) */
  uint32_t has_transform; /* 0: identity (TextureBinding::transform == None) */
  float transform[6];
} pt_texture_binding;

typedef enum pt_alpha_mode { PT_ALPHA_OPAQUE = 0, PT_ALPHA_MASK = 1, PT_ALPHA_BLEND = 2 } pt_alpha_mode;

/* Presence bits of oxideav_mesh3d::MaterialExt's Option<...> members. */
enum {
  PT_EXT_SPECULAR = 1u << 0,
  PT_EXT_TRANSMISSION = 1u << 1,
  PT_EXT_VOLUME = 1u << 2,
  PT_EXT_CLEARCOAT = 1u << 3,
  PT_EXT_SHEEN = 1u << 4,
  PT_EXT_ANISOTROPY = 1u << 5,
  PT_EXT_IRIDESCENCE = 1u << 6,
  PT_EXT_DIFFUSE_TRANSMISSION = 1u << 7,
  PT_EXT_DISPERSION = 1u << 8
};

/* PreparedMaterial (src/prepare.rs:437-476, factors resolved as in
 * from_material :625-670) plus the raw MaterialExt values the path tracer
 * reads in TraceScene::material_oriented (src/trace.rs:757-890). Extension
 * values are passed verbatim (non-finite values are defaulted on the device
 * exactly as the reference's `fin` helper does). */
typedef struct pt_material {
  float base_color[4];
  pt_texture_binding base_color_texture;
  float metallic;
  float roughness;
  pt_texture_binding metallic_roughness_texture;
  pt_texture_binding normal_texture;
  float normal_scale;
  pt_texture_binding occlusion_texture;
  float occlusion_strength;
  float emissive[3]; /* emissive_strength already multiplied in */
  pt_texture_binding emissive_texture;
  uint32_t alpha_mode; /* pt_alpha_mode */
  float alpha_cutoff;
  uint32_t double_sided;
  uint32_t unlit;
  float ior;
  uint32_t ext_flags; /* PT_EXT_* */
  /* KHR_materials_specular */
  float specular_factor;
  pt_texture_binding specular_texture;
  float specular_color_factor[3];
  pt_texture_binding specular_color_texture;
  /* KHR_materials_transmission */
  float transmission_factor;
  pt_texture_binding transmission_texture;
  /* KHR_materials_volume (attenuation_distance = effective value, +inf = none) */
  float thickness_factor;
  pt_texture_binding thickness_texture;
  float attenuation_distance;
  float attenuation_color[3];
  /* KHR_materials_clearcoat */
  float clearcoat_factor;
  pt_texture_binding clearcoat_texture;
  float clearcoat_roughness_factor;
  pt_texture_binding clearcoat_roughness_texture;
  pt_texture_binding clearcoat_normal_texture;
  float clearcoat_normal_scale;
  /* KHR_materials_sheen */
  float sheen_color_factor[3];
  pt_texture_binding sheen_color_texture;
  float sheen_roughness_factor;
  pt_texture_binding sheen_roughness_texture;
  /* KHR_materials_anisotropy */
  float anisotropy_strength;
  float anisotropy_rotation;
  pt_texture_binding anisotropy_texture;
  /* KHR_materials_iridescence */
  float iridescence_factor;
  pt_texture_binding iridescence_texture;
  float iridescence_ior;
  float iridescence_thickness_min;
  float iridescence_thickness_max;
  pt_texture_binding iridescence_thickness_texture;
  /* KHR_materials_diffuse_transmission */
  float diffuse_transmission_factor;
  pt_texture_binding diffuse_transmission_texture;
  float diffuse_transmission_color_factor[3];
  pt_texture_binding diffuse_transmission_color_texture;
  /* KHR_materials_dispersion */
  float dispersion;
} pt_material;

typedef enum pt_filter { PT_FILTER_NEAREST = 0, PT_FILTER_LINEAR = 1 } pt_filter;
typedef enum pt_min_filter {
  PT_MIN_NEAREST = 0,
  PT_MIN_LINEAR = 1,
  PT_MIN_NEAREST_MIP_NEAREST = 2,
  PT_MIN_LINEAR_MIP_NEAREST = 3,
  PT_MIN_NEAREST_MIP_LINEAR = 4,
  PT_MIN_LINEAR_MIP_LINEAR = 5
} pt_min_filter;
typedef enum pt_wrap { PT_WRAP_REPEAT = 0, PT_WRAP_CLAMP = 1, PT_WRAP_MIRROR = 2 } pt_wrap;
typedef enum pt_pixel_format { PT_PIXELS_RGBA8 = 0, PT_PIXELS_RGBA_F32 = 1 } pt_pixel_format;

/* PreparedTexture (src/texture.rs:386-410): a decoded image (DecodedImage,
 * src/texture.rs:108-116) plus the glTF sampler with the mesh3d
 * effective_{mag,min}_filter already applied. The library builds the sRGB
 * and linear mip chains itself (build_mips, src/texture.rs:324-383).
 * pixels == NULL marks an unresolved texture (PreparedScene::textures[i] ==
 * None). */
typedef struct pt_texture {
  uint32_t width;
  uint32_t height;
  uint32_t format; /* pt_pixel_format */
  const void *pixels;
  uint32_t mag_filter; /* pt_filter */
  uint32_t min_filter; /* pt_min_filter */
  uint32_t wrap_s;     /* pt_wrap */
  uint32_t wrap_t;
} pt_texture;

/* One triangle DrawItem (src/prepare.rs:170-211): world-space, de-indexed,
 * CCW front. Line / point items carry no area and are not passed. Optional
 * streams are NULL when absent (or when their length does not match the
 * positions, which the reference treats as absent). */
typedef struct pt_draw_item {
  uint32_t triangle_count;            /* corners = 3 * triangle_count */
  const float *positions;             /* [corners][3] */
  const float *normals;               /* [corners][3] or NULL */
  uint32_t has_vertex_normals;        /* DrawItem::has_vertex_normals */
  const float *tangents;              /* [corners][4] or NULL */
  const float *uvs[PT_MAX_UV_SETS];   /* [corners][2] or NULL, per TEXCOORD_n */
  const float *colors;                /* [corners][4] (COLOR_0, linear) or NULL */
  uint32_t material;                  /* index into pt_scene_desc::materials */
} pt_draw_item;

typedef enum pt_light_kind { PT_LIGHT_DIRECTIONAL = 0, PT_LIGHT_POINT = 1, PT_LIGHT_SPOT = 2 } pt_light_kind;

/* PreparedLight (src/prepare.rs:687-713). */
typedef struct pt_light {
  uint32_t kind; /* pt_light_kind */
  float color[3];
  float intensity;
  float position[3];
  float direction[3]; /* unit direction the light travels */
  uint32_t has_range;
  float range;
  float inner_cone_angle;
  float outer_cone_angle;
} pt_light;

/* PreparedScene (src/prepare.rs:1028-1048) restricted to what the path
 * tracer reads: triangle items in order (their concatenation is the
 * TraceScene soup, src/trace.rs:328-351, so the global triangle id of item
 * i's triangle t is the running triangle count before i plus t), materials,
 * textures and the punctual lights (scene lights or the options fallback). */
typedef struct pt_scene_desc {
  uint32_t item_count;
  const pt_draw_item *items;
  uint32_t material_count;
  const pt_material *materials;
  uint32_t texture_count;
  const pt_texture *textures;
  uint32_t light_count;
  const pt_light *lights;
} pt_scene_desc;

/* Equirectangular environment (EnvironmentMap::new, src/pathtrace.rs:1575):
 * scene-linear RGBA f32, row 0 = +Y, scaled by intensity. The library builds
 * the luminance x sin(theta) sampling CDFs. */
typedef struct pt_environment {
  uint32_t width;
  uint32_t height;
  const float *pixels; /* [height][width][4] */
  float intensity;
} pt_environment;

/* ------------------------------------------------------------------ camera / options */

typedef enum pt_projection { PT_PERSPECTIVE = 0, PT_ORTHOGRAPHIC = 1 } pt_projection;

/* Camera (src/camera.rs:63-91): the placement fields primary_ray reads. */
typedef struct pt_camera {
  float eye[3];
  float forward[3];
  float side[3];
  float up[3];
  float half_w;
  float half_h;
  uint32_t projection; /* pt_projection */
} pt_camera;

typedef enum pt_light_strategy { PT_MIS = 0, PT_LIGHT_ONLY = 1, PT_BSDF_ONLY = 2 } pt_light_strategy;
typedef enum pt_tone_map { PT_TONE_CLAMP = 0, PT_TONE_REINHARD = 1, PT_TONE_ACES = 2 } pt_tone_map;

/* PathTraceOptions (src/options.rs:67-89). */
typedef struct pt_path_trace_options {
  uint32_t samples_per_pixel;
  uint32_t max_bounces;
  uint32_t rr_start;
  float clamp;
  uint32_t seed;
  uint32_t strategy; /* pt_light_strategy */
} pt_path_trace_options;

/* The RenderOptions fields the path tracer reads (the camera fields are
 * consumed by Camera::resolve on the host and arrive as pt_camera). */
typedef struct pt_render_options {
  uint32_t width;
  uint32_t height;
  uint8_t background[4]; /* BackgroundColor, RGBA8 */
  uint32_t tone_map;     /* pt_tone_map */
  float exposure;
  float ambient;
  pt_path_trace_options path_trace;
} pt_render_options;

/* ------------------------------------------------------------------ context / scenes */

typedef struct pt_context pt_context;

/* Create a context on CUDA device `device` (one per GPU). */
PT_API pt_status pt_create(pt_context **out, int device);
/* Destroys the context and its resident scenes; destroy its tracers first
 * (a tracer refers to its context). */
PT_API void pt_destroy(pt_context *ctx);
/* Message of the last failing call on ctx (or of pt_create when ctx is NULL). */
PT_API const char *pt_last_error(const pt_context *ctx);
PT_API uint32_t pt_abi_version(void);

/* Upload a prepared scene: the emissive-triangle table (EmissiveLights::build,
 * src/pathtrace.rs:1479-1543) on the host; the BVH (on the device for large
 * scenes, replaced by a host binned-SAH tree built in the background; see
 * pt_set_bvh_builder) and the texture mip chains on the device. The scene
 * stays in device memory until pt_scene_release (or until the serving cache
 * evicts it). */
PT_API pt_status pt_scene_upload(pt_context *ctx, const pt_scene_desc *desc, uint32_t *scene_id);
PT_API pt_status pt_scene_release(pt_context *ctx, uint32_t scene_id);
/* An animated frame of resident scene `scene_id` (no counterpart in the
 * reference, which re-prepares the scene every frame:
 * PreparedScene::build, src/prepare.rs:1110-1119, then TraceScene::new):
 * `desc` is the scene at another time with the same draw items and triangle
 * counts. Its streams and tables replace the old ones; the BVH keeps its
 * structure and is refitted on the device (records rewritten, node bounds
 * recomputed bottom up) instead of rebuilt. Images equal those of a fresh
 * pt_scene_upload of `desc` bit for bit (closest hits do not depend on the
 * tree); tracers on the scene must sync again (their accumulation resets).
 * PT_ERR_INVALID_ARG when the topology differs. */
PT_API pt_status pt_scene_refit(pt_context *ctx, uint32_t scene_id, const pt_scene_desc *desc);
/* Device bytes held by a resident scene. */
PT_API pt_status pt_scene_device_bytes(pt_context *ctx, uint32_t scene_id, uint64_t *bytes);
PT_API pt_status pt_scene_triangle_count(pt_context *ctx, uint32_t scene_id, uint64_t *count);

/* ------------------------------------------------------------------ progressive tracer */

/* PathTracer (src/pathtrace.rs:2369-2735) with a device-resident accumulator
 * (per pixel: sum r, sum g, sum b over covered samples, covered count, f64). */
typedef struct pt_tracer pt_tracer;

PT_API pt_status pt_tracer_create(pt_context *ctx, pt_tracer **out);
PT_API void pt_tracer_destroy(pt_tracer *tr);
/* PathTracer::sync: bind scene + camera + options. Resets the accumulator
 * exactly when the scene changed (other id, or invalidate_scene was called)
 * or the radiance key changed (radiance_key, src/pathtrace.rs:2402-2418:
 * everything except background, tone map, exposure and spp). *reset receives
 * 1 when it reset. */
PT_API pt_status pt_tracer_sync(pt_tracer *tr, uint32_t scene_id, const pt_camera *camera,
                         const pt_render_options *opts, int *reset);
/* PathTracer::refine: add `samples` samples to every pixel; sample indices
 * continue from pt_tracer_samples, so refine(a); refine(b) == refine(a + b)
 * bit for bit. Blocks until the device work is done. */
PT_API pt_status pt_tracer_refine(pt_tracer *tr, uint32_t samples);
PT_API pt_status pt_tracer_samples(const pt_tracer *tr, uint32_t *samples);
/* Batched refine (no counterpart in the reference, which refines one
 * tracer at a time): adds samples[i] samples to tracers[i] for every i, all
 * in shared waves of path slots on the context's device, each path reading
 * its own tracer's scene, camera, options and accumulator. Every tracer ends
 * bit-identical to pt_tracer_refine(tracers[i], samples[i]) run alone. All
 * tracers must belong to ctx and appear once. */
PT_API pt_status pt_tracer_refine_many(pt_context *ctx, pt_tracer *const *tracers, const uint32_t *samples,
                                       uint32_t count);
/* Device time, wave count and rays traced of the last refine / batch. */
PT_API pt_status pt_batch_stats(const pt_context *ctx, float *ms, uint32_t *waves, uint64_t *rays);
PT_API pt_status pt_tracer_is_converged(const pt_tracer *tr, int *converged);
PT_API pt_status pt_tracer_reset(pt_tracer *tr);
PT_API pt_status pt_tracer_invalidate_scene(pt_tracer *tr);
/* PathTracer::set_environment: env == NULL removes it. Resets accumulation. */
PT_API pt_status pt_tracer_set_environment(pt_tracer *tr, const pt_environment *env);
/* PathTracer::hdr (src/pathtrace.rs:2717-2734): width*height*4 floats. */
PT_API pt_status pt_tracer_read_hdr(pt_tracer *tr, float *out_rgba, size_t out_floats);
/* PathTracer::image (src/pathtrace.rs:2687-2713): width*height*4 bytes. */
PT_API pt_status pt_tracer_read_image(pt_tracer *tr, uint8_t *out_rgba, size_t out_bytes);
/* Raw accumulator: width*height*4 doubles (sum r, g, b, covered count). */
PT_API pt_status pt_tracer_read_accum(pt_tracer *tr, double *out, size_t out_doubles);
/* Rays traced by the last refine: closest-hit (extension) and any-hit (shadow). */
PT_API pt_status pt_tracer_ray_counts(const pt_tracer *tr, uint64_t *extension_rays, uint64_t *shadow_rays);

/* PathTraceRenderer::render / render_hdr (src/pathtrace.rs:2761-2777):
 * invalidate -> sync -> refine(max(spp, 1)) -> image / hdr, on a temporary
 * tracer. env may be NULL. */
PT_API pt_status pt_render_hdr(pt_context *ctx, uint32_t scene_id, const pt_camera *camera,
                        const pt_render_options *opts, const pt_environment *env,
                        float *out_rgba, size_t out_floats);
/* Refine without allocating. This entry point has no counterpart in the
 * reference. It is for callers that cannot allocate device memory inside a
 * call — a render loop whose frame budget forbids cudaMalloc / cudaFree
 * (they can synchronise the device), or a host whose memory all comes from
 * its own pool. The caller owns the output: `d_accum` is a device buffer of
 * width*height*4 doubles (sum r, g, b, covered count per pixel) that this
 * call adds `samples` samples to, starting at sample index `first_sample`
 * (so consecutive calls continue the sequence exactly like
 * pt_tracer_refine). `d_accum` must be 16-byte aligned, on the context's
 * device, and lie inside one device allocation with room for the whole
 * image; anything else is rejected with PT_ERR_INVALID_ARG before any
 * launch. The per-wave path samples live in a fixed scratch array compiled
 * into the library (1,048,576 path slots, 16 MiB, held by every GPU that
 * loads the library until the process exits); images above 1,048,576
 * pixels are rejected with PT_ERR_INVALID_ARG. No environment map (the sky is
 * `ambient`). The samples are traced by the megakernel schedule whatever
 * the context's schedule and tuned choices say: the image equals
 * pt_tracer_refine's, the speed is the megakernel's. The call waits for its
 * work (it synchronises the context's stream) before returning. The first
 * call on a device looks up the scratch address for that device and keeps
 * it for the life of the process (a cudaDeviceReset makes it stale); make
 * that first call before any stream capture. Every call reuses the same
 * scratch, so calls that overlap on the GPU race: serialise them. */
PT_API pt_status pt_refine_noalloc(pt_context *ctx, uint32_t scene_id, const pt_camera *camera,
                                   const pt_render_options *opts, uint32_t first_sample, uint32_t samples,
                                   double *d_accum);

PT_API pt_status pt_render_image(pt_context *ctx, uint32_t scene_id, const pt_camera *camera,
                          const pt_render_options *opts, const pt_environment *env,
                          uint8_t *out_rgba, size_t out_bytes);

/* ------------------------------------------------------------------ raycast */

/* ShadingMode (src/options.rs:150-187). */
typedef enum pt_shading_mode {
  PT_SHADE_FLAT = 0,
  PT_SHADE_GOURAUD = 1,
  PT_SHADE_PHONG = 2,
  PT_SHADE_WIREFRAME = 3,
  PT_SHADE_NORMAL_DEBUG = 4,
  PT_SHADE_DEPTH_DEBUG = 5,
  PT_SHADE_PBR = 6
} pt_shading_mode;

/* What the raycast backend reads of RenderOptions (src/options.rs) plus the
 * camera's clip planes (Camera::near / far, src/camera.rs:80-84). */
typedef struct pt_raycast_options {
  uint32_t width, height;  /* output pixels */
  uint32_t aa;             /* SSAA factor per axis, 1..=8 */
  uint32_t shading;        /* pt_shading_mode */
  float light_azimuth_deg, light_elevation_deg, light_intensity; /* LightSpec */
  uint8_t background[4];
  uint32_t tone_map;       /* pt_tone_map */
  float exposure;
  uint32_t max_ray_depth;  /* capped at 16 */
  float near_plane, far_plane;
  /* PT_SHADE_PBR only: */
  float ambient;                     /* uniform environment radiance (>= 0) */
  uint32_t shadows;                  /* ray-traced hard shadows for every light */
  float reflection_roughness_cutoff; /* in [0, 1]; 0 = no mirror rays */
} pt_raycast_options;

/* The Whitted ray tracer behind RenderBackend::Raycast (src/raycast.rs:145-560)
 * on a resident scene: one ray per render sample (width·aa × height·aa,
 * through Camera::primary_ray at the sample centre, `camera` resolved for
 * that resolution), the legacy shading modes (Flat, Gouraud, Phong with
 * Whitted's shadow, mirror and refraction rays up to max_ray_depth,
 * Wireframe, NormalDebug, DepthDebug), then the scanline backend's frame
 * resolve (src/scanline.rs:124-221): SSAA box filter, premultiplied
 * averages, exposure + tone map + sRGB for RGBA8. PT_SHADE_PBR evaluates the
 * glTF metallic-roughness model at every hit (src/raycast.rs:518-740):
 * ambient, emissive and direct light from every scene light (hard shadow
 * rays when `shadows` is set, passing MASK cut-outs, BLEND and transmissive
 * occluders), a mirror ray below reflection_roughness_cutoff, refraction
 * through thin walls and KHR_materials_volume bodies with Beer-Lambert
 * absorption, BLEND composited per ray, texture LOD from ray differentials
 * at camera hits and ray cones after a bounce. Writes the scene-linear HDR
 * image (width*height*4 floats) and/or the RGBA8 image (width*height*4
 * bytes); either pointer may be NULL. */
PT_API pt_status pt_raycast_render(pt_context *ctx, uint32_t scene_id, const pt_camera *camera,
                                   const pt_raycast_options *opts, float *out_hdr, size_t hdr_floats,
                                   uint8_t *out_rgba, size_t rgba_bytes);

#ifdef __cplusplus
}
#endif

#endif /* PT_B200_H */
