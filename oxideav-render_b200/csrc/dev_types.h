// Device-resident scene / request layout shared by host and device code.
//
// HBM layout of one resident scene (all arrays 256-byte aligned):
//   nodes     BvhNode[node_count]        64 B  two child boxes + child refs
//   nodes4    Bvh4Node[node4_count]     128 B  the same tree, four children per node
//   tris      float4[3 * tri_count]      48 B  leaf-ordered triangle records:
//                                              (v0.xyz, global id), v1, v2
//   tri_info  uint2[tri_count]            8 B  (material, attribute flags) by global id
//   pos       float[9 * tri_count]       36 B  corner positions by global id
//   nrm/tan/uv[s]/col                          optional corner streams by global id
//   materials, textures (+ one float4 texel pool for every mip level of
//   every texture, sRGB and linear chains), lights, emissive table.
// Per request: the camera, options, an f64 accumulator (32 B / pixel).
#pragma once

#include <cstdint>

#include <vector_types.h>

#include "../../include/pt_b200.h"

namespace ptd {

// Two-child node, 64 bytes, fetched as four float4:
//   a = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)
//   b = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//   c = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
//   d = (child0, child1, count0, count1) as int: child >= 0 is an interior
//       node index, child < 0 is a leaf whose first triangle record is ~child.
struct alignas(16) BvhNode {
  float4 a, b, c;
  int4 d;
};

// Four-child node, 128 bytes (one cache line), the same tree collapsed so
// each node holds up to four children, boxes stored by axis:
//   lo_x / hi_x / lo_y / hi_y / lo_z / hi_z  = that bound of children 0..3
//   child = child refs as in BvhNode (>= 0 node, < 0 leaf), kEmptyChild
//           for unused slots.
struct alignas(128) Bvh4Node {
  float4 lo_x, hi_x, lo_y, hi_y, lo_z, hi_z;
  int4 child;
  int4 pad;
};
constexpr int kEmptyChild = 0x7fffffff;
// Node layout per ray kind in the wavefront (DevRequest::wide_nodes).
enum WideNodes : uint32_t { WIDE_EXTENSION = 1u, WIDE_SHADOW = 2u };

enum TriFlags : uint32_t {
  TRI_HAS_VN = 1u << 0,       // has_vertex_normals and a normal stream
  TRI_HAS_TANGENTS = 1u << 1,
  TRI_HAS_COLORS = 1u << 2,
  TRI_UV0 = 1u << 3,          // TRI_UV0 << s: UV set s present
};

// Triangle record flags (second record's w): what the any-hit filter needs
// without touching the material table.
enum RecordFlags : uint32_t { REC_OPAQUE = 1u, REC_DOUBLE_SIDED = 2u };

constexpr int kMaxMipLevels = 16;

struct DevTexture {
  uint32_t img_w, img_h, levels;
  uint32_t mag, min, wrap_s, wrap_t, pad;
  uint32_t lw[kMaxMipLevels], lh[kMaxMipLevels];
  uint64_t srgb_off[kMaxMipLevels], lin_off[kMaxMipLevels];  // texel offsets into the pool
  // The uploaded source texels the chains are generated from: byte offset
  // in the scene's source-texel part, PT_PIXELS_* format.
  uint64_t src_off;
  uint32_t src_format, pad2;
};

// pt_material plus values the host precomputes so the device never
// evaluates a transcendental of a scene constant.
struct DevMaterial {
  pt_material m;
  float aniso_sin, aniso_cos;  // sin / cos of fin(anisotropy_rotation, 0)
  uint32_t emissive_nonblack;  // !is_black(emissive)
  uint32_t pad;
};

struct DevLight {
  pt_light l;
  float cos_outer, cos_inner;  // spot cone cosines
};

struct DevScene {
  const BvhNode *nodes;
  const float4 *tris;
  const uint2 *tri_info;
  const float *pos, *nrm, *tan, *uv[PT_MAX_UV_SETS], *col;
  const DevMaterial *materials;
  const DevTexture *textures;
  const float4 *texels;
  const DevLight *lights;
  const uint32_t *em_tris;
  const float *em_pmf, *em_cdf;
  const uint32_t *em_lookup;
  uint32_t node_count, tri_count, material_count, texture_count, light_count, em_count;
  uint32_t max_depth, node4_count;
  const Bvh4Node *nodes4;  // the same tree with four-child nodes
};

struct DevEnv {
  uint32_t w, h, uniform, pad;
  float intensity, pad1, pad2, pad3;
  const float4 *pixels;       // w * h texels (scene-linear RGBA)
  const float *marginal;      // h + 1
  const float *conditional;   // h * (w + 1)
  const float *mass;          // w * h
};

// Everything one accumulation needs (the reference's Integrator,
// src/pathtrace.rs:1878-1890): scene, environment, camera, options.
struct DevRequest {
  const DevScene *scene;
  const DevEnv *env;  // nullptr: constant sky `ambient`
  pt_camera cam;
  uint32_t width, height;
  float ambient, pixel_spread;
  uint32_t orthographic, max_bounces, rr_start, seed, strategy;
  float clamp;
  float p_env;  // probability the area-light sampler picks the environment
  uint32_t wide_nodes;  // WIDE_* bits: which rays walk the four-child layout
  double *accum;  // width * height * 4 (sum r, g, b, covered count)
};

// A contiguous run of path slots of one request within a wave: slot
// `slot_begin + s * pixel_count + i` traces sample `sample_begin + s` of
// pixel `pixel_begin + i` (i < pixel_count, s < spp).
struct WaveSegment {
  uint32_t request;
  uint32_t slot_begin;
  uint32_t pixel_begin, pixel_count;
  uint32_t sample_begin, spp;
  uint32_t pad0, pad1;
};

// Structure-of-arrays path state of one wave of the wavefront schedule
// (wavefront.cuh), `capacity` slots, `shadow_slots` queued shadow rays per
// slot.
// Per iteration: [0] active count, [1] shadow-queue count, [2] extend claim
// cursor, [3] shadow claim cursor, [4] most shadow rays of a queued path,
// [5..7] spare.
constexpr uint32_t kWfCounterStride = 8;

struct WaveBuffers {
  float4 *o, *d, *beta, *rad, *prev, *sigma;
  uint4 *seed;                 // pixel_seed, sample index, path_seed, request
  float4 *hit_tb;              // t, b0, b1, b2
  uint32_t *hit_g;             // global id | front << 31 | found << 30
  float4 *sh_o, *sh_d, *sh_c;  // [shadow_slots][capacity]: (o, tmax), (d, ray id), (contrib, skip)
  uint32_t *sh_n;              // shadow rays queued per slot
  uint8_t *sh_vis;             // [shadow_slots][capacity]: 1 where the shadow ray reached its light
  uint32_t *q[2];              // active queues (ping-pong by iteration)
  uint32_t *q_shadow;
  uint32_t *counters;          // [iterations][kWfCounterStride]
  uint32_t *q_sorted;          // the active queue bucketed by material (material sort on)
  uint32_t *sort_keys;         // material-sort key of each active-queue position (set by extend)
  uint32_t *sort_counts;       // [iterations][2][kSortBuckets]: bucket sizes, then cursors
  float4 *nee;                 // [3][capacity]: the NEE kernel's area sample and emission pdf per slot
  struct WaveDesc *desc;       // this wave's requests and segments (written before each wave)
  uint32_t capacity, shadow_slots, iterations, sort_materials;
  uint32_t shade_blocks;       // 3 or 4: the k_wf_shade instantiation (blocks per SM)
  uint32_t trav_threads;       // 128 or 256: block size of the traversal kernels (1,024 threads per SM)
  uint32_t claim_chunk;        // 1, 2 or 4: queue entries a traversal lane claims per refill
  uint32_t all_wide;           // WIDE_* bits that hold for every request of the wave (host-side launch choice)
};

// What changes from one wave to the next, read by the kernels from device
// memory, so a wave's launch sequence is the same for every wave of the same
// bounce count (and can be replayed as one CUDA graph).
struct WaveDesc {
  const DevRequest *reqs;
  const WaveSegment *segs;
  uint32_t nseg, total, max_pix;
  uint32_t flags;  // WAVE_AREA_LIGHTS: some request has emissive triangles or an environment
};
enum WaveFlags : uint32_t { WAVE_AREA_LIGHTS = 1u };
constexpr uint32_t kSortBuckets = 256;

// Per-launch device counters (rays traced, traversal work, errors).
struct DevCounters {
  unsigned long long ext_rays, shadow_rays;
  unsigned long long ext_nodes, ext_tris;  // traversal work of closest-hit rays
  unsigned long long sh_nodes, sh_tris;    // traversal work of any-hit (shadow) rays
  unsigned int error_flags, pad;
};

// Stages timed by the optional per-stage CUDA events.
enum Stage : int { STAGE_RAYGEN = 0, STAGE_EXTEND, STAGE_SHADE, STAGE_SHADOW, STAGE_ACCUMULATE, STAGE_MEGAKERNEL,
                   STAGE_SORT, STAGE_NEE, STAGE_END, STAGE_COUNT = STAGE_END };
enum ErrorFlags : uint32_t { ERR_STACK_OVERFLOW = 1u };

}  // namespace ptd
