// Host-side scene preparation: BVH build, attribute streams, materials,
// texture mip chains, emissive-triangle table, environment CDFs, and the
// single device arena each resident scene lives in.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "dev_types.h"

namespace ptd {

struct BvhBuildStats {
  uint32_t nodes = 0, leaves = 0, max_depth = 0;
  double sah_cost = 0.0, seconds = 0.0;
  uint64_t references = 0;  // triangle records (above the triangle count with spatial splits)
};

// Binned-SAH BVH over the soup (positions: 9 floats per triangle), laid out
// as two-child 64-byte nodes, as the same tree collapsed to four-child
// 128-byte nodes, plus 48-byte leaf-ordered triangle records shared by both.
// `rec_flags[g]` goes into each record (REC_* bits).
void build_bvh(const float *pos, uint32_t tri_count, const uint32_t *rec_flags, std::vector<BvhNode> &nodes,
               std::vector<Bvh4Node> &nodes4, std::vector<float4> &records, BvhBuildStats &stats, int threads);
// The same outputs from a spatial-split BVH: fewer overlapping leaves for
// scenes of many small overlapping triangles, at a few times the build time
// and up to 4x the triangle records (a triangle cut by split planes is
// referenced from several leaves).
void build_bvh_spatial(const float *pos, uint32_t tri_count, const uint32_t *rec_flags,
                       std::vector<BvhNode> &nodes, std::vector<Bvh4Node> &nodes4, std::vector<float4> &records,
                       BvhBuildStats &stats, int threads);

// One device allocation holding a scene (or an environment) plus the
// device copy of its descriptor. `stream` non-null: the allocation is
// stream-ordered (cudaMallocAsync) and is freed in that stream's order.
struct DeviceArena {
  void *base = nullptr;
  uint64_t bytes = 0;
  cudaStream_t stream = nullptr;
  void release();
};

// A scene fully prepared on the host: the exact bytes of its device arena
// (attribute streams, materials, texel pool, lights, emissive tables), its
// BVH (nodes and triangle records, a second device allocation) and a
// descriptor whose pointer fields hold arena offsets + 1 (0 = absent).
// Uploading it is two allocations and a few copies, so an evicted scene
// comes back without another BVH build.
// Uninitialised host bytes (a scene image is written part by part; the
// alignment gaps are zeroed).
struct HostBlob {
  std::unique_ptr<uint8_t[]> p;
  uint8_t *ext = nullptr;  // borrowed memory (a HostStaging buffer) instead of p
  size_t n = 0;
  void allocate(size_t bytes) {
    p.reset(new uint8_t[bytes]);
    ext = nullptr;
    n = bytes;
  }
  void use(uint8_t *q, size_t bytes) {
    p.reset();
    ext = q;
    n = bytes;
  }
  uint8_t *data() { return ext ? ext : p.get(); }
  const uint8_t *data() const { return ext ? ext : p.get(); }
  size_t size() const { return n; }
};

// Page-locked host memory reused by every upload of a context (grow-only,
// up to kMaxStagingBytes): the image is written straight into it and the
// copy to the device runs at DMA speed.
struct HostStaging {
  static constexpr size_t kMaxStagingBytes = size_t(4) << 30;
  uint8_t *p = nullptr;
  size_t cap = 0;
  // `bytes` of pinned memory, or nullptr (too large, or pinning failed).
  uint8_t *reserve(size_t bytes);
  void release();
  ~HostStaging() { release(); }
};

// A BVH in its device layouts, in host memory.
struct HostTree {
  std::vector<BvhNode> nodes;
  std::vector<Bvh4Node> nodes4;
  std::vector<float4> records;
  uint64_t bytes() const;  // of its device allocation
};

struct SceneImage {
  HostBlob blob;   // everything but the BVH
  HostTree tree;   // empty when built without a BVH
  // Textures: the table (as in the blob), the source texels' offset in the
  // blob, and the device-only texel pool that follows the blob in the arena
  // (its mip chains are generated on the device at commit).
  std::vector<DevTexture> textures;
  uint64_t tex_src_off = 0, pool_off = 0, pool_bytes = 0;
  uint64_t device_bytes() const { return std::max<uint64_t>(blob.size(), pool_off + pool_bytes) + tree.bytes(); }
  DevScene rel{};
  uint64_t desc_off = 0;
  uint64_t tri_count = 0;
  BvhBuildStats bvh;
  uint32_t light_count = 0;
  // Host time of build_scene_image: total, tables (textures and their mips,
  // materials, lights, emissive tables), BVH build, the blob fill (corner
  // streams and tables copied into place).
  double seconds[4] = {0.0, 0.0, 0.0, 0.0};
};

struct SceneHost {
  DevScene dev{};           // pointers into `arena` (and `bvh_arena`)
  DevScene *d_desc = nullptr;
  DeviceArena arena;
  DeviceArena bvh_arena;    // nodes and records of a device-built BVH
  uint64_t tri_count = 0;
  uint64_t pool_texels = 0;  // texels of every mip chain (dev.texels)
  BvhBuildStats bvh;
  uint32_t light_count = 0;
  bool device_bvh = false;  // the BVH was built on the GPU
  // Host wall time of upload_scene: host image, arena allocation + copy,
  // device BVH build, total.
  double upload_seconds[4] = {0.0, 0.0, 0.0, 0.0};
  // Triangle count of every draw item, in order: a refit needs the same.
  std::vector<uint32_t> item_tris;
  uint64_t device_bytes() const { return arena.bytes + bvh_arena.bytes; }
};

// Validates `desc` and builds its device image on the host. Returns an
// empty string on success, else an error message. `with_bvh` false leaves
// the BVH parts out (node counts 0) for a build on the device.
// `spatial` builds the spatial-split tree (build_bvh_spatial) instead.
std::string build_scene_image(const pt_scene_desc &desc, SceneImage &img, bool with_bvh = true,
                              HostStaging *staging = nullptr, bool spatial = false);
// Allocates the arena and copies `img` into it (stream-ordered when `stream`
// is non-null). `oom` is set when the failure was a device allocation.
std::string commit_scene(const SceneImage &img, SceneHost &out, bool &oom, cudaStream_t stream = nullptr);
// Deepest leaf a tree may have: the traversal stacks hold 64 two-child
// entries and 3 * 56 + 8 four-child entries.
constexpr uint32_t kMaxTreeDepth = 56;
// Where upload_scene builds the BVH.
// BVH_BUILD_AUTO: scenes of at least kAutoDeviceBuildTris triangles build
// on the device with the binned-SAH rule (the host builder's tree, in
// milliseconds), smaller ones on the host. BVH_BUILD_DEVICE_PLOC clusters
// on the device instead (faster to build, 3-12 % more node visits).
// BVH_BUILD_HOST_SPATIAL builds the spatial-split tree on the host (seconds
// for large soups; for scenes that stay resident).
enum BvhBuilder : int {
  BVH_BUILD_AUTO = 0,
  BVH_BUILD_HOST = 1,
  BVH_BUILD_DEVICE = 2,
  BVH_BUILD_DEVICE_PLOC = 3,
  BVH_BUILD_HOST_SPATIAL = 4
};
constexpr uint64_t kAutoDeviceBuildTris = 16384;
// build_scene_image + commit_scene, with the BVH built where `builder`
// says (`stream`: the device build's stream). A device-built tree deeper
// than the traversal stacks allow is rebuilt on the host.
std::string upload_scene(const pt_scene_desc &desc, SceneHost &out, bool &oom, int builder = BVH_BUILD_HOST,
                         cudaStream_t stream = nullptr, HostStaging *staging = nullptr);
void release_scene(SceneHost &s);
// An animated frame of a resident scene with the same draw items and
// triangle counts: the new host image (no BVH) replaces the scene arena, the
// tree keeps its structure and is refitted on the device
// (device_refit_bvh). upload_seconds then holds: host image, arena copy,
// refit, total.
std::string refit_scene(const pt_scene_desc &desc, SceneHost &sc, bool &oom, cudaStream_t stream,
                        HostStaging *staging);
// Records rewritten from the scene's positions and both node layouts'
// bounds recomputed bottom up (bvh_refit.cu); `records` triangle records.
std::string device_refit_bvh(SceneHost &sc, uint64_t records, cudaStream_t stream);
struct EnvHost {
  DevEnv dev{};
  DevEnv *d_desc = nullptr;
  DeviceArena arena;
};
// Builds the environment's CDFs and uploads them (stream-ordered when
// `stream` is non-null).
std::string upload_env(const pt_environment &env, EnvHost &out, bool &oom, cudaStream_t stream = nullptr);
void release_env(EnvHost &e);

// Host-built tables the kernels read (sheen albedo, sRGB thresholds).
void host_sheen_lut(float out[512]);
void host_srgb_thresholds(float out[255]);
float host_srgb_to_linear(float c);

}  // namespace ptd
