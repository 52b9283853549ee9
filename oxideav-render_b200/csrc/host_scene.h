// Host-side scene preparation: BVH build, attribute streams, materials,
// texture mip chains, emissive-triangle table, environment CDFs, and the
// single device arena each resident scene lives in.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "dev_types.h"

namespace ptd {

struct BvhBuildStats {
  uint32_t nodes = 0, leaves = 0, max_depth = 0;
  double sah_cost = 0.0, seconds = 0.0;
};

// Binned-SAH BVH over the soup (positions: 9 floats per triangle), laid out
// as two-child 64-byte nodes plus 48-byte leaf-ordered triangle records.
// `rec_flags[g]` goes into each record (REC_* bits).
void build_bvh(const float *pos, uint32_t tri_count, const uint32_t *rec_flags, std::vector<BvhNode> &nodes,
               std::vector<float4> &records, BvhBuildStats &stats, int threads);

// One device allocation holding a scene (or an environment) plus the
// device copy of its descriptor.
struct DeviceArena {
  void *base = nullptr;
  uint64_t bytes = 0;
  void release();
};

struct SceneHost {
  DevScene dev{};           // pointers into `arena`
  DevScene *d_desc = nullptr;
  DeviceArena arena;
  uint64_t tri_count = 0;
  BvhBuildStats bvh;
  uint32_t light_count = 0;
};

// Validates `desc`, builds everything on the host and uploads it.
// Returns an empty string on success, else an error message
// (`oom` set when the failure was a device allocation).
std::string upload_scene(const pt_scene_desc &desc, SceneHost &out, bool &oom);
void release_scene(SceneHost &s);

struct EnvHost {
  DevEnv dev{};
  DevEnv *d_desc = nullptr;
  DeviceArena arena;
};
std::string upload_env(const pt_environment &env, EnvHost &out, bool &oom);
void release_env(EnvHost &e);

// Host-built tables the kernels read (sheen albedo, sRGB thresholds).
void host_sheen_lut(float out[512]);
void host_srgb_thresholds(float out[255]);
float host_srgb_to_linear(float c);

}  // namespace ptd
