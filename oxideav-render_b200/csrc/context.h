// The context object behind the opaque pt_context handle, shared by the C
// entry points (capi.cpp, noalloc.cu).
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/pt_b200.h"
#include "../../include/pt_b200_debug.h"
#include "host_scene.h"

struct pt_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  std::map<uint32_t, std::unique_ptr<ptd::SceneHost>> scenes;
  uint32_t next_id = 1;
  uint32_t schedule = PT_SCHEDULE_MEGAKERNEL;
  uint32_t wave_slots = 1u << 22;
  float4 *d_out = nullptr;
  size_t out_cap = 0;
  ptd::WaveSegment *d_segs = nullptr;
  size_t seg_cap = 0;
  ptd::DevRequest *d_reqs = nullptr;  // requests of the running batch
  size_t req_cap = 0;
  float last_batch_ms = 0.0f;
  uint32_t last_batch_waves = 0;
  uint64_t last_batch_rays = 0;
  ptd::DevCounters *d_ctr = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int num_sms = 148;
  bool stage_timing = false;
  std::vector<cudaEvent_t> stage_events;
  // Wavefront schedule: one arena holding the SoA path state and queues.
  ptd::WaveBuffers wf{};
  void *wf_arena = nullptr;
  size_t wf_bytes = 0;
};

namespace ptd {
// Records `msg` as the context's last error and returns `st`.
pt_status ctx_fail(pt_context *ctx, pt_status st, const std::string &msg);
// The resident scene `id`, or nullptr.
SceneHost *ctx_find_scene(pt_context *ctx, uint32_t id);
}  // namespace ptd
