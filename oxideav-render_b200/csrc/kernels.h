// Host-side declarations of the kernel launchers (kernels.cu, wavefront.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "dev_types.h"

namespace ptd {

// Optional per-stage CUDA events: mark(kind) records the next event of a
// caller-owned pool on the stream; consecutive events bracket one stage.
struct StageTimer {
  cudaEvent_t *events = nullptr;
  size_t capacity = 0;
  std::vector<int> kinds;
  size_t count() const { return kinds.size(); }
  void mark(int kind, cudaStream_t st) {
    if (!events || kinds.size() >= capacity) return;
    cudaEventRecord(events[kinds.size()], st);
    kinds.push_back(kind);
  }
};

cudaError_t set_tables(const float *sheen_lut, const float *srgb_thresh);
cudaError_t launch_megakernel(const DevRequest *reqs, const WaveSegment *segs, uint32_t nseg, uint32_t total,
                              float4 *out, DevCounters *ctr, cudaStream_t st);
// One wave of the wavefront schedule (counter reset, ray generation,
// `w.iterations` bounces, and unless `accumulate` is false the in-order
// accumulate), driven by the wave descriptor `w.desc` that the caller has
// written on `st` beforehand.
cudaError_t launch_wavefront(const WaveBuffers &w, DevCounters *ctr, int num_sms, cudaStream_t st,
                             StageTimer *timer = nullptr, bool accumulate = true);
// The in-order accumulate of a traced wave on its own (k_wf_accumulate).
cudaError_t launch_wave_accumulate(const WaveBuffers &w, int num_sms, cudaStream_t st);
// The same launch sequence captured once as an executable CUDA graph; it
// stays valid while `w`'s buffers, `ctr` and the bounce count are unchanged.
cudaError_t capture_wavefront(const WaveBuffers &w, DevCounters *ctr, int num_sms, cudaGraphExec_t *out,
                              bool accumulate = true);
cudaError_t launch_accumulate(const DevRequest *reqs, const WaveSegment *segs, uint32_t nseg, uint32_t max_pixels,
                              const float4 *out, cudaStream_t st);
cudaError_t launch_resolve_hdr(const double *accum, uint32_t n, uint32_t samples, float4 bg, float4 *out,
                               cudaStream_t st);
cudaError_t launch_resolve_image(const double *accum, uint32_t n, uint32_t samples, float4 bg, uchar4 bg_bytes,
                                 uint32_t tone_map, float exposure, uchar4 *out, cudaStream_t st);
cudaError_t launch_debug_sobol(uint32_t n, uint32_t seed, float4 *out, cudaStream_t st);
// RenderBackend::Raycast (raycast.cuh): one sample per render pixel
// (rw x rh), then the aa x aa box resolve into HDR and / or RGBA8.
cudaError_t launch_raycast(const DevScene &s, const pt_camera &cam, uint32_t rw, uint32_t rh, uint32_t mode,
                           uint32_t max_depth, const float light_dir[3], float light_intensity, float near_plane,
                           float far_plane, const float decode[256], float4 *samples, uint8_t *covered,
                           uint32_t *err, int num_sms, cudaStream_t st);
// ShadingMode::Pbr (raycast_pbr.cuh): every sample with a short frame stack,
// then the samples listed in ovf_list again with deep stacks (`deep` holds
// deep_slots * raycast_pbr_frame_bytes()).
size_t raycast_pbr_frame_bytes();
cudaError_t launch_raycast_pbr(const DevScene &s, const pt_camera &cam, uint32_t rw, uint32_t rh, uint32_t max_depth,
                               bool shadows, float ambient, float cutoff, float spread, float4 bg, float4 *samples,
                               uint8_t *covered, uint32_t *err, uint32_t *ovf_list, uint32_t *ovf_count, void *deep,
                               uint32_t deep_slots, int num_sms, cudaStream_t st);
cudaError_t launch_raycast_resolve(const float4 *samples, const uint8_t *covered, uint32_t out_w, uint32_t out_h,
                                   uint32_t aa, float4 bg, uint32_t tone, float exposure, float4 *hdr, uchar4 *rgba,
                                   cudaStream_t st);
cudaError_t launch_debug_pattern(const DevRequest *rq, uint32_t npix, uint32_t index, uint32_t pattern, float4 *out,
                                 cudaStream_t st);
cudaError_t launch_debug_primary(const DevRequest *rq, uint32_t npix, uint32_t index, uint32_t *out_g, float4 *out_tb,
                                 DevCounters *ctr, cudaStream_t st);
cudaError_t launch_debug_bsdf(const float *params, const float *dirs, const float *us, uint32_t n, float *out,
                              cudaStream_t st);

}  // namespace ptd
