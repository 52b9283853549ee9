// Kernels of the plain (one path per thread) schedule, the in-order f64
// accumulator, the resolve kernels and the test hooks.
#include <algorithm>
#include <cstdio>

#include "dev_integrator.cuh"
#include "kernels.h"
#include "wavefront.cuh"

namespace ptd {

__device__ float g_srgb_thresh[255];  // srgb_to_linear((k + 0.5) / 255)

PT_DEV const WaveSegment &find_segment(const WaveSegment *segs, uint32_t nseg, uint32_t slot) {
  uint32_t lo = 0, hi = nseg;
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (segs[mid].slot_begin <= slot)
      lo = mid;
    else
      hi = mid;
  }
  return segs[lo];
}

PT_DEV void slot_pixel(const DevRequest &rq, const WaveSegment &seg, uint32_t slot, uint32_t &x, uint32_t &y,
                       uint32_t &index) {
  uint32_t local = slot - seg.slot_begin;
  uint32_t s = local / seg.pixel_count, i = local - s * seg.pixel_count;
  uint32_t p = seg.pixel_begin + i;
  y = p / rq.width;
  x = p - y * rq.width;
  index = seg.sample_begin + s;
}

struct ImmediateSink {
  const DevRequest *rq;
  PathState *ps;
  ThreadStats *ts;
  PT_DEV void emit(const ShadowRay &sr) {
    if (trace_shadow(*rq, *ps, sr, *ts)) ps->radiance = vadd(ps->radiance, sr.contrib);
  }
};

// One thread traces one (pixel, sample) path to the end.
__global__ void __launch_bounds__(128, 3) k_megakernel(const DevRequest *reqs, const WaveSegment *segs, uint32_t nseg,
                                                    uint32_t total, float4 *out, DevCounters *ctr) {
  uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
  ThreadStats ts{0, 0, 0, 0, 0, 0, 0};
  if (slot < total) {
    const WaveSegment &seg = find_segment(segs, nseg, slot);
    const DevRequest &rq = reqs[seg.request];
    uint32_t x, y, index;
    slot_pixel(rq, seg, slot, x, y, index);
    PathState ps;
    init_path(rq, x, y, index, ps);
    ImmediateSink sink{&rq, &ps, &ts};
    for (;;) {
      Hit h;
      bool found = trace_extension(rq, ps, h, ts);
      if (!shade(rq, ps, found, h, sink)) break;
    }
    out[slot] = path_result(ps);
  }
  flush_stats(ctr, ts);
}

// accum[p] += covered samples of pixel p in sample order (f64, as the
// reference's refine loop adds them, src/pathtrace.rs:2569-2578).
__global__ void k_accumulate(const DevRequest *reqs, const WaveSegment *segs, const float4 *out) {
  const WaveSegment &seg = segs[blockIdx.y];
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= seg.pixel_count) return;
  const DevRequest &rq = reqs[seg.request];
  double4 *acc = reinterpret_cast<double4 *>(rq.accum) + seg.pixel_begin + i;
  double4 a = *acc;
  const float4 *src = out + seg.slot_begin + i;
  for (uint32_t s = 0; s < seg.spp; ++s) {
    float4 v = src[(size_t)s * seg.pixel_count];
    if (v.w > 0.0f) {
      // Non-finite radiance counts as a covered black sample (src/pathtrace.rs:2324-2328).
      if (!(isfinite(v.x) && isfinite(v.y) && isfinite(v.z))) v = make_float4(0.0f, 0.0f, 0.0f, v.w);
      a.x += (double)v.x;
      a.y += (double)v.y;
      a.z += (double)v.z;
      a.w += 1.0;
    }
  }
  *acc = a;
}

// ---------------------------------------------------------------- resolve
PT_DEV bool resolve_pixel(const double *a, uint32_t samples, float4 bg, float m_out[3], float &f) {
  if (a[3] <= 0.0 || samples == 0) return false;
  m_out[0] = (float)(a[0] / a[3]);
  m_out[1] = (float)(a[1] / a[3]);
  m_out[2] = (float)(a[2] / a[3]);
  f = (float)clampd(a[3] / (double)samples, 0.0, 1.0);
  return true;
}
PT_DEV float4 mix_bg(const float c[3], float f, float4 bg) {
  float a_sum = f + (1.0f - f) * bg.w;
  if (a_sum > 0.0f)
    return make_float4((f * c[0] + (1.0f - f) * bg.x * bg.w) / a_sum, (f * c[1] + (1.0f - f) * bg.y * bg.w) / a_sum,
                       (f * c[2] + (1.0f - f) * bg.z * bg.w) / a_sum, a_sum);
  return make_float4(f * c[0] + (1.0f - f) * bg.x, f * c[1] + (1.0f - f) * bg.y, f * c[2] + (1.0f - f) * bg.z, 0.0f);
}
PT_DEV float sanitize(float v) { return isnan(v) ? 0.0f : v; }
PT_DEV float aces(float x) {
  x = x * 0.6f;
  float v = (x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f);
  return clampr(v, 0.0f, 1.0f);
}
// ToneMap::apply, src/hdr.rs:44-67.
PT_DEV void tone_apply(uint32_t tm, float c[3]) {
  float r = fmaxf(sanitize(c[0]), 0.0f), g = fmaxf(sanitize(c[1]), 0.0f), b = fmaxf(sanitize(c[2]), 0.0f);
  if (tm == PT_TONE_REINHARD) {
    float l = 0.2126f * r + 0.7152f * g + 0.0722f * b;
    if (l <= 0.0f) {
      c[0] = c[1] = c[2] = 0.0f;
      return;
    }
    float s = 1.0f / (1.0f + l);
    c[0] = fminf(r * s, 1.0f);
    c[1] = fminf(g * s, 1.0f);
    c[2] = fminf(b * s, 1.0f);
  } else if (tm == PT_TONE_ACES) {
    c[0] = aces(r);
    c[1] = aces(g);
    c[2] = aces(b);
  } else {
    c[0] = fminf(r, 1.0f);
    c[1] = fminf(g, 1.0f);
    c[2] = fminf(b, 1.0f);
  }
}
// linear_to_srgb_byte, src/hdr.rs:116-129 (partition point over the thresholds).
PT_DEV uint8_t srgb_byte(float c) {
  if (isnan(c)) return 0;
  uint32_t lo = 0, hi = 255;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (g_srgb_thresh[mid] <= c)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (uint8_t)lo;
}

}  // namespace ptd

#include "raycast.cuh"
#include "raycast_pbr.cuh"

namespace ptd {

// PathTracer::hdr, src/pathtrace.rs:2717-2734.
__global__ void k_resolve_hdr(const double *accum, uint32_t n, uint32_t samples, float4 bg, float4 *out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 a4 = reinterpret_cast<const double4 *>(accum)[i];
  double a[4] = {a4.x, a4.y, a4.z, a4.w};
  float m[3], f;
  if (!resolve_pixel(a, samples, bg, m, f)) {
    out[i] = bg;
    return;
  }
  out[i] = f >= 1.0f ? make_float4(m[0], m[1], m[2], 1.0f) : mix_bg(m, f, bg);
}

// PathTracer::image, src/pathtrace.rs:2687-2713.
__global__ void k_resolve_image(const double *accum, uint32_t n, uint32_t samples, float4 bg, uchar4 bg_bytes,
                                uint32_t tone_map, float exposure, uchar4 *out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 a4 = reinterpret_cast<const double4 *>(accum)[i];
  double a[4] = {a4.x, a4.y, a4.z, a4.w};
  float m[3], f;
  if (!resolve_pixel(a, samples, bg, m, f)) {
    out[i] = bg_bytes;
    return;
  }
  float c[3] = {m[0] * exposure, m[1] * exposure, m[2] * exposure};
  tone_apply(tone_map, c);
  float4 r = f >= 1.0f ? make_float4(c[0], c[1], c[2], 1.0f) : mix_bg(c, f, bg);
  out[i] = make_uchar4(srgb_byte(r.x), srgb_byte(r.y), srgb_byte(r.z),
                       (uint8_t)f2u32(roundf(clampr(r.w, 0.0f, 1.0f) * 255.0f)));
}

// ---------------------------------------------------------------- test hooks
__global__ void k_debug_sobol(uint32_t n, uint32_t seed, float4 *out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float v[4];
  sobol_owen_4d(i, seed, v);
  out[i] = make_float4(v[0], v[1], v[2], v[3]);
}

// Pattern `pattern` of sample `index` for every pixel of the request.
__global__ void k_debug_pattern(const DevRequest *rq, uint32_t index, uint32_t pattern, float4 *out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rq->width * rq->height) return;
  Sampler smp;
  smp.init(rq->seed, i % rq->width, i / rq->width, index);
  float v[4];
  smp.pattern(pattern, v);
  out[i] = make_float4(v[0], v[1], v[2], v[3]);
}

// Primary hit (k = 0 acceptance) of sample `index` for every pixel.
__global__ void k_debug_primary(const DevRequest *rq, uint32_t index, uint32_t *out_g, float4 *out_tb,
                                DevCounters *ctr) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  ThreadStats ts{0, 0, 0, 0, 0, 0, 0};
  if (i < rq->width * rq->height) {
    PathState ps;
    init_path(*rq, i % rq->width, i / rq->width, index, ps);
    Hit h;
    if (trace_extension(*rq, ps, h, ts)) {
      out_g[i] = h.g;
      out_tb[i] = make_float4(h.t, h.b0, h.b1, h.b2);
    } else {
      out_g[i] = 0xffffffffu;
      out_tb[i] = make_float4(inf(), 0.0f, 0.0f, 0.0f);
    }
  }
  flush_stats(ctr, ts);
}

PT_DEV MaterialSample ms_from(const float *a) {
  MaterialSample m;
  for (int k = 0; k < 4; ++k) m.base_color[k] = a[k];
  m.metallic = a[4];
  m.roughness = a[5];
  m.normal = {a[6], a[7], a[8]};
  m.specular = a[9];
  m.specular_color = {a[10], a[11], a[12]};
  m.transmission = a[13];
  m.thickness = a[14];
  m.ior = a[15];
  m.clearcoat = a[16];
  m.clearcoat_roughness = a[17];
  m.clearcoat_normal = {a[18], a[19], a[20]};
  m.sheen_color = {a[21], a[22], a[23]};
  m.sheen_roughness = a[24];
  m.anisotropy = a[25];
  m.anisotropy_direction = {a[26], a[27], a[28]};
  m.iridescence = a[29];
  m.iridescence_ior = a[30];
  m.iridescence_thickness = a[31];
  m.diffuse_transmission = a[32];
  m.diffuse_transmission_color = {a[33], a[34], a[35]};
  m.emissive = vzero();
  m.unlit = 0;
  m.double_sided = 0;
  m.attenuation_color = {1.0f, 1.0f, 1.0f};
  m.attenuation_distance = inf();
  m.dispersion = 0.0f;
  return m;
}

// BSDF eval of n directions and BSDF sampling of n lobe triples
// (params: 36 MaterialSample floats, v, ng, front).
__global__ void k_debug_bsdf(const float *params, const float *dirs, const float *us, uint32_t n, float *out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  MaterialSample m = ms_from(params);
  Bsdf b;
  b.init(m, {params[36], params[37], params[38]}, {params[39], params[40], params[41]}, params[42] != 0.0f);
  V3 f;
  float pdf;
  b.eval({dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]}, f, pdf);
  float *o = out + 12 * i;
  o[0] = f.x;
  o[1] = f.y;
  o[2] = f.z;
  o[3] = pdf;
  V3 l, fs;
  float ps;
  bool ok = b.sample(us + 3 * i, l, fs, ps);
  o[4] = ok ? 1.0f : 0.0f;
  o[5] = ok ? l.x : 0.0f;
  o[6] = ok ? l.y : 0.0f;
  o[7] = ok ? l.z : 0.0f;
  o[8] = ok ? fs.x : 0.0f;
  o[9] = ok ? fs.y : 0.0f;
  o[10] = ok ? fs.z : 0.0f;
  o[11] = ok ? ps : 0.0f;
}

// ---------------------------------------------------------------- launchers
#define LAUNCH_CHECK() cudaGetLastError()

cudaError_t set_tables(const float *sheen_lut, const float *srgb_thresh) {
  cudaError_t e = cudaMemcpyToSymbol(g_sheen_lut, sheen_lut, sizeof(float) * SHEEN_LUT_COS * SHEEN_LUT_ROUGH);
  if (e != cudaSuccess) return e;
  return cudaMemcpyToSymbol(g_srgb_thresh, srgb_thresh, sizeof(float) * 255);
}

cudaError_t launch_megakernel(const DevRequest *reqs, const WaveSegment *segs, uint32_t nseg, uint32_t total,
                              float4 *out, DevCounters *ctr, cudaStream_t st) {
  if (total == 0) return cudaSuccess;
  k_megakernel<<<(total + 127) / 128, 128, 0, st>>>(reqs, segs, nseg, total, out, ctr);
  return LAUNCH_CHECK();
}
// One wave of the wavefront schedule: raygen, then `w.iterations` rounds of
// extend / shade / shadow over device-side queue counters (no host sync).
// The traversal kernels are persistent: exactly the blocks that fit at once
// (occupancy queried once, outside any stream capture).
// Index [t][o]: t = 0 the 256-thread instantiations, 1 the 128-thread ones;
// o = 1 the four-child-only ones.
void persistent_blocks(int per_sm_ext[2][2], int per_sm_sh[2][2]) {
  static int ext[2][2] = {}, sh[2][2] = {};
  if (ext[0][0] == 0) {
    // The traversal kernels are register-bound at 1,024 threads per SM and
    // need shared memory only for their short stacks: ask for the smallest
    // shared-memory carveout that holds those blocks, so the rest of the
    // SM's on-chip memory serves as L1 for nodes and triangle records (the
    // default carveout left 102 KB of shared memory for 37 KB of stacks;
    // the 64 KB configuration traced the request mix 1 % faster).
    int dev = 0, smem_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess)
      smem_sm = 0;
    cudaGetLastError();
    auto q = [smem_sm](int &v, const void *fn, int threads) {
      if (smem_sm > 0) {
        const long need = (1024L / threads) * ((long)kShortStack * threads * (long)sizeof(int) + 1024L);
        const int pct = (int)std::min(100L, (need * 100L + smem_sm - 1) / smem_sm + 1);
        if (cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, pct) != cudaSuccess)
          cudaGetLastError();
      }
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, fn, threads, 0) != cudaSuccess || v < 1) v = 1;
    };
    q(ext[0][0], (const void *)k_wf_extend<256, false>, 256);
    q(ext[0][1], (const void *)k_wf_extend<256, true>, 256);
    q(sh[0][0], (const void *)k_wf_shadow<256, false>, 256);
    q(sh[0][1], (const void *)k_wf_shadow<256, true>, 256);
    q(ext[1][0], (const void *)k_wf_extend<128, false>, 128);
    q(ext[1][1], (const void *)k_wf_extend<128, true>, 128);
    q(sh[1][0], (const void *)k_wf_shadow<128, false>, 128);
    q(sh[1][1], (const void *)k_wf_shadow<128, true>, 128);
  }
  for (int t = 0; t < 2; ++t)
    for (int o = 0; o < 2; ++o) {
      per_sm_ext[t][o] = ext[t][o];
      per_sm_sh[t][o] = sh[t][o];
    }
}

// The traversal launches of one bounce iteration: block size and node
// layout choose the instantiation.
template <int kThreads>
void launch_extend(const WaveBuffers &w, uint32_t it, DevCounters *ctr, uint32_t grid, bool only4, cudaStream_t st) {
  if (only4)
    k_wf_extend<kThreads, true><<<grid, kThreads, 0, st>>>(w, it, ctr);
  else
    k_wf_extend<kThreads, false><<<grid, kThreads, 0, st>>>(w, it, ctr);
}
template <int kThreads>
void launch_shadow(const WaveBuffers &w, uint32_t it, DevCounters *ctr, uint32_t grid, bool only4, cudaStream_t st) {
  if (only4)
    k_wf_shadow<kThreads, true><<<grid, kThreads, 0, st>>>(w, it, ctr);
  else
    k_wf_shadow<kThreads, false><<<grid, kThreads, 0, st>>>(w, it, ctr);
}

cudaError_t launch_wavefront(const WaveBuffers &w, DevCounters *ctr, int num_sms, cudaStream_t st,
                             StageTimer *timer, bool accumulate) {
  StageTimer none;
  StageTimer &tm = timer ? *timer : none;
  cudaError_t e = cudaMemsetAsync(w.counters, 0, sizeof(uint32_t) * kWfCounterStride * (w.iterations + 1), st);
  if (e == cudaSuccess && w.sort_materials)
    e = cudaMemsetAsync(w.sort_counts, 0, sizeof(uint32_t) * 2 * kSortBuckets * (w.iterations + 1), st);
  if (e != cudaSuccess) return e;
  int per_sm_ext[2][2], per_sm_sh[2][2];
  persistent_blocks(per_sm_ext, per_sm_sh);
  const bool shade4 = w.shade_blocks == 4;
  const bool t128 = w.trav_threads == 128;
  const bool ext4 = (w.all_wide & WIDE_EXTENSION) != 0, sh4 = (w.all_wide & WIDE_SHADOW) != 0;
  const uint32_t g_ext = (uint32_t)(num_sms * per_sm_ext[t128 ? 1 : 0][ext4 ? 1 : 0]),
                 g_shade = (uint32_t)num_sms * (shade4 ? 8 : 6),
                 g_sh = (uint32_t)(num_sms * per_sm_sh[t128 ? 1 : 0][sh4 ? 1 : 0]), g_wide = (uint32_t)num_sms * 16,
                 g_nee = (uint32_t)num_sms * 8;
  tm.mark(STAGE_RAYGEN, st);
  k_wf_raygen<<<g_wide, 256, 0, st>>>(w);
  for (uint32_t it = 0; it < w.iterations; ++it) {
    tm.mark(STAGE_EXTEND, st);
    if (t128)
      launch_extend<128>(w, it, ctr, g_ext, ext4, st);
    else
      launch_extend<256>(w, it, ctr, g_ext, ext4, st);
    if (w.sort_materials) {
      tm.mark(STAGE_SORT, st);
      k_wf_sort_count<<<g_shade, 256, 0, st>>>(w, it);
      k_wf_sort_scan<<<1, kSortBuckets, 0, st>>>(w, it);
      k_wf_sort_scatter<<<g_shade, 256, 0, st>>>(w, it);
    }
    tm.mark(STAGE_NEE, st);
    k_wf_nee<<<g_nee, 256, 0, st>>>(w, it);
    tm.mark(STAGE_SHADE, st);
    if (shade4)
      k_wf_shade<4><<<g_shade, 128, 0, st>>>(w, it);
    else
      k_wf_shade<3><<<g_shade, 128, 0, st>>>(w, it);
    tm.mark(STAGE_SHADOW, st);
    if (t128)
      launch_shadow<128>(w, it, ctr, g_sh, sh4, st);
    else
      launch_shadow<256>(w, it, ctr, g_sh, sh4, st);
    k_wf_shadow_add<<<g_wide, 256, 0, st>>>(w, it);
  }
  if (accumulate) {
    tm.mark(STAGE_ACCUMULATE, st);
    k_wf_accumulate<<<g_wide, 256, 0, st>>>(w);
  }
  return LAUNCH_CHECK();
}

cudaError_t launch_wave_accumulate(const WaveBuffers &w, int num_sms, cudaStream_t st) {
  k_wf_accumulate<<<(unsigned)num_sms * 16, 256, 0, st>>>(w);
  return LAUNCH_CHECK();
}

cudaError_t capture_wavefront(const WaveBuffers &w, DevCounters *ctr, int num_sms, cudaGraphExec_t *out,
                              bool accumulate) {
  *out = nullptr;
  int a[2][2], b[2][2];
  persistent_blocks(a, b);
  cudaStream_t cs = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (e != cudaSuccess) return e;
  cudaGraph_t g = nullptr;
  e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    cudaError_t le = launch_wavefront(w, ctr, num_sms, cs, nullptr, accumulate);
    e = cudaStreamEndCapture(cs, &g);
    if (e == cudaSuccess) e = le;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(out, g, 0);
  if (g) cudaGraphDestroy(g);
  cudaStreamDestroy(cs);
  return e;
}

cudaError_t launch_accumulate(const DevRequest *reqs, const WaveSegment *segs, uint32_t nseg, uint32_t max_pixels,
                              const float4 *out, cudaStream_t st) {
  if (nseg == 0 || max_pixels == 0) return cudaSuccess;
  dim3 grid((max_pixels + 255) / 256, nseg);
  k_accumulate<<<grid, 256, 0, st>>>(reqs, segs, out);
  return LAUNCH_CHECK();
}
cudaError_t launch_resolve_hdr(const double *accum, uint32_t n, uint32_t samples, float4 bg, float4 *out,
                               cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_resolve_hdr<<<(n + 255) / 256, 256, 0, st>>>(accum, n, samples, bg, out);
  return LAUNCH_CHECK();
}
cudaError_t launch_resolve_image(const double *accum, uint32_t n, uint32_t samples, float4 bg, uchar4 bg_bytes,
                                 uint32_t tone_map, float exposure, uchar4 *out, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_resolve_image<<<(n + 255) / 256, 256, 0, st>>>(accum, n, samples, bg, bg_bytes, tone_map, exposure, out);
  return LAUNCH_CHECK();
}
cudaError_t launch_debug_sobol(uint32_t n, uint32_t seed, float4 *out, cudaStream_t st) {
  k_debug_sobol<<<(n + 255) / 256, 256, 0, st>>>(n, seed, out);
  return LAUNCH_CHECK();
}
cudaError_t launch_debug_pattern(const DevRequest *rq, uint32_t npix, uint32_t index, uint32_t pattern, float4 *out,
                                 cudaStream_t st) {
  k_debug_pattern<<<(npix + 255) / 256, 256, 0, st>>>(rq, index, pattern, out);
  return LAUNCH_CHECK();
}
cudaError_t launch_debug_primary(const DevRequest *rq, uint32_t npix, uint32_t index, uint32_t *out_g, float4 *out_tb,
                                 DevCounters *ctr, cudaStream_t st) {
  k_debug_primary<<<(npix + 127) / 128, 128, 0, st>>>(rq, index, out_g, out_tb, ctr);
  return LAUNCH_CHECK();
}
cudaError_t launch_debug_bsdf(const float *params, const float *dirs, const float *us, uint32_t n, float *out,
                              cudaStream_t st) {
  k_debug_bsdf<<<(n + 127) / 128, 128, 0, st>>>(params, dirs, us, n, out);
  return LAUNCH_CHECK();
}

// RenderBackend::Raycast: trace every render sample, then resolve.
cudaError_t launch_raycast(const DevScene &s, const pt_camera &cam, uint32_t rw, uint32_t rh, uint32_t mode,
                           uint32_t max_depth, const float light_dir[3], float light_intensity, float near_plane,
                           float far_plane, const float decode[256], float4 *samples, uint8_t *covered,
                           uint32_t *err, int num_sms, cudaStream_t st) {
  RaycastParams p;
  p.s = s;
  p.cam = cam;
  p.rw = rw;
  p.rh = rh;
  p.mode = mode;
  p.max_depth = max_depth < kRayDepthCap ? max_depth : kRayDepthCap;
  p.light_dir = {light_dir[0], light_dir[1], light_dir[2]};
  p.light_intensity = light_intensity;
  p.near_plane = near_plane;
  p.far_plane = far_plane;
  for (int k = 0; k < 256; ++k) p.decode[k] = decode[k];
  p.samples = samples;
  p.covered = covered;
  p.err = err;
  const uint64_t n = (uint64_t)rw * rh;
  const uint64_t blocks = std::min<uint64_t>((n + 127) / 128, (uint64_t)num_sms * 16);
  k_raycast<<<(unsigned)std::max<uint64_t>(blocks, 1), 128, 0, st>>>(p);
  return cudaGetLastError();
}

size_t raycast_pbr_frame_bytes() { return sizeof(PbrFrame) * (size_t)kPbrDeepFrames; }

cudaError_t launch_raycast_pbr(const DevScene &s, const pt_camera &cam, uint32_t rw, uint32_t rh, uint32_t max_depth,
                               bool shadows, float ambient, float cutoff, float spread, float4 bg, float4 *samples,
                               uint8_t *covered, uint32_t *err, uint32_t *ovf_list, uint32_t *ovf_count, void *deep,
                               uint32_t deep_slots, int num_sms, cudaStream_t st) {
  PbrParams p;
  p.s = s;
  p.cam = cam;
  p.rw = rw;
  p.rh = rh;
  p.max_depth = max_depth < kRayDepthCap ? max_depth : kRayDepthCap;
  p.shadows = shadows ? 1u : 0u;
  p.ambient = ambient;
  p.cutoff = cutoff;
  p.spread = spread;
  p.bg = bg;
  p.samples = samples;
  p.covered = covered;
  p.err = err;
  p.ovf_list = ovf_list;
  p.ovf_count = ovf_count;
  p.deep = static_cast<PbrFrame *>(deep);
  p.deep_slots = deep_slots;
  const uint64_t n = (uint64_t)rw * rh;
  const uint64_t blocks = std::min<uint64_t>((n + 127) / 128, (uint64_t)num_sms * 16);
  k_raycast_pbr<<<(unsigned)std::max<uint64_t>(blocks, 1), 128, 0, st>>>(p);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_raycast_pbr_deep<<<(deep_slots + 63) / 64, 64, 0, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_raycast_resolve(const float4 *samples, const uint8_t *covered, uint32_t out_w, uint32_t out_h,
                                   uint32_t aa, float4 bg, uint32_t tone, float exposure, float4 *hdr, uchar4 *rgba,
                                   cudaStream_t st) {
  const uint64_t n = (uint64_t)out_w * out_h;
  const unsigned blocks = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 1u << 16));
  k_raycast_resolve<<<blocks, 256, 0, st>>>(samples, covered, out_w, out_h, aa, bg, tone, exposure, hdr, rgba);
  return cudaGetLastError();
}

}  // namespace ptd
