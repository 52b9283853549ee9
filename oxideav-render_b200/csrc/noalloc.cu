// pt_refine_noalloc: the refine pass for callers that must not allocate
// device memory during a call.
//
// Who needs it: hosts that own every device allocation themselves — a
// render loop with a frame-time budget that forbids cudaMalloc / cudaFree
// (both can synchronise the whole device), an engine or plugin host whose
// memory all comes from its own pool allocator, or code running where a
// hidden allocation would break the caller's memory accounting. Such a
// caller allocates the accumulator itself and passes it in; the path
// samples of each wave go to a fixed scratch array compiled into this
// library instead of the context's growable wave buffer.
//
// The scratch is a file-scope `static __device__` array of
// kNoAllocSlots path slots (16 MiB of samples plus a few hundred bytes of
// launch descriptors). Every GPU that loads the library holds it until the
// process exits. Each call overwrites it; calls that overlap on the GPU
// (two contexts, or two threads, on the same device at the same time) race
// on it and must be serialised by the caller.
//
// The samples are traced by the one-launch megakernel schedule: the
// wavefront's path-state arenas are far larger than a fixed scratch can
// hold. Images are identical to pt_tracer_refine's (whose default is the
// wavefront), but the speed is the megakernel's, and the context's schedule
// and tuned per-class knobs are not consulted here.
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdint>
#include <mutex>
#include <new>
#include <string>

#include "context.h"
#include "kernels.h"

namespace {

// Path slots of the static scratch: one wave holds at most this many
// (pixel, sample) paths, so images up to this many pixels are accepted.
constexpr uint32_t kNoAllocSlots = 1u << 20;
constexpr int kMaxDevices = 64;

struct NoAllocScratch {
  ptd::DevRequest request;
  ptd::WaveSegment segment;
  ptd::DevCounters counters;
  float4 samples[kNoAllocSlots];
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

std::mutex g_setup_mu;
NoAllocScratch *g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch on the current device (looked up once per
// device; host code cannot use the symbol itself as a device pointer).
cudaError_t scratch_address(int device, NoAllocScratch **out) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_addr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[device] = static_cast<NoAllocScratch *>(p);
  }
  *out = g_scratch_addr[device];
  return cudaSuccess;
}

// The caller's accumulator must be device (or managed) memory of this
// context's device, 16-byte aligned (the accumulate kernel reads and writes
// it as double4), and lie wholly inside one allocation of at least `bytes`
// from `p`: a kernel given anything else would fault on a shared GPU.
// The allocation range comes from the driver (cuMemGetAddressRange, fetched
// through the runtime's entry-point query, so no libcuda link is needed).
std::string check_accumulator(int device, const void *p, uint64_t bytes) {
  if (reinterpret_cast<uintptr_t>(p) % 16 != 0) return "d_accum must be 16-byte aligned";
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return "d_accum is not a pointer the CUDA runtime knows";
  }
  if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
    return "d_accum must point to device (or managed) memory";
  if (a.type == cudaMemoryTypeDevice && a.device != device)
    return "d_accum belongs to device " + std::to_string(a.device) + ", the context to device " +
           std::to_string(device);
  static PFN_cuMemGetAddressRange_v3020 range_fn = [] {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuMemGetAddressRange", &fn, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      fn = nullptr;
    return reinterpret_cast<PFN_cuMemGetAddressRange_v3020>(fn);
  }();
  if (!range_fn) return "the driver does not report allocation ranges; d_accum cannot be checked";
  CUdeviceptr_v2 base = 0;
  size_t size = 0;
  const CUdeviceptr_v2 at = static_cast<CUdeviceptr_v2>(reinterpret_cast<uintptr_t>(p));
  if (range_fn(&base, &size, at) != CUDA_SUCCESS) return "d_accum is not inside a device allocation";
  if (at + bytes > base + size)
    return "d_accum holds " + std::to_string((base + size - at) / 32) + " pixels, the image needs " +
           std::to_string(bytes / 32);
  return std::string();
}

#define NA_CHECK(call)                                                                                     \
  do {                                                                                                     \
    cudaError_t e_ = (call);                                                                               \
    if (e_ != cudaSuccess)                                                                                 \
      return ptd::ctx_fail(ctx, PT_ERR_DEVICE, std::string(#call) + ": " + cudaGetErrorString(e_));       \
  } while (0)

pt_status refine_noalloc_impl(pt_context *ctx, uint32_t scene_id, const pt_camera *camera,
                              const pt_render_options *opts, uint32_t first_sample, uint32_t samples,
                              double *d_accum) {
  if (!camera || !opts || !d_accum) return ptd::ctx_fail(ctx, PT_ERR_INVALID_ARG, "camera / options / accum is NULL");
  if (opts->path_trace.max_bounces > 1024)
    return ptd::ctx_fail(ctx, PT_ERR_INVALID_ARG, "path_trace.max_bounces must be <= 1024");
  if (opts->path_trace.strategy > PT_BSDF_ONLY || camera->projection > PT_ORTHOGRAPHIC)
    return ptd::ctx_fail(ctx, PT_ERR_INVALID_ARG, "unknown light strategy or projection");
  if (ctx->device < 0 || ctx->device >= kMaxDevices)
    return ptd::ctx_fail(ctx, PT_ERR_INVALID_ARG, "device index out of range for pt_refine_noalloc");
  const uint32_t w = opts->width ? opts->width : 1u, h = opts->height ? opts->height : 1u;
  const uint64_t npix = (uint64_t)w * h;
  if (npix > kNoAllocSlots)
    return ptd::ctx_fail(ctx, PT_ERR_INVALID_ARG,
                         "pt_refine_noalloc: image has " + std::to_string(npix) +
                             " pixels; its static scratch holds at most " + std::to_string(kNoAllocSlots) +
                             " (use pt_tracer_refine for larger images)");
  ptd::SceneHost *sc = ptd::ctx_find_scene(ctx, scene_id);
  if (!sc) return ptd::ctx_fail(ctx, PT_ERR_NOT_FOUND, "unknown scene " + std::to_string(scene_id));
  if (samples == 0) return PT_OK;
  NA_CHECK(cudaSetDevice(ctx->device));
  const std::string bad = check_accumulator(ctx->device, d_accum, npix * 4 * sizeof(double));
  if (!bad.empty()) return ptd::ctx_fail(ctx, PT_ERR_INVALID_ARG, "pt_refine_noalloc: " + bad);
  NoAllocScratch *scratch = nullptr;
  NA_CHECK(scratch_address(ctx->device, &scratch));

  ptd::DevRequest rq{};
  rq.scene = sc->d_desc;
  rq.env = nullptr;
  rq.cam = *camera;
  rq.width = w;
  rq.height = h;
  rq.ambient = std::isfinite(opts->ambient) ? std::fmax(opts->ambient, 0.0f) : 0.0f;
  rq.pixel_spread = 2.0f * camera->half_h / (float)h;
  rq.orthographic = camera->projection == PT_ORTHOGRAPHIC ? 1u : 0u;
  rq.max_bounces = opts->path_trace.max_bounces;
  rq.rr_start = opts->path_trace.rr_start;
  rq.seed = opts->path_trace.seed;
  rq.strategy = opts->path_trace.strategy;
  rq.clamp = opts->path_trace.clamp;
  rq.p_env = 0.0f;
  rq.accum = d_accum;
  NA_CHECK(cudaMemcpyAsync(&scratch->request, &rq, sizeof rq, cudaMemcpyHostToDevice, ctx->stream));
  // The counters keep the previous call's totals: clear them.
  NA_CHECK(cudaMemsetAsync(&scratch->counters, 0, sizeof(ptd::DevCounters), ctx->stream));
  const uint32_t per_wave = (uint32_t)(kNoAllocSlots / npix);
  for (uint32_t done = 0; done < samples;) {
    uint32_t c = samples - done < per_wave ? samples - done : per_wave;
    ptd::WaveSegment seg{0, 0, 0, (uint32_t)npix, first_sample + done, c, 0, 0};
    // Pageable H2D copies are stream-ordered after the previous wave's kernels.
    NA_CHECK(cudaMemcpyAsync(&scratch->segment, &seg, sizeof seg, cudaMemcpyHostToDevice, ctx->stream));
    NA_CHECK(ptd::launch_megakernel(&scratch->request, &scratch->segment, 1, (uint32_t)npix * c, scratch->samples,
                                    &scratch->counters, ctx->stream));
    NA_CHECK(ptd::launch_accumulate(&scratch->request, &scratch->segment, 1, (uint32_t)npix, scratch->samples,
                                    ctx->stream));
    done += c;
  }
  ptd::DevCounters counters;
  NA_CHECK(cudaMemcpyAsync(&counters, &scratch->counters, sizeof counters, cudaMemcpyDeviceToHost, ctx->stream));
  NA_CHECK(cudaStreamSynchronize(ctx->stream));
  if (counters.error_flags & ptd::ERR_STACK_OVERFLOW)
    return ptd::ctx_fail(ctx, PT_ERR_DEVICE, "BVH traversal stack overflow");
  return PT_OK;
}
}  // namespace

extern "C" pt_status pt_refine_noalloc(pt_context *ctx, uint32_t scene_id, const pt_camera *camera,
                                       const pt_render_options *opts, uint32_t first_sample, uint32_t samples,
                                       double *d_accum) {
  if (!ctx) return PT_ERR_INVALID_ARG;
  // No exception crosses the C ABI.
  try {
    return refine_noalloc_impl(ctx, scene_id, camera, opts, first_sample, samples, d_accum);
  } catch (const std::bad_alloc &) {
    ctx->err = "host allocation failed";
    return PT_ERR_OOM;
  } catch (...) {
    return PT_ERR_DEVICE;
  }
}
