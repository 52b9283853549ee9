// Texture mip chains built on the device (src/texture.rs:324-383,
// build_mips): level 0 decoded from the uploaded source texels (sRGB
// through the 256-entry decode table for the colour chain, byte / 255 for
// the linear chain; f32 sources copied), then each level the 2x2 box
// average of the one above with clamped edges, summed in the same order as
// the host build (((0 + a) + b) + c) + d, then * 0.25) so the texels are
// bit-identical to it.
#include "mip_build.h"

namespace ptd {
namespace {

struct DecodeTable {
  float v[256];
};

__global__ void k_mip_level0(const DevTexture *tex, uint32_t ntex, const uint8_t *src, float4 *pool, DecodeTable lut) {
  const uint32_t ti = blockIdx.y;
  if (ti >= ntex) return;
  const DevTexture t = tex[ti];
  if (t.levels == 0) return;
  const uint64_t n = (uint64_t)t.img_w * t.img_h;
  float4 *s = pool + t.srgb_off[0], *l = pool + t.lin_off[0];
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    if (t.src_format == PT_PIXELS_RGBA8) {
      const uchar4 c = reinterpret_cast<const uchar4 *>(src + t.src_off)[i];
      const float a = (float)c.w / 255.0f;
      s[i] = make_float4(lut.v[c.x], lut.v[c.y], lut.v[c.z], a);
      l[i] = make_float4((float)c.x / 255.0f, (float)c.y / 255.0f, (float)c.z / 255.0f, a);
    } else {
      const float *p = reinterpret_cast<const float *>(src + t.src_off) + 4 * i;
      const float4 c = make_float4(p[0], p[1], p[2], p[3]);
      s[i] = c;
      l[i] = c;
    }
  }
}

__device__ __forceinline__ float4 box4(const float4 *prev, uint32_t pw, uint32_t ph, uint32_t x, uint32_t y) {
  const uint64_t x0 = min(2 * x, pw - 1), x1 = min(2 * x + 1, pw - 1);
  const uint64_t y0 = min(2 * y, ph - 1), y1 = min(2 * y + 1, ph - 1);
  const float4 q[4] = {prev[y0 * pw + x0], prev[y0 * pw + x1], prev[y1 * pw + x0], prev[y1 * pw + x1]};
  float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    a0 += q[k].x;
    a1 += q[k].y;
    a2 += q[k].z;
    a3 += q[k].w;
  }
  return make_float4(a0 * 0.25f, a1 * 0.25f, a2 * 0.25f, a3 * 0.25f);
}

__global__ void k_mip_level(const DevTexture *tex, uint32_t ntex, float4 *pool, uint32_t level) {
  const uint32_t ti = blockIdx.y;
  if (ti >= ntex) return;
  const DevTexture &t = tex[ti];
  if (level >= t.levels) return;
  const uint32_t pw = t.lw[level - 1], ph = t.lh[level - 1], w = t.lw[level], h = t.lh[level];
  const uint64_t n = (uint64_t)w * h;
  const float4 *ps = pool + t.srgb_off[level - 1], *pl = pool + t.lin_off[level - 1];
  float4 *s = pool + t.srgb_off[level], *l = pool + t.lin_off[level];
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t y = (uint32_t)(i / w), x = (uint32_t)(i - (uint64_t)y * w);
    s[i] = box4(ps, pw, ph, x, y);
    l[i] = box4(pl, pw, ph, x, y);
  }
}

}  // namespace

std::string device_build_mips(const std::vector<DevTexture> &host_tex, const DevTexture *d_tex, const uint8_t *d_src,
                              float4 *d_pool, const float decode[256], cudaStream_t st) {
  const uint32_t ntex = (uint32_t)host_tex.size();
  uint32_t max_levels = 0;
  uint64_t max_texels = 0;
  for (const DevTexture &t : host_tex) {
    max_levels = std::max(max_levels, t.levels);
    if (t.levels) max_texels = std::max<uint64_t>(max_texels, (uint64_t)t.img_w * t.img_h);
  }
  if (max_levels == 0) return "";
  DecodeTable lut;
  for (int k = 0; k < 256; ++k) lut.v[k] = decode[k];
  constexpr uint32_t kThreads = 256, kMaxY = 65535;
  for (uint32_t t0 = 0; t0 < ntex; t0 += kMaxY) {
    const uint32_t nt = std::min(ntex - t0, kMaxY);
    auto blocks = [&](uint64_t texels) {
      return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((texels + kThreads - 1) / kThreads, 4096));
    };
    k_mip_level0<<<dim3(blocks(max_texels), nt), kThreads, 0, st>>>(d_tex + t0, nt, d_src, d_pool, lut);
    uint64_t lvl_texels = max_texels;
    for (uint32_t k = 1; k < max_levels; ++k) {
      lvl_texels = std::max<uint64_t>(lvl_texels / 4, 1);
      k_mip_level<<<dim3(blocks(lvl_texels), nt), kThreads, 0, st>>>(d_tex + t0, nt, d_pool, k);
    }
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? std::string() : std::string("mip generation failed: ") + cudaGetErrorString(e);
}

}  // namespace ptd
