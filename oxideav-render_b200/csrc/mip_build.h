// Texture mip chains generated on the device at scene upload: the host
// image carries each texture's source texels; both chains (sRGB-decoded
// colour and linear data) of every level are written into the scene's
// texel pool by kernels.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "dev_types.h"

namespace ptd {

// Level sizes of a w x h texture's chain (halving, at least 1, down to 1x1).
inline uint32_t mip_levels(uint32_t w, uint32_t h, uint32_t *lw = nullptr, uint32_t *lh = nullptr,
                           uint32_t cap = 0) {
  uint32_t n = 0;
  for (;;) {
    if (lw && n < cap) {
      lw[n] = w;
      lh[n] = h;
    }
    ++n;
    if (w == 1 && h == 1) break;
    w = w / 2 > 1 ? w / 2 : 1;
    h = h / 2 > 1 ? h / 2 : 1;
  }
  return n;
}

// Fills every chain of `host_tex` (the same table the device holds at
// `d_tex`) from the sources at d_src + src_off into d_pool, on `st`.
// `decode` maps an sRGB byte to linear.
std::string device_build_mips(const std::vector<DevTexture> &host_tex, const DevTexture *d_tex, const uint8_t *d_src,
                              float4 *d_pool, const float decode[256], cudaStream_t st);

}  // namespace ptd
