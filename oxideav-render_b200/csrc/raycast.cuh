// RenderBackend::Raycast on the device: the Whitted ray tracer of
// src/raycast.rs (legacy shading modes, :382-516) over the scene's device
// BVH, and the scanline backend's frame resolve (src/scanline.rs:124-221).
//
// One thread per render sample traces the camera ray through the sample
// centre and shades it; Phong mode follows Whitted's recursion (a hard
// shadow ray toward the options' directional light, a mirror ray weighted
// by metallic·(1 − roughness) and Schlick's Fresnel, a refraction ray for
// KHR_materials_transmission) with an explicit frame stack of at most
// kRayDepthCap + 1 frames instead of device recursion, combining each
// child's colour into its parent in the reference's order. A second kernel
// box-filters the aa × aa samples of every output pixel and applies the
// display transform.
#pragma once

#include "dev_integrator.cuh"

namespace ptd {

constexpr uint32_t kRayDepthCap = 16;           // MAX_DEPTH_CAP, src/raycast.rs:121
constexpr float kLegacyAmbient = 0.2f;          // AMBIENT, src/shade.rs:13
constexpr float kSecondaryRayThreshold = 1.0e-2f;  // src/raycast.rs:130
constexpr float kWireframeEdge = 0.03f;          // src/raycast.rs:134

struct RaycastParams {
  DevScene s;
  pt_camera cam;
  uint32_t rw, rh, mode, max_depth;
  V3 light_dir;
  float light_intensity;
  float near_plane, far_plane;
  float decode[256];  // srgb_u8_lut: sRGB byte -> linear
  float4 *samples;     // rw * rh colours
  uint8_t *covered;    // rw * rh
  uint32_t *err;
};

struct AcceptAll {
  PT_DEV bool operator()(uint32_t, uint32_t, float, float, float, float, bool) const { return true; }
};
struct AcceptNotSelf {
  uint32_t skip;
  PT_DEV bool operator()(uint32_t g, uint32_t, float, float, float, float, bool) const { return g != skip; }
};

// shade_pixel, src/shade.rs:40-50: Lambert + constant ambient.
PT_DEV float4 shade_legacy(float4 base, V3 n, V3 l, float intensity) {
  float cos_theta = fmaxf(vdot(n, l), 0.0f);
  float diffuse = kLegacyAmbient + (1.0f - kLegacyAmbient) * cos_theta * intensity;
  float f = clampr(diffuse, 0.0f, 1.0f);
  return make_float4(base.x * f, base.y * f, base.z * f, base.w);
}

// reflect / refract / schlick, src/trace.rs:1087-1116.
PT_DEV V3 reflect_dir(V3 d, V3 n) {
  float k = 2.0f * vdot(d, n);
  return {d.x - k * n.x, d.y - k * n.y, d.z - k * n.z};
}
PT_DEV bool refract_dir(V3 d, V3 n, float eta, V3 &out) {
  float cos_i = clampr(-vdot(d, n), -1.0f, 1.0f);
  float sin2_t = eta * eta * (1.0f - cos_i * cos_i);
  if (sin2_t > 1.0f) return false;
  float cos_t = sqrtf(1.0f - sin2_t);
  float k = eta * cos_i - cos_t;
  out = vnormalise({eta * d.x + k * n.x, eta * d.y + k * n.y, eta * d.z + k * n.z});
  return true;
}
PT_DEV float schlick_scalar(float f0, float c) { return f0 + (1.0f - f0) * powi5(1.0f - clampr(c, 0.0f, 1.0f)); }

// normal_to_byte / depth_to_byte, src/scanline.rs:840-858.
PT_DEV uint32_t normal_byte(float n) {
  if (!isfinite(n)) return 128;
  float v = roundf((clampr(n, -1.0f, 1.0f) + 1.0f) * 0.5f * 255.0f);
  return (uint32_t)clampr(v, 0.0f, 255.0f);
}
PT_DEV uint32_t depth_byte(float z) {
  if (!isfinite(z)) return 0;
  float zc = clampr(z, -1.0f, 1.0f);
  float v = roundf((1.0f - (zc * 0.5f + 0.5f)) * 255.0f);
  return (uint32_t)clampr(v, 0.0f, 255.0f);
}

// Camera::ndc_z (src/camera.rs:521-538) of Camera::view_depth (:541-543).
PT_DEV float ndc_depth(const RaycastParams &p, V3 pos) {
  V3 eye = {p.cam.eye[0], p.cam.eye[1], p.cam.eye[2]}, fw = {p.cam.forward[0], p.cam.forward[1], p.cam.forward[2]};
  float vd = vdot(vsub(pos, eye), fw);
  const float nr = p.near_plane, fr = p.far_plane;
  if (p.cam.projection == PT_PERSPECTIVE) {
    float nf = 1.0f / (nr - fr);
    float d = fmaxf(vd, F32_MIN_POSITIVE);
    return -(fr + nr) * nf + 2.0f * fr * nr * nf / d;
  }
  float fne = fr - nr;
  if (fabsf(fne) < F32_EPSILON) return 0.0f;
  return (2.0f * vd - (fr + nr)) / fne;
}

PT_DEV V3 corner_normal(const DevScene &s, uint32_t g, int k) {
  if (s.nrm) return ld3(s.nrm + 9u * g + 3u * k);
  return surface(s, g, 1.0f / 3.0f, 1.0f / 3.0f, 1.0f / 3.0f, 0u).ng;
}
PT_DEV V3 hit_normal(const DevScene &s, const Hit &h) {
  if (s.nrm) return interp3(s.nrm, h.g, h.b0, h.b1, h.b2);
  return surface(s, h.g, h.b0, h.b1, h.b2, 0u).ng;
}

// One Whitted call: `whitted(d, hit, depth)` of src/raycast.rs:433-516.
struct WhittedFrame {
  V3 d, p, n;
  float4 out, a;
  uint32_t skip, depth;
  float kr, kt, ior, gloss;
  bool entering;
  uint8_t phase;    // 0: the mirror ray is next; 1: the transmission ray; 2: done
  uint8_t pending;  // what the child on top combines into: 1 mirror, 2 refraction, 3 total internal reflection
};

// Shades the frame's hit up to its secondary rays; false when the frame is
// already finished (unlit, or at the depth limit).
PT_DEV bool whitted_enter(const RaycastParams &p, WhittedFrame &f, V3 d, const Hit &h, uint32_t depth,
                          uint32_t &err) {
  const DevScene &s = p.s;
  const pt_material &m = s.materials[__ldg(s.tri_info + h.g).x].m;
  f.a = make_float4(m.base_color[0], m.base_color[1], m.base_color[2], m.base_color[3]);
  f.d = d;
  f.depth = depth;
  f.phase = 2;
  f.pending = 0;
  if (m.unlit) {
    f.out = f.a;
    return false;
  }
  V3 raw = vnormalise(hit_normal(s, h));
  f.entering = vdot(d, raw) < 0.0f;
  f.n = f.entering ? raw : V3{raw.x * -1.0f, raw.y * -1.0f, raw.z * -1.0f};
  f.p = interp3(s.pos, h.g, h.b0, h.b1, h.b2);
  f.skip = h.g;
  V3 so = offset_ray_origin(f.p, f.n);
  TraversalStats st{0, 0};
  bool shadowed = occluded(s, so, p.light_dir, 0.0f, inf(), AcceptNotSelf{f.skip}, st, err);
  f.out = shadowed ? make_float4(f.a.x * kLegacyAmbient, f.a.y * kLegacyAmbient, f.a.z * kLegacyAmbient, f.a.w)
                   : shade_legacy(f.a, f.n, p.light_dir, p.light_intensity);
  f.out.x += m.emissive[0];
  f.out.y += m.emissive[1];
  f.out.z += m.emissive[2];
  if (depth >= p.max_depth) return false;
  float cos_in = clampr(-vdot(d, f.n), 0.0f, 1.0f);
  f.gloss = m.metallic * (1.0f - m.roughness);
  f.kr = 0.0f;
  if (f.gloss > kSecondaryRayThreshold) {
    float f0 = 0.04f + 0.96f * m.metallic;
    f.kr = clampr(schlick_scalar(f0, cos_in), 0.0f, 1.0f) * f.gloss;
  }
  f.kt = (m.ext_flags & PT_EXT_TRANSMISSION) ? clampr(m.transmission_factor, 0.0f, 1.0f) : 0.0f;
  f.ior = m.ior;
  f.phase = 0;
  return true;
}

PT_DEV void whitted_combine(WhittedFrame &f, uint8_t how, float4 c) {
  if (how == 1) {
    f.out.x = f.out.x * (1.0f - f.kr) + c.x * f.a.x * f.kr;
    f.out.y = f.out.y * (1.0f - f.kr) + c.y * f.a.y * f.kr;
    f.out.z = f.out.z * (1.0f - f.kr) + c.z * f.a.z * f.kr;
  } else if (how == 2) {
    f.out.x = f.out.x * (1.0f - f.kt) + c.x * f.a.x * f.kt;
    f.out.y = f.out.y * (1.0f - f.kt) + c.y * f.a.y * f.kt;
    f.out.z = f.out.z * (1.0f - f.kt) + c.z * f.a.z * f.kt;
  } else if (how == 3) {
    f.out.x = f.out.x * (1.0f - f.kt) + c.x * f.kt;
    f.out.y = f.out.y * (1.0f - f.kt) + c.y * f.kt;
    f.out.z = f.out.z * (1.0f - f.kt) + c.z * f.kt;
  }
}

PT_DEV float4 whitted(const RaycastParams &p, V3 d0, const Hit &h0, uint32_t &err) {
  WhittedFrame fr[kRayDepthCap + 1];
  int top = 0;
  if (!whitted_enter(p, fr[0], d0, h0, 0, err)) return fr[0].out;
  for (;;) {
    WhittedFrame &f = fr[top];
    V3 o, dir;
    uint8_t how = 0;
    bool child = false;
    if (f.phase == 0) {
      f.phase = 1;
      if (f.gloss > kSecondaryRayThreshold) {
        o = offset_ray_origin(f.p, f.n);
        dir = reflect_dir(f.d, f.n);
        how = 1;
        child = true;
      }
    } else if (f.phase == 1) {
      f.phase = 2;
      if (f.kt > kSecondaryRayThreshold) {
        float eta = f.entering ? 1.0f / f.ior : f.ior;
        V3 t;
        if (refract_dir(f.d, f.n, eta, t)) {
          o = offset_ray_origin(f.p, V3{f.n.x * -1.0f, f.n.y * -1.0f, f.n.z * -1.0f});
          dir = t;
          how = 2;
        } else {
          o = offset_ray_origin(f.p, f.n);
          dir = reflect_dir(f.d, f.n);
          how = 3;
        }
        child = true;
      }
    } else {
      if (top == 0) return f.out;
      const float4 c = f.out;
      --top;
      whitted_combine(fr[top], fr[top].pending, c);
      continue;
    }
    if (!child) continue;
    Hit h;
    TraversalStats st{0, 0};
    if (!closest_hit(p.s, o, dir, 0.0f, inf(), AcceptNotSelf{f.skip}, h, st, err)) {
      // Escaping rays: black for the mirror ray, nothing through the
      // transmission, no change for total internal reflection.
      if (how == 1) whitted_combine(f, 1, make_float4(0.0f, 0.0f, 0.0f, 1.0f));
      if (how == 2) whitted_combine(f, 2, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
      continue;
    }
    f.pending = how;
    WhittedFrame &c = fr[top + 1];
    if (whitted_enter(p, c, dir, h, f.depth + 1, err)) {
      ++top;
    } else {
      whitted_combine(f, how, c.out);
    }
  }
}

// Ctx::pixel + Ctx::legacy, src/raycast.rs:349-431.
__global__ void __launch_bounds__(128) k_raycast(RaycastParams p) {
  const uint64_t n = (uint64_t)p.rw * p.rh;
  uint32_t err = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t y = (uint32_t)(i / p.rw), x = (uint32_t)(i - (uint64_t)y * p.rw);
    const float px = (float)x + 0.5f, py = (float)y + 0.5f;
    const float ndc_x = (px / fmaxf((float)p.rw, 1.0f)) * 2.0f - 1.0f;
    const float ndc_y = 1.0f - (py / fmaxf((float)p.rh, 1.0f)) * 2.0f;
    const V3 side = {p.cam.side[0], p.cam.side[1], p.cam.side[2]}, up = {p.cam.up[0], p.cam.up[1], p.cam.up[2]};
    const V3 fw = {p.cam.forward[0], p.cam.forward[1], p.cam.forward[2]};
    const V3 off = vadd(vscale(side, ndc_x * p.cam.half_w), vscale(up, ndc_y * p.cam.half_h));
    V3 o, d;
    if (p.cam.projection == PT_PERSPECTIVE) {
      o = {p.cam.eye[0], p.cam.eye[1], p.cam.eye[2]};
      d = vnormalise(vadd(off, fw));
    } else {
      o = vadd(V3{p.cam.eye[0], p.cam.eye[1], p.cam.eye[2]}, off);
      d = fw;
    }
    Hit h;
    TraversalStats st{0, 0};
    bool covered = closest_hit(p.s, o, d, 0.0f, inf(), AcceptAll{}, h, st, err);
    float4 c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (covered) {
      const pt_material &m = p.s.materials[__ldg(p.s.tri_info + h.g).x].m;
      const float4 base = make_float4(m.base_color[0], m.base_color[1], m.base_color[2], m.base_color[3]);
      switch (p.mode) {
        case PT_SHADE_FLAT:
          c = base;
          break;
        case PT_SHADE_WIREFRAME:
          if (fminf(fminf(fminf(INFINITY, h.b0), h.b1), h.b2) > kWireframeEdge)
            covered = false;
          else
            c = base;
          break;
        case PT_SHADE_GOURAUD: {
          float4 ca = shade_legacy(base, corner_normal(p.s, h.g, 0), p.light_dir, p.light_intensity);
          float4 cb = shade_legacy(base, corner_normal(p.s, h.g, 1), p.light_dir, p.light_intensity);
          float4 cc = shade_legacy(base, corner_normal(p.s, h.g, 2), p.light_dir, p.light_intensity);
          c = make_float4(ca.x * h.b0 + cb.x * h.b1 + cc.x * h.b2, ca.y * h.b0 + cb.y * h.b1 + cc.y * h.b2,
                          ca.z * h.b0 + cb.z * h.b1 + cc.z * h.b2, ca.w * h.b0 + cb.w * h.b1 + cc.w * h.b2);
          break;
        }
        case PT_SHADE_NORMAL_DEBUG: {
          V3 nn = vnormalise(hit_normal(p.s, h));
          c = make_float4(p.decode[normal_byte(nn.x)], p.decode[normal_byte(nn.y)], p.decode[normal_byte(nn.z)], 1.0f);
          break;
        }
        case PT_SHADE_DEPTH_DEBUG: {
          float g = p.decode[depth_byte(ndc_depth(p, interp3(p.s.pos, h.g, h.b0, h.b1, h.b2)))];
          c = make_float4(g, g, g, 1.0f);
          break;
        }
        default:
          c = whitted(p, d, h, err);
          break;
      }
    }
    p.samples[i] = covered ? c : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    p.covered[i] = covered ? 1 : 0;
  }
  if (err) atomicOr(p.err, err);
}

// Frame::resolve + to_rgba8 / to_hdr, src/scanline.rs:136-221.
__global__ void k_raycast_resolve(const float4 *samples, const uint8_t *covered, uint32_t out_w, uint32_t out_h,
                                  uint32_t aa, float4 bg, uint32_t tone, float exposure, float4 *hdr, uchar4 *rgba) {
  const uint64_t n = (uint64_t)out_w * out_h;
  const uint64_t rw = (uint64_t)out_w * aa;
  const float cnt = (float)(aa * aa);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t oy = (uint32_t)(i / out_w), ox = (uint32_t)(i - (uint64_t)oy * out_w);
    float pre_h[3] = {0, 0, 0}, str_h[3] = {0, 0, 0}, a_h = 0.0f;
    float pre_d[3] = {0, 0, 0}, str_d[3] = {0, 0, 0}, a_d = 0.0f;
    for (uint32_t j = 0; j < aa; ++j)
      for (uint32_t k = 0; k < aa; ++k) {
        const uint64_t si = ((uint64_t)oy * aa + j) * rw + (uint64_t)ox * aa + k;
        float4 ch = bg, cd = bg;
        if (covered[si]) {
          const float4 c = samples[si];
          ch = c;
          float m[3] = {c.x * exposure, c.y * exposure, c.z * exposure};
          tone_apply(tone, m);
          cd = make_float4(m[0], m[1], m[2], clampr(c.w, 0.0f, 1.0f));
        }
        const float hv[4] = {ch.x, ch.y, ch.z, ch.w}, dv[4] = {cd.x, cd.y, cd.z, cd.w};
        for (int q = 0; q < 3; ++q) {
          pre_h[q] += hv[q] * hv[3];
          str_h[q] += hv[q];
          pre_d[q] += dv[q] * dv[3];
          str_d[q] += dv[q];
        }
        a_h += hv[3];
        a_d += dv[3];
      }
    if (hdr)
      hdr[i] = a_h > 0.0f ? make_float4(pre_h[0] / a_h, pre_h[1] / a_h, pre_h[2] / a_h, a_h / cnt)
                          : make_float4(str_h[0] / cnt, str_h[1] / cnt, str_h[2] / cnt, 0.0f);
    if (rgba) {
      const float4 o = a_d > 0.0f ? make_float4(pre_d[0] / a_d, pre_d[1] / a_d, pre_d[2] / a_d, a_d / cnt)
                                  : make_float4(str_d[0] / cnt, str_d[1] / cnt, str_d[2] / cnt, 0.0f);
      rgba[i] = make_uchar4(srgb_byte(o.x), srgb_byte(o.y), srgb_byte(o.z),
                            (uint8_t)roundf(clampr(o.w, 0.0f, 1.0f) * 255.0f));
    }
  }
}

}  // namespace ptd
