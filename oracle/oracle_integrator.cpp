// ORACLE — test infrastructure only (see oracle_core.hpp).
// Integrator::sample (src/pathtrace.rs:1878-2330), the progressive
// accumulator and its band scheduler (:2526-2591), the resolve
// (:2593-2734) with ToneMap / sRGB (src/hdr.rs:41-129), and the C entry
// points the Python test harness calls through ctypes.
#include <algorithm>
#include <atomic>
#include <thread>

#include "oracle_scene.hpp"

namespace oracle {

struct Integrator {
  const Scene *ts;
  const EnvironmentMap *env;
  pt_camera cam;
  uint32_t width, height;
  float ambient;
  pt_path_trace_options pt;
  float pixel_spread;
  bool orthographic;
  mutable uint64_t ext_rays = 0, shadow_rays = 0;

  V3 cv(const float *a) const { return {a[0], a[1], a[2]}; }
  // Camera::primary_ray, src/camera.rs:489-514.
  void primary_ray(float px, float py, V3 &o, V3 &d) const {
    float ndc_x = (px / fmaxr((float)width, 1.0f)) * 2.0f - 1.0f;
    float ndc_y = 1.0f - (py / fmaxr((float)height, 1.0f)) * 2.0f;
    V3 off = add(scale(cv(cam.side), ndc_x * cam.half_w), scale(cv(cam.up), ndc_y * cam.half_h));
    if (cam.projection == PT_PERSPECTIVE) {
      o = cv(cam.eye);
      d = normalise(add(off, cv(cam.forward)));
    } else {
      o = add(cv(cam.eye), off);
      d = cv(cam.forward);
    }
  }
  V3 clamp(V3 c) const {
    float m = max3(c);
    if (pt.clamp > 0.0f && m > pt.clamp) return scale(c, pt.clamp / m);
    return c;
  }
  float p_env() const {
    if (env && !ts->emissive.empty()) return 0.5f;
    if (env) return 1.0f;
    return 0.0f;
  }
  // Integrator::accept, src/pathtrace.rs:1924-1934.
  bool accept(const Hit &c, const Sampler &s, uint32_t ray, bool primary) const {
    const pt_material &mat = ts->material_of(c);
    if (primary && !c.front && !mat.double_sided) return false;
    switch (mat.alpha_mode) {
      case PT_ALPHA_MASK:
        return ts->alpha(c) >= mat.alpha_cutoff;
      case PT_ALPHA_BLEND:
        return s.coin(ray, c.global) < ts->alpha(c);
      default:
        return true;
    }
  }
  bool visible(V3 o, V3 d, float t_max, const Sampler &s, uint32_t ray, uint32_t skip) const {
    shadow_rays++;
    return !ts->occluded_filtered(o, d, 0.0f, t_max,
                                  [&](const Hit &c) { return c.global != skip && accept(c, s, ray, false); });
  }
  // Integrator::emission, src/pathtrace.rs:1951-1966.
  V3 emission(const Hit &hit) const {
    const Item &item = ts->item_of(hit);
    const pt_material &mat = ts->material_of(hit);
    V3 e = cv(mat.emissive);
    if (mat.unlit || is_black(e)) return {0, 0, 0};
    V4 t;
    if (ts->sample_binding(item, mat.emissive_texture, 3 * (size_t)hit.tri, hit.bary, TexLod{}, true, t))
      e = mul(e, {t[0], t[1], t[2]});
    return e;
  }
  // Integrator::tri_pdf, src/pathtrace.rs:1972-1991.
  float tri_pdf(size_t li, uint32_t g, V3 p, V3 q) const {
    V3 a, b, c;
    ts->triangle_positions(g, a, b, c);
    float sel = (1.0f - p_env()) * ts->emissive.pmf[li];
    float omega = triangle_solid_angle(p, a, b, c);
    if (omega >= MIN_SPHERICAL_SOLID_ANGLE) return sel / omega;
    V3 cr = cross(sub(b, a), sub(c, a));
    float len = std::sqrt(dot(cr, cr));
    V3 to = sub(q, p);
    float d2 = dot(to, to);
    if (len <= 0.0f || d2 <= 0.0f) return 0.0f;
    float cos = std::fabs(dot(cr, to) / (len * std::sqrt(d2)));
    if (cos <= 0.0f) return 0.0f;
    return sel * d2 / (0.5f * len * cos);
  }
  float light_pdf(const Hit &hit, V3 p, V3 q) const {
    if (hit.global >= ts->emissive.lookup.size()) return 0.0f;
    uint32_t li = ts->emissive.lookup[hit.global];
    if (li == UINT32_MAX) return 0.0f;
    return tri_pdf(li, hit.global, p, q);
  }
  static float power_heuristic(float a, float b) {
    float a2 = a * a, b2 = b * b;
    if (a2 + b2 > 0.0f && std::isfinite(a2 + b2)) return a2 / (a2 + b2);
    if (std::isinf(a)) return 1.0f;
    return 0.0f;
  }
  static V3 offset_ray_origin(V3 p, V3 n) {
    const float ORIGIN = 1.0f / 32.0f, FLOAT_SCALE = 1.0f / 65536.0f, INT_SCALE = 256.0f;
    V3 out;
    for (int k = 0; k < 3; ++k) {
      int32_t of_i = f2i32(INT_SCALE * n[k]);
      int32_t bits;
      std::memcpy(&bits, &p[k], 4);
      int32_t moved = p[k] < 0.0f ? (int32_t)((uint32_t)bits - (uint32_t)of_i) : (int32_t)((uint32_t)bits + (uint32_t)of_i);
      float p_i;
      std::memcpy(&p_i, &moved, 4);
      if (std::fabs(p[k]) < ORIGIN)
        out[k] = p[k] + FLOAT_SCALE * n[k];
      else if (std::isfinite(p_i))
        out[k] = p_i;
      else
        out[k] = p[k];
    }
    return out;
  }

  // Integrator::sample, src/pathtrace.rs:2004-2329. Returns false when the
  // sample is uncovered.
  bool sample(uint32_t x, uint32_t y, uint32_t index, V3 &out) const {
    Sampler s(pt.seed, x, y, index);
    float p0[4];
    s.pattern(0, p0);
    V3 o, d;
    primary_ray((float)x + p0[0], (float)y + p0[1], o, d);
    V3 beta = {1, 1, 1}, radiance = {0, 0, 0};
    float prev_pdf = 0.0f;
    V3 prev_pos = {0, 0, 0};
    bool has_medium = false;
    V3 sigma = {0, 0, 0};
    int hero = -1;
    uint32_t strategy = pt.strategy;
    uint32_t k = 0;
    for (;;) {
      uint32_t ray_id = k << 16;
      Hit hit;
      ext_rays++;
      bool found = ts->closest_hit_filtered(o, d, 0.0f, INF, [&](const Hit &c) { return accept(c, s, ray_id, k == 0); },
                                            hit);
      if (has_medium) {
        if (!found) break;
        for (int c = 0; c < 3; ++c) beta[c] *= std::exp(-sigma[c] * hit.t);
      }
      if (!found) {
        if (k == 0) return false;
        V3 le;
        float w;
        if (env) {
          le = env->radiance(d);
          if (strategy == PT_MIS)
            w = power_heuristic(prev_pdf, p_env() * env->pdf(d));
          else if (strategy == PT_LIGHT_ONLY)
            w = 0.0f;
          else
            w = 1.0f;
        } else {
          le = {ambient, ambient, ambient};
          w = 1.0f;
        }
        if (w > 0.0f) radiance = add(radiance, clamp(scale(mul(beta, le), w)));
        break;
      }
      Surface surf = ts->surface(hit);
      const pt_material &pmat = ts->material_of(hit);
      V3 pem = cv(pmat.emissive);
      if ((hit.front || pmat.double_sided) && !pmat.unlit && !is_black(pem)) {
        V3 le = emission(hit);
        if (!is_black(le)) {
          if (k == 0) {
            radiance = add(radiance, mul(beta, le));
          } else {
            float pl = light_pdf(hit, prev_pos, surf.position);
            float w;
            if (pl <= 0.0f)
              w = 1.0f;
            else if (strategy == PT_MIS)
              w = power_heuristic(prev_pdf, pl);
            else if (strategy == PT_LIGHT_ONLY)
              w = 0.0f;
            else
              w = 1.0f;
            if (w > 0.0f) radiance = add(radiance, clamp(scale(mul(beta, le), w)));
          }
        }
      }
      TexLod lod;
      if (k == 0) {
        lod.kind = TexLodKind::Cone;
        lod.width = orthographic ? pixel_spread : pixel_spread * hit.t;
        lod.dir = d;
      }
      bool flip = !hit.front && pmat.double_sided;
      MaterialSample mat = ts->material_oriented(hit, surf, lod, flip);
      if (flip) {
        mat.normal = neg(mat.normal);
        mat.clearcoat_normal = neg(mat.clearcoat_normal);
      }
      if (mat.unlit) {
        V3 c = {mat.base_color[0], mat.base_color[1], mat.base_color[2]};
        V3 contrib = mul(beta, c);
        radiance = add(radiance, k == 0 ? contrib : clamp(contrib));
        break;
      }
      if (k >= pt.max_bounces) break;
      if (mat.dispersion > 0.0f && mat.thickness > 0.0f && mat.transmission > 0.0f) {
        int c;
        if (hero >= 0) {
          c = hero;
        } else {
          c = (int)std::min<uint64_t>(f2usize(s.coin(ray_id | 0x7fffu, UINT32_MAX) * 3.0f), 2);
          for (int i = 0; i < 3; ++i) beta[i] = i == c ? beta[i] * 3.0f : 0.0f;
          hero = c;
        }
        float iors[3];
        dispersion_iors(mat.ior, mat.dispersion, iors);
        mat.ior = iors[c];
      }
      V3 v = neg(d);
      Bsdf bsdf(mat, v, surf.geometric_normal, hit.front);
      if (bsdf.is_black()) break;
      V3 p = surf.position;
      V3 ng = bsdf.ng;
      auto spawn = [&](V3 dir) { return dot(dir, ng) >= 0.0f ? offset_ray_origin(p, ng) : offset_ray_origin(p, neg(ng)); };

      // NEE: punctual lights.
      for (size_t j = 0; j < ts->lights.size(); ++j) {
        LightSample ls;
        if (!light_sample(ts->lights[j], p, ls)) continue;
        V3 f;
        float pdf_unused;
        bsdf.eval(ls.l, f, pdf_unused);
        if (is_black(f)) continue;
        V3 o2 = spawn(ls.l);
        float tmax = std::isfinite(ls.distance) ? ls.distance * (1.0f - 1.0e-4f) : INF;
        if (visible(o2, ls.l, tmax, s, ray_id | 0x8000u | ((uint32_t)j & 0x7fffu), UINT32_MAX))
          radiance = add(radiance, clamp(mul(mul(beta, f), ls.radiance)));
      }

      // NEE: area set.
      float pl_u[4];
      s.pattern(2 + 2 * k, pl_u);
      if (strategy != PT_BSDF_ONLY && (env || !ts->emissive.empty())) {
        float pe = p_env();
        uint32_t shadow_id = ray_id | 0xffffu;
        if (pl_u[2] < pe) {
          V3 l, le;
          float pdf;
          if (env && env->sample(pl_u[0], pl_u[1], l, le, pdf)) {
            float pl = pe * pdf;
            V3 f;
            float pb;
            bsdf.eval(l, f, pb);
            if (!is_black(f) && !is_black(le) && pl > 0.0f) {
              float w = strategy == PT_MIS ? power_heuristic(pl, pb) : 1.0f;
              if (visible(spawn(l), l, INF, s, shadow_id, UINT32_MAX))
                radiance = add(radiance, clamp(scale(mul(mul(beta, f), le), w / pl)));
            }
          }
        } else if (!ts->emissive.empty()) {
          float us = pe > 0.0f ? clampr((pl_u[2] - pe) / (1.0f - pe), 0.0f, 0.999999f) : pl_u[2];
          size_t li = ts->emissive.pick(us);
          uint32_t g = ts->emissive.tris[li];
          V3 a, b, c;
          ts->triangle_positions(g, a, b, c);
          bool have_target = false;
          V3 q;
          if (triangle_solid_angle(p, a, b, c) >= MIN_SPHERICAL_SOLID_ANGLE) {
            V3 l;
            if (sample_spherical_triangle(p, a, b, c, pl_u[0], pl_u[1], l)) {
              V3 n = cross(sub(b, a), sub(c, a));
              float dn = dot(l, n);
              if (dn != 0.0f) {
                float t = dot(sub(a, p), n) / dn;
                if (t > 0.0f && std::isfinite(t)) {
                  q = add(p, scale(l, t));
                  have_target = true;
                }
              }
            }
          } else {
            float su = std::sqrt(pl_u[0]);
            float w[3] = {1.0f - su, su * (1.0f - pl_u[1]), su * pl_u[1]};
            q = {a.x * w[0] + b.x * w[1] + c.x * w[2], a.y * w[0] + b.y * w[1] + c.y * w[2],
                 a.z * w[0] + b.z * w[1] + c.z * w[2]};
            have_target = true;
          }
          float bary[3];
          bool have_bary = false;
          if (have_target) {
            // barycentric_of, src/trace.rs:1120-1133.
            V3 e1 = sub(b, a), e2 = sub(c, a), r = sub(q, a);
            float d11 = dot(e1, e1), d12 = dot(e1, e2), d22 = dot(e2, e2);
            float r1 = dot(r, e1), r2 = dot(r, e2);
            float det = d11 * d22 - d12 * d12;
            if (std::isfinite(det) && std::fabs(det) > FLT_MIN) {
              float u = (d22 * r1 - d12 * r2) / det;
              float vv = (d11 * r2 - d12 * r1) / det;
              bary[0] = 1.0f - u - vv;
              bary[1] = u;
              bary[2] = vv;
              have_bary = true;
            }
          }
          if (have_target && have_bary) {
            for (float &bb : bary) bb = clampr(bb, 0.0f, 1.0f);
            V3 to = sub(q, p);
            float dist2 = dot(to, to);
            Hit lh = ts->make_hit(g, std::sqrt(dist2), bary, true);
            Surface lsurf = ts->surface(lh);
            const pt_material &lmat = ts->material_of(lh);
            if (dist2 > 1.0e-12f) {
              float dist = std::sqrt(dist2);
              V3 l = scale(to, 1.0f / dist);
              float cos_l = -dot(lsurf.geometric_normal, l);
              float pl = tri_pdf(li, g, p, q);
              if ((cos_l > 0.0f || (lmat.double_sided && cos_l < 0.0f)) && pl > 0.0f && std::isfinite(pl)) {
                V3 f;
                float pb;
                bsdf.eval(l, f, pb);
                V3 le = emission(lh);
                if (!is_black(f) && !is_black(le)) {
                  float w = strategy == PT_MIS ? power_heuristic(pl, pb) : 1.0f;
                  V3 o2 = spawn(l);
                  float tmax = fmaxr(dist * (1.0f - 1.0e-4f), 0.0f);
                  if (visible(o2, l, tmax, s, shadow_id, g))
                    radiance = add(radiance, clamp(scale(mul(mul(beta, f), le), w / pl)));
                }
              }
            }
          }
        }
      }

      // BSDF sampling.
      float pb_u[4];
      s.pattern(1 + 2 * k, pb_u);
      V3 l, f;
      float pdf;
      if (!bsdf.sample(pb_u, l, f, pdf)) break;
      beta = mul(beta, scale(f, 1.0f / pdf));
      if (!finite3(beta)) break;
      prev_pdf = pdf;
      prev_pos = p;
      if (dot(l, ng) < 0.0f && mat.thickness > 0.0f && mat.transmission > 0.0f) {
        if (hit.front) {
          float dist = mat.attenuation_distance;
          if (std::isfinite(dist)) {
            V3 c = mat.attenuation_color;
            sigma = {-std::log(fmaxr(c.x, 1.0e-6f)) / dist, -std::log(fmaxr(c.y, 1.0e-6f)) / dist,
                     -std::log(fmaxr(c.z, 1.0e-6f)) / dist};
            has_medium = true;
          } else {
            has_medium = false;
          }
        } else {
          has_medium = false;
        }
      }
      if (k + 1 >= pt.rr_start) {
        float q = clampr(max3(beta), 0.05f, 1.0f);
        if (q < 1.0f) {
          if (pb_u[3] >= q) break;
          beta = scale(beta, 1.0f / q);
        }
      }
      o = spawn(l);
      d = l;
      k += 1;
    }
    out = finite3(radiance) ? radiance : V3{0, 0, 0};
    return true;
  }
};

static Integrator make_integrator(const Scene *sc, const EnvironmentMap *env, const pt_camera &cam,
                                  const pt_render_options &o) {
  Integrator it;
  it.ts = sc;
  it.env = env;
  it.cam = cam;
  it.width = std::max(o.width, 1u);
  it.height = std::max(o.height, 1u);
  it.ambient = std::isfinite(o.ambient) ? fmaxr(o.ambient, 0.0f) : 0.0f;
  it.pt = o.path_trace;
  it.orthographic = cam.projection == PT_ORTHOGRAPHIC;
  it.pixel_spread = 2.0f * cam.half_h / (float)it.height;
  return it;
}

// ---- resolve (src/hdr.rs:41-129, src/pathtrace.rs:2593-2734) ----------------
static float srgb_to_linear_f(float c) {
  if (c <= 0.04045f) return c / 12.92f;
  return std::pow((c + 0.055f) / 1.055f, 2.4f);
}
static float sanitize(float v) { return std::isnan(v) ? 0.0f : v; }
static float aces(float x) {
  x = x * 0.6f;
  float v = (x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f);
  return clampr(v, 0.0f, 1.0f);
}
static V3 tone_apply(uint32_t tm, V3 rgb) {
  rgb = {fmaxr(sanitize(rgb.x), 0.0f), fmaxr(sanitize(rgb.y), 0.0f), fmaxr(sanitize(rgb.z), 0.0f)};
  if (tm == PT_TONE_REINHARD) {
    float l = 0.2126f * rgb.x + 0.7152f * rgb.y + 0.0722f * rgb.z;
    if (l <= 0.0f) return {0, 0, 0};
    float s = 1.0f / (1.0f + l);
    return {fminr(rgb.x * s, 1.0f), fminr(rgb.y * s, 1.0f), fminr(rgb.z * s, 1.0f)};
  }
  if (tm == PT_TONE_ACES) return {aces(rgb.x), aces(rgb.y), aces(rgb.z)};
  return {fminr(rgb.x, 1.0f), fminr(rgb.y, 1.0f), fminr(rgb.z, 1.0f)};
}
static uint8_t linear_to_srgb_byte(float c) {
  static float t[255];
  static bool init = [] {
    for (int k = 0; k < 255; ++k) t[k] = srgb_to_linear_f(((float)k + 0.5f) / 255.0f);
    return true;
  }();
  (void)init;
  if (std::isnan(c)) return 0;
  return (uint8_t)(std::upper_bound(t, t + 255, c) - t);
}
static void bg_linear(const pt_render_options &o, float bg[4]) {
  for (int k = 0; k < 3; ++k) bg[k] = srgb_to_linear_f((float)o.background[k] / 255.0f);
  bg[3] = (float)o.background[3] / 255.0f;
}
static void mix(const float m[3], float f, const float bg[4], float out[4]) {
  float a_sum = f + (1.0f - f) * bg[3];
  if (a_sum > 0.0f) {
    for (int k = 0; k < 3; ++k) out[k] = (f * m[k] + (1.0f - f) * bg[k] * bg[3]) / a_sum;
    out[3] = a_sum;
  } else {
    for (int k = 0; k < 3; ++k) out[k] = f * m[k] + (1.0f - f) * bg[k];
    out[3] = 0.0f;
  }
}
static bool resolve_pixel(const double *a, uint32_t samples, const float bg[4], bool tone, const pt_render_options &o,
                          float out[4]) {
  if (a[3] <= 0.0 || samples == 0) return false;
  float m[3] = {(float)(a[0] / a[3]), (float)(a[1] / a[3]), (float)(a[2] / a[3])};
  float f = (float)clampd(a[3] / (double)samples, 0.0, 1.0);
  V3 c = {m[0], m[1], m[2]};
  if (tone) c = tone_apply(o.tone_map, scale(c, o.exposure));
  float cm[3] = {c.x, c.y, c.z};
  if (f >= 1.0f) {
    out[0] = c.x;
    out[1] = c.y;
    out[2] = c.z;
    out[3] = 1.0f;
  } else {
    mix(cm, f, bg, out);
  }
  return true;
}

// ---- RenderBackend::Raycast, legacy shading modes ------------------------
// Ctx::pixel / legacy / whitted (src/raycast.rs:349-516) with shade_pixel and
// build_light (src/shade.rs:26-50), reflect / refract / schlick
// (src/trace.rs:1087-1116), normal_to_byte / depth_to_byte
// (src/scanline.rs:840-858), Camera::ndc_z / view_depth
// (src/camera.rs:521-543), and the frame resolve (src/scanline.rs:124-221).
namespace {
constexpr float kAmbient = 0.2f;
constexpr float kSecondary = 1.0e-2f;
constexpr float kWireEdge = 0.03f;
constexpr uint32_t kDepthCap = 16;

V3 interp3v(const std::vector<V3> &v, size_t base, const float b[3]) {
  V3 x = v[base], y = v[base + 1], z = v[base + 2];
  return {x.x * b[0] + y.x * b[1] + z.x * b[2], x.y * b[0] + y.y * b[1] + z.y * b[2],
          x.z * b[0] + y.z * b[1] + z.z * b[2]};
}

struct Raycaster {
  const Scene *ts;
  pt_camera cam;
  uint32_t rw, rh, mode, max_depth;
  V3 light;
  float intensity, near_p, far_p;
  float lut[256];

  V3 cv(const float *a) const { return {a[0], a[1], a[2]}; }
  void primary_ray(float px, float py, V3 &o, V3 &d) const {
    float ndc_x = (px / fmaxr((float)rw, 1.0f)) * 2.0f - 1.0f;
    float ndc_y = 1.0f - (py / fmaxr((float)rh, 1.0f)) * 2.0f;
    V3 off = add(scale(cv(cam.side), ndc_x * cam.half_w), scale(cv(cam.up), ndc_y * cam.half_h));
    if (cam.projection == PT_PERSPECTIVE) {
      o = cv(cam.eye);
      d = normalise(add(off, cv(cam.forward)));
    } else {
      o = add(cv(cam.eye), off);
      d = cv(cam.forward);
    }
  }
  V4 shade_pixel(V4 base, V3 n) const {
    float cos_theta = fmaxr(dot(n, light), 0.0f);
    float diffuse = kAmbient + (1.0f - kAmbient) * cos_theta * intensity;
    float f = clampr(diffuse, 0.0f, 1.0f);
    return V4{{base[0] * f, base[1] * f, base[2] * f, base[3]}};
  }
  V3 corner_normal(const Item &it, size_t c, const Hit &h) const {
    if (it.normals.size() > c) return it.normals[c];
    return ts->surface(h).geometric_normal;
  }
  V3 hit_normal(const Item &it, const Hit &h) const {
    if (it.normals.size() == it.positions.size()) return interp3v(it.normals, 3 * (size_t)h.tri, h.bary);
    return ts->surface(h).geometric_normal;
  }
  static V3 reflect(V3 d, V3 n) {
    float k = 2.0f * dot(d, n);
    return {d.x - k * n.x, d.y - k * n.y, d.z - k * n.z};
  }
  static bool refract(V3 d, V3 n, float eta, V3 &out) {
    float cos_i = clampr(-dot(d, n), -1.0f, 1.0f);
    float sin2_t = eta * eta * (1.0f - cos_i * cos_i);
    if (sin2_t > 1.0f) return false;
    float cos_t = std::sqrt(1.0f - sin2_t);
    float k = eta * cos_i - cos_t;
    out = normalise({eta * d.x + k * n.x, eta * d.y + k * n.y, eta * d.z + k * n.z});
    return true;
  }
  static float schlick(float f0, float c) { return f0 + (1.0f - f0) * powi5(1.0f - clampr(c, 0.0f, 1.0f)); }
  static uint32_t normal_byte(float n) {
    if (!std::isfinite(n)) return 128;
    float v = std::round((clampr(n, -1.0f, 1.0f) + 1.0f) * 0.5f * 255.0f);
    return (uint32_t)clampr(v, 0.0f, 255.0f);
  }
  static uint32_t depth_byte(float z) {
    if (!std::isfinite(z)) return 0;
    float zc = clampr(z, -1.0f, 1.0f);
    float v = std::round((1.0f - (zc * 0.5f + 0.5f)) * 255.0f);
    return (uint32_t)clampr(v, 0.0f, 255.0f);
  }
  float ndc_z(float vd) const {
    if (cam.projection == PT_PERSPECTIVE) {
      float nf = 1.0f / (near_p - far_p);
      float d = fmaxr(vd, FLT_MIN);
      return -(far_p + near_p) * nf + 2.0f * far_p * near_p * nf / d;
    }
    float fne = far_p - near_p;
    if (std::fabs(fne) < FLT_EPSILON) return 0.0f;
    return (2.0f * vd - (far_p + near_p)) / fne;
  }

  V4 whitted(V3 d, const Hit &hit, uint32_t depth) const {
    const Item &it = ts->item_of(hit);
    const pt_material &mat = ts->material_of(hit);
    const V4 a{{mat.base_color[0], mat.base_color[1], mat.base_color[2], mat.base_color[3]}};
    if (mat.unlit) return a;
    V3 raw = normalise(hit_normal(it, hit));
    bool entering = dot(d, raw) < 0.0f;
    V3 n = entering ? raw : scale(raw, -1.0f);
    V3 p = interp3v(it.positions, 3 * (size_t)hit.tri, hit.bary);
    uint32_t skip = hit.global;
    auto not_self = [&](const Hit &h) { return h.global != skip; };
    V3 so = Integrator::offset_ray_origin(p, n);
    bool shadowed = ts->occluded_filtered(so, light, 0.0f, INF, not_self);
    V4 out = shadowed ? V4{{a[0] * kAmbient, a[1] * kAmbient, a[2] * kAmbient, a[3]}} : shade_pixel(a, n);
    for (int k = 0; k < 3; ++k) out[k] += mat.emissive[k];
    if (depth >= max_depth) return out;
    float cos_in = clampr(-dot(d, n), 0.0f, 1.0f);
    auto trace = [&](V3 o, V3 dir, V4 &c) {
      Hit h;
      if (!ts->closest_hit_filtered(o, dir, 0.0f, INF, not_self, h)) return false;
      c = whitted(dir, h, depth + 1);
      return true;
    };
    float gloss = mat.metallic * (1.0f - mat.roughness);
    if (gloss > kSecondary) {
      float f0 = 0.04f + 0.96f * mat.metallic;
      float kr = clampr(schlick(f0, cos_in), 0.0f, 1.0f) * gloss;
      V4 rc{{0.0f, 0.0f, 0.0f, 1.0f}};
      trace(so, reflect(d, n), rc);
      for (int k = 0; k < 3; ++k) out[k] = out[k] * (1.0f - kr) + rc[k] * a[k] * kr;
    }
    float kt = (mat.ext_flags & PT_EXT_TRANSMISSION) ? clampr(mat.transmission_factor, 0.0f, 1.0f) : 0.0f;
    if (kt > kSecondary) {
      float eta = entering ? 1.0f / mat.ior : mat.ior;
      V3 tdir;
      if (refract(d, n, eta, tdir)) {
        V3 ro = Integrator::offset_ray_origin(p, scale(n, -1.0f));
        V4 tc{{0.0f, 0.0f, 0.0f, 0.0f}};
        trace(ro, tdir, tc);
        for (int k = 0; k < 3; ++k) out[k] = out[k] * (1.0f - kt) + tc[k] * a[k] * kt;
      } else {
        V4 rc;
        if (trace(so, reflect(d, n), rc))
          for (int k = 0; k < 3; ++k) out[k] = out[k] * (1.0f - kt) + rc[k] * kt;
      }
    }
    return out;
  }

  // ---- Pbr: Ctx::radiance / miss / secondary / shade (src/raycast.rs:518-740)
  // with TraceScene::shadow_transmittance, direct_light and
  // barycentric_differentials (src/trace.rs:947-1082) and the glTF
  // metallic-roughness BRDF (src/brdf.rs:24-148).
  float ambient = 0.0f, cutoff = 0.0f, spread = 0.0f;
  bool shadows = false;
  float bg[4] = {0, 0, 0, 0};
  static constexpr uint32_t kMaxLayers = 64;  // MAX_LAYERS, src/raycast.rs:126
  static constexpr float kPi = 3.14159265358979323846f;

  struct RayState {
    uint32_t depth = 0, layers = 0;
    bool camera = true;
    bool inside = false;  // Some(sigma)
    V3 sigma = {0, 0, 0};
    bool has_skip = false;
    uint32_t skip = 0;
  };
  struct Footprint {
    bool diff = true;
    V3 dxo, dxd, dyo, dyd;        // Diff: neighbouring camera rays
    float width = 0.0f, spr = 0.0f;  // Cone
  };
  struct BrdfParams {
    V3 c_diff, f0;
    float alpha;
  };
  // BrdfParams::metallic_roughness, src/brdf.rs:96-123.
  static BrdfParams metallic_roughness(V3 base, float metallic, float roughness, float f0d) {
    float m = clampr(metallic, 0.0f, 1.0f), r = clampr(roughness, 0.0f, 1.0f);
    return {{base.x * (1.0f - m), base.y * (1.0f - m), base.z * (1.0f - m)},
            {f0d + (base.x - f0d) * m, f0d + (base.y - f0d) * m, f0d + (base.z - f0d) * m},
            fmaxr(r * r, 1.0e-3f)};
  }
  // d_ggx / v_smith_ggx_correlated / f_schlick / eval, src/brdf.rs:31-148.
  static float gltf_d_ggx(float n_dot_h, float alpha) {
    float a2 = alpha * alpha;
    float d = n_dot_h * n_dot_h * (a2 - 1.0f) + 1.0f;
    return a2 / fmaxr(kPi * d * d, 1.0e-12f);
  }
  static float v_smith(float n_dot_l, float n_dot_v, float alpha) {
    float a2 = alpha * alpha;
    float gv = n_dot_l * std::sqrt(n_dot_v * n_dot_v * (1.0f - a2) + a2);
    float gl = n_dot_v * std::sqrt(n_dot_l * n_dot_l * (1.0f - a2) + a2);
    float s = gv + gl;
    return s > 0.0f ? 0.5f / s : 0.0f;
  }
  static V3 f_schlick3(V3 f0, float v_dot_h) {
    float k = powi5(1.0f - clampr(v_dot_h, 0.0f, 1.0f));
    return {f0.x + (1.0f - f0.x) * k, f0.y + (1.0f - f0.y) * k, f0.z + (1.0f - f0.z) * k};
  }
  static V3 brdf_eval(const BrdfParams &p, V3 n, V3 v, V3 l) {
    float n_dot_l = dot(n, l);
    if (n_dot_l <= 0.0f) return {0.0f, 0.0f, 0.0f};
    float n_dot_v = fmaxr(dot(n, v), 1.0e-4f);
    V3 h = {l.x + v.x, l.y + v.y, l.z + v.z};
    float hl = std::sqrt(dot(h, h));
    h = hl > 0.0f ? V3{h.x / hl, h.y / hl, h.z / hl} : n;
    float n_dot_h = fmaxr(dot(n, h), 0.0f), v_dot_h = fmaxr(dot(v, h), 0.0f);
    V3 f = f_schlick3(p.f0, v_dot_h);
    float spec = gltf_d_ggx(n_dot_h, p.alpha) * v_smith(n_dot_l, n_dot_v, p.alpha);
    return {((1.0f - f.x) * p.c_diff.x / kPi + f.x * spec) * n_dot_l,
            ((1.0f - f.y) * p.c_diff.y / kPi + f.y * spec) * n_dot_l,
            ((1.0f - f.z) * p.c_diff.z / kPi + f.z * spec) * n_dot_l};
  }
  bool masked_out(const Hit &h) const {
    const pt_material &mat = ts->material_of(h);
    return mat.alpha_mode == PT_ALPHA_MASK && ts->alpha(h) < mat.alpha_cutoff;
  }
  // TraceScene::shadow_transmittance, src/trace.rs:947-1005. The product
  // runs in f64 and is rounded once, so it does not depend on the order in
  // which the BVH reports the partial occluders.
  V3 shadow_transmittance(V3 origin, V3 dir, float t_max, const RayState &st) const {
    double tr[3] = {1.0, 1.0, 1.0};
    const double eps = (double)1.0e-4f;
    bool blocked = ts->occluded_filtered(origin, dir, 0.0f, t_max, [&](const Hit &h) {
      if (st.has_skip && h.global == st.skip) return false;
      const pt_material &mat = ts->material_of(h);
      float pass[3] = {0.0f, 0.0f, 0.0f};
      if (mat.alpha_mode == PT_ALPHA_MASK) {
        if (ts->alpha(h) < mat.alpha_cutoff) return false;
      } else if (mat.alpha_mode == PT_ALPHA_BLEND) {
        float a = 1.0f - clampr(ts->alpha(h), 0.0f, 1.0f);
        pass[0] = pass[1] = pass[2] = a;
      }
      bool has_tr = (mat.ext_flags & PT_EXT_TRANSMISSION) && std::isfinite(mat.transmission_factor) &&
                    mat.transmission_factor > 0.0f;
      if (has_tr) {
        Surface surf = ts->surface(h);
        MaterialSample m = ts->material_oriented(h, surf, TexLod{}, false);
        if (m.transmission > 0.0f) {
          if (m.thickness > 0.0f && !h.front) return false;
          float kt = m.transmission * (1.0f - m.metallic);
          float a = mat.alpha_mode == PT_ALPHA_BLEND ? pass[0] : 0.0f;
          for (int k = 0; k < 3; ++k) pass[k] = a + (1.0f - a) * kt * m.base_color[k];
        }
      }
      for (int k = 0; k < 3; ++k) tr[k] *= (double)clampr(pass[k], 0.0f, 1.0f);
      return tr[0] <= eps && tr[1] <= eps && tr[2] <= eps;
    });
    if (blocked) return {0.0f, 0.0f, 0.0f};
    return {(float)tr[0], (float)tr[1], (float)tr[2]};
  }
  // TraceScene::direct_light, src/trace.rs:1007-1048.
  V3 direct_light(V3 p, V3 n, V3 ng, V3 v, const BrdfParams &bp, const RayState &skip) const {
    float out[3] = {0.0f, 0.0f, 0.0f};
    for (const pt_light &L : ts->lights) {
      LightSample s;
      if (!light_sample(L, p, s)) continue;
      V3 f = brdf_eval(bp, n, v, s.l);
      if (f.x == 0.0f && f.y == 0.0f && f.z == 0.0f) continue;
      V3 vis = {1.0f, 1.0f, 1.0f};
      if (shadows) {
        float side = dot(ng, s.l) >= 0.0f ? 1.0f : -1.0f;
        V3 o = Integrator::offset_ray_origin(p, {ng.x * side, ng.y * side, ng.z * side});
        float t_max = std::isfinite(s.distance) ? s.distance * (1.0f - 1.0e-4f) : INF;
        vis = shadow_transmittance(o, s.l, t_max, skip);
      }
      out[0] += f.x * s.radiance.x * vis.x;
      out[1] += f.y * s.radiance.y * vis.y;
      out[2] += f.z * s.radiance.z * vis.z;
    }
    return {out[0], out[1], out[2]};
  }
  // barycentric_of, src/trace.rs:1120-1133.
  static bool barycentric_of(V3 q, V3 p0, V3 p1, V3 p2, float out[3]) {
    V3 e1 = sub(p1, p0), e2 = sub(p2, p0), r = sub(q, p0);
    float d11 = dot(e1, e1), d12 = dot(e1, e2), d22 = dot(e2, e2);
    float r1 = dot(r, e1), r2 = dot(r, e2);
    float det = d11 * d22 - d12 * d12;
    if (!std::isfinite(det) || std::fabs(det) <= FLT_MIN) return false;
    float u = (d22 * r1 - d12 * r2) / det;
    float v = (d11 * r2 - d12 * r1) / det;
    out[0] = 1.0f - u - v;
    out[1] = u;
    out[2] = v;
    return true;
  }
  // TraceScene::barycentric_differentials, src/trace.rs:1050-1082.
  bool barycentric_differentials(const Hit &hit, const Footprint &fp, TexLod &lod, float &width) const {
    V3 p0, p1, p2;
    ts->triangle_positions(hit.global, p0, p1, p2);
    V3 ng = cross(sub(p1, p0), sub(p2, p0));
    const float *b = hit.bary;
    V3 p = {p0.x * b[0] + p1.x * b[1] + p2.x * b[2], p0.y * b[0] + p1.y * b[1] + p2.y * b[2],
            p0.z * b[0] + p1.z * b[1] + p2.z * b[2]};
    auto on_plane = [&](V3 o, V3 d, float g[3], float &w) {
      float denom = dot(ng, d);
      if (std::fabs(denom) <= FLT_MIN) return false;
      float t = dot(ng, sub(p0, o)) / denom;
      V3 q = {o.x + d.x * t, o.y + d.y * t, o.z + d.z * t};
      float bq[3];
      if (!barycentric_of(q, p0, p1, p2, bq)) return false;
      V3 wv = sub(q, p);
      float wl = std::sqrt(dot(wv, wv));
      if (!std::isfinite(wl)) return false;
      for (int k = 0; k < 3; ++k) g[k] = bq[k] - b[k];
      w = wl;
      return true;
    };
    float wx, wy;
    if (!on_plane(fp.dxo, fp.dxd, lod.gx, wx)) return false;
    if (!on_plane(fp.dyo, fp.dyd, lod.gy, wy)) return false;
    lod.kind = TexLodKind::Grad;
    width = fmaxr(wx, wy);
    return true;
  }
  // Straight-alpha Porter-Duff over, src/raycast.rs:754-768.
  static V4 over(V4 src, V4 dst) {
    float a = clampr(src[3], 0.0f, 1.0f), ad = clampr(dst[3], 0.0f, 1.0f);
    float ao = a + ad * (1.0f - a);
    if (ao <= 0.0f) return V4{{0.0f, 0.0f, 0.0f, 0.0f}};
    V4 c;
    for (int k = 0; k < 3; ++k) c[k] = (src[k] * a + dst[k] * ad * (1.0f - a)) / ao;
    c[3] = ao;
    return c;
  }
  // attenuation_sigma, src/raycast.rs:744-751.
  static V3 attenuation_sigma(V3 c, float distance) {
    if (!(std::isfinite(distance) && distance > 0.0f)) return {0.0f, 0.0f, 0.0f};
    return {-std::log(clampr(c.x, 1.0e-6f, 1.0f)) / distance, -std::log(clampr(c.y, 1.0e-6f, 1.0f)) / distance,
            -std::log(clampr(c.z, 1.0e-6f, 1.0f)) / distance};
  }
  V4 miss(const RayState &st) const {
    if (st.camera) return V4{{bg[0], bg[1], bg[2], bg[3]}};
    return V4{{ambient, ambient, ambient, 1.0f}};
  }
  bool radiance(V3 o, V3 d, const Footprint &fp, const RayState &st, V4 &c) const {
    const bool cull = !st.inside;
    Hit hit;
    auto filter = [&](const Hit &h) {
      if (st.has_skip && h.global == st.skip) return false;
      if (cull && !h.front && !ts->material_of(h).double_sided) return false;
      return !masked_out(h);
    };
    if (!ts->closest_hit_filtered(o, d, 0.0f, INF, filter, hit)) return false;
    c = shade(d, hit, fp, st);
    if (st.inside) {
      c[0] *= std::exp(-st.sigma.x * hit.t);
      c[1] *= std::exp(-st.sigma.y * hit.t);
      c[2] *= std::exp(-st.sigma.z * hit.t);
    }
    return true;
  }
  V3 secondary(V3 o, V3 d, const Footprint &fp, const RayState &st) const {
    V4 c;
    if (!radiance(o, d, fp, st, c)) c = miss(st);
    return {c[0], c[1], c[2]};
  }
  V4 shade(V3 d, const Hit &hit, const Footprint &fp, const RayState &st) const {
    Surface surf = ts->surface(hit);
    TexLod lod;
    float width = 0.0f;
    if (fp.diff) {
      if (!barycentric_differentials(hit, fp, lod, width)) {
        lod = TexLod{};
        width = 0.0f;
      }
    } else {
      float w = fmaxr(fp.width + fp.spr * hit.t, 0.0f);
      lod.kind = TexLodKind::Cone;
      lod.width = w;
      lod.dir = d;
      width = w;
    }
    const pt_material &pm = ts->material_of(hit);
    MaterialSample m = ts->material_oriented(hit, surf, lod, !hit.front);
    V3 p = surf.position;
    V3 ng = hit.front ? surf.geometric_normal : scale(surf.geometric_normal, -1.0f);
    V3 n = m.normal;
    V3 v = scale(d, -1.0f);
    RayState skip_st;
    skip_st.has_skip = true;
    skip_st.skip = hit.global;
    Footprint bounce;
    bounce.diff = false;
    bounce.width = width;
    bounce.spr = spread;
    const bool can_bounce = st.depth < max_depth;
    float r0 = (m.ior - 1.0f) / (m.ior + 1.0f);
    const float f0_d = r0 * r0;
    auto next = [&](bool inside, V3 sigma) {
      RayState s;
      s.depth = st.depth + 1;
      s.layers = st.layers;
      s.camera = false;
      s.inside = inside;
      s.sigma = sigma;
      s.has_skip = true;
      s.skip = hit.global;
      return s;
    };
    const V3 neg_ng = scale(ng, -1.0f);

    if (st.inside && !hit.front && m.transmission > 0.0f && m.thickness > 0.0f) {
      if (!can_bounce) {
        V4 e = miss(next(false, {0, 0, 0}));
        return V4{{e[0], e[1], e[2], 1.0f}};
      }
      float cos_i = clampr(dot(v, n), 0.0f, 1.0f);
      V3 t;
      if (refract(d, n, m.ior, t)) {
        float sin2_t = m.ior * m.ior * (1.0f - cos_i * cos_i);
        float f = schlick(f0_d, std::sqrt(fmaxr(1.0f - sin2_t, 0.0f)));
        V3 out = secondary(Integrator::offset_ray_origin(p, neg_ng), t, bounce, next(false, {0, 0, 0}));
        V3 inn = secondary(Integrator::offset_ray_origin(p, ng), reflect(d, n), bounce, next(true, st.sigma));
        return V4{{f * inn.x + (1.0f - f) * out.x, f * inn.y + (1.0f - f) * out.y, f * inn.z + (1.0f - f) * out.z,
                   1.0f}};
      }
      V3 inn = secondary(Integrator::offset_ray_origin(p, ng), reflect(d, n), bounce, next(true, st.sigma));
      return V4{{inn.x, inn.y, inn.z, 1.0f}};
    }

    const float *col = m.base_color;
    const float alpha = pm.alpha_mode == PT_ALPHA_BLEND ? clampr(col[3], 0.0f, 1.0f) : 1.0f;
    float out[3] = {0.0f, 0.0f, 0.0f};
    if (m.unlit) {
      out[0] = col[0];
      out[1] = col[1];
      out[2] = col[2];
    } else {
      BrdfParams params = metallic_roughness({col[0], col[1], col[2]}, m.metallic, m.roughness, f0_d);
      float kt = (can_bounce && m.transmission > 0.0f) ? m.transmission : 0.0f;
      params.c_diff = scale(params.c_diff, 1.0f - kt);
      float g = 0.0f;
      if (can_bounce && m.roughness < cutoff) {
        float x = 1.0f - m.roughness / cutoff;
        g = x * x;
      }
      const float cd[3] = {params.c_diff.x, params.c_diff.y, params.c_diff.z};
      const float f0[3] = {params.f0.x, params.f0.y, params.f0.z};
      const float em[3] = {m.emissive.x, m.emissive.y, m.emissive.z};
      for (int k = 0; k < 3; ++k) out[k] = em[k] + ambient * m.occlusion * (cd[k] + (1.0f - g) * f0[k]);
      V3 direct = direct_light(p, n, ng, v, params, skip_st);
      out[0] += direct.x;
      out[1] += direct.y;
      out[2] += direct.z;
      if (g > 0.0f) {
        float n_dot_v = clampr(dot(n, v), 0.0f, 1.0f);
        V3 f = f_schlick3(params.f0, n_dot_v);
        V3 r = reflect(d, n);
        if (dot(r, ng) <= 0.0f) r = reflect(d, ng);
        V3 l = secondary(Integrator::offset_ray_origin(p, ng), r, bounce, next(st.inside, st.sigma));
        out[0] += g * f.x * l.x;
        out[1] += g * f.y * l.y;
        out[2] += g * f.z * l.z;
      }
      if (kt > 0.0f) {
        float share = kt * (1.0f - m.metallic);
        float cos_i = clampr(dot(v, n), 0.0f, 1.0f);
        V3 through = Integrator::offset_ray_origin(p, neg_ng);
        float f;
        V3 l;
        if (m.thickness > 0.0f && hit.front) {
          V3 sigma = attenuation_sigma(m.attenuation_color, m.attenuation_distance);
          V3 t;
          if (refract(d, n, 1.0f / m.ior, t)) {
            f = schlick(f0_d, cos_i);
            l = secondary(through, t, bounce, next(true, sigma));
          } else {
            f = 1.0f;
            l = {0.0f, 0.0f, 0.0f};
          }
        } else {
          RayState st2 = next(st.inside, st.sigma);
          st2.layers = st.layers + 1;
          f = schlick(f0_d, cos_i);
          l = secondary(through, d, fp, st2);
        }
        out[0] += share * (1.0f - f) * col[0] * l.x;
        out[1] += share * (1.0f - f) * col[1] * l.y;
        out[2] += share * (1.0f - f) * col[2] * l.z;
      }
    }
    if (alpha >= 1.0f) return V4{{out[0], out[1], out[2], 1.0f}};
    V4 dst;
    if (st.layers < kMaxLayers) {
      RayState st2 = st;
      st2.layers = st.layers + 1;
      st2.has_skip = true;
      st2.skip = hit.global;
      if (!radiance(Integrator::offset_ray_origin(p, neg_ng), d, fp, st2, dst)) dst = miss(st);
    } else {
      dst = miss(st);
    }
    return over(V4{{out[0], out[1], out[2], alpha}}, dst);
  }
  bool pbr_pixel(float px, float py, V4 &c) const {
    V3 o, d;
    primary_ray(px, py, o, d);
    Footprint fp;
    primary_ray(px + 1.0f, py, fp.dxo, fp.dxd);
    primary_ray(px, py + 1.0f, fp.dyo, fp.dyd);
    return radiance(o, d, fp, RayState{}, c);
  }

  bool legacy(V3 o, V3 d, V4 &c) const {
    Hit hit;
    if (!ts->closest_hit_filtered(o, d, 0.0f, INF, [](const Hit &) { return true; }, hit)) return false;
    const Item &it = ts->item_of(hit);
    const pt_material &mat = ts->material_of(hit);
    const V4 base{{mat.base_color[0], mat.base_color[1], mat.base_color[2], mat.base_color[3]}};
    const size_t b0 = 3 * (size_t)hit.tri;
    switch (mode) {
      case PT_SHADE_FLAT:
        c = base;
        return true;
      case PT_SHADE_WIREFRAME: {
        float m = INF;
        for (int k = 0; k < 3; ++k) m = fminr(m, hit.bary[k]);
        if (m > kWireEdge) return false;
        c = base;
        return true;
      }
      case PT_SHADE_GOURAUD: {
        V4 ca = shade_pixel(base, corner_normal(it, b0, hit));
        V4 cb = shade_pixel(base, corner_normal(it, b0 + 1, hit));
        V4 cc = shade_pixel(base, corner_normal(it, b0 + 2, hit));
        for (int k = 0; k < 4; ++k) c[k] = ca[k] * hit.bary[0] + cb[k] * hit.bary[1] + cc[k] * hit.bary[2];
        return true;
      }
      case PT_SHADE_NORMAL_DEBUG: {
        V3 n = normalise(hit_normal(it, hit));
        c = V4{{lut[normal_byte(n.x)], lut[normal_byte(n.y)], lut[normal_byte(n.z)], 1.0f}};
        return true;
      }
      case PT_SHADE_DEPTH_DEBUG: {
        V3 pp = interp3v(it.positions, b0, hit.bary);
        float g = lut[depth_byte(ndc_z(dot(sub(pp, cv(cam.eye)), cv(cam.forward))))];
        c = V4{{g, g, g, 1.0f}};
        return true;
      }
      default:
        c = whitted(d, hit, 0);
        return true;
    }
  }
};
}  // namespace

}  // namespace oracle

using namespace oracle;

extern "C" {

// RenderBackend::Raycast render (legacy modes): HDR (w*h*4 floats) and/or
// RGBA8 (w*h*4 bytes); returns 0, or -1 for options it does not cover.
int oracle_raycast(const pt_scene_desc *desc, const pt_camera *cam, const pt_raycast_options *o, float *hdr,
                   uint8_t *rgba) {
  if (o->shading > PT_SHADE_PBR || o->aa < 1 || o->aa > 8) return -1;
  Scene sc(*desc);
  Raycaster rc;
  rc.ts = &sc;
  rc.cam = *cam;
  rc.rw = o->width * o->aa;
  rc.rh = o->height * o->aa;
  rc.mode = o->shading;
  rc.max_depth = std::min(o->max_ray_depth, kDepthCap);
  {
    const float deg = 3.14159265358979323846f / 180.0f;
    float az = o->light_azimuth_deg * deg, el = o->light_elevation_deg * deg;
    float cos_el = std::cos(el);
    rc.light = normalise({cos_el * std::sin(az), std::sin(el), cos_el * std::cos(az)});
  }
  rc.intensity = o->light_intensity;
  rc.near_p = o->near_plane;
  rc.far_p = o->far_plane;
  for (int i = 0; i < 256; ++i) rc.lut[i] = srgb_to_linear_f((float)i / 255.0f);
  rc.ambient = std::isfinite(o->ambient) ? fmaxr(o->ambient, 0.0f) : 0.0f;
  rc.cutoff = std::isfinite(o->reflection_roughness_cutoff) ? clampr(o->reflection_roughness_cutoff, 0.0f, 1.0f) : 0.0f;
  rc.shadows = o->shadows != 0;
  // trace::pixel_spread, src/trace.rs:1139-1146.
  rc.spread = cam->projection == PT_PERSPECTIVE ? std::atan(2.0f * cam->half_h / (float)std::max(rc.rh, 1u)) : 0.0f;
  for (int k = 0; k < 3; ++k) rc.bg[k] = rc.lut[o->background[k]];
  rc.bg[3] = (float)o->background[3] / 255.0f;
  const size_t ns = (size_t)rc.rw * rc.rh;
  std::vector<V4> col(ns);
  std::vector<uint8_t> cov(ns, 0);
  const unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  std::atomic<size_t> next{0};
  auto work = [&] {
    for (size_t y; (y = next.fetch_add(1)) < rc.rh;)
      for (uint32_t x = 0; x < rc.rw; ++x) {
        V3 ro, rd;
        rc.primary_ray((float)x + 0.5f, (float)y + 0.5f, ro, rd);
        V4 c{{0, 0, 0, 0}};
        bool hit = o->shading == PT_SHADE_PBR ? rc.pbr_pixel((float)x + 0.5f, (float)y + 0.5f, c) : rc.legacy(ro, rd, c);
        col[y * rc.rw + x] = hit ? c : V4{{0, 0, 0, 0}};
        cov[y * rc.rw + x] = hit ? 1 : 0;
      }
  };
  std::vector<std::thread> pool;
  for (unsigned k = 1; k < nt; ++k) pool.emplace_back(work);
  work();
  for (auto &th : pool) th.join();
  const bool display = o->shading == PT_SHADE_NORMAL_DEBUG || o->shading == PT_SHADE_DEPTH_DEBUG;
  const uint32_t tm = display ? (uint32_t)PT_TONE_CLAMP : o->tone_map;
  const float exposure = display ? 1.0f : o->exposure;
  float bg[4] = {rc.lut[o->background[0]], rc.lut[o->background[1]], rc.lut[o->background[2]],
                 (float)o->background[3] / 255.0f};
  const uint32_t aa = o->aa;
  const float n = (float)(aa * aa);
  for (uint32_t oy = 0; oy < o->height; ++oy)
    for (uint32_t ox = 0; ox < o->width; ++ox) {
      float pre_h[3] = {0, 0, 0}, str_h[3] = {0, 0, 0}, a_h = 0.0f;
      float pre_d[3] = {0, 0, 0}, str_d[3] = {0, 0, 0}, a_d = 0.0f;
      for (uint32_t j = 0; j < aa; ++j)
        for (uint32_t i = 0; i < aa; ++i) {
          size_t si = ((size_t)oy * aa + j) * rc.rw + (size_t)ox * aa + i;
          float ch[4] = {bg[0], bg[1], bg[2], bg[3]}, cd[4] = {bg[0], bg[1], bg[2], bg[3]};
          if (cov[si]) {
            const V4 &c = col[si];
            for (int k = 0; k < 4; ++k) ch[k] = c[k];
            V3 m = tone_apply(tm, {c[0] * exposure, c[1] * exposure, c[2] * exposure});
            cd[0] = m.x;
            cd[1] = m.y;
            cd[2] = m.z;
            cd[3] = clampr(c[3], 0.0f, 1.0f);
          }
          for (int k = 0; k < 3; ++k) {
            pre_h[k] += ch[k] * ch[3];
            str_h[k] += ch[k];
            pre_d[k] += cd[k] * cd[3];
            str_d[k] += cd[k];
          }
          a_h += ch[3];
          a_d += cd[3];
        }
      const size_t op = (size_t)oy * o->width + ox;
      float oh[4], od[4];
      if (a_h > 0.0f) {
        for (int k = 0; k < 3; ++k) oh[k] = pre_h[k] / a_h;
        oh[3] = a_h / n;
      } else {
        for (int k = 0; k < 3; ++k) oh[k] = str_h[k] / n;
        oh[3] = 0.0f;
      }
      if (a_d > 0.0f) {
        for (int k = 0; k < 3; ++k) od[k] = pre_d[k] / a_d;
        od[3] = a_d / n;
      } else {
        for (int k = 0; k < 3; ++k) od[k] = str_d[k] / n;
        od[3] = 0.0f;
      }
      if (hdr)
        for (int k = 0; k < 4; ++k) hdr[4 * op + k] = oh[k];
      if (rgba) {
        for (int k = 0; k < 3; ++k) rgba[4 * op + k] = linear_to_srgb_byte(od[k]);
        rgba[4 * op + 3] = (uint8_t)std::round(clampr(od[3], 0.0f, 1.0f) * 255.0f);
      }
    }
  return 0;
}

// The glTF metallic-roughness BRDF of src/brdf.rs: `params` = c_diff[3],
// f0[3], alpha of BrdfParams::metallic_roughness; `out` = eval(n, v, l).
void oracle_gltf_brdf(const float base[3], float metallic, float roughness, float f0_dielectric, const float n[3],
                      const float v[3], const float l[3], float params[7], float out[3]) {
  Raycaster::BrdfParams p =
      Raycaster::metallic_roughness({base[0], base[1], base[2]}, metallic, roughness, f0_dielectric);
  V3 e = Raycaster::brdf_eval(p, {n[0], n[1], n[2]}, {v[0], v[1], v[2]}, {l[0], l[1], l[2]});
  const float pv[7] = {p.c_diff.x, p.c_diff.y, p.c_diff.z, p.f0.x, p.f0.y, p.f0.z, p.alpha};
  for (int k = 0; k < 7; ++k) params[k] = pv[k];
  out[0] = e.x;
  out[1] = e.y;
  out[2] = e.z;
}
float oracle_gltf_d_ggx(float n_dot_h, float alpha) { return Raycaster::gltf_d_ggx(n_dot_h, alpha); }
void oracle_gltf_schlick(const float f0[3], float v_dot_h, float out[3]) {
  V3 f = Raycaster::f_schlick3({f0[0], f0[1], f0[2]}, v_dot_h);
  out[0] = f.x;
  out[1] = f.y;
  out[2] = f.z;
}

void *oracle_scene_create(const pt_scene_desc *desc) {
  try {
    return new Scene(*desc);
  } catch (...) {
    return nullptr;
  }
}
void oracle_scene_destroy(void *s) { delete (Scene *)s; }
uint64_t oracle_scene_triangles(const void *s) { return ((const Scene *)s)->triangle_count(); }
void *oracle_env_create(const pt_environment *env) { return new EnvironmentMap(*env); }
void oracle_env_destroy(void *e) { delete (EnvironmentMap *)e; }

// PathTracer::refine over a caller-owned f64 accumulator (width*height*4):
// threads pull 4-row bands, each pixel runs samples first..first+n in order.
int oracle_refine(const void *scene, const void *env, const pt_camera *cam, const pt_render_options *opts,
                  uint32_t first, uint32_t samples, int threads, double *accum, uint64_t *ray_counts) {
  const Scene *sc = (const Scene *)scene;
  Integrator base = make_integrator(sc, (const EnvironmentMap *)env, *cam, *opts);
  uint32_t w = base.width, h = base.height;
  const uint32_t BAND_ROWS = 4;
  uint32_t bands = (h + BAND_ROWS - 1) / BAND_ROWS;
  std::atomic<uint32_t> next{0};
  std::atomic<uint64_t> ext{0}, sh{0};
  int nthreads = std::max(1, std::min<int>(threads > 0 ? threads : (int)std::thread::hardware_concurrency(),
                                           (int)(h / BAND_ROWS + 1)));
  auto work = [&]() {
    Integrator it = base;
    for (;;) {
      uint32_t band = next.fetch_add(1);
      if (band >= bands) break;
      for (uint32_t y = band * BAND_ROWS; y < std::min(h, (band + 1) * BAND_ROWS); ++y)
        for (uint32_t x = 0; x < w; ++x) {
          double *px = accum + ((size_t)y * w + x) * 4;
          for (uint32_t si = 0; si < samples; ++si) {
            V3 c;
            if (it.sample(x, y, first + si, c)) {
              px[0] += (double)c.x;
              px[1] += (double)c.y;
              px[2] += (double)c.z;
              px[3] += 1.0;
            }
          }
        }
    }
    ext += it.ext_rays;
    sh += it.shadow_rays;
  };
  if (nthreads <= 1) {
    work();
  } else {
    std::vector<std::thread> pool;
    for (int i = 0; i < nthreads; ++i) pool.emplace_back(work);
    for (auto &t : pool) t.join();
  }
  if (ray_counts) {
    ray_counts[0] = ext.load();
    ray_counts[1] = sh.load();
  }
  return 0;
}

// refine over a strided subset of rows (row0 + i * stride, i < count) of the
// full frame: the bounded CPU baseline sample. accum holds width*count*4.
int oracle_refine_rows(const void *scene, const void *env, const pt_camera *cam, const pt_render_options *opts,
                       uint32_t row0, uint32_t stride, uint32_t count, uint32_t first, uint32_t samples, int threads,
                       double *accum, uint64_t *ray_counts) {
  const Scene *sc = (const Scene *)scene;
  Integrator base = make_integrator(sc, (const EnvironmentMap *)env, *cam, *opts);
  uint32_t w = base.width;
  std::atomic<uint32_t> next{0};
  std::atomic<uint64_t> ext{0}, sh{0};
  int nthreads = std::max(1, std::min<int>(threads > 0 ? threads : (int)std::thread::hardware_concurrency(),
                                           (int)count));
  auto work = [&]() {
    Integrator it = base;
    for (;;) {
      uint32_t r = next.fetch_add(1);
      if (r >= count) break;
      uint32_t y = row0 + r * stride;
      if (y >= base.height) continue;
      for (uint32_t x = 0; x < w; ++x) {
        double *px = accum + ((size_t)r * w + x) * 4;
        for (uint32_t si = 0; si < samples; ++si) {
          V3 c;
          if (it.sample(x, y, first + si, c)) {
            px[0] += (double)c.x;
            px[1] += (double)c.y;
            px[2] += (double)c.z;
            px[3] += 1.0;
          }
        }
      }
    }
    ext += it.ext_rays;
    sh += it.shadow_rays;
  };
  std::vector<std::thread> pool;
  for (int i = 0; i < nthreads; ++i) pool.emplace_back(work);
  for (auto &t : pool) t.join();
  if (ray_counts) {
    ray_counts[0] = ext.load();
    ray_counts[1] = sh.load();
  }
  return 0;
}

// One sample of one pixel (radiance, covered flag); for per-sample checks.
int oracle_sample(const void *scene, const void *env, const pt_camera *cam, const pt_render_options *opts, uint32_t x,
                  uint32_t y, uint32_t index, float out_rgb[3]) {
  Integrator it = make_integrator((const Scene *)scene, (const EnvironmentMap *)env, *cam, *opts);
  V3 c;
  bool cov = it.sample(x, y, index, c);
  out_rgb[0] = c.x;
  out_rgb[1] = c.y;
  out_rgb[2] = c.z;
  return cov ? 1 : 0;
}

void oracle_resolve_hdr(const double *accum, uint32_t samples, const pt_render_options *o, float *out) {
  float bg[4];
  bg_linear(*o, bg);
  size_t n = (size_t)std::max(o->width, 1u) * std::max(o->height, 1u);
  for (size_t i = 0; i < n; ++i) {
    float px[4];
    if (!resolve_pixel(accum + 4 * i, samples, bg, false, *o, px)) std::memcpy(px, bg, sizeof px);
    std::memcpy(out + 4 * i, px, sizeof px);
  }
}

void oracle_resolve_image(const double *accum, uint32_t samples, const pt_render_options *o, uint8_t *out) {
  float bg[4];
  bg_linear(*o, bg);
  size_t n = (size_t)std::max(o->width, 1u) * std::max(o->height, 1u);
  for (size_t i = 0; i < n; ++i) {
    float c[4];
    if (!resolve_pixel(accum + 4 * i, samples, bg, true, *o, c)) {
      std::memcpy(out + 4 * i, o->background, 4);
      continue;
    }
    for (int k = 0; k < 3; ++k) out[4 * i + k] = linear_to_srgb_byte(c[k]);
    out[4 * i + 3] = (uint8_t)f2usize(std::round(clampr(c[3], 0.0f, 1.0f) * 255.0f));
  }
}

// Primary (k = 0) closest hit of sample `index` for every pixel, with the
// camera-ray acceptance filter. global = UINT32_MAX on a miss.
void oracle_primary_hits(const void *scene, const pt_camera *cam, const pt_render_options *opts, uint32_t index,
                         uint32_t *out_global, float *out_t, float *out_bary) {
  Integrator it = make_integrator((const Scene *)scene, nullptr, *cam, *opts);
  for (uint32_t y = 0; y < it.height; ++y)
    for (uint32_t x = 0; x < it.width; ++x) {
      Sampler s(it.pt.seed, x, y, index);
      float p0[4];
      s.pattern(0, p0);
      V3 o, d;
      it.primary_ray((float)x + p0[0], (float)y + p0[1], o, d);
      Hit h;
      size_t i = (size_t)y * it.width + x;
      if (it.ts->closest_hit_filtered(o, d, 0.0f, INF, [&](const Hit &c) { return it.accept(c, s, 0, true); }, h)) {
        out_global[i] = h.global;
        out_t[i] = h.t;
        if (out_bary)
          for (int k = 0; k < 3; ++k) out_bary[3 * i + k] = h.bary[k];
      } else {
        out_global[i] = UINT32_MAX;
        out_t[i] = INF;
      }
    }
}

// Unfiltered closest hit / occlusion (TraceScene::closest_hit, ::occluded).
int oracle_closest_hit(const void *scene, const float o[3], const float d[3], float t_min, float t_max,
                       uint32_t *global, float *t, float bary[3], int *front) {
  const Scene *sc = (const Scene *)scene;
  Hit h;
  if (!sc->closest_hit_filtered({o[0], o[1], o[2]}, {d[0], d[1], d[2]}, t_min, t_max, [](const Hit &) { return true; },
                                h))
    return 0;
  *global = h.global;
  *t = h.t;
  for (int k = 0; k < 3; ++k) bary[k] = h.bary[k];
  *front = h.front ? 1 : 0;
  return 1;
}
int oracle_occluded(const void *scene, const float o[3], const float d[3], float t_min, float t_max) {
  const Scene *sc = (const Scene *)scene;
  return sc->occluded_filtered({o[0], o[1], o[2]}, {d[0], d[1], d[2]}, t_min, t_max, [](const Hit &) { return true; })
             ? 1
             : 0;
}
void oracle_surface(const void *scene, uint32_t global, const float bary[3], float out_pos[3], float out_ng[3],
                    float out_sn[3]) {
  const Scene *sc = (const Scene *)scene;
  float b[3] = {bary[0], bary[1], bary[2]};
  Hit h = sc->make_hit(global, 0.0f, b, true);
  Surface s = sc->surface(h);
  for (int k = 0; k < 3; ++k) {
    out_pos[k] = s.position[k];
    out_ng[k] = s.geometric_normal[k];
    out_sn[k] = s.shading_normal[k];
  }
}
// Material base colour / metallic / roughness at a hit (TexLod::Base).
void oracle_material_base(const void *scene, uint32_t global, const float bary[3], float out[6]) {
  const Scene *sc = (const Scene *)scene;
  float b[3] = {bary[0], bary[1], bary[2]};
  Hit h = sc->make_hit(global, 0.0f, b, true);
  Surface s = sc->surface(h);
  MaterialSample m = sc->material_oriented(h, s, TexLod{}, false);
  for (int k = 0; k < 4; ++k) out[k] = m.base_color[k];
  out[4] = m.metallic;
  out[5] = m.roughness;
}
void oracle_emissive_table(const void *scene, uint32_t *count, const uint32_t **tris, const float **pmf,
                           const float **cdf) {
  const Scene *sc = (const Scene *)scene;
  *count = (uint32_t)sc->emissive.tris.size();
  *tris = sc->emissive.tris.data();
  *pmf = sc->emissive.pmf.data();
  *cdf = sc->emissive.cdf.data();
}

// PreparedTexture::sample_lod on a one-texture scene; also reports the
// number of mip levels and the last level's first texel.
void oracle_texture_sample(const pt_texture *t, float u, float v, float lod, int srgb, float out[4],
                           uint32_t *levels, float top[4]) {
  pt_material m{};
  m.base_color_texture.texture = -1;
  pt_scene_desc d{};
  d.material_count = 1;
  d.materials = &m;
  d.texture_count = 1;
  d.textures = t;
  Scene sc(d);
  const Texture *tex = sc.textures[0].get();
  V4 r = tex->sample_lod(u, v, lod, srgb != 0);
  for (int k = 0; k < 4; ++k) out[k] = r[k];
  const std::vector<MipLevel> &mips = tex->mips(srgb != 0);
  if (levels) *levels = (uint32_t)mips.size();
  if (top)
    for (int k = 0; k < 4; ++k) top[k] = mips.back().texels[0][k];
}

// Every level of one chain of a texture (build_mips, src/texture.rs:324-383),
// concatenated level by level as RGBA f32; returns the texel count and
// writes at most `cap` texels.
uint64_t oracle_texture_mips(const pt_texture *t, int srgb, float *out, uint64_t cap) {
  pt_material m{};
  m.base_color_texture.texture = -1;
  pt_scene_desc d{};
  d.material_count = 1;
  d.materials = &m;
  d.texture_count = 1;
  d.textures = t;
  Scene sc(d);
  const std::vector<MipLevel> &mips = sc.textures[0]->mips(srgb != 0);
  uint64_t n = 0;
  for (const MipLevel &lv : mips)
    for (const auto &px : lv.texels) {
      if (n < cap)
        for (int k = 0; k < 4; ++k) out[4 * n + k] = px[k];
      ++n;
    }
  return n;
}

void oracle_sobol_owen_4d(uint32_t index, uint32_t seed, float out[4]) { sobol_owen_4d(index, seed, out); }
uint32_t oracle_sobol(uint32_t index, uint32_t dim) { return sobol(index, (int)dim); }
void oracle_sampler_pattern(uint32_t seed, uint32_t x, uint32_t y, uint32_t index, uint32_t pattern, float out[4]) {
  Sampler s(seed, x, y, index);
  s.pattern(pattern, out);
}
float oracle_sampler_coin(uint32_t seed, uint32_t x, uint32_t y, uint32_t index, uint32_t ray, uint32_t tri) {
  return Sampler(seed, x, y, index).coin(ray, tri);
}
uint32_t oracle_pcg_hash(uint32_t x) { return pcg_hash(x); }

float oracle_triangle_solid_angle(const float p[3], const float a[3], const float b[3], const float c[3]) {
  return triangle_solid_angle({p[0], p[1], p[2]}, {a[0], a[1], a[2]}, {b[0], b[1], b[2]}, {c[0], c[1], c[2]});
}
int oracle_sample_spherical_triangle(const float p[3], const float a[3], const float b[3], const float c[3], float u0,
                                     float u1, float out[3]) {
  V3 o;
  if (!sample_spherical_triangle({p[0], p[1], p[2]}, {a[0], a[1], a[2]}, {b[0], b[1], b[2]}, {c[0], c[1], c[2]}, u0,
                                 u1, o))
    return 0;
  out[0] = o.x;
  out[1] = o.y;
  out[2] = o.z;
  return 1;
}
void oracle_iridescent_fresnel(float outside, float film, const float f0[3], float thick, float cos1, float out[3]) {
  V3 r = iridescent_fresnel(outside, film, {f0[0], f0[1], f0[2]}, thick, cos1);
  out[0] = r.x;
  out[1] = r.y;
  out[2] = r.z;
}
void oracle_dispersion_iors(float ior, float dispersion, float out[3]) { dispersion_iors(ior, dispersion, out); }
const float *oracle_sheen_lut(void) { return sheen_lut().data(); }

float oracle_env_pdf(const void *env, const float d[3]) { return ((const EnvironmentMap *)env)->pdf({d[0], d[1], d[2]}); }
int oracle_env_sample(const void *env, float u0, float u1, float d[3], float le[3], float *pdf) {
  V3 dd, l;
  if (!((const EnvironmentMap *)env)->sample(u0, u1, dd, l, *pdf)) return 0;
  d[0] = dd.x;
  d[1] = dd.y;
  d[2] = dd.z;
  le[0] = l.x;
  le[1] = l.y;
  le[2] = l.z;
  return 1;
}

// MaterialSample as a flat float array for the BSDF tests (layout below).
// [0..4) base_color, 4 metallic, 5 roughness, [6..9) normal, 9 specular,
// [10..13) specular_color, 13 transmission, 14 thickness, 15 ior,
// 16 clearcoat, 17 clearcoat_roughness, [18..21) clearcoat_normal,
// [21..24) sheen_color, 24 sheen_roughness, 25 anisotropy,
// [26..29) anisotropy_direction, 29 iridescence, 30 iridescence_ior,
// 31 iridescence_thickness, 32 diffuse_transmission, [33..36) dt_color.
static MaterialSample ms_from(const float *a) {
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
  return m;
}
void oracle_bsdf_eval(const float *ms, const float v[3], const float ng[3], int front, const float l[3], float f[3],
                      float *pdf, float probs[6]) {
  Bsdf b(ms_from(ms), {v[0], v[1], v[2]}, {ng[0], ng[1], ng[2]}, front != 0);
  V3 ff;
  b.eval({l[0], l[1], l[2]}, ff, *pdf);
  f[0] = ff.x;
  f[1] = ff.y;
  f[2] = ff.z;
  if (probs)
    for (int i = 0; i < 6; ++i) probs[i] = b.probs[i];
}
// Batched eval over n directions (quadrature in the tests).
void oracle_bsdf_eval_many(const float *ms, const float v[3], const float ng[3], int front, uint32_t n, const float *l,
                           float *f, float *pdf) {
  Bsdf b(ms_from(ms), {v[0], v[1], v[2]}, {ng[0], ng[1], ng[2]}, front != 0);
  for (uint32_t i = 0; i < n; ++i) {
    V3 ff;
    b.eval({l[3 * i], l[3 * i + 1], l[3 * i + 2]}, ff, pdf[i]);
    f[3 * i] = ff.x;
    f[3 * i + 1] = ff.y;
    f[3 * i + 2] = ff.z;
  }
}
// Batched sample over n lobe/direction triples u[3*i..].
void oracle_bsdf_sample_many(const float *ms, const float v[3], const float ng[3], int front, uint32_t n,
                             const float *u, float *l, float *f, float *pdf, uint8_t *ok) {
  Bsdf b(ms_from(ms), {v[0], v[1], v[2]}, {ng[0], ng[1], ng[2]}, front != 0);
  for (uint32_t i = 0; i < n; ++i) {
    V3 ll, ff;
    float p = 0.0f;
    bool good = b.sample(u + 3 * i, ll, ff, p);
    ok[i] = good ? 1 : 0;
    if (!good) continue;
    l[3 * i] = ll.x;
    l[3 * i + 1] = ll.y;
    l[3 * i + 2] = ll.z;
    f[3 * i] = ff.x;
    f[3 * i + 1] = ff.y;
    f[3 * i + 2] = ff.z;
    pdf[i] = p;
  }
}

}  // extern "C"
