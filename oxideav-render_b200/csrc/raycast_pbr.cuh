// RenderBackend::Raycast, ShadingMode::Pbr on the device: Ctx::radiance /
// miss / secondary / shade of src/raycast.rs:518-740 with
// TraceScene::shadow_transmittance, ::direct_light and
// ::barycentric_differentials (src/trace.rs:947-1082) and the glTF 2.0
// metallic-roughness BRDF of src/brdf.rs.
//
// One thread per render sample. The reference recurses: a hit is shaded
// (ambient + emissive + direct light from every prepared light, with
// ray-traced hard shadows through MASK cut-outs, BLEND and transmissive
// occluders), then up to three rays continue from it — a mirror ray, a
// transmission ray (thin wall straight through, or a volume entered by
// Snell's law), and for BLEND surfaces the same ray behind the surface,
// composited with the straight-alpha over operator — and a volume's exit
// face splits into a refracted and an internally reflected ray. Every
// child's colour combines into its parent's sums in the reference's
// order, so the device evaluates the same expression tree post-order with
// an explicit stack of frames (one per pending radiance call that hit)
// instead of device recursion: the result is bit-identical to the
// recursion wherever the math functions agree.
//
// Nesting is bounded by the reference's caps: every child adds a
// reflection/refraction bounce (at most 16) or a see-through layer (at most
// 64), so a sample needs at most 81 frames. The main kernel keeps
// kPbrLocalFrames in local memory and hands the rare samples that nest
// deeper to a second kernel, which re-traces them with the full stack in a
// global buffer sized for its small fixed grid.
#pragma once

#include "raycast.cuh"

namespace ptd {

constexpr uint32_t kMaxLayers = 64;  // MAX_LAYERS, src/raycast.rs:126
constexpr int kPbrLocalFrames = 8;
constexpr int kPbrDeepFrames = (int)(kRayDepthCap + kMaxLayers + 1);
constexpr uint32_t kNoTriangle = 0xffffffffu;

// RayState (src/raycast.rs:331-345) of one radiance call.
struct PbrState {
  uint16_t depth, layers;
  uint8_t camera, inside;
  uint32_t skip;  // kNoTriangle: none
  V3 sigma;       // absorption of the volume the ray travels in (inside)
};

enum : uint8_t {
  // Where a child's colour goes in its parent.
  RET_ROOT = 0,
  RET_MIRROR,      // out += (g F) L
  RET_TRANSMIT,    // out += (share (1 - F) col) L
  RET_EXIT_OUT,    // volume exit: the refracted ray, kept for the final mix
  RET_EXIT_IN,     // volume exit: the internally reflected ray
  RET_BEHIND,      // BLEND: the surface composited over what is behind it
};
enum : uint8_t { PROG_SURFACE = 0, PROG_EXIT };
enum : uint8_t {
  // Surface program: the next child to consider. Exit program: 0 = refracted
  // ray next, 1 = internal ray next.
  PH_MIRROR = 0,
  PH_TRANSMIT,
  PH_BEHIND,
  PH_DONE,
};
enum : uint8_t { TR_NONE = 0, TR_THIN, TR_VOLUME, TR_TIR };

// One pending Ctx::shade of a radiance call that hit.
struct PbrFrame {
  PbrState st;
  float t;  // hit distance (volume absorption on return)
  uint8_t ret, prog, phase, trans;
  uint8_t fp_diff;             // footprint of the ray: differentials (camera) or a cone
  uint8_t has_mirror, has_exit_out;
  float fp_width, fp_spread;  // cone footprint of the ray
  float bwidth;               // cone width the bounces start with
  uint32_t g;                 // hit triangle: what every child skips
  V3 d;                       // ray direction
  V3 o_up, o_down;            // origins offset along +/- the oriented geometric normal
  V3 rdir, tdir;              // mirror / transmission (or exit refraction) directions
  float out[3], alpha;        // running colour; the frame's result once done
  float wr[3], wt[3];         // mirror / transmission weights (exit program: wr = refracted colour)
  V3 tsig;                    // absorption inside a volume the transmission ray enters
  float f;                    // exit program: Fresnel of the refraction
};

struct PbrParams {
  DevScene s;
  pt_camera cam;
  uint32_t rw, rh, max_depth, shadows;
  float ambient, cutoff, spread;
  float4 bg;             // linear background (camera misses)
  float4 *samples;       // rw * rh colours
  uint8_t *covered;      // rw * rh
  uint32_t *err;
  uint32_t *ovf_list;    // samples that need more than kPbrLocalFrames
  uint32_t *ovf_count;
  PbrFrame *deep;        // deep_slots * kPbrDeepFrames
  uint32_t deep_slots;
};

// Camera::primary_ray (src/camera.rs:489-514).
PT_DEV void primary_ray(const pt_camera &cam, uint32_t rw, uint32_t rh, float px, float py, V3 &o, V3 &d) {
  const float ndc_x = (px / fmaxf((float)rw, 1.0f)) * 2.0f - 1.0f;
  const float ndc_y = 1.0f - (py / fmaxf((float)rh, 1.0f)) * 2.0f;
  const V3 side = {cam.side[0], cam.side[1], cam.side[2]}, up = {cam.up[0], cam.up[1], cam.up[2]};
  const V3 fw = {cam.forward[0], cam.forward[1], cam.forward[2]};
  const V3 off = vadd(vscale(side, ndc_x * cam.half_w), vscale(up, ndc_y * cam.half_h));
  if (cam.projection == PT_PERSPECTIVE) {
    o = {cam.eye[0], cam.eye[1], cam.eye[2]};
    d = vnormalise(vadd(off, fw));
  } else {
    o = vadd(V3{cam.eye[0], cam.eye[1], cam.eye[2]}, off);
    d = fw;
  }
}

// ---------------------------------------------------------------- glTF BRDF
struct GltfBrdf {
  V3 c_diff, f0;
  float alpha;
};
// BrdfParams::metallic_roughness, src/brdf.rs:96-123.
PT_DEV GltfBrdf gltf_metallic_roughness(V3 base, float metallic, float roughness, float f0d) {
  const float m = clampr(metallic, 0.0f, 1.0f), r = clampr(roughness, 0.0f, 1.0f);
  GltfBrdf p;
  p.c_diff = {base.x * (1.0f - m), base.y * (1.0f - m), base.z * (1.0f - m)};
  p.f0 = {f0d + (base.x - f0d) * m, f0d + (base.y - f0d) * m, f0d + (base.z - f0d) * m};
  p.alpha = fmaxf(r * r, 1.0e-3f);
  return p;
}
// d_ggx / v_smith_ggx_correlated / f_schlick / eval, src/brdf.rs:31-148.
PT_DEV float gltf_d_ggx(float n_dot_h, float alpha) {
  const float a2 = alpha * alpha;
  const float d = n_dot_h * n_dot_h * (a2 - 1.0f) + 1.0f;
  return a2 / fmaxf(PI * d * d, 1.0e-12f);
}
PT_DEV float gltf_v_smith(float n_dot_l, float n_dot_v, float alpha) {
  const float a2 = alpha * alpha;
  const float gv = n_dot_l * sqrtf(n_dot_v * n_dot_v * (1.0f - a2) + a2);
  const float gl = n_dot_v * sqrtf(n_dot_l * n_dot_l * (1.0f - a2) + a2);
  const float s = gv + gl;
  return s > 0.0f ? 0.5f / s : 0.0f;
}
PT_DEV V3 gltf_schlick(V3 f0, float v_dot_h) {
  const float k = powi5(1.0f - clampr(v_dot_h, 0.0f, 1.0f));
  return {f0.x + (1.0f - f0.x) * k, f0.y + (1.0f - f0.y) * k, f0.z + (1.0f - f0.z) * k};
}
PT_DEV V3 gltf_eval(const GltfBrdf &p, V3 n, V3 v, V3 l) {
  const float n_dot_l = vdot(n, l);
  if (n_dot_l <= 0.0f) return vzero();
  const float n_dot_v = fmaxf(vdot(n, v), 1.0e-4f);
  V3 h = {l.x + v.x, l.y + v.y, l.z + v.z};
  const float hl = sqrtf(vdot(h, h));
  h = hl > 0.0f ? V3{h.x / hl, h.y / hl, h.z / hl} : n;
  const float n_dot_h = fmaxf(vdot(n, h), 0.0f), v_dot_h = fmaxf(vdot(v, h), 0.0f);
  const V3 f = gltf_schlick(p.f0, v_dot_h);
  const float spec = gltf_d_ggx(n_dot_h, p.alpha) * gltf_v_smith(n_dot_l, n_dot_v, p.alpha);
  return {((1.0f - f.x) * p.c_diff.x / PI + f.x * spec) * n_dot_l,
          ((1.0f - f.y) * p.c_diff.y / PI + f.y * spec) * n_dot_l,
          ((1.0f - f.z) * p.c_diff.z / PI + f.z * spec) * n_dot_l};
}

// ---------------------------------------------------------------- visibility
// Closest-hit filter of Ctx::radiance (src/raycast.rs:522-533): the surface
// the ray leaves, back faces of single-sided materials outside volumes, and
// MASK cut-outs are skipped.
struct AcceptPbr {
  const DevScene *s;
  uint32_t skip;
  bool cull;
  PT_DEV bool operator()(uint32_t g, uint32_t, float, float b0, float b1, float b2, bool front) const {
    if (g == skip) return false;
    const uint2 info = __ldg(s->tri_info + g);
    const pt_material &m = s->materials[info.x].m;
    if (cull && !front && !m.double_sided) return false;
    if (m.alpha_mode == PT_ALPHA_MASK && hit_alpha(*s, m, g, info.y, b0, b1, b2) < m.alpha_cutoff) return false;
    return true;
  }
};

// The part of material_oriented (src/trace.rs:700-923) the shadow filter
// reads: base colour, metallic, transmission and thickness at level 0.
PT_DEV void shadow_material(const DevScene &s, const pt_material &mat, uint32_t g, uint32_t flags, float b0, float b1,
                            float b2, float col[3], float &metallic, float &transmission, float &thickness) {
  const TexLod base{false, 0.0f, vzero()};
  float4 t;
  col[0] = mat.base_color[0];
  col[1] = mat.base_color[1];
  col[2] = mat.base_color[2];
  if (sample_binding(s, mat.base_color_texture, g, flags, b0, b1, b2, base, true, t)) {
    col[0] *= t.x;
    col[1] *= t.y;
    col[2] *= t.z;
  }
  if (flags & TRI_HAS_COLORS) {
    const float4 v = interp4(s.col, g, b0, b1, b2);
    col[0] *= v.x;
    col[1] *= v.y;
    col[2] *= v.z;
  }
  float m = mat.metallic;
  if (sample_binding(s, mat.metallic_roughness_texture, g, flags, b0, b1, b2, base, false, t)) m *= t.z;
  metallic = clampr(m, 0.0f, 1.0f);
  transmission = 0.0f;
  if (mat.ext_flags & PT_EXT_TRANSMISSION) {
    transmission = clampr(fin(mat.transmission_factor, 0.0f), 0.0f, 1.0f);
    if (sample_binding(s, mat.transmission_texture, g, flags, b0, b1, b2, base, false, t)) transmission *= t.x;
  }
  thickness = 0.0f;
  if (mat.ext_flags & PT_EXT_VOLUME) {
    thickness = fmaxf(fin(mat.thickness_factor, 0.0f), 0.0f);
    if (sample_binding(s, mat.thickness_texture, g, flags, b0, b1, b2, base, false, t)) thickness *= t.y;
  }
}

// Any-hit filter of TraceScene::shadow_transmittance (src/trace.rs:947-1005):
// multiplies the light each partial occluder passes into `tr` and stops the
// traversal once every channel is at most 1e-4. The product runs in f64 and
// is rounded once, so it does not depend on the order in which the tree
// reports the occluders.
struct AcceptShadowPbr {
  const DevScene *s;
  uint32_t skip;
  double *tr;
  PT_DEV bool operator()(uint32_t g, uint32_t, float, float b0, float b1, float b2, bool front) const {
    if (g == skip) return false;
    const uint2 info = __ldg(s->tri_info + g);
    const pt_material &mat = s->materials[info.x].m;
    float pass[3] = {0.0f, 0.0f, 0.0f};
    if (mat.alpha_mode == PT_ALPHA_MASK) {
      if (hit_alpha(*s, mat, g, info.y, b0, b1, b2) < mat.alpha_cutoff) return false;
    } else if (mat.alpha_mode == PT_ALPHA_BLEND) {
      const float a = 1.0f - clampr(hit_alpha(*s, mat, g, info.y, b0, b1, b2), 0.0f, 1.0f);
      pass[0] = pass[1] = pass[2] = a;
    }
    if ((mat.ext_flags & PT_EXT_TRANSMISSION) && isfinite(mat.transmission_factor) && mat.transmission_factor > 0.0f) {
      float col[3], metallic, transmission, thickness;
      shadow_material(*s, mat, g, info.y, b0, b1, b2, col, metallic, transmission, thickness);
      if (transmission > 0.0f) {
        if (thickness > 0.0f && !front) return false;
        const float kt = transmission * (1.0f - metallic);
        const float a = mat.alpha_mode == PT_ALPHA_BLEND ? pass[0] : 0.0f;
        for (int k = 0; k < 3; ++k) pass[k] = a + (1.0f - a) * kt * col[k];
      }
    }
    const double eps = (double)1.0e-4f;
    for (int k = 0; k < 3; ++k) tr[k] *= (double)clampr(pass[k], 0.0f, 1.0f);
    return tr[0] <= eps && tr[1] <= eps && tr[2] <= eps;
  }
};

// TraceScene::direct_light, src/trace.rs:1007-1048.
PT_DEV V3 pbr_direct_light(const PbrParams &P, V3 p, V3 n, V3 ng, V3 v, const GltfBrdf &bp, uint32_t skip,
                           uint32_t &err) {
  const DevScene &s = P.s;
  float out[3] = {0.0f, 0.0f, 0.0f};
  for (uint32_t i = 0; i < s.light_count; ++i) {
    LightSample ls;
    if (!light_sample(s.lights[i], p, ls)) continue;
    const V3 f = gltf_eval(bp, n, v, ls.l);
    if (f.x == 0.0f && f.y == 0.0f && f.z == 0.0f) continue;
    V3 vis = {1.0f, 1.0f, 1.0f};
    if (P.shadows) {
      const float side = vdot(ng, ls.l) >= 0.0f ? 1.0f : -1.0f;
      const V3 o = offset_ray_origin(p, {ng.x * side, ng.y * side, ng.z * side});
      const float t_max = isfinite(ls.distance) ? ls.distance * (1.0f - 1.0e-4f) : inf();
      double tr[3] = {1.0, 1.0, 1.0};
      TraversalStats st{0, 0};
      if (occluded(s, o, ls.l, 0.0f, t_max, AcceptShadowPbr{&s, skip, tr}, st, err))
        vis = vzero();
      else
        vis = {(float)tr[0], (float)tr[1], (float)tr[2]};
    }
    out[0] += f.x * ls.radiance.x * vis.x;
    out[1] += f.y * ls.radiance.y * vis.y;
    out[2] += f.z * ls.radiance.z * vis.z;
  }
  return {out[0], out[1], out[2]};
}

// barycentric_of, src/trace.rs:1120-1133.
PT_DEV bool barycentric_of(V3 q, V3 p0, V3 p1, V3 p2, float out[3]) {
  const V3 e1 = vsub(p1, p0), e2 = vsub(p2, p0), r = vsub(q, p0);
  const float d11 = vdot(e1, e1), d12 = vdot(e1, e2), d22 = vdot(e2, e2);
  const float r1 = vdot(r, e1), r2 = vdot(r, e2);
  const float det = d11 * d22 - d12 * d12;
  if (!isfinite(det) || fabsf(det) <= F32_MIN_POSITIVE) return false;
  const float u = (d22 * r1 - d12 * r2) / det;
  const float v = (d11 * r2 - d12 * r1) / det;
  out[0] = 1.0f - u - v;
  out[1] = u;
  out[2] = v;
  return true;
}

// TraceScene::barycentric_differentials (src/trace.rs:1050-1082) for the
// camera rays through the neighbouring samples (px + 1, py) and (px, py + 1).
PT_DEV bool barycentric_differentials(const PbrParams &P, uint32_t g, float b0, float b1, float b2, float px,
                                      float py, RayTexLod &lod, float &width) {
  const float *pp = P.s.pos + 9u * g;
  const V3 p0 = ld3(pp), p1 = ld3(pp + 3), p2 = ld3(pp + 6);
  const V3 ng = vcross(vsub(p1, p0), vsub(p2, p0));
  const float b[3] = {b0, b1, b2};
  const V3 p = {p0.x * b0 + p1.x * b1 + p2.x * b2, p0.y * b0 + p1.y * b1 + p2.y * b2,
                p0.z * b0 + p1.z * b1 + p2.z * b2};
  float w[2];
  for (int axis = 0; axis < 2; ++axis) {
    V3 o, d;
    primary_ray(P.cam, P.rw, P.rh, axis == 0 ? px + 1.0f : px, axis == 0 ? py : py + 1.0f, o, d);
    const float denom = vdot(ng, d);
    if (fabsf(denom) <= F32_MIN_POSITIVE) return false;
    const float t = vdot(ng, vsub(p0, o)) / denom;
    const V3 q = {o.x + d.x * t, o.y + d.y * t, o.z + d.z * t};
    float bq[3];
    if (!barycentric_of(q, p0, p1, p2, bq)) return false;
    const V3 wv = vsub(q, p);
    const float wl = sqrtf(vdot(wv, wv));
    if (!isfinite(wl)) return false;
    float *gd = axis == 0 ? lod.gx : lod.gy;
    for (int k = 0; k < 3; ++k) gd[k] = bq[k] - b[k];
    w[axis] = wl;
  }
  lod.grad = true;
  width = fmaxf(w[0], w[1]);
  return true;
}

// attenuation_sigma, src/raycast.rs:744-751.
PT_DEV V3 attenuation_sigma(V3 c, float distance) {
  if (!(isfinite(distance) && distance > 0.0f)) return vzero();
  return {-logf(clampr(c.x, 1.0e-6f, 1.0f)) / distance, -logf(clampr(c.y, 1.0e-6f, 1.0f)) / distance,
          -logf(clampr(c.z, 1.0e-6f, 1.0f)) / distance};
}

// over, src/raycast.rs:754-768: straight-alpha Porter-Duff over in linear
// space.
PT_DEV float4 pbr_over(float4 src, float4 dst) {
  const float a = clampr(src.w, 0.0f, 1.0f), ad = clampr(dst.w, 0.0f, 1.0f);
  const float ao = a + ad * (1.0f - a);
  if (ao <= 0.0f) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  return make_float4((src.x * a + dst.x * ad * (1.0f - a)) / ao, (src.y * a + dst.y * ad * (1.0f - a)) / ao,
                     (src.z * a + dst.z * ad * (1.0f - a)) / ao, ao);
}

// ---------------------------------------------------------------- shading
// The part of Ctx::shade (src/raycast.rs:578-740) before its first child
// ray: material, local terms and direct light, and everything the children
// need. Leaves f.phase at PH_DONE when the shade needs no child.
PT_DEV void pbr_enter(const PbrParams &P, PbrFrame &f, const Hit &h, float px, float py, uint32_t &err) {
  const DevScene &s = P.s;
  const uint2 info = __ldg(s.tri_info + h.g);
  const DevMaterial &dm = s.materials[info.x];
  const Surface surf = surface(s, h.g, h.b0, h.b1, h.b2, info.y);
  RayTexLod lod{false, 0.0f, vzero(), false, {0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}};
  float width = 0.0f;
  if (f.fp_diff) {
    if (!barycentric_differentials(P, h.g, h.b0, h.b1, h.b2, px, py, lod, width)) {
      lod.grad = false;
      width = 0.0f;
    }
  } else {
    const float w = fmaxf(f.fp_width + f.fp_spread * h.t, 0.0f);
    lod.cone = true;
    lod.width = w;
    lod.dir = f.d;
    width = w;
  }
  MaterialSample m;
  material_oriented<true>(s, dm, h.g, info.y, h.b0, h.b1, h.b2, surf.sn, lod, !h.front, m);
  const V3 p = surf.position;
  const V3 ng = h.front ? surf.ng : vscale(surf.ng, -1.0f);
  const V3 n = m.normal;
  const V3 d = f.d;
  const V3 v = vscale(d, -1.0f);
  f.bwidth = width;
  f.o_up = offset_ray_origin(p, ng);
  f.o_down = offset_ray_origin(p, vscale(ng, -1.0f));
  const bool can_bounce = f.st.depth < P.max_depth;
  const float r0 = (m.ior - 1.0f) / (m.ior + 1.0f);
  const float f0_d = r0 * r0;

  if (f.st.inside && !h.front && m.transmission > 0.0f && m.thickness > 0.0f) {
    // Leaving a volume through its boundary.
    f.prog = PROG_EXIT;
    f.alpha = 1.0f;
    if (!can_bounce) {
      f.out[0] = f.out[1] = f.out[2] = P.ambient;
      f.phase = PH_DONE;
      return;
    }
    const float cos_i = clampr(vdot(v, n), 0.0f, 1.0f);
    f.rdir = reflect_dir(d, n);
    V3 t;
    if (refract_dir(d, n, m.ior, t)) {
      const float sin2_t = m.ior * m.ior * (1.0f - cos_i * cos_i);
      f.f = schlick_scalar(f0_d, sqrtf(fmaxf(1.0f - sin2_t, 0.0f)));
      f.tdir = t;
      f.has_exit_out = 1;
      f.phase = 0;
    } else {
      f.has_exit_out = 0;
      f.phase = 1;
    }
    return;
  }

  f.prog = PROG_SURFACE;
  const pt_material &pm = dm.m;
  const float col[3] = {m.base_color[0], m.base_color[1], m.base_color[2]};
  f.alpha = pm.alpha_mode == PT_ALPHA_BLEND ? clampr(m.base_color[3], 0.0f, 1.0f) : 1.0f;
  f.has_mirror = 0;
  f.trans = TR_NONE;
  f.phase = PH_MIRROR;
  if (m.unlit) {
    f.out[0] = col[0];
    f.out[1] = col[1];
    f.out[2] = col[2];
    return;
  }
  GltfBrdf bp = gltf_metallic_roughness({col[0], col[1], col[2]}, m.metallic, m.roughness, f0_d);
  const float kt = (can_bounce && m.transmission > 0.0f) ? m.transmission : 0.0f;
  bp.c_diff = vscale(bp.c_diff, 1.0f - kt);
  float g = 0.0f;
  if (can_bounce && m.roughness < P.cutoff) {
    const float x = 1.0f - m.roughness / P.cutoff;
    g = x * x;
  }
  const float cd[3] = {bp.c_diff.x, bp.c_diff.y, bp.c_diff.z}, f0[3] = {bp.f0.x, bp.f0.y, bp.f0.z};
  const float em[3] = {m.emissive.x, m.emissive.y, m.emissive.z};
  for (int k = 0; k < 3; ++k) f.out[k] = em[k] + P.ambient * m.occlusion * (cd[k] + (1.0f - g) * f0[k]);
  const V3 direct = pbr_direct_light(P, p, n, ng, v, bp, h.g, err);
  f.out[0] += direct.x;
  f.out[1] += direct.y;
  f.out[2] += direct.z;
  if (g > 0.0f) {
    const V3 fr = gltf_schlick(bp.f0, clampr(vdot(n, v), 0.0f, 1.0f));
    V3 r = reflect_dir(d, n);
    // A normal-mapped normal sending the mirror ray under the surface:
    // reflect about the geometric normal.
    if (vdot(r, ng) <= 0.0f) r = reflect_dir(d, ng);
    f.rdir = r;
    f.wr[0] = g * fr.x;
    f.wr[1] = g * fr.y;
    f.wr[2] = g * fr.z;
    f.has_mirror = 1;
  }
  if (kt > 0.0f) {
    const float share = kt * (1.0f - m.metallic);
    const float cos_i = clampr(vdot(v, n), 0.0f, 1.0f);
    float fr;
    if (m.thickness > 0.0f && h.front) {
      // Entering a volume: Snell bend, absorption inside.
      f.tsig = attenuation_sigma(m.attenuation_color, m.attenuation_distance);
      V3 t;
      if (refract_dir(d, n, 1.0f / m.ior, t)) {
        fr = schlick_scalar(f0_d, cos_i);
        f.tdir = t;
        f.trans = TR_VOLUME;
      } else {
        fr = 1.0f;
        f.trans = TR_TIR;
      }
    } else {
      // Thin wall: straight through, footprint unchanged.
      fr = schlick_scalar(f0_d, cos_i);
      f.tdir = d;
      f.trans = TR_THIN;
    }
    for (int k = 0; k < 3; ++k) f.wt[k] = share * (1.0f - fr) * col[k];
  }
}

// A radiance call about to be traced.
struct PbrCall {
  V3 o, d;
  PbrState st;
  uint8_t ret, fp_diff;
  float fp_width, fp_spread;
};

PT_DEV PbrState pbr_next(const PbrFrame &f, bool inside, V3 sigma) {
  PbrState s;
  s.depth = (uint16_t)(f.st.depth + 1);
  s.layers = f.st.layers;
  s.camera = 0;
  s.inside = inside ? 1 : 0;
  s.sigma = sigma;
  s.skip = f.g;
  return s;
}

// The frame's next child call, if any; false when the frame is finished
// (its result in out / alpha).
PT_DEV bool pbr_next_child(const PbrParams &P, PbrFrame &f, PbrCall &c) {
  c.fp_diff = 0;
  c.fp_width = f.bwidth;
  c.fp_spread = P.spread;
  if (f.prog == PROG_EXIT) {
    if (f.phase == 0) {
      f.phase = 1;
      c.o = f.o_down;
      c.d = f.tdir;
      c.st = pbr_next(f, false, vzero());
      c.ret = RET_EXIT_OUT;
      return true;
    }
    if (f.phase == 1) {
      f.phase = PH_DONE;
      c.o = f.o_up;
      c.d = f.rdir;
      c.st = pbr_next(f, true, f.st.sigma);
      c.ret = RET_EXIT_IN;
      return true;
    }
    return false;
  }
  for (;;) {
    switch (f.phase) {
      case PH_MIRROR:
        f.phase = PH_TRANSMIT;
        if (f.has_mirror) {
          c.o = f.o_up;
          c.d = f.rdir;
          c.st = pbr_next(f, f.st.inside, f.st.sigma);
          c.ret = RET_MIRROR;
          return true;
        }
        break;
      case PH_TRANSMIT:
        f.phase = PH_BEHIND;
        if (f.trans == TR_TIR) {
          // Total internal reflection on entry: F = 1 and no ray.
          for (int k = 0; k < 3; ++k) f.out[k] += f.wt[k] * 0.0f;
        } else if (f.trans != TR_NONE) {
          c.o = f.o_down;
          c.d = f.tdir;
          c.ret = RET_TRANSMIT;
          if (f.trans == TR_VOLUME) {
            c.st = pbr_next(f, true, f.tsig);
          } else {
            c.st = pbr_next(f, f.st.inside, f.st.sigma);
            c.st.layers = (uint16_t)(f.st.layers + 1);
            c.fp_diff = f.fp_diff;
            c.fp_width = f.fp_width;
            c.fp_spread = f.fp_spread;
          }
          return true;
        }
        break;
      case PH_BEHIND:
        f.phase = PH_DONE;
        if (f.alpha >= 1.0f) {
          f.alpha = 1.0f;
          return false;
        }
        if (f.st.layers < kMaxLayers) {
          // BLEND: continue the ray behind the surface.
          c.o = f.o_down;
          c.d = f.d;
          c.st = f.st;
          c.st.layers = (uint16_t)(f.st.layers + 1);
          c.st.skip = f.g;
          c.fp_diff = f.fp_diff;
          c.fp_width = f.fp_width;
          c.fp_spread = f.fp_spread;
          c.ret = RET_BEHIND;
          return true;
        } else {
          const float4 dst = f.st.camera ? P.bg : make_float4(P.ambient, P.ambient, P.ambient, 1.0f);
          const float4 o = pbr_over(make_float4(f.out[0], f.out[1], f.out[2], f.alpha), dst);
          f.out[0] = o.x;
          f.out[1] = o.y;
          f.out[2] = o.z;
          f.alpha = o.w;
          return false;
        }
      default:
        return false;
    }
  }
}

// Folds a finished child's colour (`have` false: the child ray escaped)
// into its parent.
PT_DEV void pbr_combine(const PbrParams &P, PbrFrame &f, uint8_t ret, bool have, float4 c) {
  // Escaping secondary rays see the uniform environment (Ctx::miss of a
  // non-camera state); a BLEND continuation sees what its own ray sees.
  const float a = P.ambient;
  const float l[3] = {have ? c.x : a, have ? c.y : a, have ? c.z : a};
  switch (ret) {
    case RET_MIRROR:
      for (int k = 0; k < 3; ++k) f.out[k] += f.wr[k] * l[k];
      break;
    case RET_TRANSMIT:
      for (int k = 0; k < 3; ++k) f.out[k] += f.wt[k] * l[k];
      break;
    case RET_EXIT_OUT:
      for (int k = 0; k < 3; ++k) f.wr[k] = l[k];
      break;
    case RET_EXIT_IN:
      if (f.has_exit_out) {
        for (int k = 0; k < 3; ++k) f.out[k] = f.f * l[k] + (1.0f - f.f) * f.wr[k];
      } else {
        for (int k = 0; k < 3; ++k) f.out[k] = l[k];
      }
      f.alpha = 1.0f;
      break;
    case RET_BEHIND: {
      const float4 dst = have ? c : (f.st.camera ? P.bg : make_float4(a, a, a, 1.0f));
      const float4 o = pbr_over(make_float4(f.out[0], f.out[1], f.out[2], f.alpha), dst);
      f.out[0] = o.x;
      f.out[1] = o.y;
      f.out[2] = o.z;
      f.alpha = o.w;
      break;
    }
    default:
      break;
  }
}

// A finished frame's radiance: Beer-Lambert absorption over the hit
// distance when the ray travelled inside a volume (Ctx::radiance).
PT_DEV float4 pbr_result(const PbrFrame &f) {
  float4 c = make_float4(f.out[0], f.out[1], f.out[2], f.alpha);
  if (f.st.inside) {
    c.x *= expf(-f.st.sigma.x * f.t);
    c.y *= expf(-f.st.sigma.y * f.t);
    c.z *= expf(-f.st.sigma.z * f.t);
  }
  return c;
}

// Ctx::pixel for ShadingMode::Pbr: 1 covered (colour in `out`), 0 the camera
// ray escaped, -1 the sample needs more than `cap` frames.
PT_DEV int pbr_sample(const PbrParams &P, float px, float py, PbrFrame *fr, int cap, float4 &out, uint32_t &err) {
  PbrCall c;
  primary_ray(P.cam, P.rw, P.rh, px, py, c.o, c.d);
  c.st = PbrState{0, 0, 1, 0, kNoTriangle, vzero()};
  c.ret = RET_ROOT;
  c.fp_diff = 1;
  c.fp_width = 0.0f;
  c.fp_spread = 0.0f;
  int top = -1;
  for (;;) {
    Hit h;
    TraversalStats ts{0, 0};
    const bool hit = closest_hit(P.s, c.o, c.d, 0.0f, inf(), AcceptPbr{&P.s, c.st.skip, c.st.inside == 0}, h, ts, err);
    bool have = false;
    float4 val = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    uint8_t ret = c.ret;
    if (hit) {
      if (top + 1 >= cap) return -1;
      PbrFrame &f = fr[++top];
      f.st = c.st;
      f.t = h.t;
      f.ret = c.ret;
      f.fp_diff = c.fp_diff;
      f.fp_width = c.fp_width;
      f.fp_spread = c.fp_spread;
      f.g = h.g;
      f.d = c.d;
      pbr_enter(P, f, h, px, py, err);
      if (pbr_next_child(P, f, c)) continue;
      have = true;
      val = pbr_result(f);
      --top;
    }
    // Deliver upward until a frame launches another child.
    for (;;) {
      if (ret == RET_ROOT) {
        out = val;
        return have ? 1 : 0;
      }
      PbrFrame &f = fr[top];
      pbr_combine(P, f, ret, have, val);
      if (pbr_next_child(P, f, c)) break;
      have = true;
      val = pbr_result(f);
      ret = f.ret;
      --top;
    }
  }
}

PT_DEV void pbr_store(const PbrParams &P, uint64_t i, int r, float4 c) {
  P.samples[i] = r > 0 ? c : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  P.covered[i] = r > 0 ? 1 : 0;
}

// Every render sample with a kPbrLocalFrames-deep stack; samples that nest
// deeper are listed for k_raycast_pbr_deep.
__global__ void __launch_bounds__(128) k_raycast_pbr(PbrParams P) {
  const uint64_t n = (uint64_t)P.rw * P.rh;
  uint32_t err = 0;
  PbrFrame fr[kPbrLocalFrames];
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t y = (uint32_t)(i / P.rw), x = (uint32_t)(i - (uint64_t)y * P.rw);
    float4 c;
    const int r = pbr_sample(P, (float)x + 0.5f, (float)y + 0.5f, fr, kPbrLocalFrames, c, err);
    if (r < 0) {
      const uint32_t slot = atomicAdd(P.ovf_count, 1u);
      P.ovf_list[slot] = (uint32_t)i;
      pbr_store(P, i, 0, c);
    } else {
      pbr_store(P, i, r, c);
    }
  }
  if (err) atomicOr(P.err, err);
}

// The listed samples again, each thread with a full kPbrDeepFrames stack in
// the global buffer (deep_slots threads in all).
__global__ void __launch_bounds__(64) k_raycast_pbr_deep(PbrParams P) {
  const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= P.deep_slots) return;
  PbrFrame *fr = P.deep + (size_t)slot * kPbrDeepFrames;
  const uint32_t count = *P.ovf_count;
  uint32_t err = 0;
  for (uint32_t j = slot; j < count; j += P.deep_slots) {
    const uint64_t i = P.ovf_list[j];
    const uint32_t y = (uint32_t)(i / P.rw), x = (uint32_t)(i - (uint64_t)y * P.rw);
    float4 c;
    const int r = pbr_sample(P, (float)x + 0.5f, (float)y + 0.5f, fr, kPbrDeepFrames, c, err);
    if (r < 0) err |= ERR_STACK_OVERFLOW;
    pbr_store(P, i, r, c);
  }
  if (err) atomicOr(P.err, err);
}

}  // namespace ptd
