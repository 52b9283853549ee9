// Per-vertex path construction (Integrator::sample, src/pathtrace.rs:2004-2329)
// split into the three steps a wavefront schedules separately:
//   trace_extension  closest hit of the path's current ray (step 1);
//   shade            medium, miss, emission + MIS, material, NEE shadow-ray
//                    generation, BSDF sampling, roulette (steps 2-9);
//   shadow rays      resolved by a ShadowSink: traced in place by the
//                    megakernel, queued and traced by the shadow kernel in
//                    the wavefront.
// Every contribution is added to the path radiance in the reference's order
// (emission of vertex k, punctual lights 0.., the area sample, then vertex
// k+1), so the float sums round identically in both schedules.
#pragma once

#include "dev_scene.cuh"

namespace ptd {

struct PathState {
  V3 o, d;
  V3 beta, radiance;
  V3 prev_pos, sigma;
  float prev_pdf;
  uint32_t k;
  int32_t hero;        // -1 until a dispersive volume picks the channel
  uint32_t has_medium;
  uint32_t covered;    // primary ray found geometry
  Sampler smp;
};

struct ShadowRay {
  V3 o, d;
  float tmax;
  uint32_t ray_id, skip;
  V3 contrib;  // clamped contribution added when the ray is unoccluded
};

struct ThreadStats {
  uint32_t ext_rays, shadow_rays, ext_nodes, ext_tris, sh_nodes, sh_tris, err;
};

// Warp-reduces the per-thread counters into the launch's DevCounters.
PT_DEV void flush_stats(DevCounters *ctr, const ThreadStats &ts) {
  unsigned long long v[6] = {ts.ext_rays, ts.shadow_rays, ts.ext_nodes, ts.ext_tris, ts.sh_nodes, ts.sh_tris};
  unsigned int err = ts.err;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int k = 0; k < 6; ++k) v[k] += __shfl_down_sync(0xffffffffu, v[k], off);
    err |= __shfl_down_sync(0xffffffffu, err, off);
  }
  if ((threadIdx.x & 31) == 0) {
    unsigned long long *dst[6] = {&ctr->ext_rays, &ctr->shadow_rays, &ctr->ext_nodes,
                                  &ctr->ext_tris, &ctr->sh_nodes, &ctr->sh_tris};
#pragma unroll
    for (int k = 0; k < 6; ++k)
      if (v[k]) atomicAdd(dst[k], v[k]);
    if (err) atomicOr(&ctr->error_flags, err);
  }
}

PT_DEV V3 clamp_contrib(const DevRequest &rq, V3 c) {
  float m = max3(c);
  if (rq.clamp > 0.0f && m > rq.clamp) return vscale(c, rq.clamp / m);
  return c;
}
PT_DEV float power_heuristic(float a, float b) {
  float a2 = a * a, b2 = b * b;
  if (a2 + b2 > 0.0f && isfinite(a2 + b2)) return a2 / (a2 + b2);
  if (isinf(a)) return 1.0f;
  return 0.0f;
}
// offset_ray_origin (Waechter & Binder 2019), src/trace.rs:1152-1175.
PT_DEV V3 offset_ray_origin(V3 p, V3 n) {
  const float ORIGIN = 1.0f / 32.0f, FLOAT_SCALE = 1.0f / 65536.0f, INT_SCALE = 256.0f;
  float pc[3] = {p.x, p.y, p.z}, nc[3] = {n.x, n.y, n.z}, out[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    int32_t of_i = f2i32(INT_SCALE * nc[k]);
    uint32_t bits = __float_as_uint(pc[k]);
    uint32_t moved = pc[k] < 0.0f ? bits - (uint32_t)of_i : bits + (uint32_t)of_i;
    float p_i = __uint_as_float(moved);
    if (fabsf(pc[k]) < ORIGIN)
      out[k] = pc[k] + FLOAT_SCALE * nc[k];
    else if (isfinite(p_i))
      out[k] = p_i;
    else
      out[k] = pc[k];
  }
  return {out[0], out[1], out[2]};
}

// Camera::primary_ray, src/camera.rs:489-514.
PT_DEV void primary_ray(const DevRequest &rq, float px, float py, V3 &o, V3 &d) {
  const pt_camera &c = rq.cam;
  float ndc_x = (px / fmaxf((float)rq.width, 1.0f)) * 2.0f - 1.0f;
  float ndc_y = 1.0f - (py / fmaxf((float)rq.height, 1.0f)) * 2.0f;
  V3 side = {c.side[0], c.side[1], c.side[2]}, up = {c.up[0], c.up[1], c.up[2]};
  V3 off = vadd(vscale(side, ndc_x * c.half_w), vscale(up, ndc_y * c.half_h));
  V3 eye = {c.eye[0], c.eye[1], c.eye[2]}, fwd = {c.forward[0], c.forward[1], c.forward[2]};
  if (c.projection == PT_PERSPECTIVE) {
    o = eye;
    d = vnormalise(vadd(off, fwd));
  } else {
    o = vadd(eye, off);
    d = fwd;
  }
}

PT_DEV void init_path(const DevRequest &rq, uint32_t x, uint32_t y, uint32_t index, PathState &ps) {
  ps.smp.init(rq.seed, x, y, index);
  float p0[4];
  ps.smp.pattern(0, p0);
  primary_ray(rq, (float)x + p0[0], (float)y + p0[1], ps.o, ps.d);
  ps.beta = {1.0f, 1.0f, 1.0f};
  ps.radiance = vzero();
  ps.prev_pdf = 0.0f;
  ps.prev_pos = vzero();
  ps.sigma = vzero();
  ps.k = 0;
  ps.hero = -1;
  ps.has_medium = 0;
  ps.covered = 0;
}

// Integrator::accept (src/pathtrace.rs:1924-1934): the any-hit filter.
struct AcceptFilter {
  const DevScene *s;
  const Sampler *smp;
  uint32_t ray;
  bool primary;
  uint32_t skip;
  PT_DEV bool operator()(uint32_t g, uint32_t rflags, float, float b0, float b1, float b2, bool front) const {
    if (g == skip) return false;
    if (primary && !front && !(rflags & REC_DOUBLE_SIDED)) return false;
    if (rflags & REC_OPAQUE) return true;
    uint2 info = __ldg(s->tri_info + g);
    const pt_material &m = s->materials[info.x].m;
    float a = hit_alpha(*s, m, g, info.y, b0, b1, b2);
    if (m.alpha_mode == PT_ALPHA_MASK) return a >= m.alpha_cutoff;
    return smp->coin(ray, g) < a;
  }
};

PT_DEV bool trace_extension(const DevRequest &rq, const PathState &ps, Hit &hit, ThreadStats &ts) {
  const DevScene &s = *rq.scene;
  AcceptFilter acc{&s, &ps.smp, ps.k << 16, ps.k == 0, 0xffffffffu};
  TraversalStats st{0, 0};
  ts.ext_rays++;
  bool found = closest_hit(s, ps.o, ps.d, 0.0f, inf(), acc, hit, st, ts.err);
  ts.ext_nodes += st.nodes;
  ts.ext_tris += st.tris;
  return found;
}

PT_DEV bool trace_shadow(const DevRequest &rq, const PathState &ps, const ShadowRay &sr, ThreadStats &ts) {
  const DevScene &s = *rq.scene;
  AcceptFilter acc{&s, &ps.smp, sr.ray_id, false, sr.skip};
  TraversalStats st{0, 0};
  ts.shadow_rays++;
  bool occ = occluded(s, sr.o, sr.d, 0.0f, sr.tmax, acc, st, ts.err);
  ts.sh_nodes += st.nodes;
  ts.sh_tris += st.tris;
  return !occ;
}

// Integrator::emission, src/pathtrace.rs:1951-1966.
PT_DEV V3 emission(const DevScene &s, const DevMaterial &dm, uint32_t g, uint32_t flags, float b0, float b1, float b2) {
  const pt_material &m = dm.m;
  if (m.unlit || !dm.emissive_nonblack) return vzero();
  V3 e = {m.emissive[0], m.emissive[1], m.emissive[2]};
  float4 t;
  TexLod base{false, 0.0f, vzero()};
  if (sample_binding(s, m.emissive_texture, g, flags, b0, b1, b2, base, true, t)) e = vmul(e, {t.x, t.y, t.z});
  return e;
}

PT_DEV void tri_positions(const DevScene &s, uint32_t g, V3 &a, V3 &b, V3 &c) {
  const float *p = s.pos + 9u * g;
  a = ld3(p);
  b = ld3(p + 3);
  c = ld3(p + 6);
}

// Integrator::tri_pdf, src/pathtrace.rs:1972-1991, for emitter li with
// corners a, b, c whose solid angle seen from p is omega.
PT_DEV float tri_pdf_omega(const DevRequest &rq, uint32_t li, V3 a, V3 b, V3 c, float omega, V3 p, V3 q) {
  float sel = (1.0f - rq.p_env) * __ldg(rq.scene->em_pmf + li);
  if (omega >= 1.0e-4f) return sel / omega;
  V3 cr = vcross(vsub(b, a), vsub(c, a));
  float len = sqrtf(vdot(cr, cr));
  V3 to = vsub(q, p);
  float d2 = vdot(to, to);
  if (len <= 0.0f || d2 <= 0.0f) return 0.0f;
  float cs = fabsf(vdot(cr, to) / (len * sqrtf(d2)));
  if (cs <= 0.0f) return 0.0f;
  return sel * d2 / (0.5f * len * cs);
}
PT_DEV float tri_pdf(const DevRequest &rq, uint32_t li, uint32_t g, V3 p, V3 q) {
  V3 a, b, c;
  tri_positions(*rq.scene, g, a, b, c);
  return tri_pdf_omega(rq, li, a, b, c, triangle_solid_angle(p, a, b, c), p, q);
}

// Integrator::tri_pdf of the emissive triangle g hit at q from prev_pos
// (the light-sampling pdf of the emission MIS weight); 0 when g is not in
// the emissive table.
PT_DEV float emission_light_pdf(const DevRequest &rq, const DevScene &s, uint32_t g, V3 prev_pos, V3 q) {
  const uint32_t li = __ldg(s.em_lookup + g);
  return li != 0xffffffffu ? tri_pdf(rq, li, g, prev_pos, q) : 0.0f;
}

// Whether the request samples area lights (environment or emissive
// triangles) in its next-event estimation.
PT_DEV bool area_nee(const DevRequest &rq, const DevScene &s) {
  return rq.strategy != PT_BSDF_ONLY && (rq.env || s.em_count > 0);
}

// The area-set light sample of next-event estimation at p
// (Integrator::sample, src/pathtrace.rs:2171-2290, its environment /
// emissive-triangle branch): direction, radiance, pdf, shadow-ray extent and
// skipped triangle; `go` false when no sample.
struct AreaSample {
  V3 l, le;
  float pl, tmax;
  uint32_t skip;
  bool go;
};
PT_DEV AreaSample sample_area_light(const DevRequest &rq, const DevScene &s, V3 p, const float pl_u[4]) {
  AreaSample out;
  out.l = vzero();
  out.le = vzero();
  out.pl = 0.0f;
  out.tmax = inf();
  out.skip = 0xffffffffu;
  out.go = false;
  const float pe = rq.p_env;
  if (pl_u[2] < pe) {
    float epdf;
    if (rq.env && env_sample(*rq.env, pl_u[0], pl_u[1], out.l, out.le, epdf)) {
      out.pl = pe * epdf;
      out.go = true;
    }
  } else if (s.em_count > 0) {
    float us = pe > 0.0f ? clampr((pl_u[2] - pe) / (1.0f - pe), 0.0f, 0.999999f) : pl_u[2];
    uint32_t li = min(upper_bound(s.em_cdf, s.em_count, us), s.em_count - 1);
    uint32_t g = __ldg(s.em_tris + li);
    V3 a, b, cc;
    tri_positions(s, g, a, b, cc);
    bool have_target = false;
    V3 q = vzero();
    // The solid angle picks the sampling method and is the pdf's
    // denominator (one evaluation serves both).
    const float omega = triangle_solid_angle(p, a, b, cc);
    if (omega >= 1.0e-4f) {
      V3 ld;
      if (sample_spherical_triangle(p, a, b, cc, pl_u[0], pl_u[1], ld)) {
        V3 n = vcross(vsub(b, a), vsub(cc, a));
        float dn = vdot(ld, n);
        if (dn != 0.0f) {
          float t = vdot(vsub(a, p), n) / dn;
          if (t > 0.0f && isfinite(t)) {
            q = vadd(p, vscale(ld, t));
            have_target = true;
          }
        }
      }
    } else {
      float su = sqrtf(pl_u[0]);
      float w0 = 1.0f - su, w1 = su * (1.0f - pl_u[1]), w2 = su * pl_u[1];
      q = {a.x * w0 + b.x * w1 + cc.x * w2, a.y * w0 + b.y * w1 + cc.y * w2, a.z * w0 + b.z * w1 + cc.z * w2};
      have_target = true;
    }
    if (have_target) {
      // barycentric_of, src/trace.rs:1120-1133.
      V3 e1 = vsub(b, a), e2 = vsub(cc, a), r = vsub(q, a);
      float d11 = vdot(e1, e1), d12 = vdot(e1, e2), d22 = vdot(e2, e2);
      float r1 = vdot(r, e1), r2 = vdot(r, e2);
      float det = d11 * d22 - d12 * d12;
      if (isfinite(det) && fabsf(det) > F32_MIN_POSITIVE) {
        float u = (d22 * r1 - d12 * r2) / det;
        float vv = (d11 * r2 - d12 * r1) / det;
        float lb0 = clampr(1.0f - u - vv, 0.0f, 1.0f), lb1 = clampr(u, 0.0f, 1.0f), lb2 = clampr(vv, 0.0f, 1.0f);
        V3 to = vsub(q, p);
        float dist2 = vdot(to, to);
        uint2 linfo = __ldg(s.tri_info + g);
        const DevMaterial &lmat = s.materials[linfo.x];
        Surface lsurf = surface(s, g, lb0, lb1, lb2, linfo.y);
        if (dist2 > 1.0e-12f) {
          float dist = sqrtf(dist2);
          out.l = vscale(to, 1.0f / dist);
          float cos_l = -vdot(lsurf.ng, out.l);
          out.pl = tri_pdf_omega(rq, li, a, b, cc, omega, p, q);
          if ((cos_l > 0.0f || (lmat.m.double_sided && cos_l < 0.0f)) && out.pl > 0.0f && isfinite(out.pl)) {
            out.le = emission(s, lmat, g, linfo.y, lb0, lb1, lb2);
            out.tmax = fmaxf(dist * (1.0f - 1.0e-4f), 0.0f);
            out.skip = g;
            out.go = true;
          }
        }
      }
    }
  }
  return out;
}

// What the wavefront's NEE kernel computed for a vertex ahead of shade:
// the area-light sample and the emission MIS pdf. The megakernel computes
// both inline; the values are the same either way.
struct NeeInput {
  AreaSample area;
  float pl_emit;
};

// Shade vertex k of the path whose extension ray produced (found, hit).
// Shadow rays go to `sink.emit(ray)` in the reference's order. Returns false
// when the path terminated (the sink may still hold shadow rays of this
// vertex that contribute). With kPre, the area-light sample and the
// emission MIS pdf come from `pre` instead of being computed here, which
// keeps the f64 spherical-triangle and environment sampling code out of
// this (large) function's instruction footprint.
template <class Sink, bool kPre = false>
PT_DEV bool shade(const DevRequest &rq, PathState &ps, bool found, const Hit &hit, Sink &sink,
                  const NeeInput *pre = nullptr) {
  const DevScene &s = *rq.scene;
  const uint32_t k = ps.k;
  const uint32_t ray_id = k << 16;
  const uint32_t strategy = rq.strategy;
  if (ps.has_medium) {
    if (!found) return false;
    ps.beta = {ps.beta.x * expf(-ps.sigma.x * hit.t), ps.beta.y * expf(-ps.sigma.y * hit.t),
               ps.beta.z * expf(-ps.sigma.z * hit.t)};
  }
  if (!found) {
    if (k == 0) return false;  // uncovered
    V3 le;
    float w;
    if (rq.env) {
      le = env_radiance(*rq.env, ps.d);
      if (strategy == PT_MIS)
        w = power_heuristic(ps.prev_pdf, rq.p_env * env_pdf(*rq.env, ps.d));
      else if (strategy == PT_LIGHT_ONLY)
        w = 0.0f;
      else
        w = 1.0f;
    } else {
      le = {rq.ambient, rq.ambient, rq.ambient};
      w = 1.0f;
    }
    if (w > 0.0f) ps.radiance = vadd(ps.radiance, clamp_contrib(rq, vscale(vmul(ps.beta, le), w)));
    return false;
  }
  if (k == 0) ps.covered = 1;
  const uint2 info = __ldg(s.tri_info + hit.g);
  const uint32_t flags = info.y;
  const DevMaterial &dm = s.materials[info.x];
  const Surface surf = surface(s, hit.g, hit.b0, hit.b1, hit.b2, flags);
  const bool ds = dm.m.double_sided != 0;

  // Emission.
  if ((hit.front || ds) && !dm.m.unlit && dm.emissive_nonblack) {
    V3 le = emission(s, dm, hit.g, flags, hit.b0, hit.b1, hit.b2);
    if (!is_black(le)) {
      if (k == 0) {
        ps.radiance = vadd(ps.radiance, vmul(ps.beta, le));
      } else {
        float pl;
        if constexpr (kPre)
          pl = pre->pl_emit;
        else
          pl = emission_light_pdf(rq, s, hit.g, ps.prev_pos, surf.position);
        float w;
        if (pl <= 0.0f)
          w = 1.0f;
        else if (strategy == PT_MIS)
          w = power_heuristic(ps.prev_pdf, pl);
        else if (strategy == PT_LIGHT_ONLY)
          w = 0.0f;
        else
          w = 1.0f;
        if (w > 0.0f) ps.radiance = vadd(ps.radiance, clamp_contrib(rq, vscale(vmul(ps.beta, le), w)));
      }
    }
  }
  TexLod lod{false, 0.0f, vzero()};
  if (k == 0) {
    lod.cone = true;
    lod.width = rq.orthographic ? rq.pixel_spread : rq.pixel_spread * hit.t;
    lod.dir = ps.d;
  }
  const bool flip = !hit.front && ds;
  MaterialSample mat;
  material_oriented(s, dm, hit.g, flags, hit.b0, hit.b1, hit.b2, surf.sn, lod, flip, mat);
  if (flip) {
    mat.normal = vneg(mat.normal);
    mat.clearcoat_normal = vneg(mat.clearcoat_normal);
  }
  if (mat.unlit) {
    V3 c = {mat.base_color[0], mat.base_color[1], mat.base_color[2]};
    V3 contrib = vmul(ps.beta, c);
    ps.radiance = vadd(ps.radiance, k == 0 ? contrib : clamp_contrib(rq, contrib));
    return false;
  }
  if (k >= rq.max_bounces) return false;
  if (mat.dispersion > 0.0f && mat.thickness > 0.0f && mat.transmission > 0.0f) {
    int c;
    if (ps.hero >= 0) {
      c = ps.hero;
    } else {
      c = (int)min(f2u32(ps.smp.coin(ray_id | 0x7fffu, 0xffffffffu) * 3.0f), 2u);
      ps.beta = {c == 0 ? ps.beta.x * 3.0f : 0.0f, c == 1 ? ps.beta.y * 3.0f : 0.0f, c == 2 ? ps.beta.z * 3.0f : 0.0f};
      ps.hero = c;
    }
    float iors[3];
    dispersion_iors(mat.ior, mat.dispersion, iors);
    mat.ior = c == 0 ? iors[0] : (c == 1 ? iors[1] : iors[2]);
  }
  const V3 v = vneg(ps.d);
  Bsdf bsdf;
  bsdf.init(mat, v, surf.ng, hit.front);
  if (bsdf.is_black()) return false;
  const V3 p = surf.position;
  const V3 ng = bsdf.ng;
  const V3 off_pos = offset_ray_origin(p, ng), off_neg = offset_ray_origin(p, vneg(ng));

  // Next-event estimation and BSDF sampling share one Bsdf::eval call site:
  // candidate c < light_count is punctual light c, c == light_count the
  // area-set sample (environment or emissive triangle), the last one the
  // BSDF-sampled continuation. Shadow rays leave in the reference's order
  // (punctual lights, then the area sample) and every value is computed as
  // in Integrator::sample (src/pathtrace.rs:2171-2290); only the code path
  // to eval is shared, which keeps the kernel's instruction footprint small.
  float pb_u[4];
  ps.smp.pattern(1 + 2 * k, pb_u);
  const uint32_t nl = s.light_count;
  const bool area = area_nee(rq, s);
  const uint32_t shadow_id = ray_id | 0xffffu;
  V3 l, f;
  float pdf;
  for (uint32_t c = 0;; ++c) {
    V3 le = vzero();
    float pl = 0.0f, tmax = inf();
    uint32_t skip = 0xffffffffu, rid = shadow_id;
    bool go = false;
    if (c < nl) {
      LightSample ls;
      if (light_sample(s.lights[c], p, ls)) {
        l = ls.l;
        le = ls.radiance;
        tmax = isfinite(ls.distance) ? ls.distance * (1.0f - 1.0e-4f) : inf();
        rid = ray_id | 0x8000u | (c & 0x7fffu);
        go = true;
      }
    } else if (c == nl) {
      if (!area) continue;
      AreaSample as;
      if constexpr (kPre) {
        as = pre->area;
      } else {
        float pl_u[4];
        ps.smp.pattern(2 + 2 * k, pl_u);
        as = sample_area_light(rq, s, p, pl_u);
      }
      if (as.go) {
        l = as.l;
        le = as.le;
        pl = as.pl;
        tmax = as.tmax;
        skip = as.skip;
        go = true;
      }
    } else {
      if (!bsdf.sample_dir(pb_u, l)) return false;
      go = true;
    }
    if (!go) continue;
    bsdf.eval(l, f, pdf);
    if (c > nl) break;  // the BSDF sample: continue the path below
    if (is_black(f)) continue;
    ShadowRay sr;
    if (c < nl) {
      sr.contrib = clamp_contrib(rq, vmul(vmul(ps.beta, f), le));
    } else {
      if (is_black(le) || !(pl > 0.0f)) continue;
      float w = strategy == PT_MIS ? power_heuristic(pl, pdf) : 1.0f;
      sr.contrib = clamp_contrib(rq, vscale(vmul(vmul(ps.beta, f), le), w / pl));
    }
    if (sr.contrib.x == 0.0f && sr.contrib.y == 0.0f && sr.contrib.z == 0.0f) continue;  // adds nothing
    sr.o = vdot(l, ng) >= 0.0f ? off_pos : off_neg;
    sr.d = l;
    sr.tmax = tmax;
    sr.ray_id = rid;
    sr.skip = skip;
    sink.emit(sr);
  }
  if (!Bsdf::sample_accept(f, pdf)) return false;
  ps.beta = vmul(ps.beta, vscale(f, 1.0f / pdf));
  if (!finite3(ps.beta)) return false;
  ps.prev_pdf = pdf;
  ps.prev_pos = p;
  if (vdot(l, ng) < 0.0f && mat.thickness > 0.0f && mat.transmission > 0.0f) {
    if (hit.front) {
      float dist = mat.attenuation_distance;
      if (isfinite(dist)) {
        V3 c = mat.attenuation_color;
        ps.sigma = {-logf(fmaxf(c.x, 1.0e-6f)) / dist, -logf(fmaxf(c.y, 1.0e-6f)) / dist,
                    -logf(fmaxf(c.z, 1.0e-6f)) / dist};
        ps.has_medium = 1;
      } else {
        ps.has_medium = 0;
      }
    } else {
      ps.has_medium = 0;
    }
  }
  if (k + 1 >= rq.rr_start) {
    float q = clampr(max3(ps.beta), 0.05f, 1.0f);
    if (q < 1.0f) {
      if (pb_u[3] >= q) return false;
      ps.beta = vscale(ps.beta, 1.0f / q);
    }
  }
  ps.o = vdot(l, ng) >= 0.0f ? off_pos : off_neg;
  ps.d = l;
  ps.k = k + 1;
  return true;
}

// Final per-sample value: radiance (non-finite -> 0) and the covered flag.
PT_DEV float4 path_result(const PathState &ps) {
  if (!ps.covered) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  V3 r = finite3(ps.radiance) ? ps.radiance : vzero();
  return make_float4(r.x, r.y, r.z, 1.0f);
}

}  // namespace ptd
