// Device BSDF: microfacet terms, the layered glTF metallic-roughness BSDF
// with KHR_materials_{specular,transmission,volume,clearcoat,sheen,
// anisotropy,iridescence,diffuse_transmission,dispersion}, thin-film
// iridescence and spherical-triangle sampling.
// Formulas follow src/pathtrace.rs:508-1425 and :1743-1871 term by term.
#pragma once

#include "dev_common.cuh"

namespace ptd {

constexpr int SHEEN_LUT_COS = 32, SHEEN_LUT_ROUGH = 16;
// Sheen directional albedo E(cos, roughness), tabulated on the host by the
// reference's quadrature (sheen_lut, src/pathtrace.rs:645-674). All device
// code lives in one translation unit (kernels.cu), which sets it.
__device__ float g_sheen_lut[SHEEN_LUT_COS * SHEEN_LUT_ROUGH];

constexpr float MIN_ALPHA = 1.0e-3f;
enum { LOBE_DIFFUSE = 0, LOBE_SPECULAR, LOBE_TRANSMISSION, LOBE_CLEARCOAT, LOBE_SHEEN, LOBE_DIFFUSE_T };

// MaterialSample (src/trace.rs:202-305).
struct MaterialSample {
  float base_color[4];
  float metallic, roughness;
  V3 normal;
  float occlusion;  // set by material_oriented<true> only
  V3 emissive;
  uint32_t unlit, double_sided;
  float ior, specular;
  V3 specular_color;
  float transmission, thickness;
  V3 attenuation_color;
  float attenuation_distance;
  float clearcoat, clearcoat_roughness;
  V3 clearcoat_normal;
  V3 sheen_color;
  float sheen_roughness, anisotropy;
  V3 anisotropy_direction;
  float iridescence, iridescence_ior, iridescence_thickness;
  float diffuse_transmission;
  V3 diffuse_transmission_color;
  float dispersion;
};

PT_DEV float d_ggx(float n_dot_h, float a) {
  if (n_dot_h <= 0.0f) return 0.0f;
  float a2 = a * a;
  float d = n_dot_h * n_dot_h * (a2 - 1.0f) + 1.0f;
  return a2 / (PI * d * d);
}
PT_DEV float lambda_iso(float cos, float a) {
  float c = fmaxf(fabsf(cos), 1.0e-7f);
  float a2 = a * a;
  return (sqrtf(a2 + (1.0f - a2) * c * c) / c - 1.0f) * 0.5f;
}
PT_DEV float g1_iso(float cos, float a) { return 1.0f / (1.0f + lambda_iso(cos, a)); }
PT_DEV float g2_iso(float cv, float cl, float a) { return 1.0f / (1.0f + lambda_iso(cv, a) + lambda_iso(cl, a)); }
PT_DEV V3 schlick(V3 f0, float cos) {
  float k = powi5(1.0f - clampr(cos, 0.0f, 1.0f));
  return {f0.x + (1.0f - f0.x) * k, f0.y + (1.0f - f0.y) * k, f0.z + (1.0f - f0.z) * k};
}

// GGX visible normals (Heitz 2018), isotropic and stretched.
PT_DEV V3 sample_vndf_at(V3 v, float at, float ab, float u0, float u1) {
  V3 vh = vnormalise({at * v.x, ab * v.y, v.z});
  float lensq = vh.x * vh.x + vh.y * vh.y;
  V3 t1;
  if (lensq > 0.0f) {
    float il = 1.0f / sqrtf(lensq);
    t1 = {-vh.y * il, vh.x * il, 0.0f};
  } else {
    t1 = {1.0f, 0.0f, 0.0f};
  }
  V3 t2 = vcross(vh, t1);
  float r = sqrtf(u0);
  float phi = 2.0f * PI * u1;
  float p1 = r * cosf(phi);
  float p2 = r * sinf(phi);
  float s = 0.5f * (1.0f + vh.z);
  p2 = (1.0f - s) * sqrtf(fmaxf(1.0f - p1 * p1, 0.0f)) + s * p2;
  float pz = sqrtf(fmaxf(1.0f - p1 * p1 - p2 * p2, 0.0f));
  V3 nh = {p1 * t1.x + p2 * t2.x + pz * vh.x, p1 * t1.y + p2 * t2.y + pz * vh.y, p1 * t1.z + p2 * t2.z + pz * vh.z};
  return vnormalise({at * nh.x, ab * nh.y, fmaxf(nh.z, 1.0e-6f)});
}
PT_DEV float vndf_reflect_pdf(V3 n, V3 v, V3 h, float a) {
  float nv = vdot(n, v), nh = vdot(n, h);
  if (nv <= 0.0f || nh <= 0.0f || vdot(v, h) <= 0.0f) return 0.0f;
  return g1_iso(nv, a) * d_ggx(nh, a) / (4.0f * nv);
}
PT_DEV V3 reflect(V3 v, V3 h) {
  float d = 2.0f * vdot(v, h);
  return {d * h.x - v.x, d * h.y - v.y, d * h.z - v.z};
}
PT_DEV bool refract(V3 v, V3 h, float eta, V3 &out) {
  float ci = vdot(v, h);
  float s2 = eta * eta * fmaxf(1.0f - ci * ci, 0.0f);
  if (s2 >= 1.0f) return false;
  float ct = sqrtf(1.0f - s2);
  float k = eta * ci - ct;
  out = vnormalise({-eta * v.x + k * h.x, -eta * v.y + k * h.y, -eta * v.z + k * h.z});
  return true;
}
PT_DEV V3 cosine_hemisphere(float u0, float u1) {
  float a = 2.0f * u0 - 1.0f;
  float b = 2.0f * u1 - 1.0f;
  float r, phi;
  if (a == 0.0f && b == 0.0f) {
    r = 0.0f;
    phi = 0.0f;
  } else if (fabsf(a) > fabsf(b)) {
    r = a;
    phi = FRAC_PI_4 * (b / a);
  } else {
    r = b;
    phi = FRAC_PI_2 - FRAC_PI_4 * (a / b);
  }
  float x = r * cosf(phi), y = r * sinf(phi);
  return {x, y, sqrtf(fmaxf(1.0f - x * x - y * y, 0.0f))};
}

// Sheen (Charlie + Neubelt-Pettineo), src/pathtrace.rs:617-692.
PT_DEV float d_charlie(float n_dot_h, float a) {
  float inv = 1.0f / fmaxf(a, 1.0e-3f);
  float sin2 = fmaxf(1.0f - n_dot_h * n_dot_h, 0.0f);
  return (2.0f + inv) * powf(sin2, inv * 0.5f) / (2.0f * PI);
}
PT_DEV float v_neubelt(float nl, float nv) { return 1.0f / fmaxf(4.0f * (nl + nv - nl * nv), 1.0e-6f); }
PT_DEV float sheen_albedo(float cos, float rough) {
  float x = clampr(clampr(cos, 0.0f, 1.0f) * (float)SHEEN_LUT_COS - 0.5f, 0.0f, (float)(SHEEN_LUT_COS - 1));
  float y = clampr(clampr(rough, 0.0f, 1.0f) * (float)(SHEEN_LUT_ROUGH - 1), 0.0f, (float)(SHEEN_LUT_ROUGH - 1));
  uint32_t x0 = f2u32(floorf(x)), y0 = f2u32(floorf(y));
  uint32_t x1 = min(x0 + 1, (uint32_t)SHEEN_LUT_COS - 1), y1 = min(y0 + 1, (uint32_t)SHEEN_LUT_ROUGH - 1);
  float fx = x - (float)x0, fy = y - (float)y0;
  const float *lut = g_sheen_lut;
  float a00 = __ldg(lut + y0 * SHEEN_LUT_COS + x0), a10 = __ldg(lut + y0 * SHEEN_LUT_COS + x1);
  float a01 = __ldg(lut + y1 * SHEEN_LUT_COS + x0), a11 = __ldg(lut + y1 * SHEEN_LUT_COS + x1);
  float a = a00 + (a10 - a00) * fx;
  float b = a01 + (a11 - a01) * fx;
  return a + (b - a) * fy;
}

// Thin-film iridescence (Belcour & Barla 2017), src/pathtrace.rs:1326-1417.
PT_DEV V3 eval_sensitivity(float opd, V3 shift) {
  float phase = 2.0f * PI * opd * 1.0e-9f;
  const float val[3] = {5.4856e-13f, 4.4201e-13f, 5.2481e-13f};
  const float pos[3] = {1.6810e6f, 1.7953e6f, 2.2084e6f};
  const float var[3] = {4.3278e9f, 9.3046e9f, 6.6121e9f};
  float sh[3] = {shift.x, shift.y, shift.z};
  float xyz[3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
    xyz[k] = val[k] * sqrtf(2.0f * PI * var[k]) * cosf(pos[k] * phase + sh[k]) * expf(-phase * phase * var[k]);
  xyz[0] += 9.7470e-14f * sqrtf(2.0f * PI * 4.5282e9f) * cosf(2.2399e6f * phase + sh[0]) *
            expf(-4.5282e9f * phase * phase);
#pragma unroll
  for (int k = 0; k < 3; ++k) xyz[k] /= 1.0685e-7f;
  return {3.2404542f * xyz[0] - 1.5371385f * xyz[1] - 0.4985314f * xyz[2],
          -0.969266f * xyz[0] + 1.8760108f * xyz[1] + 0.041556f * xyz[2],
          0.0556434f * xyz[0] - 0.2040259f * xyz[1] + 1.0572252f * xyz[2]};
}
PT_DEV V3 iridescent_fresnel(float outside_ior, float film_ior, V3 base_f0, float thickness_nm, float cos1) {
  cos1 = clampr(cos1, 0.0f, 1.0f);
  float r0 = powi2((film_ior - outside_ior) / (film_ior + outside_ior));
  float r12 = r0 + (1.0f - r0) * powi5(1.0f - cos1);
  float t121 = 1.0f - r12;
  float sin2_2 = powi2(outside_ior / film_ior) * (1.0f - cos1 * cos1);
  float cos2_sq = 1.0f - sin2_2;
  if (cos2_sq < 0.0f) return {1.0f, 1.0f, 1.0f};
  float cos2 = sqrtf(cos2_sq);
  float bf[3] = {base_f0.x, base_f0.y, base_f0.z};
  float r23[3], phi23[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float f0 = clampr(bf[k] + 1.0e-4f, 0.0f, 0.9999f);
    float sq = sqrtf(f0);
    float base_ior = (1.0f + sq) / (1.0f - sq);
    float r1 = powi2((base_ior - film_ior) / (base_ior + film_ior));
    r23[k] = r1 + (1.0f - r1) * powi5(1.0f - cos2);
    if (base_ior < film_ior) phi23[k] = PI;
  }
  float opd = 2.0f * film_ior * thickness_nm * cos2;
  float phi12 = film_ior < outside_ior ? PI : 0.0f;
  float phi21 = PI - phi12;
  float phi[3] = {phi21 + phi23[0], phi21 + phi23[1], phi21 + phi23[2]};
  float out[3], r123[3], rs[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    r123[k] = clampr(r12 * r23[k], 1.0e-5f, 0.9999f);
    rs[k] = t121 * t121 * r23[k] / (1.0f - r123[k]);
    out[k] = r12 + rs[k];
  }
  float cm[3] = {rs[0] - t121, rs[1] - t121, rs[2] - t121};
#pragma unroll
  for (int m = 1; m <= 2; ++m) {
#pragma unroll
    for (int k = 0; k < 3; ++k) cm[k] *= sqrtf(r123[k]);
    V3 sm = eval_sensitivity((float)m * opd, {(float)m * phi[0], (float)m * phi[1], (float)m * phi[2]});
    out[0] += cm[0] * 2.0f * sm.x;
    out[1] += cm[1] * 2.0f * sm.y;
    out[2] += cm[2] * 2.0f * sm.z;
  }
  return {clampr(out[0], 0.0f, 1.0f), clampr(out[1], 0.0f, 1.0f), clampr(out[2], 0.0f, 1.0f)};
}
PT_DEV void dispersion_iors(float ior, float dispersion, float out[3]) {
  float hs = (ior - 1.0f) * 0.025f * fmaxf(dispersion, 0.0f);
  out[0] = fmaxf(ior - hs, 1.0f);
  out[1] = fmaxf(ior, 1.0f);
  out[2] = fmaxf(ior + hs, 1.0f);
}

// ---------------------------------------------------------------- Microfacet
struct Microfacet {
  V3 t, b, n;
  float at, ab;
  bool aniso;
  PT_DEV V3 local(V3 w) const { return {vdot(w, t), vdot(w, b), vdot(w, n)}; }
  PT_DEV float d(V3 h) const {
    if (!aniso) return d_ggx(vdot(n, h), at);
    V3 hl = local(h);
    if (hl.z <= 0.0f) return 0.0f;
    float x = hl.x / at, y = hl.y / ab;
    float e = x * x + y * y + hl.z * hl.z;
    return 1.0f / (PI * at * ab * e * e);
  }
  PT_DEV float lambda(V3 w) const {
    if (!aniso) return lambda_iso(vdot(n, w), at);
    V3 wl = local(w);
    float cz = fmaxf(fabsf(wl.z), 1.0e-7f);
    float a2 = powi2(at * wl.x) + powi2(ab * wl.y);
    return (sqrtf(1.0f + a2 / (cz * cz)) - 1.0f) * 0.5f;
  }
  PT_DEV float g1(V3 v) const { return 1.0f / (1.0f + lambda(v)); }
  PT_DEV float g2(V3 v, V3 l) const { return 1.0f / (1.0f + lambda(v) + lambda(l)); }
  PT_DEV float pdf_reflect(V3 v, V3 h) const {
    if (!aniso) return vndf_reflect_pdf(n, v, h, at);
    float nv = vdot(n, v), nh = vdot(n, h);
    if (nv <= 0.0f || nh <= 0.0f || vdot(v, h) <= 0.0f) return 0.0f;
    return g1(v) * d(h) / (4.0f * nv);
  }
  PT_DEV bool sample(V3 v, float u0, float u1, V3 &out) const {
    V3 vl = local(v);
    if (vl.z <= 0.0f) return false;
    V3 h = aniso ? sample_vndf_at(vl, at, ab, u0, u1) : sample_vndf_at(vl, at, at, u0, u1);
    out = to_world(t, b, n, h);
    return true;
  }
};

// ---------------------------------------------------------------- Bsdf
struct Bsdf {
  V3 v, n, ng, ncc, base;
  float metallic;
  Microfacet mf;
  float specular;
  V3 f0d;
  float transmission;
  bool thin;
  float eta_i, eta_t;
  float clearcoat, cc_alpha;
  V3 sheen;
  float sheen_rough, sheen_alpha;
  float irid, irid_ior, irid_thick;
  float dt;
  V3 dt_color;
  float w_cc;
  float probs[6];

  // Bsdf::new, src/pathtrace.rs:853-986.
  PT_DEV void init(const MaterialSample &m, V3 v_, V3 ng_, bool front) {
    v = v_;
    ng = front ? ng_ : vneg(ng_);
    n = front ? m.normal : vneg(m.normal);
    if (vdot(n, v) <= 1.0e-4f) n = ng;
    ncc = front ? m.clearcoat_normal : vneg(m.clearcoat_normal);
    if (vdot(ncc, v) <= 1.0e-4f) ncc = n;
    thin = m.thickness <= 0.0f;
    float ior = (isfinite(m.ior) && m.ior >= 1.0f) ? m.ior : 1.5f;
    if (thin || front) {
      eta_i = 1.0f;
      eta_t = ior;
    } else {
      eta_i = ior;
      eta_t = 1.0f;
    }
    bool inside = !thin && !front;
    float r0 = powi2((ior - 1.0f) / (ior + 1.0f));
    base = {m.base_color[0], m.base_color[1], m.base_color[2]};
    float alpha = fmaxf(m.roughness * m.roughness, MIN_ALPHA);
    float aniso = clampr(m.anisotropy, 0.0f, 1.0f);
    basis(n, mf.t, mf.b);
    mf.n = n;
    mf.at = alpha;
    mf.ab = alpha;
    mf.aniso = false;
    if (aniso > 0.0f) {
      V3 d0 = m.anisotropy_direction;
      float dn = vdot(d0, n);
      V3 t = vnormalise({d0.x - n.x * dn, d0.y - n.y * dn, d0.z - n.z * dn});
      if (vdot(t, t) > 0.5f) {
        float at = alpha + (1.0f - alpha) * aniso * aniso;
        if (at > alpha) {
          mf.t = t;
          mf.b = vcross(n, t);
          mf.n = n;
          mf.at = at;
          mf.ab = alpha;
          mf.aniso = true;
        }
      }
    }
    metallic = m.metallic;
    specular = clampr(m.specular, 0.0f, 1.0f);
    f0d = {fminf(r0 * m.specular_color.x, 1.0f), fminf(r0 * m.specular_color.y, 1.0f),
           fminf(r0 * m.specular_color.z, 1.0f)};
    transmission = m.transmission;
    clearcoat = inside ? 0.0f : m.clearcoat;
    cc_alpha = fmaxf(m.clearcoat_roughness * m.clearcoat_roughness, MIN_ALPHA);
    sheen = inside ? vzero() : m.sheen_color;
    sheen_rough = m.sheen_roughness;
    sheen_alpha = fmaxf(m.sheen_roughness * m.sheen_roughness, 1.0e-3f);
    irid = inside ? 0.0f : clampr(m.iridescence, 0.0f, 1.0f);
    irid_ior = isfinite(m.iridescence_ior) ? fmaxf(m.iridescence_ior, 1.0f) : 1.3f;
    irid_thick = isfinite(m.iridescence_thickness) ? fmaxf(m.iridescence_thickness, 0.0f) : 400.0f;
    dt = clampr(m.diffuse_transmission, 0.0f, 1.0f);
    dt_color = {clampr(m.diffuse_transmission_color.x, 0.0f, 1.0f),
                clampr(m.diffuse_transmission_color.y, 0.0f, 1.0f),
                clampr(m.diffuse_transmission_color.z, 0.0f, 1.0f)};
    w_cc = 0.0f;
#pragma unroll
    for (int i = 0; i < 6; ++i) probs[i] = 0.0f;

    float cv = fmaxf(vdot(n, v), 1.0e-4f);
    w_cc = clearcoat > 0.0f ? clearcoat * schlick({0.04f, 0.04f, 0.04f}, vdot(ncc, v)).x : 0.0f;
    float sheen_max = max3(sheen);
    float e_v = sheen_max > 0.0f ? sheen_albedo(cv, sheen_rough) : 0.0f;
    float s_scale = (1.0f - w_cc) * (1.0f - sheen_max * e_v);
    V3 fd_v, fm_v;
    fresnel_pair(cv, fd_v, fm_v);
    float fd = max3(fd_v);
    float fm = mean3(fm_v);
    float m_ = metallic;
    float base_mean = fmaxf(mean3(base), 0.0f);
    float t = transmission;
    float p[6] = {
        s_scale * (1.0f - m_) * (1.0f - t) * (1.0f - dt) * (1.0f - fd) * base_mean,
        s_scale * ((1.0f - m_) * fd + m_ * fm),
        s_scale * (1.0f - m_) * t * (1.0f - fd) * base_mean,
        w_cc,
        (1.0f - w_cc) * sheen_max * e_v,
        s_scale * (1.0f - m_) * (1.0f - t) * dt * (1.0f - fd) * fmaxf(mean3(dt_color), 0.0f),
    };
    float sum = 0.0f;
#pragma unroll
    for (int i = 0; i < 6; ++i) sum += p[i];
    if (sum > 0.0f && isfinite(sum)) {
#pragma unroll
      for (int i = 0; i < 6; ++i) probs[i] = p[i] / sum;
    }
  }
  PT_DEV bool is_black() const {
#pragma unroll
    for (int i = 0; i < 6; ++i)
      if (probs[i] > 0.0f) return false;
    return true;
  }
  PT_DEV V3 fresnel_d(float c) const {
    if (eta_i > eta_t) {
      float eta = eta_i / eta_t;
      float s2 = eta * eta * fmaxf(1.0f - c * c, 0.0f);
      if (s2 >= 1.0f) return {1.0f, 1.0f, 1.0f};
      return schlick(f0d, sqrtf(1.0f - s2));
    }
    return schlick(f0d, c);
  }
  PT_DEV void fresnel_pair(float c, V3 &fd_out, V3 &fm_out) const {
    V3 fd = vscale(fresnel_d(c), specular);
    V3 fm = schlick(base, c);
    if (irid <= 0.0f) {
      fd_out = fd;
      fm_out = fm;
      return;
    }
    float i = irid;
    V3 fd_i = metallic < 1.0f ? iridescent_fresnel(1.0f, irid_ior, vscale(f0d, specular), irid_thick, c) : fd;
    V3 fm_i = metallic > 0.0f ? iridescent_fresnel(1.0f, irid_ior, base, irid_thick, c) : fm;
    fd_out = {fd.x + (fd_i.x - fd.x) * i, fd.y + (fd_i.y - fd.y) * i, fd.z + (fd_i.z - fd.z) * i};
    fm_out = {fm.x + (fm_i.x - fm.x) * i, fm.y + (fm_i.y - fm.y) * i, fm.z + (fm_i.z - fm.z) * i};
  }

  // Bsdf::eval, src/pathtrace.rs:1075-1211: f(v,l)|n.l| and the mixture pdf.
  PT_DEV void eval(V3 l, V3 &f_out, float &pdf_out) const {
    float nv = fmaxf(vdot(n, v), 1.0e-4f);
    if (vdot(ng, l) > 0.0f) {
      float nl = vdot(n, l);
      V3 h = vnormalise(vadd(v, l));
      float vh = fmaxf(vdot(v, h), 0.0f);
      V3 f = vzero();
      float pdf = 0.0f;
      if (nl > 0.0f) {
        V3 fd, fm;
        fresnel_pair(vh, fd, fm);
        float spec_c = mf.d(h) * mf.g2(v, l) / (4.0f * nv * nl);
        float m = metallic;
        float diff_k = (1.0f - m) * (1.0f - transmission) * (1.0f - dt) * (1.0f - max3(fd)) / PI;
        V3 layer = {spec_c * ((1.0f - m) * fd.x + m * fm.x) + diff_k * base.x,
                    spec_c * ((1.0f - m) * fd.y + m * fm.y) + diff_k * base.y,
                    spec_c * ((1.0f - m) * fd.z + m * fm.z) + diff_k * base.z};
        float smax = max3(sheen);
        if (smax > 0.0f) {
          float sc = fminf(1.0f - smax * sheen_albedo(nv, sheen_rough), 1.0f - smax * sheen_albedo(nl, sheen_rough));
          float nh = vdot(n, h);
          float sh = d_charlie(nh, sheen_alpha) * v_neubelt(nl, nv);
          layer = {layer.x * sc + sheen.x * sh, layer.y * sc + sheen.y * sh, layer.z * sc + sheen.z * sh};
        }
        f = {layer.x * (1.0f - w_cc), layer.y * (1.0f - w_cc), layer.z * (1.0f - w_cc)};
        pdf += (probs[LOBE_DIFFUSE] + probs[LOBE_SHEEN]) * nl / PI;
        pdf += probs[LOBE_SPECULAR] * mf.pdf_reflect(v, h);
      }
      if (clearcoat > 0.0f) {
        float cnv = fmaxf(vdot(ncc, v), 1.0e-4f);
        float cnl = vdot(ncc, l);
        if (cnl > 0.0f) {
          float cnh = vdot(ncc, h);
          float c = w_cc * d_ggx(cnh, cc_alpha) * g2_iso(cnv, cnl, cc_alpha) / (4.0f * cnv * cnl);
          f = {f.x + c, f.y + c, f.z + c};
          pdf += probs[LOBE_CLEARCOAT] * vndf_reflect_pdf(ncc, v, h, cc_alpha);
        }
      }
      float cos = fmaxf(nl, 0.0f);
      f_out = vscale(f, cos);
      pdf_out = pdf;
      return;
    }
    f_out = vzero();
    pdf_out = 0.0f;
    if (metallic >= 1.0f || (transmission <= 0.0f && dt <= 0.0f)) return;
    float nl = -vdot(n, l);
    if (nl <= 0.0f) return;
    float smax = max3(sheen);
    float layer_scale = (1.0f - w_cc) * (smax > 0.0f ? 1.0f - smax * sheen_albedo(nv, sheen_rough) : 1.0f);
    V3 f = vzero();
    float pdf = 0.0f;
    if (dt > 0.0f && transmission < 1.0f) {
      V3 fd, fm;
      fresnel_pair(nv, fd, fm);
      float w = (1.0f - metallic) * (1.0f - transmission) * dt * (1.0f - max3(fd)) * layer_scale / PI;
      f = {f.x + w * dt_color.x * nl, f.y + w * dt_color.y * nl, f.z + w * dt_color.z * nl};
      pdf += probs[LOBE_DIFFUSE_T] * nl / PI;
    }
    if (transmission <= 0.0f) {
      f_out = f;
      pdf_out = pdf;
      return;
    }
    float w = (1.0f - metallic) * transmission * layer_scale;
    float val, pdf_t;
    if (thin) {
      V3 lm = vadd(l, vscale(n, 2.0f * nl));
      V3 h = vnormalise(vadd(v, lm));
      float vh = vdot(v, h), nh = vdot(n, h);
      if (vh <= 0.0f || nh <= 0.0f) {
        f_out = f;
        pdf_out = pdf;
        return;
      }
      V3 fdv, fmv;
      fresnel_pair(vh, fdv, fmv);
      float fd = max3(fdv);
      val = mf.d(h) * mf.g2(v, lm) / (4.0f * nv * nl) * (1.0f - fd);
      pdf_t = mf.pdf_reflect(v, h);
    } else {
      float ei = eta_i, et = eta_t;
      V3 h = vnormalise({-(ei * v.x + et * l.x), -(ei * v.y + et * l.y), -(ei * v.z + et * l.z)});
      if (vdot(h, n) < 0.0f) h = vneg(h);
      float vh = vdot(v, h), lh = vdot(l, h), nh = vdot(n, h);
      if (vh <= 0.0f || lh >= 0.0f || nh <= 0.0f) {
        f_out = f;
        pdf_out = pdf;
        return;
      }
      float denom = ei * vh + et * lh;
      if (fabsf(denom) < 1.0e-6f) {
        f_out = f;
        pdf_out = pdf;
        return;
      }
      float d = mf.d(h);
      V3 fdv, fmv;
      fresnel_pair(vh, fdv, fmv);
      float fd = max3(fdv);
      float jac = et * et * fabsf(lh) / (denom * denom);
      val = vh * fabsf(lh) * d * mf.g2(v, l) * et * et * (1.0f - fd) / (nv * nl * denom * denom);
      pdf_t = mf.g1(v) * vh * d / nv * jac;
    }
    f = {f.x + base.x * w * val * nl, f.y + base.y * w * val * nl, f.z + base.z * w * val * nl};
    f_out = f;
    pdf_out = pdf + probs[LOBE_TRANSMISSION] * pdf_t;
  }

  // Bsdf::sample, src/pathtrace.rs:1216-1279: sample_dir picks the lobe and
  // direction, eval gives (f, pdf) and sample_accept applies the final
  // checks. Split so a caller can share one eval call site.
  PT_DEV bool sample(const float u[3], V3 &l_out, V3 &f_out, float &pdf_out) const {
    V3 l;
    if (!sample_dir(u, l)) return false;
    V3 f;
    float pdf;
    eval(l, f, pdf);
    if (!sample_accept(f, pdf)) return false;
    l_out = l;
    f_out = f;
    pdf_out = pdf;
    return true;
  }
  PT_DEV static bool sample_accept(V3 f, float pdf) {
    return !(pdf <= 0.0f || !isfinite(pdf) || ptd::is_black(f) || !finite3(f));
  }
  PT_DEV bool sample_dir(const float u[3], V3 &l_out) const {
    float acc = 0.0f;
    int lobe = -1;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      acc += probs[i];
      if (lobe < 0 && probs[i] > 0.0f && u[2] < acc) lobe = i;
    }
    if (lobe < 0) {
#pragma unroll
      for (int i = 0; i < 6; ++i)
        if (probs[i] > 0.0f) lobe = i;
      if (lobe < 0) return false;
    }
    V3 l;
    if (lobe == LOBE_DIFFUSE || lobe == LOBE_SHEEN) {
      V3 t, b;
      basis(n, t, b);
      l = to_world(t, b, n, cosine_hemisphere(u[0], u[1]));
    } else if (lobe == LOBE_DIFFUSE_T) {
      V3 t, b;
      basis(n, t, b);
      V3 d = cosine_hemisphere(u[0], u[1]);
      l = to_world(t, b, n, {d.x, d.y, -d.z});
    } else if (lobe == LOBE_CLEARCOAT) {
      V3 t, b;
      basis(ncc, t, b);
      V3 vl = {vdot(v, t), vdot(v, b), vdot(v, ncc)};
      if (vl.z <= 0.0f) return false;
      V3 h = to_world(t, b, ncc, sample_vndf_at(vl, cc_alpha, cc_alpha, u[0], u[1]));
      l = reflect(v, h);
    } else {
      V3 h;
      if (!mf.sample(v, u[0], u[1], h)) return false;
      if (lobe == LOBE_SPECULAR) {
        l = reflect(v, h);
      } else if (thin) {
        V3 r = reflect(v, h);
        float d = vdot(r, n);
        l = vadd(r, vscale(n, -2.0f * d));
      } else {
        if (!refract(v, h, eta_i / eta_t, l)) return false;
      }
    }
    if (!finite3(l) || vdot(l, l) < 0.5f) return false;
    bool reflection = vdot(ng, l) > 0.0f;
    bool transmits = lobe == LOBE_TRANSMISSION || lobe == LOBE_DIFFUSE_T;
    if (reflection == transmits) return false;
    l_out = l;
    return true;
  }
};

// ---------------------------------------------------------------- spherical triangles
// triangle_solid_angle (Van Oosterom & Strackee 1983), src/pathtrace.rs:1755-1784.
PT_DEV float triangle_solid_angle(V3 p, V3 a_, V3 b_, V3 c_) {
  double a[3], b[3], c[3];
  V3 q3[3] = {a_, b_, c_};
  double *o3[3] = {a, b, c};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double d0 = (double)(q3[i].x - p.x), d1 = (double)(q3[i].y - p.y), d2 = (double)(q3[i].z - p.z);
    double l = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    if (l > 0.0) {
      o3[i][0] = d0 / l;
      o3[i][1] = d1 / l;
      o3[i][2] = d2 / l;
    } else {
      o3[i][0] = o3[i][1] = o3[i][2] = 0.0;
    }
  }
  double bc0 = b[1] * c[2] - b[2] * c[1], bc1 = b[2] * c[0] - b[0] * c[2], bc2 = b[0] * c[1] - b[1] * c[0];
  double num = fabs(a[0] * bc0 + a[1] * bc1 + a[2] * bc2);
  double den = 1.0 + (a[0] * b[0] + a[1] * b[1] + a[2] * b[2]) + (b[0] * c[0] + b[1] * c[1] + b[2] * c[2]) +
               (c[0] * a[0] + c[1] * a[1] + c[2] * a[2]);
  double o = 2.0 * atan2(num, den);
  if (isfinite(o)) return (float)fmax(o, 0.0);
  return 0.0f;
}

struct D3 {
  double x, y, z;
};
PT_DEV double ddot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PT_DEV D3 dcross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
PT_DEV bool dnorm(D3 x, D3 &o) {
  double l = sqrt(ddot(x, x));
  if (!(l > 1.0e-300 && isfinite(l))) return false;
  o = {x.x / l, x.y / l, x.z / l};
  return true;
}
// Arvo 1995, src/pathtrace.rs:1789-1871.
PT_DEV bool sample_spherical_triangle(V3 p, V3 a_, V3 b_, V3 c_, float u0, float u1, V3 &out) {
  auto sub = [&](V3 x) { return D3{(double)(x.x - p.x), (double)(x.y - p.y), (double)(x.z - p.z)}; };
  D3 a, b, c;
  if (!dnorm(sub(a_), a) || !dnorm(sub(b_), b) || !dnorm(sub(c_), c)) return false;
  D3 nab, nbc, nca;
  if (!dnorm(dcross(a, b), nab) || !dnorm(dcross(b, c), nbc) || !dnorm(dcross(c, a), nca)) return false;
  double alpha = acos(clampd(-ddot(nab, nca), -1.0, 1.0));
  double beta = acos(clampd(-ddot(nbc, nab), -1.0, 1.0));
  double gamma = acos(clampd(-ddot(nca, nbc), -1.0, 1.0));
  double area = alpha + beta + gamma - 3.14159265358979323846;
  if (isnan(area) || area <= 0.0) return false;
  double ap = (double)u0 * area;
  double s = sin(ap - alpha), t = cos(ap - alpha);
  double sa = sin(alpha), ca = cos(alpha);
  double cos_c = ddot(a, b);
  double uu = t - ca;
  double vv = s + sa * cos_c;
  double den = (vv * s + uu * t) * sa;
  if (fabs(den) < 1.0e-300) return false;
  double q = clampd(((vv * t - uu * s) * ca - vv) / den, -1.0, 1.0);
  double dca = ddot(c, a);
  D3 ca_perp;
  if (!dnorm({c.x - dca * a.x, c.y - dca * a.y, c.z - dca * a.z}, ca_perp)) return false;
  double r = sqrt(fmax(1.0 - q * q, 0.0));
  D3 cp = {q * a.x + r * ca_perp.x, q * a.y + r * ca_perp.y, q * a.z + r * ca_perp.z};
  double z = 1.0 - (double)u1 * (1.0 - ddot(cp, b));
  double dcpb = ddot(cp, b);
  D3 cb_perp;
  bool has_perp = dnorm({cp.x - dcpb * b.x, cp.y - dcpb * b.y, cp.z - dcpb * b.z}, cb_perp);
  double w = sqrt(fmax(1.0 - z * z, 0.0));
  D3 d = has_perp ? D3{z * b.x + w * cb_perp.x, z * b.y + w * cb_perp.y, z * b.z + w * cb_perp.z} : b;
  D3 dn;
  if (!dnorm(d, dn)) return false;
  out = {(float)dn.x, (float)dn.y, (float)dn.z};
  return true;
}

}  // namespace ptd
