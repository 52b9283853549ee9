// ORACLE — test infrastructure only (see oracle_core.hpp).
// Microfacet terms, the layered glTF BSDF, sheen table, thin-film
// iridescence, dispersion and spherical-triangle sampling, restated from
// src/pathtrace.rs:508-1425 and :1743-1871.
#include "oracle_core.hpp"

#include <mutex>

namespace oracle {

const SobolMatrices &sobol_matrices() {
  static SobolMatrices m;
  return m;
}

constexpr float MIN_ALPHA = 1.0e-3f;  // src/pathtrace.rs:513
enum { LOBE_DIFFUSE = 0, LOBE_SPECULAR, LOBE_TRANSMISSION, LOBE_CLEARCOAT, LOBE_SHEEN, LOBE_DIFFUSE_T };

// src/pathtrace.rs:515-550
static float d_ggx(float n_dot_h, float a) {
  if (n_dot_h <= 0.0f) return 0.0f;
  float a2 = a * a;
  float d = n_dot_h * n_dot_h * (a2 - 1.0f) + 1.0f;
  return a2 / (PI * d * d);
}
static float lambda_iso(float cos, float a) {
  float c = fmaxr(std::fabs(cos), 1.0e-7f);
  float a2 = a * a;
  return (std::sqrt(a2 + (1.0f - a2) * c * c) / c - 1.0f) * 0.5f;
}
static float g1_iso(float cos, float a) { return 1.0f / (1.0f + lambda_iso(cos, a)); }
static float g2_iso(float cv, float cl, float a) { return 1.0f / (1.0f + lambda_iso(cv, a) + lambda_iso(cl, a)); }
static V3 schlick(V3 f0, float cos) {
  float k = powi5(1.0f - clampr(cos, 0.0f, 1.0f));
  return {f0.x + (1.0f - f0.x) * k, f0.y + (1.0f - f0.y) * k, f0.z + (1.0f - f0.z) * k};
}

// sample_vndf / sample_vndf_aniso, src/pathtrace.rs:554-577, 1288-1311.
static V3 sample_vndf_at(V3 v, float at, float ab, float u0, float u1) {
  V3 vh = normalise({at * v.x, ab * v.y, v.z});
  float lensq = vh.x * vh.x + vh.y * vh.y;
  V3 t1;
  if (lensq > 0.0f) {
    float il = 1.0f / std::sqrt(lensq);
    t1 = {-vh.y * il, vh.x * il, 0.0f};
  } else {
    t1 = {1.0f, 0.0f, 0.0f};
  }
  V3 t2 = cross(vh, t1);
  float r = std::sqrt(u0);
  float phi = 2.0f * PI * u1;
  float p1 = r * std::cos(phi);
  float p2 = r * std::sin(phi);
  float s = 0.5f * (1.0f + vh.z);
  p2 = (1.0f - s) * std::sqrt(fmaxr(1.0f - p1 * p1, 0.0f)) + s * p2;
  float pz = std::sqrt(fmaxr(1.0f - p1 * p1 - p2 * p2, 0.0f));
  V3 nh = {p1 * t1.x + p2 * t2.x + pz * vh.x, p1 * t1.y + p2 * t2.y + pz * vh.y,
           p1 * t1.z + p2 * t2.z + pz * vh.z};
  return normalise({at * nh.x, ab * nh.y, fmaxr(nh.z, 1.0e-6f)});
}
static V3 sample_vndf(V3 v, float a, float u0, float u1) { return sample_vndf_at(v, a, a, u0, u1); }

static float vndf_reflect_pdf(V3 n, V3 v, V3 h, float a) {
  float nv = dot(n, v), nh = dot(n, h);
  if (nv <= 0.0f || nh <= 0.0f || dot(v, h) <= 0.0f) return 0.0f;
  return g1_iso(nv, a) * d_ggx(nh, a) / (4.0f * nv);
}
static V3 reflect(V3 v, V3 h) {
  float d = 2.0f * dot(v, h);
  return {d * h.x - v.x, d * h.y - v.y, d * h.z - v.z};
}
static bool refract(V3 v, V3 h, float eta, V3 &out) {
  float ci = dot(v, h);
  float s2 = eta * eta * fmaxr(1.0f - ci * ci, 0.0f);
  if (s2 >= 1.0f) return false;
  float ct = std::sqrt(1.0f - s2);
  float k = eta * ci - ct;
  out = normalise({-eta * v.x + k * h.x, -eta * v.y + k * h.y, -eta * v.z + k * h.z});
  return true;
}

// Sheen, src/pathtrace.rs:617-692.
static float d_charlie(float n_dot_h, float a) {
  float inv = 1.0f / fmaxr(a, 1.0e-3f);
  float sin2 = fmaxr(1.0f - n_dot_h * n_dot_h, 0.0f);
  return (2.0f + inv) * std::pow(sin2, inv * 0.5f) / (2.0f * PI);
}
static float v_neubelt(float nl, float nv) { return 1.0f / fmaxr(4.0f * (nl + nv - nl * nv), 1.0e-6f); }
constexpr int SHEEN_LUT_COS = 32, SHEEN_LUT_ROUGH = 16;
const std::vector<float> &sheen_lut() {
  static std::vector<float> lut;
  static std::once_flag once;
  std::call_once(once, [] {
    const int nt = 48, np = 24;
    lut.assign(SHEEN_LUT_COS * SHEEN_LUT_ROUGH, 0.0f);
    for (int ri = 0; ri < SHEEN_LUT_ROUGH; ++ri) {
      float r = (float)ri / (float)(SHEEN_LUT_ROUGH - 1);
      float a = fmaxr(r * r, 1.0e-3f);
      for (int ci = 0; ci < SHEEN_LUT_COS; ++ci) {
        float cv = fmaxr(((float)ci + 0.5f) / (float)SHEEN_LUT_COS, 1.0e-3f);
        V3 v = {std::sqrt(1.0f - cv * cv), 0.0f, cv};
        float sum = 0.0f;
        for (int i = 0; i < nt; ++i) {
          float th = ((float)i + 0.5f) / (float)nt * FRAC_PI_2;
          float st = std::sin(th), ct = std::cos(th);
          for (int j = 0; j < np; ++j) {
            float ph = ((float)j + 0.5f) / (float)np * PI;
            V3 l = {st * std::cos(ph), st * std::sin(ph), ct};
            V3 h = normalise(add(v, l));
            float f = d_charlie(h.z, a) * v_neubelt(ct, cv);
            sum += f * ct * st;
          }
        }
        float dw = (FRAC_PI_2 / (float)nt) * (PI / (float)np) * 2.0f;
        lut[ri * SHEEN_LUT_COS + ci] = clampr(sum * dw, 0.0f, 1.0f);
      }
    }
  });
  return lut;
}
float sheen_albedo(float cos, float rough) {
  const std::vector<float> &lut = sheen_lut();
  float x = clampr(clampr(cos, 0.0f, 1.0f) * (float)SHEEN_LUT_COS - 0.5f, 0.0f, (float)(SHEEN_LUT_COS - 1));
  float y = clampr(clampr(rough, 0.0f, 1.0f) * (float)(SHEEN_LUT_ROUGH - 1), 0.0f, (float)(SHEEN_LUT_ROUGH - 1));
  size_t x0 = (size_t)f2usize(std::floor(x)), y0 = (size_t)f2usize(std::floor(y));
  size_t x1 = std::min<size_t>(x0 + 1, SHEEN_LUT_COS - 1), y1 = std::min<size_t>(y0 + 1, SHEEN_LUT_ROUGH - 1);
  float fx = x - (float)x0, fy = y - (float)y0;
  auto at = [&](size_t xx, size_t yy) { return lut[yy * SHEEN_LUT_COS + xx]; };
  float a = at(x0, y0) + (at(x1, y0) - at(x0, y0)) * fx;
  float b = at(x0, y1) + (at(x1, y1) - at(x0, y1)) * fx;
  return a + (b - a) * fy;
}

// Microfacet methods, src/pathtrace.rs:720-811.
static Microfacet mf_isotropic(V3 n, float a) {
  Microfacet m;
  basis(n, m.t, m.b);
  m.n = n;
  m.at = a;
  m.ab = a;
  m.aniso = false;
  return m;
}
static V3 mf_local(const Microfacet &m, V3 w) { return {dot(w, m.t), dot(w, m.b), dot(w, m.n)}; }
static float mf_d(const Microfacet &m, V3 h) {
  if (!m.aniso) return d_ggx(dot(m.n, h), m.at);
  V3 hl = mf_local(m, h);
  if (hl.z <= 0.0f) return 0.0f;
  float x = hl.x / m.at, y = hl.y / m.ab;
  float e = x * x + y * y + hl.z * hl.z;
  return 1.0f / (PI * m.at * m.ab * e * e);
}
static float mf_lambda(const Microfacet &m, V3 w) {
  if (!m.aniso) return lambda_iso(dot(m.n, w), m.at);
  V3 wl = mf_local(m, w);
  float cz = fmaxr(std::fabs(wl.z), 1.0e-7f);
  float a2 = powi2(m.at * wl.x) + powi2(m.ab * wl.y);
  return (std::sqrt(1.0f + a2 / (cz * cz)) - 1.0f) * 0.5f;
}
static float mf_g1(const Microfacet &m, V3 v) { return 1.0f / (1.0f + mf_lambda(m, v)); }
static float mf_g2(const Microfacet &m, V3 v, V3 l) { return 1.0f / (1.0f + mf_lambda(m, v) + mf_lambda(m, l)); }
static float mf_pdf_reflect(const Microfacet &m, V3 v, V3 h) {
  if (!m.aniso) return vndf_reflect_pdf(m.n, v, h, m.at);
  float nv = dot(m.n, v), nh = dot(m.n, h);
  if (nv <= 0.0f || nh <= 0.0f || dot(v, h) <= 0.0f) return 0.0f;
  return mf_g1(m, v) * mf_d(m, h) / (4.0f * nv);
}
static bool mf_sample(const Microfacet &m, V3 v, float u0, float u1, V3 &out) {
  V3 vl = mf_local(m, v);
  if (vl.z <= 0.0f) return false;
  V3 h = m.aniso ? sample_vndf_at(vl, m.at, m.ab, u0, u1) : sample_vndf(vl, m.at, u0, u1);
  out = to_world(m.t, m.b, m.n, h);
  return true;
}

// Bsdf::new, src/pathtrace.rs:853-986.
Bsdf::Bsdf(const MaterialSample &m, V3 v_, V3 ng_, bool front) {
  auto flip = [&](V3 a) { return front ? a : neg(a); };
  v = v_;
  ng = flip(ng_);
  n = flip(m.normal);
  if (dot(n, v) <= 1.0e-4f) n = ng;
  ncc = flip(m.clearcoat_normal);
  if (dot(ncc, v) <= 1.0e-4f) ncc = n;
  thin = m.thickness <= 0.0f;
  float ior = (std::isfinite(m.ior) && m.ior >= 1.0f) ? m.ior : 1.5f;
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
  float alpha = fmaxr(m.roughness * m.roughness, MIN_ALPHA);
  float aniso = clampr(m.anisotropy, 0.0f, 1.0f);
  mf = mf_isotropic(n, alpha);
  if (aniso > 0.0f) {
    V3 d0 = m.anisotropy_direction;
    float dn = dot(d0, n);
    V3 t = normalise({d0.x - n.x * dn, d0.y - n.y * dn, d0.z - n.z * dn});
    if (dot(t, t) > 0.5f) {
      float at = alpha + (1.0f - alpha) * aniso * aniso;
      if (at > alpha) {
        mf.t = t;
        mf.b = cross(n, t);
        mf.n = n;
        mf.at = at;
        mf.ab = alpha;
        mf.aniso = true;
      }
    }
  }
  metallic = m.metallic;
  specular = clampr(m.specular, 0.0f, 1.0f);
  f0d = {fminr(r0 * m.specular_color.x, 1.0f), fminr(r0 * m.specular_color.y, 1.0f),
         fminr(r0 * m.specular_color.z, 1.0f)};
  transmission = m.transmission;
  clearcoat = inside ? 0.0f : m.clearcoat;
  cc_alpha = fmaxr(m.clearcoat_roughness * m.clearcoat_roughness, MIN_ALPHA);
  sheen = inside ? V3{0, 0, 0} : m.sheen_color;
  sheen_rough = m.sheen_roughness;
  sheen_alpha = fmaxr(m.sheen_roughness * m.sheen_roughness, 1.0e-3f);
  irid = inside ? 0.0f : clampr(m.iridescence, 0.0f, 1.0f);
  irid_ior = std::isfinite(m.iridescence_ior) ? fmaxr(m.iridescence_ior, 1.0f) : 1.3f;
  irid_thick = std::isfinite(m.iridescence_thickness) ? fmaxr(m.iridescence_thickness, 0.0f) : 400.0f;
  dt = clampr(m.diffuse_transmission, 0.0f, 1.0f);
  dt_color = {clampr(m.diffuse_transmission_color.x, 0.0f, 1.0f), clampr(m.diffuse_transmission_color.y, 0.0f, 1.0f),
              clampr(m.diffuse_transmission_color.z, 0.0f, 1.0f)};
  w_cc = 0.0f;
  for (float &p : probs) p = 0.0f;

  float cv = fmaxr(dot(n, v), 1.0e-4f);
  w_cc = clearcoat > 0.0f ? clearcoat * schlick({0.04f, 0.04f, 0.04f}, dot(ncc, v)).x : 0.0f;
  float sheen_max = max3(sheen);
  float e_v = sheen_max > 0.0f ? sheen_albedo(cv, sheen_rough) : 0.0f;
  float s_scale = (1.0f - w_cc) * (1.0f - sheen_max * e_v);
  V3 fd_v, fm_v;
  fresnel_pair(cv, fd_v, fm_v);
  float fd = max3(fd_v);
  float fm = mean3(fm_v);
  float m_ = metallic;
  float base_mean = fmaxr(mean3(base), 0.0f);
  float t = transmission;
  float p[6] = {
      s_scale * (1.0f - m_) * (1.0f - t) * (1.0f - dt) * (1.0f - fd) * base_mean,
      s_scale * ((1.0f - m_) * fd + m_ * fm),
      s_scale * (1.0f - m_) * t * (1.0f - fd) * base_mean,
      w_cc,
      (1.0f - w_cc) * sheen_max * e_v,
      s_scale * (1.0f - m_) * (1.0f - t) * dt * (1.0f - fd) * fmaxr(mean3(dt_color), 0.0f),
  };
  float sum = 0.0f;
  for (float x : p) sum += x;
  if (sum > 0.0f && std::isfinite(sum)) {
    for (int i = 0; i < 6; ++i) probs[i] = p[i] / sum;
  }
}

// src/pathtrace.rs:1021-1031
V3 Bsdf::fresnel_d(float c) const {
  if (eta_i > eta_t) {
    float eta = eta_i / eta_t;
    float s2 = eta * eta * fmaxr(1.0f - c * c, 0.0f);
    if (s2 >= 1.0f) return {1.0f, 1.0f, 1.0f};
    return schlick(f0d, std::sqrt(1.0f - s2));
  }
  return schlick(f0d, c);
}

// src/pathtrace.rs:1039-1072
void Bsdf::fresnel_pair(float c, V3 &fd_out, V3 &fm_out) const {
  V3 fd = scale(fresnel_d(c), specular);
  V3 fm = schlick(base, c);
  if (irid <= 0.0f) {
    fd_out = fd;
    fm_out = fm;
    return;
  }
  float i = irid;
  auto mix3 = [&](V3 a, V3 b) {
    return V3{a.x + (b.x - a.x) * i, a.y + (b.y - a.y) * i, a.z + (b.z - a.z) * i};
  };
  V3 fd_i = metallic < 1.0f ? iridescent_fresnel(1.0f, irid_ior, scale(f0d, specular), irid_thick, c) : fd;
  V3 fm_i = metallic > 0.0f ? iridescent_fresnel(1.0f, irid_ior, base, irid_thick, c) : fm;
  fd_out = mix3(fd, fd_i);
  fm_out = mix3(fm, fm_i);
}

// Bsdf::eval, src/pathtrace.rs:1075-1211.
void Bsdf::eval(V3 l, V3 &f_out, float &pdf_out) const {
  float nv = fmaxr(dot(n, v), 1.0e-4f);
  const float *p = probs;
  if (dot(ng, l) > 0.0f) {
    float nl = dot(n, l);
    V3 h = normalise(add(v, l));
    float vh = fmaxr(dot(v, h), 0.0f);
    V3 f = {0, 0, 0};
    float pdf = 0.0f;
    if (nl > 0.0f) {
      V3 fd, fm;
      fresnel_pair(vh, fd, fm);
      float spec_c = mf_d(mf, h) * mf_g2(mf, v, l) / (4.0f * nv * nl);
      float m = metallic;
      float diff_k = (1.0f - m) * (1.0f - transmission) * (1.0f - dt) * (1.0f - max3(fd)) / PI;
      V3 layer;
      for (int k = 0; k < 3; ++k) layer[k] = spec_c * ((1.0f - m) * fd[k] + m * fm[k]) + diff_k * base[k];
      float smax = max3(sheen);
      if (smax > 0.0f) {
        float sc = fminr(1.0f - smax * sheen_albedo(nv, sheen_rough), 1.0f - smax * sheen_albedo(nl, sheen_rough));
        float nh = dot(n, h);
        float sh = d_charlie(nh, sheen_alpha) * v_neubelt(nl, nv);
        for (int k = 0; k < 3; ++k) layer[k] = layer[k] * sc + sheen[k] * sh;
      }
      for (int k = 0; k < 3; ++k) f[k] = layer[k] * (1.0f - w_cc);
      pdf += (p[LOBE_DIFFUSE] + p[LOBE_SHEEN]) * nl / PI;
      pdf += p[LOBE_SPECULAR] * mf_pdf_reflect(mf, v, h);
    }
    if (clearcoat > 0.0f) {
      float cnv = fmaxr(dot(ncc, v), 1.0e-4f);
      float cnl = dot(ncc, l);
      if (cnl > 0.0f) {
        float cnh = dot(ncc, h);
        float c = w_cc * d_ggx(cnh, cc_alpha) * g2_iso(cnv, cnl, cc_alpha) / (4.0f * cnv * cnl);
        for (int k = 0; k < 3; ++k) f[k] += c;
        pdf += p[LOBE_CLEARCOAT] * vndf_reflect_pdf(ncc, v, h, cc_alpha);
      }
    }
    float cos = fmaxr(nl, 0.0f);
    f_out = scale(f, cos);
    pdf_out = pdf;
    return;
  }
  // Transmission.
  f_out = {0, 0, 0};
  pdf_out = 0.0f;
  if (metallic >= 1.0f || (transmission <= 0.0f && dt <= 0.0f)) return;
  float nl = -dot(n, l);
  if (nl <= 0.0f) return;
  float smax = max3(sheen);
  float layer_scale = (1.0f - w_cc) * (smax > 0.0f ? 1.0f - smax * sheen_albedo(nv, sheen_rough) : 1.0f);
  V3 f = {0, 0, 0};
  float pdf = 0.0f;
  if (dt > 0.0f && transmission < 1.0f) {
    V3 fd, fm;
    fresnel_pair(nv, fd, fm);
    float w = (1.0f - metallic) * (1.0f - transmission) * dt * (1.0f - max3(fd)) * layer_scale / PI;
    for (int k = 0; k < 3; ++k) f[k] += w * dt_color[k] * nl;
    pdf += p[LOBE_DIFFUSE_T] * nl / PI;
  }
  if (transmission <= 0.0f) {
    f_out = f;
    pdf_out = pdf;
    return;
  }
  float w = (1.0f - metallic) * transmission * layer_scale;
  float val, pdf_t;
  if (thin) {
    V3 lm = add(l, scale(n, 2.0f * nl));
    V3 h = normalise(add(v, lm));
    float vh = dot(v, h), nh = dot(n, h);
    if (vh <= 0.0f || nh <= 0.0f) {
      f_out = f;
      pdf_out = pdf;
      return;
    }
    V3 fdv, fmv;
    fresnel_pair(vh, fdv, fmv);
    float fd = max3(fdv);
    val = mf_d(mf, h) * mf_g2(mf, v, lm) / (4.0f * nv * nl) * (1.0f - fd);
    pdf_t = mf_pdf_reflect(mf, v, h);
  } else {
    float ei = eta_i, et = eta_t;
    V3 h = normalise({-(ei * v.x + et * l.x), -(ei * v.y + et * l.y), -(ei * v.z + et * l.z)});
    if (dot(h, n) < 0.0f) h = neg(h);
    float vh = dot(v, h), lh = dot(l, h), nh = dot(n, h);
    if (vh <= 0.0f || lh >= 0.0f || nh <= 0.0f) {
      f_out = f;
      pdf_out = pdf;
      return;
    }
    float denom = ei * vh + et * lh;
    if (std::fabs(denom) < 1.0e-6f) {
      f_out = f;
      pdf_out = pdf;
      return;
    }
    float d = mf_d(mf, h);
    V3 fdv, fmv;
    fresnel_pair(vh, fdv, fmv);
    float fd = max3(fdv);
    float jac = et * et * std::fabs(lh) / (denom * denom);
    val = vh * std::fabs(lh) * d * mf_g2(mf, v, l) * et * et * (1.0f - fd) / (nv * nl * denom * denom);
    pdf_t = mf_g1(mf, v) * vh * d / nv * jac;
  }
  for (int k = 0; k < 3; ++k) f[k] += base[k] * w * val * nl;
  f_out = f;
  pdf_out = pdf + p[LOBE_TRANSMISSION] * pdf_t;
}

// Bsdf::sample, src/pathtrace.rs:1216-1279.
bool Bsdf::sample(const float u[3], V3 &l_out, V3 &f_out, float &pdf_out) const {
  float acc = 0.0f;
  int lobe = -1;
  for (int i = 0; i < 6; ++i) {
    acc += probs[i];
    if (probs[i] > 0.0f && u[2] < acc) {
      lobe = i;
      break;
    }
  }
  if (lobe < 0) {
    for (int i = 5; i >= 0; --i)
      if (probs[i] > 0.0f) {
        lobe = i;
        break;
      }
    if (lobe < 0) return false;
  }
  V3 l;
  switch (lobe) {
    case LOBE_DIFFUSE:
    case LOBE_SHEEN: {
      V3 t, b;
      basis(n, t, b);
      l = to_world(t, b, n, cosine_hemisphere(u[0], u[1]));
      break;
    }
    case LOBE_DIFFUSE_T: {
      V3 t, b;
      basis(n, t, b);
      V3 d = cosine_hemisphere(u[0], u[1]);
      l = to_world(t, b, n, {d.x, d.y, -d.z});
      break;
    }
    case LOBE_CLEARCOAT: {
      V3 t, b;
      basis(ncc, t, b);
      V3 vl = {dot(v, t), dot(v, b), dot(v, ncc)};
      if (vl.z <= 0.0f) return false;
      V3 h = to_world(t, b, ncc, sample_vndf(vl, cc_alpha, u[0], u[1]));
      l = reflect(v, h);
      break;
    }
    case LOBE_SPECULAR:
    case LOBE_TRANSMISSION: {
      V3 h;
      if (!mf_sample(mf, v, u[0], u[1], h)) return false;
      if (lobe == LOBE_SPECULAR) {
        l = reflect(v, h);
      } else if (thin) {
        V3 r = reflect(v, h);
        float d = dot(r, n);
        l = add(r, scale(n, -2.0f * d));
      } else {
        if (!refract(v, h, eta_i / eta_t, l)) return false;
      }
      break;
    }
    default:
      return false;
  }
  if (!finite3(l) || dot(l, l) < 0.5f) return false;
  bool reflection = dot(ng, l) > 0.0f;
  bool transmits = lobe == LOBE_TRANSMISSION || lobe == LOBE_DIFFUSE_T;
  if (reflection == transmits) return false;
  V3 f;
  float pdf;
  eval(l, f, pdf);
  if (pdf <= 0.0f || !std::isfinite(pdf) || oracle::is_black(f) || !finite3(f)) return false;
  l_out = l;
  f_out = f;
  pdf_out = pdf;
  return true;
}

// eval_sensitivity, src/pathtrace.rs:1393-1417.
static V3 eval_sensitivity(float opd, V3 shift) {
  float phase = 2.0f * PI * opd * 1.0e-9f;
  const float val[3] = {5.4856e-13f, 4.4201e-13f, 5.2481e-13f};
  const float pos[3] = {1.6810e6f, 1.7953e6f, 2.2084e6f};
  const float var[3] = {4.3278e9f, 9.3046e9f, 6.6121e9f};
  float xyz[3];
  for (int k = 0; k < 3; ++k)
    xyz[k] = val[k] * std::sqrt(2.0f * PI * var[k]) * std::cos(pos[k] * phase + shift[k]) *
             std::exp(-phase * phase * var[k]);
  xyz[0] += 9.7470e-14f * std::sqrt(2.0f * PI * 4.5282e9f) * std::cos(2.2399e6f * phase + shift[0]) *
            std::exp(-4.5282e9f * phase * phase);
  for (float &x : xyz) x /= 1.0685e-7f;
  return {3.2404542f * xyz[0] - 1.5371385f * xyz[1] - 0.4985314f * xyz[2],
          -0.969266f * xyz[0] + 1.8760108f * xyz[1] + 0.041556f * xyz[2],
          0.0556434f * xyz[0] - 0.2040259f * xyz[1] + 1.0572252f * xyz[2]};
}

// iridescent_fresnel, src/pathtrace.rs:1326-1387.
V3 iridescent_fresnel(float outside_ior, float film_ior, V3 base_f0, float thickness_nm, float cos1) {
  cos1 = clampr(cos1, 0.0f, 1.0f);
  float r0 = powi2((film_ior - outside_ior) / (film_ior + outside_ior));
  float r12 = r0 + (1.0f - r0) * powi5(1.0f - cos1);
  float t121 = 1.0f - r12;
  float sin2_2 = powi2(outside_ior / film_ior) * (1.0f - cos1 * cos1);
  float cos2_sq = 1.0f - sin2_2;
  if (cos2_sq < 0.0f) return {1.0f, 1.0f, 1.0f};
  float cos2 = std::sqrt(cos2_sq);
  float r23[3], phi23[3] = {0, 0, 0};
  for (int k = 0; k < 3; ++k) {
    float f0 = clampr(base_f0[k] + 1.0e-4f, 0.0f, 0.9999f);
    float sq = std::sqrt(f0);
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
  for (int k = 0; k < 3; ++k) {
    r123[k] = clampr(r12 * r23[k], 1.0e-5f, 0.9999f);
    rs[k] = t121 * t121 * r23[k] / (1.0f - r123[k]);
    out[k] = r12 + rs[k];
  }
  float cm[3] = {rs[0] - t121, rs[1] - t121, rs[2] - t121};
  for (int m = 1; m <= 2; ++m) {
    for (int k = 0; k < 3; ++k) cm[k] *= std::sqrt(r123[k]);
    V3 sm = eval_sensitivity((float)m * opd, {(float)m * phi[0], (float)m * phi[1], (float)m * phi[2]});
    for (int k = 0; k < 3; ++k) out[k] += cm[k] * 2.0f * sm[k];
  }
  return {clampr(out[0], 0.0f, 1.0f), clampr(out[1], 0.0f, 1.0f), clampr(out[2], 0.0f, 1.0f)};
}

// dispersion_iors, src/pathtrace.rs:1422-1425.
void dispersion_iors(float ior, float dispersion, float out[3]) {
  float hs = (ior - 1.0f) * 0.025f * fmaxr(dispersion, 0.0f);
  out[0] = fmaxr(ior - hs, 1.0f);
  out[1] = fmaxr(ior, 1.0f);
  out[2] = fmaxr(ior + hs, 1.0f);
}

// triangle_solid_angle (Van Oosterom & Strackee), src/pathtrace.rs:1755-1784.
float triangle_solid_angle(V3 p, V3 a_, V3 b_, V3 c_) {
  auto u = [&](V3 q, double o[3]) {
    double d[3] = {(double)(q.x - p.x), (double)(q.y - p.y), (double)(q.z - p.z)};
    double l = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (l > 0.0) {
      o[0] = d[0] / l;
      o[1] = d[1] / l;
      o[2] = d[2] / l;
    } else {
      o[0] = o[1] = o[2] = 0.0;
    }
  };
  double a[3], b[3], c[3];
  u(a_, a);
  u(b_, b);
  u(c_, c);
  auto dt = [](const double x[3], const double y[3]) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; };
  double bc[3] = {b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0]};
  double num = std::fabs(dt(a, bc));
  double den = 1.0 + dt(a, b) + dt(b, c) + dt(c, a);
  double o = 2.0 * std::atan2(num, den);
  if (std::isfinite(o)) return (float)std::fmax(o, 0.0);
  return 0.0f;
}

// sample_spherical_triangle (Arvo 1995), src/pathtrace.rs:1789-1871.
bool sample_spherical_triangle(V3 p, V3 a_, V3 b_, V3 c_, float u0, float u1, V3 &out) {
  struct D3 {
    double v[3];
  };
  auto sub = [&](V3 x) { return D3{{(double)(x.x - p.x), (double)(x.y - p.y), (double)(x.z - p.z)}}; };
  auto dt = [](D3 x, D3 y) { return x.v[0] * y.v[0] + x.v[1] * y.v[1] + x.v[2] * y.v[2]; };
  auto cr = [](D3 x, D3 y) {
    return D3{{x.v[1] * y.v[2] - x.v[2] * y.v[1], x.v[2] * y.v[0] - x.v[0] * y.v[2], x.v[0] * y.v[1] - x.v[1] * y.v[0]}};
  };
  auto norm = [&](D3 x, D3 &o) {
    double l = std::sqrt(dt(x, x));
    if (!(l > 1.0e-300 && std::isfinite(l))) return false;
    o = D3{{x.v[0] / l, x.v[1] / l, x.v[2] / l}};
    return true;
  };
  D3 a, b, c;
  if (!norm(sub(a_), a) || !norm(sub(b_), b) || !norm(sub(c_), c)) return false;
  D3 nab, nbc, nca;
  if (!norm(cr(a, b), nab) || !norm(cr(b, c), nbc) || !norm(cr(c, a), nca)) return false;
  auto ang = [&](D3 x, D3 y) { return std::acos(clampd(-dt(x, y), -1.0, 1.0)); };
  double alpha = ang(nab, nca), beta = ang(nbc, nab), gamma = ang(nca, nbc);
  double area = alpha + beta + gamma - 3.14159265358979323846;
  if (std::isnan(area) || area <= 0.0) return false;
  double ap = (double)u0 * area;
  double s = std::sin(ap - alpha), t = std::cos(ap - alpha);
  double sa = std::sin(alpha), ca = std::cos(alpha);
  double cos_c = dt(a, b);
  double uu = t - ca;
  double vv = s + sa * cos_c;
  double den = (vv * s + uu * t) * sa;
  if (std::fabs(den) < 1.0e-300) return false;
  double q = clampd(((vv * t - uu * s) * ca - vv) / den, -1.0, 1.0);
  D3 ca_perp;
  double dca = dt(c, a);
  if (!norm(D3{{c.v[0] - dca * a.v[0], c.v[1] - dca * a.v[1], c.v[2] - dca * a.v[2]}}, ca_perp)) return false;
  double r = std::sqrt(std::fmax(1.0 - q * q, 0.0));
  D3 cp = {{q * a.v[0] + r * ca_perp.v[0], q * a.v[1] + r * ca_perp.v[1], q * a.v[2] + r * ca_perp.v[2]}};
  double z = 1.0 - (double)u1 * (1.0 - dt(cp, b));
  double dcpb = dt(cp, b);
  D3 cb_perp;
  bool has_perp = norm(D3{{cp.v[0] - dcpb * b.v[0], cp.v[1] - dcpb * b.v[1], cp.v[2] - dcpb * b.v[2]}}, cb_perp);
  double w = std::sqrt(std::fmax(1.0 - z * z, 0.0));
  D3 d = has_perp ? D3{{z * b.v[0] + w * cb_perp.v[0], z * b.v[1] + w * cb_perp.v[1], z * b.v[2] + w * cb_perp.v[2]}}
                  : b;
  D3 dn;
  if (!norm(d, dn)) return false;
  out = {(float)dn.v[0], (float)dn.v[1], (float)dn.v[2]};
  return true;
}

}  // namespace oracle
