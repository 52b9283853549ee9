// ORACLE — test infrastructure only. A CPU restatement of oxideav-render's
// PathTrace backend used to check the CUDA library (tests/, smoke() and the
// bench's cpu_baseline leg are its only users; nothing in the product links it).
//
// Parity status: the reference is Rust and cannot be built in this container
// (no cargo/rustc; the BVH / ray crate oxideav-mesh3d "0.0" is not vendored).
// This restatement is pinned to the reference's own known-answer tests
// (src/pathtrace.rs:2866-3750, src/trace.rs:1222-1308), which tests/ port.
//
// Compiled with -O2 -ffp-contract=off and no fast-math: Rust never fuses
// multiply-adds, so every f32 expression below rounds in the order written,
// exactly like the reference's source.
//
// This header: vector helpers (src/math.rs, src/pathtrace.rs:431-506),
// sampling (src/pathtrace.rs:297-425), microfacet + BSDF (src/pathtrace.rs:508-1311),
// iridescence (:1313-1425), spherical triangles (:1743-1871).
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <optional>
#include <vector>

namespace oracle {

constexpr float PI = 3.14159265358979323846f;
constexpr float FRAC_PI_2 = 1.57079632679489661923f;
constexpr float FRAC_PI_4 = 0.785398163397448309616f;
constexpr float INF = std::numeric_limits<float>::infinity();

struct V3 {
  float x, y, z;
  float &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
struct V4 {
  float v[4];
  float &operator[](int i) { return v[i]; }
  float operator[](int i) const { return v[i]; }
};

// ---- Rust float semantics ------------------------------------------------
// f32::max / f32::min ignore a NaN operand (like fmax / fmin).
inline float fmaxr(float a, float b) { return std::fmax(a, b); }
inline float fminr(float a, float b) { return std::fmin(a, b); }
// f32::clamp keeps NaN (src: core::f32::clamp).
inline float clampr(float x, float lo, float hi) {
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}
inline double clampd(double x, double lo, double hi) {
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}
// `as usize` / `as i64` / `as i32` casts saturate and map NaN to 0.
inline uint64_t f2usize(float f) {
  if (!(f > 0.0f)) return 0;
  if (f >= 18446744073709551616.0f) return UINT64_MAX;
  return (uint64_t)f;
}
inline int64_t f2i64(float f) {
  if (std::isnan(f)) return 0;
  if (f <= -9223372036854775808.0f) return INT64_MIN;
  if (f >= 9223372036854775808.0f) return INT64_MAX;
  return (int64_t)f;
}
inline int32_t f2i32(float f) {
  if (std::isnan(f)) return 0;
  if (f <= -2147483648.0f) return INT32_MIN;
  if (f >= 2147483648.0f) return INT32_MAX;
  return (int32_t)f;
}
// f32::powi for the constant exponents the reference uses (LLVM expands
// powi by binary exponentiation: x^5 = x * (x^2)^2).
inline float powi2(float x) { return x * x; }
inline float powi5(float x) {
  float x2 = x * x;
  float x4 = x2 * x2;
  return x * x4;
}

// ---- vector helpers (src/math.rs:53-91, src/pathtrace.rs:431-466) --------
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 scale(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 mul(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V3 neg(V3 a) { return {-a.x, -a.y, -a.z}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// vec3_normalise: zero vector (len < f32::EPSILON) maps to zero.
inline V3 normalise(V3 v) {
  float len = std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
  if (len < FLT_EPSILON) return {0.0f, 0.0f, 0.0f};
  return {v.x / len, v.y / len, v.z / len};
}
inline float max3(V3 a) { return fmaxr(fmaxr(a.x, a.y), a.z); }
inline float mean3(V3 a) { return (a.x + a.y + a.z) * (1.0f / 3.0f); }
inline float luminance(V3 a) { return 0.2126f * a.x + 0.7152f * a.y + 0.0722f * a.z; }
inline bool is_black(V3 a) { return !(a.x > 0.0f || a.y > 0.0f || a.z > 0.0f); }
inline bool finite3(V3 a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }

// basis (Duff et al. 2017), src/pathtrace.rs:470-478.
inline void basis(V3 n, V3 &t, V3 &b) {
  float sign = std::copysign(1.0f, n.z);
  float a = -1.0f / (sign + n.z);
  float bb = n.x * n.y * a;
  t = {1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x};
  b = {bb, sign + n.y * n.y * a, -n.y};
}
inline V3 to_world(V3 t, V3 b, V3 n, V3 v) {
  return {t.x * v.x + b.x * v.y + n.x * v.z, t.y * v.x + b.y * v.y + n.y * v.z,
          t.z * v.x + b.z * v.y + n.z * v.z};
}
// cosine_hemisphere, src/pathtrace.rs:491-506.
inline V3 cosine_hemisphere(float u0, float u1) {
  float a = 2.0f * u0 - 1.0f;
  float b = 2.0f * u1 - 1.0f;
  float r, phi;
  if (a == 0.0f && b == 0.0f) {
    r = 0.0f;
    phi = 0.0f;
  } else if (std::fabs(a) > std::fabs(b)) {
    r = a;
    phi = FRAC_PI_4 * (b / a);
  } else {
    r = b;
    phi = FRAC_PI_2 - FRAC_PI_4 * (a / b);
  }
  float x = r * std::cos(phi), y = r * std::sin(phi);
  return {x, y, std::sqrt(fmaxr(1.0f - x * x - y * y, 0.0f))};
}

// ---- sampling (src/pathtrace.rs:297-425) ---------------------------------
inline uint32_t pcg_hash(uint32_t x) {
  uint32_t state = x * 747796405u + 2891336453u;
  uint32_t word = ((state >> ((state >> 28) + 4u)) ^ state) * 277803737u;
  return (word >> 22) ^ word;
}
inline uint32_t hash_mix(uint32_t a, uint32_t b) { return pcg_hash(a ^ pcg_hash(b)); }
inline uint32_t reverse_bits(uint32_t x) {
  x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
  x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
  x = ((x >> 4) & 0x0F0F0F0Fu) | ((x & 0x0F0F0F0Fu) << 4);
  x = ((x >> 8) & 0x00FF00FFu) | ((x & 0x00FF00FFu) << 8);
  return (x >> 16) | (x << 16);
}
// Joe & Kuo direction numbers for dims 1-3, van der Corput for dim 0
// (sobol_matrices, src/pathtrace.rs:319-346).
struct SobolMatrices {
  uint32_t m[4][32];
  SobolMatrices() {
    for (int k = 0; k < 32; ++k) m[0][k] = 1u << (31 - k);
    const int s_[3] = {1, 2, 3};
    const uint32_t a_[3] = {0, 1, 1};
    const uint32_t init[3][3] = {{1, 0, 0}, {1, 3, 0}, {1, 3, 1}};
    for (int d = 0; d < 3; ++d) {
      int s = s_[d];
      uint32_t a = a_[d];
      uint32_t mm[32] = {0};
      for (int i = 0; i < s; ++i) mm[i] = init[d][i];
      for (int k = s; k < 32; ++k) {
        uint32_t v = mm[k - s] ^ (mm[k - s] << s);
        for (int j = 1; j < s; ++j)
          if ((a >> (s - 1 - j)) & 1u) v ^= mm[k - j] << j;
        mm[k] = v;
      }
      for (int k = 0; k < 32; ++k) m[d + 1][k] = mm[k] << (31 - k);
    }
  }
};
const SobolMatrices &sobol_matrices();
inline uint32_t sobol(uint32_t index, int dim) {
  const uint32_t *m = sobol_matrices().m[dim];
  uint32_t r = 0, i = index;
  int k = 0;
  while (i != 0) {
    if (i & 1u) r ^= m[k];
    i >>= 1;
    k += 1;
  }
  return r;
}
inline uint32_t laine_karras(uint32_t x, uint32_t seed) {
  x += seed;
  x ^= x * 0x6c50b47cu;
  x ^= x * 0xb82f1e52u;
  x ^= x * 0xc7afe638u;
  x ^= x * 0x8d22f6e6u;
  return x;
}
inline uint32_t nested_uniform_scramble(uint32_t x, uint32_t seed) {
  return reverse_bits(laine_karras(reverse_bits(x), seed));
}
inline float to_unit(uint32_t v) { return (float)(v >> 8) * (1.0f / 16777216.0f); }
inline void sobol_owen_4d(uint32_t index, uint32_t pattern_seed, float out[4]) {
  uint32_t i = nested_uniform_scramble(index, pattern_seed);
  for (int d = 0; d < 4; ++d)
    out[d] = to_unit(nested_uniform_scramble(sobol(i, d), hash_mix(pattern_seed, (uint32_t)d)));
}
struct Sampler {
  uint32_t pixel_seed, index, path_seed;
  Sampler(uint32_t seed, uint32_t x, uint32_t y, uint32_t idx) {
    pixel_seed = hash_mix(hash_mix(seed, y), x);
    index = idx;
    path_seed = hash_mix(pixel_seed, idx);
  }
  void pattern(uint32_t p, float out[4]) const { sobol_owen_4d(index, hash_mix(pixel_seed, p), out); }
  float coin(uint32_t ray, uint32_t tri) const { return to_unit(hash_mix(hash_mix(path_seed, ray), tri)); }
};

// ---- MaterialSample (src/trace.rs:202-305) -------------------------------
struct MaterialSample {
  float base_color[4] = {1, 1, 1, 1};
  float metallic = 1.0f;
  float roughness = 1.0f;
  V3 normal = {0, 0, 1};
  float occlusion = 1.0f;
  V3 emissive = {0, 0, 0};
  bool unlit = false;
  uint32_t alpha_mode = 0;
  float alpha_cutoff = 0.5f;
  bool double_sided = false;
  float ior = 1.5f;
  float specular = 1.0f;
  V3 specular_color = {1, 1, 1};
  float transmission = 0.0f;
  float thickness = 0.0f;
  V3 attenuation_color = {1, 1, 1};
  float attenuation_distance = INF;
  float clearcoat = 0.0f;
  float clearcoat_roughness = 0.0f;
  V3 clearcoat_normal = {0, 0, 1};
  V3 sheen_color = {0, 0, 0};
  float sheen_roughness = 0.0f;
  float anisotropy = 0.0f;
  V3 anisotropy_direction = {0, 0, 0};
  float iridescence = 0.0f;
  float iridescence_ior = 1.3f;
  float iridescence_thickness = 400.0f;
  float diffuse_transmission = 0.0f;
  V3 diffuse_transmission_color = {1, 1, 1};
  float dispersion = 0.0f;
};

// ---- BSDF ------------------------------------------------------------------
struct Microfacet {
  V3 t, b, n;
  float at, ab;
  bool aniso;
};

class Bsdf {
 public:
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

  Bsdf(const MaterialSample &m, V3 v, V3 ng, bool front);
  bool is_black() const {
    for (float p : probs)
      if (p > 0.0f) return false;
    return true;
  }
  V3 fresnel_d(float c) const;
  void fresnel_pair(float c, V3 &fd, V3 &fm) const;
  // f(v,l)|n.l| and mixture pdf.
  void eval(V3 l, V3 &f, float &pdf) const;
  // Returns false when the sample carries no energy.
  bool sample(const float u[3], V3 &l, V3 &f, float &pdf) const;
};

V3 iridescent_fresnel(float outside_ior, float film_ior, V3 base_f0, float thickness_nm, float cos1);
void dispersion_iors(float ior, float dispersion, float out[3]);
float sheen_albedo(float cos, float rough);
const std::vector<float> &sheen_lut();
float triangle_solid_angle(V3 p, V3 a, V3 b, V3 c);
bool sample_spherical_triangle(V3 p, V3 a, V3 b, V3 c, float u0, float u1, V3 &out);
constexpr float MIN_SPHERICAL_SOLID_ANGLE = 1.0e-4f;

}  // namespace oracle
