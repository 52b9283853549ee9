// Device math shared by every kernel: f32 vector helpers with the
// reference's rounding order (src/math.rs:53-91, src/pathtrace.rs:431-506),
// Rust float semantics (max/min ignore NaN, clamp keeps NaN, saturating
// casts), and the Owen-scrambled Sobol' sampler (src/pathtrace.rs:297-425).
//
// The library is compiled with --fmad=false, -prec-div=true and
// -prec-sqrt=true: every + - * / sqrt below rounds exactly once in source
// order, like the reference's Rust, so integer work and the geometry chain
// (sampler -> primary ray -> watertight test) reproduce bit for bit.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define PT_DEV __device__ __forceinline__
#define PT_HD __host__ __device__ __forceinline__

namespace ptd {

constexpr float PI = 3.14159265358979323846f;
constexpr float FRAC_PI_2 = 1.57079632679489661923f;
constexpr float FRAC_PI_4 = 0.785398163397448309616f;
constexpr float F32_EPSILON = 1.1920928955078125e-07f;
constexpr float F32_MIN_POSITIVE = 1.17549435e-38f;

PT_DEV float inf() { return __int_as_float(0x7f800000); }

struct V3 {
  float x, y, z;
  PT_DEV float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
PT_DEV V3 v3(float x, float y, float z) { return V3{x, y, z}; }
PT_DEV V3 vadd(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
PT_DEV V3 vsub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
PT_DEV V3 vscale(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
PT_DEV V3 vmul(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
PT_DEV V3 vneg(V3 a) { return {-a.x, -a.y, -a.z}; }
PT_DEV float vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PT_DEV V3 vcross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
// vec3_normalise: vectors shorter than f32::EPSILON map to zero.
PT_DEV V3 vnormalise(V3 v) {
  float len = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
  if (len < F32_EPSILON) return {0.0f, 0.0f, 0.0f};
  return {v.x / len, v.y / len, v.z / len};
}
PT_DEV float max3(V3 a) { return fmaxf(fmaxf(a.x, a.y), a.z); }
PT_DEV float mean3(V3 a) { return (a.x + a.y + a.z) * (1.0f / 3.0f); }
PT_DEV float luminance(V3 a) { return 0.2126f * a.x + 0.7152f * a.y + 0.0722f * a.z; }
PT_DEV bool is_black(V3 a) { return !(a.x > 0.0f || a.y > 0.0f || a.z > 0.0f); }
PT_DEV bool finite3(V3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
PT_DEV V3 vzero() { return {0.0f, 0.0f, 0.0f}; }

// f32::clamp keeps NaN.
PT_DEV float clampr(float x, float lo, float hi) {
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}
PT_DEV double clampd(double x, double lo, double hi) {
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}
// Saturating float -> int casts (Rust `as`), NaN -> 0.
PT_DEV uint32_t f2u32(float f) {
  if (!(f > 0.0f)) return 0u;
  if (f >= 4294967296.0f) return 0xffffffffu;
  return (uint32_t)f;
}
PT_DEV int64_t f2i64(float f) {
  if (isnan(f)) return 0;
  if (f <= -9223372036854775808.0f) return INT64_MIN;
  if (f >= 9223372036854775808.0f) return INT64_MAX;
  return (int64_t)f;
}
PT_DEV int32_t f2i32(float f) {
  if (isnan(f)) return 0;
  if (f <= -2147483648.0f) return INT32_MIN;
  if (f >= 2147483648.0f) return INT32_MAX;
  return (int32_t)f;
}
// f32::powi with the constant exponents the reference uses.
PT_DEV float powi2(float x) { return x * x; }
PT_DEV float powi5(float x) {
  float x2 = x * x;
  float x4 = x2 * x2;
  return x * x4;
}

// Orthonormal basis (Duff et al. 2017), src/pathtrace.rs:470-478.
PT_DEV void basis(V3 n, V3 &t, V3 &b) {
  float sign = copysignf(1.0f, n.z);
  float a = -1.0f / (sign + n.z);
  float bb = n.x * n.y * a;
  t = {1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x};
  b = {bb, sign + n.y * n.y * a, -n.y};
}
PT_DEV V3 to_world(V3 t, V3 b, V3 n, V3 v) {
  return {t.x * v.x + b.x * v.y + n.x * v.z, t.y * v.x + b.y * v.y + n.y * v.z, t.z * v.x + b.z * v.y + n.z * v.z};
}

// ---------------------------------------------------------------- sampler

PT_HD uint32_t pcg_hash(uint32_t x) {
  uint32_t state = x * 747796405u + 2891336453u;
  uint32_t word = ((state >> ((state >> 28) + 4u)) ^ state) * 277803737u;
  return (word >> 22) ^ word;
}
PT_HD uint32_t hash_mix(uint32_t a, uint32_t b) { return pcg_hash(a ^ pcg_hash(b)); }

// Generator matrices of dims 1-3 (Joe & Kuo polynomials (1,0,[1]),
// (2,1,[1,3]), (3,1,[1,3,1])); dim 0 is the bit reversal. Built at compile
// time so the Sobol' loop below XORs immediates.
struct SobolTable {
  uint32_t m[3][32];
};
constexpr SobolTable make_sobol() {
  SobolTable t{};
  const int s_[3] = {1, 2, 3};
  const uint32_t a_[3] = {0, 1, 1};
  const uint32_t init[3][3] = {{1, 0, 0}, {1, 3, 0}, {1, 3, 1}};
  for (int d = 0; d < 3; ++d) {
    uint32_t mm[32] = {};
    int s = s_[d];
    for (int i = 0; i < s; ++i) mm[i] = init[d][i];
    for (int k = s; k < 32; ++k) {
      uint32_t v = mm[k - s] ^ (mm[k - s] << s);
      for (int j = 1; j < s; ++j)
        if ((a_[d] >> (s - 1 - j)) & 1u) v ^= mm[k - j] << j;
      mm[k] = v;
    }
    for (int k = 0; k < 32; ++k) t.m[d][k] = mm[k] << (31 - k);
  }
  return t;
}
// Constant-initialised per translation unit; the unrolled loop reads it at
// warp-uniform addresses (constant-cache broadcast).
static __constant__ SobolTable c_sobol = make_sobol();

template <int D>
PT_DEV uint32_t sobol_dim(uint32_t index) {
  if (D == 0) return __brev(index);
  uint32_t r = 0;
#pragma unroll
  for (int k = 0; k < 32; ++k) r ^= ((index >> k) & 1u) ? c_sobol.m[D - 1][k] : 0u;
  return r;
}
PT_DEV uint32_t laine_karras(uint32_t x, uint32_t seed) {
  x += seed;
  x ^= x * 0x6c50b47cu;
  x ^= x * 0xb82f1e52u;
  x ^= x * 0xc7afe638u;
  x ^= x * 0x8d22f6e6u;
  return x;
}
PT_DEV uint32_t nested_uniform_scramble(uint32_t x, uint32_t seed) { return __brev(laine_karras(__brev(x), seed)); }
PT_DEV float to_unit(uint32_t v) { return (float)(v >> 8) * (1.0f / 16777216.0f); }

// sobol_owen_4d (src/pathtrace.rs:388-398).
PT_DEV void sobol_owen_4d(uint32_t index, uint32_t pattern_seed, float out[4]) {
  uint32_t i = nested_uniform_scramble(index, pattern_seed);
  out[0] = to_unit(nested_uniform_scramble(sobol_dim<0>(i), hash_mix(pattern_seed, 0u)));
  out[1] = to_unit(nested_uniform_scramble(sobol_dim<1>(i), hash_mix(pattern_seed, 1u)));
  out[2] = to_unit(nested_uniform_scramble(sobol_dim<2>(i), hash_mix(pattern_seed, 2u)));
  out[3] = to_unit(nested_uniform_scramble(sobol_dim<3>(i), hash_mix(pattern_seed, 3u)));
}

// Sampler (src/pathtrace.rs:401-425).
struct Sampler {
  uint32_t pixel_seed, index, path_seed;
  PT_DEV void init(uint32_t seed, uint32_t x, uint32_t y, uint32_t idx) {
    pixel_seed = hash_mix(hash_mix(seed, y), x);
    index = idx;
    path_seed = hash_mix(pixel_seed, idx);
  }
  PT_DEV void pattern(uint32_t p, float out[4]) const { sobol_owen_4d(index, hash_mix(pixel_seed, p), out); }
  PT_DEV float coin(uint32_t ray, uint32_t tri) const { return to_unit(hash_mix(hash_mix(path_seed, ray), tri)); }
};

}  // namespace ptd
