// Device scene queries: BVH traversal with the watertight triangle test
// (TraceScene::closest_hit_filtered / occluded_filtered,
// src/trace.rs:405-450, over a host-built binned-SAH tree; Woop, Benthin &
// Wald, JCGT 2(1) 2013), hit surfaces (:459-488), texture sampling
// (src/texture.rs:277-515), material evaluation (src/trace.rs:491-923),
// punctual lights (src/prepare.rs:921-963) and the environment map
// (src/pathtrace.rs:1557-1741).
//
// Closest hit = the accepted candidate with the smallest t, ties broken by
// the lowest global triangle id, so the answer does not depend on the tree
// or the traversal order. Node boxes are padded on the host and the slab
// test widens t_far by 1 + 2*gamma(3), so a triangle the watertight test
// accepts is never culled by a box.
#pragma once

#include "dev_bsdf.cuh"
#include "dev_types.h"

namespace ptd {

constexpr int kStackSize = 64;  // the host builder caps tree depth below this
constexpr uint32_t kLeafCountShift = 27;
constexpr uint32_t kLeafFirstMask = (1u << kLeafCountShift) - 1u;

struct Hit {
  float t;
  uint32_t g;
  float b0, b1, b2;
  bool front;
};

struct Ray {
  V3 o, d;
  int kx, ky, kz;
  float sx, sy, sz;
  V3 inv;  // box-test reciprocal (zero components nudged to +-1e-30)
};

PT_DEV Ray make_ray(V3 o, V3 d) {
  Ray r;
  r.o = o;
  r.d = d;
  int kz = 0;
  if (fabsf(d.y) > fabsf(d.x)) kz = 1;
  if (fabsf(d.z) > fabsf(kz == 0 ? d.x : d.y)) kz = 2;
  int kx = kz == 2 ? 0 : kz + 1;
  int ky = kx == 2 ? 0 : kx + 1;
  float dk = d[kz];
  if (dk < 0.0f) {
    int t = kx;
    kx = ky;
    ky = t;
  }
  r.kx = kx;
  r.ky = ky;
  r.kz = kz;
  r.sx = d[kx] / dk;
  r.sy = d[ky] / dk;
  r.sz = 1.0f / dk;
  auto nz = [](float v) { return fabsf(v) < 1.0e-30f ? copysignf(1.0e-30f, v) : v; };
  r.inv = {1.0f / nz(d.x), 1.0f / nz(d.y), 1.0f / nz(d.z)};
  return r;
}

PT_DEV float comp(V3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// Woop et al. 2013, identical arithmetic to the oracle.
PT_DEV bool intersect_watertight(const Ray &r, V3 v0, V3 v1, V3 v2, float &t, float &b0, float &b1, float &b2,
                                 bool &front) {
  V3 a = vsub(v0, r.o), b = vsub(v1, r.o), c = vsub(v2, r.o);
  float akz = comp(a, r.kz), bkz = comp(b, r.kz), ckz = comp(c, r.kz);
  float ax = comp(a, r.kx) - r.sx * akz, ay = comp(a, r.ky) - r.sy * akz;
  float bx = comp(b, r.kx) - r.sx * bkz, by = comp(b, r.ky) - r.sy * bkz;
  float cx = comp(c, r.kx) - r.sx * ckz, cy = comp(c, r.ky) - r.sy * ckz;
  float u = cx * by - cy * bx;
  float v = ax * cy - ay * cx;
  float w = bx * ay - by * ax;
  if (u == 0.0f || v == 0.0f || w == 0.0f) {
    u = (float)((double)cx * (double)by - (double)cy * (double)bx);
    v = (float)((double)ax * (double)cy - (double)ay * (double)cx);
    w = (float)((double)bx * (double)ay - (double)by * (double)ax);
  }
  if ((u < 0.0f || v < 0.0f || w < 0.0f) && (u > 0.0f || v > 0.0f || w > 0.0f)) return false;
  float det = u + v + w;
  if (det == 0.0f) return false;
  float az = r.sz * akz, bz = r.sz * bkz, cz = r.sz * ckz;
  float tt = u * az + v * bz + w * cz;
  float rcp = 1.0f / det;
  t = tt * rcp;
  b0 = u * rcp;
  b1 = v * rcp;
  b2 = w * rcp;
  front = det > 0.0f;
  return true;
}

PT_DEV float4 ldg4(const float4 *p) { return __ldg(p); }

// Slab test of both children of a node against [t0, t1]; returns entry distances.
PT_DEV void node_boxes(const BvhNode *node, const Ray &r, float t0, float t1, bool &h0, bool &h1, float &e0,
                       float &e1, int4 &d) {
  const float grow = 1.0000003576f;  // 1 + 2 * gamma(3)
  float4 a = ldg4(&node->a), b = ldg4(&node->b), c = ldg4(&node->c);
  d = __ldg(&node->d);
  float ox = r.o.x, oy = r.o.y, oz = r.o.z;
  float ix = r.inv.x, iy = r.inv.y, iz = r.inv.z;
  {
    float lx = (a.x - ox) * ix, hx = (a.y - ox) * ix;
    float ly = (a.z - oy) * iy, hy = (a.w - oy) * iy;
    float lz = (c.x - oz) * iz, hz = (c.y - oz) * iz;
    float tn = fmaxf(fmaxf(fminf(lx, hx), fminf(ly, hy)), fmaxf(fminf(lz, hz), t0));
    float tf = fminf(fminf(fmaxf(lx, hx), fmaxf(ly, hy)), fmaxf(lz, hz)) * grow;
    tf = fminf(tf, t1);
    h0 = tn <= tf;
    e0 = tn;
  }
  {
    float lx = (b.x - ox) * ix, hx = (b.y - ox) * ix;
    float ly = (b.z - oy) * iy, hy = (b.w - oy) * iy;
    float lz = (c.z - oz) * iz, hz = (c.w - oz) * iz;
    float tn = fmaxf(fmaxf(fminf(lx, hx), fminf(ly, hy)), fmaxf(fminf(lz, hz), t0));
    float tf = fminf(fminf(fmaxf(lx, hx), fmaxf(ly, hy)), fmaxf(lz, hz)) * grow;
    tf = fminf(tf, t1);
    h1 = tn <= tf;
    e1 = tn;
  }
}

struct TraversalStats {
  uint32_t nodes, tris;
};

// Closest accepted hit in [t_min, t_max]. `accept(g, t, b0, b1, b2, front)`
// is the any-hit filter (alpha mask, stochastic blend, primary culling).
template <class Accept>
PT_DEV bool closest_hit(const DevScene &s, V3 o, V3 d, float t_min, float t_max, Accept &&accept, Hit &best,
                        TraversalStats &st, uint32_t &err) {
  if (s.node_count == 0) return false;
  Ray r = make_ray(o, d);
  bool have = false;
  best.t = t_max;
  best.g = 0xffffffffu;
  int stack[kStackSize];
  int sp = 0;
  int cur = 0;
  for (;;) {
    if (cur >= 0) {
      st.nodes++;
      bool h0, h1;
      float e0, e1;
      int4 dd;
      node_boxes(s.nodes + cur, r, t_min, best.t, h0, h1, e0, e1, dd);
      if (h0 && h1) {
        int nearc = e1 < e0 ? dd.y : dd.x;
        int farc = e1 < e0 ? dd.x : dd.y;
        if (sp < kStackSize) {
          stack[sp++] = farc;
        } else {
          err |= ERR_STACK_OVERFLOW;
        }
        cur = nearc;
        continue;
      }
      if (h0) {
        cur = dd.x;
        continue;
      }
      if (h1) {
        cur = dd.y;
        continue;
      }
    } else {
      // Leaf reference ~(first | count << 27): records [first, first + count).
      uint32_t first = (uint32_t)(~cur);
      uint32_t count = first >> kLeafCountShift;
      first &= kLeafFirstMask;
      for (uint32_t i = 0; i < count; ++i) {
        const float4 *tr = s.tris + 3u * (first + i);
        float4 p0 = ldg4(tr), p1 = ldg4(tr + 1), p2 = ldg4(tr + 2);
        st.tris++;
        float t, b0, b1, b2;
        bool front;
        if (!intersect_watertight(r, {p0.x, p0.y, p0.z}, {p1.x, p1.y, p1.z}, {p2.x, p2.y, p2.z}, t, b0, b1, b2, front))
          continue;
        if (!(t >= t_min)) continue;
        uint32_t g = __float_as_uint(p0.w);
        bool better = have ? (t < best.t || (t == best.t && g < best.g)) : (t <= t_max);
        if (!better) continue;
        if (accept(g, __float_as_uint(p1.w), t, b0, b1, b2, front)) {
          best.t = t;
          best.g = g;
          best.b0 = b0;
          best.b1 = b1;
          best.b2 = b2;
          best.front = front;
          have = true;
        }
      }
    }
    if (sp == 0) break;
    cur = stack[--sp];
  }
  return have;
}

// Any accepted hit in [t_min, t_max].
template <class Accept>
PT_DEV bool occluded(const DevScene &s, V3 o, V3 d, float t_min, float t_max, Accept &&accept, TraversalStats &st,
                     uint32_t &err) {
  if (s.node_count == 0) return false;
  Ray r = make_ray(o, d);
  int stack[kStackSize];
  int sp = 0;
  int cur = 0;
  for (;;) {
    if (cur >= 0) {
      st.nodes++;
      bool h0, h1;
      float e0, e1;
      int4 dd;
      node_boxes(s.nodes + cur, r, t_min, t_max, h0, h1, e0, e1, dd);
      if (h0 && h1) {
        if (sp < kStackSize) {
          stack[sp++] = dd.y;
        } else {
          err |= ERR_STACK_OVERFLOW;
        }
        cur = dd.x;
        continue;
      }
      if (h0) {
        cur = dd.x;
        continue;
      }
      if (h1) {
        cur = dd.y;
        continue;
      }
    } else {
      uint32_t first = (uint32_t)(~cur);
      uint32_t count = first >> kLeafCountShift;
      first &= kLeafFirstMask;
      for (uint32_t i = 0; i < count; ++i) {
        const float4 *tr = s.tris + 3u * (first + i);
        float4 p0 = ldg4(tr), p1 = ldg4(tr + 1), p2 = ldg4(tr + 2);
        st.tris++;
        float t, b0, b1, b2;
        bool front;
        if (!intersect_watertight(r, {p0.x, p0.y, p0.z}, {p1.x, p1.y, p1.z}, {p2.x, p2.y, p2.z}, t, b0, b1, b2, front))
          continue;
        if (!(t >= t_min && t <= t_max)) continue;
        if (accept(__float_as_uint(p0.w), __float_as_uint(p1.w), t, b0, b1, b2, front)) return true;
      }
    }
    if (sp == 0) break;
    cur = stack[--sp];
  }
  return false;
}

// ---------------------------------------------------------------- attributes
PT_DEV V3 ld3(const float *p) { return {__ldg(p), __ldg(p + 1), __ldg(p + 2)}; }
PT_DEV float4 ld4f(const float *p) { return make_float4(__ldg(p), __ldg(p + 1), __ldg(p + 2), __ldg(p + 3)); }

// interp3 / interp2 / interp4 (src/trace.rs:1178-1204) over corners 3g..3g+2.
PT_DEV V3 interp3(const float *s, uint32_t g, float b0, float b1, float b2) {
  const float *p = s + 9u * g;
  V3 x = ld3(p), y = ld3(p + 3), z = ld3(p + 6);
  return {x.x * b0 + y.x * b1 + z.x * b2, x.y * b0 + y.y * b1 + z.y * b2, x.z * b0 + y.z * b1 + z.z * b2};
}
PT_DEV void interp2(const float *s, uint32_t g, float b0, float b1, float b2, float out[2]) {
  const float *p = s + 6u * g;
  float x0 = __ldg(p), x1 = __ldg(p + 1), y0 = __ldg(p + 2), y1 = __ldg(p + 3), z0 = __ldg(p + 4), z1 = __ldg(p + 5);
  out[0] = x0 * b0 + y0 * b1 + z0 * b2;
  out[1] = x1 * b0 + y1 * b1 + z1 * b2;
}
PT_DEV float4 interp4(const float *s, uint32_t g, float b0, float b1, float b2) {
  const float *p = s + 12u * g;
  float4 x = ld4f(p), y = ld4f(p + 4), z = ld4f(p + 8);
  return make_float4(x.x * b0 + y.x * b1 + z.x * b2, x.y * b0 + y.y * b1 + z.y * b2, x.z * b0 + y.z * b1 + z.z * b2,
                     x.w * b0 + y.w * b1 + z.w * b2);
}

struct Surface {
  V3 position, ng, sn;
};

// TraceScene::surface, src/trace.rs:459-488.
PT_DEV Surface surface(const DevScene &s, uint32_t g, float b0, float b1, float b2, uint32_t flags) {
  Surface out;
  out.position = interp3(s.pos, g, b0, b1, b2);
  const float *p = s.pos + 9u * g;
  V3 p0 = ld3(p), p1 = ld3(p + 3), p2 = ld3(p + 6);
  V3 cr = vcross(vsub(p1, p0), vsub(p2, p0));
  float len = sqrtf(vdot(cr, cr));
  out.ng = len > 0.0f ? V3{cr.x / len, cr.y / len, cr.z / len} : V3{0.0f, 0.0f, 1.0f};
  out.sn = out.ng;
  if (flags & TRI_HAS_VN) {
    V3 n = vnormalise(interp3(s.nrm, g, b0, b1, b2));
    out.sn = vdot(n, n) > 0.5f ? n : out.ng;
  }
  return out;
}

// ---------------------------------------------------------------- textures
PT_DEV uint32_t wrap_index(int64_t i, int64_t n, uint32_t mode) {
  int64_t r;
  if (mode == PT_WRAP_REPEAT) {
    r = i % n;
    if (r < 0) r += n;
  } else if (mode == PT_WRAP_CLAMP) {
    r = i < 0 ? 0 : (i > n - 1 ? n - 1 : i);
  } else {
    int64_t m = i % (2 * n);
    if (m < 0) m += 2 * n;
    r = m >= n ? 2 * n - 1 - m : m;
  }
  return (uint32_t)r;
}
PT_DEV float4 lerp4(float4 a, float4 b, float t) {
  return make_float4(a.x + (b.x - a.x) * t, a.y + (b.y - a.y) * t, a.z + (b.z - a.z) * t, a.w + (b.w - a.w) * t);
}
// filter_level, src/texture.rs:486-515.
PT_DEV float4 filter_level(const float4 *texels, uint32_t w, uint32_t h, float u, float v, bool linear, uint32_t ws,
                           uint32_t wt) {
  u = isfinite(u) ? u : 0.0f;
  v = isfinite(v) ? v : 0.0f;
  u = clampr(u, -1.0e6f, 1.0e6f);
  v = clampr(v, -1.0e6f, 1.0e6f);
  float x = u * (float)w, y = v * (float)h;
  if (!linear) {
    uint32_t xi = wrap_index(f2i64(floorf(x)), w, ws), yi = wrap_index(f2i64(floorf(y)), h, wt);
    return __ldg(texels + (size_t)yi * w + xi);
  }
  float xf = x - 0.5f, yf = y - 0.5f;
  float x0 = floorf(xf), y0 = floorf(yf);
  float fx = xf - x0, fy = yf - y0;
  int64_t ix = f2i64(x0), iy = f2i64(y0);
  uint32_t xa = wrap_index(ix, w, ws), xb = wrap_index(ix + 1, w, ws);
  uint32_t ya = wrap_index(iy, h, wt), yb = wrap_index(iy + 1, h, wt);
  float4 a = __ldg(texels + (size_t)ya * w + xa), b = __ldg(texels + (size_t)ya * w + xb);
  float4 c = __ldg(texels + (size_t)yb * w + xa), d = __ldg(texels + (size_t)yb * w + xb);
  return lerp4(lerp4(a, b, fx), lerp4(c, d, fx), fy);
}
// PreparedTexture::sample_lod, src/texture.rs:420-451.
PT_DEV float4 sample_lod(const DevScene &s, const DevTexture &t, float u, float v, float lod, bool srgb) {
  const uint64_t *off = srgb ? t.srgb_off : t.lin_off;
  if (isnan(lod) || lod <= 0.0f)
    return filter_level(s.texels + off[0], t.lw[0], t.lh[0], u, v, t.mag == PT_FILTER_LINEAR, t.wrap_s, t.wrap_t);
  uint32_t mn = t.min;
  bool lin = (mn == PT_MIN_LINEAR || mn == PT_MIN_LINEAR_MIP_NEAREST || mn == PT_MIN_LINEAR_MIP_LINEAR);
  float max_level = (float)(t.levels - 1);
  if (mn == PT_MIN_NEAREST || mn == PT_MIN_LINEAR)
    return filter_level(s.texels + off[0], t.lw[0], t.lh[0], u, v, lin, t.wrap_s, t.wrap_t);
  if (mn == PT_MIN_NEAREST_MIP_NEAREST || mn == PT_MIN_LINEAR_MIP_NEAREST) {
    uint32_t l = f2u32(clampr(roundf(lod), 0.0f, max_level));
    return filter_level(s.texels + off[l], t.lw[l], t.lh[l], u, v, lin, t.wrap_s, t.wrap_t);
  }
  float l = clampr(lod, 0.0f, max_level);
  uint32_t l0 = f2u32(floorf(l));
  uint32_t l1 = min(l0 + 1, t.levels - 1);
  float f = l - (float)l0;
  float4 a = filter_level(s.texels + off[l0], t.lw[l0], t.lh[l0], u, v, lin, t.wrap_s, t.wrap_t);
  if (f <= 0.0f || l0 == l1) return a;
  float4 b = filter_level(s.texels + off[l1], t.lw[l1], t.lh[l1], u, v, lin, t.wrap_s, t.wrap_t);
  return lerp4(a, b, f);
}

// Texture LOD of a hit: ray cone at the camera vertex, level 0 after.
struct TexLod {
  bool cone;
  float width;
  V3 dir;
  static constexpr bool kGrad = false;
};

// TexLod of the raycast backend (src/trace.rs:171-195): level 0, a ray cone,
// or ray differentials — the barycentric change per output pixel along x
// (gx) and y (gy).
struct RayTexLod {
  bool cone;
  float width;
  V3 dir;
  bool grad;
  float gx[3], gy[3];
  static constexpr bool kGrad = true;
};

// f32::hypot as glibc's hypotf computes it: the f64 root of the f64 sum of
// the (exact) f64 squares, rounded once to f32.
PT_DEV float hypot_f32(float a, float b) {
  const double x = (double)a, y = (double)b;
  return (float)sqrt(x * x + y * y);
}

PT_DEV void transform_uv(const pt_texture_binding &b, float uv[2]) {
  if (!b.has_transform) return;
  float u = uv[0], v = uv[1];
  uv[0] = b.transform[0] * u + b.transform[1] * v + b.transform[2];
  uv[1] = b.transform[3] * u + b.transform[4] * v + b.transform[5];
}

// TraceScene::lod (src/trace.rs:518-554) + ::sample / ::sample_at, and for
// ray differentials ::sample_grad (:596-620) with Texture::sample_grad
// (src/texture.rs:456-474).
template <class Lod>
PT_DEV bool sample_binding(const DevScene &s, const pt_texture_binding &bd, uint32_t g, uint32_t flags, float b0,
                           float b1, float b2, const Lod &lod, bool srgb, float4 &out) {
  int ti = bd.texture;
  if (ti < 0 || (uint32_t)ti >= s.texture_count) return false;
  uint32_t set = bd.uv_set;
  if (set >= PT_MAX_UV_SETS || !(flags & (TRI_UV0 << set))) return false;
  const DevTexture &tex = s.textures[ti];
  const float *uvs = s.uv[set];
  if constexpr (Lod::kGrad) {
    if (lod.grad) {
      // Move the barycentrics by one pixel, difference the transformed UVs.
      const float *q = uvs + 6u * g;
      const float u0 = __ldg(q), v0 = __ldg(q + 1), u1 = __ldg(q + 2), v1 = __ldg(q + 3), u2 = __ldg(q + 4),
                  v2 = __ldg(q + 5);
      float uv[2];
      interp2(uvs, g, b0, b1, b2, uv);
      float tuv[2] = {uv[0], uv[1]};
      transform_uv(bd, tuv);
      float dx[2] = {uv[0] + u0 * lod.gx[0] + u1 * lod.gx[1] + u2 * lod.gx[2],
                     uv[1] + v0 * lod.gx[0] + v1 * lod.gx[1] + v2 * lod.gx[2]};
      float dy[2] = {uv[0] + u0 * lod.gy[0] + u1 * lod.gy[1] + u2 * lod.gy[2],
                     uv[1] + v0 * lod.gy[0] + v1 * lod.gy[1] + v2 * lod.gy[2]};
      transform_uv(bd, dx);
      transform_uv(bd, dy);
      const float w = (float)tex.img_w, h = (float)tex.img_h;
      const float lx = hypot_f32((dx[0] - tuv[0]) * w, (dx[1] - tuv[1]) * h);
      const float ly = hypot_f32((dy[0] - tuv[0]) * w, (dy[1] - tuv[1]) * h);
      const float rho = fmaxf(lx, ly);
      const float l = (isfinite(rho) && rho > 0.0f) ? log2f(rho) : 0.0f;
      out = sample_lod(s, tex, tuv[0], tuv[1], l, srgb);
      return true;
    }
  }
  float l = 0.0f;
  if (lod.cone) {
    const float *q = uvs + 6u * g;
    float uv0[2] = {__ldg(q), __ldg(q + 1)}, uv1[2] = {__ldg(q + 2), __ldg(q + 3)}, uv2[2] = {__ldg(q + 4), __ldg(q + 5)};
    transform_uv(bd, uv0);
    transform_uv(bd, uv1);
    transform_uv(bd, uv2);
    float ta = (float)tex.img_w * (float)tex.img_h *
               fabsf((uv1[0] - uv0[0]) * (uv2[1] - uv0[1]) - (uv2[0] - uv0[0]) * (uv1[1] - uv0[1]));
    const float *p = s.pos + 9u * g;
    V3 p0 = ld3(p), p1 = ld3(p + 3), p2 = ld3(p + 6);
    V3 cr = vcross(vsub(p1, p0), vsub(p2, p0));
    float pa = sqrtf(vdot(cr, cr));
    if (ta > 0.0f && pa > 0.0f && lod.width > 0.0f) {
      V3 n = {cr.x / pa, cr.y / pa, cr.z / pa};
      float cs = fmaxf(fabsf(vdot(n, lod.dir)), 1.0e-3f);
      float lv = 0.5f * log2f(ta / pa) + log2f(lod.width / cs);
      l = isfinite(lv) ? lv : 0.0f;
    }
  }
  float uv[2];
  interp2(uvs, g, b0, b1, b2, uv);
  transform_uv(bd, uv);
  out = sample_lod(s, tex, uv[0], uv[1], l, srgb);
  return true;
}

// TraceScene::alpha, src/trace.rs:492-506.
PT_DEV float hit_alpha(const DevScene &s, const pt_material &mat, uint32_t g, uint32_t flags, float b0, float b1,
                       float b2) {
  float a = mat.base_color[3];
  float4 t;
  TexLod base{false, 0.0f, vzero()};
  if (sample_binding(s, mat.base_color_texture, g, flags, b0, b1, b2, base, true, t)) a *= t.w;
  if (flags & TRI_HAS_COLORS) a *= interp4(s.col, g, b0, b1, b2).w;
  return a;
}

// tangent_frame / perturb, src/trace.rs:640-687.
PT_DEV bool tangent_frame(const DevScene &s, uint32_t g, uint32_t flags, float b0, float b1, float b2, V3 n, V3 &tt,
                          V3 &bt) {
  if (!(flags & TRI_HAS_TANGENTS)) return false;
  float4 tg = interp4(s.tan, g, b0, b1, b2);
  float w = __ldg(s.tan + 12u * g + 3) < 0.0f ? -1.0f : 1.0f;
  V3 t3 = {tg.x, tg.y, tg.z};
  float d = vdot(n, t3);
  tt = vnormalise({t3.x - n.x * d, t3.y - n.y * d, t3.z - n.z * d});
  if (vdot(tt, tt) < 0.5f) return false;
  V3 c = vcross(n, tt);
  bt = {c.x * w, c.y * w, c.z * w};
  return true;
}
PT_DEV V3 perturb(const DevScene &s, uint32_t g, uint32_t flags, float b0, float b1, float b2, V3 n, float4 t,
                  float sc) {
  V3 tt, bt;
  if (!tangent_frame(s, g, flags, b0, b1, b2, n, tt, bt)) return n;
  float ts0 = (t.x * 2.0f - 1.0f) * sc, ts1 = (t.y * 2.0f - 1.0f) * sc, ts2 = t.z * 2.0f - 1.0f;
  V3 nn = vnormalise({tt.x * ts0 + bt.x * ts1 + n.x * ts2, tt.y * ts0 + bt.y * ts1 + n.y * ts2,
                      tt.z * ts0 + bt.z * ts1 + n.z * ts2});
  return vdot(nn, nn) > 0.5f ? nn : n;
}
PT_DEV float fin(float v, float d) { return isfinite(v) ? v : d; }

// TraceScene::material_oriented, src/trace.rs:700-923 (the occlusion
// input is evaluated only when kOcclusion is set: the path tracer never
// reads it).
template <bool kOcclusion = false, class Lod>
PT_DEV void material_oriented(const DevScene &s, const DevMaterial &dm, uint32_t g, uint32_t flags, float b0, float b1,
                              float b2, V3 shading_normal, const Lod &lod, bool flip, MaterialSample &m) {
  const pt_material &mat = dm.m;
  V3 sn = flip ? vneg(shading_normal) : shading_normal;
  float4 t;
  float col[4] = {mat.base_color[0], mat.base_color[1], mat.base_color[2], mat.base_color[3]};
  if (sample_binding(s, mat.base_color_texture, g, flags, b0, b1, b2, lod, true, t)) {
    col[0] *= t.x;
    col[1] *= t.y;
    col[2] *= t.z;
    col[3] *= t.w;
  }
  if (flags & TRI_HAS_COLORS) {
    float4 v = interp4(s.col, g, b0, b1, b2);
    col[0] *= v.x;
    col[1] *= v.y;
    col[2] *= v.z;
    col[3] *= v.w;
  }
  float metallic = mat.metallic, roughness = mat.roughness;
  if (sample_binding(s, mat.metallic_roughness_texture, g, flags, b0, b1, b2, lod, false, t)) {
    roughness *= t.y;
    metallic *= t.z;
  }
  V3 normal = sn;
  if (sample_binding(s, mat.normal_texture, g, flags, b0, b1, b2, lod, false, t))
    normal = perturb(s, g, flags, b0, b1, b2, normal, t, mat.normal_scale);
  if constexpr (kOcclusion) {
    float occlusion = 1.0f;
    if (sample_binding(s, mat.occlusion_texture, g, flags, b0, b1, b2, lod, false, t))
      occlusion = 1.0f + mat.occlusion_strength * (t.x - 1.0f);
    m.occlusion = clampr(occlusion, 0.0f, 1.0f);
  }
  V3 emissive = {mat.emissive[0], mat.emissive[1], mat.emissive[2]};
  if (sample_binding(s, mat.emissive_texture, g, flags, b0, b1, b2, lod, true, t)) {
    emissive.x *= t.x;
    emissive.y *= t.y;
    emissive.z *= t.z;
  }
  uint32_t ext = mat.ext_flags;
  float specular = 1.0f;
  V3 specular_color = {1.0f, 1.0f, 1.0f};
  if (ext & PT_EXT_SPECULAR) {
    specular = clampr(fin(mat.specular_factor, 1.0f), 0.0f, 1.0f);
    if (sample_binding(s, mat.specular_texture, g, flags, b0, b1, b2, lod, false, t)) specular *= t.w;
    specular_color = {fmaxf(fin(mat.specular_color_factor[0], 1.0f), 0.0f),
                      fmaxf(fin(mat.specular_color_factor[1], 1.0f), 0.0f),
                      fmaxf(fin(mat.specular_color_factor[2], 1.0f), 0.0f)};
    if (sample_binding(s, mat.specular_color_texture, g, flags, b0, b1, b2, lod, true, t)) {
      specular_color.x *= t.x;
      specular_color.y *= t.y;
      specular_color.z *= t.z;
    }
  }
  float transmission = 0.0f;
  if (ext & PT_EXT_TRANSMISSION) {
    transmission = clampr(fin(mat.transmission_factor, 0.0f), 0.0f, 1.0f);
    if (sample_binding(s, mat.transmission_texture, g, flags, b0, b1, b2, lod, false, t)) transmission *= t.x;
  }
  float thickness = 0.0f, attenuation_distance = inf();
  V3 attenuation_color = {1.0f, 1.0f, 1.0f};
  if (ext & PT_EXT_VOLUME) {
    thickness = fmaxf(fin(mat.thickness_factor, 0.0f), 0.0f);
    if (sample_binding(s, mat.thickness_texture, g, flags, b0, b1, b2, lod, false, t)) thickness *= t.y;
    attenuation_color = {clampr(fin(mat.attenuation_color[0], 1.0f), 0.0f, 1.0f),
                         clampr(fin(mat.attenuation_color[1], 1.0f), 0.0f, 1.0f),
                         clampr(fin(mat.attenuation_color[2], 1.0f), 0.0f, 1.0f)};
    float d = mat.attenuation_distance;
    attenuation_distance = (isfinite(d) && d > 0.0f) ? d : inf();
  }
  float clearcoat = 0.0f, clearcoat_roughness = 0.0f;
  V3 clearcoat_normal = sn;
  if (ext & PT_EXT_CLEARCOAT) {
    clearcoat = clampr(fin(mat.clearcoat_factor, 0.0f), 0.0f, 1.0f);
    if (sample_binding(s, mat.clearcoat_texture, g, flags, b0, b1, b2, lod, false, t)) clearcoat *= t.x;
    clearcoat_roughness = clampr(fin(mat.clearcoat_roughness_factor, 0.0f), 0.0f, 1.0f);
    if (sample_binding(s, mat.clearcoat_roughness_texture, g, flags, b0, b1, b2, lod, false, t))
      clearcoat_roughness *= t.y;
    if (sample_binding(s, mat.clearcoat_normal_texture, g, flags, b0, b1, b2, lod, false, t))
      clearcoat_normal = perturb(s, g, flags, b0, b1, b2, sn, t, fin(mat.clearcoat_normal_scale, 1.0f));
  }
  V3 sheen_color = vzero();
  float sheen_roughness = 0.0f;
  if (ext & PT_EXT_SHEEN) {
    sheen_color = {clampr(fin(mat.sheen_color_factor[0], 0.0f), 0.0f, 1.0f),
                   clampr(fin(mat.sheen_color_factor[1], 0.0f), 0.0f, 1.0f),
                   clampr(fin(mat.sheen_color_factor[2], 0.0f), 0.0f, 1.0f)};
    if (sample_binding(s, mat.sheen_color_texture, g, flags, b0, b1, b2, lod, true, t)) {
      sheen_color.x *= t.x;
      sheen_color.y *= t.y;
      sheen_color.z *= t.z;
    }
    sheen_roughness = clampr(fin(mat.sheen_roughness_factor, 0.0f), 0.0f, 1.0f);
    if (sample_binding(s, mat.sheen_roughness_texture, g, flags, b0, b1, b2, lod, false, t)) sheen_roughness *= t.w;
  }
  float anisotropy = 0.0f;
  V3 anisotropy_direction = vzero();
  if (ext & PT_EXT_ANISOTROPY) {
    anisotropy = clampr(fin(mat.anisotropy_strength, 0.0f), 0.0f, 1.0f);
    float dir0 = 1.0f, dir1 = 0.0f;
    if (sample_binding(s, mat.anisotropy_texture, g, flags, b0, b1, b2, lod, false, t)) {
      dir0 = t.x * 2.0f - 1.0f;
      dir1 = t.y * 2.0f - 1.0f;
      anisotropy *= clampr(t.z, 0.0f, 1.0f);
    }
    float sr = dm.aniso_sin, cr = dm.aniso_cos;
    float rot0 = cr * dir0 - sr * dir1, rot1 = sr * dir0 + cr * dir1;
    V3 tt, bt;
    if (tangent_frame(s, g, flags, b0, b1, b2, sn, tt, bt)) {
      V3 d = vnormalise({tt.x * rot0 + bt.x * rot1, tt.y * rot0 + bt.y * rot1, tt.z * rot0 + bt.z * rot1});
      if (vdot(d, d) > 0.5f) anisotropy_direction = d;
    }
    if (vdot(anisotropy_direction, anisotropy_direction) < 0.5f) anisotropy = 0.0f;
  }
  float iridescence = 0.0f, iridescence_ior = 1.3f, iridescence_thickness = 400.0f;
  if (ext & PT_EXT_IRIDESCENCE) {
    iridescence = clampr(fin(mat.iridescence_factor, 0.0f), 0.0f, 1.0f);
    if (sample_binding(s, mat.iridescence_texture, g, flags, b0, b1, b2, lod, false, t)) iridescence *= t.x;
    iridescence_ior = fmaxf(fin(mat.iridescence_ior, 1.3f), 1.0f);
    float lo = fin(mat.iridescence_thickness_min, 100.0f), hi = fin(mat.iridescence_thickness_max, 400.0f);
    float gg = 1.0f;
    if (sample_binding(s, mat.iridescence_thickness_texture, g, flags, b0, b1, b2, lod, false, t))
      gg = clampr(t.y, 0.0f, 1.0f);
    iridescence_thickness = fmaxf(lo + (hi - lo) * gg, 0.0f);
  }
  float dtr = 0.0f;
  V3 dt_color = {1.0f, 1.0f, 1.0f};
  if (ext & PT_EXT_DIFFUSE_TRANSMISSION) {
    dtr = clampr(fin(mat.diffuse_transmission_factor, 0.0f), 0.0f, 1.0f);
    if (sample_binding(s, mat.diffuse_transmission_texture, g, flags, b0, b1, b2, lod, false, t)) dtr *= t.w;
    dt_color = {clampr(fin(mat.diffuse_transmission_color_factor[0], 1.0f), 0.0f, 1.0f),
                clampr(fin(mat.diffuse_transmission_color_factor[1], 1.0f), 0.0f, 1.0f),
                clampr(fin(mat.diffuse_transmission_color_factor[2], 1.0f), 0.0f, 1.0f)};
    if (sample_binding(s, mat.diffuse_transmission_color_texture, g, flags, b0, b1, b2, lod, true, t)) {
      dt_color.x *= t.x;
      dt_color.y *= t.y;
      dt_color.z *= t.z;
    }
  }
  m.base_color[0] = col[0];
  m.base_color[1] = col[1];
  m.base_color[2] = col[2];
  m.base_color[3] = col[3];
  m.metallic = clampr(metallic, 0.0f, 1.0f);
  m.roughness = clampr(roughness, 0.0f, 1.0f);
  m.normal = normal;
  m.emissive = emissive;
  m.unlit = mat.unlit;
  m.double_sided = mat.double_sided;
  m.ior = mat.ior;
  m.specular = specular;
  m.specular_color = specular_color;
  m.transmission = transmission;
  m.thickness = thickness;
  m.attenuation_color = attenuation_color;
  m.attenuation_distance = attenuation_distance;
  m.clearcoat = clearcoat;
  m.clearcoat_roughness = clearcoat_roughness;
  m.clearcoat_normal = clearcoat_normal;
  m.sheen_color = sheen_color;
  m.sheen_roughness = sheen_roughness;
  m.anisotropy = anisotropy;
  m.anisotropy_direction = anisotropy_direction;
  m.iridescence = iridescence;
  m.iridescence_ior = iridescence_ior;
  m.iridescence_thickness = iridescence_thickness;
  m.diffuse_transmission = dtr;
  m.diffuse_transmission_color = dt_color;
  m.dispersion = (ext & PT_EXT_DISPERSION) ? fmaxf(fin(mat.dispersion, 0.0f), 0.0f) : 0.0f;
}

// ---------------------------------------------------------------- lights
struct LightSample {
  V3 l;
  float distance;
  V3 radiance;
};
// PreparedLight::sample, src/prepare.rs:921-963.
PT_DEV bool light_sample(const DevLight &dl, V3 p, LightSample &out) {
  const pt_light &L = dl.l;
  V3 base = {L.color[0] * L.intensity, L.color[1] * L.intensity, L.color[2] * L.intensity};
  if (L.kind == PT_LIGHT_DIRECTIONAL) {
    out.l = {-L.direction[0], -L.direction[1], -L.direction[2]};
    out.distance = inf();
    out.radiance = base;
    return true;
  }
  V3 to = vsub({L.position[0], L.position[1], L.position[2]}, p);
  float d2 = vdot(to, to);
  if (isnan(d2) || d2 <= 1.0e-12f) return false;
  float d = sqrtf(d2);
  V3 l = {to.x / d, to.y / d, to.z / d};
  float att = 1.0f / d2;
  if (L.has_range) {
    float x = d / L.range;
    att *= clampr(1.0f - x * x * x * x, 0.0f, 1.0f);
  }
  if (L.kind == PT_LIGHT_SPOT) {
    float sc = 1.0f / fmaxf(dl.cos_inner - dl.cos_outer, 0.001f);
    float offset = -dl.cos_outer * sc;
    float cd = vdot({L.direction[0], L.direction[1], L.direction[2]}, {-l.x, -l.y, -l.z});
    float a = clampr(cd * sc + offset, 0.0f, 1.0f);
    att *= a * a;
  }
  if (att <= 0.0f) return false;
  out.l = l;
  out.distance = d;
  out.radiance = {base.x * att, base.y * att, base.z * att};
  return true;
}

// EmissiveLights::pick (partition_point(c <= u)), src/pathtrace.rs:1550-1554.
PT_DEV uint32_t upper_bound(const float *a, uint32_t n, float u) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (__ldg(a + mid) <= u)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// ---------------------------------------------------------------- environment
PT_DEV void env_texel_of(const DevEnv &e, V3 d, uint32_t &x, uint32_t &y, float &st) {
  float u = 0.5f + atan2f(d.x, -d.z) / (2.0f * PI);
  float th = acosf(clampr(d.y, -1.0f, 1.0f));
  float v = th / PI;
  x = min(f2u32(u * (float)e.w), e.w - 1);
  y = min(f2u32(v * (float)e.h), e.h - 1);
  st = sinf(th);
}
PT_DEV V3 env_radiance(const DevEnv &e, V3 d) {
  uint32_t x, y;
  float st;
  env_texel_of(e, d, x, y, st);
  if (e.uniform || !e.pixels) return vzero();
  float4 c = __ldg(e.pixels + (size_t)y * e.w + x);
  V3 cc = {c.x, c.y, c.z};
  if (!finite3(cc)) return vzero();
  return vscale({fmaxf(cc.x, 0.0f), fmaxf(cc.y, 0.0f), fmaxf(cc.z, 0.0f)}, e.intensity);
}
PT_DEV float env_pdf(const DevEnv &e, V3 d) {
  uint32_t x, y;
  float st;
  env_texel_of(e, d, x, y, st);
  if (st <= 1.0e-6f) return 0.0f;
  return __ldg(e.mass + (size_t)y * e.w + x) * (float)(e.w * e.h) / (2.0f * PI * PI * st);
}
PT_DEV bool env_sample(const DevEnv &e, float u0, float u1, V3 &d, V3 &le, float &p) {
  uint32_t yy = upper_bound(e.marginal, e.h + 1, u0);
  uint32_t y = min(max(yy, 1u), e.h) - 1;
  const float *row = e.conditional + (size_t)y * (e.w + 1);
  uint32_t xx = upper_bound(row, e.w + 1, u1);
  uint32_t x = min(max(xx, 1u), e.w) - 1;
  float my = (u0 - __ldg(e.marginal + y)) / fmaxf(__ldg(e.marginal + y + 1) - __ldg(e.marginal + y), 1e-12f);
  float mx = (u1 - __ldg(row + x)) / fmaxf(__ldg(row + x + 1) - __ldg(row + x), 1e-12f);
  float u = ((float)x + clampr(mx, 0.0f, 0.99999f)) / (float)e.w;
  float v = ((float)y + clampr(my, 0.0f, 0.99999f)) / (float)e.h;
  float phi = 2.0f * PI * (u - 0.5f);
  float th = PI * v;
  float st = sinf(th), ct = cosf(th);
  d = {st * sinf(phi), ct, -st * cosf(phi)};
  p = env_pdf(e, d);
  if (p <= 0.0f || !isfinite(p)) return false;
  le = env_radiance(e, d);
  return true;
}

}  // namespace ptd
