// ORACLE — test infrastructure only (see oracle_core.hpp).
// Scene side of the restatement: texture mip chains and sampling
// (src/texture.rs:268-515), the traced triangle soup with a BVH and the
// watertight triangle test (src/trace.rs:307-450 over oxideav-mesh3d's Bvh,
// restated from Wald 2007 / Woop, Benthin & Wald 2013), hit surfaces and
// material evaluation (src/trace.rs:459-923, 1118-1204), punctual lights
// (src/prepare.rs:921-963), emissive-triangle table and environment map
// (src/pathtrace.rs:1431-1741).
#pragma once

#include <array>
#include <memory>

#include "../include/pt_b200.h"
#include "oracle_core.hpp"

namespace oracle {

struct MipLevel {
  uint32_t w = 0, h = 0;
  std::vector<V4> texels;
};

struct Texture {
  uint32_t img_w = 0, img_h = 0;
  std::vector<MipLevel> srgb, linear;
  uint32_t mag = PT_FILTER_LINEAR, min = PT_MIN_LINEAR_MIP_LINEAR, wrap_s = 0, wrap_t = 0;
  const std::vector<MipLevel> &mips(bool srgb_space) const { return srgb_space ? srgb : linear; }
  V4 sample_lod(float u, float v, float lod, bool srgb_space) const;
};

struct Item {
  uint32_t tri_count = 0;
  std::vector<V3> positions, normals;
  bool has_vertex_normals = false;
  std::vector<V4> tangents;
  std::vector<std::array<float, 2>> uvs[PT_MAX_UV_SETS];
  std::vector<V4> colors;
  uint32_t material = 0;
  const std::vector<std::array<float, 2>> *uv_set(uint32_t s) const {
    if (s >= PT_MAX_UV_SETS || uvs[s].empty()) return nullptr;
    return &uvs[s];
  }
};

struct TriRef {
  uint32_t item, tri;
};

struct Hit {
  float t = 0.0f;
  uint32_t global = 0, item = 0, tri = 0;
  float bary[3] = {0, 0, 0};
  bool front = false;
};

struct Surface {
  V3 position, geometric_normal, shading_normal;
  float area;
  uint32_t material;
};

struct BvhNode {
  float bmin[3], bmax[3];
  uint32_t left_or_first;  // interior: left child index; leaf: first slot
  uint32_t count;          // 0 = interior (right child = left + 1... stored in right)
  uint32_t right;
};

struct PreparedRay {
  V3 o, d;
  int kx, ky, kz;
  float sx, sy, sz;
};

PreparedRay prepare_ray(V3 o, V3 d);
// Woop et al. 2013 watertight test. Barycentrics are the weights of the
// triangle's corners 0, 1, 2 (the reference's [w, u, v]).
bool intersect_watertight(const PreparedRay &r, V3 v0, V3 v1, V3 v2, float &t, float bary[3], bool &front);

// TexLod, src/trace.rs:171-195: level 0, a ray cone, or ray differentials
// (barycentric change per pixel along x and y).
enum class TexLodKind { Base, Cone, Grad };
struct TexLod {
  TexLodKind kind = TexLodKind::Base;
  float width = 0.0f;
  V3 dir = {0, 0, 0};
  float gx[3] = {0, 0, 0}, gy[3] = {0, 0, 0};
};

// f32::hypot as glibc's hypotf computes it: the f64 root of the f64 sum of
// squares (exact squares), rounded once.
inline float hypot_f32(float a, float b) {
  double x = (double)a, y = (double)b;
  return (float)std::sqrt(x * x + y * y);
}

struct LightSample {
  V3 l;
  float distance;
  V3 radiance;
};
bool light_sample(const pt_light &light, V3 p, LightSample &out);

struct EmissiveLights {
  std::vector<uint32_t> tris;
  std::vector<float> pmf, cdf;
  std::vector<uint32_t> lookup;
  bool empty() const { return tris.empty(); }
  size_t pick(float u) const;
};

struct EnvironmentMap {
  uint32_t w = 1, h = 1;
  std::vector<float> pixels;  // w*h*4
  float intensity = 0.0f;
  std::vector<float> marginal, conditional, mass;
  bool uniform = true;
  explicit EnvironmentMap(const pt_environment &env);
  void texel_of(V3 d, size_t &x, size_t &y, float &st) const;
  V3 radiance(V3 d) const;
  float pdf(V3 d) const;
  bool sample(float u0, float u1, V3 &d, V3 &le, float &pdf) const;
};

class Scene {
 public:
  explicit Scene(const pt_scene_desc &desc);
  std::vector<Item> items;
  std::vector<pt_material> materials;
  std::vector<std::unique_ptr<Texture>> textures;  // null = unresolved
  std::vector<pt_light> lights;
  std::vector<V3> soup;  // 3 per global triangle
  std::vector<TriRef> tri_refs;
  std::vector<BvhNode> nodes;
  std::vector<uint32_t> slots;  // leaf slot -> global triangle
  EmissiveLights emissive;

  size_t triangle_count() const { return tri_refs.size(); }
  void triangle_positions(uint32_t g, V3 &a, V3 &b, V3 &c) const {
    a = soup[3 * g];
    b = soup[3 * g + 1];
    c = soup[3 * g + 2];
  }
  Hit make_hit(uint32_t g, float t, const float bary[3], bool front) const;

  template <class F>
  bool closest_hit_filtered(V3 o, V3 d, float t_min, float t_max, F &&filter, Hit &out) const;
  template <class F>
  bool occluded_filtered(V3 o, V3 d, float t_min, float t_max, F &&filter) const;

  const Item &item_of(const Hit &h) const { return items[h.item]; }
  const pt_material &material_of(const Hit &h) const { return materials[items[h.item].material]; }
  Surface surface(const Hit &h) const;
  float alpha(const Hit &h) const;
  MaterialSample material_oriented(const Hit &h, const Surface &s, const TexLod &lod, bool flip) const;
  const Texture *texture(const pt_texture_binding &b) const {
    if (b.texture < 0 || (size_t)b.texture >= textures.size()) return nullptr;
    return textures[b.texture].get();
  }
  // Samples `b` at the hit (TraceScene::sample / sample_at); false = None.
  bool sample_binding(const Item &item, const pt_texture_binding &b, size_t base, const float bary[3],
                      const TexLod &lod, bool srgb, V4 &out) const;
  mutable uint64_t counter_nodes = 0, counter_tris = 0;

 private:
  void build_bvh();
  bool box_hit(const BvhNode &n, const V3 &o, const V3 &inv, const V3 &d, float t0, float t1) const;
};

inline std::array<float, 2> transform_uv(const pt_texture_binding &b, std::array<float, 2> uv) {
  if (!b.has_transform) return uv;
  const float *m = b.transform;
  return {m[0] * uv[0] + m[1] * uv[1] + m[2], m[3] * uv[0] + m[4] * uv[1] + m[5]};
}

// ---- traversal (templated on the filter) --------------------------------
template <class F>
bool Scene::closest_hit_filtered(V3 o, V3 d, float t_min, float t_max, F &&filter, Hit &out) const {
  if (nodes.empty()) return false;
  PreparedRay r = prepare_ray(o, d);
  V3 inv = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
  bool have = false;
  Hit best;
  uint32_t stack[128];
  int sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    const BvhNode &n = nodes[stack[--sp]];
    counter_nodes++;
    if (!box_hit(n, o, inv, d, t_min, have ? best.t : t_max)) continue;
    if (n.count > 0) {
      for (uint32_t i = 0; i < n.count; ++i) {
        uint32_t g = slots[n.left_or_first + i];
        counter_tris++;
        float t, bary[3];
        bool front;
        if (!intersect_watertight(r, soup[3 * g], soup[3 * g + 1], soup[3 * g + 2], t, bary, front)) continue;
        if (!(t >= t_min)) continue;
        bool better = have ? (t < best.t || (t == best.t && g < best.global)) : (t <= t_max);
        if (!better) continue;
        Hit h = make_hit(g, t, bary, front);
        if (filter(h)) {
          best = h;
          have = true;
        }
      }
    } else {
      stack[sp++] = n.left_or_first;
      stack[sp++] = n.right;
    }
  }
  if (have) out = best;
  return have;
}

template <class F>
bool Scene::occluded_filtered(V3 o, V3 d, float t_min, float t_max, F &&filter) const {
  if (nodes.empty()) return false;
  PreparedRay r = prepare_ray(o, d);
  V3 inv = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
  uint32_t stack[128];
  int sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    const BvhNode &n = nodes[stack[--sp]];
    counter_nodes++;
    if (!box_hit(n, o, inv, d, t_min, t_max)) continue;
    if (n.count > 0) {
      for (uint32_t i = 0; i < n.count; ++i) {
        uint32_t g = slots[n.left_or_first + i];
        counter_tris++;
        float t, bary[3];
        bool front;
        if (!intersect_watertight(r, soup[3 * g], soup[3 * g + 1], soup[3 * g + 2], t, bary, front)) continue;
        if (!(t >= t_min && t <= t_max)) continue;
        if (filter(make_hit(g, t, bary, front))) return true;
      }
    } else {
      stack[sp++] = n.left_or_first;
      stack[sp++] = n.right;
    }
  }
  return false;
}

}  // namespace oracle
