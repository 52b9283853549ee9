// ORACLE — test infrastructure only (see oracle_core.hpp).
#include "oracle_scene.hpp"

#include <algorithm>
#include <numeric>

namespace oracle {

// ---------------------------------------------------------------- textures

// srgb_to_linear / srgb_u8_lut, src/hdr.rs:80-109.
static float srgb_to_linear(float c) {
  if (c <= 0.04045f) return c / 12.92f;
  return std::pow((c + 0.055f) / 1.055f, 2.4f);
}
static const float *srgb_lut() {
  static float t[256];
  static bool init = [] {
    for (int i = 0; i < 256; ++i) t[i] = srgb_to_linear((float)i / 255.0f);
    return true;
  }();
  (void)init;
  return t;
}

// build_mips, src/texture.rs:324-383.
static std::vector<MipLevel> build_mips(const pt_texture &img, bool srgb_space) {
  const float *lut = srgb_lut();
  size_t n = (size_t)img.width * img.height;
  MipLevel l0;
  l0.w = img.width;
  l0.h = img.height;
  l0.texels.resize(n);
  if (img.format == PT_PIXELS_RGBA8) {
    const uint8_t *p = (const uint8_t *)img.pixels;
    for (size_t i = 0; i < n; ++i) {
      auto c = [&](uint8_t v) { return srgb_space ? lut[v] : (float)v / 255.0f; };
      l0.texels[i] = V4{{c(p[4 * i]), c(p[4 * i + 1]), c(p[4 * i + 2]), (float)p[4 * i + 3] / 255.0f}};
    }
  } else {
    const float *p = (const float *)img.pixels;
    for (size_t i = 0; i < n; ++i) l0.texels[i] = V4{{p[4 * i], p[4 * i + 1], p[4 * i + 2], p[4 * i + 3]}};
  }
  std::vector<MipLevel> levels;
  levels.push_back(std::move(l0));
  for (;;) {
    const MipLevel &prev = levels.back();
    if (prev.w == 1 && prev.h == 1) break;
    MipLevel nx;
    nx.w = std::max(prev.w / 2, 1u);
    nx.h = std::max(prev.h / 2, 1u);
    nx.texels.reserve((size_t)nx.w * nx.h);
    for (uint32_t y = 0; y < nx.h; ++y) {
      for (uint32_t x = 0; x < nx.w; ++x) {
        size_t x0 = std::min(2 * x, prev.w - 1), x1 = std::min(2 * x + 1, prev.w - 1);
        size_t y0 = std::min(2 * y, prev.h - 1), y1 = std::min(2 * y + 1, prev.h - 1);
        size_t pw = prev.w;
        float acc[4] = {0, 0, 0, 0};
        size_t idx[4] = {y0 * pw + x0, y0 * pw + x1, y1 * pw + x0, y1 * pw + x1};
        for (size_t id : idx)
          for (int c = 0; c < 4; ++c) acc[c] += prev.texels[id][c];
        nx.texels.push_back(V4{{acc[0] * 0.25f, acc[1] * 0.25f, acc[2] * 0.25f, acc[3] * 0.25f}});
      }
    }
    levels.push_back(std::move(nx));
  }
  return levels;
}

// wrap_index, src/texture.rs:277-286.
static size_t wrap_index(int64_t i, int64_t n, uint32_t mode) {
  auto rem_euclid = [](int64_t a, int64_t m) {
    int64_t r = a % m;
    return r < 0 ? r + m : r;
  };
  int64_t r;
  if (mode == PT_WRAP_REPEAT) {
    r = rem_euclid(i, n);
  } else if (mode == PT_WRAP_CLAMP) {
    r = std::min(std::max(i, (int64_t)0), n - 1);
  } else {
    int64_t m = rem_euclid(i, 2 * n);
    r = m >= n ? 2 * n - 1 - m : m;
  }
  return (size_t)r;
}
static V4 fetch(const MipLevel &l, int64_t x, int64_t y, uint32_t ws, uint32_t wt) {
  size_t xi = wrap_index(x, l.w, ws), yi = wrap_index(y, l.h, wt);
  return l.texels[yi * l.w + xi];
}
static V4 lerp4(V4 a, V4 b, float t) {
  return V4{{a[0] + (b[0] - a[0]) * t, a[1] + (b[1] - a[1]) * t, a[2] + (b[2] - a[2]) * t, a[3] + (b[3] - a[3]) * t}};
}
// filter_level, src/texture.rs:486-515.
static V4 filter_level(const MipLevel &lvl, float u, float v, bool linear, uint32_t ws, uint32_t wt) {
  u = std::isfinite(u) ? u : 0.0f;
  v = std::isfinite(v) ? v : 0.0f;
  u = clampr(u, -1.0e6f, 1.0e6f);
  v = clampr(v, -1.0e6f, 1.0e6f);
  float x = u * (float)lvl.w, y = v * (float)lvl.h;
  if (!linear) return fetch(lvl, f2i64(std::floor(x)), f2i64(std::floor(y)), ws, wt);
  float xf = x - 0.5f, yf = y - 0.5f;
  float x0 = std::floor(xf), y0 = std::floor(yf);
  float fx = xf - x0, fy = yf - y0;
  int64_t ix = f2i64(x0), iy = f2i64(y0);
  V4 a = fetch(lvl, ix, iy, ws, wt), b = fetch(lvl, ix + 1, iy, ws, wt);
  V4 c = fetch(lvl, ix, iy + 1, ws, wt), d = fetch(lvl, ix + 1, iy + 1, ws, wt);
  return lerp4(lerp4(a, b, fx), lerp4(c, d, fx), fy);
}
// PreparedTexture::sample_lod, src/texture.rs:420-451.
V4 Texture::sample_lod(float u, float v, float lod, bool srgb_space) const {
  const std::vector<MipLevel> &m = mips(srgb_space);
  if (std::isnan(lod) || lod <= 0.0f) return filter_level(m[0], u, v, mag == PT_FILTER_LINEAR, wrap_s, wrap_t);
  bool lin = (min == PT_MIN_LINEAR || min == PT_MIN_LINEAR_MIP_NEAREST || min == PT_MIN_LINEAR_MIP_LINEAR);
  float max_level = (float)(m.size() - 1);
  switch (min) {
    case PT_MIN_NEAREST:
    case PT_MIN_LINEAR:
      return filter_level(m[0], u, v, lin, wrap_s, wrap_t);
    case PT_MIN_NEAREST_MIP_NEAREST:
    case PT_MIN_LINEAR_MIP_NEAREST: {
      size_t l = (size_t)f2usize(clampr(std::round(lod), 0.0f, max_level));
      return filter_level(m[l], u, v, lin, wrap_s, wrap_t);
    }
    default: {
      float l = clampr(lod, 0.0f, max_level);
      size_t l0 = (size_t)f2usize(std::floor(l));
      size_t l1 = std::min(l0 + 1, m.size() - 1);
      float f = l - (float)l0;
      V4 a = filter_level(m[l0], u, v, lin, wrap_s, wrap_t);
      if (f <= 0.0f || l0 == l1) return a;
      V4 b = filter_level(m[l1], u, v, lin, wrap_s, wrap_t);
      return lerp4(a, b, f);
    }
  }
}

// ---------------------------------------------------------------- ray / triangle

PreparedRay prepare_ray(V3 o, V3 d) {
  PreparedRay r;
  r.o = o;
  r.d = d;
  int kz = 0;
  if (std::fabs(d.y) > std::fabs(d[kz])) kz = 1;
  if (std::fabs(d.z) > std::fabs(d[kz])) kz = 2;
  int kx = (kz + 1) % 3, ky = (kx + 1) % 3;
  if (d[kz] < 0.0f) std::swap(kx, ky);
  r.kx = kx;
  r.ky = ky;
  r.kz = kz;
  r.sx = d[kx] / d[kz];
  r.sy = d[ky] / d[kz];
  r.sz = 1.0f / d[kz];
  return r;
}

bool intersect_watertight(const PreparedRay &r, V3 v0, V3 v1, V3 v2, float &t, float bary[3], bool &front) {
  V3 a = sub(v0, r.o), b = sub(v1, r.o), c = sub(v2, r.o);
  float ax = a[r.kx] - r.sx * a[r.kz], ay = a[r.ky] - r.sy * a[r.kz];
  float bx = b[r.kx] - r.sx * b[r.kz], by = b[r.ky] - r.sy * b[r.kz];
  float cx = c[r.kx] - r.sx * c[r.kz], cy = c[r.ky] - r.sy * c[r.kz];
  float u = cx * by - cy * bx;
  float v = ax * cy - ay * cx;
  float w = bx * ay - by * ax;
  if (u == 0.0f || v == 0.0f || w == 0.0f) {
    double cxby = (double)cx * (double)by, cybx = (double)cy * (double)bx;
    u = (float)(cxby - cybx);
    double axcy = (double)ax * (double)cy, aycx = (double)ay * (double)cx;
    v = (float)(axcy - aycx);
    double bxay = (double)bx * (double)ay, byax = (double)by * (double)ax;
    w = (float)(bxay - byax);
  }
  if ((u < 0.0f || v < 0.0f || w < 0.0f) && (u > 0.0f || v > 0.0f || w > 0.0f)) return false;
  float det = u + v + w;
  if (det == 0.0f) return false;
  float az = r.sz * a[r.kz], bz = r.sz * b[r.kz], cz = r.sz * c[r.kz];
  float tt = u * az + v * bz + w * cz;
  float rcp = 1.0f / det;
  t = tt * rcp;
  bary[0] = u * rcp;
  bary[1] = v * rcp;
  bary[2] = w * rcp;
  front = det > 0.0f;
  return true;
}

bool Scene::box_hit(const BvhNode &n, const V3 &o, const V3 &inv, const V3 &d, float t0, float t1) const {
  const float grow = 1.0f + 2.0f * (3.0f * 5.9604645e-8f) / (1.0f - 3.0f * 5.9604645e-8f);
  float tn = t0, tf = t1;
  for (int k = 0; k < 3; ++k) {
    if (d[k] == 0.0f) {
      if (o[k] < n.bmin[k] || o[k] > n.bmax[k]) return false;
      continue;
    }
    float a = (n.bmin[k] - o[k]) * inv[k];
    float b = (n.bmax[k] - o[k]) * inv[k];
    if (a > b) std::swap(a, b);
    b *= grow;
    if (a > tn) tn = a;
    if (b < tf) tf = b;
    if (tn > tf) return false;
  }
  return true;
}

// Binned-SAH BVH2 (Wald 2007) over the soup; only conservativeness matters
// for results (closest accepted hit with the lowest-id tie-break is
// independent of the tree).
void Scene::build_bvh() {
  size_t nt = tri_refs.size();
  nodes.clear();
  slots.resize(nt);
  std::iota(slots.begin(), slots.end(), 0u);
  if (nt == 0) return;
  std::vector<V3> cmin(nt), cmax(nt), cen(nt);
  for (size_t g = 0; g < nt; ++g) {
    V3 a = soup[3 * g], b = soup[3 * g + 1], c = soup[3 * g + 2];
    cmin[g] = {std::min({a.x, b.x, c.x}), std::min({a.y, b.y, c.y}), std::min({a.z, b.z, c.z})};
    cmax[g] = {std::max({a.x, b.x, c.x}), std::max({a.y, b.y, c.y}), std::max({a.z, b.z, c.z})};
    cen[g] = {(cmin[g].x + cmax[g].x) * 0.5f, (cmin[g].y + cmax[g].y) * 0.5f, (cmin[g].z + cmax[g].z) * 0.5f};
  }
  struct Task {
    uint32_t node, first, count, depth;
  };
  nodes.push_back(BvhNode{});
  std::vector<Task> work{{0, 0, (uint32_t)nt, 0}};
  auto area = [](V3 lo, V3 hi) {
    float dx = hi.x - lo.x, dy = hi.y - lo.y, dz = hi.z - lo.z;
    return dx * dy + dy * dz + dz * dx;
  };
  while (!work.empty()) {
    Task tk = work.back();
    work.pop_back();
    V3 lo = {INF, INF, INF}, hi = {-INF, -INF, -INF}, clo = lo, chi = hi;
    for (uint32_t i = tk.first; i < tk.first + tk.count; ++i) {
      uint32_t g = slots[i];
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], cmin[g][k]);
        hi[k] = std::max(hi[k], cmax[g][k]);
        clo[k] = std::min(clo[k], cen[g][k]);
        chi[k] = std::max(chi[k], cen[g][k]);
      }
    }
    BvhNode &node = nodes[tk.node];
    float ext = std::max({hi.x - lo.x, hi.y - lo.y, hi.z - lo.z, std::fabs(lo.x), std::fabs(lo.y),
                          std::fabs(lo.z), std::fabs(hi.x), std::fabs(hi.y), std::fabs(hi.z)});
    float pad = ext * 1.0e-5f + 1.0e-30f;
    for (int k = 0; k < 3; ++k) {
      node.bmin[k] = lo[k] - pad;
      node.bmax[k] = hi[k] + pad;
    }
    if (tk.count <= 4 || tk.depth >= 60) {
      node.left_or_first = tk.first;
      node.count = tk.count;
      node.right = 0;
      continue;
    }
    const int B = 16;
    int best_axis = -1;
    int best_bin = 0;
    float best_cost = INF;
    for (int k = 0; k < 3; ++k) {
      float span = chi[k] - clo[k];
      if (!(span > 0.0f)) continue;
      uint32_t cnt[B] = {0};
      V3 blo[B], bhi[B];
      for (int i = 0; i < B; ++i) {
        blo[i] = {INF, INF, INF};
        bhi[i] = {-INF, -INF, -INF};
      }
      for (uint32_t i = tk.first; i < tk.first + tk.count; ++i) {
        uint32_t g = slots[i];
        int bi = std::min(B - 1, (int)((cen[g][k] - clo[k]) / span * B));
        cnt[bi]++;
        for (int a = 0; a < 3; ++a) {
          blo[bi][a] = std::min(blo[bi][a], cmin[g][a]);
          bhi[bi][a] = std::max(bhi[bi][a], cmax[g][a]);
        }
      }
      for (int s = 1; s < B; ++s) {
        V3 l0 = {INF, INF, INF}, l1 = {-INF, -INF, -INF}, r0 = l0, r1 = l1;
        uint32_t nl = 0, nr = 0;
        for (int i = 0; i < s; ++i) {
          nl += cnt[i];
          for (int a = 0; a < 3; ++a) {
            l0[a] = std::min(l0[a], blo[i][a]);
            l1[a] = std::max(l1[a], bhi[i][a]);
          }
        }
        for (int i = s; i < B; ++i) {
          nr += cnt[i];
          for (int a = 0; a < 3; ++a) {
            r0[a] = std::min(r0[a], blo[i][a]);
            r1[a] = std::max(r1[a], bhi[i][a]);
          }
        }
        if (nl == 0 || nr == 0) continue;
        float cost = area(l0, l1) * nl + area(r0, r1) * nr;
        if (cost < best_cost) {
          best_cost = cost;
          best_axis = k;
          best_bin = s;
        }
      }
    }
    uint32_t mid;
    if (best_axis < 0) {
      mid = tk.first + tk.count / 2;
    } else {
      float span = chi[best_axis] - clo[best_axis];
      auto it = std::partition(slots.begin() + tk.first, slots.begin() + tk.first + tk.count, [&](uint32_t g) {
        int bi = std::min(B - 1, (int)((cen[g][best_axis] - clo[best_axis]) / span * B));
        return bi < best_bin;
      });
      mid = (uint32_t)(it - slots.begin());
      if (mid == tk.first || mid == tk.first + tk.count) mid = tk.first + tk.count / 2;
    }
    uint32_t left = (uint32_t)nodes.size();
    nodes.push_back(BvhNode{});
    nodes.push_back(BvhNode{});
    BvhNode &nd = nodes[tk.node];
    nd.left_or_first = left;
    nd.right = left + 1;
    nd.count = 0;
    work.push_back({left, tk.first, mid - tk.first, tk.depth + 1});
    work.push_back({left + 1, mid, tk.first + tk.count - mid, tk.depth + 1});
  }
}

// ---------------------------------------------------------------- scene

Scene::Scene(const pt_scene_desc &desc) {
  for (uint32_t i = 0; i < desc.material_count; ++i) materials.push_back(desc.materials[i]);
  for (uint32_t i = 0; i < desc.texture_count; ++i) {
    const pt_texture &t = desc.textures[i];
    if (!t.pixels || t.width == 0 || t.height == 0) {
      textures.emplace_back(nullptr);
      continue;
    }
    auto tex = std::make_unique<Texture>();
    tex->img_w = t.width;
    tex->img_h = t.height;
    tex->srgb = build_mips(t, true);
    tex->linear = build_mips(t, false);
    tex->mag = t.mag_filter;
    tex->min = t.min_filter;
    tex->wrap_s = t.wrap_s;
    tex->wrap_t = t.wrap_t;
    textures.push_back(std::move(tex));
  }
  for (uint32_t i = 0; i < desc.light_count; ++i) lights.push_back(desc.lights[i]);
  for (uint32_t ii = 0; ii < desc.item_count; ++ii) {
    const pt_draw_item &d = desc.items[ii];
    Item it;
    it.tri_count = d.triangle_count;
    size_t nc = 3 * (size_t)d.triangle_count;
    it.positions.resize(nc);
    for (size_t c = 0; c < nc; ++c) it.positions[c] = {d.positions[3 * c], d.positions[3 * c + 1], d.positions[3 * c + 2]};
    if (d.normals) {
      it.normals.resize(nc);
      for (size_t c = 0; c < nc; ++c) it.normals[c] = {d.normals[3 * c], d.normals[3 * c + 1], d.normals[3 * c + 2]};
    }
    it.has_vertex_normals = d.has_vertex_normals != 0;
    if (d.tangents) {
      it.tangents.resize(nc);
      for (size_t c = 0; c < nc; ++c)
        it.tangents[c] = V4{{d.tangents[4 * c], d.tangents[4 * c + 1], d.tangents[4 * c + 2], d.tangents[4 * c + 3]}};
    }
    for (int s = 0; s < PT_MAX_UV_SETS; ++s) {
      if (!d.uvs[s]) continue;
      it.uvs[s].resize(nc);
      for (size_t c = 0; c < nc; ++c) it.uvs[s][c] = {d.uvs[s][2 * c], d.uvs[s][2 * c + 1]};
    }
    if (d.colors) {
      it.colors.resize(nc);
      for (size_t c = 0; c < nc; ++c)
        it.colors[c] = V4{{d.colors[4 * c], d.colors[4 * c + 1], d.colors[4 * c + 2], d.colors[4 * c + 3]}};
    }
    it.material = d.material < materials.size() ? d.material : (uint32_t)materials.size() - 1;
    for (uint32_t t = 0; t < d.triangle_count; ++t) {
      soup.push_back(it.positions[3 * t]);
      soup.push_back(it.positions[3 * t + 1]);
      soup.push_back(it.positions[3 * t + 2]);
      tri_refs.push_back({ii, t});
    }
    items.push_back(std::move(it));
  }
  build_bvh();

  // EmissiveLights::build, src/pathtrace.rs:1479-1543.
  std::vector<V3> mean_e(materials.size());
  for (size_t m = 0; m < materials.size(); ++m) {
    const pt_material &mt = materials[m];
    if (mt.unlit) {
      mean_e[m] = {0, 0, 0};
      continue;
    }
    V3 e = {mt.emissive[0], mt.emissive[1], mt.emissive[2]};
    if (const Texture *t = texture(mt.emissive_texture)) {
      const V4 &c = t->srgb.back().texels[0];
      e = mul(e, {c[0], c[1], c[2]});
    }
    mean_e[m] = e;
  }
  emissive.lookup.assign(tri_refs.size(), UINT32_MAX);
  std::vector<float> power;
  for (size_t g = 0; g < tri_refs.size(); ++g) {
    const Item &item = items[tri_refs[g].item];
    V3 e = mean_e[item.material];
    float lum = luminance(e);
    if (std::isnan(lum) || lum <= 0.0f) continue;
    V3 a, b, c;
    triangle_positions((uint32_t)g, a, b, c);
    V3 cr = cross(sub(b, a), sub(c, a));
    float ar = 0.5f * std::sqrt(dot(cr, cr));
    if (std::isnan(ar) || ar <= 0.0f || !std::isfinite(ar)) continue;
    float sides = materials[item.material].double_sided ? 2.0f : 1.0f;
    emissive.lookup[g] = (uint32_t)emissive.tris.size();
    emissive.tris.push_back((uint32_t)g);
    power.push_back(ar * lum * sides);
  }
  double total = 0.0;
  for (float p : power) total += (double)p;
  double acc = 0.0;
  for (float pw : power) {
    emissive.pmf.push_back((float)((double)pw / total));
    acc += (double)pw / total;
    emissive.cdf.push_back((float)acc);
  }
  if (!emissive.cdf.empty()) emissive.cdf.back() = 1.0f;
}

size_t EmissiveLights::pick(float u) const {
  size_t i = (size_t)(std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
  return std::min(i, tris.size() - 1);
}

Hit Scene::make_hit(uint32_t g, float t, const float bary[3], bool front) const {
  Hit h;
  h.t = t;
  h.global = g;
  h.item = tri_refs[g].item;
  h.tri = tri_refs[g].tri;
  h.bary[0] = bary[0];
  h.bary[1] = bary[1];
  h.bary[2] = bary[2];
  h.front = front;
  return h;
}

static V3 interp3(const std::vector<V3> &v, size_t base, const float b[3]) {
  V3 x = v[base], y = v[base + 1], z = v[base + 2];
  return {x.x * b[0] + y.x * b[1] + z.x * b[2], x.y * b[0] + y.y * b[1] + z.y * b[2],
          x.z * b[0] + y.z * b[1] + z.z * b[2]};
}
static std::array<float, 2> interp2(const std::vector<std::array<float, 2>> &v, size_t base, const float b[3]) {
  auto x = v[base], y = v[base + 1], z = v[base + 2];
  return {x[0] * b[0] + y[0] * b[1] + z[0] * b[2], x[1] * b[0] + y[1] * b[1] + z[1] * b[2]};
}
static V4 interp4(const std::vector<V4> &v, size_t base, const float b[3]) {
  V4 x = v[base], y = v[base + 1], z = v[base + 2], o;
  for (int k = 0; k < 4; ++k) o[k] = x[k] * b[0] + y[k] * b[1] + z[k] * b[2];
  return o;
}

// TraceScene::surface, src/trace.rs:459-488.
Surface Scene::surface(const Hit &h) const {
  const Item &item = items[h.item];
  size_t base = 3 * (size_t)h.tri;
  const std::vector<V3> &p = item.positions;
  Surface s;
  s.position = interp3(p, base, h.bary);
  V3 cr = cross(sub(p[base + 1], p[base]), sub(p[base + 2], p[base]));
  float len = std::sqrt(dot(cr, cr));
  V3 ng = len > 0.0f ? V3{cr.x / len, cr.y / len, cr.z / len} : V3{0.0f, 0.0f, 1.0f};
  V3 sn = ng;
  if (item.has_vertex_normals && item.normals.size() == p.size()) {
    V3 n = normalise(interp3(item.normals, base, h.bary));
    sn = dot(n, n) > 0.5f ? n : ng;
  }
  s.geometric_normal = ng;
  s.shading_normal = sn;
  s.area = 0.5f * len;
  s.material = item.material;
  return s;
}

// TraceScene::lod, src/trace.rs:518-554.
static bool lod_of(const Scene &sc, const Item &item, const pt_texture_binding &bd, size_t base, const TexLod &lod,
                   float &out) {
  if (lod.kind != TexLodKind::Cone) return false;
  const Texture *tex = sc.texture(bd);
  if (!tex) return false;
  const auto *uvs = item.uv_set(bd.uv_set);
  if (!uvs) return false;
  const std::vector<V3> &p = item.positions;
  std::array<float, 2> uv[3] = {transform_uv(bd, (*uvs)[base]), transform_uv(bd, (*uvs)[base + 1]),
                                transform_uv(bd, (*uvs)[base + 2])};
  float ta = (float)tex->img_w * (float)tex->img_h *
             std::fabs((uv[1][0] - uv[0][0]) * (uv[2][1] - uv[0][1]) - (uv[2][0] - uv[0][0]) * (uv[1][1] - uv[0][1]));
  V3 cr = cross(sub(p[base + 1], p[base]), sub(p[base + 2], p[base]));
  float pa = std::sqrt(dot(cr, cr));
  if (!(ta > 0.0f && pa > 0.0f && lod.width > 0.0f)) {
    out = 0.0f;
    return true;
  }
  V3 n = {cr.x / pa, cr.y / pa, cr.z / pa};
  float cos = fmaxr(std::fabs(dot(n, lod.dir)), 1.0e-3f);
  float l = 0.5f * std::log2(ta / pa) + std::log2(lod.width / cos);
  out = std::isfinite(l) ? l : 0.0f;
  return true;
}

bool Scene::sample_binding(const Item &item, const pt_texture_binding &bd, size_t base, const float bary[3],
                           const TexLod &lod, bool srgb, V4 &out) const {
  if (bd.texture < 0) return false;
  if (lod.kind == TexLodKind::Grad) {
    // TraceScene::sample_grad (src/trace.rs:596-620) + Texture::sample_grad
    // (src/texture.rs:456-474): move the barycentrics by one pixel,
    // difference the transformed UVs, LOD = log2 of the longer texel step.
    const Texture *tex = texture(bd);
    if (!tex) return false;
    const auto *uvs = item.uv_set(bd.uv_set);
    if (!uvs || uvs->size() != item.positions.size()) return false;
    const auto &u = *uvs;
    std::array<float, 2> uv = interp2(u, base, bary);
    std::array<float, 2> tuv = transform_uv(bd, uv);
    auto duv = [&](const float d[3]) {
      std::array<float, 2> moved = {uv[0] + u[base][0] * d[0] + u[base + 1][0] * d[1] + u[base + 2][0] * d[2],
                                    uv[1] + u[base][1] * d[0] + u[base + 1][1] * d[1] + u[base + 2][1] * d[2]};
      std::array<float, 2> m = transform_uv(bd, moved);
      return std::array<float, 2>{m[0] - tuv[0], m[1] - tuv[1]};
    };
    std::array<float, 2> gx = duv(lod.gx), gy = duv(lod.gy);
    float w = (float)tex->img_w, h = (float)tex->img_h;
    float lx = hypot_f32(gx[0] * w, gx[1] * h), ly = hypot_f32(gy[0] * w, gy[1] * h);
    float rho = fmaxr(lx, ly);
    float l = (std::isfinite(rho) && rho > 0.0f) ? std::log2(rho) : 0.0f;
    out = tex->sample_lod(tuv[0], tuv[1], l, srgb);
    return true;
  }
  float l = 0.0f;
  if (!lod_of(*this, item, bd, base, lod, l)) l = 0.0f;
  const Texture *tex = texture(bd);
  if (!tex) return false;
  const auto *uvs = item.uv_set(bd.uv_set);
  if (!uvs || uvs->size() != item.positions.size()) return false;
  auto uv = transform_uv(bd, interp2(*uvs, base, bary));
  out = tex->sample_lod(uv[0], uv[1], l, srgb);
  return true;
}

// TraceScene::alpha, src/trace.rs:492-506.
float Scene::alpha(const Hit &h) const {
  const Item &item = items[h.item];
  const pt_material &mat = materials[item.material];
  size_t base = 3 * (size_t)h.tri;
  float a = mat.base_color[3];
  V4 t;
  if (sample_binding(item, mat.base_color_texture, base, h.bary, TexLod{}, true, t)) a *= t[3];
  if (item.colors.size() == item.positions.size()) a *= interp4(item.colors, base, h.bary)[3];
  return a;
}

// TraceScene::tangent_frame / perturb, src/trace.rs:640-687.
static bool tangent_frame(const Item &item, size_t base, const float b[3], V3 n, V3 &tt, V3 &bt) {
  if (item.tangents.size() != item.positions.size()) return false;
  V4 tg = interp4(item.tangents, base, b);
  float w = item.tangents[base][3] < 0.0f ? -1.0f : 1.0f;
  V3 t3 = {tg[0], tg[1], tg[2]};
  float d = dot(n, t3);
  tt = normalise({t3.x - n.x * d, t3.y - n.y * d, t3.z - n.z * d});
  if (dot(tt, tt) < 0.5f) return false;
  V3 c = cross(n, tt);
  bt = {c.x * w, c.y * w, c.z * w};
  return true;
}
static V3 perturb(const Item &item, size_t base, const float b[3], V3 n, V4 t, float sc) {
  V3 tt, bt;
  if (!tangent_frame(item, base, b, n, tt, bt)) return n;
  float ts[3] = {(t[0] * 2.0f - 1.0f) * sc, (t[1] * 2.0f - 1.0f) * sc, t[2] * 2.0f - 1.0f};
  V3 nn = normalise({tt.x * ts[0] + bt.x * ts[1] + n.x * ts[2], tt.y * ts[0] + bt.y * ts[1] + n.y * ts[2],
                     tt.z * ts[0] + bt.z * ts[1] + n.z * ts[2]});
  return dot(nn, nn) > 0.5f ? nn : n;
}

static float fin(float v, float d) { return std::isfinite(v) ? v : d; }

// TraceScene::material_oriented, src/trace.rs:700-923.
MaterialSample Scene::material_oriented(const Hit &h, const Surface &surf, const TexLod &lod, bool flip) const {
  V3 sn = flip ? neg(surf.shading_normal) : surf.shading_normal;
  const Item &item = items[h.item];
  const pt_material &mat = materials[item.material];
  size_t base = 3 * (size_t)h.tri;
  const float *b = h.bary;
  auto samp = [&](const pt_texture_binding &bd, bool srgb, V4 &t) {
    return sample_binding(item, bd, base, b, lod, srgb, t);
  };
  MaterialSample m;
  V4 t;
  float col[4] = {mat.base_color[0], mat.base_color[1], mat.base_color[2], mat.base_color[3]};
  if (samp(mat.base_color_texture, true, t))
    for (int k = 0; k < 4; ++k) col[k] *= t[k];
  if (item.colors.size() == item.positions.size()) {
    V4 v = interp4(item.colors, base, b);
    for (int k = 0; k < 4; ++k) col[k] *= v[k];
  }
  float metallic = mat.metallic, roughness = mat.roughness;
  if (samp(mat.metallic_roughness_texture, false, t)) {
    roughness *= t[1];
    metallic *= t[2];
  }
  V3 normal = sn;
  if (samp(mat.normal_texture, false, t)) normal = perturb(item, base, b, normal, t, mat.normal_scale);
  float occlusion = 1.0f;
  if (samp(mat.occlusion_texture, false, t)) occlusion = 1.0f + mat.occlusion_strength * (t[0] - 1.0f);
  V3 emissive = {mat.emissive[0], mat.emissive[1], mat.emissive[2]};
  if (samp(mat.emissive_texture, true, t))
    for (int k = 0; k < 3; ++k) emissive[k] *= t[k];

  uint32_t ext = mat.ext_flags;
  float specular = 1.0f;
  V3 specular_color = {1, 1, 1};
  if (ext & PT_EXT_SPECULAR) {
    specular = clampr(fin(mat.specular_factor, 1.0f), 0.0f, 1.0f);
    if (samp(mat.specular_texture, false, t)) specular *= t[3];
    for (int k = 0; k < 3; ++k) specular_color[k] = fmaxr(fin(mat.specular_color_factor[k], 1.0f), 0.0f);
    if (samp(mat.specular_color_texture, true, t))
      for (int k = 0; k < 3; ++k) specular_color[k] *= t[k];
  }
  float transmission = 0.0f;
  if (ext & PT_EXT_TRANSMISSION) {
    transmission = clampr(fin(mat.transmission_factor, 0.0f), 0.0f, 1.0f);
    if (samp(mat.transmission_texture, false, t)) transmission *= t[0];
  }
  float thickness = 0.0f, attenuation_distance = INF;
  V3 attenuation_color = {1, 1, 1};
  if (ext & PT_EXT_VOLUME) {
    thickness = fmaxr(fin(mat.thickness_factor, 0.0f), 0.0f);
    if (samp(mat.thickness_texture, false, t)) thickness *= t[1];
    for (int k = 0; k < 3; ++k) attenuation_color[k] = clampr(fin(mat.attenuation_color[k], 1.0f), 0.0f, 1.0f);
    float d = mat.attenuation_distance;
    attenuation_distance = (std::isfinite(d) && d > 0.0f) ? d : INF;
  }
  float clearcoat = 0.0f, clearcoat_roughness = 0.0f;
  V3 clearcoat_normal = sn;
  if (ext & PT_EXT_CLEARCOAT) {
    clearcoat = clampr(fin(mat.clearcoat_factor, 0.0f), 0.0f, 1.0f);
    if (samp(mat.clearcoat_texture, false, t)) clearcoat *= t[0];
    clearcoat_roughness = clampr(fin(mat.clearcoat_roughness_factor, 0.0f), 0.0f, 1.0f);
    if (samp(mat.clearcoat_roughness_texture, false, t)) clearcoat_roughness *= t[1];
    if (samp(mat.clearcoat_normal_texture, false, t))
      clearcoat_normal = perturb(item, base, b, sn, t, fin(mat.clearcoat_normal_scale, 1.0f));
  }
  V3 sheen_color = {0, 0, 0};
  float sheen_roughness = 0.0f;
  if (ext & PT_EXT_SHEEN) {
    for (int k = 0; k < 3; ++k) sheen_color[k] = clampr(fin(mat.sheen_color_factor[k], 0.0f), 0.0f, 1.0f);
    if (samp(mat.sheen_color_texture, true, t))
      for (int k = 0; k < 3; ++k) sheen_color[k] *= t[k];
    sheen_roughness = clampr(fin(mat.sheen_roughness_factor, 0.0f), 0.0f, 1.0f);
    if (samp(mat.sheen_roughness_texture, false, t)) sheen_roughness *= t[3];
  }
  float anisotropy = 0.0f;
  V3 anisotropy_direction = {0, 0, 0};
  if (ext & PT_EXT_ANISOTROPY) {
    anisotropy = clampr(fin(mat.anisotropy_strength, 0.0f), 0.0f, 1.0f);
    float dir[2] = {1.0f, 0.0f};
    if (samp(mat.anisotropy_texture, false, t)) {
      dir[0] = t[0] * 2.0f - 1.0f;
      dir[1] = t[1] * 2.0f - 1.0f;
      anisotropy *= clampr(t[2], 0.0f, 1.0f);
    }
    float rot_angle = fin(mat.anisotropy_rotation, 0.0f);
    float sr = std::sin(rot_angle), cr = std::cos(rot_angle);
    float rot[2] = {cr * dir[0] - sr * dir[1], sr * dir[0] + cr * dir[1]};
    V3 tt, bt;
    if (tangent_frame(item, base, b, sn, tt, bt)) {
      V3 d = normalise({tt.x * rot[0] + bt.x * rot[1], tt.y * rot[0] + bt.y * rot[1], tt.z * rot[0] + bt.z * rot[1]});
      if (dot(d, d) > 0.5f) anisotropy_direction = d;
    }
    if (dot(anisotropy_direction, anisotropy_direction) < 0.5f) anisotropy = 0.0f;
  }
  float iridescence = 0.0f, iridescence_ior = 1.3f, iridescence_thickness = 400.0f;
  if (ext & PT_EXT_IRIDESCENCE) {
    iridescence = clampr(fin(mat.iridescence_factor, 0.0f), 0.0f, 1.0f);
    if (samp(mat.iridescence_texture, false, t)) iridescence *= t[0];
    iridescence_ior = fmaxr(fin(mat.iridescence_ior, 1.3f), 1.0f);
    float lo = fin(mat.iridescence_thickness_min, 100.0f), hi = fin(mat.iridescence_thickness_max, 400.0f);
    float g = 1.0f;
    if (samp(mat.iridescence_thickness_texture, false, t)) g = clampr(t[1], 0.0f, 1.0f);
    iridescence_thickness = fmaxr(lo + (hi - lo) * g, 0.0f);
  }
  float diffuse_transmission = 0.0f;
  V3 dt_color = {1, 1, 1};
  if (ext & PT_EXT_DIFFUSE_TRANSMISSION) {
    diffuse_transmission = clampr(fin(mat.diffuse_transmission_factor, 0.0f), 0.0f, 1.0f);
    if (samp(mat.diffuse_transmission_texture, false, t)) diffuse_transmission *= t[3];
    for (int k = 0; k < 3; ++k)
      dt_color[k] = clampr(fin(mat.diffuse_transmission_color_factor[k], 1.0f), 0.0f, 1.0f);
    if (samp(mat.diffuse_transmission_color_texture, true, t))
      for (int k = 0; k < 3; ++k) dt_color[k] *= t[k];
  }
  float dispersion = (ext & PT_EXT_DISPERSION) ? fmaxr(fin(mat.dispersion, 0.0f), 0.0f) : 0.0f;

  for (int k = 0; k < 4; ++k) m.base_color[k] = col[k];
  m.metallic = clampr(metallic, 0.0f, 1.0f);
  m.roughness = clampr(roughness, 0.0f, 1.0f);
  m.normal = normal;
  m.occlusion = clampr(occlusion, 0.0f, 1.0f);
  m.emissive = emissive;
  m.unlit = mat.unlit != 0;
  m.alpha_mode = mat.alpha_mode;
  m.alpha_cutoff = mat.alpha_cutoff;
  m.double_sided = mat.double_sided != 0;
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
  m.diffuse_transmission = diffuse_transmission;
  m.diffuse_transmission_color = dt_color;
  m.dispersion = dispersion;
  return m;
}

// ---------------------------------------------------------------- lights

// PreparedLight::sample, src/prepare.rs:921-963.
bool light_sample(const pt_light &L, V3 p, LightSample &out) {
  V3 base = {L.color[0] * L.intensity, L.color[1] * L.intensity, L.color[2] * L.intensity};
  if (L.kind == PT_LIGHT_DIRECTIONAL) {
    out.l = {-L.direction[0], -L.direction[1], -L.direction[2]};
    out.distance = INF;
    out.radiance = base;
    return true;
  }
  V3 to = sub({L.position[0], L.position[1], L.position[2]}, p);
  float d2 = dot(to, to);
  if (std::isnan(d2) || d2 <= 1.0e-12f) return false;
  float d = std::sqrt(d2);
  V3 l = {to.x / d, to.y / d, to.z / d};
  float att = 1.0f / d2;
  if (L.has_range) {
    float x = d / L.range;
    att *= clampr(1.0f - x * x * x * x, 0.0f, 1.0f);
  }
  if (L.kind == PT_LIGHT_SPOT) {
    float cos_outer = std::cos(L.outer_cone_angle);
    float cos_inner = std::cos(L.inner_cone_angle);
    float sc = 1.0f / fmaxr(cos_inner - cos_outer, 0.001f);
    float offset = -cos_outer * sc;
    float cd = dot({L.direction[0], L.direction[1], L.direction[2]}, {-l.x, -l.y, -l.z});
    float a = clampr(cd * sc + offset, 0.0f, 1.0f);
    att *= a * a;
  }
  if (att <= 0.0f) return false;
  out.l = l;
  out.distance = d;
  out.radiance = {base.x * att, base.y * att, base.z * att};
  return true;
}

// EnvironmentMap::new, src/pathtrace.rs:1575-1638.
EnvironmentMap::EnvironmentMap(const pt_environment &env) {
  w = std::max(env.width, 1u);
  h = std::max(env.height, 1u);
  bool valid = env.pixels != nullptr && env.width > 0 && env.height > 0;
  if (valid) pixels.assign(env.pixels, env.pixels + (size_t)w * h * 4);
  std::vector<double> weights((size_t)w * h, 0.0);
  if (valid) {
    for (uint32_t y = 0; y < h; ++y) {
      double st = (double)std::sin(PI * ((float)y + 0.5f) / (float)h);
      for (uint32_t x = 0; x < w; ++x) {
        size_t i = ((size_t)y * w + x) * 4;
        float l = luminance({pixels[i], pixels[i + 1], pixels[i + 2]});
        weights[(size_t)y * w + x] = (std::isfinite(l) && l > 0.0f) ? (double)l * st : 0.0;
      }
    }
  }
  double total = 0.0;
  for (double x : weights) total += x;
  uniform = !(total > 0.0 && std::isfinite(total));
  if (uniform)
    for (size_t i = 0; i < weights.size(); ++i) {
      size_t y = i / w;
      weights[i] = (double)std::sin(PI * ((float)y + 0.5f) / (float)h);
    }
  total = 0.0;
  for (double x : weights) total += x;
  double acc = 0.0;
  marginal.push_back(0.0f);
  for (uint32_t y = 0; y < h; ++y) {
    double row = 0.0;
    for (uint32_t x = 0; x < w; ++x) row += weights[(size_t)y * w + x];
    double racc = 0.0;
    conditional.push_back(0.0f);
    for (uint32_t x = 0; x < w; ++x) {
      racc += weights[(size_t)y * w + x];
      conditional.push_back(row > 0.0 ? (float)(racc / row) : (float)(x + 1) / (float)w);
    }
    acc += row;
    marginal.push_back((float)(acc / total));
  }
  marginal.back() = 1.0f;
  mass.resize(weights.size());
  for (size_t i = 0; i < weights.size(); ++i) mass[i] = (float)(weights[i] / total);
  intensity = std::isfinite(env.intensity) ? fmaxr(env.intensity, 0.0f) : 0.0f;
}

void EnvironmentMap::texel_of(V3 d, size_t &x, size_t &y, float &st) const {
  float u = 0.5f + std::atan2(d.x, -d.z) / (2.0f * PI);
  float th = std::acos(clampr(d.y, -1.0f, 1.0f));
  float v = th / PI;
  x = std::min((size_t)f2usize(u * (float)w), (size_t)w - 1);
  y = std::min((size_t)f2usize(v * (float)h), (size_t)h - 1);
  st = std::sin(th);
}
V3 EnvironmentMap::radiance(V3 d) const {
  size_t x, y;
  float st;
  texel_of(d, x, y, st);
  size_t i = (y * w + x) * 4;
  if (uniform || i + 3 > pixels.size()) return {0, 0, 0};
  V3 c = {pixels[i], pixels[i + 1], pixels[i + 2]};
  if (!finite3(c)) return {0, 0, 0};
  return scale({fmaxr(c.x, 0.0f), fmaxr(c.y, 0.0f), fmaxr(c.z, 0.0f)}, intensity);
}
float EnvironmentMap::pdf(V3 d) const {
  size_t x, y;
  float st;
  texel_of(d, x, y, st);
  if (st <= 1.0e-6f) return 0.0f;
  return mass[y * w + x] * (float)(w * h) / (2.0f * PI * PI * st);
}
bool EnvironmentMap::sample(float u0, float u1, V3 &d, V3 &le, float &p) const {
  size_t yy = (size_t)(std::upper_bound(marginal.begin(), marginal.end(), u0) - marginal.begin());
  size_t y = std::min(std::max(yy, (size_t)1), (size_t)h) - 1;
  const float *row = &conditional[y * (w + 1)];
  size_t xx = (size_t)(std::upper_bound(row, row + w + 1, u1) - row);
  size_t x = std::min(std::max(xx, (size_t)1), (size_t)w) - 1;
  float my = (u0 - marginal[y]) / fmaxr(marginal[y + 1] - marginal[y], 1e-12f);
  float mx = (u1 - row[x]) / fmaxr(row[x + 1] - row[x], 1e-12f);
  float u = ((float)x + clampr(mx, 0.0f, 0.99999f)) / (float)w;
  float v = ((float)y + clampr(my, 0.0f, 0.99999f)) / (float)h;
  float phi = 2.0f * PI * (u - 0.5f);
  float th = PI * v;
  float st = std::sin(th), ct = std::cos(th);
  d = {st * std::sin(phi), ct, -st * std::cos(phi)};
  p = pdf(d);
  if (p <= 0.0f || !std::isfinite(p)) return false;
  le = radiance(d);
  return true;
}

}  // namespace oracle
