// Host-side scene preparation and upload (see host_scene.h).
//
// Reference behaviour restated here (host side, computed once per scene):
//   - TraceScene soup + TriRef order (src/trace.rs:328-351): global triangle
//     ids follow item order, then triangle order within an item;
//   - build_mips (src/texture.rs:324-383) for the sRGB and linear chains;
//   - EmissiveLights::build (src/pathtrace.rs:1479-1543), f64 CDF;
//   - EnvironmentMap::new (src/pathtrace.rs:1575-1638), f64 CDFs;
//   - sheen_lut (src/pathtrace.rs:645-674) and the sRGB byte thresholds
//     (src/hdr.rs:116-129).
// The BVH is this library's own: binned SAH (Wald, "On fast Construction of
// SAH-based Bounding Volume Hierarchies", 2007), built in parallel over
// subtrees, emitted depth-first as two-child nodes.
#include "host_scene.h"
#include "bvh_build.h"
#include "mip_build.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <numeric>
#include <thread>

#include <cuda_runtime.h>

namespace ptd {

// ============================================================ tables
float host_srgb_to_linear(float c) {
  if (c <= 0.04045f) return c / 12.92f;
  return std::pow((c + 0.055f) / 1.055f, 2.4f);
}
void host_srgb_thresholds(float out[255]) {
  for (int k = 0; k < 255; ++k) out[k] = host_srgb_to_linear(((float)k + 0.5f) / 255.0f);
}

static float h_d_charlie(float n_dot_h, float a) {
  float inv = 1.0f / std::fmax(a, 1.0e-3f);
  float sin2 = std::fmax(1.0f - n_dot_h * n_dot_h, 0.0f);
  return (2.0f + inv) * std::pow(sin2, inv * 0.5f) / (2.0f * 3.14159265358979323846f);
}
static float h_v_neubelt(float nl, float nv) { return 1.0f / std::fmax(4.0f * (nl + nv - nl * nv), 1.0e-6f); }
void host_sheen_lut(float out[512]) {
  const float PI = 3.14159265358979323846f, HALF_PI = 1.57079632679489661923f;
  const int nt = 48, np = 24, NC = 32, NR = 16;
  for (int ri = 0; ri < NR; ++ri) {
    float r = (float)ri / (float)(NR - 1);
    float a = std::fmax(r * r, 1.0e-3f);
    for (int ci = 0; ci < NC; ++ci) {
      float cv = std::fmax(((float)ci + 0.5f) / (float)NC, 1.0e-3f);
      float v[3] = {std::sqrt(1.0f - cv * cv), 0.0f, cv};
      float sum = 0.0f;
      for (int i = 0; i < nt; ++i) {
        float th = ((float)i + 0.5f) / (float)nt * HALF_PI;
        float st = std::sin(th), ct = std::cos(th);
        for (int j = 0; j < np; ++j) {
          float ph = ((float)j + 0.5f) / (float)np * PI;
          float l[3] = {st * std::cos(ph), st * std::sin(ph), ct};
          float h[3] = {v[0] + l[0], v[1] + l[1], v[2] + l[2]};
          float len = std::sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
          float hz = len < 1.1920929e-07f ? 0.0f : h[2] / len;
          float f = h_d_charlie(hz, a) * h_v_neubelt(ct, cv);
          sum += f * ct * st;
        }
      }
      float dw = (HALF_PI / (float)nt) * (PI / (float)np) * 2.0f;
      float x = sum * dw;
      out[ri * NC + ci] = x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x);
    }
  }
}

// ============================================================ BVH build
namespace {

struct BNode {
  float lo[3], hi[3];
  uint32_t left;         // interior: children left, left + 1
  uint32_t first, count;  // leaf when count > 0
};

struct Builder {
  const float *pos;
  uint32_t n;
  // Per-triangle bounds in build order: a node's triangles are one
  // contiguous run, partitioned in place as the tree splits.
  struct Prim {
    float lo[3], hi[3], c[3];
    uint32_t g;
  };
  std::vector<Prim> prims;
  std::vector<BNode> nodes;
  std::atomic<uint32_t> node_count{1};
  std::atomic<uint32_t> max_depth{0};

  struct Task {
    uint32_t node, begin, end, depth;
  };
  std::mutex mu;
  std::condition_variable cv;
  std::vector<Task> stack;
  int active = 0;
  bool done = false;

  static constexpr int kBins = 16;
  static constexpr uint32_t kMaxLeaf = 8;
  static constexpr uint32_t kLocalThreshold = 32768;
  static constexpr uint32_t kParallelNode = 65536;
  int wide = 1;  // threads for one large node's passes

  // Bin of a centroid offset times the bin scale: truncation, clamped to
  // the bins (a NaN offset lands in bin 0).
  static int bin_of(float f) { return f >= 1.0f ? std::min(kBins - 1, (int)std::min(f, 16.0f)) : 0; }
  static float area(const float lo[3], const float hi[3]) {
    float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    if (!(dx >= 0.0f) || !(dy >= 0.0f) || !(dz >= 0.0f)) return 0.0f;
    return dx * dy + dy * dz + dz * dx;
  }

  void make_leaf(BNode &nd, uint32_t b, uint32_t e) {
    nd.first = b;
    nd.count = e - b;
    nd.left = 0;
  }

  // Bin counts and bounds of a run of triangles, per axis (one pass over
  // the run for all three axes). Merging per-chunk bins gives exactly the
  // sequential result: sums of counts, min / max of the same values.
  struct Bins {
    uint32_t c[3][kBins];
    float l[3][kBins][3], h[3][kBins][3];
    void clear() {
      for (int k = 0; k < 3; ++k)
        for (int b = 0; b < kBins; ++b) {
          c[k][b] = 0;
          for (int a = 0; a < 3; ++a) {
            l[k][b][a] = INFINITY;
            h[k][b][a] = -INFINITY;
          }
        }
    }
    void merge(const Bins &o) {
      for (int k = 0; k < 3; ++k)
        for (int b = 0; b < kBins; ++b) {
          c[k][b] += o.c[k][b];
          for (int a = 0; a < 3; ++a) {
            l[k][b][a] = std::min(l[k][b][a], o.l[k][b][a]);
            h[k][b][a] = std::max(h[k][b][a], o.h[k][b][a]);
          }
        }
    }
  };
  void bin_range(Bins &B, uint32_t begin, uint32_t end, const float clo[3], const float scale[3],
                 const bool use[3]) const {
    for (uint32_t i = begin; i < end; ++i) {
      const Prim &pr = prims[i];
      for (int k = 0; k < 3; ++k) {
        if (!use[k]) continue;
        int b = bin_of((pr.c[k] - clo[k]) * scale[k]);
        B.c[k][b]++;
        for (int a = 0; a < 3; ++a) {
          B.l[k][b][a] = std::min(B.l[k][b][a], pr.lo[a]);
          B.h[k][b][a] = std::max(B.h[k][b][a], pr.hi[a]);
        }
      }
    }
  }
  void bounds_range(uint32_t begin, uint32_t end, float lo[3], float hi[3], float clo[3], float chi[3]) const {
    for (uint32_t i = begin; i < end; ++i) {
      const Prim &pr = prims[i];
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], pr.lo[k]);
        hi[k] = std::max(hi[k], pr.hi[k]);
        clo[k] = std::min(clo[k], pr.c[k]);
        chi[k] = std::max(chi[k], pr.c[k]);
      }
    }
  }
  // Runs fn(chunk, begin, end) over `chunks` slices of [begin, end) on threads.
  template <class F>
  static void parallel_chunks(uint32_t begin, uint32_t end, int chunks, F &&fn) {
    std::vector<std::thread> th;
    const uint32_t n = end - begin;
    for (int c = 0; c < chunks; ++c) {
      uint32_t b = begin + (uint32_t)((uint64_t)n * c / chunks), e = begin + (uint32_t)((uint64_t)n * (c + 1) / chunks);
      th.emplace_back([&fn, c, b, e] { fn(c, b, e); });
    }
    for (auto &x : th) x.join();
  }

  // Processes one node; returns the child tasks (0 or 2). Nodes of at least
  // kParallelNode triangles (the top of the tree, before the task pool has
  // enough subtrees) spread their passes over `wide` threads.
  int split(const Task &t, Task out[2]) {
    BNode &nd = nodes[t.node];
    uint32_t cnt = t.end - t.begin;
    const int par = cnt >= kParallelNode ? wide : 1;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
    if (par > 1) {
      std::vector<std::array<float, 12>> part(par);
      parallel_chunks(t.begin, t.end, par, [&](int c, uint32_t b, uint32_t e) {
        float l[3] = {INFINITY, INFINITY, INFINITY}, h[3] = {-INFINITY, -INFINITY, -INFINITY};
        float cl[3] = {INFINITY, INFINITY, INFINITY}, ch[3] = {-INFINITY, -INFINITY, -INFINITY};
        bounds_range(b, e, l, h, cl, ch);
        for (int k = 0; k < 3; ++k) {
          part[c][k] = l[k];
          part[c][3 + k] = h[k];
          part[c][6 + k] = cl[k];
          part[c][9 + k] = ch[k];
        }
      });
      for (int c = 0; c < par; ++c)
        for (int k = 0; k < 3; ++k) {
          lo[k] = std::min(lo[k], part[c][k]);
          hi[k] = std::max(hi[k], part[c][3 + k]);
          clo[k] = std::min(clo[k], part[c][6 + k]);
          chi[k] = std::max(chi[k], part[c][9 + k]);
        }
    } else {
      bounds_range(t.begin, t.end, lo, hi, clo, chi);
    }
    for (int k = 0; k < 3; ++k) {
      nd.lo[k] = lo[k];
      nd.hi[k] = hi[k];
    }
    uint32_t d = max_depth.load(std::memory_order_relaxed);
    while (t.depth > d && !max_depth.compare_exchange_weak(d, t.depth)) {
    }
    if (cnt <= 1) {
      make_leaf(nd, t.begin, t.end);
      return 0;
    }
    // Keep the tree shallow enough for a 64-entry traversal stack: near
    // the limit, split at the object median (halves the count per level).
    uint32_t need = 0;
    for (uint32_t c = cnt; c > kMaxLeaf; c = (c + 1) / 2) ++need;
    bool median = t.depth + need >= 56;
    int axis = -1;
    uint32_t mid = 0;
    int best_bin = 0;
    float best_cost = INFINITY;
    float scale[3] = {0.0f, 0.0f, 0.0f};
    if (!median) {
      float parent = area(lo, hi);
      bool use[3];
      for (int k = 0; k < 3; ++k) {
        float span = chi[k] - clo[k];
        use[k] = span > 0.0f;
        scale[k] = use[k] ? (float)kBins / span : 0.0f;
      }
      Bins B;
      B.clear();
      if (par > 1) {
        std::vector<Bins> part(par);
        parallel_chunks(t.begin, t.end, par, [&](int c, uint32_t b, uint32_t e) {
          part[c].clear();
          bin_range(part[c], b, e, clo, scale, use);
        });
        for (int c = 0; c < par; ++c) B.merge(part[c]);
      } else {
        bin_range(B, t.begin, t.end, clo, scale, use);
      }
      for (int k = 0; k < 3; ++k) {
        if (!use[k]) continue;
        const uint32_t *bc = B.c[k];
        float rl[kBins][3], rh[kBins][3];
        uint32_t rc[kBins];
        float accl[3] = {INFINITY, INFINITY, INFINITY}, acch[3] = {-INFINITY, -INFINITY, -INFINITY};
        uint32_t acc = 0;
        for (int b = kBins - 1; b >= 1; --b) {
          acc += bc[b];
          for (int a = 0; a < 3; ++a) {
            accl[a] = std::min(accl[a], B.l[k][b][a]);
            acch[a] = std::max(acch[a], B.h[k][b][a]);
          }
          rc[b] = acc;
          for (int a = 0; a < 3; ++a) {
            rl[b][a] = accl[a];
            rh[b][a] = acch[a];
          }
        }
        float ll[3] = {INFINITY, INFINITY, INFINITY}, lh[3] = {-INFINITY, -INFINITY, -INFINITY};
        uint32_t lc = 0;
        for (int s = 1; s < kBins; ++s) {
          lc += bc[s - 1];
          for (int a = 0; a < 3; ++a) {
            ll[a] = std::min(ll[a], B.l[k][s - 1][a]);
            lh[a] = std::max(lh[a], B.h[k][s - 1][a]);
          }
          if (lc == 0 || rc[s] == 0) continue;
          float cost = 1.0f + (area(ll, lh) * (float)lc + area(rl[s], rh[s]) * (float)rc[s]) / std::max(parent, 1e-30f);
          if (cost < best_cost) {
            best_cost = cost;
            axis = k;
            best_bin = s;
          }
        }
      }
      if (cnt <= kMaxLeaf && (axis < 0 || (float)cnt <= best_cost)) {
        make_leaf(nd, t.begin, t.end);
        return 0;
      }
    }
    if (axis >= 0) {
      const float sc = scale[axis], base = clo[axis];
      auto left = [&](const Prim &pr) { return bin_of((pr.c[axis] - base) * sc) < best_bin; };
      if (par > 1) {
        // Two passes: count each chunk's left side, then scatter every chunk
        // into its place (stable within chunks) and copy back.
        std::vector<uint32_t> nl(par, 0);
        parallel_chunks(t.begin, t.end, par, [&](int c, uint32_t b, uint32_t e) {
          uint32_t k = 0;
          for (uint32_t i = b; i < e; ++i) k += left(prims[i]) ? 1u : 0u;
          nl[c] = k;
        });
        std::vector<uint32_t> lofs(par), rofs(par);
        uint32_t total_left = 0;
        for (int c = 0; c < par; ++c) total_left += nl[c];
        uint32_t lacc = 0, racc = total_left;
        for (int c = 0; c < par; ++c) {
          uint32_t b = t.begin + (uint32_t)((uint64_t)cnt * c / par), e = t.begin + (uint32_t)((uint64_t)cnt * (c + 1) / par);
          lofs[c] = lacc;
          rofs[c] = racc;
          lacc += nl[c];
          racc += (e - b) - nl[c];
        }
        std::vector<Prim> tmp(cnt);
        parallel_chunks(t.begin, t.end, par, [&](int c, uint32_t b, uint32_t e) {
          uint32_t li = lofs[c], ri = rofs[c];
          for (uint32_t i = b; i < e; ++i) tmp[left(prims[i]) ? li++ : ri++] = prims[i];
        });
        parallel_chunks(0, cnt, par, [&](int, uint32_t b, uint32_t e) {
          std::copy(tmp.begin() + b, tmp.begin() + e, prims.begin() + t.begin + b);
        });
        mid = t.begin + total_left;
      } else {
        auto it = std::partition(prims.begin() + t.begin, prims.begin() + t.end, left);
        mid = (uint32_t)(it - prims.begin());
      }
    }
    if (axis < 0 || mid == t.begin || mid == t.end) {
      // Object median along the widest centroid axis (or index halves when
      // every centroid coincides).
      int ax = 0;
      float w = chi[0] - clo[0];
      for (int k = 1; k < 3; ++k)
        if (chi[k] - clo[k] > w) {
          w = chi[k] - clo[k];
          ax = k;
        }
      mid = t.begin + cnt / 2;
      if (w > 0.0f)
        std::nth_element(prims.begin() + t.begin, prims.begin() + mid, prims.begin() + t.end,
                         [&](const Prim &a, const Prim &b) { return a.c[ax] < b.c[ax]; });
    }
    uint32_t c = node_count.fetch_add(2);
    nd.left = c;
    nd.count = 0;
    out[0] = {c, t.begin, mid, t.depth + 1};
    out[1] = {c + 1, mid, t.end, t.depth + 1};
    return 2;
  }

  void local_build(Task t) {
    std::vector<Task> st{t};
    while (!st.empty()) {
      Task cur = st.back();
      st.pop_back();
      Task ch[2];
      if (split(cur, ch) == 2) {
        st.push_back(ch[1]);
        st.push_back(ch[0]);
      }
    }
  }

  void worker() {
    for (;;) {
      Task t;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return done || !stack.empty(); });
        if (stack.empty()) return;
        t = stack.back();
        stack.pop_back();
        ++active;
      }
      if (t.end - t.begin <= kLocalThreshold) {
        local_build(t);
      } else {
        Task ch[2];
        if (split(t, ch) == 2) {
          std::lock_guard<std::mutex> lk(mu);
          stack.push_back(ch[0]);
          stack.push_back(ch[1]);
          cv.notify_all();
        }
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        --active;
        if (active == 0 && stack.empty()) {
          done = true;
          cv.notify_all();
        }
      }
    }
  }

  void run(int threads) {
    nodes.resize(std::max<size_t>(2 * (size_t)n, 1));
    if (threads <= 1 || n <= kLocalThreshold) {
      local_build({0, 0, n, 0});
    } else {
      stack.push_back({0, 0, n, 0});
      std::vector<std::thread> pool;
      for (int i = 0; i < threads; ++i) pool.emplace_back([this] { worker(); });
      for (auto &th : pool) th.join();
    }
    nodes.resize(node_count.load());
  }
};

void pad_box(const float lo[3], const float hi[3], float plo[3], float phi[3]) {
  float ext = 0.0f;
  for (int k = 0; k < 3; ++k)
    ext = std::max({ext, hi[k] - lo[k], std::fabs(lo[k]), std::fabs(hi[k])});
  float pad = ext * 1.0e-5f + 1.0e-30f;
  for (int k = 0; k < 3; ++k) {
    plo[k] = lo[k] - pad;
    phi[k] = hi[k] + pad;
  }
}

// Spatial-split BVH (Stich, Friedrich & Dietrich, "Spatial Splits in
// Bounding Volume Hierarchies", HPG 2009). At every node the binned object
// split (Builder's rule: SAH over centroid bins) competes with a spatial
// split, which cuts the node's box at a plane and every triangle reference
// straddling it into two references bounding the clipped triangle. A
// spatial split is tried only where the object split's two children
// overlap by more than kAlpha of the root's surface area, and only while
// the node's subtree stays within its share of the reference budget
// (kMaxGrowth times the triangle count overall). A triangle may end
// up in several leaves; its record is repeated. Traversal answers do not
// change: the closest hit is the accepted candidate of smallest t (ties to
// the lowest global id) wherever it is found, and every point of a triangle
// lies in the box of some leaf that references it.
struct SpatialBuilder {
  struct Ref {
    float lo[3], hi[3];
    uint32_t g;
  };
  // A node to split: its references and the most references its subtree
  // may end with (the root's is the whole budget; a split hands each child
  // a share in proportion to its references, so the tree does not depend
  // on thread timing).
  struct Task {
    uint32_t node, depth;
    std::vector<Ref> refs;
    uint64_t budget;
  };
  static constexpr int kObjBins = 16, kSpatialBins = 32;
  // Leaves of at most four references: a warp's leaf phase waits for its
  // largest leaf, and on the request mix 4 traced 1 % faster than 8.
  static constexpr uint32_t kMaxLeaf = 4;
  static constexpr uint32_t kLocalThreshold = 4096;
  static constexpr uint32_t kParallelNode = 262144;  // nodes binned on three threads
  static constexpr float kAlpha = 1e-5f;
  static constexpr double kMaxGrowth = 4.0;

  const float *pos = nullptr;
  uint32_t n = 0;
  std::vector<BNode> nodes;
  std::atomic<uint32_t> node_count{1};
  std::vector<uint32_t> order;
  std::atomic<uint64_t> order_fill{0};
  uint64_t max_refs = 0;
  float min_overlap = 0.0f;
  std::atomic<uint32_t> max_depth{0};
  std::mutex mu;
  std::condition_variable cv;
  std::vector<Task> stack;
  int active = 0;
  bool done = false;

  static void grow(float lo[3], float hi[3], const float p[3]) {
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], p[k]);
      hi[k] = std::max(hi[k], p[k]);
    }
  }
  static void grow_box(float lo[3], float hi[3], const float blo[3], const float bhi[3]) {
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], blo[k]);
      hi[k] = std::max(hi[k], bhi[k]);
    }
  }
  static bool valid(const float lo[3], const float hi[3]) {
    return lo[0] <= hi[0] && lo[1] <= hi[1] && lo[2] <= hi[2];
  }
  static void empty_box(float lo[3], float hi[3]) {
    for (int k = 0; k < 3; ++k) {
      lo[k] = INFINITY;
      hi[k] = -INFINITY;
    }
  }

  // The parts of reference `r` (its triangle clipped to its box) on either
  // side of `plane` on `axis`: bounds of the triangle's vertices and edge
  // crossings on each side, cut at the plane and intersected with r's box.
  void split_ref(const Ref &r, int axis, float plane, Ref &L, Ref &R) const {
    const float *p = pos + 9 * (size_t)r.g;
    empty_box(L.lo, L.hi);
    empty_box(R.lo, R.hi);
    for (int i = 0; i < 3; ++i) {
      const float *v0 = p + 3 * i, *v1 = p + 3 * ((i + 1) % 3);
      if (v0[axis] <= plane) grow(L.lo, L.hi, v0);
      if (v0[axis] >= plane) grow(R.lo, R.hi, v0);
      if ((v0[axis] < plane && v1[axis] > plane) || (v0[axis] > plane && v1[axis] < plane)) {
        const float t = (plane - v0[axis]) / (v1[axis] - v0[axis]);
        float q[3];
        for (int k = 0; k < 3; ++k) q[k] = v0[k] + t * (v1[k] - v0[k]);
        q[axis] = plane;
        grow(L.lo, L.hi, q);
        grow(R.lo, R.hi, q);
      }
    }
    L.hi[axis] = std::min(L.hi[axis], plane);
    R.lo[axis] = std::max(R.lo[axis], plane);
    for (int k = 0; k < 3; ++k) {
      L.lo[k] = std::max(L.lo[k], r.lo[k]);
      L.hi[k] = std::min(L.hi[k], r.hi[k]);
      R.lo[k] = std::max(R.lo[k], r.lo[k]);
      R.hi[k] = std::min(R.hi[k], r.hi[k]);
    }
    L.g = R.g = r.g;
  }

  void make_leaf(BNode &nd, const std::vector<Ref> &refs) {
    const uint64_t first = order_fill.fetch_add(refs.size());
    for (size_t i = 0; i < refs.size(); ++i) order[first + i] = refs[i].g;
    nd.first = (uint32_t)first;
    nd.count = (uint32_t)refs.size();
    nd.left = 0;
  }

  // Processes one node: a leaf, or two child tasks in `out`.
  int split(Task &t, Task out[2]) {
    BNode &nd = nodes[t.node];
    std::vector<Ref> &refs = t.refs;
    const uint32_t cnt = (uint32_t)refs.size();
    float lo[3], hi[3], clo[3], chi[3];
    empty_box(lo, hi);
    empty_box(clo, chi);
    for (const Ref &r : refs) {
      grow_box(lo, hi, r.lo, r.hi);
      float c[3] = {(r.lo[0] + r.hi[0]) * 0.5f, (r.lo[1] + r.hi[1]) * 0.5f, (r.lo[2] + r.hi[2]) * 0.5f};
      grow(clo, chi, c);
    }
    for (int k = 0; k < 3; ++k) {
      nd.lo[k] = lo[k];
      nd.hi[k] = hi[k];
    }
    uint32_t d = max_depth.load(std::memory_order_relaxed);
    while (t.depth > d && !max_depth.compare_exchange_weak(d, t.depth)) {
    }
    if (cnt <= 1) {
      make_leaf(nd, refs);
      return 0;
    }
    uint32_t need = 0;
    for (uint32_t c = cnt; c > kMaxLeaf; c = (c + 1) / 2) ++need;
    const bool median = t.depth + need >= 56;
    const float parent = std::max(Builder::area(lo, hi), 1e-30f);
    // Object split over centroid bins, and (where the object split's
    // children overlap enough and the reference budget allows) a spatial
    // split over bins of the node's box; each axis is an independent pass,
    // run on its own thread for large nodes.
    struct ObjAxis {
      float cost = INFINITY, scale = 0.0f, lo_l[3], hi_l[3], lo_r[3], hi_r[3];
      int bin = 0;
    } oa[3];
    struct SpAxis {
      float cost = INFINITY, plane = 0.0f;
    } sa[3];
    auto object_axis = [&](int k) {
      ObjAxis &res = oa[k];
      const float span = chi[k] - clo[k];
      if (!(span > 0.0f)) return;
      const float sc = (float)kObjBins / span;
      uint32_t bc[kObjBins] = {};
      float bl[kObjBins][3], bh[kObjBins][3];
      for (int b = 0; b < kObjBins; ++b) empty_box(bl[b], bh[b]);
      for (const Ref &r : refs) {
        const float c = (r.lo[k] + r.hi[k]) * 0.5f;
        const int b = std::min(kObjBins - 1, std::max(0, (int)((c - clo[k]) * sc)));
        bc[b]++;
        grow_box(bl[b], bh[b], r.lo, r.hi);
      }
      float rl[kObjBins][3], rh[kObjBins][3];
      uint32_t rc[kObjBins];
      float al[3], ah[3];
      empty_box(al, ah);
      uint32_t acc = 0;
      for (int b = kObjBins - 1; b >= 1; --b) {
        acc += bc[b];
        grow_box(al, ah, bl[b], bh[b]);
        rc[b] = acc;
        std::copy(al, al + 3, rl[b]);
        std::copy(ah, ah + 3, rh[b]);
      }
      float ll[3], lh[3];
      empty_box(ll, lh);
      uint32_t lc = 0;
      for (int sp = 1; sp < kObjBins; ++sp) {
        lc += bc[sp - 1];
        grow_box(ll, lh, bl[sp - 1], bh[sp - 1]);
        if (lc == 0 || rc[sp] == 0) continue;
        const float cost =
            1.0f + (Builder::area(ll, lh) * (float)lc + Builder::area(rl[sp], rh[sp]) * (float)rc[sp]) / parent;
        if (cost < res.cost) {
          res.cost = cost;
          res.bin = sp;
          res.scale = sc;
          std::copy(ll, ll + 3, res.lo_l);
          std::copy(lh, lh + 3, res.hi_l);
          std::copy(rl[sp], rl[sp] + 3, res.lo_r);
          std::copy(rh[sp], rh[sp] + 3, res.hi_r);
        }
      }
    };
    auto spatial_axis = [&](int k) {
      SpAxis &res = sa[k];
      const float span = hi[k] - lo[k];
      if (!(span > 0.0f)) return;
      const float w = span / (float)kSpatialBins;
      auto bin_of = [&](float x) { return std::min(kSpatialBins - 1, std::max(0, (int)((x - lo[k]) / w))); };
      uint32_t entry[kSpatialBins] = {}, exit[kSpatialBins] = {};
      float bl[kSpatialBins][3], bh[kSpatialBins][3];
      for (int b = 0; b < kSpatialBins; ++b) empty_box(bl[b], bh[b]);
      for (const Ref &r : refs) {
        const int fb = bin_of(r.lo[k]), lb = std::max(fb, bin_of(r.hi[k]));
        entry[fb]++;
        exit[lb]++;
        Ref cur = r;
        for (int b = fb; b < lb; ++b) {
          Ref L, R;
          split_ref(cur, k, lo[k] + w * (float)(b + 1), L, R);
          if (valid(L.lo, L.hi)) grow_box(bl[b], bh[b], L.lo, L.hi);
          cur = R;
          if (!valid(cur.lo, cur.hi)) break;
        }
        if (valid(cur.lo, cur.hi)) grow_box(bl[lb], bh[lb], cur.lo, cur.hi);
      }
      float rl[kSpatialBins][3], rh[kSpatialBins][3];
      uint32_t rc[kSpatialBins];
      float al[3], ah[3];
      empty_box(al, ah);
      uint32_t acc = 0;
      for (int b = kSpatialBins - 1; b >= 1; --b) {
        acc += exit[b];
        grow_box(al, ah, bl[b], bh[b]);
        rc[b] = acc;
        std::copy(al, al + 3, rl[b]);
        std::copy(ah, ah + 3, rh[b]);
      }
      float ll[3], lh[3];
      empty_box(ll, lh);
      uint32_t lc = 0;
      for (int sp = 1; sp < kSpatialBins; ++sp) {
        lc += entry[sp - 1];
        grow_box(ll, lh, bl[sp - 1], bh[sp - 1]);
        if (lc == 0 || rc[sp] == 0 || !valid(ll, lh) || !valid(rl[sp], rh[sp])) continue;
        const float cost =
            1.0f + (Builder::area(ll, lh) * (float)lc + Builder::area(rl[sp], rh[sp]) * (float)rc[sp]) / parent;
        if (cost < res.cost) {
          res.cost = cost;
          res.plane = lo[k] + w * (float)sp;
        }
      }
    };
    const bool par = cnt >= kParallelNode;
    auto each_axis = [&](auto &&fn) {
      if (par) {
        std::thread t1([&] { fn(1); }), t2([&] { fn(2); });
        fn(0);
        t1.join();
        t2.join();
      } else {
        for (int k = 0; k < 3; ++k) fn(k);
      }
    };
    int oaxis = -1, obin = 0;
    float ocost = INFINITY, oscale = 0.0f;
    if (!median) {
      each_axis(object_axis);
      for (int k = 0; k < 3; ++k)
        if (oa[k].cost < ocost) {
          ocost = oa[k].cost;
          oaxis = k;
          obin = oa[k].bin;
          oscale = oa[k].scale;
        }
    }
    int saxis = -1;
    float scost = INFINITY, splane = 0.0f;
    if (!median && oaxis >= 0 && t.budget > cnt) {
      const ObjAxis &o = oa[oaxis];
      float ilo[3], ihi[3];
      for (int k = 0; k < 3; ++k) {
        ilo[k] = std::max(o.lo_l[k], o.lo_r[k]);
        ihi[k] = std::min(o.hi_l[k], o.hi_r[k]);
      }
      const float overlap = valid(ilo, ihi) ? Builder::area(ilo, ihi) : 0.0f;
      if (overlap > min_overlap) {
        each_axis(spatial_axis);
        for (int k = 0; k < 3; ++k)
          if (sa[k].cost < scost) {
            scost = sa[k].cost;
            saxis = k;
            splane = sa[k].plane;
          }
      }
    }
    const float best = std::min(ocost, scost);
    if (cnt <= kMaxLeaf && (oaxis < 0 || (float)cnt <= best)) {
      make_leaf(nd, refs);
      return 0;
    }
    std::vector<Ref> left, right;
    if (saxis >= 0 && scost < ocost) {
      uint64_t straddle = 0;
      for (const Ref &r : refs)
        if (r.lo[saxis] < splane && r.hi[saxis] > splane) ++straddle;
      if (cnt + straddle <= t.budget) {
        left.reserve(cnt);
        right.reserve(cnt);
        for (const Ref &r : refs) {
          if (r.hi[saxis] <= splane) {
            left.push_back(r);
          } else if (r.lo[saxis] >= splane) {
            right.push_back(r);
          } else {
            Ref L, R;
            split_ref(r, saxis, splane, L, R);
            const bool vl = valid(L.lo, L.hi), vr = valid(R.lo, R.hi);
            if (vl) left.push_back(L);
            if (vr) right.push_back(R);
            if (!vl && !vr) right.push_back(r);  // degenerate clip: keep the reference whole
          }
        }
        if (left.empty() || right.empty()) {
          left.clear();
          right.clear();
        }
      }
    }
    if (left.empty() && right.empty() && oaxis >= 0) {
      for (const Ref &r : refs) {
        const float c = (r.lo[oaxis] + r.hi[oaxis]) * 0.5f;
        const int b = std::min(kObjBins - 1, std::max(0, (int)((c - clo[oaxis]) * oscale)));
        (b < obin ? left : right).push_back(r);
      }
      if (left.empty() || right.empty()) {
        left.clear();
        right.clear();
      }
    }
    if (left.empty() || right.empty()) {
      // Object median along the widest centroid axis (or index halves).
      left.clear();
      right.clear();
      int ax = 0;
      float wd = chi[0] - clo[0];
      for (int k = 1; k < 3; ++k)
        if (chi[k] - clo[k] > wd) {
          wd = chi[k] - clo[k];
          ax = k;
        }
      const uint32_t mid = cnt / 2;
      if (wd > 0.0f)
        std::nth_element(refs.begin(), refs.begin() + mid, refs.end(), [&](const Ref &a, const Ref &b) {
          return a.lo[ax] + a.hi[ax] < b.lo[ax] + b.hi[ax];
        });
      left.assign(refs.begin(), refs.begin() + mid);
      right.assign(refs.begin() + mid, refs.end());
    }
    std::vector<Ref>().swap(refs);
    const uint32_t c = node_count.fetch_add(2);
    nd.left = c;
    nd.count = 0;
    const uint64_t nl = left.size(), nr = right.size();
    const uint64_t bl = std::max<uint64_t>(nl, (uint64_t)((double)t.budget * (double)nl / (double)(nl + nr)));
    out[0].node = c;
    out[0].depth = t.depth + 1;
    out[0].refs = std::move(left);
    out[0].budget = bl;
    out[1].node = c + 1;
    out[1].depth = t.depth + 1;
    out[1].refs = std::move(right);
    out[1].budget = std::max<uint64_t>(nr, t.budget > bl ? t.budget - bl : 0);
    return 2;
  }

  void local_build(Task t) {
    std::vector<Task> st;
    st.push_back(std::move(t));
    while (!st.empty()) {
      Task cur = std::move(st.back());
      st.pop_back();
      Task ch[2];
      if (split(cur, ch) == 2) {
        st.push_back(std::move(ch[1]));
        st.push_back(std::move(ch[0]));
      }
    }
  }

  void worker() {
    for (;;) {
      Task t;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return done || !stack.empty(); });
        if (stack.empty()) return;
        t = std::move(stack.back());
        stack.pop_back();
        ++active;
      }
      if (t.refs.size() <= kLocalThreshold) {
        local_build(std::move(t));
      } else {
        Task ch[2];
        if (split(t, ch) == 2) {
          std::lock_guard<std::mutex> lk(mu);
          stack.push_back(std::move(ch[0]));
          stack.push_back(std::move(ch[1]));
          cv.notify_all();
        }
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        --active;
        if (active == 0 && stack.empty()) {
          done = true;
          cv.notify_all();
        }
      }
    }
  }

  void run(std::vector<Ref> refs, int threads) {
    max_refs = (uint64_t)std::ceil(kMaxGrowth * (double)n);
    order.resize(max_refs);
    nodes.resize(2 * max_refs + 2);
    float lo[3], hi[3];
    empty_box(lo, hi);
    for (const Ref &r : refs) grow_box(lo, hi, r.lo, r.hi);
    min_overlap = kAlpha * Builder::area(lo, hi);
    Task root{0, 0, std::move(refs), max_refs};
    if (threads <= 1 || root.refs.size() <= kLocalThreshold) {
      local_build(std::move(root));
    } else {
      stack.push_back(std::move(root));
      std::vector<std::thread> pool;
      for (int i = 0; i < threads; ++i) pool.emplace_back([this] { worker(); });
      for (auto &th : pool) th.join();
    }
    nodes.resize(node_count.load());
    order.resize(order_fill.load());
  }
};

// Lays out a built binary tree (`nodes`, leaves indexing `order`, the
// global triangle id of each leaf slot) as two-child nodes, four-child nodes
// and leaf-ordered triangle records.
void emit_tree(const std::vector<BNode> &nodes, const std::vector<uint32_t> &order, uint32_t max_depth,
               const float *pos, const uint32_t *rec_flags, std::vector<BvhNode> &out_nodes,
               std::vector<Bvh4Node> &out_nodes4, std::vector<float4> &records, BvhBuildStats &stats);

}  // namespace

void build_bvh(const float *pos, uint32_t tri_count, const uint32_t *rec_flags, std::vector<BvhNode> &out_nodes,
               std::vector<Bvh4Node> &out_nodes4, std::vector<float4> &records, BvhBuildStats &stats, int threads) {
  auto t0 = std::chrono::steady_clock::now();
  out_nodes.clear();
  out_nodes4.clear();
  records.clear();
  stats = BvhBuildStats{};
  if (tri_count == 0) return;
  Builder b;
  b.pos = pos;
  b.n = tri_count;
  b.prims.resize(tri_count);
  for (size_t g = 0; g < tri_count; ++g) {
    const float *p = pos + 9 * g;
    Builder::Prim &pr = b.prims[g];
    pr.g = (uint32_t)g;
    for (int k = 0; k < 3; ++k) {
      float lo = std::min({p[k], p[3 + k], p[6 + k]}), hi = std::max({p[k], p[3 + k], p[6 + k]});
      pr.lo[k] = lo;
      pr.hi[k] = hi;
      pr.c[k] = (lo + hi) * 0.5f;
    }
  }
  b.wide = std::max(1, threads);
  b.run(std::max(1, threads));
  std::vector<uint32_t> order(tri_count);
  for (size_t i = 0; i < tri_count; ++i) order[i] = b.prims[i].g;
  emit_tree(b.nodes, order, b.max_depth.load(), pos, rec_flags, out_nodes, out_nodes4, records, stats);
  stats.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void build_bvh_spatial(const float *pos, uint32_t tri_count, const uint32_t *rec_flags,
                       std::vector<BvhNode> &out_nodes, std::vector<Bvh4Node> &out_nodes4,
                       std::vector<float4> &records, BvhBuildStats &stats, int threads) {
  auto t0 = std::chrono::steady_clock::now();
  out_nodes.clear();
  out_nodes4.clear();
  records.clear();
  stats = BvhBuildStats{};
  if (tri_count == 0) return;
  SpatialBuilder b;
  b.pos = pos;
  b.n = tri_count;
  std::vector<SpatialBuilder::Ref> refs(tri_count);
  for (size_t g = 0; g < tri_count; ++g) {
    const float *p = pos + 9 * g;
    SpatialBuilder::Ref &r = refs[g];
    r.g = (uint32_t)g;
    for (int k = 0; k < 3; ++k) {
      r.lo[k] = std::min({p[k], p[3 + k], p[6 + k]});
      r.hi[k] = std::max({p[k], p[3 + k], p[6 + k]});
    }
  }
  b.run(std::move(refs), std::max(1, threads));
  emit_tree(b.nodes, b.order, b.max_depth.load(), pos, rec_flags, out_nodes, out_nodes4, records, stats);
  stats.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

namespace {

void emit_tree(const std::vector<BNode> &in_nodes, const std::vector<uint32_t> &in_order, uint32_t max_depth,
               const float *pos, const uint32_t *rec_flags, std::vector<BvhNode> &out_nodes,
               std::vector<Bvh4Node> &out_nodes4, std::vector<float4> &records, BvhBuildStats &stats) {
  // Records in depth-first leaf order (left child first), whatever order
  // the builder's threads filled `in_order` in: the layout is deterministic
  // and a subtree's triangles are contiguous.
  std::vector<BNode> nodes(in_nodes);
  std::vector<uint32_t> order;
  order.reserve(in_order.size());
  {
    std::vector<uint32_t> st{0};
    while (!st.empty()) {
      BNode &nd = nodes[st.back()];
      st.pop_back();
      if (nd.count > 0) {
        const uint32_t first = (uint32_t)order.size();
        order.insert(order.end(), in_order.begin() + nd.first, in_order.begin() + nd.first + nd.count);
        nd.first = first;
      } else {
        st.push_back(nd.left + 1);
        st.push_back(nd.left);
      }
    }
  }
  // Depth-first two-child layout.
  auto leaf_ref = [](uint32_t first, uint32_t count) { return (int)~(first | (count << 27)); };
  std::vector<uint32_t> gstack;
  const BNode &root = nodes[0];
  auto child_box = [&](const BNode &c, float lo[3], float hi[3]) { pad_box(c.lo, c.hi, lo, hi); };
  auto fill = [&](BvhNode &gn, const BNode &c0, const BNode &c1, int r0, int r1) {
    float l0[3], h0[3], l1[3], h1[3];
    child_box(c0, l0, h0);
    child_box(c1, l1, h1);
    gn.a = make_float4(l0[0], h0[0], l0[1], h0[1]);
    gn.b = make_float4(l1[0], h1[0], l1[1], h1[1]);
    gn.c = make_float4(l0[2], h0[2], l1[2], h1[2]);
    gn.d = make_int4(r0, r1, (int)c0.count, (int)c1.count);
  };
  if (root.count > 0) {
    BvhNode gn;
    BNode empty = root;
    empty.count = 0;
    fill(gn, root, root, leaf_ref(root.first, root.count), leaf_ref(root.first, 0));
    out_nodes.push_back(gn);
    stats.leaves = 1;
  } else {
    // Iterative DFS: each interior binary node becomes one GPU node.
    struct Item {
      uint32_t bin, gpu;
    };
    std::vector<Item> st;
    out_nodes.push_back(BvhNode{});
    st.push_back({0, 0});
    while (!st.empty()) {
      Item it = st.back();
      st.pop_back();
      const BNode &nd = nodes[it.bin];
      const BNode &c0 = nodes[nd.left];
      const BNode &c1 = nodes[nd.left + 1];
      int r[2];
      const BNode *cs[2] = {&c0, &c1};
      for (int k = 0; k < 2; ++k) {
        if (cs[k]->count > 0) {
          r[k] = leaf_ref(cs[k]->first, cs[k]->count);
          stats.leaves++;
        } else {
          r[k] = (int)out_nodes.size();
          out_nodes.push_back(BvhNode{});
        }
      }
      fill(out_nodes[it.gpu], c0, c1, r[0], r[1]);
      // Right first on the stack so the left subtree is laid out first.
      if (cs[1]->count == 0) st.push_back({nd.left + 1, (uint32_t)r[1]});
      if (cs[0]->count == 0) st.push_back({nd.left, (uint32_t)r[0]});
    }
  }
  // Four-child layout: a node starts from its two binary children and opens
  // the interior child of largest surface area until it holds four.
  {
    auto set_child = [&](Bvh4Node &n, int slot, const BNode *c, int ref) {
      float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
      if (c) pad_box(c->lo, c->hi, lo, hi);
      reinterpret_cast<float *>(&n.lo_x)[slot] = lo[0];
      reinterpret_cast<float *>(&n.hi_x)[slot] = hi[0];
      reinterpret_cast<float *>(&n.lo_y)[slot] = lo[1];
      reinterpret_cast<float *>(&n.hi_y)[slot] = hi[1];
      reinterpret_cast<float *>(&n.lo_z)[slot] = lo[2];
      reinterpret_cast<float *>(&n.hi_z)[slot] = hi[2];
      reinterpret_cast<int *>(&n.child)[slot] = ref;
    };
    struct Item {
      uint32_t bin, gpu;
    };
    out_nodes4.push_back(Bvh4Node{});
    out_nodes4[0].pad = make_int4(0, 0, 0, 0);
    if (root.count > 0) {
      set_child(out_nodes4[0], 0, &root, leaf_ref(root.first, root.count));
      for (int k = 1; k < 4; ++k) set_child(out_nodes4[0], k, nullptr, kEmptyChild);
    } else {
      std::vector<Item> st{{0, 0}};
      while (!st.empty()) {
        Item it = st.back();
        st.pop_back();
        const BNode &nd = nodes[it.bin];
        uint32_t ch[4] = {nd.left, nd.left + 1, 0, 0};
        int nch = 2;
        while (nch < 4) {
          int best = -1;
          float best_area = -1.0f;
          for (int i = 0; i < nch; ++i) {
            const BNode &c = nodes[ch[i]];
            if (c.count > 0) continue;
            float a = Builder::area(c.lo, c.hi);
            if (a > best_area) {
              best_area = a;
              best = i;
            }
          }
          if (best < 0) break;
          uint32_t opened = ch[best];
          for (int i = nch; i > best + 1; --i) ch[i] = ch[i - 1];
          ch[best] = nodes[opened].left;
          ch[best + 1] = nodes[opened].left + 1;
          ++nch;
        }
        std::vector<Item> next;
        for (int k = 0; k < 4; ++k) {
          if (k >= nch) {
            set_child(out_nodes4[it.gpu], k, nullptr, kEmptyChild);
            continue;
          }
          const BNode &c = nodes[ch[k]];
          int ref;
          if (c.count > 0) {
            ref = leaf_ref(c.first, c.count);
          } else {
            ref = (int)out_nodes4.size();
            out_nodes4.push_back(Bvh4Node{});
            out_nodes4.back().pad = make_int4(0, 0, 0, 0);
            next.push_back({ch[k], (uint32_t)ref});
          }
          set_child(out_nodes4[it.gpu], k, &c, ref);
        }
        for (auto r = next.rbegin(); r != next.rend(); ++r) st.push_back(*r);
      }
    }
  }
  records.resize(3 * order.size());
  for (size_t i = 0; i < order.size(); ++i) {
    uint32_t g = order[i];
    const float *p = pos + 9 * (size_t)g;
    float gid, fl;
    std::memcpy(&gid, &g, 4);
    uint32_t f = rec_flags ? rec_flags[g] : 0u;
    std::memcpy(&fl, &f, 4);
    records[3 * i] = make_float4(p[0], p[1], p[2], gid);
    records[3 * i + 1] = make_float4(p[3], p[4], p[5], fl);
    records[3 * i + 2] = make_float4(p[6], p[7], p[8], 0.0f);
  }
  stats.nodes = (uint32_t)out_nodes.size();
  stats.max_depth = max_depth;
  stats.references = (uint64_t)order.size();
  // SAH cost of the tree (traversal 1, intersection 1, relative to the root box).
  double root_area = Builder::area(nodes[0].lo, nodes[0].hi);
  double cost = 0.0;
  for (const BNode &nd : nodes) {
    double a = Builder::area(nd.lo, nd.hi) / std::max(root_area, 1e-30);
    cost += nd.count > 0 ? a * nd.count : a;
  }
  stats.sah_cost = cost;
}

}  // namespace

// ============================================================ arena
void DeviceArena::release() {
  if (base) {
    if (stream)
      cudaFreeAsync(base, stream);
    else
      cudaFree(base);
  }
  base = nullptr;
  bytes = 0;
  stream = nullptr;
}

namespace {

struct ArenaPlan {
  std::vector<std::pair<const void *, size_t>> parts;  // host source, bytes
  std::vector<size_t> offsets;
  size_t total = 0;
  size_t add(const void *src, size_t bytes) {
    size_t off = (total + 255) & ~(size_t)255;
    parts.push_back({src, bytes});
    offsets.push_back(off);
    total = off + bytes;
    return parts.size() - 1;
  }
};

std::string commit(ArenaPlan &plan, DeviceArena &arena, bool &oom, cudaStream_t stream) {
  if (plan.total == 0) plan.total = 256;
  cudaError_t e = stream ? cudaMallocAsync(&arena.base, plan.total, stream) : cudaMalloc(&arena.base, plan.total);
  if (e != cudaSuccess) {
    oom = e == cudaErrorMemoryAllocation;
    arena.base = nullptr;
    cudaGetLastError();
    return std::string("device allocation of ") + std::to_string(plan.total) + " bytes failed: " +
           cudaGetErrorString(e);
  }
  arena.bytes = plan.total;
  arena.stream = stream;
  std::vector<uint8_t> staging(plan.total, 0);
  for (size_t i = 0; i < plan.parts.size(); ++i)
    if (plan.parts[i].second) std::memcpy(staging.data() + plan.offsets[i], plan.parts[i].first, plan.parts[i].second);
  // A pageable-source async copy returns once the bytes are staged.
  e = stream ? cudaMemcpyAsync(arena.base, staging.data(), plan.total, cudaMemcpyHostToDevice, stream)
             : cudaMemcpy(arena.base, staging.data(), plan.total, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return std::string("upload failed: ") + cudaGetErrorString(e);
  return "";
}

template <class T>
const T *dptr(const DeviceArena &a, const ArenaPlan &p, size_t part) {
  return reinterpret_cast<const T *>(static_cast<uint8_t *>(a.base) + p.offsets[part]);
}

struct MipChain {
  std::vector<uint32_t> w, h;
  std::vector<std::vector<float4>> levels;
};

void build_mips(const pt_texture &img, bool srgb, MipChain &out) {
  static float lut[256];
  static bool init = [] {
    for (int i = 0; i < 256; ++i) lut[i] = host_srgb_to_linear((float)i / 255.0f);
    return true;
  }();
  (void)init;
  size_t n = (size_t)img.width * img.height;
  std::vector<float4> l0(n);
  if (img.format == PT_PIXELS_RGBA8) {
    const uint8_t *p = (const uint8_t *)img.pixels;
    for (size_t i = 0; i < n; ++i) {
      auto c = [&](uint8_t v) { return srgb ? lut[v] : (float)v / 255.0f; };
      l0[i] = make_float4(c(p[4 * i]), c(p[4 * i + 1]), c(p[4 * i + 2]), (float)p[4 * i + 3] / 255.0f);
    }
  } else {
    const float *p = (const float *)img.pixels;
    for (size_t i = 0; i < n; ++i) l0[i] = make_float4(p[4 * i], p[4 * i + 1], p[4 * i + 2], p[4 * i + 3]);
  }
  out.w.push_back(img.width);
  out.h.push_back(img.height);
  out.levels.push_back(std::move(l0));
  for (;;) {
    uint32_t pw = out.w.back(), ph = out.h.back();
    if (pw == 1 && ph == 1) break;
    uint32_t w = std::max(pw / 2, 1u), h = std::max(ph / 2, 1u);
    const std::vector<float4> &prev = out.levels.back();
    std::vector<float4> nx((size_t)w * h);
    for (uint32_t y = 0; y < h; ++y)
      for (uint32_t x = 0; x < w; ++x) {
        size_t x0 = std::min(2 * x, pw - 1), x1 = std::min(2 * x + 1, pw - 1);
        size_t y0 = std::min(2 * y, ph - 1), y1 = std::min(2 * y + 1, ph - 1);
        const float4 *q[4] = {&prev[y0 * pw + x0], &prev[y0 * pw + x1], &prev[y1 * pw + x0], &prev[y1 * pw + x1]};
        float acc[4] = {0, 0, 0, 0};
        for (const float4 *t : q) {
          acc[0] += t->x;
          acc[1] += t->y;
          acc[2] += t->z;
          acc[3] += t->w;
        }
        nx[(size_t)y * w + x] = make_float4(acc[0] * 0.25f, acc[1] * 0.25f, acc[2] * 0.25f, acc[3] * 0.25f);
      }
    out.w.push_back(w);
    out.h.push_back(h);
    out.levels.push_back(std::move(nx));
  }
}

}  // namespace

// ============================================================ scene upload
uint8_t *HostStaging::reserve(size_t bytes) {
  if (bytes > kMaxStagingBytes) return nullptr;
  if (bytes <= cap) return p;
  release();
  size_t want = std::max(bytes, std::min(kMaxStagingBytes, cap * 2));
  void *q = nullptr;
  if (cudaHostAlloc(&q, want, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  p = static_cast<uint8_t *>(q);
  cap = want;
  return p;
}

void HostStaging::release() {
  if (p) cudaFreeHost(p);
  p = nullptr;
  cap = 0;
}

std::string build_scene_image(const pt_scene_desc &desc, SceneImage &img, bool with_bvh, HostStaging *staging,
                              bool spatial) {
  using clk = std::chrono::steady_clock;
  const auto t_start = clk::now();
  auto since = [](clk::time_point a) { return std::chrono::duration<double>(clk::now() - a).count(); };
  if (desc.item_count && !desc.items) return "pt_scene_desc.items is NULL";
  if (desc.material_count == 0 || !desc.materials) return "pt_scene_desc needs at least one material";
  if (desc.texture_count && !desc.textures) return "pt_scene_desc.textures is NULL";
  if (desc.light_count && !desc.lights) return "pt_scene_desc.lights is NULL";
  uint64_t T = 0;
  for (uint32_t i = 0; i < desc.item_count; ++i) {
    const pt_draw_item &it = desc.items[i];
    if (it.triangle_count && !it.positions) return "item " + std::to_string(i) + " has no positions";
    if (it.material >= desc.material_count) return "item " + std::to_string(i) + " material index out of range";
    T += it.triangle_count;
  }
  if (T >= (1ull << 27)) return "scene has " + std::to_string(T) + " triangles; the limit is 134217727";
  const uint32_t tc = (uint32_t)T;

  // Textures: each chain's level sizes and texel offsets in the pool (the
  // pool itself is generated on the device from the source texels).
  std::vector<DevTexture> texs(desc.texture_count);
  std::vector<bool> tex_ok(desc.texture_count, false);
  uint64_t pool_texels = 0, src_bytes = 0;
  for (uint32_t i = 0; i < desc.texture_count; ++i) {
    const pt_texture &t = desc.textures[i];
    DevTexture &d = texs[i];
    std::memset(&d, 0, sizeof d);
    if (!t.pixels || t.width == 0 || t.height == 0) continue;
    if (t.format > PT_PIXELS_RGBA_F32) return "texture " + std::to_string(i) + " has an unknown pixel format";
    if (mip_levels(t.width, t.height) > (uint32_t)kMaxMipLevels) return "texture " + std::to_string(i) + " is too large";
    d.img_w = t.width;
    d.img_h = t.height;
    d.levels = mip_levels(t.width, t.height, d.lw, d.lh, kMaxMipLevels);
    d.mag = t.mag_filter;
    d.min = t.min_filter;
    d.wrap_s = t.wrap_s;
    d.wrap_t = t.wrap_t;
    for (uint32_t k = 0; k < d.levels; ++k) {
      const uint64_t n = (uint64_t)d.lw[k] * d.lh[k];
      d.srgb_off[k] = pool_texels;
      d.lin_off[k] = pool_texels + n;
      pool_texels += 2 * n;
    }
    d.src_format = t.format;
    d.src_off = src_bytes;
    src_bytes += ((uint64_t)t.width * t.height * (t.format == PT_PIXELS_RGBA8 ? 4 : 16) + 15) & ~uint64_t(15);
    tex_ok[i] = true;
  }
  auto fix_binding = [&](pt_texture_binding &b) {
    if (b.texture >= 0 && ((uint32_t)b.texture >= desc.texture_count || !tex_ok[b.texture])) b.texture = -1;
  };

  // Materials.
  std::vector<DevMaterial> mats(desc.material_count);
  for (uint32_t m = 0; m < desc.material_count; ++m) {
    DevMaterial &dm = mats[m];
    std::memset(&dm, 0, sizeof dm);
    dm.m = desc.materials[m];
    pt_texture_binding *bs[] = {&dm.m.base_color_texture, &dm.m.metallic_roughness_texture, &dm.m.normal_texture,
                                &dm.m.occlusion_texture, &dm.m.emissive_texture, &dm.m.specular_texture,
                                &dm.m.specular_color_texture, &dm.m.transmission_texture, &dm.m.thickness_texture,
                                &dm.m.clearcoat_texture, &dm.m.clearcoat_roughness_texture,
                                &dm.m.clearcoat_normal_texture, &dm.m.sheen_color_texture,
                                &dm.m.sheen_roughness_texture, &dm.m.anisotropy_texture, &dm.m.iridescence_texture,
                                &dm.m.iridescence_thickness_texture, &dm.m.diffuse_transmission_texture,
                                &dm.m.diffuse_transmission_color_texture};
    for (pt_texture_binding *b : bs) fix_binding(*b);
    float rot = std::isfinite(dm.m.anisotropy_rotation) ? dm.m.anisotropy_rotation : 0.0f;
    dm.aniso_sin = std::sin(rot);
    dm.aniso_cos = std::cos(rot);
    dm.emissive_nonblack = (dm.m.emissive[0] > 0.0f || dm.m.emissive[1] > 0.0f || dm.m.emissive[2] > 0.0f) ? 1u : 0u;
  }

  // Which optional corner streams the scene has, and each item's first
  // global triangle id.
  bool any_vn = false, any_tan = false, any_col = false, any_uv[PT_MAX_UV_SETS] = {false, false, false, false};
  std::vector<uint64_t> first_tri(desc.item_count + 1, 0);
  for (uint32_t i = 0; i < desc.item_count; ++i) {
    const pt_draw_item &it = desc.items[i];
    any_vn |= it.normals != nullptr;
    any_tan |= it.tangents != nullptr;
    any_col |= it.colors != nullptr;
    for (int s = 0; s < PT_MAX_UV_SETS; ++s) any_uv[s] |= it.uvs[s] != nullptr;
    first_tri[i + 1] = first_tri[i] + it.triangle_count;
  }

  // Lights.
  std::vector<DevLight> lights(desc.light_count);
  for (uint32_t j = 0; j < desc.light_count; ++j) {
    lights[j].l = desc.lights[j];
    lights[j].cos_outer = std::cos(desc.lights[j].outer_cone_angle);
    lights[j].cos_inner = std::cos(desc.lights[j].inner_cone_angle);
  }

  // EmissiveLights::build: the mean emitted radiance of each material, then
  // every emitting triangle of positive area (read from the items' own
  // position arrays) in global id order.
  // An emissive texture's mean is its 1x1 colour level, built here on the
  // host for the textures bound as emission (the same texels the device
  // chain holds).
  std::vector<float> mean_e(3 * (size_t)desc.material_count);
  std::vector<float4> tex_mean(desc.texture_count);
  std::vector<bool> have_mean(desc.texture_count, false);
  for (uint32_t m = 0; m < desc.material_count; ++m) {
    const pt_material &mt = mats[m].m;
    float e[3] = {0.0f, 0.0f, 0.0f};
    if (!mt.unlit) {
      e[0] = mt.emissive[0];
      e[1] = mt.emissive[1];
      e[2] = mt.emissive[2];
      int ti = mt.emissive_texture.texture;
      if (ti >= 0) {
        if (!have_mean[ti]) {
          MipChain s;
          build_mips(desc.textures[ti], true, s);
          tex_mean[ti] = s.levels.back()[0];
          have_mean[ti] = true;
        }
        const float4 &c = tex_mean[ti];
        e[0] = e[0] * c.x;
        e[1] = e[1] * c.y;
        e[2] = e[2] * c.z;
      }
    }
    std::memcpy(&mean_e[3 * m], e, sizeof e);
  }
  std::vector<uint32_t> em_tris;
  std::vector<float> power;
  for (uint32_t i = 0; i < desc.item_count; ++i) {
    const pt_draw_item &it = desc.items[i];
    const float *e = &mean_e[3 * (size_t)it.material];
    float lum = 0.2126f * e[0] + 0.7152f * e[1] + 0.0722f * e[2];
    if (std::isnan(lum) || lum <= 0.0f) continue;
    const float sides = mats[it.material].m.double_sided ? 2.0f : 1.0f;
    for (uint64_t t = 0; t < it.triangle_count; ++t) {
      const float *p = it.positions + 9 * t;
      float e1[3] = {p[3] - p[0], p[4] - p[1], p[5] - p[2]}, e2[3] = {p[6] - p[0], p[7] - p[1], p[8] - p[2]};
      float cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
      float ar = 0.5f * std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
      if (std::isnan(ar) || ar <= 0.0f || !std::isfinite(ar)) continue;
      em_tris.push_back((uint32_t)(first_tri[i] + t));
      power.push_back(ar * lum * sides);
    }
  }
  double total_power = 0.0;
  for (float p : power) total_power += (double)p;
  std::vector<float> pmf, cdf;
  double acc = 0.0;
  for (float pw : power) {
    pmf.push_back((float)((double)pw / total_power));
    acc += (double)pw / total_power;
    cdf.push_back((float)acc);
  }
  if (!cdf.empty()) cdf.back() = 1.0f;
  img.seconds[1] = since(t_start);

  // The arena plan: every part's offset (256-byte aligned) from its size.
  struct Plan {
    std::vector<size_t> off, bytes;
    size_t total = 0;
    size_t add(size_t b) {
      size_t o = (total + 255) & ~(size_t)255;
      off.push_back(o);
      bytes.push_back(b);
      total = o + b;
      return off.size() - 1;
    }
  } plan;
  const size_t p_info = plan.add(T * sizeof(uint2));
  const size_t p_pos = plan.add(T * 36);
  const size_t p_nrm = plan.add(any_vn ? T * 36 : 0);
  const size_t p_tan = plan.add(any_tan ? T * 48 : 0);
  const size_t p_col = plan.add(any_col ? T * 48 : 0);
  size_t p_uv[PT_MAX_UV_SETS];
  for (int s = 0; s < PT_MAX_UV_SETS; ++s) p_uv[s] = plan.add(any_uv[s] ? T * 24 : 0);
  const size_t p_mat = plan.add(mats.size() * sizeof(DevMaterial));
  const size_t p_tex = plan.add(texs.size() * sizeof(DevTexture));
  const size_t p_src = plan.add(src_bytes);
  const size_t p_lights = plan.add(lights.size() * sizeof(DevLight));
  const size_t p_emt = plan.add(em_tris.size() * 4);
  const size_t p_pmf = plan.add(pmf.size() * 4);
  const size_t p_cdf = plan.add(cdf.size() * 4);
  const size_t p_lookup = plan.add(T * 4);
  const size_t p_desc = plan.add(sizeof(DevScene));
  // The texel pool comes last and exists on the device only: the host
  // image ends where it starts.
  const size_t p_pool = plan.add(pool_texels * sizeof(float4));
  const size_t total = std::max<size_t>(plan.off[p_pool], 256);
  const auto t_fill = clk::now();
  const int threads = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  if (uint8_t *pinned = staging ? staging->reserve(total) : nullptr)
    img.blob.use(pinned, total);
  else
    img.blob.allocate(total);
  uint8_t *const dst = img.blob.data();
  std::vector<uint32_t> rec_flags(T);

  // Fill: every byte of the blob is written once, by tasks spread over
  // threads (copies in slices of at most 16 MiB, first touch included).
  std::vector<std::function<void()>> tasks;
  const size_t kSlice = size_t(16) << 20;
  auto copy_task = [&](size_t off, const void *src, size_t bytes) {
    for (size_t o = 0; o < bytes; o += kSlice) {
      const size_t b = std::min(kSlice, bytes - o);
      const uint8_t *s = src ? static_cast<const uint8_t *>(src) + o : nullptr;
      tasks.push_back([dst, off, o, s, b] {
        if (s)
          std::memcpy(dst + off + o, s, b);
        else
          std::memset(dst + off + o, 0, b);
      });
    }
  };
  {
    size_t cursor = 0;  // zero the alignment gaps and the tail
    for (size_t k = 0; k < p_pool; ++k) {
      if (plan.off[k] > cursor) copy_task(cursor, nullptr, plan.off[k] - cursor);
      cursor = plan.off[k] + plan.bytes[k];
    }
    if (total > cursor) copy_task(cursor, nullptr, total - cursor);
  }
  copy_task(plan.off[p_mat], mats.data(), plan.bytes[p_mat]);
  copy_task(plan.off[p_tex], texs.data(), plan.bytes[p_tex]);
  for (uint32_t i = 0; i < desc.texture_count; ++i)
    if (tex_ok[i]) {
      const pt_texture &tx = desc.textures[i];
      const size_t b = (size_t)tx.width * tx.height * (tx.format == PT_PIXELS_RGBA8 ? 4 : 16);
      copy_task(plan.off[p_src] + texs[i].src_off, tx.pixels, b);
    }
  copy_task(plan.off[p_lights], lights.data(), plan.bytes[p_lights]);
  copy_task(plan.off[p_emt], em_tris.data(), plan.bytes[p_emt]);
  copy_task(plan.off[p_pmf], pmf.data(), plan.bytes[p_pmf]);
  copy_task(plan.off[p_cdf], cdf.data(), plan.bytes[p_cdf]);
  copy_task(plan.off[p_desc], nullptr, plan.bytes[p_desc]);
  // Corner streams by global triangle id: each item's array, or zeros for
  // an item without it.
  for (uint32_t i = 0; i < desc.item_count; ++i) {
    const pt_draw_item &it = desc.items[i];
    const size_t g0 = first_tri[i], n = it.triangle_count;
    copy_task(plan.off[p_pos] + 36 * g0, it.positions, 36 * n);
    // Every item's corner normals (face normals when it has no vertex
    // normals: the raycast backend shades with them); TRI_HAS_VN tells the
    // path tracer which are vertex normals.
    if (any_vn) copy_task(plan.off[p_nrm] + 36 * g0, it.normals, 36 * n);
    if (any_tan) copy_task(plan.off[p_tan] + 48 * g0, it.tangents, 48 * n);
    if (any_col) copy_task(plan.off[p_col] + 48 * g0, it.colors, 48 * n);
    for (int s = 0; s < PT_MAX_UV_SETS; ++s)
      if (any_uv[s]) copy_task(plan.off[p_uv[s]] + 24 * g0, it.uvs[s], 24 * n);
    // (material, attribute flags) and the record flags of its triangles.
    uint32_t flags = 0;
    if (it.normals && it.has_vertex_normals) flags |= TRI_HAS_VN;
    if (it.tangents) flags |= TRI_HAS_TANGENTS;
    if (it.colors) flags |= TRI_HAS_COLORS;
    for (int s = 0; s < PT_MAX_UV_SETS; ++s)
      if (it.uvs[s]) flags |= TRI_UV0 << s;
    const pt_material &mm = desc.materials[it.material];
    const uint32_t rf = (mm.alpha_mode == PT_ALPHA_OPAQUE ? REC_OPAQUE : 0u) | (mm.double_sided ? REC_DOUBLE_SIDED : 0u);
    const uint2 inf = make_uint2(it.material, flags);
    uint2 *info = reinterpret_cast<uint2 *>(dst + plan.off[p_info]);
    uint32_t *rec = rec_flags.data();
    const size_t kTris = size_t(1) << 20;
    for (size_t a = 0; a < n; a += kTris) {
      const size_t b = std::min(n, a + kTris);
      tasks.push_back([info, rec, inf, rf, g0, a, b] {
        for (size_t t = a; t < b; ++t) {
          info[g0 + t] = inf;
          rec[g0 + t] = rf;
        }
      });
    }
  }
  // Emissive lookup by global id: "none" everywhere, then the emitters.
  {
    uint32_t *lookup = reinterpret_cast<uint32_t *>(dst + plan.off[p_lookup]);
    const size_t kTris = size_t(4) << 20;
    for (size_t a = 0; a < T; a += kTris) {
      const size_t b = std::min(T, a + kTris);
      tasks.push_back([lookup, a, b] { std::fill(lookup + a, lookup + b, 0xffffffffu); });
    }
  }
  {
    std::atomic<size_t> next{0};
    auto work = [&] {
      for (size_t k; (k = next.fetch_add(1)) < tasks.size();) tasks[k]();
    };
    const int nt = (int)std::min<size_t>(tasks.size(), (size_t)threads);
    std::vector<std::thread> pool_threads;
    for (int k = 1; k < nt; ++k) pool_threads.emplace_back(work);
    work();
    for (auto &th : pool_threads) th.join();
  }
  {
    uint32_t *lookup = reinterpret_cast<uint32_t *>(dst + plan.off[p_lookup]);
    for (size_t k = 0; k < em_tris.size(); ++k) lookup[em_tris[k]] = (uint32_t)k;
  }
  img.seconds[3] = since(t_fill);

  // BVH (host build) from the positions now in the blob.
  const auto t_bvh = clk::now();
  const float *pos = reinterpret_cast<const float *>(dst + plan.off[p_pos]);
  if (with_bvh && spatial)
    build_bvh_spatial(pos, tc, rec_flags.data(), img.tree.nodes, img.tree.nodes4, img.tree.records, img.bvh, threads);
  else if (with_bvh)
    build_bvh(pos, tc, rec_flags.data(), img.tree.nodes, img.tree.nodes4, img.tree.records, img.bvh, threads);
  img.seconds[2] = since(t_bvh);
  img.textures = texs;
  img.tex_src_off = plan.off[p_src];
  img.pool_off = plan.off[p_pool];
  img.pool_bytes = plan.bytes[p_pool];

  // Pointer fields hold offset + 1 until commit_scene rebases them; the
  // tree's are set when it is committed.
  auto rel = [&](size_t part, size_t bytes) -> uintptr_t { return bytes ? (uintptr_t)plan.off[part] + 1 : 0; };
  DevScene &d = img.rel;
  std::memset(&d, 0, sizeof d);
  d.tri_info = (const uint2 *)rel(p_info, 1);
  d.pos = (const float *)rel(p_pos, 1);
  d.nrm = (const float *)rel(p_nrm, plan.bytes[p_nrm]);
  d.tan = (const float *)rel(p_tan, plan.bytes[p_tan]);
  d.col = (const float *)rel(p_col, plan.bytes[p_col]);
  for (int s = 0; s < PT_MAX_UV_SETS; ++s) d.uv[s] = (const float *)rel(p_uv[s], plan.bytes[p_uv[s]]);
  d.materials = (const DevMaterial *)rel(p_mat, 1);
  d.textures = (const DevTexture *)rel(p_tex, 1);
  d.texels = (const float4 *)rel(p_pool, 1);
  d.lights = (const DevLight *)rel(p_lights, 1);
  d.em_tris = (const uint32_t *)rel(p_emt, 1);
  d.em_pmf = (const float *)rel(p_pmf, 1);
  d.em_cdf = (const float *)rel(p_cdf, 1);
  d.em_lookup = (const uint32_t *)rel(p_lookup, 1);
  d.tri_count = tc;
  d.material_count = desc.material_count;
  d.texture_count = desc.texture_count;
  d.light_count = desc.light_count;
  d.em_count = (uint32_t)em_tris.size();
  img.desc_off = plan.off[p_desc];
  img.tri_count = tc;
  img.light_count = desc.light_count;
  img.seconds[0] = since(t_start);
  return "";
}

uint64_t HostTree::bytes() const {
  auto al = [](uint64_t x) { return (x + 255) & ~uint64_t(255); };
  return al(nodes.size() * sizeof(BvhNode)) + al(nodes4.size() * sizeof(Bvh4Node)) + al(records.size() * sizeof(float4));
}

namespace {

template <class P>
void rebase(const P *&p, uint8_t *base) {
  p = p ? reinterpret_cast<const P *>(base + (reinterpret_cast<uintptr_t>(p) - 1)) : nullptr;
}

// Allocates `a` for `t` and copies it (stream-ordered when `stream` is
// non-null), pointing d's tree fields into it.
std::string commit_tree(const HostTree &t, uint32_t max_depth, DeviceArena &a, DevScene &d, bool &oom,
                        cudaStream_t stream) {
  auto al = [](uint64_t x) { return (x + 255) & ~uint64_t(255); };
  const uint64_t b2 = t.nodes.size() * sizeof(BvhNode), b4 = t.nodes4.size() * sizeof(Bvh4Node);
  const uint64_t br = t.records.size() * sizeof(float4);
  const uint64_t off4 = al(b2), offr = off4 + al(b4), total = std::max<uint64_t>(offr + al(br), 256);
  cudaError_t e = stream ? cudaMallocAsync(&a.base, total, stream) : cudaMalloc(&a.base, total);
  if (e != cudaSuccess) {
    oom = e == cudaErrorMemoryAllocation;
    a.base = nullptr;
    cudaGetLastError();
    return std::string("device allocation of ") + std::to_string(total) + " BVH bytes failed: " + cudaGetErrorString(e);
  }
  a.bytes = total;
  a.stream = stream;
  uint8_t *base = static_cast<uint8_t *>(a.base);
  const void *src[3] = {t.nodes.data(), t.nodes4.data(), t.records.data()};
  const uint64_t off[3] = {0, off4, offr}, len[3] = {b2, b4, br};
  for (int k = 0; k < 3 && e == cudaSuccess; ++k)
    if (len[k])
      e = stream ? cudaMemcpyAsync(base + off[k], src[k], len[k], cudaMemcpyHostToDevice, stream)
                 : cudaMemcpy(base + off[k], src[k], len[k], cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    a.release();
    return std::string("BVH upload failed: ") + cudaGetErrorString(e);
  }
  d.nodes = t.nodes.empty() ? nullptr : reinterpret_cast<const BvhNode *>(base);
  d.nodes4 = t.nodes4.empty() ? nullptr : reinterpret_cast<const Bvh4Node *>(base + off4);
  d.tris = reinterpret_cast<const float4 *>(base + offr);
  d.node_count = (uint32_t)t.nodes.size();
  d.node4_count = (uint32_t)t.nodes4.size();
  d.max_depth = max_depth;
  return "";
}

}  // namespace

std::string commit_scene(const SceneImage &img, SceneHost &out, bool &oom, cudaStream_t stream) {
  oom = false;
  const size_t total = std::max<uint64_t>(img.blob.size(), img.pool_off + img.pool_bytes);
  cudaError_t e = stream ? cudaMallocAsync(&out.arena.base, total, stream) : cudaMalloc(&out.arena.base, total);
  if (e != cudaSuccess) {
    oom = e == cudaErrorMemoryAllocation;
    out.arena.base = nullptr;
    cudaGetLastError();
    return std::string("device allocation of ") + std::to_string(total) + " bytes failed: " + cudaGetErrorString(e);
  }
  out.arena.bytes = total;
  out.arena.stream = stream;
  uint8_t *base = static_cast<uint8_t *>(out.arena.base);
  DevScene d = img.rel;
  rebase(d.tri_info, base);
  rebase(d.pos, base);
  rebase(d.nrm, base);
  rebase(d.tan, base);
  rebase(d.col, base);
  for (int s = 0; s < PT_MAX_UV_SETS; ++s) rebase(d.uv[s], base);
  rebase(d.materials, base);
  rebase(d.textures, base);
  rebase(d.texels, base);
  rebase(d.lights, base);
  rebase(d.em_tris, base);
  rebase(d.em_pmf, base);
  rebase(d.em_cdf, base);
  rebase(d.em_lookup, base);
  out.d_desc = reinterpret_cast<DevScene *>(base + img.desc_off);
  // Pageable sources: the copies return once the bytes are staged, and run
  // in the stream's order (before any later wave).
  e = stream ? cudaMemcpyAsync(base, img.blob.data(), img.blob.size(), cudaMemcpyHostToDevice, stream)
             : cudaMemcpy(base, img.blob.data(), img.blob.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    out.arena.release();
    return std::string("scene upload failed: ") + cudaGetErrorString(e);
  }
  if (img.pool_bytes) {
    static float decode[256];
    static bool init = [] {
      for (int i = 0; i < 256; ++i) decode[i] = host_srgb_to_linear((float)i / 255.0f);
      return true;
    }();
    (void)init;
    std::string err = device_build_mips(img.textures, d.textures, base + img.tex_src_off,
                                        reinterpret_cast<float4 *>(base + img.pool_off), decode, stream);
    // Without a stream the commit is synchronous: the chains are done when
    // it returns (later work may run on any stream).
    if (err.empty() && !stream && cudaStreamSynchronize(nullptr) != cudaSuccess)
      err = std::string("mip generation failed: ") + cudaGetErrorString(cudaGetLastError());
    if (!err.empty()) {
      out.arena.release();
      return err;
    }
  }
  if (!img.tree.nodes.empty()) {
    std::string err = commit_tree(img.tree, img.bvh.max_depth, out.bvh_arena, d, oom, stream);
    if (!err.empty()) {
      out.arena.release();
      return err;
    }
  }
  e = stream ? cudaMemcpyAsync(out.d_desc, &d, sizeof(DevScene), cudaMemcpyHostToDevice, stream)
             : cudaMemcpy(out.d_desc, &d, sizeof(DevScene), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    out.arena.release();
    out.bvh_arena.release();
    return std::string("scene upload failed: ") + cudaGetErrorString(e);
  }
  out.dev = d;
  out.tri_count = img.tri_count;
  out.pool_texels = img.pool_bytes / sizeof(float4);
  out.bvh = img.bvh;
  out.light_count = img.light_count;
  return "";
}

std::string upload_scene(const pt_scene_desc &desc, SceneHost &out, bool &oom, int builder, cudaStream_t stream,
                         HostStaging *staging) {
  oom = false;
  out.item_tris.clear();
  for (uint32_t i = 0; desc.items && i < desc.item_count; ++i) out.item_tris.push_back(desc.items[i].triangle_count);
  using clk = std::chrono::steady_clock;
  const auto t0 = clk::now();
  auto secs = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
  uint64_t tris = 0;
  for (uint32_t i = 0; desc.items && i < desc.item_count; ++i) tris += desc.items[i].triangle_count;
  const bool device = builder == BVH_BUILD_DEVICE || builder == BVH_BUILD_DEVICE_PLOC ||
                      (builder == BVH_BUILD_AUTO && tris >= kAutoDeviceBuildTris);
  if (device && tris >= 64) {
    SceneImage img;
    std::string err = build_scene_image(desc, img, false, staging);
    if (!err.empty()) return err;
    const auto t1 = clk::now();
    err = commit_scene(img, out, oom);
    if (!err.empty()) return err;
    const auto t2 = clk::now();
    err = builder == BVH_BUILD_DEVICE_PLOC ? device_build_bvh(out, stream, kMaxTreeDepth, oom)
                                           : device_build_bvh_sah(out, stream, kMaxTreeDepth, oom);
    if (err.empty()) {
      const auto t3 = clk::now();
      out.upload_seconds[0] = secs(t0, t1);
      out.upload_seconds[1] = secs(t1, t2);
      out.upload_seconds[2] = secs(t2, t3);
      out.upload_seconds[3] = secs(t0, t3);
      out.device_bvh = true;
      return "";
    }
    release_scene(out);
    if (err.rfind("depth", 0) != 0) return err;
    oom = false;
  }
  SceneImage img;
  const auto t1 = clk::now();
  std::string err = build_scene_image(desc, img, true, nullptr, builder == BVH_BUILD_HOST_SPATIAL);
  if (!err.empty()) return err;
  const auto t2 = clk::now();
  err = commit_scene(img, out, oom);
  const auto t3 = clk::now();
  out.upload_seconds[0] = secs(t1, t2);
  out.upload_seconds[1] = secs(t2, t3);
  out.upload_seconds[2] = 0.0;
  out.upload_seconds[3] = secs(t0, t3);
  return err;
}

std::string refit_scene(const pt_scene_desc &desc, SceneHost &sc, bool &oom, cudaStream_t stream,
                        HostStaging *staging) {
  oom = false;
  using clk = std::chrono::steady_clock;
  auto secs = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
  const auto t0 = clk::now();
  std::vector<uint32_t> tris;
  for (uint32_t i = 0; desc.items && i < desc.item_count; ++i) tris.push_back(desc.items[i].triangle_count);
  if (tris != sc.item_tris)
    return "refit needs the same draw items with the same triangle counts (upload the scene instead)";
  SceneImage img;
  std::string err = build_scene_image(desc, img, false, staging);
  if (!err.empty()) return err;
  const auto t1 = clk::now();
  SceneHost fresh;
  err = commit_scene(img, fresh, oom, stream);
  if (!err.empty()) return err;
  const auto t2 = clk::now();
  // The old tree, refitted to the new positions, goes with the new arena.
  fresh.bvh_arena = sc.bvh_arena;
  fresh.dev.nodes = sc.dev.nodes;
  fresh.dev.nodes4 = sc.dev.nodes4;
  fresh.dev.tris = sc.dev.tris;
  fresh.dev.node_count = sc.dev.node_count;
  fresh.dev.node4_count = sc.dev.node4_count;
  fresh.dev.max_depth = sc.dev.max_depth;
  fresh.bvh = sc.bvh;
  fresh.device_bvh = sc.device_bvh;
  fresh.item_tris = sc.item_tris;
  err = device_refit_bvh(fresh, sc.bvh.references, stream);
  cudaError_t e = cudaSuccess;
  if (err.empty()) e = cudaMemcpyAsync(fresh.d_desc, &fresh.dev, sizeof(DevScene), cudaMemcpyHostToDevice, stream);
  if (err.empty() && e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (err.empty() && e != cudaSuccess) err = std::string("refit: ") + cudaGetErrorString(e);
  if (!err.empty()) {
    // The tree stays with the old scene, which is still whole.
    fresh.bvh_arena = DeviceArena{};
    fresh.arena.release();
    return err;
  }
  sc.arena.release();
  sc.bvh_arena = DeviceArena{};
  const auto t3 = clk::now();
  fresh.upload_seconds[0] = secs(t0, t1);
  fresh.upload_seconds[1] = secs(t1, t2);
  fresh.upload_seconds[2] = secs(t2, t3);
  fresh.upload_seconds[3] = secs(t0, t3);
  sc = std::move(fresh);
  return "";
}

void release_scene(SceneHost &s) {
  s.arena.release();
  s.bvh_arena.release();
  s.d_desc = nullptr;
  s.device_bvh = false;
}

// ============================================================ environment
std::string upload_env(const pt_environment &env, EnvHost &out, bool &oom, cudaStream_t stream) {
  oom = false;
  const float PI = 3.14159265358979323846f;
  uint32_t w = std::max(env.width, 1u), h = std::max(env.height, 1u);
  bool valid = env.pixels != nullptr && env.width > 0 && env.height > 0;
  std::vector<float4> px;
  if (valid) {
    px.resize((size_t)w * h);
    std::memcpy(px.data(), env.pixels, px.size() * sizeof(float4));
  }
  std::vector<double> weights((size_t)w * h, 0.0);
  if (valid)
    for (uint32_t y = 0; y < h; ++y) {
      double st = (double)std::sin(PI * ((float)y + 0.5f) / (float)h);
      for (uint32_t x = 0; x < w; ++x) {
        const float4 &c = px[(size_t)y * w + x];
        float l = 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z;
        weights[(size_t)y * w + x] = (std::isfinite(l) && l > 0.0f) ? (double)l * st : 0.0;
      }
    }
  double total = 0.0;
  for (double x : weights) total += x;
  bool uniform = !(total > 0.0 && std::isfinite(total));
  if (uniform)
    for (size_t i = 0; i < weights.size(); ++i)
      weights[i] = (double)std::sin(PI * ((float)(i / w) + 0.5f) / (float)h);
  total = 0.0;
  for (double x : weights) total += x;
  std::vector<float> marginal, conditional, mass(weights.size());
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
  for (size_t i = 0; i < weights.size(); ++i) mass[i] = (float)(weights[i] / total);

  ArenaPlan plan;
  size_t p_px = plan.add(px.data(), px.size() * sizeof(float4));
  size_t p_m = plan.add(marginal.data(), marginal.size() * 4);
  size_t p_c = plan.add(conditional.data(), conditional.size() * 4);
  size_t p_mass = plan.add(mass.data(), mass.size() * 4);
  DevEnv tmp{};
  size_t p_desc = plan.add(&tmp, sizeof(DevEnv));
  std::string err = commit(plan, out.arena, oom, stream);
  if (!err.empty()) {
    out.arena.release();
    return err;
  }
  DevEnv &d = out.dev;
  d.w = w;
  d.h = h;
  d.uniform = uniform ? 1u : 0u;
  d.intensity = std::isfinite(env.intensity) ? std::fmax(env.intensity, 0.0f) : 0.0f;
  d.pixels = valid ? dptr<float4>(out.arena, plan, p_px) : nullptr;
  d.marginal = dptr<float>(out.arena, plan, p_m);
  d.conditional = dptr<float>(out.arena, plan, p_c);
  d.mass = dptr<float>(out.arena, plan, p_mass);
  out.d_desc = const_cast<DevEnv *>(dptr<DevEnv>(out.arena, plan, p_desc));
  cudaError_t e = stream ? cudaMemcpyAsync(out.d_desc, &d, sizeof(DevEnv), cudaMemcpyHostToDevice, stream)
                         : cudaMemcpy(out.d_desc, &d, sizeof(DevEnv), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    out.arena.release();
    return std::string("environment upload failed: ") + cudaGetErrorString(e);
  }
  return "";
}

void release_env(EnvHost &e) {
  e.arena.release();
  e.d_desc = nullptr;
}

}  // namespace ptd
