// Persistent-thread traversal for the wavefront's extend and shadow kernels.
//
// Each lane owns one ray at a time and asks for the next queue entry the
// moment its ray finishes (one warp-aggregated atomic per refill), so the
// lanes of a warp stay busy instead of idling behind the warp's slowest ray
// (Aila & Laine, "Understanding the Efficiency of Ray Traversal on GPUs",
// HPG 2009: persistent threads with dynamic fetch) and the warp alternates a
// speculative node phase with a leaf phase (their while-while traversal
// with postponed leaves), so lanes rarely idle behind each other; the node
// phase does not wait for its last few searching lanes
// (node_phase_goes_on).
//
// The traversal stack keeps its top entries in shared memory (one column
// per thread, conflict-free) and spills deeper entries to local memory.
// Rays walk either node layout of the scene: two-child 64-byte nodes or the
// same tree as four-child 128-byte nodes (fewer, wider steps).
//
// Results equal closest_hit / occluded of dev_scene.cuh: the closest hit is
// the accepted candidate with the smallest t (ties: lowest global id), a
// definition that does not depend on traversal order, and the any-hit
// answer is a yes/no.
#pragma once

#include "dev_scene.cuh"

namespace ptd {

// Shared-memory entries per thread. Eight keep the blocks' shared memory
// small, which leaves more of the SM's L1 to node and triangle data; the
// request mix traced 1 % faster than with 16 (24: no change).
constexpr int kShortStack = 8;
constexpr int kTravDone = kEmptyChild;  // "no next node" (never a node index)
// A four-child node pushes at most three entries per level and the builder
// keeps the binary tree (hence the four-child tree) at most 56 levels deep.
constexpr int kTravStackSize = 3 * 56 + 8;

struct TravStack {
  int *sm;        // this thread's column: entry i at sm[i * stride]
  int stride;
  int spill[kTravStackSize - kShortStack];
  PT_DEV void push(int &sp, int v, uint32_t &err) {
    if (sp < kShortStack)
      sm[sp * stride] = v;
    else if (sp < kTravStackSize)
      spill[sp - kShortStack] = v;
    else {
      err |= ERR_STACK_OVERFLOW;
      return;
    }
    ++sp;
  }
  // Callers pop only a non-empty stack; an empty one reads as "done".
  PT_DEV int pop(int &sp) {
    if (sp <= 0) return kTravDone;
    --sp;
    return sp < kShortStack ? sm[sp * stride] : spill[sp - kShortStack];
  }
};

// Slab test of one child box against [t0, t1] (the test node_boxes applies).
PT_DEV bool child_box(float lox, float hix, float loy, float hiy, float loz, float hiz, const Ray &r, float t0,
                      float t1, float &entry) {
  const float grow = 1.0000003576f;  // 1 + 2 * gamma(3)
  float lx = (lox - r.o.x) * r.inv.x, hx = (hix - r.o.x) * r.inv.x;
  float ly = (loy - r.o.y) * r.inv.y, hy = (hiy - r.o.y) * r.inv.y;
  float lz = (loz - r.o.z) * r.inv.z, hz = (hiz - r.o.z) * r.inv.z;
  float tn = fmaxf(fmaxf(fminf(lx, hx), fminf(ly, hy)), fmaxf(fminf(lz, hz), t0));
  float tf = fminf(fminf(fmaxf(lx, hx), fmaxf(ly, hy)), fmaxf(lz, hz)) * grow;
  tf = fminf(tf, t1);
  entry = tn;
  return tn <= tf;
}

PT_DEV void cswap(float &ea, int &ca, float &eb, int &cb) {
  if (eb < ea) {
    float te = ea;
    ea = eb;
    eb = te;
    int tc = ca;
    ca = cb;
    cb = tc;
  }
}

// Tests the children of node `cur` and returns the nearest hit child
// (kTravDone when none), pushing the other hit children farthest first.
// Children are ordered by entry distance when `ordered`.
PT_DEV int visit_node2(const DevScene &s, const Ray &r, float t_min, float t_far, int cur, int &sp, TravStack &stk,
                       uint32_t &err, bool ordered) {
  bool h0, h1;
  float e0, e1;
  int4 dd;
  node_boxes(s.nodes + cur, r, t_min, t_far, h0, h1, e0, e1, dd);
  if (h0 && h1) {
    bool swap = ordered && e1 < e0;
    stk.push(sp, swap ? dd.x : dd.y, err);
    return swap ? dd.y : dd.x;
  }
  if (h0) return dd.x;
  if (h1) return dd.y;
  return kTravDone;
}

PT_DEV int visit_node4(const DevScene &s, const Ray &r, float t_min, float t_far, int cur, int &sp, TravStack &stk,
                       uint32_t &err, bool ordered) {
  const Bvh4Node *nd = s.nodes4 + cur;
  const float4 lx = ldg4(&nd->lo_x), hx = ldg4(&nd->hi_x), ly = ldg4(&nd->lo_y), hy = ldg4(&nd->hi_y);
  const float4 lz = ldg4(&nd->lo_z), hz = ldg4(&nd->hi_z);
  const int4 ch = __ldg(&nd->child);
  float e0, e1, e2, e3;
  int c0 = child_box(lx.x, hx.x, ly.x, hy.x, lz.x, hz.x, r, t_min, t_far, e0) && ch.x != kEmptyChild ? ch.x : kTravDone;
  int c1 = child_box(lx.y, hx.y, ly.y, hy.y, lz.y, hz.y, r, t_min, t_far, e1) && ch.y != kEmptyChild ? ch.y : kTravDone;
  int c2 = child_box(lx.z, hx.z, ly.z, hy.z, lz.z, hz.z, r, t_min, t_far, e2) && ch.z != kEmptyChild ? ch.z : kTravDone;
  int c3 = child_box(lx.w, hx.w, ly.w, hy.w, lz.w, hz.w, r, t_min, t_far, e3) && ch.w != kEmptyChild ? ch.w : kTravDone;
  if (ordered) {
    if (c0 == kTravDone) e0 = inf();
    if (c1 == kTravDone) e1 = inf();
    if (c2 == kTravDone) e2 = inf();
    if (c3 == kTravDone) e3 = inf();
    cswap(e0, c0, e1, c1);
    cswap(e2, c2, e3, c3);
    cswap(e0, c0, e2, c2);
    cswap(e1, c1, e3, c3);
    cswap(e1, c1, e2, c2);
  }
  int next = kTravDone;
  if (c3 != kTravDone) next = c3;
  if (c2 != kTravDone) {
    if (next != kTravDone) stk.push(sp, next, err);
    next = c2;
  }
  if (c1 != kTravDone) {
    if (next != kTravDone) stk.push(sp, next, err);
    next = c1;
  }
  if (c0 != kTravDone) {
    if (next != kTravDone) stk.push(sp, next, err);
    next = c0;
  }
  return next;
}

// Traversal position of one ray for speculative while-while traversal
// (Aila & Laine 2009): in a warp's node phase every lane walks nodes; a lane
// that reaches a leaf parks it in `leaf` and keeps walking until it meets a
// second leaf, and the phase lasts while any lane is still looking for its
// first one. The warp then tests the parked leaves together.
struct TravCore {
  Ray r;
  int cur, sp, leaf;
  bool wide;
  PT_DEV void start(const DevScene &s, V3 o, V3 d, bool wide_nodes) {
    r = make_ray(o, d);
    cur = s.node_count ? 0 : kTravDone;
    sp = 0;
    leaf = kTravDone;
    wide = wide_nodes && s.nodes4;
  }
  PT_DEV bool searching() const { return leaf == kTravDone && (cur != kTravDone || sp > 0); }
  // kTravDone is positive: "a node to visit" is cur >= 0 && cur != kTravDone.
  PT_DEV bool can_step() const {
    return leaf == kTravDone ? (cur != kTravDone || sp > 0)
                             : ((cur >= 0 && cur != kTravDone) || (cur == kTravDone && sp > 0));
  }
  PT_DEV bool finished() const { return leaf == kTravDone && cur == kTravDone && sp == 0; }
  // One node-phase step; the caller checks can_step(). kOnly4: the caller
  // knows the ray walks the four-child layout (`wide`), so the two-child
  // visit is not compiled in.
  template <bool kOnly4>
  PT_DEV void node_step(const DevScene &s, float t_min, float t_far, TravStack &stk, uint32_t &nodes,
                        uint32_t &err, bool ordered) {
    if (cur < 0) {  // a leaf met in the previous node phase
      leaf = cur;
      cur = kTravDone;
      return;
    }
    if (cur == kTravDone) {
      cur = stk.pop(sp);
      if (cur == kTravDone) return;
      if (cur < 0) {
        if (leaf == kTravDone) {
          leaf = cur;
          cur = kTravDone;
        }
        return;
      }
    }
    nodes++;
    cur = kOnly4 || wide ? visit_node4(s, r, t_min, t_far, cur, sp, stk, err, ordered)
                         : visit_node2(s, r, t_min, t_far, cur, sp, stk, err, ordered);
    if (cur < 0 && leaf == kTravDone) {
      leaf = cur;
      cur = kTravDone;
    }
  }
  // The parked leaf's triangle records [first, first + count).
  PT_DEV void leaf_range(uint32_t &first, uint32_t &count) const {
    first = (uint32_t)(~leaf);
    count = first >> kLeafCountShift;
    first &= kLeafFirstMask;
  }
};

// Closest-hit state of one ray.
struct ClosestRay {
  TravCore core;
  float t_min, t_max;
  Hit best;
  bool have;
  PT_DEV void init(const DevScene &s, V3 o, V3 d, float tmin, float tmax, bool wide_nodes) {
    core.start(s, o, d, wide_nodes);
    t_min = tmin;
    t_max = tmax;
    best.t = tmax;
    best.g = 0xffffffffu;
    have = false;
  }
  template <bool kOnly4>
  PT_DEV void node_step(const DevScene &s, TravStack &stk, uint32_t &nodes, uint32_t &err) {
    core.node_step<kOnly4>(s, t_min, best.t, stk, nodes, err, true);
  }
  // Tests the parked leaf (if any) and clears it.
  template <class Accept>
  PT_DEV void leaf_step(const DevScene &s, Accept &accept, uint32_t &tris) {
    if (core.leaf == kTravDone) return;
    uint32_t first, count;
    core.leaf_range(first, count);
    core.leaf = kTravDone;
    for (uint32_t i = 0; i < count; ++i) {
      const float4 *tr = s.tris + 3u * (first + i);
      float4 p0 = ldg4(tr), p1 = ldg4(tr + 1), p2 = ldg4(tr + 2);
      tris++;
      float t, b0, b1, b2;
      bool front;
      if (!intersect_watertight(core.r, {p0.x, p0.y, p0.z}, {p1.x, p1.y, p1.z}, {p2.x, p2.y, p2.z}, t, b0, b1, b2,
                                front))
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
};

// Any-hit state of one ray.
struct ShadowTrav {
  TravCore core;
  float t_max;
  bool occluded;
  PT_DEV void init(const DevScene &s, V3 o, V3 d, float tmax, bool wide_nodes) {
    core.start(s, o, d, wide_nodes);
    t_max = tmax;
    occluded = false;
  }
  template <bool kOnly4>
  PT_DEV void node_step(const DevScene &s, TravStack &stk, uint32_t &nodes, uint32_t &err) {
    core.node_step<kOnly4>(s, 0.0f, t_max, stk, nodes, err, false);
  }
  template <class Accept>
  PT_DEV void leaf_step(const DevScene &s, Accept &accept, uint32_t &tris) {
    if (core.leaf == kTravDone) return;
    uint32_t first, count;
    core.leaf_range(first, count);
    core.leaf = kTravDone;
    for (uint32_t i = 0; i < count; ++i) {
      const float4 *tr = s.tris + 3u * (first + i);
      float4 p0 = ldg4(tr), p1 = ldg4(tr + 1), p2 = ldg4(tr + 2);
      tris++;
      float t, b0, b1, b2;
      bool front;
      if (!intersect_watertight(core.r, {p0.x, p0.y, p0.z}, {p1.x, p1.y, p1.z}, {p2.x, p2.y, p2.z}, t, b0, b1, b2,
                                front))
        continue;
      if (!(t >= 0.0f && t <= t_max)) continue;
      if (accept(__float_as_uint(p0.w), __float_as_uint(p1.w), t, b0, b1, b2, front)) {
        occluded = true;
        return;
      }
    }
  }
  PT_DEV bool done() const { return occluded || core.finished(); }
};

// The node phase of while-while traversal ends once at most this many lanes
// of the warp are still looking for their first leaf, instead of when the
// last one finds it: the stragglers keep their traversal state and go on in
// the next round, and the warp's other lanes test their parked leaves
// meanwhile. Measured on the request mix: closest-hit traversal 701 -> 652
// ms and shadow rays 519 -> 493 ms per step with 4 (2: 677 / 498, 8: 648 /
// 487, 12: 672 / 496); on the sphere grid frame 36.6 -> 35.6 ms extend.
// With the four-child-only kernels, 6 traced the mix 1 % faster than 4 and
// the sphere grid frame within 0.2 %.
constexpr int kNodePhaseStragglers = 6;

// Warp-collective: whether the node phase goes on, given this lane's
// `searching` (it has a ray and no parked leaf yet) and `ready` (it has a
// parked leaf to test or a finished ray to write). The phase also goes on
// while no lane is ready, so every round makes progress.
PT_DEV bool node_phase_goes_on(bool searching, bool ready) {
  const int n = __popc(__ballot_sync(0xffffffffu, searching));
  return n > kNodePhaseStragglers || (n > 0 && !__any_sync(0xffffffffu, ready));
}

// Warp-aggregated claim of `chunk` consecutive queue entries for each lane
// with `need`; returns this lane's first entry index (meaningful when
// `need`). `exhausted` turns true (warp-uniformly) once the claims pass `n`,
// after which no atomics are issued.
PT_DEV uint32_t warp_claim(uint32_t *counter, bool need, uint32_t n, bool &exhausted, uint32_t chunk = 1) {
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t mask = __ballot_sync(0xffffffffu, need);
  if (mask == 0 || exhausted) return 0xffffffffu;
  uint32_t leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask) * chunk);
  base = __shfl_sync(0xffffffffu, base, leader);
  if (base + (uint32_t)__popc(mask) * chunk >= n) exhausted = true;
  return base + (uint32_t)__popc(mask & ((1u << lane) - 1u)) * chunk;
}

// A lane's claimed queue entries not yet started: entries [next, next + left).
struct ClaimedRun {
  uint32_t next = 0, left = 0;
  // Refills the run (warp-collective: every lane calls it) for lanes with
  // no ray and no entries left, then hands out this lane's next entry in
  // `idx` when it has no ray. Returns whether a new entry was taken.
  PT_DEV bool take(uint32_t *counter, bool has, uint32_t n, bool &exhausted, uint32_t chunk, uint32_t &idx) {
    const bool need = !has && left == 0;
    const uint32_t first = warp_claim(counter, need, n, exhausted, chunk);
    if (need && first < n) {
      next = first;
      left = min(chunk, n - first);
    }
    if (has || left == 0) return false;
    idx = next++;
    --left;
    return true;
  }
};

}  // namespace ptd
