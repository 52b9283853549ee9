// Persistent-thread traversal for the wavefront's extend and shadow kernels.
//
// Each lane owns one ray at a time and asks for the next queue entry the
// moment its ray finishes (one warp-aggregated atomic per refill), so the
// lanes of a warp stay busy instead of idling behind the warp's slowest ray
// (Aila & Laine, "Understanding the Efficiency of Ray Traversal on GPUs",
// HPG 2009: persistent threads with dynamic fetch). A loop iteration takes
// a lane from its current position down to its next leaf (inner-node steps)
// and then tests that leaf, so lanes reconverge once per leaf.
//
// The traversal stack keeps its top entries in shared memory (one column
// per thread, conflict-free) and spills deeper entries to local memory.
//
// Results equal closest_hit / occluded of dev_scene.cuh: the closest hit is
// the accepted candidate with the smallest t (ties: lowest global id), a
// definition that does not depend on traversal order, and the any-hit
// answer is a yes/no.
#pragma once

#include "dev_scene.cuh"

namespace ptd {

constexpr int kShortStack = 16;     // shared-memory entries per thread
constexpr int kTravDone = 0x7fffffff;  // "no next node" (never a node index)

struct TravStack {
  int *sm;        // this thread's column: entry i at sm[i * stride]
  int stride;
  int spill[kStackSize - kShortStack];
  PT_DEV void push(int &sp, int v, uint32_t &err) {
    if (sp < kShortStack)
      sm[sp * stride] = v;
    else if (sp < kStackSize)
      spill[sp - kShortStack] = v;
    else {
      err |= ERR_STACK_OVERFLOW;
      return;
    }
    ++sp;
  }
  PT_DEV int pop(int &sp) {
    --sp;
    return sp < kShortStack ? sm[sp * stride] : spill[sp - kShortStack];
  }
};

// Walks inner nodes from `cur` until a leaf reference (< 0) is reached, or
// returns kTravDone when the stack runs dry. `t_far` culls boxes (the best
// hit so far, or t_max). Near child first when `ordered`.
PT_DEV int descend(const DevScene &s, const Ray &r, float t_min, float t_far, int cur, int &sp, TravStack &stk,
                   uint32_t &nodes, uint32_t &err, bool ordered) {
  for (;;) {
    if (cur == kTravDone) {
      if (sp == 0) return kTravDone;
      cur = stk.pop(sp);
      continue;
    }
    if (cur < 0) return cur;
    nodes++;
    bool h0, h1;
    float e0, e1;
    int4 dd;
    node_boxes(s.nodes + cur, r, t_min, t_far, h0, h1, e0, e1, dd);
    if (h0 && h1) {
      bool swap = ordered && e1 < e0;
      stk.push(sp, swap ? dd.x : dd.y, err);
      cur = swap ? dd.y : dd.x;
    } else if (h0) {
      cur = dd.x;
    } else if (h1) {
      cur = dd.y;
    } else {
      cur = kTravDone;
    }
  }
}

// Closest-hit traversal of one ray, resumable leaf by leaf.
struct ClosestRay {
  Ray r;
  float t_min;
  Hit best;
  bool have;
  int cur, sp;
  PT_DEV void init(V3 o, V3 d, float tmin, float tmax) {
    r = make_ray(o, d);
    t_min = tmin;
    best.t = tmax;
    best.g = 0xffffffffu;
    have = false;
    cur = 0;
    sp = 0;
  }
  // One iteration: descend to the next leaf and test it. Returns true when
  // the ray is finished.
  template <class Accept>
  PT_DEV bool step(const DevScene &s, TravStack &stk, Accept &accept, uint32_t &nodes, uint32_t &tris,
                   uint32_t &err) {
    if (s.node_count == 0) return true;
    const float t_max = best.t;
    cur = descend(s, r, t_min, best.t, cur, sp, stk, nodes, err, true);
    if (cur == kTravDone) return true;
    uint32_t first = (uint32_t)(~cur);
    uint32_t count = first >> kLeafCountShift;
    first &= kLeafFirstMask;
    for (uint32_t i = 0; i < count; ++i) {
      const float4 *tr = s.tris + 3u * (first + i);
      float4 p0 = ldg4(tr), p1 = ldg4(tr + 1), p2 = ldg4(tr + 2);
      tris++;
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
    cur = kTravDone;  // next: pop
    return sp == 0;
  }
};

// Any-hit traversal of one ray, resumable leaf by leaf.
struct ShadowTrav {
  Ray r;
  float t_max;
  int cur, sp;
  PT_DEV void init(V3 o, V3 d, float tmax) {
    r = make_ray(o, d);
    t_max = tmax;
    cur = 0;
    sp = 0;
  }
  // Returns 0 while running, 1 when finished unoccluded, 2 when occluded.
  template <class Accept>
  PT_DEV int step(const DevScene &s, TravStack &stk, Accept &accept, uint32_t &nodes, uint32_t &tris,
                  uint32_t &err) {
    if (s.node_count == 0) return 1;
    cur = descend(s, r, 0.0f, t_max, cur, sp, stk, nodes, err, false);
    if (cur == kTravDone) return 1;
    uint32_t first = (uint32_t)(~cur);
    uint32_t count = first >> kLeafCountShift;
    first &= kLeafFirstMask;
    for (uint32_t i = 0; i < count; ++i) {
      const float4 *tr = s.tris + 3u * (first + i);
      float4 p0 = ldg4(tr), p1 = ldg4(tr + 1), p2 = ldg4(tr + 2);
      tris++;
      float t, b0, b1, b2;
      bool front;
      if (!intersect_watertight(r, {p0.x, p0.y, p0.z}, {p1.x, p1.y, p1.z}, {p2.x, p2.y, p2.z}, t, b0, b1, b2, front))
        continue;
      if (!(t >= 0.0f && t <= t_max)) continue;
      if (accept(__float_as_uint(p0.w), __float_as_uint(p1.w), t, b0, b1, b2, front)) return 2;
    }
    cur = kTravDone;
    return sp == 0 ? 1 : 0;
  }
};

// Warp-aggregated claim of queue entries for the lanes with `need`; returns
// this lane's entry index (meaningful when `need`). `exhausted` turns true
// (warp-uniformly) once the claims pass `n`, after which no atomics are
// issued.
PT_DEV uint32_t warp_claim(uint32_t *counter, bool need, uint32_t n, bool &exhausted) {
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t mask = __ballot_sync(0xffffffffu, need);
  if (mask == 0 || exhausted) return 0xffffffffu;
  uint32_t leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (base + (uint32_t)__popc(mask) >= n) exhausted = true;
  return base + __popc(mask & ((1u << lane) - 1u));
}

}  // namespace ptd
