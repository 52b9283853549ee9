// Wavefront schedule of the path loop: the per-vertex steps of
// dev_integrator.cuh run as separate kernels over compacted queues of path
// slots, with the path state held in structure-of-arrays form.
//
//   k_wf_raygen   camera rays for every slot of the wave (active queue 0);
//   k_wf_extend   closest hit of each queued path (traversal only: small
//                 register footprint, high occupancy);
//   k_wf_nee      per queued vertex, the area-light sample of next-event
//                 estimation and the emission MIS pdf (the f64
//                 spherical-triangle and environment sampling), kept out of
//                 the shade kernel's instruction footprint;
//   k_wf_shade    emission, material, BSDF, NEE shadow-ray generation,
//                 BSDF sampling, roulette; survivors are appended to the next
//                 active queue and paths with shadow rays to the shadow queue
//                 (warp-aggregated atomics);
//   k_wf_shadow   one lane per queued shadow ray (ray k of every path
//                 before ray k + 1): whether it reaches its light;
//   k_wf_shadow_add  each path's visible contributions, added to its
//                 radiance in generation order.
// The contributions of a vertex therefore reach the radiance sum in the
// reference's order (emission, punctual lights, area sample, next vertex):
// the per-sample radiance is bit-identical to the megakernel's.
// Queue lengths live in device memory (one counter block per bounce), so a
// wave runs max_bounces + 1 iterations without a host round trip; kernels
// of an exhausted iteration exit at once.
#pragma once

#include "dev_integrator.cuh"
#include "dev_traverse.cuh"

namespace ptd {

enum : uint32_t { HIT_FRONT = 1u << 31, HIT_FOUND = 1u << 30, HIT_G_MASK = (1u << 30) - 1u };
enum : uint32_t { PF_MEDIUM = 1u, PF_COVERED = 2u, PF_HERO_SHIFT = 2u };

PT_DEV void wf_store(const WaveBuffers &w, uint32_t slot, const PathState &ps, uint32_t request) {
  w.o[slot] = make_float4(ps.o.x, ps.o.y, ps.o.z, __uint_as_float(ps.k));
  w.d[slot] = make_float4(ps.d.x, ps.d.y, ps.d.z, ps.prev_pdf);
  uint32_t flags = (ps.has_medium ? PF_MEDIUM : 0u) | (ps.covered ? PF_COVERED : 0u) |
                   ((uint32_t)(ps.hero + 1) << PF_HERO_SHIFT);
  w.beta[slot] = make_float4(ps.beta.x, ps.beta.y, ps.beta.z, __uint_as_float(flags));
  w.rad[slot] = make_float4(ps.radiance.x, ps.radiance.y, ps.radiance.z, ps.covered ? 1.0f : 0.0f);
  w.prev[slot] = make_float4(ps.prev_pos.x, ps.prev_pos.y, ps.prev_pos.z, 0.0f);
  w.sigma[slot] = make_float4(ps.sigma.x, ps.sigma.y, ps.sigma.z, 0.0f);
  w.seed[slot] = make_uint4(ps.smp.pixel_seed, ps.smp.index, ps.smp.path_seed, request);
}

// wf_store without the sampler seeds and request, which never change after
// ray generation (shade writes back only what a vertex can change).
PT_DEV void wf_store_vertex(const WaveBuffers &w, uint32_t slot, const PathState &ps) {
  w.o[slot] = make_float4(ps.o.x, ps.o.y, ps.o.z, __uint_as_float(ps.k));
  w.d[slot] = make_float4(ps.d.x, ps.d.y, ps.d.z, ps.prev_pdf);
  uint32_t flags = (ps.has_medium ? PF_MEDIUM : 0u) | (ps.covered ? PF_COVERED : 0u) |
                   ((uint32_t)(ps.hero + 1) << PF_HERO_SHIFT);
  w.beta[slot] = make_float4(ps.beta.x, ps.beta.y, ps.beta.z, __uint_as_float(flags));
  w.rad[slot] = make_float4(ps.radiance.x, ps.radiance.y, ps.radiance.z, ps.covered ? 1.0f : 0.0f);
  w.prev[slot] = make_float4(ps.prev_pos.x, ps.prev_pos.y, ps.prev_pos.z, 0.0f);
  if (ps.has_medium) w.sigma[slot] = make_float4(ps.sigma.x, ps.sigma.y, ps.sigma.z, 0.0f);
}

PT_DEV uint32_t wf_load(const WaveBuffers &w, uint32_t slot, PathState &ps) {
  float4 o = w.o[slot], d = w.d[slot], b = w.beta[slot], r = w.rad[slot], p = w.prev[slot];
  uint4 sd = w.seed[slot];
  // The medium coefficients are read (and written) only inside a medium.
  const float4 s = (__float_as_uint(b.w) & PF_MEDIUM) ? w.sigma[slot] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  ps.o = {o.x, o.y, o.z};
  ps.k = __float_as_uint(o.w);
  ps.d = {d.x, d.y, d.z};
  ps.prev_pdf = d.w;
  uint32_t flags = __float_as_uint(b.w);
  ps.beta = {b.x, b.y, b.z};
  ps.has_medium = (flags & PF_MEDIUM) ? 1u : 0u;
  ps.covered = (flags & PF_COVERED) ? 1u : 0u;
  ps.hero = (int32_t)(flags >> PF_HERO_SHIFT) - 1;
  ps.radiance = {r.x, r.y, r.z};
  ps.prev_pos = {p.x, p.y, p.z};
  ps.sigma = {s.x, s.y, s.z};
  ps.smp.pixel_seed = sd.x;
  ps.smp.index = sd.y;
  ps.smp.path_seed = sd.z;
  return sd.w;
}

// Warp-aggregated append: one atomic per warp for the lanes with `pred`.
PT_DEV void wf_append(uint32_t *queue, uint32_t *count, bool pred, uint32_t value) {
  uint32_t active = __activemask();
  uint32_t mask = __ballot_sync(active, pred);
  if (mask == 0) return;
  uint32_t lane = threadIdx.x & 31u;
  uint32_t leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(count, (uint32_t)__popc(mask));
  base = __shfl_sync(active, base, leader);
  if (pred) queue[base + __popc(mask & ((1u << lane) - 1u))] = value;
}

// Warp-aggregated maximum: one atomic per warp.
PT_DEV void wf_max(uint32_t *dst, uint32_t v) {
  const uint32_t active = __activemask();
  const uint32_t m = __reduce_max_sync(active, v);
  if ((threadIdx.x & 31u) == (uint32_t)(__ffs(active) - 1) && m) atomicMax(dst, m);
}

struct DeferredSink {
  const WaveBuffers *w;
  uint32_t slot, count;
  PT_DEV void emit(const ShadowRay &sr) {
    if (count >= w->shadow_slots) return;  // host sizes shadow_slots >= lights + 1
    size_t i = (size_t)count * w->capacity + slot;
    w->sh_o[i] = make_float4(sr.o.x, sr.o.y, sr.o.z, sr.tmax);
    w->sh_d[i] = make_float4(sr.d.x, sr.d.y, sr.d.z, __uint_as_float(sr.ray_id));
    w->sh_c[i] = make_float4(sr.contrib.x, sr.contrib.y, sr.contrib.z, __uint_as_float(sr.skip));
    ++count;
  }
};

// Camera rays for every slot of the wave (grid-stride over the wave's
// slots, read from the wave descriptor).
__global__ void __launch_bounds__(256) k_wf_raygen(WaveBuffers w) {
  const WaveDesc wd = *w.desc;
  if (blockIdx.x == 0 && threadIdx.x == 0) w.counters[0] = wd.total;
  for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < wd.total; slot += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = wd.nseg;
    while (hi - lo > 1) {
      uint32_t mid = (lo + hi) >> 1;
      if (wd.segs[mid].slot_begin <= slot)
        lo = mid;
      else
        hi = mid;
    }
    const WaveSegment &seg = wd.segs[lo];
    const DevRequest &rq = wd.reqs[seg.request];
    uint32_t local = slot - seg.slot_begin;
    uint32_t sidx = local / seg.pixel_count, i = local - sidx * seg.pixel_count;
    uint32_t p = seg.pixel_begin + i;
    uint32_t y = p / rq.width, x = p - y * rq.width;
    PathState ps;
    init_path(rq, x, y, seg.sample_begin + sidx, ps);
    wf_store(w, slot, ps, seg.request);
    w.q[0][slot] = slot;
  }
}

// In-order f64 accumulation of the wave's per-slot results into each
// request's accumulator (a pixel's samples in index order, as the
// reference's per-pixel loop adds them).
__global__ void __launch_bounds__(256) k_wf_accumulate(WaveBuffers w) {
  const WaveDesc wd = *w.desc;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t sg = 0; sg < wd.nseg; ++sg) {
    const WaveSegment seg = wd.segs[sg];
    double4 *accum = reinterpret_cast<double4 *>(wd.reqs[seg.request].accum) + seg.pixel_begin;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < seg.pixel_count; i += stride) {
      double4 a = accum[i];
      const float4 *src = w.rad + seg.slot_begin + i;
      for (uint32_t k = 0; k < seg.spp; ++k) {
        float4 v = src[(size_t)k * seg.pixel_count];
        if (v.w > 0.0f) {
          // Non-finite radiance counts as a covered black sample (src/pathtrace.rs:2324-2328).
          if (!(isfinite(v.x) && isfinite(v.y) && isfinite(v.z))) v = make_float4(0.0f, 0.0f, 0.0f, v.w);
          a.x += (double)v.x;
          a.y += (double)v.y;
          a.z += (double)v.z;
          a.w += 1.0;
        }
      }
      accum[i] = a;
    }
  }
}

// Computed by extend when the ray finishes and stored by queue position, so
// the count / scatter passes read keys and slots contiguously.
PT_DEV uint32_t sort_key(const DevScene *s, bool found, uint32_t g) {
  if (!found) return 0;
  uint32_t m = __ldg(s->tri_info + g).x;
  uint32_t sh = (uint32_t)((uintptr_t)s >> 8) * 0x9E3779B1u;
  return 1u + (m + sh) % (kSortBuckets - 1u);
}

// Closest hit of every queued path: persistent lanes, one ray each, refilled
// from the queue as rays finish (dev_traverse.cuh), in runs of
// w.claim_chunk entries. kThreads per block, 1,024 threads per SM.
// kOnly4: every request of the wave walks the four-child layout for
// extension rays (WaveBuffers::all_wide).
template <int kThreads, bool kOnly4>
__global__ void __launch_bounds__(kThreads, 1024 / kThreads) k_wf_extend(WaveBuffers w, uint32_t iter,
                                                                       DevCounters *ctr) {
  const DevRequest *reqs = w.desc->reqs;
  __shared__ int s_stack[kShortStack * kThreads];
  const uint32_t n = w.counters[iter * kWfCounterStride + 0];
  const uint32_t *q = w.q[iter & 1u];
  uint32_t *claim = w.counters + iter * kWfCounterStride + 2;
  TravStack stk;
  stk.sm = s_stack + threadIdx.x;
  stk.stride = blockDim.x;
  ThreadStats ts{0, 0, 0, 0, 0, 0, 0};
  bool has = false, exhausted = false;
  uint32_t slot = 0, k = 0, qpos = 0;
  const DevRequest *rq = nullptr;
  Sampler smp;
  ClosestRay cr;
  ClaimedRun run;
  for (;;) {
    uint32_t idx = 0;
    if (run.take(claim, has, n, exhausted, w.claim_chunk, idx)) {
      qpos = idx;
      slot = q[idx];
      float4 o = w.o[slot], d = w.d[slot];
      uint4 sd = w.seed[slot];
      rq = reqs + sd.w;
      smp.pixel_seed = sd.x;
      smp.index = sd.y;
      smp.path_seed = sd.z;
      k = __float_as_uint(o.w);
      cr.init(*rq->scene, {o.x, o.y, o.z}, {d.x, d.y, d.z}, 0.0f, inf(), (rq->wide_nodes & WIDE_EXTENSION) != 0);
      has = true;
      ts.ext_rays++;
    }
    if (!__any_sync(0xffffffffu, has)) break;
    // Node phase: until at most kNodePhaseStragglers lanes still look for
    // their first leaf (they go on in the next round).
    while (node_phase_goes_on(has && cr.core.searching(),
                              has && (cr.core.leaf != kTravDone || cr.core.finished()))) {
      if (has && cr.core.can_step()) cr.template node_step<kOnly4>(*rq->scene, stk, ts.ext_nodes, ts.err);
    }
    // Leaf phase.
    if (has) {
      const DevScene &s = *rq->scene;
      AcceptFilter acc{&s, &smp, k << 16, k == 0, 0xffffffffu};
      cr.leaf_step(s, acc, ts.ext_tris);
      if (cr.core.finished()) {
        if (cr.have) {
          const Hit &h = cr.best;
          w.hit_tb[slot] = make_float4(h.t, h.b0, h.b1, h.b2);
          w.hit_g[slot] = (h.g & HIT_G_MASK) | HIT_FOUND | (h.front ? HIT_FRONT : 0u);
        } else {
          w.hit_g[slot] = 0u;
        }
        if (w.sort_materials) w.sort_keys[qpos] = sort_key(&s, cr.have, cr.best.g);
        has = false;
      }
    }
  }
  flush_stats(ctr, ts);
}

// ---- material sort: the active queue bucketed by (scene, material) before
// shade, stable within each warp's group of equal keys. Bucket 0 holds the
// paths whose ray missed.
// Tiles of kSortTile queue entries per block: a shared-memory histogram per
// tile, then one global atomic per non-empty bucket (the hot buckets - the
// material most paths hit - would serialise per-warp global atomics).
constexpr uint32_t kSortPerThread = 8, kSortTile = 256 * kSortPerThread;

__global__ void __launch_bounds__(256) k_wf_sort_count(WaveBuffers w, uint32_t iter) {
  __shared__ uint32_t hist[kSortBuckets];
  const uint32_t n = w.counters[iter * kWfCounterStride + 0];
  uint32_t *count = w.sort_counts + (size_t)iter * 2 * kSortBuckets;
  const uint32_t t = threadIdx.x;
  for (uint32_t base = blockIdx.x * kSortTile; base < n; base += gridDim.x * kSortTile) {
    hist[t] = 0;
    __syncthreads();
#pragma unroll
    for (uint32_t e = 0; e < kSortPerThread; ++e) {
      const uint32_t i = base + e * 256 + t;
      if (i < n) atomicAdd(&hist[w.sort_keys[i]], 1u);
    }
    __syncthreads();
    if (hist[t]) atomicAdd(count + t, hist[t]);
    __syncthreads();
  }
}

// One block of kSortBuckets threads: bucket sizes -> start cursors.
__global__ void __launch_bounds__(kSortBuckets) k_wf_sort_scan(WaveBuffers w, uint32_t iter) {
  __shared__ uint32_t s[kSortBuckets];
  uint32_t *count = w.sort_counts + (size_t)iter * 2 * kSortBuckets;
  const uint32_t t = threadIdx.x;
  const uint32_t own = count[t];
  s[t] = own;
  __syncthreads();
  for (uint32_t off = 1; off < kSortBuckets; off <<= 1) {
    uint32_t v = t >= off ? s[t - off] : 0u;
    __syncthreads();
    s[t] += v;
    __syncthreads();
  }
  count[kSortBuckets + t] = s[t] - own;
}

__global__ void __launch_bounds__(256) k_wf_sort_scatter(WaveBuffers w, uint32_t iter) {
  __shared__ uint32_t hist[kSortBuckets], start[kSortBuckets];
  const uint32_t n = w.counters[iter * kWfCounterStride + 0];
  const uint32_t *q = w.q[iter & 1u];
  uint32_t *cursor = w.sort_counts + (size_t)iter * 2 * kSortBuckets + kSortBuckets;
  const uint32_t t = threadIdx.x;
  for (uint32_t base = blockIdx.x * kSortTile; base < n; base += gridDim.x * kSortTile) {
    hist[t] = 0;
    __syncthreads();
    uint32_t key[kSortPerThread], rank[kSortPerThread];
#pragma unroll
    for (uint32_t e = 0; e < kSortPerThread; ++e) {
      const uint32_t i = base + e * 256 + t;
      key[e] = i < n ? w.sort_keys[i] : 0u;
      rank[e] = i < n ? atomicAdd(&hist[key[e]], 1u) : 0u;
    }
    __syncthreads();
    if (hist[t]) start[t] = atomicAdd(cursor + t, hist[t]);
    __syncthreads();
#pragma unroll
    for (uint32_t e = 0; e < kSortPerThread; ++e) {
      const uint32_t i = base + e * 256 + t;
      if (i < n) w.q_sorted[start[key[e]] + rank[e]] = q[i];
    }
    __syncthreads();
  }
}

// The area-light sample and emission MIS pdf of every queued vertex that
// hit something, in the order shade will read them (its queue). Values are
// those shade would compute inline (the same functions on the same inputs).
// Four blocks of 256 per SM (64 registers, a few spills): the sampling is
// latency bound (CDF searches, dependent f64 steps), so occupancy beats the
// spill-free 106-register form (NEE stage 128 -> 120 ms per mix step).
__global__ void __launch_bounds__(256, 4) k_wf_nee(WaveBuffers w, uint32_t iter) {
  if (!(w.desc->flags & WAVE_AREA_LIGHTS)) return;  // nothing to sample in this wave
  const DevRequest *reqs = w.desc->reqs;
  const uint32_t n = w.counters[iter * kWfCounterStride + 0];
  const uint32_t *q = w.sort_materials ? w.q_sorted : w.q[iter & 1u];
  const size_t cap = w.capacity;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t slot = q[i];
    const uint32_t hg = w.hit_g[slot];
    if (!(hg & HIT_FOUND)) continue;
    const uint4 sd = w.seed[slot];
    const DevRequest &rq = reqs[sd.w];
    const DevScene &s = *rq.scene;
    if (!rq.env && s.em_count == 0) continue;  // shade reads nothing for this request
    const uint32_t k = __float_as_uint(w.o[slot].w);
    const uint32_t g = hg & HIT_G_MASK;
    const float4 tb = w.hit_tb[slot];
    const V3 pos = interp3(s.pos, g, tb.y, tb.z, tb.w);
    float pl_emit = 0.0f;
    if (k > 0) {
      const float4 pv = w.prev[slot];
      pl_emit = emission_light_pdf(rq, s, g, {pv.x, pv.y, pv.z}, pos);
    }
    AreaSample as;
    as.go = false;
    if (k < rq.max_bounces && area_nee(rq, s)) {
      Sampler smp;
      smp.pixel_seed = sd.x;
      smp.index = sd.y;
      smp.path_seed = sd.z;
      float pl_u[4];
      smp.pattern(2 + 2 * k, pl_u);
      as = sample_area_light(rq, s, pos, pl_u);
    }
    if (as.go) {
      w.nee[slot] = make_float4(as.l.x, as.l.y, as.l.z, as.pl);
      w.nee[cap + slot] = make_float4(as.le.x, as.le.y, as.le.z, as.tmax);
    }
    w.nee[2 * cap + slot] = make_float4(__uint_as_float(as.skip), as.go ? 1.0f : 0.0f, pl_emit, 0.0f);
  }
}

// kBlocks 128-thread blocks per SM. Three (168 registers) measured faster
// than the unconstrained 234-register build despite a few spills, and than
// four on scenes with light shading (C1); four (128 registers, more
// spills) is faster where shading is heavy (C2's f64 area-light sampling).
// The tuner picks per scene class.
template <int kBlocks>
__global__ void __launch_bounds__(128, kBlocks) k_wf_shade(WaveBuffers w, uint32_t iter) {
  const DevRequest *reqs = w.desc->reqs;
  const uint32_t n = w.counters[iter * kWfCounterStride + 0];
  const uint32_t *q = w.sort_materials ? w.q_sorted : w.q[iter & 1u];
  uint32_t *q_next = w.q[(iter + 1) & 1u];
  uint32_t *n_next = w.counters + (iter + 1) * kWfCounterStride + 0;
  uint32_t *n_shadow = w.counters + iter * kWfCounterStride + 1;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t slot = q[i];
    PathState ps;
    uint32_t request = wf_load(w, slot, ps);
    const DevRequest &rq = reqs[request];
    uint32_t hg = w.hit_g[slot];
    bool found = (hg & HIT_FOUND) != 0;
    Hit h;
    if (found) {
      float4 tb = w.hit_tb[slot];
      h.t = tb.x;
      h.b0 = tb.y;
      h.b1 = tb.z;
      h.b2 = tb.w;
      h.g = hg & HIT_G_MASK;
      h.front = (hg & HIT_FRONT) != 0;
    }
    DeferredSink sink{&w, slot, 0};
    NeeInput pre;
    pre.area.go = false;
    pre.pl_emit = 0.0f;
    if (found && (rq.env || rq.scene->em_count > 0)) {
      const size_t cap = w.capacity;
      const float4 n2 = w.nee[2 * cap + slot];
      pre.area.go = n2.y != 0.0f;
      pre.area.skip = __float_as_uint(n2.x);
      pre.pl_emit = n2.z;
      if (pre.area.go) {
        const float4 n0 = w.nee[slot], n1 = w.nee[cap + slot];
        pre.area.l = {n0.x, n0.y, n0.z};
        pre.area.pl = n0.w;
        pre.area.le = {n1.x, n1.y, n1.z};
        pre.area.tmax = n1.w;
      }
    }
    bool alive = shade<DeferredSink, true>(rq, ps, found, h, sink, &pre);
    wf_store_vertex(w, slot, ps);
    w.sh_n[slot] = sink.count;
    wf_append(q_next, n_next, alive, slot);
    wf_append(w.q_shadow, n_shadow, sink.count > 0, slot);
    wf_max(n_shadow + 3, sink.count);
  }
}

// Shadow rays of the queued paths, one lane per ray: entry i of the
// flattened queue is ray k = i / n of queued path i % n (n paths, k below
// the wave's largest per-path count), so neighbouring lanes trace the same
// light's rays from neighbouring queue positions. A lane records whether
// its ray reached the light (sh_vis); k_wf_shadow_add then adds each path's
// visible contributions in generation order. Entries past a path's own
// count carry no ray. n times the largest count fits 32 bits: the arena
// holds 48 bytes per (ray, slot).
// kOnly4: every request of the wave walks the four-child layout for shadow
// rays.
template <int kThreads, bool kOnly4>
__global__ void __launch_bounds__(kThreads, 1024 / kThreads) k_wf_shadow(WaveBuffers w, uint32_t iter,
                                                                       DevCounters *ctr) {
  const DevRequest *reqs = w.desc->reqs;
  __shared__ int s_stack[kShortStack * kThreads];
  const uint32_t n = w.counters[iter * kWfCounterStride + 1];
  const uint32_t kmax = min(w.counters[iter * kWfCounterStride + 4], w.shadow_slots);
  const uint32_t total = n * kmax;
  uint32_t *claim = w.counters + iter * kWfCounterStride + 3;
  TravStack stk;
  stk.sm = s_stack + threadIdx.x;
  stk.stride = blockDim.x;
  ThreadStats ts{0, 0, 0, 0, 0, 0, 0};
  bool has = false, exhausted = false;
  size_t e = 0;
  uint32_t ray_id = 0, skip = 0;
  const DevRequest *rq = nullptr;
  Sampler smp;
  ShadowTrav tr;
  ClaimedRun run;
  for (;;) {
    uint32_t idx = 0;
    if (run.take(claim, has, total, exhausted, w.claim_chunk, idx)) {
      const uint32_t k = idx / n, q = idx - k * n;
      const uint32_t slot = w.q_shadow[q];
      if (k < w.sh_n[slot]) {
        const uint4 sd = w.seed[slot];
        rq = reqs + sd.w;
        smp.pixel_seed = sd.x;
        smp.index = sd.y;
        smp.path_seed = sd.z;
        e = (size_t)k * w.capacity + slot;
        const float4 so = w.sh_o[e], sdd = w.sh_d[e];
        tr.init(*rq->scene, {so.x, so.y, so.z}, {sdd.x, sdd.y, sdd.z}, so.w, (rq->wide_nodes & WIDE_SHADOW) != 0);
        ray_id = __float_as_uint(sdd.w);
        skip = __float_as_uint(w.sh_c[e].w);
        ts.shadow_rays++;
        has = true;
      }
    }
    if (!__any_sync(0xffffffffu, has)) {
      // Lanes that drew entries without a ray draw again; the warp ends
      // once the queue is exhausted and no lane holds unstarted entries.
      if (exhausted && !__any_sync(0xffffffffu, run.left > 0)) break;
      continue;
    }
    // Node phase: until at most kNodePhaseStragglers lanes still search.
    while (node_phase_goes_on(has && tr.core.searching(),
                              has && (tr.core.leaf != kTravDone || tr.core.finished()))) {
      if (has && tr.core.can_step()) tr.template node_step<kOnly4>(*rq->scene, stk, ts.sh_nodes, ts.err);
    }
    // Leaf phase.
    if (has) {
      const DevScene &s = *rq->scene;
      AcceptFilter acc{&s, &smp, ray_id, false, skip};
      tr.leaf_step(s, acc, ts.sh_tris);
      if (tr.done()) {
        w.sh_vis[e] = tr.occluded ? 0 : 1;
        has = false;
      }
    }
  }
  flush_stats(ctr, ts);
}

// Each queued path's visible shadow-ray contributions, added to its
// radiance in generation order (the order the reference adds them).
__global__ void __launch_bounds__(256) k_wf_shadow_add(WaveBuffers w, uint32_t iter) {
  const uint32_t n = w.counters[iter * kWfCounterStride + 1];
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const uint32_t slot = w.q_shadow[q];
    const uint32_t cnt = w.sh_n[slot];
    const float4 r = w.rad[slot];
    V3 rad = {r.x, r.y, r.z};
    for (uint32_t k = 0; k < cnt; ++k) {
      const size_t e = (size_t)k * w.capacity + slot;
      if (w.sh_vis[e]) {
        const float4 c = w.sh_c[e];
        rad = vadd(rad, {c.x, c.y, c.z});
      }
    }
    w.rad[slot] = make_float4(rad.x, rad.y, rad.z, r.w);
  }
}

}  // namespace ptd
