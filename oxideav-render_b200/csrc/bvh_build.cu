// Device BVH construction (bvh_build.h): Morton order, radix sort, parallel
// locally-ordered clustering, SAH leaf collapse, and the two node layouts.
//
// Data layout during the build (n triangles, 2n - 1 binary nodes):
//   node v < n        leaf of the triangle at sorted position v
//   node v >= n       interior node created by the (v - n)-th merge; merges
//                     of one clustering round get consecutive ids, so every
//                     parent has a larger id (and a later round) than its
//                     children
//   nlo / nhi         node boxes (float4, w unused)
//   ncount / ncost    triangles below the node / its SAH cost
//   nstate            NS_* bits; nfirst / ndepth from the top-down pass
//   nchild[v - n]     the two children of interior node v
// The output layouts number the surviving interior nodes in decreasing id
// order (root first).
#include <algorithm>
#include <type_traits>
#include <chrono>
#include <cstdio>
#include <vector>

#include "bvh_build.h"
#include "dev_types.h"

namespace ptd {
namespace {

constexpr int kPlocRadius = 16;
// Morton code bits per axis: 10 (30-bit codes in 32-bit keys) or 21 (63-bit
// codes in 64-bit keys).
constexpr int kMortonAxisBits = 10;
using MortonKey = std::conditional_t<(kMortonAxisBits > 10), unsigned long long, uint32_t>;
constexpr int kMortonBits = 3 * kMortonAxisBits;
constexpr uint32_t kMaxLeafTris = 8;
// SAH weights of a node visit and of a triangle test.
constexpr float kTraversalCost = 1.0f, kTriangleCost = 1.0f;
// Smallest scene built on the device; smaller ones build on the host.
constexpr uint32_t kMinDeviceTris = 64;
constexpr uint32_t kMaxRounds = 1u << 16;

constexpr int kThreads = 256;
constexpr int kScanItems = 8, kScanTile = kThreads * kScanItems;
constexpr int kRadixRounds = 8, kRadixTile = kThreads * kRadixRounds, kRadixBins = 256;
constexpr uint32_t kLeafShift = 27;

enum NodeState : uint32_t { NS_COVERED = 1u, NS_WIDE = 2u, NS_COLLAPSED = 4u };

__device__ __forceinline__ float box_area(float4 lo, float4 hi) {
  float dx = fmaxf(hi.x - lo.x, 0.0f), dy = fmaxf(hi.y - lo.y, 0.0f), dz = fmaxf(hi.z - lo.z, 0.0f);
  float a = dx * dy + dy * dz + dz * dx;
  return isnan(a) ? INFINITY : a;
}
__device__ __forceinline__ float4 fmin4(float4 a, float4 b) {
  return make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), 0.0f);
}
__device__ __forceinline__ float4 fmax4(float4 a, float4 b) {
  return make_float4(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z), 0.0f);
}
// Order-preserving map of floats to unsigned ints (for atomicMin / Max).
__device__ __forceinline__ uint32_t ord_of(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float float_of(uint32_t u) {
  return (u & 0x80000000u) ? __uint_as_float(u & 0x7fffffffu) : __uint_as_float(~u);
}
// The low `kMortonAxisBits` bits of x spread to every third bit.
__device__ __forceinline__ MortonKey spread_bits(uint32_t x) {
  MortonKey r = 0;
#pragma unroll
  for (int b = 0; b < kMortonAxisBits; ++b) r |= (MortonKey)((x >> b) & 1u) << (3 * b);
  return r;
}

// ---------------------------------------------------------------- scans
// Exclusive prefix sums in tiles of kScanTile items: each block scans one
// tile and leaves the tile total in `sums`; a scan of the totals, added
// back, completes the multi-tile scan.
template <class T>
__global__ void __launch_bounds__(kThreads) k_scan_tile(const T *in, T *out, uint64_t n, T *sums) {
  __shared__ T warp_tot[kThreads / 32];
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  T v[kScanItems];
  T run = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = base + k < n ? in[base + k] : T(0);
    T x = v[k];
    v[k] = run;
    run += x;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T incl = run;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += y;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  T before = 0, total = 0;
  for (int w = 0; w < kThreads / 32; ++w) {
    if (w < warp) before += warp_tot[w];
    total += warp_tot[w];
  }
  const T excl = before + incl - run;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) out[base + k] = excl + v[k];
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

template <class T>
__global__ void k_scan_add(T *out, uint64_t n, const T *offs) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] += offs[i / kScanTile];
}

uint64_t tiles_of(uint64_t n, uint64_t tile) { return (n + tile - 1) / tile; }

// Scratch for every level of a scan of up to `n` items.
uint64_t scan_scratch_items(uint64_t n) {
  uint64_t total = 0;
  do {
    n = tiles_of(n, kScanTile);
    total += n + 1;
  } while (n > 1);
  return total;
}

unsigned grid_for(uint64_t n, int per_block = kThreads) {
  uint64_t g = (n + per_block - 1) / per_block;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(g, 1u << 20));
}

// Exclusive scan in -> out (in == out allowed). Returns the device address
// of the grand total.
template <class T>
T *scan_exclusive(const T *in, T *out, uint64_t n, T *scratch, cudaStream_t st) {
  const uint64_t nt = tiles_of(std::max<uint64_t>(n, 1), kScanTile);
  T *sums = scratch;
  k_scan_tile<T><<<(unsigned)nt, kThreads, 0, st>>>(in, out, n, sums);
  if (nt == 1) return sums;
  T *total = scan_exclusive<T>(sums, sums, nt, scratch + nt + 1, st);
  k_scan_add<T><<<grid_for(n), kThreads, 0, st>>>(out, n, sums);
  return total;
}

// ---------------------------------------------------------------- radix sort
__global__ void __launch_bounds__(kThreads) k_radix_hist(const MortonKey *keys, uint32_t n, int shift, uint32_t *hist,
                                                         uint32_t ntiles) {
  __shared__ uint32_t h[kRadixBins];
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * kRadixTile;
#pragma unroll
  for (int r = 0; r < kRadixRounds; ++r) {
    uint64_t i = base + (uint64_t)r * kThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(uint32_t)(keys[i] >> shift) & 0xffu], 1u);
  }
  __syncthreads();
  hist[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one tile: items are ranked in input order, a round of
// kThreads items at a time (warp match for equal digits inside a warp,
// per-warp digit counts across warps, a running count across rounds).
__global__ void __launch_bounds__(kThreads) k_radix_scatter(const MortonKey *keys, const uint32_t *vals, MortonKey *keys_out,
                                                            uint32_t *vals_out, uint32_t n, int shift,
                                                            const uint32_t *offs, uint32_t ntiles) {
  __shared__ uint32_t run[kRadixBins];
  __shared__ uint32_t wc[kThreads / 32][kRadixBins];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  run[threadIdx.x] = offs[(uint64_t)threadIdx.x * ntiles + blockIdx.x];
#pragma unroll
  for (int w = 0; w < kThreads / 32; ++w) wc[w][threadIdx.x] = 0;
  __syncthreads();
  const uint32_t lt = (1u << lane) - 1u;
  const uint64_t base = (uint64_t)blockIdx.x * kRadixTile;
  for (int r = 0; r < kRadixRounds; ++r) {
    const uint64_t i = base + (uint64_t)r * kThreads + threadIdx.x;
    const bool valid = i < n;
    MortonKey key = 0;
    uint32_t val = 0, d = kRadixBins;
    if (valid) {
      key = keys[i];
      val = vals[i];
      d = (uint32_t)(key >> shift) & 0xffu;
    }
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t rank = __popc(peers & lt);
    const bool leader = lane == __ffs(peers) - 1;
    if (valid && leader) wc[warp][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      uint32_t pos = run[d] + rank;
      for (int w = 0; w < warp; ++w) pos += wc[w][d];
      keys_out[pos] = key;
      vals_out[pos] = val;
    }
    __syncthreads();
    uint32_t add = 0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) add += wc[w][threadIdx.x];
    run[threadIdx.x] += add;
    __syncthreads();
    if (valid && leader) wc[warp][d] = 0;
    __syncthreads();
  }
}

// ---------------------------------------------------------------- primitives
// Triangle boxes (a triangle with a NaN coordinate gets an empty box: it
// can never be hit) and the bounds of the finite centroids.
__global__ void __launch_bounds__(kThreads) k_prim_boxes(const float *pos, uint32_t n, float4 *lo, float4 *hi,
                                                         uint32_t *cb) {
  float cl[3] = {INFINITY, INFINITY, INFINITY}, ch[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float *p = pos + 9ull * i;
    float v[9];
    bool nan = false;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      v[k] = __ldg(p + k);
      nan |= isnan(v[k]);
    }
    float4 l, h;
    if (nan) {
      l = make_float4(INFINITY, INFINITY, INFINITY, 0.0f);
      h = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.0f);
    } else {
      l = make_float4(fminf(fminf(v[0], v[3]), v[6]), fminf(fminf(v[1], v[4]), v[7]), fminf(fminf(v[2], v[5]), v[8]),
                      0.0f);
      h = make_float4(fmaxf(fmaxf(v[0], v[3]), v[6]), fmaxf(fmaxf(v[1], v[4]), v[7]), fmaxf(fmaxf(v[2], v[5]), v[8]),
                      0.0f);
      float c[3] = {(l.x + h.x) * 0.5f, (l.y + h.y) * 0.5f, (l.z + h.z) * 0.5f};
      if (isfinite(c[0]) && isfinite(c[1]) && isfinite(c[2]))
        for (int k = 0; k < 3; ++k) {
          cl[k] = fminf(cl[k], c[k]);
          ch[k] = fmaxf(ch[k], c[k]);
        }
    }
    lo[i] = l;
    hi[i] = h;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k)
    for (int d = 16; d > 0; d >>= 1) {
      cl[k] = fminf(cl[k], __shfl_xor_sync(0xffffffffu, cl[k], d));
      ch[k] = fmaxf(ch[k], __shfl_xor_sync(0xffffffffu, ch[k], d));
    }
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 3; ++k) {
      atomicMin(cb + k, ord_of(cl[k]));
      atomicMax(cb + 3 + k, ord_of(ch[k]));
    }
}

__global__ void k_morton(const float4 *lo, const float4 *hi, uint32_t n, const uint32_t *cb, MortonKey *keys,
                         uint32_t *vals) {
  float cmin[3], ext[3];
  for (int k = 0; k < 3; ++k) {
    cmin[k] = float_of(cb[k]);
    ext[k] = float_of(cb[3 + k]) - cmin[k];
  }
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 l = lo[i], h = hi[i];
    float c[3] = {(l.x + h.x) * 0.5f, (l.y + h.y) * 0.5f, (l.z + h.z) * 0.5f};
    uint32_t q[3];
    for (int k = 0; k < 3; ++k) {
      float x = ext[k] > 0.0f ? (c[k] - cmin[k]) / ext[k] : 0.0f;
      if (!(x >= 0.0f)) x = 0.0f;
      x = fminf(x, 1.0f);
      const uint32_t cells = 1u << kMortonAxisBits;
      q[k] = min((uint32_t)(x * (float)cells), cells - 1u);
    }
    keys[i] = (spread_bits(q[0]) << 2) | (spread_bits(q[1]) << 1) | spread_bits(q[2]);
    vals[i] = i;
  }
}

// ---------------------------------------------------------------- clustering
struct Nodes {
  float4 *lo, *hi;
  uint32_t *count;
  float *cost;
  uint32_t *state, *first, *depth;
  int2 *child;  // indexed v - n
  uint32_t n;
};

__global__ void k_leaves(const uint32_t *vals, const float4 *plo, const float4 *phi, Nodes nd, uint32_t *clusters) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nd.n; j += gridDim.x * blockDim.x) {
    uint32_t g = vals[j];
    float4 l = plo[g], h = phi[g];
    nd.lo[j] = l;
    nd.hi[j] = h;
    nd.count[j] = 1;
    nd.cost[j] = kTriangleCost * box_area(l, h);
    nd.state[j] = 0;
    clusters[j] = j;
  }
}

// Nearest neighbour of every cluster within kPlocRadius positions: the
// smallest area of the merged box, ties to the lower position. Under that
// order the globally closest pair is mutual, so every round merges.
// Clustering state on the device, so rounds run back to back without the
// host reading the cluster count in between.
struct PlocState {
  uint32_t m;        // clusters left
  uint32_t merged;   // interior nodes created so far
  uint32_t rounds;   // rounds done (round r created nodes n + round_begin[r-1] ..)
  uint32_t error;    // a round merged nothing
};

__global__ void __launch_bounds__(kThreads) k_nearest(const uint32_t *clusters, const PlocState *ps, const float4 *nlo,
                                                      const float4 *nhi, uint32_t *nn) {
  const uint32_t m = ps->m;
  if (m <= 1 || (uint64_t)blockIdx.x * kThreads >= m) return;
  __shared__ float4 slo[kThreads + 2 * kPlocRadius], shi[kThreads + 2 * kPlocRadius];
  const int64_t b0 = (int64_t)blockIdx.x * kThreads;
  for (int t = threadIdx.x; t < kThreads + 2 * kPlocRadius; t += kThreads) {
    int64_t idx = b0 - kPlocRadius + t;
    if (idx >= 0 && idx < (int64_t)m) {
      uint32_t c = clusters[idx];
      slo[t] = nlo[c];
      shi[t] = nhi[c];
    }
  }
  __syncthreads();
  const int64_t i = b0 + threadIdx.x;
  if (i >= (int64_t)m) return;
  const float4 l = slo[threadIdx.x + kPlocRadius], h = shi[threadIdx.x + kPlocRadius];
  const int64_t j0 = i - kPlocRadius > 0 ? i - kPlocRadius : 0;
  const int64_t j1 = i + kPlocRadius < (int64_t)m - 1 ? i + kPlocRadius : (int64_t)m - 1;
  float best = INFINITY;
  uint32_t best_j = 0xffffffffu;
  for (int64_t j = j0; j <= j1; ++j) {
    if (j == i) continue;
    const int t = (int)(j - b0) + kPlocRadius;
    const float a = box_area(fmin4(l, slo[t]), fmax4(h, shi[t]));
    if (best_j == 0xffffffffu || a < best) {
      best = a;
      best_j = (uint32_t)j;
    }
  }
  nn[i] = best_j;
}

// keep (high word) and merge (low word) flags of every cluster; zeros for
// positions from m up to `bound` (the scan covers the host's bound).
__global__ void k_mark(const uint32_t *nn, const PlocState *ps, uint32_t bound, uint64_t *flags) {
  const uint32_t m = ps->m;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < bound; i += gridDim.x * blockDim.x) {
    if (m <= 1 || i >= m) {
      flags[i] = 0;
      continue;
    }
    uint32_t j = nn[i];
    bool mutual = nn[j] == i;
    uint64_t keep = (mutual && i > j) ? 0u : 1u;
    uint64_t merge = (mutual && i < j) ? 1u : 0u;
    flags[i] = (keep << 32) | merge;
  }
}

__global__ void k_compact(const uint32_t *clusters, uint32_t *next, const PlocState *ps, const uint32_t *nn,
                          const uint64_t *flags, const uint64_t *offs, Nodes nd) {
  const uint32_t m = ps->m, merged_before = ps->merged;
  if (m <= 1) return;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const uint64_t f = flags[i];
    if (!(f >> 32)) continue;
    const uint64_t o = offs[i];
    const uint32_t pos = (uint32_t)(o >> 32);
    if (!(f & 1u)) {
      next[pos] = clusters[i];
      continue;
    }
    const uint32_t a = clusters[i], b = clusters[nn[i]];
    const uint32_t k = merged_before + (uint32_t)o;
    const uint32_t v = nd.n + k;
    const float4 l = fmin4(nd.lo[a], nd.lo[b]), h = fmax4(nd.hi[a], nd.hi[b]);
    const uint32_t cnt = nd.count[a] + nd.count[b];
    const float area = box_area(l, h);
    const float split = kTraversalCost * area + nd.cost[a] + nd.cost[b];
    const float leaf = kTriangleCost * (float)cnt * area;
    const bool collapse = cnt <= kMaxLeafTris && leaf <= split;
    nd.lo[v] = l;
    nd.hi[v] = h;
    nd.count[v] = cnt;
    nd.cost[v] = collapse ? leaf : split;
    nd.state[v] = collapse ? NS_COLLAPSED : 0u;
    nd.child[k] = make_int2((int)a, (int)b);
    next[pos] = v;
  }
}

// Ends a round: the scan total gives the clusters kept and the merges made.
__global__ void k_advance(PlocState *ps, const uint64_t *total, uint32_t *round_begin, uint32_t max_rounds) {
  if (ps->m <= 1 || ps->error) return;
  const uint64_t t = *total;
  const uint32_t kept = (uint32_t)(t >> 32), merges = (uint32_t)t;
  if (merges == 0 || kept + merges != ps->m || ps->rounds >= max_rounds) {
    ps->error = 1;
    ps->m = 1;
    return;
  }
  ps->merged += merges;
  ps->m = kept;
  ps->rounds += 1;
  round_begin[ps->rounds] = ps->merged;
}

// ---------------------------------------------------------------- layouts
__device__ __forceinline__ bool interior(const Nodes &nd, uint32_t c) {
  return c >= nd.n && !(nd.state[c] & NS_COLLAPSED);
}

// Children of the four-child node of interior node v: start from its two
// children and open the interior child of largest surface area until there
// are four (or none is left to open).
__device__ int wide_children(const Nodes &nd, uint32_t v, uint32_t ch[4]) {
  const int2 c = nd.child[v - nd.n];
  ch[0] = (uint32_t)c.x;
  ch[1] = (uint32_t)c.y;
  int nch = 2;
  while (nch < 4) {
    int best = -1;
    float best_area = -1.0f;
    for (int i = 0; i < nch; ++i) {
      if (!interior(nd, ch[i])) continue;
      float a = box_area(nd.lo[ch[i]], nd.hi[ch[i]]);
      if (a > best_area) {
        best_area = a;
        best = i;
      }
    }
    if (best < 0) break;
    const int2 oc = nd.child[ch[best] - nd.n];
    for (int i = nch; i > best + 1; --i) ch[i] = ch[i - 1];
    ch[best] = (uint32_t)oc.x;
    ch[best + 1] = (uint32_t)oc.y;
    ++nch;
  }
  return nch;
}

__global__ void k_root(Nodes nd, uint32_t root) {
  nd.first[root] = 0;
  nd.depth[root] = 0;
  nd.state[root] |= NS_WIDE;
}

// Top-down pass over the interior nodes of one clustering round (parents of
// later rounds are done): record offsets, depths, coverage by a collapsed
// ancestor, and the four-child node marks.
__global__ void k_topdown(Nodes nd, uint32_t v0, uint32_t v1, uint32_t *max_depth, uint32_t *leaves) {
  for (uint32_t v = v0 + blockIdx.x * blockDim.x + threadIdx.x; v < v1; v += gridDim.x * blockDim.x) {
    const uint32_t st = nd.state[v];
    const int2 c = nd.child[v - nd.n];
    const uint32_t a = (uint32_t)c.x, b = (uint32_t)c.y;
    const uint32_t f = nd.first[v], d = nd.depth[v];
    nd.first[a] = f;
    nd.first[b] = f + nd.count[a];
    nd.depth[a] = d + 1;
    nd.depth[b] = d + 1;
    if (st & (NS_COVERED | NS_COLLAPSED)) {
      nd.state[a] |= NS_COVERED;
      nd.state[b] |= NS_COVERED;
      continue;
    }
    uint32_t leaf_kids = 0;
    if (!interior(nd, a)) ++leaf_kids;
    if (!interior(nd, b)) ++leaf_kids;
    if (leaf_kids) {
      atomicMax(max_depth, d + 1);
      atomicAdd(leaves, leaf_kids);
    }
    if (st & NS_WIDE) {
      uint32_t ch[4];
      const int nch = wide_children(nd, v, ch);
      for (int i = 0; i < nch; ++i)
        if (interior(nd, ch[i])) nd.state[ch[i]] |= NS_WIDE;
    }
  }
}

// In decreasing id order: (two-child node) << 32 | (four-child node).
__global__ void k_layout_flags(Nodes nd, uint64_t *flags) {
  const uint32_t m = nd.n - 1;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < m; p += gridDim.x * blockDim.x) {
    const uint32_t v = 2 * nd.n - 2 - p;
    const uint32_t st = nd.state[v];
    const uint64_t two = (st & (NS_COVERED | NS_COLLAPSED)) ? 0u : 1u;
    const uint64_t four = (two && (st & NS_WIDE)) ? 1u : 0u;
    flags[p] = (two << 32) | four;
  }
}

__device__ __forceinline__ void pad_box(float4 lo, float4 hi, float plo[3], float phi[3]) {
  const float l[3] = {lo.x, lo.y, lo.z}, h[3] = {hi.x, hi.y, hi.z};
  float ext = 0.0f;
  for (int k = 0; k < 3; ++k) ext = fmaxf(fmaxf(ext, h[k] - l[k]), fmaxf(fabsf(l[k]), fabsf(h[k])));
  const float pad = ext * 1.0e-5f + 1.0e-30f;
  for (int k = 0; k < 3; ++k) {
    plo[k] = l[k] - pad;
    phi[k] = h[k] + pad;
  }
}

// Reference to child c from a two-child node (`wide` false: the index in
// the two-child array) or a four-child node (the index in the four-child
// array); leaves encode their record range.
__device__ __forceinline__ int child_ref(const Nodes &nd, const uint64_t *offs, uint32_t c, bool wide,
                                         uint32_t &count) {
  if (interior(nd, c)) {
    count = 0;
    const uint64_t o = offs[2 * nd.n - 2 - c];
    return (int)(wide ? (uint32_t)o : (uint32_t)(o >> 32));
  }
  count = nd.count[c];
  return (int)~(nd.first[c] | (count << kLeafShift));
}

__global__ void k_write_nodes(Nodes nd, const uint64_t *offs, BvhNode *out2, Bvh4Node *out4) {
  const uint32_t m = nd.n - 1;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < m; p += gridDim.x * blockDim.x) {
    const uint32_t v = 2 * nd.n - 2 - p;
    const uint32_t st = nd.state[v];
    if (st & (NS_COVERED | NS_COLLAPSED)) continue;
    const uint64_t o = offs[p];
    const int2 c = nd.child[v - nd.n];
    {
      float l0[3], h0[3], l1[3], h1[3];
      pad_box(nd.lo[c.x], nd.hi[c.x], l0, h0);
      pad_box(nd.lo[c.y], nd.hi[c.y], l1, h1);
      uint32_t n0, n1;
      const int r0 = child_ref(nd, offs, (uint32_t)c.x, false, n0), r1 = child_ref(nd, offs, (uint32_t)c.y, false, n1);
      BvhNode g;
      g.a = make_float4(l0[0], h0[0], l0[1], h0[1]);
      g.b = make_float4(l1[0], h1[0], l1[1], h1[1]);
      g.c = make_float4(l0[2], h0[2], l1[2], h1[2]);
      g.d = make_int4(r0, r1, (int)n0, (int)n1);
      out2[o >> 32] = g;
    }
    if (st & NS_WIDE) {
      uint32_t ch[4];
      const int nch = wide_children(nd, v, ch);
      float bl[3][4], bh[3][4];
      int ref[4];
      for (int i = 0; i < 4; ++i) {
        if (i < nch) {
          float l[3], h[3];
          pad_box(nd.lo[ch[i]], nd.hi[ch[i]], l, h);
          for (int k = 0; k < 3; ++k) {
            bl[k][i] = l[k];
            bh[k][i] = h[k];
          }
          uint32_t cnt;
          ref[i] = child_ref(nd, offs, ch[i], true, cnt);
        } else {
          for (int k = 0; k < 3; ++k) {
            bl[k][i] = INFINITY;
            bh[k][i] = -INFINITY;
          }
          ref[i] = kEmptyChild;
        }
      }
      Bvh4Node q;
      q.lo_x = make_float4(bl[0][0], bl[0][1], bl[0][2], bl[0][3]);
      q.hi_x = make_float4(bh[0][0], bh[0][1], bh[0][2], bh[0][3]);
      q.lo_y = make_float4(bl[1][0], bl[1][1], bl[1][2], bl[1][3]);
      q.hi_y = make_float4(bh[1][0], bh[1][1], bh[1][2], bh[1][3]);
      q.lo_z = make_float4(bl[2][0], bl[2][1], bl[2][2], bl[2][3]);
      q.hi_z = make_float4(bh[2][0], bh[2][1], bh[2][2], bh[2][3]);
      q.child = make_int4(ref[0], ref[1], ref[2], ref[3]);
      q.pad = make_int4(0, 0, 0, 0);
      out4[(uint32_t)o] = q;
    }
  }
}

// Leaf-ordered triangle records: (v0, global id), (v1, REC_* flags), (v2, 0).
__global__ void k_write_records(Nodes nd, const uint32_t *vals, const float *pos, const uint2 *tri_info,
                                const DevMaterial *materials, float4 *records) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nd.n; j += gridDim.x * blockDim.x) {
    const uint32_t g = vals[j];
    const uint32_t r = nd.first[j];
    const float *p = pos + 9ull * g;
    const pt_material &m = materials[__ldg(&tri_info[g].x)].m;
    const uint32_t fl = (m.alpha_mode == PT_ALPHA_OPAQUE ? REC_OPAQUE : 0u) | (m.double_sided ? REC_DOUBLE_SIDED : 0u);
    records[3ull * r] = make_float4(p[0], p[1], p[2], __uint_as_float(g));
    records[3ull * r + 1] = make_float4(p[3], p[4], p[5], __uint_as_float(fl));
    records[3ull * r + 2] = make_float4(p[6], p[7], p[8], 0.0f);
  }
}

// ---------------------------------------------------------------- binned SAH, top down
// The host builder's split rule, level by level on the device: per active
// node the bounds of its triangles and centroids, 16 bins per axis of the
// centroid extent, the sweep for the cheapest split (cost 1 + (A_L n_L +
// A_R n_R) / A_parent, leaf when at most 8 triangles cost no more), a
// stable partition, the children. Nodes near the depth limit, or without a
// valid split, halve their range by index.
constexpr int kSahBins = 16;
constexpr uint32_t kSahNone = 0xffffffffu;
constexpr uint32_t kSahHalve = 0xfffffffeu;
constexpr int kSahBinWords = 3 * kSahBins * 7;  // per axis and bin: count, lo.xyz, hi.xyz

struct SahNodes {
  float4 *lo, *hi;          // node bounds
  uint32_t *begin, *count;  // triangle range
  uint32_t *depth;
  int *left;                // first of two consecutive children, -1 for a leaf
  uint32_t *state;          // NS_WIDE marks (four-child layout)
};

struct SahLevel {
  const uint32_t *act;  // active node ids, ranges in increasing order
  uint32_t m;           // active nodes
  uint32_t *bnd;        // 12 per active node: ord(lo), ord(hi), ord(clo), ord(chi)
  uint32_t *bins;       // kSahBinWords per active node
  uint32_t *split;      // per active node: axis << 8 | bin, kSahNone (leaf) or kSahHalve
};

// Builder::area of the host build (0 for an empty or NaN box).
__device__ __forceinline__ float host_area(float4 lo, float4 hi) {
  float dx = hi.x - lo.x, dy = hi.y - lo.y, dz = hi.z - lo.z;
  if (!(dx >= 0.0f) || !(dy >= 0.0f) || !(dz >= 0.0f)) return 0.0f;
  return dx * dy + dy * dz + dz * dx;
}

// Bin of a centroid offset times the bin scale: truncation, clamped to the
// bins (a NaN offset lands in bin 0).
__device__ __forceinline__ int sah_bin(float f) { return f >= 1.0f ? min(kSahBins - 1, (int)fminf(f, 16.0f)) : 0; }

// Active node of every triangle (binary search of the sorted ranges).
__global__ void k_sah_seg(SahNodes nd, SahLevel lv, uint32_t n, uint32_t *seg) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = lv.m;
    while (hi - lo > 1) {
      uint32_t mid = (lo + hi) >> 1;
      if (nd.begin[lv.act[mid]] <= i)
        lo = mid;
      else
        hi = mid;
    }
    const uint32_t v = lv.act[lo];
    seg[i] = (i >= nd.begin[v] && i < nd.begin[v] + nd.count[v]) ? lo : kSahNone;
  }
}

__device__ __forceinline__ void prim_box(const float4 *plo, const float4 *phi, uint32_t i, float l[3], float h[3],
                                         float c[3]) {
  const float4 a = plo[i], b = phi[i];
  l[0] = a.x, l[1] = a.y, l[2] = a.z;
  h[0] = b.x, h[1] = b.y, h[2] = b.z;
  for (int k = 0; k < 3; ++k) c[k] = (l[k] + h[k]) * 0.5f;
}

// Bounds of every active node: a warp whose 32 triangles share a node
// reduces them first (one atomic per bound), others update per lane.
__global__ void k_sah_bounds(const float4 *plo, const float4 *phi, const uint32_t *seg, uint32_t n, SahLevel lv) {
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t s = i < n ? seg[i] : kSahNone;
    float l[3] = {INFINITY, INFINITY, INFINITY}, h[3] = {-INFINITY, -INFINITY, -INFINITY};
    float cl[3] = {INFINITY, INFINITY, INFINITY}, ch[3] = {-INFINITY, -INFINITY, -INFINITY};
    if (s != kSahNone) {
      float c[3];
      prim_box(plo, phi, i, l, h, c);
      for (int k = 0; k < 3; ++k)
        if (isfinite(c[0]) && isfinite(c[1]) && isfinite(c[2])) cl[k] = ch[k] = c[k];
    }
    const uint32_t s0 = __shfl_sync(0xffffffffu, s, 0);
    if (__all_sync(0xffffffffu, s == s0)) {
      if (s0 == kSahNone) continue;
      for (int k = 0; k < 3; ++k)
        for (int d = 16; d > 0; d >>= 1) {
          l[k] = fminf(l[k], __shfl_xor_sync(0xffffffffu, l[k], d));
          h[k] = fmaxf(h[k], __shfl_xor_sync(0xffffffffu, h[k], d));
          cl[k] = fminf(cl[k], __shfl_xor_sync(0xffffffffu, cl[k], d));
          ch[k] = fmaxf(ch[k], __shfl_xor_sync(0xffffffffu, ch[k], d));
        }
      if ((threadIdx.x & 31) != 0) continue;
    } else if (s == kSahNone) {
      continue;
    }
    uint32_t *b = lv.bnd + 12ull * s;
    for (int k = 0; k < 3; ++k) {
      atomicMin(b + k, ord_of(l[k]));
      atomicMax(b + 3 + k, ord_of(h[k]));
      atomicMin(b + 6 + k, ord_of(cl[k]));
      atomicMax(b + 9 + k, ord_of(ch[k]));
    }
  }
}

__device__ __forceinline__ void node_binning(const uint32_t *b, float clo[3], float scale[3], bool use[3]) {
  for (int k = 0; k < 3; ++k) {
    clo[k] = float_of(b[6 + k]);
    float span = float_of(b[9 + k]) - clo[k];
    use[k] = span > 0.0f;
    scale[k] = use[k] ? (float)kSahBins / span : 0.0f;
  }
}

// Bin counts and bounds: a tile of triangles of one node accumulates in
// shared memory and flushes once; tiles spanning several nodes (small
// nodes) update the nodes' bins directly.
__global__ void __launch_bounds__(kThreads) k_sah_bins(const float4 *plo, const float4 *phi, const uint32_t *seg,
                                                       uint32_t n, SahLevel lv) {
  __shared__ uint32_t sb[kSahBinWords];
  constexpr uint32_t kTile = kThreads * 8;
  for (uint32_t t0 = blockIdx.x * kTile; t0 < n; t0 += gridDim.x * kTile) {
    const uint32_t t1 = min(n, t0 + kTile);
    const uint32_t sa = seg[t0], sz = seg[t1 - 1];
    const bool uniform = sa == sz && sa != kSahNone;
    if (uniform) {
      for (int w = threadIdx.x; w < kSahBinWords; w += kThreads) {
        const int f = w % 7;
        sb[w] = (f >= 1 && f <= 3) ? 0xffffffffu : 0u;
      }
      __syncthreads();
    }
    for (uint32_t i = t0 + threadIdx.x; i < t1; i += kThreads) {
      const uint32_t s = seg[i];
      if (s == kSahNone) continue;
      float clo[3], scale[3];
      bool use[3];
      node_binning(lv.bnd + 12ull * s, clo, scale, use);
      float l[3], h[3], c[3];
      prim_box(plo, phi, i, l, h, c);
      uint32_t *dst = uniform ? sb : lv.bins + (uint64_t)kSahBinWords * s;
      for (int k = 0; k < 3; ++k) {
        if (!use[k]) continue;
        const int bin = sah_bin((c[k] - clo[k]) * scale[k]);
        uint32_t *w = dst + (k * kSahBins + bin) * 7;
        atomicAdd(w, 1u);
        for (int a = 0; a < 3; ++a) {
          atomicMin(w + 1 + a, ord_of(l[a]));
          atomicMax(w + 4 + a, ord_of(h[a]));
        }
      }
    }
    if (uniform) {
      __syncthreads();
      uint32_t *g = lv.bins + (uint64_t)kSahBinWords * sa;
      for (int w = threadIdx.x; w < kSahBinWords; w += kThreads) {
        const int f = w % 7;
        if (f == 0) {
          if (sb[w]) atomicAdd(g + w, sb[w]);
        } else if (f <= 3) {
          if (sb[w] != 0xffffffffu) atomicMin(g + w, sb[w]);
        } else if (sb[w]) {
          atomicMax(g + w, sb[w]);
        }
      }
      __syncthreads();
    }
  }
}

__global__ void k_sah_init_bins(SahLevel lv) {
  const uint64_t total = (uint64_t)lv.m * kSahBinWords;
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
    const int f = (int)(w % 7);
    lv.bins[w] = (f >= 1 && f <= 3) ? 0xffffffffu : 0u;
  }
  const uint64_t tb = (uint64_t)lv.m * 12;
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < tb; w += (uint64_t)gridDim.x * blockDim.x) {
    const int f = (int)(w % 12);
    lv.bnd[w] = (f < 3 || (f >= 6 && f < 9)) ? 0xffffffffu : 0u;
  }
}

// The split of every active node (the host builder's sweep).
__global__ void k_sah_split(SahNodes nd, SahLevel lv, uint32_t *max_depth) {
  for (uint32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < lv.m; a += gridDim.x * blockDim.x) {
    const uint32_t v = lv.act[a];
    const uint32_t *b = lv.bnd + 12ull * a;
    const float4 lo = make_float4(float_of(b[0]), float_of(b[1]), float_of(b[2]), 0.0f);
    const float4 hi = make_float4(float_of(b[3]), float_of(b[4]), float_of(b[5]), 0.0f);
    nd.lo[v] = lo;
    nd.hi[v] = hi;
    const uint32_t cnt = nd.count[v], depth = nd.depth[v];
    if (cnt <= 1) {
      lv.split[a] = kSahNone;
      atomicMax(max_depth, depth);
      continue;
    }
    uint32_t need = 0;
    for (uint32_t c = cnt; c > kMaxLeafTris; c = (c + 1) / 2) ++need;
    const bool median = depth + need >= 56;
    int axis = -1, best_bin = 0;
    float best_cost = INFINITY;
    if (!median) {
      const float parent = host_area(lo, hi);
      bool use[3];
      float clo[3], scale[3];
      node_binning(b, clo, scale, use);
      const uint32_t *bins = lv.bins + (uint64_t)kSahBinWords * a;
      for (int k = 0; k < 3; ++k) {
        if (!use[k]) continue;
        float rl[kSahBins][3], rh[kSahBins][3];
        uint32_t rc[kSahBins];
        float accl[3] = {INFINITY, INFINITY, INFINITY}, acch[3] = {-INFINITY, -INFINITY, -INFINITY};
        uint32_t acc = 0;
        for (int bb = kSahBins - 1; bb >= 1; --bb) {
          const uint32_t *w = bins + (k * kSahBins + bb) * 7;
          acc += w[0];
          if (w[0])
            for (int q = 0; q < 3; ++q) {
              accl[q] = fminf(accl[q], float_of(w[1 + q]));
              acch[q] = fmaxf(acch[q], float_of(w[4 + q]));
            }
          rc[bb] = acc;
          for (int q = 0; q < 3; ++q) {
            rl[bb][q] = accl[q];
            rh[bb][q] = acch[q];
          }
        }
        float ll[3] = {INFINITY, INFINITY, INFINITY}, lh[3] = {-INFINITY, -INFINITY, -INFINITY};
        uint32_t lc = 0;
        for (int s = 1; s < kSahBins; ++s) {
          const uint32_t *w = bins + (k * kSahBins + s - 1) * 7;
          lc += w[0];
          if (w[0])
            for (int q = 0; q < 3; ++q) {
              ll[q] = fminf(ll[q], float_of(w[1 + q]));
              lh[q] = fmaxf(lh[q], float_of(w[4 + q]));
            }
          if (lc == 0 || rc[s] == 0) continue;
          const float4 l4 = make_float4(ll[0], ll[1], ll[2], 0.0f), h4 = make_float4(lh[0], lh[1], lh[2], 0.0f);
          const float4 r4l = make_float4(rl[s][0], rl[s][1], rl[s][2], 0.0f);
          const float4 r4h = make_float4(rh[s][0], rh[s][1], rh[s][2], 0.0f);
          const float cost =
              1.0f + (host_area(l4, h4) * (float)lc + host_area(r4l, r4h) * (float)rc[s]) / fmaxf(parent, 1e-30f);
          if (cost < best_cost) {
            best_cost = cost;
            axis = k;
            best_bin = s;
          }
        }
      }
      if (cnt <= kMaxLeafTris && (axis < 0 || (float)cnt <= best_cost)) {
        lv.split[a] = kSahNone;
        atomicMax(max_depth, depth);
        continue;
      }
    }
    lv.split[a] = axis >= 0 ? ((uint32_t)axis << 8 | (uint32_t)best_bin) : kSahHalve;
  }
}

// Left flags of the triangles of SAH-split nodes.
__global__ void k_sah_flags(const float4 *plo, const float4 *phi, const uint32_t *seg, uint32_t n, SahLevel lv,
                            uint32_t *flag) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t s = seg[i];
    uint32_t f = 0;
    if (s != kSahNone) {
      const uint32_t sp = lv.split[s];
      if (sp < kSahHalve) {
        const int axis = (int)(sp >> 8), bin = (int)(sp & 0xffu);
        float clo[3], scale[3];
        bool use[3];
        node_binning(lv.bnd + 12ull * s, clo, scale, use);
        float l[3], h[3], c[3];
        prim_box(plo, phi, i, l, h, c);
        f = sah_bin((c[axis] - clo[axis]) * scale[axis]) < bin ? 1u : 0u;
      }
    }
    flag[i] = f;
  }
}

// Left triangles of a split node's range from the exclusive scan of the
// flags (`end` may be n).
__device__ __forceinline__ uint32_t left_count(const uint32_t *scan, const uint32_t *flag, uint32_t n, uint32_t b0,
                                               uint32_t e0) {
  return (e0 < n ? scan[e0] : scan[n - 1] + flag[n - 1]) - scan[b0];
}

// Stable partition of the split nodes' ranges (others keep their order).
__global__ void k_sah_scatter(const float4 *plo, const float4 *phi, float4 *qlo, float4 *qhi, const uint32_t *seg,
                              const uint32_t *flag, const uint32_t *scan, uint32_t n, SahNodes nd, SahLevel lv) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t s = seg[i];
    uint32_t dst = i;
    if (s != kSahNone && lv.split[s] < kSahHalve) {
      const uint32_t v = lv.act[s], b0 = nd.begin[v], e0 = b0 + nd.count[v];
      const uint32_t total_left = left_count(scan, flag, n, b0, e0);
      const uint32_t lrank = scan[i] - scan[b0];
      dst = flag[i] ? b0 + lrank : b0 + total_left + (i - b0 - lrank);
    }
    qlo[dst] = plo[i];
    qhi[dst] = phi[i];
  }
}

__global__ void k_sah_split_flags(SahLevel lv, uint32_t *out) {
  for (uint32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < lv.m; a += gridDim.x * blockDim.x)
    out[a] = lv.split[a] != kSahNone ? 1u : 0u;
}

// Children of the split nodes: ids from a scan of the split flags.
__global__ void k_sah_children(SahNodes nd, SahLevel lv, const uint32_t *split_scan, uint32_t next_id,
                               const uint32_t *scan, const uint32_t *flag, uint32_t n, uint32_t *next_act) {
  for (uint32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < lv.m; a += gridDim.x * blockDim.x) {
    const uint32_t v = lv.act[a], sp = lv.split[a];
    if (sp == kSahNone) {
      nd.left[v] = -1;
      continue;
    }
    const uint32_t b0 = nd.begin[v], cnt = nd.count[v];
    const uint32_t nl = sp == kSahHalve ? cnt / 2 : left_count(scan, flag, n, b0, b0 + cnt);
    const uint32_t k = split_scan[a];
    const uint32_t c = next_id + 2 * k;
    nd.left[v] = (int)c;
    nd.begin[c] = b0;
    nd.count[c] = nl;
    nd.begin[c + 1] = b0 + nl;
    nd.count[c + 1] = cnt - nl;
    nd.depth[c] = nd.depth[c + 1] = nd.depth[v] + 1;
    nd.state[c] = nd.state[c + 1] = 0;
    next_act[2 * k] = c;
    next_act[2 * k + 1] = c + 1;
  }
}

__device__ __forceinline__ bool sah_interior(const SahNodes &nd, uint32_t c) { return nd.left[c] >= 0; }

// Children of the four-child node of interior node v (the host layout's
// rule: open the interior child of largest surface area until four).
__device__ int sah_wide_children(const SahNodes &nd, uint32_t v, uint32_t ch[4]) {
  ch[0] = (uint32_t)nd.left[v];
  ch[1] = ch[0] + 1;
  int nch = 2;
  while (nch < 4) {
    int best = -1;
    float best_area = -1.0f;
    for (int i = 0; i < nch; ++i) {
      if (!sah_interior(nd, ch[i])) continue;
      float a = host_area(nd.lo[ch[i]], nd.hi[ch[i]]);
      if (a > best_area) {
        best_area = a;
        best = i;
      }
    }
    if (best < 0) break;
    const uint32_t oc = (uint32_t)nd.left[ch[best]];
    for (int i = nch; i > best + 1; --i) ch[i] = ch[i - 1];
    ch[best] = oc;
    ch[best + 1] = oc + 1;
    ++nch;
  }
  return nch;
}

// Four-child marks, one level of node ids at a time (parents first).
__global__ void k_sah_mark(SahNodes nd, uint32_t v0, uint32_t v1) {
  for (uint32_t v = v0 + blockIdx.x * blockDim.x + threadIdx.x; v < v1; v += gridDim.x * blockDim.x) {
    if (!sah_interior(nd, v) || !(nd.state[v] & NS_WIDE)) continue;
    uint32_t ch[4];
    const int nch = sah_wide_children(nd, v, ch);
    for (int i = 0; i < nch; ++i)
      if (sah_interior(nd, ch[i])) nd.state[ch[i]] |= NS_WIDE;
  }
}

// (two-child node) << 32 | (four-child node), in id order.
__global__ void k_sah_layout_flags(SahNodes nd, uint32_t total, uint64_t *flags) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < total; v += gridDim.x * blockDim.x) {
    const uint64_t two = sah_interior(nd, v) ? 1u : 0u;
    const uint64_t four = (two && (nd.state[v] & NS_WIDE)) ? 1u : 0u;
    flags[v] = (two << 32) | four;
  }
}

__device__ __forceinline__ int sah_ref(const SahNodes &nd, const uint64_t *offs, uint32_t c, bool wide,
                                       uint32_t &count) {
  if (sah_interior(nd, c)) {
    count = 0;
    const uint64_t o = offs[c];
    return (int)(wide ? (uint32_t)o : (uint32_t)(o >> 32));
  }
  count = nd.count[c];
  return (int)~(nd.begin[c] | (count << kLeafShift));
}

__global__ void k_sah_write_nodes(SahNodes nd, uint32_t total, const uint64_t *offs, BvhNode *out2, Bvh4Node *out4) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < total; v += gridDim.x * blockDim.x) {
    if (!sah_interior(nd, v)) continue;
    const uint64_t o = offs[v];
    const uint32_t c0 = (uint32_t)nd.left[v], c1 = c0 + 1;
    float l0[3], h0[3], l1[3], h1[3];
    pad_box(nd.lo[c0], nd.hi[c0], l0, h0);
    pad_box(nd.lo[c1], nd.hi[c1], l1, h1);
    uint32_t n0, n1;
    const int r0 = sah_ref(nd, offs, c0, false, n0), r1 = sah_ref(nd, offs, c1, false, n1);
    BvhNode g;
    g.a = make_float4(l0[0], h0[0], l0[1], h0[1]);
    g.b = make_float4(l1[0], h1[0], l1[1], h1[1]);
    g.c = make_float4(l0[2], h0[2], l1[2], h1[2]);
    g.d = make_int4(r0, r1, (int)n0, (int)n1);
    out2[o >> 32] = g;
    if (!(nd.state[v] & NS_WIDE)) continue;
    uint32_t ch[4];
    const int nch = sah_wide_children(nd, v, ch);
    float bl[3][4], bh[3][4];
    int ref[4];
    for (int i = 0; i < 4; ++i) {
      if (i < nch) {
        float l[3], h[3];
        pad_box(nd.lo[ch[i]], nd.hi[ch[i]], l, h);
        for (int k = 0; k < 3; ++k) {
          bl[k][i] = l[k];
          bh[k][i] = h[k];
        }
        uint32_t cnt;
        ref[i] = sah_ref(nd, offs, ch[i], true, cnt);
      } else {
        for (int k = 0; k < 3; ++k) {
          bl[k][i] = INFINITY;
          bh[k][i] = -INFINITY;
        }
        ref[i] = kEmptyChild;
      }
    }
    Bvh4Node q;
    q.lo_x = make_float4(bl[0][0], bl[0][1], bl[0][2], bl[0][3]);
    q.hi_x = make_float4(bh[0][0], bh[0][1], bh[0][2], bh[0][3]);
    q.lo_y = make_float4(bl[1][0], bl[1][1], bl[1][2], bl[1][3]);
    q.hi_y = make_float4(bh[1][0], bh[1][1], bh[1][2], bh[1][3]);
    q.lo_z = make_float4(bl[2][0], bl[2][1], bl[2][2], bl[2][3]);
    q.hi_z = make_float4(bh[2][0], bh[2][1], bh[2][2], bh[2][3]);
    q.child = make_int4(ref[0], ref[1], ref[2], ref[3]);
    q.pad = make_int4(0, 0, 0, 0);
    out4[(uint32_t)o] = q;
  }
}

// Triangle boxes (min / max of the three corners, as the host build), with
// the global id in lo.w.
__global__ void k_sah_prims(const float *pos, uint32_t n, float4 *lo, float4 *hi) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float *p = pos + 9ull * i;
    float l[3], h[3];
    bool nan = false;
    for (int k = 0; k < 3; ++k) {
      const float a = __ldg(p + k), b = __ldg(p + 3 + k), c = __ldg(p + 6 + k);
      nan |= isnan(a) || isnan(b) || isnan(c);
      l[k] = fminf(fminf(a, b), c);
      h[k] = fmaxf(fmaxf(a, b), c);
    }
    if (nan)  // never hit: an empty box, outside every node's bounds
      for (int k = 0; k < 3; ++k) {
        l[k] = INFINITY;
        h[k] = -INFINITY;
      }
    lo[i] = make_float4(l[0], l[1], l[2], __uint_as_float(i));
    hi[i] = make_float4(h[0], h[1], h[2], 0.0f);
  }
}

__global__ void k_sah_records(const float4 *plo, uint32_t n, const float *pos, const uint2 *tri_info,
                              const DevMaterial *materials, float4 *records) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const uint32_t g = __float_as_uint(plo[r].w);
    const float *p = pos + 9ull * g;
    const pt_material &m = materials[__ldg(&tri_info[g].x)].m;
    const uint32_t fl = (m.alpha_mode == PT_ALPHA_OPAQUE ? REC_OPAQUE : 0u) | (m.double_sided ? REC_DOUBLE_SIDED : 0u);
    records[3ull * r] = make_float4(p[0], p[1], p[2], __uint_as_float(g));
    records[3ull * r + 1] = make_float4(p[3], p[4], p[5], __uint_as_float(fl));
    records[3ull * r + 2] = make_float4(p[6], p[7], p[8], 0.0f);
  }
}

// ---- small subtrees: nodes of at most kSahSmall triangles leave the level
// rounds and are built whole by one thread each (the same split rule, an
// in-place partition), in node ids reserved for them (2c - 2 per node of c
// triangles; unused ids stay empty leaves that nothing references).
constexpr uint32_t kSahSmall = 32;

// Splits the children of the last round into the next round's active list
// and the deferred (small) list: flags, then a scatter after their scan.
__global__ void k_sah_route_flags(const uint32_t *kids, uint32_t nk, SahNodes nd, uint32_t *flag) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nk; k += gridDim.x * blockDim.x)
    flag[k] = nd.count[kids[k]] > kSahSmall ? 1u : 0u;
}
__global__ void k_sah_route(const uint32_t *kids, uint32_t nk, const uint32_t *flag, const uint32_t *scan,
                            uint32_t *act_next, uint32_t *deferred, uint32_t def_base) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nk; k += gridDim.x * blockDim.x) {
    if (flag[k])
      act_next[scan[k]] = kids[k];
    else
      deferred[def_base + (k - scan[k])] = kids[k];
  }
}

__global__ void k_sah_small_reserve(const uint32_t *deferred, uint32_t nd_count, SahNodes nd, uint32_t *need) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nd_count; k += gridDim.x * blockDim.x) {
    const uint32_t c = nd.count[deferred[k]];
    need[k] = c > 1 ? 2 * c - 2 : 0;
  }
}

__global__ void k_add_base(uint32_t *v, uint32_t n, uint32_t base) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) v[k] += base;
}

__global__ void k_sah_small_clear(SahNodes nd, uint32_t v0, uint32_t v1) {
  for (uint32_t v = v0 + blockIdx.x * blockDim.x + threadIdx.x; v < v1; v += gridDim.x * blockDim.x) {
    nd.lo[v] = make_float4(INFINITY, INFINITY, INFINITY, 0.0f);
    nd.hi[v] = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.0f);
    nd.begin[v] = 0;
    nd.count[v] = 0;
    nd.depth[v] = 0;
    nd.left[v] = -1;
    nd.state[v] = 0;
  }
}

// The whole subtree of one small node, depth first (the host builder's
// split of a node, sequentially: bounds, 16 bins per axis, the sweep, leaf
// or split, then an in-place partition).
__global__ void k_sah_small(const uint32_t *deferred, uint32_t nd_count, const uint32_t *first_id, SahNodes nd,
                            float4 *plo, float4 *phi, uint32_t *used, uint32_t *max_depth) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nd_count; k += gridDim.x * blockDim.x) {
    const uint32_t root = deferred[k];
    uint32_t next = first_id[k];
    const uint32_t id0 = next;
    struct Task {
      uint32_t v, b, c, d;
    } st[2 * kSahSmall];
    int sp = 0;
    st[sp++] = {root, nd.begin[root], nd.count[root], nd.depth[root]};
    while (sp > 0) {
      const Task t = st[--sp];
      float4 lo = make_float4(INFINITY, INFINITY, INFINITY, 0.0f), hi = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.0f);
      float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
      for (uint32_t i = t.b; i < t.b + t.c; ++i) {
        float l[3], h[3], c[3];
        prim_box(plo, phi, i, l, h, c);
        lo = make_float4(fminf(lo.x, l[0]), fminf(lo.y, l[1]), fminf(lo.z, l[2]), 0.0f);
        hi = make_float4(fmaxf(hi.x, h[0]), fmaxf(hi.y, h[1]), fmaxf(hi.z, h[2]), 0.0f);
        if (isfinite(c[0]) && isfinite(c[1]) && isfinite(c[2]))
          for (int q = 0; q < 3; ++q) {
            clo[q] = fminf(clo[q], c[q]);
            chi[q] = fmaxf(chi[q], c[q]);
          }
      }
      nd.lo[t.v] = lo;
      nd.hi[t.v] = hi;
      nd.left[t.v] = -1;
      if (t.c <= 1) {
        atomicMax(max_depth, t.d);
        continue;
      }
      uint32_t need = 0;
      for (uint32_t c = t.c; c > kMaxLeafTris; c = (c + 1) / 2) ++need;
      const bool median = t.d + need >= 56;
      int axis = -1, best_bin = 0;
      float best_cost = INFINITY, scale[3] = {0.0f, 0.0f, 0.0f};
      if (!median) {
        const float parent = host_area(lo, hi);
        for (int ax = 0; ax < 3; ++ax) {
          const float span = chi[ax] - clo[ax];
          if (!(span > 0.0f)) continue;
          scale[ax] = (float)kSahBins / span;
          uint32_t bc[kSahBins];
          float bl[kSahBins][3], bh[kSahBins][3];
          for (int b = 0; b < kSahBins; ++b) {
            bc[b] = 0;
            for (int q = 0; q < 3; ++q) {
              bl[b][q] = INFINITY;
              bh[b][q] = -INFINITY;
            }
          }
          for (uint32_t i = t.b; i < t.b + t.c; ++i) {
            float l[3], h[3], c[3];
            prim_box(plo, phi, i, l, h, c);
            const int b = sah_bin((c[ax] - clo[ax]) * scale[ax]);
            bc[b]++;
            for (int q = 0; q < 3; ++q) {
              bl[b][q] = fminf(bl[b][q], l[q]);
              bh[b][q] = fmaxf(bh[b][q], h[q]);
            }
          }
          float rl[kSahBins][3], rh[kSahBins][3];
          uint32_t rc[kSahBins];
          float accl[3] = {INFINITY, INFINITY, INFINITY}, acch[3] = {-INFINITY, -INFINITY, -INFINITY};
          uint32_t acc = 0;
          for (int b = kSahBins - 1; b >= 1; --b) {
            acc += bc[b];
            for (int q = 0; q < 3; ++q) {
              accl[q] = fminf(accl[q], bl[b][q]);
              acch[q] = fmaxf(acch[q], bh[b][q]);
              rl[b][q] = accl[q];
              rh[b][q] = acch[q];
            }
            rc[b] = acc;
          }
          float ll[3] = {INFINITY, INFINITY, INFINITY}, lh[3] = {-INFINITY, -INFINITY, -INFINITY};
          uint32_t lc = 0;
          for (int s = 1; s < kSahBins; ++s) {
            lc += bc[s - 1];
            for (int q = 0; q < 3; ++q) {
              ll[q] = fminf(ll[q], bl[s - 1][q]);
              lh[q] = fmaxf(lh[q], bh[s - 1][q]);
            }
            if (lc == 0 || rc[s] == 0) continue;
            const float cost = 1.0f + (host_area(make_float4(ll[0], ll[1], ll[2], 0.0f), make_float4(lh[0], lh[1], lh[2], 0.0f)) *
                                           (float)lc +
                                       host_area(make_float4(rl[s][0], rl[s][1], rl[s][2], 0.0f),
                                                 make_float4(rh[s][0], rh[s][1], rh[s][2], 0.0f)) *
                                           (float)rc[s]) /
                                          fmaxf(parent, 1e-30f);
            if (cost < best_cost) {
              best_cost = cost;
              axis = ax;
              best_bin = s;
            }
          }
        }
        if (t.c <= kMaxLeafTris && (axis < 0 || (float)t.c <= best_cost)) {
          atomicMax(max_depth, t.d);
          continue;
        }
      }
      uint32_t mid;
      if (axis >= 0) {
        uint32_t i = t.b, j = t.b + t.c;  // [t.b, i) left, [j, end) right
        while (i < j) {
          float l[3], h[3], c[3];
          prim_box(plo, phi, i, l, h, c);
          if (sah_bin((c[axis] - clo[axis]) * scale[axis]) < best_bin) {
            ++i;
          } else {
            --j;
            const float4 a = plo[i], b = phi[i];
            plo[i] = plo[j];
            phi[i] = phi[j];
            plo[j] = a;
            phi[j] = b;
          }
        }
        mid = i - t.b;
      } else {
        mid = t.c / 2;
      }
      const uint32_t c0 = next;
      next += 2;
      nd.left[t.v] = (int)c0;
      nd.begin[c0] = t.b;
      nd.count[c0] = mid;
      nd.begin[c0 + 1] = t.b + mid;
      nd.count[c0 + 1] = t.c - mid;
      nd.depth[c0] = nd.depth[c0 + 1] = t.d + 1;
      st[sp++] = {c0 + 1, t.b + mid, t.c - mid, t.d + 1};
      st[sp++] = {c0, t.b, mid, t.d + 1};
    }
    used[k] = next - id0;
  }
}

// Four-child marks inside the small subtrees: the root, then its nodes in
// id order (a parent's id precedes its children's).
__global__ void k_sah_small_mark(const uint32_t *deferred, uint32_t nd_count, const uint32_t *first_id,
                                 const uint32_t *used, SahNodes nd) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nd_count; k += gridDim.x * blockDim.x) {
    const uint32_t root = deferred[k], id0 = first_id[k], id1 = id0 + used[k];
    for (uint32_t w = 0; w <= id1 - id0; ++w) {
      const uint32_t v = w == 0 ? root : id0 + w - 1;
      if (!sah_interior(nd, v) || !(nd.state[v] & NS_WIDE)) continue;
      uint32_t ch[4];
      const int nch = sah_wide_children(nd, v, ch);
      for (int i = 0; i < nch; ++i)
        if (sah_interior(nd, ch[i])) nd.state[ch[i]] |= NS_WIDE;
    }
  }
}

// SAH cost contribution of every node (traversal 1, intersection 1,
// relative to the root box), summed by a scan.
__global__ void k_sah_cost(SahNodes nd, uint32_t total, double *out) {
  const double root = fmax((double)host_area(nd.lo[0], nd.hi[0]), 1e-30);
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < total; v += gridDim.x * blockDim.x) {
    const double a = (double)host_area(nd.lo[v], nd.hi[v]) / root;
    out[v] = sah_interior(nd, v) ? a : a * (double)nd.count[v];
  }
}

__global__ void k_sah_root(SahNodes nd, uint32_t n, uint32_t *act) {
  nd.begin[0] = 0;
  nd.count[0] = n;
  nd.depth[0] = 0;
  nd.state[0] = NS_WIDE;
  act[0] = 0;
}

// ---------------------------------------------------------------- host side
struct Scratch {
  std::vector<void *> ptrs;
  cudaStream_t st;
  bool oom = false;
  std::string err;
  template <class T>
  T *get(uint64_t count) {
    void *p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, std::max<uint64_t>(count, 1) * sizeof(T), st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      if (err.empty()) err = std::string("device BVH scratch allocation failed: ") + cudaGetErrorString(e);
      oom = oom || e == cudaErrorMemoryAllocation;
      return nullptr;
    }
    ptrs.push_back(p);
    return static_cast<T *>(p);
  }
  ~Scratch() {
    for (void *p : ptrs) cudaFreeAsync(p, st);
  }
};

uint64_t align256(uint64_t x) { return (x + 255) & ~uint64_t(255); }

}  // namespace

std::string device_build_bvh_sah(SceneHost &sc, cudaStream_t st, uint32_t max_depth_allowed, bool &oom,
                                 DeviceBuildInfo *info) {
  oom = false;
  const auto t0 = std::chrono::steady_clock::now();
  const uint64_t n64 = sc.tri_count;
  if (n64 < kMinDeviceTris) return "too few triangles for the device builder";
  if (n64 >= (1ull << kLeafShift)) return "too many triangles for the leaf encoding";
  const uint32_t n = (uint32_t)n64;
  const uint32_t cap = 2 * n;  // nodes of a binary tree with non-empty leaves

  Scratch s{{}, st};
  float4 *plo = s.get<float4>(n), *phi = s.get<float4>(n), *qlo = s.get<float4>(n), *qhi = s.get<float4>(n);
  uint32_t *seg = s.get<uint32_t>(n), *flag = s.get<uint32_t>(n), *pscan = s.get<uint32_t>(n);
  uint32_t *scan32 = s.get<uint32_t>(scan_scratch_items(n));
  SahNodes nd;
  nd.lo = s.get<float4>(cap);
  nd.hi = s.get<float4>(cap);
  nd.begin = s.get<uint32_t>(cap);
  nd.count = s.get<uint32_t>(cap);
  nd.depth = s.get<uint32_t>(cap);
  nd.left = s.get<int>(cap);
  nd.state = s.get<uint32_t>(cap);
  uint32_t *act = s.get<uint32_t>(n);
  uint32_t *split = s.get<uint32_t>(n), *split_scan = s.get<uint32_t>(n), *split_flag = s.get<uint32_t>(n);
  uint64_t *flags64 = s.get<uint64_t>(cap), *offs = s.get<uint64_t>(cap);
  uint64_t *scan64 = s.get<uint64_t>(scan_scratch_items(cap));
  uint32_t *counters = s.get<uint32_t>(2);  // max leaf depth
  double *cost = s.get<double>(cap), *cost_scan = s.get<double>(scan_scratch_items(cap));
  uint32_t *kids = s.get<uint32_t>(n), *route = s.get<uint32_t>(n), *route_scan = s.get<uint32_t>(n);
  uint32_t *deferred = s.get<uint32_t>(n), *first_id = s.get<uint32_t>(n), *used = s.get<uint32_t>(n);
  if (!s.err.empty()) {
    oom = s.oom;
    return s.err;
  }
  // Bounds and bins of the widest level so far, grown on demand.
  uint32_t *bnd = nullptr, *bins = nullptr;
  uint32_t level_cap = 0;
  auto grow = [&](uint32_t m) -> bool {
    if (m <= level_cap) return true;
    const uint32_t want = std::max<uint32_t>(m, std::min<uint32_t>(n, level_cap * 2 + 1024));
    bnd = s.get<uint32_t>(12ull * want);
    bins = s.get<uint32_t>((uint64_t)kSahBinWords * want);
    level_cap = want;
    return s.err.empty();
  };

  const float *pos = sc.dev.pos;
  cudaMemsetAsync(counters, 0, 2 * sizeof(uint32_t), st);
  k_sah_prims<<<grid_for(n), kThreads, 0, st>>>(pos, n, plo, phi);
  k_sah_root<<<1, 1, 0, st>>>(nd, n, act);
  std::vector<uint32_t> level_begin{0};
  uint32_t m = 1, next_id = 1, n_deferred = 0;
  while (m > 0) {
    if (level_begin.size() > 64) return "device SAH build exceeded 64 levels";
    if (!grow(m)) {
      oom = s.oom;
      return s.err;
    }
    SahLevel lv{act, m, bnd, bins, split};
    k_sah_init_bins<<<grid_for((uint64_t)m * kSahBinWords), kThreads, 0, st>>>(lv);
    k_sah_seg<<<grid_for(n), kThreads, 0, st>>>(nd, lv, n, seg);
    k_sah_bounds<<<grid_for(n), kThreads, 0, st>>>(plo, phi, seg, n, lv);
    k_sah_bins<<<(unsigned)std::min<uint64_t>(tiles_of(n, kThreads * 8), 1u << 16), kThreads, 0, st>>>(plo, phi, seg,
                                                                                                  n, lv);
    k_sah_split<<<grid_for(m), kThreads, 0, st>>>(nd, lv, counters);
    k_sah_flags<<<grid_for(n), kThreads, 0, st>>>(plo, phi, seg, n, lv, flag);
    scan_exclusive<uint32_t>(flag, pscan, n, scan32, st);
    k_sah_scatter<<<grid_for(n), kThreads, 0, st>>>(plo, phi, qlo, qhi, seg, flag, pscan, n, nd, lv);
    k_sah_split_flags<<<grid_for(m), kThreads, 0, st>>>(lv, split_flag);
    uint32_t *tot = scan_exclusive<uint32_t>(split_flag, split_scan, m, scan32, st);
    k_sah_children<<<grid_for(m), kThreads, 0, st>>>(nd, lv, split_scan, next_id, pscan, flag, n, kids);
    std::swap(plo, qlo);
    std::swap(phi, qhi);
    uint32_t splits = 0;
    cudaError_t e = cudaMemcpyAsync(&splits, tot, sizeof splits, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return std::string("device SAH build: ") + cudaGetErrorString(e);
    if (next_id + 2ull * splits > cap) return "device SAH build ran out of nodes";
    level_begin.push_back(next_id);
    next_id += 2 * splits;
    // The children: large ones stay in the rounds, small ones wait for the
    // subtree kernel.
    const uint32_t nk = 2 * splits;
    uint32_t active = 0;
    if (nk) {
      k_sah_route_flags<<<grid_for(nk), kThreads, 0, st>>>(kids, nk, nd, route);
      uint32_t *rt = scan_exclusive<uint32_t>(route, route_scan, nk, scan32, st);
      k_sah_route<<<grid_for(nk), kThreads, 0, st>>>(kids, nk, route, route_scan, act, deferred, n_deferred);
      e = cudaMemcpyAsync(&active, rt, sizeof active, cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return std::string("device SAH build: ") + cudaGetErrorString(e);
    }
    n_deferred += nk - active;
    m = active;
  }
  // Small subtrees, one thread each, in reserved node ids.
  if (n_deferred) {
    k_sah_small_reserve<<<grid_for(n_deferred), kThreads, 0, st>>>(deferred, n_deferred, nd, route);
    uint32_t *rt = scan_exclusive<uint32_t>(route, first_id, n_deferred, scan32, st);
    uint32_t reserved = 0;
    cudaError_t e = cudaMemcpyAsync(&reserved, rt, sizeof reserved, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return std::string("device SAH build: ") + cudaGetErrorString(e);
    if ((uint64_t)next_id + reserved > cap) return "device SAH build ran out of nodes";
    if (reserved) k_sah_small_clear<<<grid_for(reserved), kThreads, 0, st>>>(nd, next_id, next_id + reserved);
    k_add_base<<<grid_for(n_deferred), kThreads, 0, st>>>(first_id, n_deferred, next_id);
    k_sah_small<<<grid_for(n_deferred, 64), 64, 0, st>>>(deferred, n_deferred, first_id, nd, plo, phi, used, counters);
    next_id += reserved;
  }
  const uint32_t total = next_id;
  // Four-child marks level by level (parents first), then both numberings.
  for (size_t l = 0; l + 1 < level_begin.size(); ++l)
    k_sah_mark<<<grid_for(level_begin[l + 1] - level_begin[l]), kThreads, 0, st>>>(nd, level_begin[l],
                                                                                   level_begin[l + 1]);
  if (n_deferred)
    k_sah_small_mark<<<grid_for(n_deferred, 64), 64, 0, st>>>(deferred, n_deferred, first_id, used, nd);
  k_sah_layout_flags<<<grid_for(total), kThreads, 0, st>>>(nd, total, flags64);
  uint64_t *tot = scan_exclusive<uint64_t>(flags64, offs, total, scan64, st);
  k_sah_cost<<<grid_for(total), kThreads, 0, st>>>(nd, total, cost);
  double *cost_total = scan_exclusive<double>(cost, cost, total, cost_scan, st);
  uint64_t t = 0;
  uint32_t depth = 0;
  double sah_cost = 0.0;
  cudaError_t e = cudaMemcpyAsync(&t, tot, sizeof t, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&sah_cost, cost_total, sizeof sah_cost, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&depth, counters, sizeof depth, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return std::string("device SAH layout: ") + cudaGetErrorString(e);
  const uint32_t n2 = (uint32_t)(t >> 32), n4 = (uint32_t)t;
  if (depth > max_depth_allowed)
    return "depth " + std::to_string(depth) + " of the device-built tree exceeds " + std::to_string(max_depth_allowed);
  if (n2 == 0 || n4 == 0) return "device BVH has no interior node";
  const uint64_t off4 = align256((uint64_t)n2 * sizeof(BvhNode));
  const uint64_t offr = off4 + align256((uint64_t)n4 * sizeof(Bvh4Node));
  const uint64_t bytes = offr + align256(3ull * n * sizeof(float4));
  DeviceArena arena;
  e = cudaMalloc(&arena.base, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    oom = e == cudaErrorMemoryAllocation;
    return std::string("device allocation of ") + std::to_string(bytes) + " BVH bytes failed: " + cudaGetErrorString(e);
  }
  arena.bytes = bytes;
  uint8_t *base = static_cast<uint8_t *>(arena.base);
  BvhNode *out2 = reinterpret_cast<BvhNode *>(base);
  Bvh4Node *out4 = reinterpret_cast<Bvh4Node *>(base + off4);
  float4 *records = reinterpret_cast<float4 *>(base + offr);
  k_sah_write_nodes<<<grid_for(total), kThreads, 0, st>>>(nd, total, offs, out2, out4);
  k_sah_records<<<grid_for(n), kThreads, 0, st>>>(plo, n, pos, sc.dev.tri_info, sc.dev.materials, records);
  DevScene d = sc.dev;
  d.nodes = out2;
  d.nodes4 = out4;
  d.tris = records;
  d.node_count = n2;
  d.node4_count = n4;
  d.max_depth = depth;
  e = cudaMemcpyAsync(sc.d_desc, &d, sizeof d, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    arena.release();
    return std::string("device BVH write: ") + cudaGetErrorString(e);
  }
  sc.dev = d;
  sc.bvh_arena.release();
  sc.bvh_arena = arena;
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  sc.bvh = BvhBuildStats{};
  sc.bvh.references = n;
  sc.bvh.nodes = n2;
  sc.bvh.leaves = n2 + 1;  // a binary tree: one leaf more than interior nodes
  sc.bvh.max_depth = depth;
  sc.bvh.sah_cost = sah_cost;
  sc.bvh.seconds = secs;
  if (info) {
    info->iterations = (uint32_t)level_begin.size() - 1;
    info->ms = 1000.0 * secs;
  }
  return "";
}

std::string device_build_bvh(SceneHost &sc, cudaStream_t st, uint32_t max_depth_allowed, bool &oom,
                             DeviceBuildInfo *info) {
  oom = false;
  const auto t0 = std::chrono::steady_clock::now();
  const uint64_t n64 = sc.tri_count;
  if (n64 < kMinDeviceTris) return "too few triangles for the device builder";
  if (n64 >= (1ull << kLeafShift)) return "too many triangles for the leaf encoding";
  const uint32_t n = (uint32_t)n64;
  const uint32_t total_nodes = 2 * n - 1;

  Scratch s{{}, st};
  float4 *plo = s.get<float4>(n), *phi = s.get<float4>(n);
  uint32_t *cb = s.get<uint32_t>(6);
  MortonKey *keys = s.get<MortonKey>(n), *keys2 = s.get<MortonKey>(n);
  uint32_t *vals = s.get<uint32_t>(n), *vals2 = s.get<uint32_t>(n);
  const uint32_t ntiles = (uint32_t)tiles_of(n, kRadixTile);
  uint32_t *hist = s.get<uint32_t>((uint64_t)kRadixBins * ntiles);
  uint32_t *scan32 = s.get<uint32_t>(scan_scratch_items((uint64_t)kRadixBins * ntiles));
  Nodes nd;
  nd.n = n;
  nd.lo = s.get<float4>(total_nodes);
  nd.hi = s.get<float4>(total_nodes);
  nd.count = s.get<uint32_t>(total_nodes);
  nd.cost = s.get<float>(total_nodes);
  nd.state = s.get<uint32_t>(total_nodes);
  nd.first = s.get<uint32_t>(total_nodes);
  nd.depth = s.get<uint32_t>(total_nodes);
  nd.child = s.get<int2>(n - 1);
  uint32_t *ca = s.get<uint32_t>(n), *cbuf = s.get<uint32_t>(n), *nn = s.get<uint32_t>(n);
  uint64_t *flags = s.get<uint64_t>(n), *offs = s.get<uint64_t>(n);
  uint64_t *scan64 = s.get<uint64_t>(scan_scratch_items(n));
  uint32_t *counters = s.get<uint32_t>(2);  // max depth, leaves
  PlocState *pstate = s.get<PlocState>(1);
  uint32_t *round_dev = s.get<uint32_t>(kMaxRounds + 1);
  if (!s.err.empty()) {
    oom = s.oom;
    return s.err;
  }
  auto check = [&](const char *what) -> std::string {
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? std::string() : std::string(what) + ": " + cudaGetErrorString(e);
  };

  // Boxes, Morton codes, sort.
  const uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
  cudaMemcpyAsync(cb, init, sizeof init, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(counters, 0, 2 * sizeof(uint32_t), st);
  const float *pos = sc.dev.pos;
  k_prim_boxes<<<grid_for(n), kThreads, 0, st>>>(pos, n, plo, phi, cb);
  k_morton<<<grid_for(n), kThreads, 0, st>>>(plo, phi, n, cb, keys, vals);
  for (int shift = 0; shift < kMortonBits; shift += 8) {
    k_radix_hist<<<ntiles, kThreads, 0, st>>>(keys, n, shift, hist, ntiles);
    scan_exclusive<uint32_t>(hist, hist, (uint64_t)kRadixBins * ntiles, scan32, st);
    k_radix_scatter<<<ntiles, kThreads, 0, st>>>(keys, vals, keys2, vals2, n, shift, hist, ntiles);
    std::swap(keys, keys2);
    std::swap(vals, vals2);
  }
  std::string err = check("device BVH sort");
  if (!err.empty()) return err;

  // Clustering rounds, in batches launched back to back; the host reads
  // the cluster count once per batch (grids are sized by that bound).
  k_leaves<<<grid_for(n), kThreads, 0, st>>>(vals, plo, phi, nd, ca);
  PlocState init_state{n, 0, 0, 0};
  cudaMemcpyAsync(pstate, &init_state, sizeof init_state, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(round_dev, 0, sizeof(uint32_t), st);
  uint32_t bound = n;
  PlocState hs = init_state;
  for (uint32_t batch = 0;; ++batch) {
    const uint32_t per_batch = bound > 65536 ? 4 : 16;
    for (uint32_t r = 0; r < per_batch; ++r) {
      k_nearest<<<(unsigned)tiles_of(bound, kThreads), kThreads, 0, st>>>(ca, pstate, nd.lo, nd.hi, nn);
      k_mark<<<grid_for(bound), kThreads, 0, st>>>(nn, pstate, bound, flags);
      uint64_t *tot = scan_exclusive<uint64_t>(flags, offs, bound, scan64, st);
      k_compact<<<grid_for(bound), kThreads, 0, st>>>(ca, cbuf, pstate, nn, flags, offs, nd);
      k_advance<<<1, 1, 0, st>>>(pstate, tot, round_dev, kMaxRounds);
      std::swap(ca, cbuf);
    }
    cudaError_t e = cudaMemcpyAsync(&hs, pstate, sizeof hs, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return std::string("device BVH clustering: ") + cudaGetErrorString(e);
    if (hs.error) return "device BVH clustering made no progress";
    if (hs.m <= 1) break;
    bound = hs.m;
  }
  const uint32_t merged = hs.merged;
  if (merged != n - 1) return "device BVH clustering left more than one root";
  std::vector<uint32_t> round_begin(hs.rounds + 1);
  if (cudaMemcpy(round_begin.data(), round_dev, round_begin.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost) !=
      cudaSuccess)
    return "device BVH clustering: round table read failed";

  // Top-down pass, latest round first.
  const uint32_t root = 2 * n - 2;
  k_root<<<1, 1, 0, st>>>(nd, root);
  for (size_t r = round_begin.size() - 1; r >= 1; --r) {
    const uint32_t v0 = n + round_begin[r - 1], v1 = n + round_begin[r];
    k_topdown<<<grid_for(v1 - v0), kThreads, 0, st>>>(nd, v0, v1, counters, counters + 1);
  }
  k_layout_flags<<<grid_for(n - 1), kThreads, 0, st>>>(nd, flags);
  uint64_t *tot = scan_exclusive<uint64_t>(flags, offs, n - 1, scan64, st);
  uint64_t t = 0;
  uint32_t cnt[2] = {0, 0};
  cudaError_t e = cudaMemcpyAsync(&t, tot, sizeof t, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(cnt, counters, sizeof cnt, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return std::string("device BVH layout: ") + cudaGetErrorString(e);
  const uint32_t n2 = (uint32_t)(t >> 32), n4 = (uint32_t)t;
  if (cnt[0] > max_depth_allowed)
    return "depth " + std::to_string(cnt[0]) + " of the device-built tree exceeds " + std::to_string(max_depth_allowed);
  if (n2 == 0 || n4 == 0) return "device BVH has no interior node";

  // The tree's own allocation: nodes, four-child nodes, records.
  const uint64_t off4 = align256((uint64_t)n2 * sizeof(BvhNode));
  const uint64_t offr = off4 + align256((uint64_t)n4 * sizeof(Bvh4Node));
  const uint64_t bytes = offr + align256(3ull * n * sizeof(float4));
  DeviceArena arena;
  e = cudaMalloc(&arena.base, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    oom = e == cudaErrorMemoryAllocation;
    return std::string("device allocation of ") + std::to_string(bytes) + " BVH bytes failed: " + cudaGetErrorString(e);
  }
  arena.bytes = bytes;
  uint8_t *base = static_cast<uint8_t *>(arena.base);
  BvhNode *out2 = reinterpret_cast<BvhNode *>(base);
  Bvh4Node *out4 = reinterpret_cast<Bvh4Node *>(base + off4);
  float4 *records = reinterpret_cast<float4 *>(base + offr);
  k_write_nodes<<<grid_for(n - 1), kThreads, 0, st>>>(nd, offs, out2, out4);
  k_write_records<<<grid_for(n), kThreads, 0, st>>>(nd, vals, pos, sc.dev.tri_info, sc.dev.materials, records);
  float root_cost = 0.0f;
  float4 rb[2];
  e = cudaMemcpyAsync(&root_cost, nd.cost + root, sizeof root_cost, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&rb[0], nd.lo + root, sizeof(float4), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&rb[1], nd.hi + root, sizeof(float4), cudaMemcpyDeviceToHost, st);
  DevScene d = sc.dev;
  d.nodes = out2;
  d.nodes4 = out4;
  d.tris = records;
  d.node_count = n2;
  d.node4_count = n4;
  d.max_depth = cnt[0];
  if (e == cudaSuccess) e = cudaMemcpyAsync(sc.d_desc, &d, sizeof d, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    arena.release();
    return std::string("device BVH write: ") + cudaGetErrorString(e);
  }
  sc.dev = d;
  sc.bvh_arena.release();
  sc.bvh_arena = arena;
  arena.base = nullptr;  // owned by the scene now
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  sc.bvh = BvhBuildStats{};
  sc.bvh.references = n;
  sc.bvh.nodes = n2;
  sc.bvh.leaves = cnt[1];
  sc.bvh.max_depth = cnt[0];
  const float dx = rb[1].x - rb[0].x, dy = rb[1].y - rb[0].y, dz = rb[1].z - rb[0].z;
  const double ra = (double)dx * dy + (double)dy * dz + (double)dz * dx;
  sc.bvh.sah_cost = ra > 0.0 ? (double)root_cost / ra : 0.0;
  sc.bvh.seconds = secs;
  if (info) {
    info->iterations = (uint32_t)round_begin.size() - 1;
    info->ms = 1000.0 * secs;
  }
  return "";
}

}  // namespace ptd
