// Refit of a resident scene's BVH for an animated frame whose topology is
// unchanged (the same draw items with the same triangle counts, so global
// triangle ids keep their meaning): the tree's structure stays, the
// triangle records are rewritten from the new corner positions and every
// node's child bounds are recomputed bottom up, for both node layouts.
// Closest hits do not depend on the tree (smallest t, ties to the lowest
// global id), so a refitted frame renders exactly as a fresh build of the
// same frame; only the traversal cost may differ.
//
// Bottom-up order without levels: every node counts its interior children;
// a node with none starts at once, and the thread that finishes a node's
// last interior child (an atomic decrement of the parent's count, after a
// fence) goes on to the parent. Child bounds written by another thread are
// read through L2 (__ldcg), so the fence makes them visible.
#include <cuda_runtime.h>

#include <string>

#include "dev_scene.cuh"
#include "host_scene.h"

namespace ptd {
namespace {

constexpr int kRefitThreads = 256;
constexpr uint32_t kNoParent = 0xffffffffu;

__device__ __forceinline__ void pad_bounds(const float lo[3], const float hi[3], float plo[3], float phi[3]) {
  float ext = 0.0f;
  for (int k = 0; k < 3; ++k) ext = fmaxf(ext, fmaxf(hi[k] - lo[k], fmaxf(fabsf(lo[k]), fabsf(hi[k]))));
  const float pad = ext * 1.0e-5f + 1.0e-30f;
  for (int k = 0; k < 3; ++k) {
    plo[k] = lo[k] - pad;
    phi[k] = hi[k] + pad;
  }
}

__device__ __forceinline__ void grow(float lo[3], float hi[3], float x, float y, float z) {
  lo[0] = fminf(lo[0], x);
  lo[1] = fminf(lo[1], y);
  lo[2] = fminf(lo[2], z);
  hi[0] = fmaxf(hi[0], x);
  hi[1] = fmaxf(hi[1], y);
  hi[2] = fmaxf(hi[2], z);
}

// Records: corner positions of each record's global id (its w), the
// any-hit flags from the triangle's material.
__global__ void k_refit_records(float4 *records, uint64_t n, const float *pos, const uint2 *tri_info,
                                const DevMaterial *materials) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t g = __float_as_uint(records[3 * r].w);
    const float *p = pos + 9ull * g;
    const pt_material &m = materials[__ldg(&tri_info[g].x)].m;
    const uint32_t fl = (m.alpha_mode == PT_ALPHA_OPAQUE ? REC_OPAQUE : 0u) | (m.double_sided ? REC_DOUBLE_SIDED : 0u);
    records[3 * r] = make_float4(p[0], p[1], p[2], __uint_as_float(g));
    records[3 * r + 1] = make_float4(p[3], p[4], p[5], __uint_as_float(fl));
    records[3 * r + 2] = make_float4(p[6], p[7], p[8], 0.0f);
  }
}

// Bounds of a leaf's records; false for an empty leaf.
__device__ bool leaf_bounds(const float4 *records, int ref, float lo[3], float hi[3]) {
  uint32_t first = (uint32_t)(~ref);
  const uint32_t count = first >> kLeafCountShift;
  first &= kLeafFirstMask;
  if (count == 0) return false;
  for (int k = 0; k < 3; ++k) {
    lo[k] = INFINITY;
    hi[k] = -INFINITY;
  }
  for (uint32_t i = 0; i < count; ++i)
    for (int v = 0; v < 3; ++v) {
      const float4 p = records[3ull * (first + i) + v];
      grow(lo, hi, p.x, p.y, p.z);
    }
  return true;
}

// ---- two-child nodes
__device__ __forceinline__ int node2_child(const BvhNode &nd, int k) { return k == 0 ? nd.d.x : nd.d.y; }

__global__ void k_refit2_links(const BvhNode *nodes, uint32_t n, uint32_t *parent, uint32_t *pending) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t c = 0;
    for (int k = 0; k < 2; ++k) {
      const int ch = node2_child(nodes[i], k);
      if (ch >= 0 && (uint32_t)ch < n) {
        parent[ch] = i;
        ++c;
      }
    }
    pending[i] = c;
  }
}

__global__ void k_refit2_up(BvhNode *nodes, uint32_t n, const float4 *records, const uint32_t *parent,
                            uint32_t *pending) {
  for (uint32_t start = blockIdx.x * blockDim.x + threadIdx.x; start < n; start += gridDim.x * blockDim.x) {
    const BvhNode s = nodes[start];
    if ((s.d.x >= 0 && (uint32_t)s.d.x < n) || (s.d.y >= 0 && (uint32_t)s.d.y < n)) continue;
    uint32_t i = start;
    for (;;) {
      BvhNode nd = nodes[i];
      float box[2][6];
      bool set[2] = {false, false};
      for (int k = 0; k < 2; ++k) {
        const int ch = node2_child(nd, k);
        float lo[3], hi[3];
        if (ch < 0) {
          set[k] = leaf_bounds(records, ch, lo, hi);
        } else if ((uint32_t)ch < n) {
          const float4 a = __ldcg(&nodes[ch].a), b = __ldcg(&nodes[ch].b), c = __ldcg(&nodes[ch].c);
          lo[0] = fminf(a.x, b.x);
          hi[0] = fmaxf(a.y, b.y);
          lo[1] = fminf(a.z, b.z);
          hi[1] = fmaxf(a.w, b.w);
          lo[2] = fminf(c.x, c.z);
          hi[2] = fmaxf(c.y, c.w);
          set[k] = true;
        }
        if (set[k]) pad_bounds(lo, hi, box[k], box[k] + 3);
      }
      if (set[0]) {
        nd.a.x = box[0][0];
        nd.a.y = box[0][3];
        nd.a.z = box[0][1];
        nd.a.w = box[0][4];
        nd.c.x = box[0][2];
        nd.c.y = box[0][5];
      }
      if (set[1]) {
        nd.b.x = box[1][0];
        nd.b.y = box[1][3];
        nd.b.z = box[1][1];
        nd.b.w = box[1][4];
        nd.c.z = box[1][2];
        nd.c.w = box[1][5];
      }
      nodes[i].a = nd.a;
      nodes[i].b = nd.b;
      nodes[i].c = nd.c;
      __threadfence();
      const uint32_t p = parent[i];
      if (p == kNoParent) break;
      if (atomicSub(&pending[p], 1u) != 1u) break;  // a sibling subtree is still open
      i = p;
    }
  }
}

// ---- four-child nodes
__global__ void k_refit4_links(const Bvh4Node *nodes, uint32_t n, uint32_t *parent, uint32_t *pending) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int ch[4] = {nodes[i].child.x, nodes[i].child.y, nodes[i].child.z, nodes[i].child.w};
    uint32_t c = 0;
    for (int k = 0; k < 4; ++k)
      if (ch[k] >= 0 && ch[k] != kEmptyChild && (uint32_t)ch[k] < n) {
        parent[ch[k]] = i;
        ++c;
      }
    pending[i] = c;
  }
}

__device__ __forceinline__ float lane(const float4 &v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w)); }
__device__ __forceinline__ void set_lane(float4 &v, int k, float x) {
  if (k == 0)
    v.x = x;
  else if (k == 1)
    v.y = x;
  else if (k == 2)
    v.z = x;
  else
    v.w = x;
}

__global__ void k_refit4_up(Bvh4Node *nodes, uint32_t n, const float4 *records, const uint32_t *parent,
                            uint32_t *pending) {
  for (uint32_t start = blockIdx.x * blockDim.x + threadIdx.x; start < n; start += gridDim.x * blockDim.x) {
    bool interior = false;
    {
      const int4 c = nodes[start].child;
      const int ch[4] = {c.x, c.y, c.z, c.w};
      for (int k = 0; k < 4; ++k) interior |= ch[k] >= 0 && ch[k] != kEmptyChild && (uint32_t)ch[k] < n;
    }
    if (interior) continue;
    uint32_t i = start;
    for (;;) {
      Bvh4Node nd = nodes[i];
      const int ch[4] = {nd.child.x, nd.child.y, nd.child.z, nd.child.w};
      for (int k = 0; k < 4; ++k) {
        float lo[3], hi[3];
        bool ok = false;
        if (ch[k] == kEmptyChild) continue;
        if (ch[k] < 0) {
          ok = leaf_bounds(records, ch[k], lo, hi);
        } else if ((uint32_t)ch[k] < n) {
          const Bvh4Node *c = nodes + ch[k];
          const float4 lx = __ldcg(&c->lo_x), hx = __ldcg(&c->hi_x), ly = __ldcg(&c->lo_y), hy = __ldcg(&c->hi_y);
          const float4 lz = __ldcg(&c->lo_z), hz = __ldcg(&c->hi_z);
          const int4 cc = __ldcg(&c->child);
          const int gch[4] = {cc.x, cc.y, cc.z, cc.w};
          for (int a = 0; a < 3; ++a) {
            lo[a] = INFINITY;
            hi[a] = -INFINITY;
          }
          for (int j = 0; j < 4; ++j) {
            if (gch[j] == kEmptyChild) continue;
            lo[0] = fminf(lo[0], lane(lx, j));
            hi[0] = fmaxf(hi[0], lane(hx, j));
            lo[1] = fminf(lo[1], lane(ly, j));
            hi[1] = fmaxf(hi[1], lane(hy, j));
            lo[2] = fminf(lo[2], lane(lz, j));
            hi[2] = fmaxf(hi[2], lane(hz, j));
            ok = true;
          }
        }
        if (!ok) continue;
        float plo[3], phi[3];
        pad_bounds(lo, hi, plo, phi);
        set_lane(nd.lo_x, k, plo[0]);
        set_lane(nd.hi_x, k, phi[0]);
        set_lane(nd.lo_y, k, plo[1]);
        set_lane(nd.hi_y, k, phi[1]);
        set_lane(nd.lo_z, k, plo[2]);
        set_lane(nd.hi_z, k, phi[2]);
      }
      nodes[i].lo_x = nd.lo_x;
      nodes[i].hi_x = nd.hi_x;
      nodes[i].lo_y = nd.lo_y;
      nodes[i].hi_y = nd.hi_y;
      nodes[i].lo_z = nd.lo_z;
      nodes[i].hi_z = nd.hi_z;
      __threadfence();
      const uint32_t p = parent[i];
      if (p == kNoParent) break;
      if (atomicSub(&pending[p], 1u) != 1u) break;
      i = p;
    }
  }
}

uint32_t grid_of(uint64_t n) {
  uint64_t g = (n + kRefitThreads - 1) / kRefitThreads;
  return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(g, 148ull * 32));
}

}  // namespace

std::string device_refit_bvh(SceneHost &sc, uint64_t records, cudaStream_t st) {
  DevScene &d = sc.dev;
  if (!d.nodes && !d.nodes4) return "";
  float4 *rec = const_cast<float4 *>(d.tris);
  if (records)
    k_refit_records<<<grid_of(records), kRefitThreads, 0, st>>>(rec, records, d.pos, d.tri_info, d.materials);
  const uint32_t n2 = d.node_count, n4 = d.node4_count;
  const uint64_t nmax = std::max<uint64_t>(std::max(n2, n4), 1);
  uint32_t *scratch = nullptr;
  cudaError_t e = cudaMallocAsync((void **)&scratch, 2 * nmax * sizeof(uint32_t), st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return std::string("refit scratch: ") + cudaGetErrorString(e);
  }
  uint32_t *parent = scratch, *pending = scratch + nmax;
  if (n2) {
    e = cudaMemsetAsync(parent, 0xff, n2 * sizeof(uint32_t), st);
    k_refit2_links<<<grid_of(n2), kRefitThreads, 0, st>>>(d.nodes, n2, parent, pending);
    k_refit2_up<<<grid_of(n2), kRefitThreads, 0, st>>>(const_cast<BvhNode *>(d.nodes), n2, d.tris, parent, pending);
  }
  if (n4 && e == cudaSuccess) {
    e = cudaMemsetAsync(parent, 0xff, n4 * sizeof(uint32_t), st);
    k_refit4_links<<<grid_of(n4), kRefitThreads, 0, st>>>(d.nodes4, n4, parent, pending);
    k_refit4_up<<<grid_of(n4), kRefitThreads, 0, st>>>(const_cast<Bvh4Node *>(d.nodes4), n4, d.tris, parent,
                                                        pending);
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaFreeAsync(scratch, st);
  if (e != cudaSuccess) return std::string("refit: ") + cudaGetErrorString(e);
  return "";
}

}  // namespace ptd
