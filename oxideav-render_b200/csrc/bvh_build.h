// Device BVH construction: the scene's BVH built on the GPU from the
// positions already resident in its arena, written in the layouts the
// traversal kernels read (two-child nodes, four-child nodes, leaf-ordered
// triangle records).
//
// Algorithm: Morton codes of the triangle centroids (30 bits), an LSD radix
// sort, then parallel locally-ordered clustering (Meister & Bittner, "Parallel
// Locally-Ordered Clustering for Bounding Volume Hierarchy Construction",
// IEEE TVCG 2018): every cluster finds its nearest neighbour (smallest merged
// surface area) among the 2 * kPlocRadius clusters around it in Morton order,
// mutual nearest neighbours merge, and the cluster list is compacted, until
// one cluster is left. Subtrees of at most kMaxLeafTris triangles whose SAH
// cost as a leaf does not exceed their cost as a node become leaves.
//
// Traversal results do not depend on the tree (the closest hit is the
// accepted candidate of smallest t, ties to the lowest global id), so images
// are identical to those rendered with the host-built tree.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "host_scene.h"

namespace ptd {

// Host statistics of the last device build, for tests and benchmarks.
struct DeviceBuildInfo {
  uint32_t iterations = 0;  // clustering rounds
  double ms = 0.0;          // host wall time of the build (synchronous)
};

// Builds the BVH of `sc` (committed without one) on the GPU: allocates
// `sc.bvh_arena`, points sc.dev's node / record fields into it, updates the
// device descriptor and sc.bvh. Returns "" on success. A tree deeper than the
// traversal stacks allow (`max_depth`) is reported as an error string that
// starts with "depth" and leaves `sc` unchanged; the caller then builds on
// the host. `oom` is set when the failure was a device allocation.
std::string device_build_bvh(SceneHost &sc, cudaStream_t stream, uint32_t max_depth, bool &oom,
                             DeviceBuildInfo *info = nullptr);

// The same contract with the host builder's binned-SAH split rule, built
// top down one tree level per round: per active node its bounds, 16 bins
// per axis of its centroid extent, the sweep for the cheapest split (or a
// leaf of at most 8 triangles), a stable partition and the children. Nodes
// at the depth limit or without a valid split halve their range by index
// (the host splits at the centroid median there).
std::string device_build_bvh_sah(SceneHost &sc, cudaStream_t stream, uint32_t max_depth, bool &oom,
                                 DeviceBuildInfo *info = nullptr);

}  // namespace ptd
