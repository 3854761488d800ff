// octree_gpu.h -- the device octree builder (octree_gpu.cu).

#ifndef SNOG_OCTREE_GPU_H
#define SNOG_OCTREE_GPU_H

#include <cstdint>
#include <vector>

#include "octree_build.h"
#include "scene.h"

namespace snog {

// A tree in the device layout of snog_common.h (nodes and 4-aligned lists),
// with the statistics of the host layout.
struct DeviceOctree {
  uint4 *nodes = nullptr;      // in the caller's arena
  uint32_t *plist = nullptr;   // in the caller's arena
  uint32_t n_nodes = 0, n_plist4 = 0;
  uint32_t n_plist_host = 0;   // entries of the host layout's list array
  uint32_t n_leaf = 0, max_depth = 0;
  uint64_t n_list_surfaces = 0;
  float origin[3] = {0, 0, 0}, size = 0;
};

// Build on the current device the tree the host builder makes from the same
// surfaces: BOXES[i] is the bounding box of the i-th surface in insertion
// order and REFS[i] the id its lists hold.  Output arrays are allocated in A.
// Throws Error (SNOG_EINVAL for trees deeper than 40 levels, SNOG_ECUDA,
// SNOG_ENOMEM).
void build_octree_device(const std::vector<Box3> &boxes, const std::vector<uint32_t> &refs, DeviceArena &A,
                         DeviceOctree &out);

// The host layout (octree_build.h) of a tree in the device layout.
OctreeArrays octree_from_device(const uint4 *d_nodes, uint32_t n_nodes, const uint32_t *d_plist, uint32_t n_plist4,
                                const float origin[3], float size, uint32_t max_depth);

}  // namespace snog

#endif
