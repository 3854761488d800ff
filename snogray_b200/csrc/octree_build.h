// octree_build.h -- host construction of the loose octree the kernels walk.
//
// The tree must be the reference's tree node for node, because hit ids are
// compared bit-exactly and the first of two equal-t hits wins
// (geometry/tripar-isec.h:158-170): the traversal order, and so the winner,
// depends on which node lists a surface sits in and in which order.  The
// construction therefore follows the reference's rules
// (space/octree-builder.cc:173-650):
//   * the first surface fixes the root cube at its bbox minimum with side
//     bbox.max_size(); a surface outside the cube grows the root by doubling
//     towards it, the old root becoming one octant of the new one;
//   * insertion is eager: a surface descends into every octant it fits in,
//     creating nodes on the way; one that straddles a midpoint stays in the
//     node unless its bbox.avg_size() < size/4, in which case it is copied
//     into every octant it touches;
//   * a node's list is last-in first-out in insertion order;
//   * the final arrays are renumbered breadth first, children in octant
//     order, each list packed and terminated.
// The implementation here is independent of the reference's classes: flat
// vectors, an explicit frame stack for the descent, and a single BFS pass
// that also yields the depth statistics.

#ifndef SNOG_OCTREE_BUILD_H
#define SNOG_OCTREE_BUILD_H

#include <cstdint>
#include <vector>

namespace snog {

struct Box3 {
  float lo[3], hi[3];
};

struct OctreeArrays {
  std::vector<uint32_t> children;   // 8 per node, BFS order
  std::vector<uint32_t> heads;      // per node, index into plist, 0 = empty
  std::vector<uint32_t> plist;      // entries = caller's refs, PREF_END ends a list
  float origin[3] = {0, 0, 0};
  float size = 0;
  uint32_t max_depth = 0;
  uint32_t n_leaf = 0;
  uint64_t n_list_surfaces = 0;
};

// Root cube of the tree being built: the first surface fixes it at its bbox
// minimum with side bbox.max_size(); a later surface outside it doubles it
// towards the surface, the old root becoming one octant of the new one
// (space/octree-builder.cc:173-247).  Shared by the host and device builders
// so both grow the root with the same float operations.
void root_start(const Box3 &box, float origin[3], float &size);
bool root_fits(const float origin[3], float size, const Box3 &box);
// Doubles the cube towards BOX; returns the octant the old root becomes.
uint32_t root_grow(const Box3 &box, float origin[3], float &size);

class OctreeBuilder {
 public:
  // Insert one surface with reference REF (stored verbatim in the lists)
  // and bounding box BOX.  Surfaces must be added in the reference's order.
  void add(uint32_t ref, const Box3 &box);

  // Produce the packed, breadth-first arrays.
  OctreeArrays finish() const;

  size_t node_count() const { return kids_.size() / 8; }

 private:
  uint32_t new_node();
  void push_ref(uint32_t node, uint32_t ref);
  void insert(uint32_t ref, const Box3 &box, uint32_t node, float x, float y, float z, float size);
  void grow_towards(const Box3 &box);

  std::vector<uint32_t> kids_;      // 8 per node, creation order
  std::vector<uint32_t> head_;      // per node: index into link_, 0 = empty
  std::vector<uint32_t> link_ref_{0};   // slot 0 is the list terminator
  std::vector<uint32_t> link_next_{0};
  float origin_[3] = {0, 0, 0};
  float size_ = 0;
};

}  // namespace snog

#endif
