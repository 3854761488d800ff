// octree_build.cc -- see octree_build.h.  All coordinate arithmetic is IEEE
// single precision in the reference's operand order, so the tree (and every
// midpoint compared against) is the same to the last bit; this file is
// compiled with -ffp-contract=off.

#include "octree_build.h"

#include <deque>
#include <stdexcept>

#include "snog_common.h"

namespace snog {

namespace {

// BBox::max_size and BBox::avg_size (geometry/bbox.h:128-158).
inline float box_max_size(const Box3 &b) {
  float ex = b.hi[0] - b.lo[0], ey = b.hi[1] - b.lo[1], ez = b.hi[2] - b.lo[2];
  float s = ex;
  if (ey > s) s = ey;
  if (ez > s) s = ez;
  return s;
}
inline float box_avg_size(const Box3 &b) {
  float ex = b.hi[0] - b.lo[0], ey = b.hi[1] - b.lo[1], ez = b.hi[2] - b.lo[2];
  return (ex + ey + ez) / 3;
}

// Whether a box belongs in the low / high half of one axis split at MID.
// A box touching the midpoint from one side counts for that side unless it is
// flat on that axis; a forced (small) box counts for every half it overlaps.
inline bool goes_low(float lo, float hi, float mid, bool force) {
  return hi < mid || (hi == mid && lo != hi) || (force && lo < mid);
}
inline bool goes_high(float lo, float hi, float mid, bool force) {
  return lo > mid || (lo == mid && lo != hi) || (force && hi > mid);
}

}  // namespace

uint32_t OctreeBuilder::new_node() {
  uint32_t id = uint32_t(head_.size());
  kids_.insert(kids_.end(), 8, 0u);
  head_.push_back(0);
  return id;
}

void OctreeBuilder::push_ref(uint32_t node, uint32_t ref) {
  uint32_t slot = uint32_t(link_ref_.size());
  link_ref_.push_back(ref);
  link_next_.push_back(head_[node]);
  head_[node] = slot;
}

void root_start(const Box3 &b, float origin[3], float &size) {
  for (int k = 0; k < 3; k++) origin[k] = b.lo[k];
  size = box_max_size(b);
}

bool root_fits(const float origin[3], float size, const Box3 &b) {
  return origin[0] <= b.lo[0] && origin[1] <= b.lo[1] && origin[2] <= b.lo[2] &&
         (origin[0] + size) >= b.hi[0] && (origin[1] + size) >= b.hi[1] && (origin[2] + size) >= b.hi[2];
}

// On each axis the cube grows to the side where B sticks out further (ties
// grow downwards); the old root keeps its position as one octant.
uint32_t root_grow(const Box3 &b, float origin[3], float &size) {
  uint32_t octant = 0;
  for (int a = 0; a < 3; a++) {
    float lo_grow = origin[a] - b.lo[a];
    float hi_grow = b.hi[a] - (origin[a] + size);
    bool grow_up = hi_grow > lo_grow;
    // Octant bit for axis a: x = 4, y = 2, z = 1 (space/octree-node.h:35-39).
    if (!grow_up) {
      octant |= 4u >> a;
      origin[a] -= size;
    }
  }
  size *= 2;
  return octant;
}

void OctreeBuilder::add(uint32_t ref, const Box3 &b) {
  if (head_.empty()) {
    new_node();
    root_start(b, origin_, size_);
    push_ref(0, ref);
    return;
  }
  while (!root_fits(origin_, size_, b)) grow_towards(b);
  insert(ref, b, 0, origin_[0], origin_[1], origin_[2], size_);
}

// Double the root cube towards B.  Node 0 stays the root, so the old root's
// record moves to a fresh slot, which becomes the new root's child.
void OctreeBuilder::grow_towards(const Box3 &b) {
  uint32_t moved = new_node();
  for (int k = 0; k < 8; k++) {
    kids_[8 * size_t(moved) + k] = kids_[k];
    kids_[k] = 0;
  }
  head_[moved] = head_[0];
  head_[0] = 0;
  kids_[root_grow(b, origin_, size_)] = moved;
}

void OctreeBuilder::insert(uint32_t ref, const Box3 &b, uint32_t node, float x, float y, float z,
                           float size) {
  // Explicit depth-first descent.  Octants are visited x-major, low before
  // high, exactly in the order the reference recurses, because the order of
  // node creation does not matter (ids are renumbered breadth first) but the
  // per-node insertion order of one surface does not either -- each node gets
  // it at most once -- so only the set of nodes reached must match.
  struct Frame { uint32_t node; float x, y, z, size; };
  Frame stack[512];
  int sp = 0;
  stack[sp++] = Frame{node, x, y, z, size};
  const float avg = box_avg_size(b);
  while (sp > 0) {
    Frame f = stack[--sp];
    float sub = f.size / 2;
    float mx = f.x + sub, my = f.y + sub, mz = f.z + sub;
    bool force = avg < f.size / 4;
    bool lx = goes_low(b.lo[0], b.hi[0], mx, force), hx = goes_high(b.lo[0], b.hi[0], mx, force);
    bool ly = goes_low(b.lo[1], b.hi[1], my, force), hy = goes_high(b.lo[1], b.hi[1], my, force);
    bool lz = goes_low(b.lo[2], b.hi[2], mz, force), hz = goes_high(b.lo[2], b.hi[2], mz, force);
    bool placed = false;
    // Children are pushed in reverse so they pop in octant order.
    for (int oc = 7; oc >= 0; oc--) {
      bool bx = oc & 4, by = oc & 2, bz = oc & 1;
      if (!((bx ? hx : lx) && (by ? hy : ly) && (bz ? hz : lz))) continue;
      placed = true;
      uint32_t child = kids_[8 * size_t(f.node) + oc];
      if (!child) {
        child = new_node();
        kids_[8 * size_t(f.node) + oc] = child;
      }
      if (sp >= 512) throw std::runtime_error("octree build: descent too deep");
      stack[sp++] = Frame{child, bx ? mx : f.x, by ? my : f.y, bz ? mz : f.z, sub};
    }
    if (!placed) push_ref(f.node, ref);
  }
}

OctreeArrays OctreeBuilder::finish() const {
  OctreeArrays out;
  const size_t n = head_.size();
  out.children.assign(8 * n, 0);
  out.heads.assign(n, 0);
  out.plist.reserve(link_ref_.size() + n + 1);
  out.plist.push_back(PREF_END);
  for (int k = 0; k < 3; k++) out.origin[k] = origin_[k];
  out.size = size_;
  if (n == 0) return out;

  std::vector<uint32_t> order;        // old node ids in BFS order
  std::vector<uint32_t> depth(n, 0);  // indexed by new id
  order.reserve(n);
  order.push_back(0);
  uint32_t next_free = 1;
  for (size_t qi = 0; qi < order.size(); qi++) {
    uint32_t old = order[qi];
    uint32_t nid = uint32_t(qi);
    if (head_[old]) {
      out.heads[nid] = uint32_t(out.plist.size());
      for (uint32_t s = head_[old]; s; s = link_next_[s]) {
        out.plist.push_back(link_ref_[s]);
        out.n_list_surfaces++;
      }
      out.plist.push_back(PREF_END);
    }
    uint32_t nkids = 0;
    for (int k = 0; k < 8; k++) {
      uint32_t c = kids_[8 * size_t(old) + k];
      if (!c) continue;
      nkids++;
      order.push_back(c);
      depth[next_free] = depth[nid] + 1;
      out.children[8 * size_t(nid) + k] = next_free++;
    }
    if (nkids == 0) {
      out.children[8 * size_t(nid) + 0] = 1;
      out.children[8 * size_t(nid) + 1] = 1;
      out.n_leaf++;
    }
    if (depth[nid] + 1 > out.max_depth) out.max_depth = depth[nid] + 1;
  }
  return out;
}

}  // namespace snog
