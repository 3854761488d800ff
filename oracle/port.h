// port.h -- CPU restatement of snogray's acceleration-structure path.
//
// TEST INFRASTRUCTURE (the oracle).  A plain, recursive C++ restatement of
// the reference's loose octree -- construction (space/octree-builder.cc:
// 173-650), traversal (space/octree.cc:101-300) with the closest-hit and
// any-hit callbacks (space/space.cc:36-129), and the primitive tests
// (geometry/tripar-isec.h:56-170, geometry/sphere-isec.h:35-94,
// geometry/quadratic-roots.h:28-66) -- in IEEE single precision evaluated in
// source order (compiled with -ffp-contract=off).  It is pinned against the
// reference's own outputs (tests/golden/, tests/test_oracle_port.py) and used
// by the GPU tests to check the CUDA path at sizes no fixture can hold.
// Nothing in the product links or calls it.

#ifndef SNOG_ORACLE_PORT_H
#define SNOG_ORACLE_PORT_H

#include <cstdint>
#include <vector>

#include "scene_spec.h"

namespace snogport {

struct V {
  float x, y, z;
};

struct Box {
  V lo, hi;
};

// A primitive in the reference's insertion order: mesh triangles by part,
// then spheres, then tripars.
struct Prim {
  int kind;          // 0 triangle, 1 sphere, 2 tripar
  V a, e1, e2;       // corner and edges (triangle / tripar); centre in a
  float radius;
  bool parallelogram;
};

struct Octree {
  std::vector<uint32_t> children;   // 8 per node (BFS order; leaf = 1,1,...)
  std::vector<uint32_t> heads;      // per node
  std::vector<int32_t> list;        // primitive ids, -1 terminates; [0] = -1
  V origin{0, 0, 0};
  float size = 0;
};

struct Scene {
  std::vector<Prim> prims;
  Octree oct;
};

Scene build(const snogspec::Scene &spec);

struct Hit {
  int32_t prim = -1;
  float t = 0;
  uint64_t nodes = 0, tests = 0;
};

// Closest hit (Space::intersect) or first hit (Space::intersects) of the ray
// o + t d, t in (0, tmax).
Hit trace(const Scene &s, V o, V d, float tmax, bool any);

}  // namespace snogport

#endif
