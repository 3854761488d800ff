// port.cc -- see port.h.  TEST INFRASTRUCTURE (the oracle).

#include "port.h"

#include <cmath>
#include <deque>
#include <stdexcept>

namespace snogport {

namespace {

V sub(V a, V b) { return V{a.x - b.x, a.y - b.y, a.z - b.z}; }
V add(V a, V b) { return V{a.x + b.x, a.y + b.y, a.z + b.z}; }
float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V cross(V a, V b) { return V{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
float fmn(float a, float b) { return a < b ? a : b; }   // util/snogmath.h:43
float fmx(float a, float b) { return a > b ? a : b; }   // util/snogmath.h:48

void grow(Box &b, V p, bool &empty) {
  if (empty) {
    b.lo = b.hi = p;
    empty = false;
    return;
  }
  b.lo = V{fmn(b.lo.x, p.x), fmn(b.lo.y, p.y), fmn(b.lo.z, p.z)};
  b.hi = V{fmx(b.hi.x, p.x), fmx(b.hi.y, p.y), fmx(b.hi.z, p.z)};
}

// ---- construction: Octree::Builder (space/octree-builder.cc) --------------

struct Builder {
  struct Node {
    uint32_t child[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint32_t head = 0;
  };
  std::vector<Node> nodes;
  std::vector<std::pair<int32_t, uint32_t>> links{{0, 0}};   // (prim, next); [0] unused
  V origin{0, 0, 0};
  float size = 0;

  void push(uint32_t node, int32_t prim) {
    links.push_back({prim, nodes[node].head});
    nodes[node].head = uint32_t(links.size() - 1);
  }

  // Octree::Builder::add, top level (octree-builder.cc:173-216)
  void add_top(int32_t prim, const Box &b) {
    if (nodes.empty()) {
      nodes.push_back(Node());
      origin = b.lo;
      V ext = sub(b.hi, b.lo);
      size = ext.x;
      if (ext.y > size) size = ext.y;
      if (ext.z > size) size = ext.z;
      push(0, prim);
      return;
    }
    if (origin.x <= b.lo.x && origin.y <= b.lo.y && origin.z <= b.lo.z && (origin.x + size) >= b.hi.x &&
        (origin.y + size) >= b.hi.y && (origin.z + size) >= b.hi.z)
      add(prim, b, 0, origin.x, origin.y, origin.z, size);
    else
      grow_to_include(prim, b);
  }

  // Octree::Builder::grow_to_include (octree-builder.cc:227-317)
  void grow_to_include(int32_t prim, const Box &b) {
    uint32_t old_root = uint32_t(nodes.size());
    nodes.push_back(nodes[0]);
    nodes[0] = Node();
    float xl = origin.x - b.lo.x, xh = b.hi.x - (origin.x + size);
    float yl = origin.y - b.lo.y, yh = b.hi.y - (origin.y + size);
    float zl = origin.z - b.lo.z, zh = b.hi.z - (origin.z + size);
    unsigned slot = (xh > xl ? 0u : 4u) | (yh > yl ? 0u : 2u) | (zh > zl ? 0u : 1u);
    nodes[0].child[slot] = old_root;
    if (xh <= xl) origin.x -= size;
    if (yh <= yl) origin.y -= size;
    if (zh <= zl) origin.z -= size;
    size *= 2;
    add_top(prim, b);
  }

  void add_to_child(int32_t prim, const Box &b, uint32_t node, unsigned slot, float x, float y, float z,
                    float sz) {
    uint32_t c = nodes[node].child[slot];
    if (!c) {
      c = uint32_t(nodes.size());
      nodes.push_back(Node());
      nodes[node].child[slot] = c;
    }
    add(prim, b, c, x, y, z, sz);
  }

  // Octree::Builder::add, general case (octree-builder.cc:337-494)
  void add(int32_t prim, const Box &b, uint32_t node, float x, float y, float z, float sz) {
    float sub_size = sz / 2;
    float mx = x + sub_size, my = y + sub_size, mz = z + sub_size;
    V ext = sub(b.hi, b.lo);
    bool force = (ext.x + ext.y + ext.z) / 3 < sz / 4;
    auto lo_side = [&](float lo, float hi, float mid) {
      return hi < mid || (hi == mid && lo != hi) || (force && lo < mid);
    };
    auto hi_side = [&](float lo, float hi, float mid) {
      return lo > mid || (lo == mid && lo != hi) || (force && hi > mid);
    };
    bool here = true;
    for (int ix = 0; ix < 2; ix++) {
      if (!(ix ? hi_side(b.lo.x, b.hi.x, mx) : lo_side(b.lo.x, b.hi.x, mx))) continue;
      for (int iy = 0; iy < 2; iy++) {
        if (!(iy ? hi_side(b.lo.y, b.hi.y, my) : lo_side(b.lo.y, b.hi.y, my))) continue;
        for (int iz = 0; iz < 2; iz++) {
          if (!(iz ? hi_side(b.lo.z, b.hi.z, mz) : lo_side(b.lo.z, b.hi.z, mz))) continue;
          add_to_child(prim, b, node, unsigned(ix * 4 + iy * 2 + iz), ix ? mx : x, iy ? my : y,
                       iz ? mz : z, sub_size);
          here = false;
        }
      }
    }
    if (here) push(node, prim);
  }

  // Octree::Builder::copy_optimized_nodes (octree-builder.cc:537-650)
  Octree finish() const {
    Octree o;
    o.origin = origin;
    o.size = size;
    o.list.push_back(-1);
    std::deque<uint32_t> q;
    if (!nodes.empty()) q.push_back(0);
    uint32_t next_free = 1;
    while (!q.empty()) {
      uint32_t from = q.front();
      q.pop_front();
      const Node &fn = nodes[from];
      size_t to = o.heads.size();
      o.heads.push_back(0);
      o.children.insert(o.children.end(), 8, 0u);
      if (fn.head) {
        o.heads[to] = uint32_t(o.list.size());
        for (uint32_t l = fn.head; l; l = links[l].second) o.list.push_back(links[l].first);
        o.list.push_back(-1);
      }
      unsigned nkids = 0;
      for (unsigned i = 0; i < 8; i++)
        if (fn.child[i]) {
          nkids++;
          q.push_back(fn.child[i]);
          o.children[8 * to + i] = next_free++;
        }
      if (!nkids) o.children[8 * to] = o.children[8 * to + 1] = 1;
    }
    return o;
  }
};

// ---- primitive tests --------------------------------------------------------

// tripar_intersects (geometry/tripar-isec.h:56-118) with t0 / t1 bounds
bool tripar_isec(const Prim &p, V o, V d, float t0, float t1, float &t) {
  V pvec = cross(d, p.e2);
  float det = dot(p.e1, pvec);
  if (det > -1e-15f && det < 1e-15f) return false;
  float inv = 1.0f / det;
  V tvec = sub(o, p.a);
  float u = dot(tvec, pvec) * inv;
  if (u < 0 || u > 1) return false;
  V qvec = cross(tvec, p.e1);
  float v = dot(d, qvec) * inv;
  if (p.parallelogram) {
    if (v < 0 || v > 1) return false;
  } else if (v < 0 || u + v > 1) {
    return false;
  }
  t = dot(p.e2, qvec) * inv;
  return t > t0 && t < t1;
}

// sphere_intersects (geometry/sphere-isec.h:35-94) with quadratic_roots
bool sphere_isec(const Prim &p, V o, V d, float t0, float t1, float &t) {
  V oo = sub(o, p.a);
  float a = dot(d, d), b = 2 * dot(d, oo), c = dot(oo, oo) - p.radius * p.radius;
  float roots[2];
  unsigned n;
  if (a == 0) {
    if (b == 0) return false;
    roots[0] = -c / b;
    n = 1;
  } else {
    float disc = b * b - 4 * a * c;
    if (disc < 0) return false;
    float sq = std::sqrt(disc);
    float q = -(b + (b < 0 ? -sq : sq)) / 2;
    roots[0] = q / a;
    if (q == 0) {
      n = 1;
    } else {
      roots[1] = c / q;
      if (roots[0] > roots[1]) std::swap(roots[0], roots[1]);
      n = 2;
    }
  }
  for (unsigned i = 0; i < n; i++) {
    t = roots[i];
    if (t > t0) return t < t1;
  }
  return false;
}

bool prim_isec(const Prim &p, V o, V d, float t0, float t1, float &t) {
  return p.kind == 1 ? sphere_isec(p, o, d, t0, t1, t) : tripar_isec(p, o, d, t0, t1, t);
}

// ---- traversal: Octree::SearchState (space/octree.cc:175-300) --------------

struct Search {
  const Scene &s;
  V o, d;
  float t0, t1;
  bool any, stop = false;
  unsigned octant;
  Hit hit;

  void visit(uint32_t node, float xmin, float xmax, float ymin, float ymax, float zmin, float zmax) {
    hit.nodes++;
    float min_t = fmx(t0, fmx(xmin, fmx(ymin, zmin)));
    float max_t = fmn(t1, fmn(xmax, fmn(ymax, zmax)));
    if (min_t >= max_t) return;
    const Octree &oc = s.oct;
    if (oc.heads[node])
      for (uint32_t k = oc.heads[node]; oc.list[k] >= 0; k++) {
        hit.tests++;
        float t;
        if (prim_isec(s.prims[oc.list[k]], o, d, t0, t1, t)) {
          hit.prim = oc.list[k];
          if (any) {
            stop = true;
            return;
          }
          t1 = t;          // Space::ClosestIntersectCallback shrinks the ray
          hit.t = t;
        }
      }
    const uint32_t *ch = &oc.children[8 * size_t(node)];
    if (ch[0] == 1 && ch[1] == 1) return;
    float xh = (xmax - xmin) / 2, yh = (ymax - ymin) / 2, zh = (zmax - zmin) / 2;
    float xm = xmin + xh, ym = ymin + yh, zm = zmin + zh;
    for (unsigned i = 0; i < 8; i++) {
      unsigned child = (i == 3) ? 4 : (i == 4) ? 3 : i;
      uint32_t c = ch[child ^ octant];
      if (c && ((child & 4) ? (t1 > xm) : (t0 < xm)) && ((child & 2) ? (t1 > ym) : (t0 < ym)) &&
          ((child & 1) ? (t1 > zm) : (t0 < zm))) {
        float cx = xmin + ((child & 4) ? xh : 0), cy = ymin + ((child & 2) ? yh : 0),
              cz = zmin + ((child & 1) ? zh : 0);
        visit(c, cx, cx + xh, cy, cy + yh, cz, cz + zh);
        if (stop) return;
      }
    }
  }
};

}  // namespace

Scene build(const snogspec::Scene &spec) {
  Scene sc;
  const auto &h = spec.h;
  Builder b;
  auto vtx = [&](uint32_t i) { return V{spec.verts[3 * i], spec.verts[3 * i + 1], spec.verts[3 * i + 2]}; };
  for (uint32_t t = 0; t < h.n_triangles; t++) {
    V p0 = vtx(spec.tris[3 * t]), p1 = vtx(spec.tris[3 * t + 1]), p2 = vtx(spec.tris[3 * t + 2]);
    Prim p{0, p0, sub(p1, p0), sub(p2, p0), 0.f, false};
    sc.prims.push_back(p);
    V n = cross(p.e2, p.e1);                        // left-handed mesh (surface/mesh.h:55)
    if (dot(n, n) > 0) {                            // surface/mesh.cc:833-846
      Box bx;
      bool empty = true;
      grow(bx, p0, empty);
      grow(bx, p1, empty);
      grow(bx, p2, empty);
      b.add_top(int32_t(t), bx);
    }
  }
  for (const auto &sp : spec.spheres) {
    Prim p{1, V{sp.center[0], sp.center[1], sp.center[2]}, V{0, 0, 0}, V{0, 0, 0}, sp.radius, false};
    sc.prims.push_back(p);
    float r = sp.radius;
    Box bx{V{p.a.x - r, p.a.y - r, p.a.z - r}, V{p.a.x + r, p.a.y + r, p.a.z + r}};
    b.add_top(int32_t(sc.prims.size() - 1), bx);
  }
  for (const auto &tp : spec.tripars) {
    Prim p{2, V{tp.v0[0], tp.v0[1], tp.v0[2]}, V{tp.e1[0], tp.e1[1], tp.e1[2]},
           V{tp.e2[0], tp.e2[1], tp.e2[2]}, 0.f, tp.parallelogram != 0};
    sc.prims.push_back(p);
    Box bx;
    bool empty = true;
    grow(bx, p.a, empty);
    grow(bx, add(p.a, p.e1), empty);
    grow(bx, add(p.a, p.e2), empty);
    if (p.parallelogram) grow(bx, add(add(p.a, p.e1), p.e2), empty);
    b.add_top(int32_t(sc.prims.size() - 1), bx);
  }
  sc.oct = b.finish();
  return sc;
}

Hit trace(const Scene &s, V o, V d, float tmax, bool any) {
  Search ss{s, o, d, 0.f, tmax, any};
  ss.octant = (d.x >= 0 ? 0u : 4u) | (d.y >= 0 ? 0u : 2u) | (d.z >= 0 ? 0u : 1u);
  if (s.oct.heads.empty()) return ss.hit;
  // root slab bounds (space/octree.cc:119-135)
  const V org = s.oct.origin;
  const float size = s.oct.size;
  float ix = d.x == 0 ? 1e9f : 1 / d.x, iy = d.y == 0 ? 1e9f : 1 / d.y, iz = d.z == 0 ? 1e9f : 1 / d.z;
  float x0 = (org.x - o.x) * ix, x1 = (org.x - o.x + size) * ix;
  float y0 = (org.y - o.y) * iy, y1 = (org.y - o.y + size) * iy;
  float z0 = (org.z - o.z) * iz, z1 = (org.z - o.z + size) * iz;
  if (x0 > x1) std::swap(x0, x1);
  if (y0 > y1) std::swap(y0, y1);
  if (z0 > z1) std::swap(z0, z1);
  ss.visit(0, x0, x1, y0, y1, z0, z1);
  return ss.hit;
}

}  // namespace snogport
