// trace.cuh -- octree closest-hit / any-hit traversal and the primitive
// tests, as device functions shared by the ray-batch kernels (trace.cu) and
// the path tracer (wavefront.cu).
//
// Exactness.  Hit ids must equal the reference's bit for bit, so every
// float operation on this path is an explicit round-to-nearest intrinsic
// (__fadd_rn, __fmul_rn, ...): nothing can be contracted into an FMA whatever
// the compile flags, and each expression rounds as the reference's
// TVec/TPos code does when evaluated left to right in IEEE single precision.
//
// Traversal order.  The reference recurses (space/octree.cc:175-300): at a
// node it first tests the node's own surface list, then visits the children
// in the order i = 0,1,2,4,3,5,6,7 (bits swapped so the number of "far" bits
// never decreases) xor the ray's origin octant, each behind a per-axis gate,
// and each child call begins with a slab cull.  Here the recursion becomes an
// explicit stack: all children that pass gate and cull *now* are pushed
// (at most 4 -- a segment meets at most 4 octants), the first of them is
// entered directly, and when an entry is popped its gate and cull are
// evaluated again with the ray's *current* extent.  Because the ray only
// ever shrinks, the push-time test admits a superset, and the pop-time test
// is exactly the test the recursion makes at that point; entries are popped
// in the recursion's order, so the set and order of surface tests -- and the
// surviving hit -- are the reference's.  The reference's negative-result
// cache (space/isec-cache.h) only skips re-testing a surface that already
// missed; a miss stays a miss for a ray that only shrinks, so omitting it
// changes work, not results.

#ifndef SNOG_TRACE_CUH
#define SNOG_TRACE_CUH

#include "snog_common.h"

namespace snog {

// -- exact float3 arithmetic ------------------------------------------------
__device__ __forceinline__ float3 xadd(float3 a, float3 b) {
  return f3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z));
}
__device__ __forceinline__ float3 xsub(float3 a, float3 b) {
  return f3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z));
}
__device__ __forceinline__ float3 xmul(float3 a, float s) {
  return f3(__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s));
}
__device__ __forceinline__ float xdot(float3 a, float3 b) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ float3 xcross(float3 a, float3 b) {
  return f3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
            __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float xlen_sq(float3 a) { return xdot(a, a); }

constexpr float kEps = 1e-15f;   // geometry/coords.h:48

// tripar_intersects (geometry/tripar-isec.h:56-118) plus the t < t1 bound of
// the ray form (tripar-isec.h:158-170).
__device__ __forceinline__ bool tripar_hit(float3 corner, float3 e1, float3 e2, bool parallelogram,
                                           float3 o, float3 d, float t0, float t1, float &t,
                                           float &u, float &v) {
  float3 pvec = xcross(d, e2);
  float det = xdot(e1, pvec);
  if (det > -kEps && det < kEps) return false;
  float inv_det = __fdiv_rn(1.0f, det);
  float3 tvec = xsub(o, corner);
  u = __fmul_rn(xdot(tvec, pvec), inv_det);
  if (u < 0.f || u > 1.f) return false;
  float3 qvec = xcross(tvec, e1);
  v = __fmul_rn(xdot(d, qvec), inv_det);
  if (parallelogram) {
    if (v < 0.f || v > 1.f) return false;
  } else {
    if (v < 0.f || __fadd_rn(u, v) > 1.f) return false;
  }
  t = __fmul_rn(xdot(e2, qvec), inv_det);
  return t > t0 && t < t1;
}

// sphere_intersects + quadratic_roots (geometry/sphere-isec.h:35-94,
// geometry/quadratic-roots.h:28-66): the first root above t0, then < t1.
__device__ __forceinline__ bool sphere_hit(float3 center, float radius, float3 o, float3 d,
                                           float t0, float t1, float &t) {
  float3 oo = xsub(o, center);
  float a = xlen_sq(d);
  float b = __fmul_rn(2.0f, xdot(d, oo));
  float c = __fsub_rn(xlen_sq(oo), __fmul_rn(radius, radius));
  float r0, r1;
  int n;
  if (a == 0.f) {
    if (b == 0.f) return false;
    r0 = __fdiv_rn(-c, b);
    r1 = r0;
    n = 1;
  } else {
    float disc = __fsub_rn(__fmul_rn(b, b), __fmul_rn(__fmul_rn(4.0f, a), c));
    if (disc < 0.f) return false;
    float sq = __fsqrt_rn(disc);
    float q = __fdiv_rn(-__fadd_rn(b, (b < 0.f ? -sq : sq)), 2.0f);
    r0 = __fdiv_rn(q, a);
    if (q == 0.f) {
      r1 = r0;
      n = 1;
    } else {
      r1 = __fdiv_rn(c, q);
      n = 2;
      if (r0 > r1) {
        float tmp = r0;
        r0 = r1;
        r1 = tmp;
      }
    }
  }
  if (r0 > t0) {
    t = r0;
    return t < t1;
  }
  if (n == 2 && r1 > t0) {
    t = r1;
    return t < t1;
  }
  return false;
}

struct TraceCounters {
  uint32_t nodes;     // node calls (space_node_intersect_calls)
  uint32_t tests;     // surface tests (surface_intersects_tests, no neg. cache)
  uint32_t overflow;  // traversal stack was too small (result invalid)
};

// Child slot IDX of a node whose 8 child ids are in K0, K1, by selects (no
// dynamically indexed local array).
__device__ __forceinline__ uint32_t pick_child(uint4 k0, uint4 k1, uint32_t idx) {
  uint4 k = (idx & 4u) ? k1 : k0;
  uint32_t a = (idx & 1u) ? k.y : k.x;
  uint32_t b = (idx & 1u) ? k.w : k.z;
  return (idx & 2u) ? b : a;
}

// Test the packed surface reference REF against the ray.  Closest queries
// shrink t1 on a hit.
__device__ __forceinline__ bool test_ref(const DevScene &s, uint32_t ref, float3 o, float3 d,
                                         float t0, float &t1) {
  const uint32_t kind = ref >> 30, idx = ref & PREF_INDEX_MASK;
  float t, u, v;
  if (kind == PK_TRI) {
    const float4 *p = s.tri + 3 * size_t(idx);
    float4 c = __ldg(p), a = __ldg(p + 1), b = __ldg(p + 2);
    if (tripar_hit(xyz(c), xyz(a), xyz(b), false, o, d, t0, t1, t, u, v)) {
      t1 = t;
      return true;
    }
  } else if (kind == PK_SPHERE) {
    float4 sp = __ldg(s.sph + idx);
    if (sphere_hit(xyz(sp), sp.w, o, d, t0, t1, t)) {
      t1 = t;
      return true;
    }
  } else {
    const float4 *p = s.tpar + 3 * size_t(idx);
    float4 c = __ldg(p), a = __ldg(p + 1), b = __ldg(p + 2);
    if (tripar_hit(xyz(c), xyz(a), xyz(b), c.w != 0.f, o, d, t0, t1, t, u, v)) {
      t1 = t;
      return true;
    }
  }
  return false;
}

// One pending octree visit: node id and gate bits packed into lo.w, the
// node's parametric slab bounds in lo.xyz (minima) and hi.xyz (maxima).
struct StackEntry {
  float4 lo, hi;
};

constexpr uint32_t kGateFlag = 8u;   // entry carries a parent gate

__device__ __forceinline__ bool slab_open(float t0, float t1, float3 lo, float3 hi) {
  float min_t = fmax_ref(t0, fmax_ref(lo.x, fmax_ref(lo.y, lo.z)));
  float max_t = fmin_ref(t1, fmin_ref(hi.x, fmin_ref(hi.y, hi.z)));
  return !(min_t >= max_t);
}

// The parent's gate for a child with octant bits CB (parametric order), at
// the current extent: a "far" half needs t1 beyond the midpoint, a "near"
// half needs t0 before it (space/octree.cc:268-272).  For the far half the
// midpoint is the child's lower bound, for the near half its upper bound --
// the very same rounded sums the reference compares against.
__device__ __forceinline__ bool gate_open(uint32_t cb, float t0, float t1, float3 lo, float3 hi) {
  bool gx = (cb & 4) ? (t1 > lo.x) : (t0 < hi.x);
  bool gy = (cb & 2) ? (t1 > lo.y) : (t0 < hi.y);
  bool gz = (cb & 1) ? (t1 > lo.z) : (t0 < hi.z);
  return gx && gy && gz;
}

// Traverse the octree.  ANY = stop at the first hit (Space::intersects /
// occludes).  Returns the surviving hit's packed reference, or PREF_END.
// t1 is shrunk to the closest hit for closest queries.  STACK entries must
// cover 3 * depth + 2 (chosen by the host from the tree depth); if they do
// not, cnt.overflow is set and the result must be discarded.
template <bool ANY, int STACK>
__device__ uint32_t traverse(const DevScene &s, float3 o, float3 d, float t0, float &t1,
                             TraceCounters &cnt) {
  if (s.n_nodes == 0) return PREF_END;
  StackEntry stk[STACK];
  int sp = 0;

  // Root slab bounds (space/octree.cc:119-135).
  float3 lo, hi;
  {
    float inv = (d.x == 0.f) ? 1e9f : __fdiv_rn(1.0f, d.x);
    float a = __fmul_rn(__fsub_rn(s.origin[0], o.x), inv);
    float b = __fmul_rn(__fadd_rn(__fsub_rn(s.origin[0], o.x), s.size), inv);
    if (a > b) { float tmp = a; a = b; b = tmp; }
    lo.x = a; hi.x = b;
    inv = (d.y == 0.f) ? 1e9f : __fdiv_rn(1.0f, d.y);
    a = __fmul_rn(__fsub_rn(s.origin[1], o.y), inv);
    b = __fmul_rn(__fadd_rn(__fsub_rn(s.origin[1], o.y), s.size), inv);
    if (a > b) { float tmp = a; a = b; b = tmp; }
    lo.y = a; hi.y = b;
    inv = (d.z == 0.f) ? 1e9f : __fdiv_rn(1.0f, d.z);
    a = __fmul_rn(__fsub_rn(s.origin[2], o.z), inv);
    b = __fmul_rn(__fadd_rn(__fsub_rn(s.origin[2], o.z), s.size), inv);
    if (a > b) { float tmp = a; a = b; b = tmp; }
    lo.z = a; hi.z = b;
  }
  const uint32_t octant = (d.x >= 0.f ? 0u : 4u) | (d.y >= 0.f ? 0u : 2u) | (d.z >= 0.f ? 0u : 1u);
  uint32_t node = 0, gate = 0;
  uint32_t hit_ref = PREF_END;

  for (;;) {
    bool open = true;
    if (gate & kGateFlag) open = gate_open(gate & 7u, t0, t1, lo, hi);
    if (open) {
      cnt.nodes++;
      open = slab_open(t0, t1, lo, hi);
    }
    if (open) {
      uint32_t h = __ldg(s.node_heads + node);
      if (h) {
        for (uint32_t ref = __ldg(s.plist + h); ref != PREF_END; ref = __ldg(s.plist + (++h))) {
          cnt.tests++;
          if (test_ref(s, ref, o, d, t0, t1)) {
            hit_ref = ref;
            if (ANY) return hit_ref;
          }
        }
      }
      const uint4 *kp = reinterpret_cast<const uint4 *>(s.node_children + 8 * size_t(node));
      uint4 k0 = __ldg(kp), k1 = __ldg(kp + 1);
      const bool leaf = (k0.x == 1u && k0.y == 1u);
      if (!leaf) {
        float3 half = f3(__fdiv_rn(__fsub_rn(hi.x, lo.x), 2.0f), __fdiv_rn(__fsub_rn(hi.y, lo.y), 2.0f),
                         __fdiv_rn(__fsub_rn(hi.z, lo.z), 2.0f));
        // Walk the visiting order backwards: every qualifying child but the
        // first is pushed (so they pop in visiting order after the first
        // child's subtree), the first is entered directly.  At most 4 pass
        // (one octant per crossing of each of the three midplanes).
        bool have = false;
        StackEntry pend;
#pragma unroll
        for (int i = 7; i >= 0; i--) {
          const uint32_t cb = (i == 3) ? 4u : (i == 4) ? 3u : uint32_t(i);
          const uint32_t c = pick_child(k0, k1, cb ^ octant);
          if (!c) continue;
          float3 clo = f3(__fadd_rn(lo.x, (cb & 4) ? half.x : 0.f), __fadd_rn(lo.y, (cb & 2) ? half.y : 0.f),
                          __fadd_rn(lo.z, (cb & 1) ? half.z : 0.f));
          float3 chi = f3(__fadd_rn(clo.x, half.x), __fadd_rn(clo.y, half.y), __fadd_rn(clo.z, half.z));
          if (!gate_open(cb, t0, t1, clo, chi) || !slab_open(t0, t1, clo, chi)) continue;
          if (have) {
            if (sp < STACK) stk[sp++] = pend;
            else cnt.overflow = 1;
          }
          pend.lo = make_float4(clo.x, clo.y, clo.z, __uint_as_float(c));
          pend.hi = make_float4(chi.x, chi.y, chi.z, __uint_as_float(cb | kGateFlag));
          have = true;
        }
        if (have) {
          node = __float_as_uint(pend.lo.w);
          gate = __float_as_uint(pend.hi.w);
          lo = xyz(pend.lo);
          hi = xyz(pend.hi);
          continue;
        }
      }
    }
    if (sp == 0) break;
    --sp;
    node = __float_as_uint(stk[sp].lo.w);
    gate = __float_as_uint(stk[sp].hi.w);
    lo = xyz(stk[sp].lo);
    hi = xyz(stk[sp].hi);
  }
  return hit_ref;
}

// Global primitive id of a packed reference: triangles, then spheres, then
// tripars.
__device__ __forceinline__ int32_t prim_id_of(const DevScene &s, uint32_t ref) {
  if (ref == PREF_END) return -1;
  uint32_t kind = ref >> 30, idx = ref & PREF_INDEX_MASK;
  if (kind == PK_TRI) return int32_t(idx);
  if (kind == PK_SPHERE) return int32_t(s.n_tri + idx);
  return int32_t(s.n_tri + s.n_sph + idx);
}

}  // namespace snog

#endif
