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
  float inv_det = __frcp_rn(det);   // = 1.0f / det, correctly rounded
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

// tripar_hit evaluated to the end without early exits: the same
// operations and the same result, but a warp whose lanes would leave at
// different tests does not diverge.  Measured faster where rounds are full
// of long lists (the intersection batch, +2.4 %), not on any-hit rounds.
__device__ __forceinline__ bool tripar_hit_flat(float3 corner, float3 e1, float3 e2, bool parallelogram,
                                                float3 o, float3 d, float t0, float t1, float &t) {
  const float3 pvec = xcross(d, e2);
  const float det = xdot(e1, pvec);
  bool ok = !(det > -kEps && det < kEps);
  const float inv_det = __frcp_rn(det);
  const float3 tvec = xsub(o, corner);
  const float u = __fmul_rn(xdot(tvec, pvec), inv_det);
  ok = ok && !(u < 0.f || u > 1.f);
  const float3 qvec = xcross(tvec, e1);
  const float v = __fmul_rn(xdot(d, qvec), inv_det);
  ok = ok && !(v < 0.f || (parallelogram ? v > 1.f : __fadd_rn(u, v) > 1.f));
  t = __fmul_rn(xdot(e2, qvec), inv_det);
  return ok && t > t0 && t < t1;
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

// A primitive's 48-byte record (snog_common.h).
struct PrimRec {
  float4 a, b, c;
};

__device__ __forceinline__ PrimRec load_prim(const DevScene &s, uint32_t id) {
  const float4 *p = s.prims + 3 * size_t(id);
  return PrimRec{__ldg(p), __ldg(p + 1), __ldg(p + 2)};
}

// Test a loaded primitive against the ray; closest queries shrink t1 on a
// hit (the surface's intersect / intersects methods, surface/mesh.cc:730-760,
// surface/sphere.cc:110-125, surface/tripar.cc:93-115).
// FLAT: triangles and tripars through tripar_hit_flat.
template <bool FLAT = false>
__device__ __forceinline__ bool test_prim(const PrimRec &r, float3 o, float3 d, float t0, float &t1) {
  const float kind = r.a.w;
  float t, u, v;
  if (kind == float(PRIM_SPHERE)) {
    if (sphere_hit(xyz(r.a), r.b.x, o, d, t0, t1, t)) {
      t1 = t;
      return true;
    }
    return false;
  }
  const bool hit = FLAT ? tripar_hit_flat(xyz(r.a), xyz(r.b), xyz(r.c), kind == float(PRIM_PARALLELOGRAM), o, d,
                                          t0, t1, t)
                       : tripar_hit(xyz(r.a), xyz(r.b), xyz(r.c), kind == float(PRIM_PARALLELOGRAM), o, d, t0, t1,
                                    t, u, v);
  if (hit) t1 = t;
  return hit;
}

// The pending children of one visited node, as one stack record: the
// node's near-half lower bounds, midpoints and far-half upper bounds (every
// child's slab bounds are a selection of these, per axis), its first child's
// index, its child mask and the visiting positions of the children not yet
// entered.  One record per visited node with two or more qualifying children,
// instead of one entry per waiting child: a visit pushes at most once, and
// the stack holds at most one record per tree level.
struct StackRec {
  float4 a;   // near_lo.xyz, first child index
  float4 b;   // mid.xyz, child mask | visiting positions still to enter << 8
  float4 c;   // far.xyz
};

// Threads per block of every trace kernel.
constexpr int kTraceBlock = 128;
// Blocks per SM the trace kernels are compiled for (register cap 64).
#ifndef SNOG_TRACE_MINBLOCKS
#define SNOG_TRACE_MINBLOCKS 8
#endif

// The newest kRing records of each thread's stack live in shared memory, as
// a ring; older ones spill to the thread's local-memory array.  Lanes of a
// warp sit at different stack depths, so a local-memory stack is read and
// written uncoalesced; the ring keeps the pushes and pops of a walk on chip
// (kRing * 48 bytes per thread, 18 KB per 128-thread block at kRing = 3).
#ifndef SNOG_RING
#define SNOG_RING 3
#endif
constexpr uint32_t kRing = SNOG_RING;

// This thread's first ring slot.  Part k (0, 1, 2) of record position e of
// thread t is float4 (3 * e + k) * kTraceBlock + t: a warp touching one part
// of one position reads 512 contiguous bytes.
__device__ __forceinline__ float4 *ring_slots() {
  __shared__ float4 ring[3 * kRing * kTraceBlock];
  return ring + threadIdx.x;
}

// Each thread's current ray in shared memory, for the lanes that test its
// list entries (a list round would otherwise move 14 values by shuffles):
// uint4 k * kTraceBlock + threadIdx.x holds, for k = 0, 1, 2, (origin, t0),
// (direction, t1) and the scene's list-record pointer.
__device__ __forceinline__ uint4 *ray_slots() {
  __shared__ uint4 rays[3 * kTraceBlock];
  return rays;
}

constexpr uint32_t kGateFlag = 8u;   // entry carries a parent gate
constexpr uint32_t kSlowSlab = 8u;   // in Traversal::octant: slab bounds may be NaN
constexpr uint32_t kAnyHit = 16u;    // in Traversal::octant: an any-hit query
enum { kClosestOnly = 0, kAnyOnly = 1, kMixed = 2 };   // queries a trace kernel runs

__device__ __forceinline__ bool slab_open(float t0, float t1, float3 lo, float3 hi) {
  float min_t = fmax_ref(t0, fmax_ref(lo.x, fmax_ref(lo.y, lo.z)));
  float max_t = fmin_ref(t1, fmin_ref(hi.x, fmin_ref(hi.y, hi.z)));
  return !(min_t >= max_t);
}

// slab_open for bounds known to be NaN-free (finite slab, t0 and t1 not
// NaN): maxima and minima are then exact and associative, so fmaxf / fminf
// in any grouping decide the same as the reference's ordered ternaries.
__device__ __forceinline__ bool slab_open_finite(float t0, float t1, float3 lo, float3 hi) {
  return fmaxf(fmaxf(t0, lo.x), fmaxf(lo.y, lo.z)) < fminf(fminf(t1, hi.x), fminf(hi.y, hi.z));
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

// Octant bits (x = 4, y = 2, z = 1) of the I-th child in the reference's
// visiting order 0,1,2,4,3,5,6,7 (before the xor with the ray's octant).
__device__ __forceinline__ uint32_t visit_bits(uint32_t i) { return i == 3u ? 4u : i == 4u ? 3u : i; }

// A resumable octree walk for one ray.  init() sets up the root's slab
// bounds (space/octree.cc:119-135); node_step() processes one octree entry --
// the child entered last, else the top of the stack -- as one call of the
// reference's recursive function does: parent gate, slab cull, then the
// node's surface list (left pending in [lp, lend) for list_round) and the
// children.  Kernels interleave the steps of many rays per warp and refill
// lanes whose ray has finished.  The stack holds one record per tree level
// on the walk's path; kRecs (from STACK, which the host picks from the tree
// depth) plus kRing records cover every tree the host admits.  Should they
// not, cnt.overflow is set and the result must be discarded.
template <int STACK>
struct Traversal {
  float3 lo, hi;
  float t0, t1;
  uint32_t node, gate, octant, hit_ref;   // octant: bits 0-2, kSlowSlab, kAnyHit
  uint32_t lp, lend;         // surface list still to test: plist[lp, lend)
  uint32_t ring;             // shared-memory ring: oldest position | count << 4 (0 when empty)
  int sp;                    // entries spilled to stk[0, sp)
  bool have;                 // a current entry (node/gate/lo/hi) is set
  const uint4 *nodes;        // the ray's scene (its list and primitive arrays are in the ray slot)
  // Records the stack may need: one per tree level.  STACK, the class the
  // host picks from the tree depth (at least 3 * depth + 4), bounds them
  // with room to spare.
  static constexpr int kRecs = (STACK + 2) / 3;
  // The spilled part of the stack: an array of kRecs records owned by the
  // caller.  It is not a member: a dynamically indexed member array puts
  // the whole object in local memory, every scalar above included.
  StackRec *stk;

  // The ray's origin and direction, from its shared-memory slot.
  __device__ __forceinline__ float3 ray_o() const {
    const uint4 a = ray_slots()[threadIdx.x];
    return f3(__uint_as_float(a.x), __uint_as_float(a.y), __uint_as_float(a.z));
  }
  __device__ __forceinline__ float3 ray_d() const {
    const uint4 a = ray_slots()[kTraceBlock + threadIdx.x];
    return f3(__uint_as_float(a.x), __uint_as_float(a.y), __uint_as_float(a.z));
  }
  // Shrink the ray (closest queries), in the register and in the slot.
  __device__ __forceinline__ void set_t1(float t) {
    t1 = t;
    reinterpret_cast<uint32_t *>(ray_slots() + kTraceBlock + threadIdx.x)[3] = __float_as_uint(t);
  }

  __device__ __forceinline__ void init(const DevScene &s, float3 o, float3 d, float t0_, float t1_) {
    t0 = t0_;
    t1 = t1_;
    hit_ref = PREF_END;
    sp = 0;
    ring = 0;
    node = 0;
    gate = 0;
    lp = lend = 0;
    have = s.n_nodes != 0;
    nodes = s.nodes;
    {
      uint4 *slot = ray_slots() + threadIdx.x;
      const unsigned long long pl = reinterpret_cast<uintptr_t>(s.lrec);
      slot[0] = make_uint4(__float_as_uint(o.x), __float_as_uint(o.y), __float_as_uint(o.z), __float_as_uint(t0_));
      slot[kTraceBlock] =
          make_uint4(__float_as_uint(d.x), __float_as_uint(d.y), __float_as_uint(d.z), __float_as_uint(t1_));
      slot[2 * kTraceBlock] = make_uint4(uint32_t(pl), uint32_t(pl >> 32), 0u, 0u);
    }
    // 1 / d rounded once, as the reference's division (__frcp_rn is the
    // correctly rounded reciprocal, the same value as 1.0f / d).
    float inv = (d.x == 0.f) ? 1e9f : __frcp_rn(d.x);
    float a = __fmul_rn(__fsub_rn(s.origin[0], o.x), inv);
    float b = __fmul_rn(__fadd_rn(__fsub_rn(s.origin[0], o.x), s.size), inv);
    if (a > b) { float tmp = a; a = b; b = tmp; }
    lo.x = a; hi.x = b;
    inv = (d.y == 0.f) ? 1e9f : __frcp_rn(d.y);
    a = __fmul_rn(__fsub_rn(s.origin[1], o.y), inv);
    b = __fmul_rn(__fadd_rn(__fsub_rn(s.origin[1], o.y), s.size), inv);
    if (a > b) { float tmp = a; a = b; b = tmp; }
    lo.y = a; hi.y = b;
    inv = (d.z == 0.f) ? 1e9f : __frcp_rn(d.z);
    a = __fmul_rn(__fsub_rn(s.origin[2], o.z), inv);
    b = __fmul_rn(__fadd_rn(__fsub_rn(s.origin[2], o.z), s.size), inv);
    if (a > b) { float tmp = a; a = b; b = tmp; }
    lo.z = a; hi.z = b;
    octant = (d.x >= 0.f ? 0u : 4u) | (d.y >= 0.f ? 0u : 2u) | (d.z >= 0.f ? 0u : 1u);
    // A node's bounds lie within its parent's (a far half's upper bound may
    // round one ulp beyond): with every root bound below 1e37 in magnitude
    // no bound below overflows, none is NaN, and with t0, t1 not NaN
    // node_step may take its fast tests.  (fabsf(NaN) < x is false.)
    const bool finite = fabsf(lo.x) < 1e37f && fabsf(lo.y) < 1e37f && fabsf(lo.z) < 1e37f &&
                        fabsf(hi.x) < 1e37f && fabsf(hi.y) < 1e37f && fabsf(hi.z) < 1e37f && !isnan(t0) &&
                        !isnan(t1);
    if (!finite) octant |= kSlowSlab;
  }

  // The walk is over: no list pending, no current entry, empty stack.
  __device__ __forceinline__ bool finished() const { return lp >= lend && !have && sp == 0 && (ring >> 4) == 0u; }

  // Push a record: into the ring, first moving the ring's oldest record to
  // local memory when the ring is full.
  __device__ __forceinline__ void push(float3 nlo, float3 mid, float3 far, uint32_t first, uint32_t bits,
                                       TraceCounters &cnt) {
    float4 *r = ring_slots();
    uint32_t base = ring & 15u, n = ring >> 4;
    if (n == kRing) {
      if (sp < kRecs) {
        stk[sp].a = r[(3 * base) * kTraceBlock];
        stk[sp].b = r[(3 * base + 1) * kTraceBlock];
        stk[sp].c = r[(3 * base + 2) * kTraceBlock];
        sp++;
      } else {
        cnt.overflow = 1;
      }
      base = base + 1u == kRing ? 0u : base + 1u;
      n--;
    }
    uint32_t pos = base + n;
    pos = pos >= kRing ? pos - kRing : pos;
    r[(3 * pos) * kTraceBlock] = make_float4(nlo.x, nlo.y, nlo.z, __uint_as_float(first));
    r[(3 * pos + 1) * kTraceBlock] = make_float4(mid.x, mid.y, mid.z, __uint_as_float(bits));
    r[(3 * pos + 2) * kTraceBlock] = make_float4(far.x, far.y, far.z, 0.f);
    ring = base | ((n + 1u) << 4);
  }

  // Make the next waiting child of the newest record the current entry (the
  // record is dropped once its last child is taken).  Returns false, leaving
  // the walk unchanged, if nothing is stacked.
  __device__ __forceinline__ bool pop() {
    float4 *r = ring_slots();
    uint32_t base = ring & 15u, n = ring >> 4;
    if (n == 0u) {
      if (sp == 0) return false;
      --sp;   // bring the newest spilled record back into the ring
      r[0] = stk[sp].a;
      r[kTraceBlock] = stk[sp].b;
      r[2 * kTraceBlock] = stk[sp].c;
      base = 0u;
      n = 1u;
    }
    uint32_t pos = base + n - 1u;
    pos = pos >= kRing ? pos - kRing : pos;
    const float4 ra = r[(3 * pos) * kTraceBlock], rb = r[(3 * pos + 1) * kTraceBlock],
                 rc = r[(3 * pos + 2) * kTraceBlock];
    const uint32_t bits = __float_as_uint(rb.w);
    const uint32_t vm = bits >> 8;
    const uint32_t i = __ffs(vm) - 1u;   // the earliest visiting position left
    const uint32_t rest = vm & (vm - 1u);
    if (rest) {
      reinterpret_cast<uint32_t *>(r + (3 * pos + 1) * kTraceBlock)[3] = (bits & 0xffu) | (rest << 8);
      ring = base | (n << 4);
    } else {
      ring = n > 1u ? (base | ((n - 1u) << 4)) : 0u;   // an emptied ring restarts at position 0
    }
    const uint32_t cb = visit_bits(i);
    const uint32_t slot = cb ^ (octant & 7u);
    node = __float_as_uint(ra.w) + __popc(bits & 0xffu & ((1u << slot) - 1u));
    gate = cb | kGateFlag;
    lo = f3((cb & 4) ? rb.x : ra.x, (cb & 2) ? rb.y : ra.y, (cb & 1) ? rb.z : ra.z);
    hi = f3((cb & 4) ? rc.x : rb.x, (cb & 2) ? rc.y : rb.y, (cb & 1) ? rc.z : rb.z);
    return true;
  }

  // One octree entry (call only with no list pending and !finished()).
  //
  // An entry is processed as one call of the reference's recursive function:
  // parent gate, slab cull, then the node's surface list, then its children.
  // Here the qualifying children are pushed when the node is visited and its
  // list is tested afterwards; the push uses the ray's extent before those
  // tests, which only admits more children (the ray can only shrink), and
  // every entry's gate and cull are evaluated again when it is entered -- so
  // the tests and their order are the reference's.
  // ANY: the queries the calling kernel runs -- kClosestOnly, kAnyOnly or
  // kMixed (checked per ray) -- so closest-hit kernels carry no any-hit branch.
  template <bool FAST = true, int ANY = kMixed>
  __device__ __forceinline__ void node_step(TraceCounters &cnt) {
    if (!have && !pop()) return;
    have = false;
    const bool slow = !FAST || (octant & kSlowSlab);
    bool open = true;
    const bool any_query = ANY == kAnyOnly || (ANY == kMixed && (octant & kAnyHit));
    if ((gate & kGateFlag) && any_query) {
      // An any-hit query's extent never changes, so an entry with a parent
      // gate passed the very gate and cull it would be given now when it
      // was pushed (or entered): the call happens and the node is open.
      cnt.nodes++;
    } else {
      if (gate & kGateFlag) open = gate_open(gate & 7u, t0, t1, lo, hi);
      if (open) {
        cnt.nodes++;
        open = slow ? slab_open(t0, t1, lo, hi) : slab_open_finite(t0, t1, lo, hi);
      }
      if (!open) return;
    }
    const uint4 nd = __ldg(nodes + node);
    lp = nd.z;
    lend = nd.z + nd.w;
    if (!nd.y) return;
    // (hi - lo) / 2: halving rounds exactly like the reference's division by 2.
    const float3 half = f3(__fmul_rn(__fsub_rn(hi.x, lo.x), 0.5f), __fmul_rn(__fsub_rn(hi.y, lo.y), 0.5f),
                           __fmul_rn(__fsub_rn(hi.z, lo.z), 0.5f));
    // Per axis the children's bounds take two values each: the near half
    // spans [lo, lo + half], the far half [lo + half, lo + half + half] --
    // the same rounded sums as the reference's child ranges.
    const float3 mid = f3(__fadd_rn(lo.x, half.x), __fadd_rn(lo.y, half.y), __fadd_rn(lo.z, half.z));
    const float3 far = f3(__fadd_rn(mid.x, half.x), __fadd_rn(mid.y, half.y), __fadd_rn(mid.z, half.z));
    const float3 near_lo = f3(__fadd_rn(lo.x, 0.f), __fadd_rn(lo.y, 0.f), __fadd_rn(lo.z, 0.f));
    // Which children pass gate and cull, by visiting position (bit i).  At
    // most 4 pass: one octant per crossing of each of the three midplanes.
    const uint32_t oct = octant & 7u;
    uint32_t vm = 0;
    if (slow) {
#pragma unroll
      for (uint32_t i = 0; i < 8; i++) {
        const uint32_t cb = visit_bits(i);
        const uint32_t slot = cb ^ oct;
        const float3 clo = f3((cb & 4) ? mid.x : near_lo.x, (cb & 2) ? mid.y : near_lo.y,
                              (cb & 1) ? mid.z : near_lo.z);
        const float3 chi = f3((cb & 4) ? far.x : mid.x, (cb & 2) ? far.y : mid.y, (cb & 1) ? far.z : mid.z);
        const bool ok = ((nd.y >> slot) & 1u) & gate_open(cb, t0, t1, clo, chi) & slab_open(t0, t1, clo, chi);
        vm |= ok ? (1u << i) : 0u;
      }
    } else {
      // The same tests from shared pieces: per axis the near and far halves'
      // gates, and the child's entry max(t0, lo.x, lo.y, lo.z) and exit
      // min(t1, hi.x, hi.y, hi.z) built from an x part and a yz part.  The
      // pieces are scalars picked by selects, not small arrays: an array
      // indexed in the loop may be placed in local memory, which a node visit
      // would then write and read a dozen times.
      const bool gx0 = t0 < mid.x, gx1 = t1 > mid.x, gy0 = t0 < mid.y, gy1 = t1 > mid.y, gz0 = t0 < mid.z,
                 gz1 = t1 > mid.z;
      const float in_x0 = fmaxf(t0, near_lo.x), in_x1 = fmaxf(t0, mid.x);
      const float out_x0 = fminf(t1, mid.x), out_x1 = fminf(t1, far.x);
      const float in_yz00 = fmaxf(near_lo.y, near_lo.z), in_yz01 = fmaxf(near_lo.y, mid.z),
                  in_yz10 = fmaxf(mid.y, near_lo.z), in_yz11 = fmaxf(mid.y, mid.z);
      const float out_yz00 = fminf(mid.y, mid.z), out_yz01 = fminf(mid.y, far.z), out_yz10 = fminf(far.y, mid.z),
                  out_yz11 = fminf(far.y, far.z);
#pragma unroll
      for (uint32_t i = 0; i < 8; i++) {
        const uint32_t cb = visit_bits(i);
        const bool bx = (cb & 4u) != 0u, by = (cb & 2u) != 0u, bz = (cb & 1u) != 0u;
        const uint32_t slot = cb ^ oct;
        const float in_yz = by ? (bz ? in_yz11 : in_yz10) : (bz ? in_yz01 : in_yz00);
        const float out_yz = by ? (bz ? out_yz11 : out_yz10) : (bz ? out_yz01 : out_yz00);
        const bool ok = ((nd.y >> slot) & 1u) && (bx ? gx1 : gx0) && (by ? gy1 : gy0) && (bz ? gz1 : gz0) &&
                        (fmaxf(bx ? in_x1 : in_x0, in_yz) < fminf(bx ? out_x1 : out_x0, out_yz));
        vm |= ok ? (1u << i) : 0u;
      }
    }
    if (!vm) return;
    // The first qualifying child becomes the current entry; the others wait
    // in one record and are entered in visiting order after the first
    // child's subtree (pop), as the reference's loop over the children does.
    const uint32_t rest = vm & (vm - 1u);
    if (rest) push(near_lo, mid, far, nd.x, (nd.y & 0xffu) | (rest << 8), cnt);
    const uint32_t i = __ffs(vm) - 1u;
    const uint32_t cb = visit_bits(i);
    const uint32_t slot = cb ^ oct;
    node = nd.x + __popc(nd.y & ((1u << slot) - 1u));
    gate = cb | kGateFlag;
    lo = f3((cb & 4) ? mid.x : near_lo.x, (cb & 2) ? mid.y : near_lo.y, (cb & 1) ? mid.z : near_lo.z);
    hi = f3((cb & 4) ? far.x : mid.x, (cb & 2) ? far.y : mid.y, (cb & 1) ? far.z : mid.z);
    have = true;
  }
};

// Position of the K-th (1-based) set bit of MASK; MASK has at least K bits set.
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t mask, uint32_t k) {
  uint32_t p = 0;
#pragma unroll
  for (uint32_t w = 16; w >= 1; w >>= 1) {
    const uint32_t c = __popc((mask >> p) & ((1u << w) - 1u));   // set bits in [p, p + w)
    if (c < k) {
      k -= c;
      p += w;
    }
  }
  return p;
}

// One warp-cooperative round of list tests.  Every lane with a list pending
// (WANT) owns the next entries of its list; the warp's pending entries, in
// lane order and list order, are dealt to its 32 lanes (one or two
// consecutive entries per lane: at most 32 or 64 per round), each lane tests
// its entries against its owner's ray, and each owner takes the result of its
// own entries:
//  * closest queries: the smallest hit t, the earliest entry among equal t.
//    This is what the sequential test with a shrinking t1 keeps -- an entry
//    hits when its t (which does not depend on t1) is below t1 -- so the
//    result equals the reference's one-by-one loop;
//  * any-hit queries (ANY): the earliest entry that hits, where the
//    reference's loop stops.
// Test counts are the reference's (all entries, or up to the stopping one).
// All 32 lanes must call it together.  Returns true for an any-hit lane whose
// search is over.
// PER: entries dealt to a lane per round, 1 or 2.  Pairs (two consecutive
// entries of one list per lane, up to 64 per round) pay where the lists a
// ray meets are long: the ray-batch kernel uses them (random-triangle
// batches: 11 % faster), and the closest-hit kernels do for scenes whose
// probe found long lists along rays (SceneImpl's pair_lists: 8 % faster on
// a 2M-triangle soup, 3 % slower on the terrain, whose lists are short).
// Any-hit rounds deal single entries: a walk stops at its first hit.
template <int STACK, int ANY = kMixed, int PER = (ANY == kMixed ? 2 : 1)>
__device__ __forceinline__ bool list_round(Traversal<STACK> &tr, bool want, bool any, TraceCounters &cnt) {
  constexpr unsigned kFull = 0xffffffffu;
  constexpr uint32_t kPer = uint32_t(PER);
  const uint32_t lane = threadIdx.x & 31u;
  __syncwarp();   // the warp's ray-slot writes (new rays, shrunk t1) are visible
  uint32_t c = want ? tr.lend - tr.lp : 0u;
  c = c < 32u * kPer ? c : 32u * kPer;
  const uint32_t np = (c + kPer - 1u) / kPer;   // dealt units: pairs (or entries)
  uint32_t incl = np;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t v = __shfl_up_sync(kFull, incl, off);
    if (lane >= uint32_t(off)) incl += v;
  }
  const uint32_t excl = incl - np;
  const bool owner = np > 0u && excl < 32u;
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  if (total == 0u) return false;
  const bool item = lane < total;
  // The owner of the unit at this lane's position.
  uint32_t own = lane;
  if (ANY == kAnyOnly) {
    // The k-th owner, k the owners whose first unit lies at or before the
    // position.
    const uint32_t owners = __ballot_sync(kFull, owner);
    const uint32_t starts = __reduce_or_sync(kFull, owner ? (1u << excl) : 0u);
    const uint32_t upto = lane == 31u ? kFull : ((2u << lane) - 1u);
    if (item) own = nth_set_bit(owners, uint32_t(__popc(starts & upto)));
  } else {
    // The first lane whose inclusive count exceeds the position (the counts
    // never decrease with the lane): a binary search of five shuffles.
    // Fewer instructions than the bit search above (the closest-hit kernel
    // 2 % faster on the terrain frame), but a longer chain of dependent
    // latencies, which the any-hit kernel's frequent sparse rounds feel (2 %
    // slower with it).
    uint32_t first = 0u;
#pragma unroll
    for (uint32_t w = 16u; w >= 1u; w >>= 1) {
      const uint32_t v = __shfl_sync(kFull, incl, first + w - 1u);
      first += v <= lane ? w : 0u;
    }
    if (item) own = first;
  }
  // The owner's ray and list.
  const uint32_t o_excl = __shfl_sync(kFull, excl, own);
  const uint32_t o_lp = __shfl_sync(kFull, tr.lp, own);
  const uint32_t o_c = __shfl_sync(kFull, c, own);
  const bool o_any = ANY != kClosestOnly && ((__ballot_sync(kFull, any) >> own) & 1u) != 0u;
  uint32_t pid = PREF_END, which = 0u;
  bool hit = false;
  float th = 0.f;
  if (item) {
    const uint4 *slot = ray_slots() + ((threadIdx.x & ~31u) + own);
    const uint4 ra = slot[0], rb = slot[kTraceBlock];
    const float3 ro = f3(__uint_as_float(ra.x), __uint_as_float(ra.y), __uint_as_float(ra.z));
    const float3 rd = f3(__uint_as_float(rb.x), __uint_as_float(rb.y), __uint_as_float(rb.z));
    const float rt0 = __uint_as_float(ra.w);
    const float rt1 = __uint_as_float(rb.w);
    const uint4 rc = slot[2 * kTraceBlock];
    // The entries' primitive records from the owner's scene's list records.
    const unsigned long long o_lrec = (unsigned long long)rc.x | ((unsigned long long)rc.y << 32);
    const uint32_t k0 = kPer * (lane - o_excl);   // the first entry's index in the owner's round
    const float4 *p = reinterpret_cast<const float4 *>(o_lrec) + 3 * size_t(o_lp + k0);
    const PrimRec r0{__ldg(p), __ldg(p + 1), __ldg(p + 2)};
    th = rt1;
    hit = test_prim<ANY != kAnyOnly>(r0, ro, rd, rt0, th);
    pid = __float_as_uint(r0.c.w);
    if (kPer == 2u && k0 + 1u < o_c && !(hit && o_any)) {
      const PrimRec r1{__ldg(p + 3), __ldg(p + 4), __ldg(p + 5)};
      float th1 = rt1;
      const bool hit1 = test_prim<ANY != kAnyOnly>(r1, ro, rd, rt0, th1);
      // The later entry wins only with a smaller t (the earlier one keeps ties).
      if (hit1 && (!hit || __float_as_uint(th1) < __float_as_uint(th))) {
        hit = true;
        th = th1;
        pid = __float_as_uint(r1.c.w);
        which = 1u;
      }
    }
  }
  // Reduce over each owner's units (positive t: its bits order like the value).
  const unsigned grp = __match_any_sync(kFull, item ? own : 32u + lane);
  const uint32_t tb = hit ? __float_as_uint(th) : kFull;
  const uint32_t tmin = __reduce_min_sync(grp, tb);
  const uint32_t best = __reduce_min_sync(grp, (hit && (o_any || tb == tmin)) ? lane : kFull);
  // Each owner reads the result at its first unit's lane.
  const uint32_t b = __shfl_sync(kFull, best, owner ? excl : lane);
  const uint32_t src = b < 32u ? b : lane;
  const uint32_t b_pid = __shfl_sync(kFull, pid, src);
  const float b_t = __shfl_sync(kFull, th, src);
  const uint32_t b_which = __shfl_sync(kFull, which, src);
  if (!owner) return false;
  const uint32_t room = kPer * (32u - excl);
  const uint32_t used = c < room ? c : room;
  if (b < 32u) {
    tr.hit_ref = b_pid;
    if (any) {
      cnt.tests += kPer * (b - excl) + b_which + 1u;
      tr.lp = tr.lend;
      return true;
    }
    tr.set_t1(b_t);
  }
  cnt.tests += used;
  tr.lp += used;
  return false;
}

// Rays a warp takes per refill: 32 (one per lane) keeps the launch's tail
// short -- 32 rather than 64 measured 1.4 % faster on the terrain frame, 16 in
// between.
#ifndef SNOG_DISPENSE_CHUNK
#define SNOG_DISPENSE_CHUNK 32
#endif

// Idle lanes a warp gathers before it refills them (1 = refill at once).
#ifndef SNOG_REFILL_MIN
#define SNOG_REFILL_MIN 4
#endif
constexpr uint32_t kRefillMin = SNOG_REFILL_MIN;

// Pending list entries a closest-hit warp gathers before a list round.
#ifndef SNOG_ROUND_MIN
#define SNOG_ROUND_MIN 24
#endif
constexpr uint32_t kRoundMin = SNOG_ROUND_MIN;
// A warp with fewer than 32 entries pending visits nodes, and one with at
// least kRoundMin runs a round; a threshold above 32 would leave a warp with
// 32..kRoundMin-1 entries pending doing neither, for ever.
static_assert(kRoundMin >= 1u && kRoundMin <= 32u, "closest-hit round threshold must not exceed the node-step cut");

// Warp-cooperative ray dispenser for the persistent trace kernels: lanes
// whose ray is finished take the next index from a warp-local range of CHUNK
// rays, refilled with one atomic on the launch's counter.  All 32 lanes of
// the warp must call fetch() together.
struct RayDispenser {
  static constexpr uint32_t kChunk = SNOG_DISPENSE_CHUNK;
  static constexpr uint32_t kIdle = 0xffffffffu;
  uint32_t next = 0, end = 0;
  bool exhausted = false;

  // Returns the new ray index for a lane that asked (NEED) and got one,
  // else kIdle.  Sets *all_idle when every lane is idle and no rays remain.
  __device__ __forceinline__ uint32_t fetch(uint32_t *counter, uint32_t n, bool need, bool busy,
                                            bool *all_idle) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t mask = __ballot_sync(0xffffffffu, need);
    uint32_t got = kIdle;
    if (mask) {
      if (next >= end && !exhausted) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(counter, kChunk);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) {
          exhausted = true;
        } else {
          next = base;
          end = base + kChunk < n ? base + kChunk : n;
        }
      }
      const uint32_t rank = __popc(mask & ((1u << lane) - 1u));
      if (need && next + rank < end) got = next + rank;
      const uint32_t take = __popc(mask);
      next = (next + take < end) ? next + take : end;
    }
    const bool idle = !busy && got == kIdle;
    *all_idle = __all_sync(0xffffffffu, idle) && exhausted && next >= end;
    return got;
  }
};

// The persistent trace loop shared by the trace kernels.  Lanes take rays
// from DISPENSER (n rays) through a RayDispenser; START(i, tr, any) begins ray
// i (calls tr.init and sets ANY for an any-hit query); DONE(i, tr, any)
// stores its result.  Each iteration, unless the warp already has a full
// round of list entries pending, every live lane without a list pending
// visits one octree entry; then the warp tests one round of pending list
// entries together.  All 32 lanes of every warp must run it.
template <int STACK, int ANY = kMixed, int PER = (ANY == kMixed ? 2 : 1), class Start, class Done>
__device__ __forceinline__ void trace_loop(uint32_t *dispenser, uint32_t n, TraceCounters &cnt, Start start,
                                           Done done) {
  StackRec stk[Traversal<STACK>::kRecs];
  Traversal<STACK> tr;
  tr.stk = stk;
  RayDispenser disp;
  uint32_t ray = RayDispenser::kIdle;
  bool any = false;
  for (;;) {
    bool all_idle;
    // Idle lanes take new rays only once kRefillMin of them are idle: a ray
    // start (queue loads, root slab set-up, ray slot) then runs on several
    // lanes at once instead of on one or two every iteration.
    const uint32_t idle_lanes = __popc(__ballot_sync(0xffffffffu, ray == RayDispenser::kIdle));
    const bool need = ray == RayDispenser::kIdle && idle_lanes >= kRefillMin;
    const uint32_t got = disp.fetch(dispenser, n, need, ray != RayDispenser::kIdle, &all_idle);
    if (all_idle) break;
    if (got != RayDispenser::kIdle) {
      ray = got;
      start(ray, tr, any);
      if (any) tr.octant |= kAnyHit;
    }
    const bool busy = ray != RayDispenser::kIdle;
    // Visit nodes only while the warp's pending list entries would not fill
    // a round: list rounds run full, node steps run with more lanes at once.
    const uint32_t pend = (busy && tr.lp < tr.lend) ? tr.lend - tr.lp : 0u;
    const uint32_t pending = __reduce_add_sync(0xffffffffu, pend < 32u ? pend : 32u);
    if (pending < 32u && busy && tr.lp >= tr.lend && !tr.finished()) tr.template node_step<true, ANY>(cnt);
    // Closest-hit kernels test lists only once at least kRoundMin entries
    // are pending, unless no lane could visit a node: fewer, fuller rounds
    // (2 % off the terrain frame; the any-hit and mixed kernels, whose
    // lists are longer or whose walks end early, measured no gain or a
    // loss).
    bool round = true;
    if (ANY == kClosestOnly) {
      const uint32_t pend2 = (busy && tr.lp < tr.lend) ? tr.lend - tr.lp : 0u;
      const uint32_t pending2 = __reduce_add_sync(0xffffffffu, pend2 < 32u ? pend2 : 32u);
      const bool can_step = busy && tr.lp >= tr.lend && !tr.finished();
      round = pending2 >= kRoundMin || __ballot_sync(0xffffffffu, can_step) == 0u;
    }
    const bool stop = round && list_round<STACK, ANY, PER>(tr, busy && tr.lp < tr.lend, any, cnt);
    if (busy && (stop || tr.finished())) {
      done(ray, tr, any);
      ray = RayDispenser::kIdle;
    }
  }
}

// Global primitive id of a packed reference: triangles, then spheres, then
// tripars.
__device__ __forceinline__ int32_t prim_id_of(const DevScene &, uint32_t ref) {
  return ref == PREF_END ? -1 : int32_t(ref);
}

}  // namespace snog

#endif
