// octree_gpu.cu -- the octree of octree_build.h built on the device, node
// for node and list entry for list entry the tree the host builder makes
// (and so the reference's, space/octree-builder.cc:29-689), in the device
// layout of snog_common.h.
//
// Why it can be parallel.  The reference inserts surfaces one at a time, but
// where a surface lands depends only on its bounding box and on the root
// cube at the time of its insertion: it descends from that root into every
// octant it fits in (or, when small, touches) and is appended to the lists
// of the nodes where it stops.  Nodes are created on the way down, so every
// node is an ancestor of a list entry; lists are last-in first-out, i.e. in
// decreasing insertion order; and the final numbering is breadth first with
// children in octant order.  The only sequential part is the root's growth,
// which the host replays on the bounding boxes alone (root_start / root_fits
// / root_grow, shared with the host builder): each run of surfaces inserted
// under one root (an "epoch") descends from that root, which sits in the
// final tree below the octants later growths gave it.
//
// Steps (one thread per surface, then per placement, then per node):
//   1. count, then emit, one record per placement: the node's path as base-8
//      digits left-aligned in a 128-bit key with the depth in the low byte
//      (so keys sort in depth-first pre-order, a node before its subtree),
//      written in decreasing surface order;
//   2. stable radix sort by key (low word, then high word): within a node
//      the surfaces stay in decreasing insertion order, the list order;
//   3. distinct keys are the nodes with lists; each one's ancestors not
//      shared with the previous distinct key are new nodes, so a scan over
//      "depth - common prefix" enumerates every node in pre-order;
//   4. a stable sort of the nodes by depth gives breadth-first order (nodes
//      of one depth stay in path order); each node finds its parent by
//      binary search one level up and sets its bit in the parent's mask;
//   5. lists are laid out 4-aligned in breadth-first node order, padded with
//      PREF_END, as the host upload does.
//
// All float arithmetic of the descent is explicit round-to-nearest single
// precision in the host builder's operand order (the file is compiled with
// -fmad=false as well).

#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <string>
#include <vector>

#include "octree_gpu.h"

namespace snog {

namespace {

typedef unsigned __int128 u128;

constexpr uint32_t kMaxDigits = 40;      // 3 bits each in key bits 127..8
// Frames of one surface's descent (32 bytes each, local memory): 4 KB per
// thread, as much as the trace kernels take, so the context's local-memory
// reservation does not grow.  A descent that needs more is reported and the
// tree is left to the host builder.
constexpr int kDescentFrames = 128;

// Device error codes (first one wins).
enum : uint32_t { OE_DEPTH = 1, OE_STACK = 2 };

struct Epoch {
  uint32_t first;          // first surface (insertion index) under this root
  uint32_t depth;          // depth of this root in the final tree
  float o[3], size;        // the root cube while this epoch's surfaces went in
  unsigned long long khi, klo;   // this root's key
};

__host__ __device__ __forceinline__ u128 make_key(unsigned long long hi, unsigned long long lo) {
  return (u128(hi) << 64) | u128(lo);
}

// Key of the OC-th child of the node with key K (depth in the low byte).
__device__ __forceinline__ u128 child_key(u128 k, uint32_t oc) {
  const uint32_t d = uint32_t(k & 0xffu);
  return ((k & ~u128(0xffu)) | (u128(oc) << (125 - 3 * d))) | u128(d + 1);
}

// The first L digits of key K, as the key of that ancestor.
__device__ __forceinline__ u128 prefix_key(u128 k, uint32_t l) {
  const u128 digits = l ? (k & (~u128(0) << (128 - 3 * l))) : u128(0);
  return digits | u128(l);
}

__device__ __forceinline__ uint32_t clz128(u128 x) {
  const unsigned long long hi = (unsigned long long)(x >> 64), lo = (unsigned long long)x;
  return hi ? __clzll(hi) : 64u + (lo ? __clzll(lo) : 64u);
}

// BBox::avg_size (geometry/bbox.h:150-158): (ex + ey + ez) / 3.
__device__ __forceinline__ float avg_size(const Box3 &b) {
  const float ex = __fsub_rn(b.hi[0], b.lo[0]), ey = __fsub_rn(b.hi[1], b.lo[1]),
              ez = __fsub_rn(b.hi[2], b.lo[2]);
  return __fdiv_rn(__fadd_rn(__fadd_rn(ex, ey), ez), 3.0f);
}

// Low / high half membership at midpoint MID (as octree_build.cc).
__device__ __forceinline__ bool goes_low(float lo, float hi, float mid, bool force) {
  return hi < mid || (hi == mid && lo != hi) || (force && lo < mid);
}
__device__ __forceinline__ bool goes_high(float lo, float hi, float mid, bool force) {
  return lo > mid || (lo == mid && lo != hi) || (force && hi > mid);
}

struct Frame {
  float x, y, z, size;
  u128 key;
};

// Descend surface box B from its epoch's root (OctreeBuilder::insert):
// count the nodes it is listed in, and with EMIT write their keys.
template <bool EMIT>
__device__ uint32_t descend(const Box3 &b, const Epoch &e, unsigned long long *khi, unsigned long long *klo,
                            uint32_t pos, uint32_t *err) {
  Frame stack[kDescentFrames];
  int sp = 0;
  stack[sp++] = Frame{e.o[0], e.o[1], e.o[2], e.size, make_key(e.khi, e.klo)};
  const float avg = avg_size(b);
  uint32_t n = 0;
  while (sp > 0) {
    const Frame f = stack[--sp];
    const float sub = __fmul_rn(f.size, 0.5f);          // f.size / 2, exactly
    const float mx = __fadd_rn(f.x, sub), my = __fadd_rn(f.y, sub), mz = __fadd_rn(f.z, sub);
    const bool force = avg < __fmul_rn(f.size, 0.25f);  // f.size / 4, exactly
    const bool lx = goes_low(b.lo[0], b.hi[0], mx, force), hx = goes_high(b.lo[0], b.hi[0], mx, force);
    const bool ly = goes_low(b.lo[1], b.hi[1], my, force), hy = goes_high(b.lo[1], b.hi[1], my, force);
    const bool lz = goes_low(b.lo[2], b.hi[2], mz, force), hz = goes_high(b.lo[2], b.hi[2], mz, force);
    const uint32_t d = uint32_t(f.key & 0xffu);
    bool placed = false;
    for (int oc = 7; oc >= 0; oc--) {
      const bool bx = oc & 4, by = oc & 2, bz = oc & 1;
      if (!((bx ? hx : lx) && (by ? hy : ly) && (bz ? hz : lz))) continue;
      placed = true;
      if (d >= kMaxDigits) {
        atomicCAS(err, 0u, uint32_t(OE_DEPTH));
        return n;
      }
      if (sp >= kDescentFrames) {
        atomicCAS(err, 0u, uint32_t(OE_STACK));
        return n;
      }
      stack[sp++] = Frame{bx ? mx : f.x, by ? my : f.y, bz ? mz : f.z, sub, child_key(f.key, uint32_t(oc))};
    }
    if (!placed) {
      if (EMIT) {
        khi[pos + n] = (unsigned long long)(f.key >> 64);
        klo[pos + n] = (unsigned long long)f.key;
      }
      n++;
    }
  }
  return n;
}

__device__ __forceinline__ uint32_t epoch_of(const Epoch *ep, uint32_t n_ep, uint32_t i) {
  uint32_t lo = 0, hi = n_ep;   // last epoch with first <= i
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (ep[mid].first <= i) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void k_oct_count(const Box3 *boxes, uint32_t n, const Epoch *ep, uint32_t n_ep, uint32_t *count,
                            uint32_t *err) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    count[i] = descend<false>(boxes[i], ep[epoch_of(ep, n_ep, i)], nullptr, nullptr, 0, err);
}

// Placements of surface i go to [P - off[i] - count[i], P - off[i]): the
// array holds the surfaces in decreasing insertion order.
__global__ void k_oct_emit(const Box3 *boxes, const uint32_t *refs, uint32_t n, const Epoch *ep, uint32_t n_ep,
                           const uint32_t *count, const uint32_t *off, uint32_t P, unsigned long long *khi,
                           unsigned long long *klo, uint32_t *pref, uint32_t *err) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t pos = P - off[i] - count[i];
    const uint32_t c = descend<true>(boxes[i], ep[epoch_of(ep, n_ep, i)], khi, klo, pos, err);
    for (uint32_t j = 0; j < c; j++) pref[pos + j] = refs[i];
  }
}

__global__ void k_iota(uint32_t *v, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

template <class T>
__global__ void k_gather(const T *src, const uint32_t *idx, T *dst, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[idx[i]];
}

// flag[j] = placement j starts a new node (key differs from j - 1).
__global__ void k_oct_flags(const unsigned long long *khi, const unsigned long long *klo, uint32_t P,
                            uint32_t *flag) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < P; j += gridDim.x * blockDim.x)
    flag[j] = (j == 0 || khi[j] != khi[j - 1] || klo[j] != klo[j - 1]) ? 1u : 0u;
}

// Distinct key u: its first placement, and the number of nodes it adds in
// pre-order (its ancestors below the prefix it shares with key u - 1).
__global__ void k_oct_runs(const unsigned long long *khi, const unsigned long long *klo, const uint32_t *flag,
                           const uint32_t *uidx, uint32_t P, uint32_t *ustart, uint32_t *ucnt_nodes) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < P; j += gridDim.x * blockDim.x) {
    if (!flag[j]) continue;
    const uint32_t u = uidx[j];
    ustart[u] = j;
    const u128 k = make_key(khi[j], klo[j]);
    const uint32_t d = uint32_t(k & 0xffu);
    uint32_t add;
    if (j == 0) {
      add = d + 1;   // root .. the node itself
    } else {
      const u128 kp = make_key(khi[j - 1], klo[j - 1]);
      const uint32_t dp = uint32_t(kp & 0xffu);
      const u128 x = (k ^ kp) & ~u128(0xffu);
      uint32_t l = x ? clz128(x) / 3u : kMaxDigits;
      l = l < dp ? l : dp;
      l = l < d ? l : d;
      add = d - l;
    }
    ucnt_nodes[u] = add;
  }
}

// Emit the nodes distinct key u adds, in pre-order: prefixes of lengths
// (d - add, d], the last one being the node holding u's list.
__global__ void k_oct_nodes(const unsigned long long *khi, const unsigned long long *klo, const uint32_t *ustart,
                            const uint32_t *ucnt_nodes, const uint32_t *nbase, uint32_t U,
                            unsigned long long *nkhi, unsigned long long *nklo, uint32_t *ndepth,
                            uint32_t *list_node) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < U; u += gridDim.x * blockDim.x) {
    const uint32_t j = ustart[u];
    const u128 k = make_key(khi[j], klo[j]);
    const uint32_t d = uint32_t(k & 0xffu), add = ucnt_nodes[u], base = nbase[u];
    for (uint32_t t = 0; t < add; t++) {
      const uint32_t l = d + 1 - add + t;
      const u128 pk = prefix_key(k, l);
      nkhi[base + t] = (unsigned long long)(pk >> 64);
      nklo[base + t] = (unsigned long long)pk;
      ndepth[base + t] = l;
    }
    list_node[u] = base + add - 1;
  }
}

// First node of each depth in breadth-first order (depths are contiguous).
__global__ void k_oct_levels(const uint32_t *bdepth, uint32_t N, uint32_t *level_start) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < N; b += gridDim.x * blockDim.x)
    if (b == 0 || bdepth[b] != bdepth[b - 1]) level_start[bdepth[b]] = b;
}

__global__ void k_oct_init_nodes(uint4 *nodes, uint32_t N) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < N; b += gridDim.x * blockDim.x)
    nodes[b] = make_uint4(0xffffffffu, 0u, 0u, 0u);
}

// Link node b (breadth-first id, depth >= 1) to its parent: binary search of
// the parent's key among the nodes one level up, which are in key order.
__global__ void k_oct_link(const unsigned long long *bkhi, const unsigned long long *bklo, const uint32_t *bdepth,
                           const uint32_t *level_start, uint32_t N, uint4 *nodes) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < N; b += gridDim.x * blockDim.x) {
    const uint32_t d = bdepth[b];
    if (d == 0) continue;
    const u128 k = make_key(bkhi[b], bklo[b]);
    const u128 pk = prefix_key(k, d - 1);
    uint32_t lo = level_start[d - 1], hi = level_start[d];   // parent in [lo, hi)
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) / 2;
      if (make_key(bkhi[mid], bklo[mid]) <= pk) lo = mid;
      else hi = mid;
    }
    const uint32_t oc = uint32_t(k >> (125 - 3 * (d - 1))) & 7u;
    atomicOr(&nodes[lo].y, 1u << oc);
    atomicMin(&nodes[lo].x, b);
  }
}

// Per breadth-first node: list length (distinct key u -> its node).
__global__ void k_oct_list_len(const uint32_t *list_node, const uint32_t *dfs2bfs, const uint32_t *ustart,
                               uint32_t U, uint32_t P, uint32_t *blen, uint32_t *bpad) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < U; u += gridDim.x * blockDim.x) {
    const uint32_t b = dfs2bfs[list_node[u]];
    const uint32_t len = (u + 1 < U ? ustart[u + 1] : P) - ustart[u];
    blen[b] = len;
    bpad[b] = (len + 3u) & ~3u;
  }
}

__global__ void k_oct_finish_nodes(uint4 *nodes, const uint32_t *blen, const uint32_t *boff, uint32_t N,
                                   uint32_t *n_leaf) {
  uint32_t leaves = 0;
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < N; b += gridDim.x * blockDim.x) {
    uint4 r = nodes[b];
    if (r.y == 0) {
      r.x = 0;
      leaves++;
    }
    r.z = blen[b] ? 4u + boff[b] : 0u;
    r.w = blen[b];
    nodes[b] = r;
  }
  if (leaves) atomicAdd(n_leaf, leaves);
}

__global__ void k_oct_fill_lists(const uint32_t *pref_sorted, const uint32_t *flag_scan, const uint32_t *flag,
                                 const uint32_t *ustart, const uint32_t *list_node, const uint32_t *dfs2bfs,
                                 const uint32_t *boff, uint32_t P, uint32_t *plist) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < P; j += gridDim.x * blockDim.x) {
    const uint32_t u = flag_scan[j] + flag[j] - 1u;
    const uint32_t b = dfs2bfs[list_node[u]];
    plist[4u + boff[b] + (j - ustart[u])] = pref_sorted[j];
  }
}

__global__ void k_scatter_inverse(const uint32_t *perm, uint32_t n, uint32_t *inv) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) inv[perm[i]] = i;
}

// Temporary device memory of one build, freed on every exit path.
struct Scratch {
  std::vector<void *> p;
  template <class T>
  T *get(size_t n) {
    void *q = nullptr;
    check_cuda(cudaMalloc(&q, n ? n * sizeof(T) : 16), "octree build scratch");
    p.push_back(q);
    return static_cast<T *>(q);
  }
  ~Scratch() {
    for (void *q : p) cudaFree(q);
  }
};

unsigned grid_for(size_t n) {
  size_t g = (n + 255) / 256;
  if (g < 1) g = 1;
  if (g > 148 * 16) g = 148 * 16;
  return unsigned(g);
}

template <class T>
void exclusive_sum(Scratch &S, const T *in, T *out, uint32_t n, cudaStream_t st) {
  size_t bytes = 0;
  check_cuda(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, st), "scan");
  void *tmp = S.get<unsigned char>(bytes);
  check_cuda(cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, n, st), "scan");
}

template <class K>
void sort_pairs(Scratch &S, const K *kin, K *kout, const uint32_t *vin, uint32_t *vout, uint32_t n, int end_bit,
                cudaStream_t st) {
  size_t bytes = 0;
  check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, n, 0, end_bit, st), "sort");
  void *tmp = S.get<unsigned char>(bytes);
  check_cuda(cub::DeviceRadixSort::SortPairs(tmp, bytes, kin, kout, vin, vout, n, 0, end_bit, st), "sort");
}

template <class T>
T read_back(const T *d, cudaStream_t st) {
  T v;
  check_cuda(cudaMemcpyAsync(&v, d, sizeof(T), cudaMemcpyDeviceToHost, st), "read back");
  check_cuda(cudaStreamSynchronize(st), "octree build");
  return v;
}

}  // namespace

void build_octree_device(const std::vector<Box3> &boxes, const std::vector<uint32_t> &refs, DeviceArena &A,
                         DeviceOctree &out) {
  out = DeviceOctree{};
  const uint32_t n = uint32_t(boxes.size());
  cudaStream_t st = nullptr;   // legacy stream: ordered with the scene's uploads
  if (n == 0) {
    std::vector<uint32_t> pl(4, PREF_END);
    out.nodes = static_cast<uint4 *>(A.alloc(0));
    out.plist = static_cast<uint32_t *>(A.upload(pl.data(), pl.size() * 4));
    out.n_plist4 = 4;
    out.n_plist_host = 1;
    return;
  }

  // ---- 0. the root's growth, replayed on the host --------------------------
  // One epoch per root a surface was inserted under; Epoch::depth first holds
  // the number of growths before the epoch, then the root's depth.
  std::vector<Epoch> ep;
  std::vector<uint32_t> grow_octant;   // octant given to the old root, per growth
  float o[3], size;
  root_start(boxes[0], o, size);
  ep.push_back(Epoch{0, 0, {o[0], o[1], o[2]}, size, 0, 0});
  for (uint32_t i = 1; i < n; i++) {
    if (root_fits(o, size, boxes[i])) continue;
    while (!root_fits(o, size, boxes[i])) grow_octant.push_back(root_grow(boxes[i], o, size));
    ep.push_back(Epoch{i, uint32_t(grow_octant.size()), {o[0], o[1], o[2]}, size, 0, 0});
  }
  const uint32_t G = uint32_t(grow_octant.size());
  if (G > kMaxDigits) throw Error{SNOG_EINVAL, "octree root grew more than 40 times"};
  // An epoch's root lies below the octants of every later growth: its digits,
  // from the final root, are the octants of growths G-1, G-2, ..., down to
  // its own number of growths.
  for (Epoch &e : ep) {
    u128 key = 0;
    uint32_t d = 0;
    for (uint32_t gi = G; gi-- > e.depth;) {
      key |= u128(grow_octant[gi]) << (125 - 3 * d);
      d++;
    }
    key |= u128(d);
    e.depth = d;
    e.khi = (unsigned long long)(key >> 64);
    e.klo = (unsigned long long)key;
  }
  for (int k = 0; k < 3; k++) out.origin[k] = o[k];
  out.size = size;

  Scratch S;
  Box3 *d_boxes = S.get<Box3>(n);
  uint32_t *d_refs = S.get<uint32_t>(n);
  Epoch *d_ep = S.get<Epoch>(ep.size());
  uint32_t *d_err = S.get<uint32_t>(2);
  check_cuda(cudaMemcpyAsync(d_boxes, boxes.data(), n * sizeof(Box3), cudaMemcpyHostToDevice, st), "upload");
  check_cuda(cudaMemcpyAsync(d_refs, refs.data(), n * 4, cudaMemcpyHostToDevice, st), "upload");
  check_cuda(cudaMemcpyAsync(d_ep, ep.data(), ep.size() * sizeof(Epoch), cudaMemcpyHostToDevice, st), "upload");
  check_cuda(cudaMemsetAsync(d_err, 0, 8, st), "memset");

  // ---- 1. placements -------------------------------------------------------
  uint32_t *d_count = S.get<uint32_t>(n + 1), *d_off = S.get<uint32_t>(n + 1);
  k_oct_count<<<grid_for(n), 256, 0, st>>>(d_boxes, n, d_ep, uint32_t(ep.size()), d_count, d_err);
  check_cuda(cudaMemsetAsync(d_count + n, 0, 4, st), "memset");
  exclusive_sum(S, d_count, d_off, n + 1, st);
  if (uint32_t e = read_back(d_err, st))
    throw Error{SNOG_EINVAL, e == OE_DEPTH ? "octree deeper than 40 levels" : "octree descent stack overflow"};
  const uint32_t P = read_back(d_off + n, st);
  unsigned long long *khi = S.get<unsigned long long>(P), *klo = S.get<unsigned long long>(P);
  uint32_t *pref = S.get<uint32_t>(P);
  k_oct_emit<<<grid_for(n), 256, 0, st>>>(d_boxes, d_refs, n, d_ep, uint32_t(ep.size()), d_count, d_off, P, khi,
                                         klo, pref, d_err);
  check_cuda(cudaGetLastError(), "octree emit");

  // ---- 2. stable sort by key -----------------------------------------------
  uint32_t *idx0 = S.get<uint32_t>(P), *idx1 = S.get<uint32_t>(P), *idx2 = S.get<uint32_t>(P);
  unsigned long long *ks = S.get<unsigned long long>(P), *kg = S.get<unsigned long long>(P);
  k_iota<<<grid_for(P), 256, 0, st>>>(idx0, P);
  sort_pairs(S, klo, ks, idx0, idx1, P, 64, st);
  k_gather<<<grid_for(P), 256, 0, st>>>(khi, idx1, kg, P);
  sort_pairs(S, kg, ks, idx1, idx2, P, 64, st);                 // ks = sorted high words
  unsigned long long *klo_s = kg;                               // reuse
  k_gather<<<grid_for(P), 256, 0, st>>>(klo, idx2, klo_s, P);
  unsigned long long *khi_s = ks;
  uint32_t *pref_s = idx0;                                      // reuse
  k_gather<<<grid_for(P), 256, 0, st>>>(pref, idx2, pref_s, P);

  // ---- 3. distinct keys and the nodes they add -------------------------------
  uint32_t *flag = S.get<uint32_t>(P + 1), *fscan = S.get<uint32_t>(P + 1);
  k_oct_flags<<<grid_for(P), 256, 0, st>>>(khi_s, klo_s, P, flag);
  check_cuda(cudaMemsetAsync(flag + P, 0, 4, st), "memset");
  exclusive_sum(S, flag, fscan, P + 1, st);
  const uint32_t U = read_back(fscan + P, st);
  uint32_t *ustart = S.get<uint32_t>(U), *uadd = S.get<uint32_t>(U + 1), *nbase = S.get<uint32_t>(U + 1);
  k_oct_runs<<<grid_for(P), 256, 0, st>>>(khi_s, klo_s, flag, fscan, P, ustart, uadd);
  check_cuda(cudaMemsetAsync(uadd + U, 0, 4, st), "memset");
  exclusive_sum(S, uadd, nbase, U + 1, st);
  const uint32_t N = read_back(nbase + U, st);
  unsigned long long *nkhi = S.get<unsigned long long>(N), *nklo = S.get<unsigned long long>(N);
  uint32_t *ndepth = S.get<uint32_t>(N), *list_node = S.get<uint32_t>(U);
  k_oct_nodes<<<grid_for(U), 256, 0, st>>>(khi_s, klo_s, ustart, uadd, nbase, U, nkhi, nklo, ndepth, list_node);

  // ---- 4. breadth-first order and links ------------------------------------
  uint32_t *dfs_iota = S.get<uint32_t>(N), *bfs2dfs = S.get<uint32_t>(N), *bdepth = S.get<uint32_t>(N);
  uint32_t *dfs2bfs = S.get<uint32_t>(N);
  k_iota<<<grid_for(N), 256, 0, st>>>(dfs_iota, N);
  sort_pairs(S, ndepth, bdepth, dfs_iota, bfs2dfs, N, 8, st);
  k_scatter_inverse<<<grid_for(N), 256, 0, st>>>(bfs2dfs, N, dfs2bfs);
  unsigned long long *bkhi = S.get<unsigned long long>(N), *bklo = S.get<unsigned long long>(N);
  k_gather<<<grid_for(N), 256, 0, st>>>(nkhi, bfs2dfs, bkhi, N);
  k_gather<<<grid_for(N), 256, 0, st>>>(nklo, bfs2dfs, bklo, N);
  const uint32_t maxd = read_back(bdepth + (N - 1), st);
  uint32_t *level_start = S.get<uint32_t>(maxd + 2);
  k_oct_levels<<<grid_for(N), 256, 0, st>>>(bdepth, N, level_start);
  check_cuda(cudaMemcpyAsync(level_start + maxd + 1, &N, 4, cudaMemcpyHostToDevice, st), "upload");
  uint4 *nodes = static_cast<uint4 *>(A.alloc(size_t(N) * sizeof(uint4)));
  k_oct_init_nodes<<<grid_for(N), 256, 0, st>>>(nodes, N);
  k_oct_link<<<grid_for(N), 256, 0, st>>>(bkhi, bklo, bdepth, level_start, N, nodes);

  // ---- 5. lists -------------------------------------------------------------
  uint32_t *blen = S.get<uint32_t>(N + 1), *bpad = S.get<uint32_t>(N + 1), *boff = S.get<uint32_t>(N + 1);
  check_cuda(cudaMemsetAsync(blen, 0, (N + 1) * 4, st), "memset");
  check_cuda(cudaMemsetAsync(bpad, 0, (N + 1) * 4, st), "memset");
  k_oct_list_len<<<grid_for(U), 256, 0, st>>>(list_node, dfs2bfs, ustart, U, P, blen, bpad);
  exclusive_sum(S, bpad, boff, N + 1, st);
  const uint32_t n_plist4 = 4 + read_back(boff + N, st);
  uint32_t *plist = static_cast<uint32_t *>(A.alloc(size_t(n_plist4) * 4));
  check_cuda(cudaMemsetAsync(plist, 0xff, size_t(n_plist4) * 4, st), "memset");
  k_oct_fill_lists<<<grid_for(P), 256, 0, st>>>(pref_s, fscan, flag, ustart, list_node, dfs2bfs, boff, P, plist);
  uint32_t *d_leaf = d_err + 1;
  k_oct_finish_nodes<<<grid_for(N), 256, 0, st>>>(nodes, blen, boff, N, d_leaf);
  check_cuda(cudaGetLastError(), "octree build");
  out.n_leaf = read_back(d_leaf, st);
  if (uint32_t e = read_back(d_err, st))
    throw Error{SNOG_EINVAL, e == OE_DEPTH ? "octree deeper than 40 levels" : "octree descent stack overflow"};

  out.nodes = nodes;
  out.plist = plist;
  out.n_nodes = N;
  out.n_plist4 = n_plist4;
  out.n_plist_host = 1 + P + U;
  out.max_depth = maxd + 1;
  out.n_list_surfaces = P;
}

// Host arrays (octree_build.h layout) of a tree in the device layout.
OctreeArrays octree_from_device(const uint4 *d_nodes, uint32_t n_nodes, const uint32_t *d_plist, uint32_t n_plist4,
                                const float origin[3], float size, uint32_t max_depth) {
  std::vector<uint4> nodes(n_nodes);
  std::vector<uint32_t> pl(n_plist4);
  if (n_nodes) check_cuda(cudaMemcpy(nodes.data(), d_nodes, n_nodes * sizeof(uint4), cudaMemcpyDeviceToHost), "download");
  if (n_plist4) check_cuda(cudaMemcpy(pl.data(), d_plist, size_t(n_plist4) * 4, cudaMemcpyDeviceToHost), "download");
  OctreeArrays o;
  o.children.assign(8 * size_t(n_nodes), 0);
  o.heads.assign(n_nodes, 0);
  o.plist.push_back(PREF_END);
  for (int k = 0; k < 3; k++) o.origin[k] = origin[k];
  o.size = size;
  o.max_depth = max_depth;
  for (uint32_t i = 0; i < n_nodes; i++) {
    const uint4 r = nodes[i];
    if (r.y == 0) {
      o.children[8 * size_t(i)] = o.children[8 * size_t(i) + 1] = 1;
      o.n_leaf++;
    } else {
      uint32_t c = r.x;
      for (uint32_t s = 0; s < 8; s++)
        if ((r.y >> s) & 1u) o.children[8 * size_t(i) + s] = c++;
    }
    if (r.w) {
      o.heads[i] = uint32_t(o.plist.size());
      for (uint32_t e = 0; e < r.w; e++) o.plist.push_back(pl[r.z + e]);
      o.plist.push_back(PREF_END);
      o.n_list_surfaces += r.w;
    }
  }
  return o;
}

}  // namespace snog
