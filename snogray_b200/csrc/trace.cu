// trace.cu -- ray-batch closest-hit / any-hit kernels behind snog_trace*.
//
// One thread per ray, SoA input (ox oy oz dx dy dz tmax), coalesced 32-bit
// loads and stores; the octree walk itself is in trace.cuh.  Counters are
// reduced per warp and added with one atomic per warp.

#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "launch.h"
#include "scene.h"
#include "trace.cuh"

namespace snog {

// The ray-batch kernel carries per-query counters and the normal output on
// top of the walk; at 7 blocks per SM (72 registers) it spills a few bytes
// instead of about a hundred at 8.
#ifndef SNOG_TRACE_BATCH_MINBLOCKS
#define SNOG_TRACE_BATCH_MINBLOCKS 7
#endif

template <int STACK>
__global__ void __launch_bounds__(kTraceBlock, SNOG_TRACE_BATCH_MINBLOCKS) k_trace_batch(DevScene s, const float *__restrict__ rays,
                                                     uint32_t n, uint32_t n_closest,
                                                     int32_t *__restrict__ prim, float *__restrict__ tout,
                                                     float *__restrict__ nrm,
                                                     unsigned long long *__restrict__ counters,
                                                     uint32_t *__restrict__ err, uint32_t *__restrict__ fetch) {
  unsigned long long cn = 0, ct = 0, an = 0, at = 0;
  TraceCounters c{0, 0, 0}, base{0, 0, 0};
  auto start = [&](uint32_t ray, Traversal<STACK> &tr, bool &any) {
    tr.init(s, f3(rays[ray], rays[size_t(n) + ray], rays[2 * size_t(n) + ray]),
            f3(rays[3 * size_t(n) + ray], rays[4 * size_t(n) + ray], rays[5 * size_t(n) + ray]), 0.f,
            rays[6 * size_t(n) + ray]);
    any = ray >= n_closest;
    base = c;
  };
  auto done = [&](uint32_t i, Traversal<STACK> &tr, bool any) {
    const bool closest = !any;
    const uint32_t ref = tr.hit_ref;
    prim[i] = prim_id_of(s, ref);
    if (tout) tout[i] = (closest && ref != PREF_END) ? tr.t1 : 0.f;
    if (nrm) {
      float3 nv = f3(0.f, 0.f, 0.f);
      if (closest && ref != PREF_END) {
        const PrimRec r = load_prim(s, ref);
        if (r.a.w == float(PRIM_SPHERE)) {
          // Sphere::IsecInfo::normal: (ray.end () - centre).unit () (surface/sphere.cc:96-100)
          float3 end = xadd(tr.ray_o(), xmul(tr.ray_d(), tr.t1));
          float3 v = xsub(end, xyz(r.a));
          nv = xmul(v, __fdiv_rn(1.0f, __fsqrt_rn(xlen_sq(v))));
        } else {
          // Triangles: (e2 x e1).unit () for a left-handed mesh, (e1 x e2)
          // for a right-handed one; tripars: e2 x e1 (surface/mesh.cc:264-271,
          // 713-718, surface/tripar.cc:78-82).
          const bool rh = r.a.w == float(PRIM_TRI) && s.right_handed;
          float3 v = rh ? xcross(xyz(r.b), xyz(r.c)) : xcross(xyz(r.c), xyz(r.b));
          nv = xmul(v, __fdiv_rn(1.0f, __fsqrt_rn(xlen_sq(v))));
        }
      }
      nrm[3 * size_t(i)] = nv.x;
      nrm[3 * size_t(i) + 1] = nv.y;
      nrm[3 * size_t(i) + 2] = nv.z;
    }
    if (closest) {
      cn += c.nodes - base.nodes;
      ct += c.tests - base.tests;
    } else {
      an += c.nodes - base.nodes;
      at += c.tests - base.tests;
    }
  };
  trace_loop<STACK>(fetch, n, c, start, done);
  if (c.overflow) atomicOr(err, 1u);
  if (counters) {
    // All lanes reach this point: reduce per warp, one atomic per warp.
    for (int off = 16; off > 0; off >>= 1) {
      cn += __shfl_down_sync(0xffffffffu, cn, off);
      ct += __shfl_down_sync(0xffffffffu, ct, off);
      an += __shfl_down_sync(0xffffffffu, an, off);
      at += __shfl_down_sync(0xffffffffu, at, off);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(counters + 0, cn);
      atomicAdd(counters + 1, ct);
      atomicAdd(counters + 2, an);
      atomicAdd(counters + 3, at);
    }
  }
}

// Stack depth needed for a tree of depth D: at most 3 pending entries per
// level (4 children can pass, one is entered), plus slack.
// One 48-byte primitive record per surface-list slot, in list order: the
// record of the slot's primitive id, with the id in c.w (padding slots get a
// zero record, never read).
__global__ void k_list_records(const uint32_t *__restrict__ plist, uint32_t n, const float4 *__restrict__ prims,
                               float4 *__restrict__ lrec) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t id = plist[i];
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a, c = a;
    if (id != PREF_END) {
      a = prims[3 * size_t(id)];
      b = prims[3 * size_t(id) + 1];
      c = prims[3 * size_t(id) + 2];
      c.w = __uint_as_float(id);
    }
    lrec[3 * size_t(i)] = a;
    lrec[3 * size_t(i) + 1] = b;
    lrec[3 * size_t(i) + 2] = c;
  }
}

cudaError_t build_list_records(const uint32_t *plist, uint32_t n, const float4 *prims, float4 *lrec,
                               cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const uint32_t blocks = (n + 255) / 256 < 65535u ? (n + 255) / 256 : 65535u;
  k_list_records<<<blocks, 256, 0, st>>>(plist, n, prims, lrec);
  return cudaGetLastError();
}

uint32_t probe_pair_lists(const DevScene &s) {
  constexpr uint32_t n = 8192;
  if (!s.n_nodes || !stack_class_for_depth(s.max_depth)) return 0;
  // Random rays through the scene's bounding box (fixed seed: the choice is
  // the same every time the scene is built).
  std::vector<float> rays(size_t(n) * 7);
  uint64_t x = 0x9e3779b97f4a7c15ull;
  auto uni = [&x]() {
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    return float(double(x >> 40) * (1.0 / 16777216.0));
  };
  for (uint32_t i = 0; i < n; i++) {
    for (int k = 0; k < 3; k++) rays[size_t(k) * n + i] = s.bbox_min[k] + (s.bbox_max[k] - s.bbox_min[k]) * uni();
    const float z = 2.f * uni() - 1.f, phi = 6.2831853f * uni(), r = std::sqrt(std::fmax(0.f, 1.f - z * z));
    rays[3 * size_t(n) + i] = r * std::cos(phi);
    rays[4 * size_t(n) + i] = r * std::sin(phi);
    rays[5 * size_t(n) + i] = z;
    rays[6 * size_t(n) + i] = INFINITY;
  }
  char *block = nullptr;
  const size_t rb = rays.size() * 4, pb = size_t(n) * 4;
  check_cuda(cudaMalloc(&block, rb + pb + 64), "probe buffers");
  unsigned long long cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  cudaError_t e = cudaMemcpy(block, rays.data(), rb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(block + rb + pb, 0, 64);
  if (e == cudaSuccess) {
    unsigned long long *c = reinterpret_cast<unsigned long long *>(block + rb + pb);
    e = launch_trace_batch(s, reinterpret_cast<const float *>(block), n, n, reinterpret_cast<int32_t *>(block + rb),
                           nullptr, nullptr, c, reinterpret_cast<uint32_t *>(c) + 8, reinterpret_cast<uint32_t *>(c) + 9,
                           nullptr, nullptr);
  }
  if (e == cudaSuccess) e = cudaMemcpy(cnt, block + rb + pb, 64, cudaMemcpyDeviceToHost);
  cudaFree(block);
  check_cuda(e, "list probe");
  // cnt[0]: node visits, cnt[1]: primitive tests of the closest-hit queries
  return cnt[1] > 5 * cnt[0] / 2 ? 1u : 0u;
}

int stack_class_for_depth(uint32_t depth) {
  uint32_t need = 3 * depth + 4;
  if (need <= 32) return 32;
  if (need <= 64) return 64;
  if (need <= 128) return 128;
  if (need <= 256) return 256;
  return 0;
}

cudaError_t launch_trace_batch(const DevScene &s, const float *rays, uint32_t n, uint32_t n_closest,
                               int32_t *prim, float *t, float *nrm, unsigned long long *counters,
                               uint32_t *err, uint32_t *fetch, cudaStream_t st, int *launches) {
  if (n == 0) return cudaSuccess;
  const int threads = kTraceBlock;
  const uint32_t want = (n + threads - 1) / threads;
  auto grid = [&](uint32_t resident) { return want < resident ? want : resident; };
  switch (stack_class_for_depth(s.max_depth)) {
    case 32: k_trace_batch<32><<<grid(resident_grid(k_trace_batch<32>, threads)), threads, 0, st>>>(s, rays, n, n_closest, prim, t, nrm, counters, err, fetch); break;
    case 64: k_trace_batch<64><<<grid(resident_grid(k_trace_batch<64>, threads)), threads, 0, st>>>(s, rays, n, n_closest, prim, t, nrm, counters, err, fetch); break;
    case 128: k_trace_batch<128><<<grid(resident_grid(k_trace_batch<128>, threads)), threads, 0, st>>>(s, rays, n, n_closest, prim, t, nrm, counters, err, fetch); break;
    case 256: k_trace_batch<256><<<grid(resident_grid(k_trace_batch<256>, threads)), threads, 0, st>>>(s, rays, n, n_closest, prim, t, nrm, counters, err, fetch); break;
    default: return cudaErrorInvalidValue;
  }
  if (launches) (*launches)++;
  return cudaGetLastError();
}

}  // namespace snog
