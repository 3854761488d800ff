// trace.cu -- ray-batch closest-hit / any-hit kernels behind snog_trace*.
//
// One thread per ray, SoA input (ox oy oz dx dy dz tmax), coalesced 32-bit
// loads and stores; the octree walk itself is in trace.cuh.  Counters are
// reduced per warp and added with one atomic per warp.

#include <cuda_runtime.h>

#include "launch.h"
#include "trace.cuh"

namespace snog {

template <int STACK>
__global__ void __launch_bounds__(128) k_trace_batch(DevScene s, const float *__restrict__ rays,
                                                     uint32_t n, uint32_t n_closest,
                                                     int32_t *__restrict__ prim, float *__restrict__ tout,
                                                     float *__restrict__ nrm,
                                                     unsigned long long *__restrict__ counters,
                                                     uint32_t *__restrict__ err) {
  const uint32_t stride = gridDim.x * blockDim.x;
  unsigned long long cn = 0, ct = 0, an = 0, at = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    float3 o = f3(rays[i], rays[size_t(n) + i], rays[2 * size_t(n) + i]);
    float3 d = f3(rays[3 * size_t(n) + i], rays[4 * size_t(n) + i], rays[5 * size_t(n) + i]);
    float t1 = rays[6 * size_t(n) + i];
    TraceCounters c{0, 0, 0};
    const bool closest = i < n_closest;
    uint32_t ref = closest ? traverse<false, STACK>(s, o, d, 0.f, t1, c)
                           : traverse<true, STACK>(s, o, d, 0.f, t1, c);
    prim[i] = prim_id_of(s, ref);
    if (tout) tout[i] = (closest && ref != PREF_END) ? t1 : 0.f;
    if (nrm) {
      float3 nv = f3(0.f, 0.f, 0.f);
      if (closest && ref != PREF_END) {
        const uint32_t kind = ref >> 30, idx = ref & PREF_INDEX_MASK;
        if (kind == PK_SPHERE) {
          // Sphere::IsecInfo::normal: (ray.end () - centre).unit () (surface/sphere.cc:96-100)
          float4 sp = s.sph[idx];
          float3 end = xadd(o, xmul(d, t1));
          float3 v = xsub(end, xyz(sp));
          nv = xmul(v, __fdiv_rn(1.0f, __fsqrt_rn(xlen_sq(v))));
        } else {
          // Triangles (left-handed mesh) and tripars: (e2 x e1).unit ()
          // (surface/mesh.cc:713-718, surface/tripar.cc:78-82).
          const float4 *p = (kind == PK_TRI ? s.tri : s.tpar) + 3 * size_t(idx);
          float3 v = xcross(xyz(p[2]), xyz(p[1]));
          nv = xmul(v, __fdiv_rn(1.0f, __fsqrt_rn(xlen_sq(v))));
        }
      }
      nrm[3 * size_t(i)] = nv.x;
      nrm[3 * size_t(i) + 1] = nv.y;
      nrm[3 * size_t(i) + 2] = nv.z;
    }
    if (c.overflow) atomicOr(err, 1u);
    if (closest) {
      cn += c.nodes;
      ct += c.tests;
    } else {
      an += c.nodes;
      at += c.tests;
    }
  }
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
                               uint32_t *err, cudaStream_t st, int *launches) {
  if (n == 0) return cudaSuccess;
  const int threads = 128;
  int sms = num_sms();
  uint32_t blocks = (n + threads - 1) / threads;
  uint32_t cap = uint32_t(sms) * 16;
  if (blocks > cap) blocks = cap;
  switch (stack_class_for_depth(s.max_depth)) {
    case 32: k_trace_batch<32><<<blocks, threads, 0, st>>>(s, rays, n, n_closest, prim, t, nrm, counters, err); break;
    case 64: k_trace_batch<64><<<blocks, threads, 0, st>>>(s, rays, n, n_closest, prim, t, nrm, counters, err); break;
    case 128: k_trace_batch<128><<<blocks, threads, 0, st>>>(s, rays, n, n_closest, prim, t, nrm, counters, err); break;
    case 256: k_trace_batch<256><<<blocks, threads, 0, st>>>(s, rays, n, n_closest, prim, t, nrm, counters, err); break;
    default: return cudaErrorInvalidValue;
  }
  if (launches) (*launches)++;
  return cudaGetLastError();
}

}  // namespace snog
