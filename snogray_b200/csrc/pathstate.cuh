// pathstate.cuh -- per-path state helpers shared by the two path tracers
// (wavefront.cu: one job in waves; engine.cu: many jobs streamed with path
// regeneration).
//
// A path's 32-bit state word holds its length (8 bits), the after-specular
// flag (1 bit), the media-stack depth (3 bits) and up to four medium ids
// (5 bits each: a scene has at most 31 distinct media besides the default).

#ifndef SNOG_PATHSTATE_CUH
#define SNOG_PATHSTATE_CUH

#include "shade.cuh"

namespace snog {

__device__ __forceinline__ uint32_t ps_len(uint32_t p) { return p & 0xffu; }
__device__ __forceinline__ bool ps_spec(uint32_t p) { return (p >> 8) & 1u; }
__device__ __forceinline__ uint32_t ps_depth(uint32_t p) { return (p >> 9) & 7u; }
__device__ __forceinline__ uint32_t ps_medium(uint32_t p, uint32_t k) { return (p >> (12 + 5 * k)) & 0x1fu; }

constexpr uint32_t kMediaStack = 4;   // media-stack entries in the path state word

// Media::update_stack_for_transmission (material/media.cc:76-118): entering a
// surface with a medium pushes it, leaving pops (never below the camera's
// medium).  The reference's stack is an unbounded list; this one holds four
// entries, and a fifth push returns false (the caller ends the path and
// reports the overflow as an error).
__device__ __forceinline__ bool ps_push(uint32_t &p, uint32_t mid) {
  const uint32_t d = ps_depth(p);
  if (d >= kMediaStack) return false;
  p = (p & ~(7u << 9)) | ((d + 1) << 9);
  p = (p & ~(0x1fu << (12 + 5 * d))) | ((mid & 0x1fu) << (12 + 5 * d));
  return true;
}
__device__ __forceinline__ uint32_t ps_pop(uint32_t p) {
  uint32_t d = ps_depth(p);
  if (d == 0) return p;
  return (p & ~(7u << 9)) | ((d - 1) << 9);
}

// RNG dimensions: vertex b, slot k.
enum : uint32_t { K_CAMERA = 0, K_BSDF = 1, K_RR = 2, K_LIGHT0 = 3 };
__device__ __forceinline__ uint32_t dim_of(uint32_t b, uint32_t k) { return (b << 12) | k; }

__device__ __forceinline__ Strata strata_for(uint32_t n) {
  // Grid::adjust_uv_sample_count (render/grid.cc:70-80)
  double sq = sqrt(double(n));
  uint32_t up = uint32_t(ceil(sq)), down = uint32_t(floor(sq + 0.5));
  if (down == 0) down = 1;
  return Strata{n, up, down, up * down};
}

// Warp-aggregated append: every lane of the warp calls it; lanes with PRED
// get consecutive slots from *COUNTER with one atomic per warp.
__device__ __forceinline__ uint32_t warp_append(uint32_t *counter, bool pred) {
  const uint32_t lane = threadIdx.x & 31u;
  unsigned mask = __ballot_sync(0xffffffffu, pred);
  if (!mask) return 0;
  uint32_t leader = __ffs(mask) - 1, base = 0;
  if (lane == leader) base = atomicAdd(counter, uint32_t(__popc(mask)));
  base = __shfl_sync(0xffffffffu, base, leader);
  return base + uint32_t(__popc(mask & ((1u << lane) - 1u)));
}

// Medium::transmittance (material/medium.h:37-40), pow (e, -absorb * d).
__device__ __forceinline__ float3 medium_transmittance(const DevMedium &m, float len) {
  if (m.absorb[0] == 0.f && m.absorb[1] == 0.f && m.absorb[2] == 0.f) return f3(1.f, 1.f, 1.f);
  return f3(expf(-m.absorb[0] * len), expf(-m.absorb[1] * len), expf(-m.absorb[2] * len));
}

}  // namespace snog

#endif
