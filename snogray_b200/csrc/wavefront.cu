// wavefront.cu -- the path integrator (render/path-integ.cc:134-407) as a
// wavefront on sm_100a.
//
// A job's render pattern (the image plus the Mitchell filter's 2-pixel
// margin, snogray.lua:543-550) times its samples per pixel is processed in
// waves of whole pixels.  Per wave:
//   k_camera                 eye rays for every path (camera/camera.cc:108-160)
//   per bounce b = 0..max_len:
//     k_trace_closest        octree closest hit for the live rays
//     k_shade                emission, BSDF continuation, Russian
//                            roulette; appends surviving rays to the other
//                            queue with warp-aggregated atomics and lists
//                            the vertices to light
//     k_direct               direct lighting with MIS of the listed
//                            vertices (emits shadow rays)
//     k_trace_shadow         any-hit for the shadow rays; unoccluded ones add
//                            their contribution to the path's radiance
//   k_splat                  Mitchell filter gather of the wave's samples
//                            into the image accumulator
// and finally k_resolve divides by the filter weight
// (image/image-sampled-output.cc:79-123).
//
// Path state is SoA of 16-byte records (float4 throughput+rr ratio, float4
// radiance+alpha) plus a 32-bit word: path length (8 bits), after-specular
// (1 bit), media-stack depth (2 bits) and up to three medium ids (7 bits
// each).  Queues hold rays as two float4 (origin+t0, direction+t1) in queue
// order, so the trace kernels read them with coalesced 128-bit loads.

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "launch.h"
#include "pathstate.cuh"
#include "scene.h"
#include "wavefront.h"

namespace snog {

namespace {

struct PathPtrs {
  float4 *thr, *rad;
  uint32_t *pstate;
  float2 *jit;
};
struct RayQ {
  float4 *o, *d;
  uint32_t *path;
};
struct ShadowQ {
  float4 *o, *d, *c;
};
struct DirectL {             // vertices to light, written by k_shade
  uint32_t *idx;             // queue index
  float4 *thr;               // throughput before the continuation, path state word in w
};

// ---- kernels -----------------------------------------------------------------

__global__ void __launch_bounds__(256) k_camera(JobConsts jc, uint64_t base, uint32_t n, PathPtrs P, RayQ q,
                                                uint32_t *counters) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    counters[0] = n;
    counters[1] = 0;
    counters[2] = 0;
    counters[4] = 0;          // closest kernel's dispenser
  }
  const Strata st = strata_for(jc.S);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
    const uint64_t g = base + p;
    const uint32_t pixel = uint32_t(g / jc.S), s = uint32_t(g % jc.S);
    const int px = jc.PX + int(pixel % jc.PW), py = jc.PY + int(pixel / jc.PW);
    Rng rng{jc.seed_lo, jc.seed_hi, uint32_t(g), uint32_t(g >> 32)};
    float2 j = strat_uv(st, rng, pixel, s, dim_of(0, K_CAMERA));
    // Renderer::render_packet (render-mgr/renderer.cc:69-88) and
    // Camera::eye_vec (camera/camera.h:384-389).
    float cu = float(px) + j.x, cv = float(py) + j.y;
    float fu = cu / float(jc.FW), fv = (float(jc.FH) - cv) / float(jc.FH);
    float x = 2.f * fu - 1.f, y = 2.f * fv - 1.f;
    float3 d = add(add(load3(jc.cam_fwd), mul(mul(load3(jc.cam_right), x), jc.tan_x)),
                   mul(mul(load3(jc.cam_up), y), jc.tan_y));
    q.o[p] = make_float4(jc.cam_pos[0], jc.cam_pos[1], jc.cam_pos[2], 0.f);
    q.d[p] = make_float4(d.x, d.y, d.z, jc.max_trace);
    q.path[p] = p;
    P.thr[p] = make_float4(1.f, 1.f, 1.f, 1.f);
    P.rad[p] = make_float4(0.f, 0.f, 0.f, 1.f);
    P.pstate[p] = 0;
    P.jit[p] = j;
  }
}

// Add a thread's node/test counts to P[0..1] with one atomic per warp; every
// lane of the block must call it.
__device__ __forceinline__ void warp_count(unsigned long long *p, unsigned long long nodes,
                                           unsigned long long tests) {
  for (int off = 16; off > 0; off >>= 1) {
    nodes += __shfl_down_sync(0xffffffffu, nodes, off);
    tests += __shfl_down_sync(0xffffffffu, tests, off);
  }
  if ((threadIdx.x & 31u) == 0) {
    atomicAdd(p, nodes);
    atomicAdd(p + 1, tests);
  }
}

// Persistent closest-hit kernel: warps take rays from the queue through a
// RayDispenser (counters[4]) and interleave one octree entry per ray per
// iteration, so finished lanes are refilled instead of idling.
template <int STACK, int PER>
__global__ void __launch_bounds__(kTraceBlock, SNOG_TRACE_MINBLOCKS) k_trace_closest(DevScene s, RayQ q, uint32_t *counters, uint32_t cur,
                                                       uint32_t *hit_ref, float *hit_t,
                                                       unsigned long long *stats, bool prof) {
  const uint32_t n = counters[cur];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    counters[cur ^ 1u] = 0;   // next queue and shadow queue start empty
    counters[2] = 0;
    counters[5] = 0;          // shadow kernel's dispenser
    counters[6] = 0;          // direct-lighting list
    stats[0] += n;
  }
  TraceCounters c{0, 0, 0};
  trace_loop<STACK, kClosestOnly, PER>(
      counters + 4, n, c,
      [&](uint32_t ray, Traversal<STACK> &tr, bool &any) {
        const float4 o = q.o[ray], d = q.d[ray];
        tr.init(s, xyz(o), xyz(d), o.w, d.w);
        any = false;
      },
      [&](uint32_t ray, Traversal<STACK> &tr, bool) {
        hit_ref[ray] = tr.hit_ref;
        hit_t[ray] = tr.t1;
      });
  if (c.overflow) atomicOr(counters + 3, 1u);
  if (prof) warp_count(stats + 2, c.nodes, c.tests);
}

// Persistent any-hit kernel for the shadow queue (dispenser counters[5]);
// an unoccluded ray adds its contribution to its path's radiance.
template <int STACK>
__global__ void __launch_bounds__(kTraceBlock, SNOG_TRACE_MINBLOCKS) k_trace_shadow(DevScene s, ShadowQ q, uint32_t *counters, float4 *rad,
                                                      unsigned long long *stats, bool prof) {
  const uint32_t n = counters[2];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    stats[1] += n;
    stats[6] += counters[6];   // vertices lit this bounce (DirectIllum::sample_all_lights calls)
  }
  TraceCounters c{0, 0, 0};
  trace_loop<STACK, kAnyOnly>(
      counters + 5, n, c,
      [&](uint32_t ray, Traversal<STACK> &tr, bool &any) {
        const float4 o = q.o[ray], d = q.d[ray];
        tr.init(s, xyz(o), xyz(d), o.w, d.w);
        any = true;
      },
      [&](uint32_t ray, Traversal<STACK> &tr, bool) {
        if (tr.hit_ref != PREF_END) return;
        const float4 cc = q.c[ray];
        float4 *r = rad + __float_as_uint(cc.w);
        atomicAdd(&r->x, cc.x);
        atomicAdd(&r->y, cc.y);
        atomicAdd(&r->z, cc.z);
      });
  if (c.overflow) atomicOr(counters + 3, 1u);
  if (prof) warp_count(stats + 4, c.nodes, c.tests);
}

// 6 blocks of 128 per SM (80 registers), as the engine's shading kernels.
__global__ void __launch_bounds__(128, 6) k_shade(DevScene s, JobConsts jc, uint64_t base, uint32_t bounce,
                                               RayQ qin, uint32_t *counters, uint32_t cur,
                                               const uint32_t *hit_ref, const float *hit_t, PathPtrs P,
                                               RayQ qout, DirectL dl) {
  const uint32_t n = counters[cur];
  if (blockIdx.x == 0 && threadIdx.x == 0) counters[4] = 0;   // next bounce's dispenser
  uint32_t *count_out = counters + (cur ^ 1u);
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const Strata st = strata_for(jc.S);
  const bool strat = bounce < jc.min_len;

  for (uint32_t wb = warp * 32; wb < n; wb += nwarps * 32) {
    const uint32_t i = wb + lane;
    const bool active = i < n;
    uint32_t path = 0, ps = 0, ref = PREF_END;
    float4 o4 = make_float4(0, 0, 0, 0), d4 = o4;
    float3 thr = f3(0, 0, 0), rad = f3(0, 0, 0);
    float rr_ratio = 1.f, alpha = 1.f;
    bool alive = false;       // path reaches direct lighting
    Isec I;
    BsdfCtx B{nullptr, 1.f, 1.f};
    DevMedium med{1.f, {0, 0, 0}};
    Rng rng{jc.seed_lo, jc.seed_hi, 0, 0};
    uint32_t pixel = 0, sidx = 0;
    if (active) {
      path = qin.path[i];
      o4 = qin.o[i];
      d4 = qin.d[i];
      ref = hit_ref[i];
      float t = hit_t[i];
      ps = P.pstate[path];
      float4 t4 = P.thr[path], r4 = P.rad[path];
      thr = xyz(t4);
      rr_ratio = t4.w;
      rad = xyz(r4);
      alpha = r4.w;
      const uint64_t g = base + path;
      pixel = uint32_t(g / jc.S);
      sidx = uint32_t(g % jc.S);
      rng.path_lo = uint32_t(g);
      rng.path_hi = uint32_t(g >> 32);
      const uint32_t depth = ps_depth(ps);
      const uint32_t mid = depth ? ps_medium(ps, depth - 1) : 0u;
      med = s.media[mid];
      const uint32_t len = ps_len(ps);
      // Volume integrator: attenuation over the ray (render/filter-volume-integ.h:55-68).
      const float t1 = ref == PREF_END ? d4.w : t;
      thr = mul3(thr, medium_transmittance(med, length(xyz(d4)) * (t1 - o4.w)));
      const bool include_emitters = len == 0 || ps_spec(ps) || jc.direct_samples == 0;
      if (ref == PREF_END) {
        if (include_emitters) rad = add(rad, mul3(background(s, xyz(d4)), thr));
        if (len == 0 && rad.x == 0.f && rad.y == 0.f && rad.z == 0.f) alpha = jc.bg_alpha;
      } else {
        I = make_isec(s, ref, xyz(o4), xyz(d4), t);
        const DevMaterial &M = s.mats[I.mat];
        // Glow::Le (material/glow.cc:37-40)
        if (include_emitters && M.type == MAT_GLOW && !I.back) rad = add(rad, mul3(load3(M.color), thr));
        const DevMaterial *bm = bsdf_material(s, I.mat);
        if (bm) {
          B.m = bm;
          B.medium_ior = med.ior;
          // Media::enclosing_medium (material/media.h:76-79)
          B.enclosing_ior = depth >= 2 ? s.media[ps_medium(ps, depth - 2)].ior : 1.f;
          alive = true;
        }
      }
    }

    // Vertices with lights to sample go to the direct-lighting list, with the
    // throughput and path state the continuation below replaces.
    const bool lit = alive && jc.direct_samples != 0u && s.n_lights != 0u;
    const uint32_t dslot = warp_append(counters + 6, lit);
    if (lit) {
      dl.idx[dslot] = i;
      dl.thr[dslot] = make_float4(thr.x, thr.y, thr.z, __uint_as_float(ps));
    }

    // ---- BSDF continuation, roulette, next ray (path-integ.cc:309-403) ----
    bool cont = false;
    float3 next_d = f3(0, 0, 0);
    if (alive) {
      const uint32_t len = ps_len(ps);
      float2 prm = strat ? strat_uv(st, rng, pixel, sidx, dim_of(bounce, K_BSDF)) : rng.uv(dim_of(bounce, K_BSDF));
      BSample bs = bsdf_sample(B, I, prm, B_ALL);
      if (bs.pdf != 0.f && !(bs.val.x == 0.f && bs.val.y == 0.f && bs.val.z == 0.f)) {
        thr = mul3(thr, mul(bs.val, fabsf(I.cos_n(bs.dir)) / bs.pdf));
        bool stop = false;
        if (len > jc.min_len) {
          float p = fminf(intensity(thr) * rr_ratio, 1.f);
          if (rng.u(dim_of(bounce, K_RR)) > p) {
            stop = true;
          } else {
            thr = mul(thr, 1.f / p);
            rr_ratio *= p;
          }
        }
        if (!stop && len != jc.max_len) {
          cont = true;
          next_d = I.nf.from(bs.dir);
          uint32_t nps = (ps & ~0x1ffu) | (len + 1) | ((bs.flags & B_SPECULAR) ? 0x100u : 0u);
          if (bs.flags & B_TRANSMISSIVE) {
            uint32_t mid = s.mats[I.mat].medium_id;
            if (mid && I.back) {
              nps = ps_pop(nps);
            } else if (mid && !ps_push(nps, mid)) {
              atomicOr(counters + 3, 2u);   // a fifth nested medium: the path ends here
              cont = false;
            }
          }
          if (cont) ps = nps;
        }
      }
    }
    uint32_t slot = warp_append(count_out, cont);
    if (cont) {
      // Intersect::recursive_ray (dir) (render/intersect.cc:196-202)
      qout.o[slot] = make_float4(I.pos.x, I.pos.y, I.pos.z, jc.min_trace);
      qout.d[slot] = make_float4(next_d.x, next_d.y, next_d.z, jc.horizon);
      qout.path[slot] = path;
    }
    if (active) {
      P.rad[path] = make_float4(rad.x, rad.y, rad.z, alpha);
      if (cont) {
        P.thr[path] = make_float4(thr.x, thr.y, thr.z, rr_ratio);
        P.pstate[path] = ps;
      }
    }
  }
}

// Direct lighting of the vertices k_shade listed (render/direct-illum.cc:83-255),
// one list entry per thread: the vertex is rebuilt from its queue entry (the
// same arithmetic as in k_shade, so the same bits) and every light sampled.
// Kept out of k_shade so neither body outgrows the instruction cache, and run
// over a compacted list so escaped and absorbed paths leave no idle lanes.
__global__ void __launch_bounds__(128, 6) k_direct(DevScene s, JobConsts jc, uint64_t base, uint32_t bounce,
                                                RayQ qin, uint32_t *counters, const uint32_t *hit_ref,
                                                const float *hit_t, DirectL dl, ShadowQ sq) {
  const uint32_t n = counters[6];
  uint32_t *count_sq = counters + 2;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const Strata st_direct = strata_for(jc.S * (jc.direct_samples ? jc.direct_samples : 1));
  const Strata st_rand = strata_for(jc.direct_samples ? jc.direct_samples : 1);
  const bool strat = bounce < jc.min_len;
  const float inv_ns = jc.direct_samples ? 1.f / float(jc.direct_samples) : 0.f;

  for (uint32_t wb = warp * 32; wb < n; wb += nwarps * 32) {
    const uint32_t k = wb + lane;
    const bool alive = k < n;
    uint32_t path = 0;
    float3 thr = f3(0, 0, 0);
    Isec I;
    BsdfCtx B{nullptr, 1.f, 1.f};
    DevMedium med{1.f, {0, 0, 0}};
    Rng rng{jc.seed_lo, jc.seed_hi, 0, 0};
    uint32_t pixel = 0, sidx = 0;
    if (alive) {
      const uint32_t i = dl.idx[k];
      const float4 t4 = dl.thr[k];
      thr = xyz(t4);
      const uint32_t ps = __float_as_uint(t4.w);
      path = qin.path[i];
      const float4 o4 = qin.o[i], d4 = qin.d[i];
      const uint64_t g = base + path;
      pixel = uint32_t(g / jc.S);
      sidx = uint32_t(g % jc.S);
      rng.path_lo = uint32_t(g);
      rng.path_hi = uint32_t(g >> 32);
      const uint32_t depth = ps_depth(ps);
      med = s.media[depth ? ps_medium(ps, depth - 1) : 0u];
      I = make_isec(s, hit_ref[i], xyz(o4), xyz(d4), hit_t[i]);
      B.m = bsdf_material(s, I.mat);
      B.medium_ior = med.ior;
      B.enclosing_ior = depth >= 2 ? s.media[ps_medium(ps, depth - 2)].ior : 1.f;
    }

    // ---- direct lighting (render/direct-illum.cc:83-255) ----------------
    // Every lane runs the same loop so that shadow-ray appends stay
    // warp-synchronous; lanes without a live vertex append nothing.
    if (jc.direct_samples) {
      const uint32_t flags = B_ALL & ~B_SPECULAR;
      for (uint32_t l = 0; l < s.n_lights; l++) {
        const DevLight &L = s.lights[l];
        const bool point = is_point_light(L);
        for (uint32_t jn = 0; jn < jc.direct_samples; jn++) {
          bool emit_l = false, emit_b = false;
          float3 c_l = f3(0, 0, 0), c_b = f3(0, 0, 0), dir_l = c_l, dir_b = c_l;
          float dist_l = 0.f, dist_b = 0.f;
          if (alive) {
            const uint32_t kl = K_LIGHT0 + 3 * l;
            float2 pl, pb;
            if (strat) {
              pl = strat_uv(st_direct, rng, pixel, sidx * jc.direct_samples + jn, dim_of(bounce, kl));
              pb = strat_uv(st_direct, rng, pixel, sidx * jc.direct_samples + jn, dim_of(bounce, kl + 1));
            } else {
              pl = strat_uv(st_rand, rng, uint32_t(rng.path_lo ^ (bounce << 24)), jn, dim_of(bounce, kl));
              pb = strat_uv(st_rand, rng, uint32_t(rng.path_lo ^ (bounce << 24)), jn, dim_of(bounce, kl + 1));
            }
            const float extra = rng.u(dim_of(bounce, kl + 2) ^ (jn << 20));
            LSample ls = light_sample(s, L, I, pl, extra);
            if (ls.pdf > 0.f && csum(ls.val) > 0.f) {
              float bpdf;
              float3 bv = bsdf_eval(B, I, ls.dir, flags, bpdf);
              if (csum(bv) > 0.f) {
                float3 c = ls.val;
                float slen = (ls.dist == 0.f ? jc.horizon : ls.dist) - 2.f * jc.min_trace;
                c = mul3(c, medium_transmittance(med, slen));
                if (!point) c = mul(c, mis_weight(ls.pdf, bpdf));
                c = mul3(c, bv);
                c = mul(c, fabsf(I.cos_n(ls.dir)) / ls.pdf);
                c_l = mul(mul3(c, thr), inv_ns);
                dir_l = ls.dir;
                dist_l = ls.dist;
                emit_l = true;
              }
            }
            if (!point) {
              BSample bs = bsdf_sample(B, I, pb, flags);
              if (bs.pdf > 0.f && csum(bs.val) > 0.f) {
                LSample lv = light_eval(s, L, I, bs.dir);
                if (lv.pdf > 0.f && csum(lv.val) > 0.f) {
                  float3 c = lv.val;
                  float slen = (lv.dist == 0.f ? jc.horizon : lv.dist) - 2.f * jc.min_trace;
                  c = mul3(c, medium_transmittance(med, slen));
                  c = mul(c, mis_weight(bs.pdf, lv.pdf));
                  c = mul3(c, bs.val);
                  c = mul(c, fabsf(I.cos_n(bs.dir)) / bs.pdf);
                  c_b = mul(mul3(c, thr), inv_ns);
                  dir_b = bs.dir;
                  dist_b = lv.dist;
                  emit_b = true;
                }
              }
            }
          }
          // Intersect::recursive_ray (dir, max_dist) (render/intersect.cc:211-218)
          uint32_t slot = warp_append(count_sq, emit_l);
          if (emit_l) {
            float3 wd = I.nf.from(dir_l);
            float t1 = (dist_l == 0.f ? jc.horizon : dist_l) - jc.min_trace;
            sq.o[slot] = make_float4(I.pos.x, I.pos.y, I.pos.z, jc.min_trace);
            sq.d[slot] = make_float4(wd.x, wd.y, wd.z, t1);
            sq.c[slot] = make_float4(c_l.x, c_l.y, c_l.z, __uint_as_float(path));
          }
          slot = warp_append(count_sq, emit_b);
          if (emit_b) {
            float3 wd = I.nf.from(dir_b);
            float t1 = (dist_b == 0.f ? jc.horizon : dist_b) - jc.min_trace;
            sq.o[slot] = make_float4(I.pos.x, I.pos.y, I.pos.z, jc.min_trace);
            sq.d[slot] = make_float4(wd.x, wd.y, wd.z, t1);
            sq.c[slot] = make_float4(c_b.x, c_b.y, c_b.z, __uint_as_float(path));
          }
        }
      }
    }

  }
}

// ImageMitchellFilt::mitchell1 with B = C = 1/3, radius 2
// (image/image-mitchell-filt.h:50-65).
__device__ __forceinline__ float mitchell1(float x) {
  const float b = 1.f / 3.f, c = 1.f / 3.f;
  x = fabsf(x);
  if (x > 2.f) return 0.f;
  if (x > 1.f)
    return ((-b - 6 * c) * x * x * x + (6 * b + 30 * c) * x * x + (-12 * b - 48 * c) * x + (8 * b + 24 * c)) *
           (1.f / 6.f);
  return ((12 - 9 * b - 6 * c) * x * x * x + (-18 + 12 * b + 6 * c) * x * x + (6 - 2 * b)) * (1.f / 6.f);
}

// Gather the wave's samples into the target pixels they reach
// (ImageFilterConv::add_sample, image/image-filter-conv.h:109-186): every
// sample within the filter's support of a target pixel centre adds
// Tint * w and w, with the negative-lobe clamp (neg_clamp = -0.1).
// G lanes (a power of two up to 32) per target pixel: they take every G-th
// sample of each neighbouring pattern pixel -- consecutive samples, so the
// group's loads coalesce -- and sum their shares with shuffles.  With one
// thread per pixel a small image at high spp left most of the GPU idle on
// long chains of loads.
template <int G>
__global__ void __launch_bounds__(256) k_splat(JobConsts jc, uint64_t base, uint32_t n, const float4 *rad,
                                               const float2 *jit, float4 *accum, float *wsum, int ty0,
                                               int nrows) {
  const uint32_t p0 = uint32_t(base / jc.S), p1 = uint32_t((base + n) / jc.S);
  const uint32_t total = uint32_t(nrows) * jc.W;
  const float neg_clamp = -0.1f;
  const uint32_t sub = threadIdx.x & uint32_t(G - 1);
  const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31u) & ~uint32_t(G - 1)));
  const uint32_t groups = (gridDim.x * blockDim.x) / G;
  // Every lane of a group has the same T, so a group runs its loop together.
  for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) / G; t < total; t += groups) {
    const int tx = int(t % jc.W), ty = ty0 + int(t / jc.W);
    // The target pixel on the film; the samples of the pattern pixels within
    // the filter's reach add to it.
    const int fx = jc.OX + tx, fy = jc.OY + ty;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    float wacc = 0.f;
    for (int dy = -2; dy <= 2; dy++) {
      const int row = fy + dy - jc.PY;
      if (row < 0 || row >= int(jc.PH)) continue;
      for (int dx = -2; dx <= 2; dx++) {
        const int col = fx + dx - jc.PX;
        if (col < 0 || col >= int(jc.PW)) continue;
        const uint32_t pidx = uint32_t(row) * jc.PW + uint32_t(col);
        if (pidx < p0 || pidx >= p1) continue;
        const uint32_t pbase = (pidx - p0) * jc.S;
        for (uint32_t k = sub; k < jc.S; k += G) {
          float2 j = jit[pbase + k];
          float sx = float(fx + dx) + j.x, sy = float(fy + dy) + j.y;
          float w = mitchell1(sx - (float(fx) + 0.5f)) * mitchell1(sy - (float(fy) + 0.5f));
          if (w == 0.f) continue;
          float4 r = rad[pbase + k];
          // Tint (radiance, alpha) stores alpha-scaled colour (color/tint.h:45-49)
          float cr = r.x * r.w * w, cg = r.y * r.w * w, cb = r.z * r.w * w, ca = r.w * w;
          if (w < 0.f) {
            float mc = fminf(cr, fminf(cg, cb));
            if (mc < neg_clamp) {
              float sc = neg_clamp / mc;
              w *= sc;
              cr *= sc; cg *= sc; cb *= sc; ca *= sc;
            }
          }
          acc.x += cr; acc.y += cg; acc.z += cb; acc.w += ca;
          wacc += w;
        }
      }
    }
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) {
      acc.x += __shfl_xor_sync(gmask, acc.x, off);
      acc.y += __shfl_xor_sync(gmask, acc.y, off);
      acc.z += __shfl_xor_sync(gmask, acc.z, off);
      acc.w += __shfl_xor_sync(gmask, acc.w, off);
      wacc += __shfl_xor_sync(gmask, wacc, off);
    }
    if (sub == 0) {
      const size_t o = size_t(ty) * jc.W + size_t(tx);
      float4 a = accum[o];
      accum[o] = make_float4(a.x + acc.x, a.y + acc.y, a.z + acc.z, a.w + acc.w);
      wsum[o] += wacc;
    }
  }
}

// The splat with the lane group that fits S samples per pixel.
void launch_splat(const JobConsts &jc, uint64_t base, uint32_t n, const float4 *rad, const float2 *jit,
                  float4 *accum, float *wsum, int ty0, int nrows, uint32_t grid256, cudaStream_t st) {
  if (jc.S >= 32) k_splat<32><<<grid256, 256, 0, st>>>(jc, base, n, rad, jit, accum, wsum, ty0, nrows);
  else if (jc.S > 8) k_splat<16><<<grid256, 256, 0, st>>>(jc, base, n, rad, jit, accum, wsum, ty0, nrows);
  else if (jc.S > 4) k_splat<8><<<grid256, 256, 0, st>>>(jc, base, n, rad, jit, accum, wsum, ty0, nrows);
  else if (jc.S > 2) k_splat<4><<<grid256, 256, 0, st>>>(jc, base, n, rad, jit, accum, wsum, ty0, nrows);
  else if (jc.S > 1) k_splat<2><<<grid256, 256, 0, st>>>(jc, base, n, rad, jit, accum, wsum, ty0, nrows);
  else k_splat<1><<<grid256, 256, 0, st>>>(jc, base, n, rad, jit, accum, wsum, ty0, nrows);
}

// ImageSampledOutput::set_raw_min_y row flush (image/image-sampled-output.cc:79-123).
__global__ void __launch_bounds__(256) k_resolve(uint32_t npix, const float4 *accum, const float *wsum, float *out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
    float4 a = accum[i];
    float w = wsum[i];
    float r = a.x, g = a.y, b = a.z, al = a.w;
    if (w > 0.f && w != 1.f) {
      float iw = 1.f / w;
      r *= iw; g *= iw; b *= iw; al *= iw;
    }
    al = fminf(fmaxf(al, 0.f), 1.f);
    r = fmaxf(r, 0.f); g = fmaxf(g, 0.f); b = fmaxf(b, 0.f);
    if (al != 0.f && al != 1.f) {
      float ia = 1.f / al;
      r *= ia; g *= ia; b *= ia;
    }
    out[3 * size_t(i)] = r;
    out[3 * size_t(i) + 1] = g;
    out[3 * size_t(i) + 2] = b;
  }
}

template <int STACK>
void launch_bounce(const DevScene &s, const JobConsts &jc, WaveBuffers &wb, uint64_t base, uint32_t b,
                   uint32_t cur, uint32_t grid128, cudaStream_t st, RenderProfile *prof, bool count) {
  RayQ qin{wb.q_o[cur], wb.q_d[cur], wb.q_path[cur]};
  RayQ qout{wb.q_o[cur ^ 1], wb.q_d[cur ^ 1], wb.q_path[cur ^ 1]};
  ShadowQ sq{wb.s_o, wb.s_d, wb.s_c};
  DirectL dl{wb.d_idx, wb.d_thr};
  PathPtrs P{wb.thr, wb.rad, wb.pstate, wb.jit};
  const bool pf = prof != nullptr || count;
  if (prof) prof->begin(st, RenderProfile::CLOSEST);
  if (s.pair_lists)
    k_trace_closest<STACK, 2><<<resident_grid(k_trace_closest<STACK, 2>, kTraceBlock), kTraceBlock, 0, st>>>(
        s, qin, wb.counters, cur, wb.hit_ref, wb.hit_t, wb.stats, pf);
  else
    k_trace_closest<STACK, 1><<<resident_grid(k_trace_closest<STACK, 1>, kTraceBlock), kTraceBlock, 0, st>>>(
        s, qin, wb.counters, cur, wb.hit_ref, wb.hit_t, wb.stats, pf);
  if (prof) prof->end(st), prof->begin(st, RenderProfile::SHADE);
  k_shade<<<grid128, 128, 0, st>>>(s, jc, base, b, qin, wb.counters, cur, wb.hit_ref, wb.hit_t, P, qout, dl);
  k_direct<<<grid128, 128, 0, st>>>(s, jc, base, b, qin, wb.counters, wb.hit_ref, wb.hit_t, dl, sq);
  if (prof) prof->end(st), prof->begin(st, RenderProfile::SHADOW);
  k_trace_shadow<STACK><<<resident_grid(k_trace_shadow<STACK>, kTraceBlock), kTraceBlock, 0, st>>>(s, sq, wb.counters, wb.rad, wb.stats, pf);
  if (prof) prof->end(st);
}

}  // namespace

cudaError_t RenderProfile::begin(cudaStream_t st, int kind) {
  if (n == cap) {
    uint32_t nc = cap ? 2 * cap : 256;
    Mark *m = new Mark[nc];
    for (uint32_t i = 0; i < n; i++) m[i] = marks[i];
    delete[] marks;
    marks = m;
    cap = nc;
  }
  Mark &mk = marks[n];
  mk.kind = kind;
  cudaError_t e = cudaEventCreate(&mk.a);
  if (e == cudaSuccess) e = cudaEventCreate(&mk.b);
  if (e == cudaSuccess) e = cudaEventRecord(mk.a, st);
  return e;
}

cudaError_t RenderProfile::end(cudaStream_t st) {
  cudaError_t e = cudaEventRecord(marks[n].b, st);
  n++;
  return e;
}

cudaError_t RenderProfile::collect() {
  cudaError_t err = cudaSuccess;
  for (uint32_t i = 0; i < n; i++) {
    float ms = 0.f;
    cudaError_t e = cudaEventElapsedTime(&ms, marks[i].a, marks[i].b);
    if (e != cudaSuccess) err = e;
    this->ms[marks[i].kind] += ms;
    launches[marks[i].kind]++;
    cudaEventDestroy(marks[i].a);
    cudaEventDestroy(marks[i].b);
  }
  n = 0;
  return err;
}

RenderProfile::~RenderProfile() {
  for (uint32_t i = 0; i < n; i++) {
    cudaEventDestroy(marks[i].a);
    cudaEventDestroy(marks[i].b);
  }
  delete[] marks;
}

uint64_t wave_bytes_per_path(uint32_t n_lights) {
  // thr 16 + rad 16 + pstate 4 + 2 queues x 36 + hit 8 + jitter 8
  // + direct-lighting list 20 + shadow queue 48 per entry, 2 entries per light sample
  return 16 + 16 + 4 + 72 + 8 + 8 + 20 + 48ull * 2 * (n_lights ? n_lights : 1);
}

cudaError_t wave_alloc(WaveBuffers &wb, uint64_t cap, uint32_t n_lights) {
  wave_free(wb);
  const uint64_t nl = n_lights ? n_lights : 1;
  size_t bytes = 0;
  auto take = [&](size_t b) {
    size_t off = bytes;
    bytes += (b + 255) & ~size_t(255);
    return off;
  };
  size_t o_thr = take(16 * cap), o_rad = take(16 * cap), o_ps = take(4 * cap);
  size_t o_qo0 = take(16 * cap), o_qd0 = take(16 * cap), o_qp0 = take(4 * cap);
  size_t o_qo1 = take(16 * cap), o_qd1 = take(16 * cap), o_qp1 = take(4 * cap);
  size_t o_href = take(4 * cap), o_ht = take(4 * cap), o_jit = take(8 * cap);
  size_t o_didx = take(4 * cap), o_dthr = take(16 * cap);
  size_t o_so = take(16 * cap * 2 * nl), o_sd = take(16 * cap * 2 * nl), o_sc = take(16 * cap * 2 * nl);
  size_t o_cnt = take(64), o_stats = take(64);
  char *base = nullptr;
  cudaError_t e = cudaMalloc(&base, bytes);
  if (e != cudaSuccess) return e;
  wb.block = base;
  wb.bytes = bytes;
  wb.wave_cap = cap;
  wb.n_lights = n_lights;
  wb.thr = reinterpret_cast<float4 *>(base + o_thr);
  wb.rad = reinterpret_cast<float4 *>(base + o_rad);
  wb.pstate = reinterpret_cast<uint32_t *>(base + o_ps);
  wb.q_o[0] = reinterpret_cast<float4 *>(base + o_qo0);
  wb.q_d[0] = reinterpret_cast<float4 *>(base + o_qd0);
  wb.q_path[0] = reinterpret_cast<uint32_t *>(base + o_qp0);
  wb.q_o[1] = reinterpret_cast<float4 *>(base + o_qo1);
  wb.q_d[1] = reinterpret_cast<float4 *>(base + o_qd1);
  wb.q_path[1] = reinterpret_cast<uint32_t *>(base + o_qp1);
  wb.hit_ref = reinterpret_cast<uint32_t *>(base + o_href);
  wb.hit_t = reinterpret_cast<float *>(base + o_ht);
  wb.jit = reinterpret_cast<float2 *>(base + o_jit);
  wb.d_idx = reinterpret_cast<uint32_t *>(base + o_didx);
  wb.d_thr = reinterpret_cast<float4 *>(base + o_dthr);
  wb.s_o = reinterpret_cast<float4 *>(base + o_so);
  wb.s_d = reinterpret_cast<float4 *>(base + o_sd);
  wb.s_c = reinterpret_cast<float4 *>(base + o_sc);
  wb.counters = reinterpret_cast<uint32_t *>(base + o_cnt);
  wb.stats = reinterpret_cast<unsigned long long *>(base + o_stats);
  return cudaSuccess;
}

void wave_free(WaveBuffers &wb) {
  if (wb.block) cudaFree(wb.block);
  wb = WaveBuffers{};
}

void check_window(const SnogRenderParams &p, const SnogRenderWindow &w) {
  if (w.pat_width == 0 || w.pat_height == 0 || w.out_width == 0 || w.out_height == 0)
    throw Error{SNOG_EINVAL, "render window: empty pattern or output"};
  if (w.out_width > 65536 || w.out_height > 65536 || w.pat_width > 65540 || w.pat_height > 65540)
    throw Error{SNOG_EINVAL, "render window too large"};
  const int64_t lim = int64_t(1) << 20;
  if (w.pat_x < -lim || w.pat_x > lim || w.pat_y < -lim || w.pat_y > lim || w.out_x < -lim || w.out_x > lim ||
      w.out_y < -lim || w.out_y > lim)
    throw Error{SNOG_EINVAL, "render window offsets out of range"};
  if (uint64_t(w.pat_width) * w.pat_height >= (1ull << 32)) throw Error{SNOG_EINVAL, "render pattern too large"};
  if (uint64_t(w.pat_width) * w.pat_height * p.spp >= (1ull << 40))
    throw Error{SNOG_EINVAL, "too many paths in one job"};
}

JobConsts make_job(const DevScene &s, const SnogCamera &cam, const SnogRenderParams &p,
                   const SnogRenderWindow *win) {
  JobConsts jc;
  std::memset(&jc, 0, sizeof jc);
  jc.FW = p.width;
  jc.FH = p.height;
  if (win) {
    jc.W = win->out_width;
    jc.H = win->out_height;
    jc.OX = win->out_x;
    jc.OY = win->out_y;
    jc.PW = win->pat_width;
    jc.PH = win->pat_height;
    jc.PX = win->pat_x;
    jc.PY = win->pat_y;
  } else {
    jc.W = p.width;
    jc.H = p.height;
    jc.OX = jc.OY = 0;
    jc.PW = p.width + 4;
    jc.PH = p.height + 4;
    jc.PX = jc.PY = -2;
  }
  jc.S = p.spp;
  jc.min_len = p.min_path_len;
  jc.max_len = p.max_path_len;
  jc.direct_samples = p.direct_samples;
  jc.min_trace = p.min_trace;
  jc.bg_alpha = p.bg_alpha;
  jc.horizon = s.horizon;
  // (scene.bbox () + camera.pos).diameter () (render-mgr/renderer.cc:54)
  float lo[3], hi[3];
  for (int k = 0; k < 3; k++) {
    lo[k] = s.bbox_min[k] < cam.pos[k] ? s.bbox_min[k] : cam.pos[k];
    hi[k] = s.bbox_max[k] > cam.pos[k] ? s.bbox_max[k] : cam.pos[k];
  }
  float ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
  jc.max_trace = std::sqrt(ex * ex + ey * ey + ez * ez);
  for (int k = 0; k < 3; k++) {
    jc.cam_pos[k] = cam.pos[k];
    jc.cam_fwd[k] = cam.forward[k];
    jc.cam_right[k] = cam.right[k];
    jc.cam_up[k] = cam.up[k];
  }
  jc.tan_x = cam.tan_half_fov_x;
  jc.tan_y = cam.tan_half_fov_y;
  jc.seed_lo = uint32_t(p.seed) * 2654435761u + 0x1234567u;
  jc.seed_hi = uint32_t(p.seed >> 32) ^ 0x9e3779b9u;
  jc.integ = p.integrator;
  return jc;
}

cudaError_t render_job(const DevScene &s, const JobConsts &jc, WaveBuffers &wb, float4 *accum, float *wsum,
                       float *out_rgb, cudaStream_t st, uint32_t *waves, uint32_t *launches,
                       RenderProfile *prof, bool count) {
  const uint64_t npix = uint64_t(jc.W) * jc.H;
  cudaError_t e = cudaMemsetAsync(accum, 0, npix * sizeof(float4), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(wsum, 0, npix * sizeof(float), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(wb.stats, 0, 64, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(wb.counters, 0, 64, st);
  if (e != cudaSuccess) return e;
  const int sms = num_sms();
  const uint32_t grid128 = uint32_t(sms) * 12, grid256 = uint32_t(sms) * 8;
  const uint64_t total = job_total(jc);
  const uint64_t wave_paths = (wb.wave_cap / jc.S) * jc.S;
  if (wave_paths == 0) return cudaErrorInvalidValue;
  const int sc = stack_class_for_depth(s.max_depth);
  uint32_t nl = 0;
  for (uint64_t base = 0; base < total; base += wave_paths) {
    const uint32_t n = uint32_t(total - base < wave_paths ? total - base : wave_paths);
    PathPtrs P{wb.thr, wb.rad, wb.pstate, wb.jit};
    RayQ q0{wb.q_o[0], wb.q_d[0], wb.q_path[0]};
    if (prof) prof->begin(st, RenderProfile::OTHER);
    k_camera<<<grid256, 256, 0, st>>>(jc, base, n, P, q0, wb.counters);
    if (prof) prof->end(st);
    nl++;
    for (uint32_t b = 0; b <= jc.max_len; b++) {
      const uint32_t cur = b & 1u;
      switch (sc) {
        case 32: launch_bounce<32>(s, jc, wb, base, b, cur, grid128, st, prof, count); break;
        case 64: launch_bounce<64>(s, jc, wb, base, b, cur, grid128, st, prof, count); break;
        case 128: launch_bounce<128>(s, jc, wb, base, b, cur, grid128, st, prof, count); break;
        case 256: launch_bounce<256>(s, jc, wb, base, b, cur, grid128, st, prof, count); break;
        default: return cudaErrorInvalidValue;
      }
      nl += 4;
    }
    // Output rows reached by this wave's pattern rows (a sample reaches
    // the film rows within 2 of its own).
    const uint32_t p0 = uint32_t(base / jc.S), p1 = uint32_t((base + n) / jc.S);
    const int r0 = int(p0 / jc.PW), r1 = int((p1 - 1) / jc.PW);
    const int a0 = jc.PY + r0 - jc.OY - 2, a1 = jc.PY + r1 - jc.OY + 2;
    const int ty0 = a0 < 0 ? 0 : a0, ty1 = a1 > int(jc.H) - 1 ? int(jc.H) - 1 : a1;
    if (ty1 >= ty0) {
      if (prof) prof->begin(st, RenderProfile::OTHER);
      launch_splat(jc, base, n, wb.rad, P.jit, accum, wsum, ty0, ty1 - ty0 + 1, grid256, st);
      if (prof) prof->end(st);
      nl++;
    }
    if (waves) (*waves)++;
  }
  if (prof) prof->begin(st, RenderProfile::OTHER);
  k_resolve<<<grid256, 256, 0, st>>>(uint32_t(npix), accum, wsum, out_rgb);
  if (prof) prof->end(st);
  nl++;
  if (launches) *launches += nl;
  return cudaGetLastError();
}

}  // namespace snog

namespace snog {

cudaError_t splat_job(const JobConsts &jc, const float4 *rad, const float2 *jit, uint64_t total, float4 *accum,
                      float *wsum, float *out_rgb, cudaStream_t st) {
  const uint64_t npix = uint64_t(jc.W) * jc.H;
  cudaError_t e = cudaMemsetAsync(accum, 0, npix * sizeof(float4), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(wsum, 0, npix * sizeof(float), st);
  if (e != cudaSuccess) return e;
  const uint32_t grid256 = uint32_t(num_sms()) * 8;
  launch_splat(jc, 0, uint32_t(total), rad, jit, accum, wsum, 0, int(jc.H), grid256, st);
  k_resolve<<<grid256, 256, 0, st>>>(uint32_t(npix), accum, wsum, out_rgb);
  return cudaGetLastError();
}

}  // namespace snog
