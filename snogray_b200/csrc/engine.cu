// engine.cu -- kernels and host loop of the streaming render engine
// (engine.h).  The per-vertex shading is the same as the wave renderer's
// (wavefront.cu) -- PathInteg::Li, render/path-integ.cc:134-407 -- with the
// path's job, scene and bounce carried in its queue entry, so one launch
// serves many jobs at different depths.  Random streams are keyed by (job
// seed, path index in the job, dimension) exactly as in the wave renderer, so
// a job renders the same image (up to float summation order) either way.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "engine.h"
#include "launch.h"
#include "pathstate.cuh"

namespace snog {

namespace {

// Rays of the direct integrator go no deeper than the path state's 8-bit
// length field; roulette beyond depth 5 makes that depth unreachable in
// practice (survival 2^-249).
constexpr uint32_t kMaxBounce = 255;

struct EQ {                 // one ray queue, SoA of 16-byte records
  float4 *o, *d, *thr, *rad;
  uint4 *meta;              // x = path state, y = job, z/w = path index lo/hi
};

struct ESQ {                // shadow queue
  float4 *o, *d, *c;        // c.w = scene index
  unsigned long long *tgt;  // address of the float4 radiance to add to
};

struct EDL {                // vertices to light, written by shade, read by direct
  uint32_t *idx;            // index in the shaded queue
  unsigned long long *tgt;  // address of the float4 radiance their light adds to
};

__global__ void k_e_plan(EngineCtl *ctl, const WorkItem *ring, uint32_t R, uint32_t N, uint32_t cur,
                         uint32_t sp_cap) {
  const uint32_t n_cur = ctl->qcount[cur];
  // Publish the branches the last shade spawned; the oldest waiting ones
  // take free queue slots before new camera paths.
  ctl->spawn_tail += ctl->spawn_n < ctl->spawn_room ? ctl->spawn_n : ctl->spawn_room;
  const unsigned long long waiting = ctl->spawn_tail - ctl->spawn_head;
  const uint32_t take = uint32_t(waiting < N - n_cur ? waiting : N - n_cur);
  ctl->regen_spawn = take;
  ctl->regen_spawn_head = ctl->spawn_head;
  ctl->spawn_head += take;
  ctl->spawn_n = 0;
  ctl->spawn_room = sp_cap - uint32_t(ctl->spawn_tail - ctl->spawn_head);
  const unsigned long long avail = ctl->avail_end - ctl->ticket;
  unsigned long long n_new = N - n_cur - take;
  if (n_new > avail) n_new = avail;
  // Retire items fully consumed before this iteration's tickets.
  unsigned long long head = ctl->item_head;
  while (head < ctl->item_tail) {
    const WorkItem &w = ring[head % R];
    if (w.cum + w.count > ctl->ticket) break;
    head++;
  }
  ctl->item_head = head;
  ctl->regen_start = ctl->ticket;
  ctl->regen_n = uint32_t(n_new);
  ctl->regen_base = n_cur;
  ctl->ticket += n_new;
  ctl->paths_started += n_new;
  ctl->qcount[cur] = n_cur + take + uint32_t(n_new);
  ctl->qcount[cur ^ 1u] = 0;
  ctl->scount = 0;
  ctl->dcount = 0;
  ctl->disp_closest = 0;
  ctl->disp_shadow = 0;
}

// New camera paths for tickets [regen_start, regen_start + regen_n).
__global__ void __launch_bounds__(256) k_e_regen(EngineCtl *ctl, const WorkItem *ring, uint32_t R,
                                                 const EngineJobDev *jobs, EQ q, EQ sp, uint32_t sp_cap) {
  const uint32_t n = ctl->regen_n, take = ctl->regen_spawn;
  const unsigned long long t0 = ctl->regen_start, head = ctl->item_head, tail = ctl->item_tail;
  const unsigned long long sp_head = ctl->regen_spawn_head;
  // Spawned branches first, into [base, base + take).
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < take; t += gridDim.x * blockDim.x) {
    const uint32_t from = uint32_t((sp_head + t) % sp_cap), slot = ctl->regen_base + t;
    q.o[slot] = sp.o[from];
    q.d[slot] = sp.d[from];
    q.thr[slot] = sp.thr[from];
    q.rad[slot] = sp.rad[from];
    q.meta[slot] = sp.meta[from];
  }
  const uint32_t base = ctl->regen_base + take;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const unsigned long long ticket = t0 + t;
    // Item holding this ticket: binary search over the ring window.
    unsigned long long lo = head, hi = tail;   // invariant: answer in [lo, hi)
    while (hi - lo > 1) {
      const unsigned long long mid = lo + (hi - lo) / 2;
      if (ring[mid % R].cum <= ticket) lo = mid;
      else hi = mid;
    }
    const WorkItem w = ring[lo % R];
    const uint32_t job = w.job;
    const unsigned long long g = w.begin + (ticket - w.cum);
    const EngineJobDev &J = jobs[job];
    const JobConsts &jc = J.jc;
    const uint32_t pixel = uint32_t(g / jc.S), s = uint32_t(g % jc.S);
    const int px = jc.PX + int(pixel % jc.PW), py = jc.PY + int(pixel / jc.PW);
    Rng rng{jc.seed_lo, jc.seed_hi, uint32_t(g), uint32_t(g >> 32)};
    const float2 j = strat_uv(strata_for(jc.S), rng, pixel, s, dim_of(0, K_CAMERA));
    // Renderer::render_packet (render-mgr/renderer.cc:69-88), Camera::eye_vec (camera/camera.h:384-389)
    const float cu = float(px) + j.x, cv = float(py) + j.y;
    const float fu = cu / float(jc.FW), fv = (float(jc.FH) - cv) / float(jc.FH);
    const float x = 2.f * fu - 1.f, y = 2.f * fv - 1.f;
    const float3 d = add(add(load3(jc.cam_fwd), mul(mul(load3(jc.cam_right), x), jc.tan_x)),
                         mul(mul(load3(jc.cam_up), y), jc.tan_y));
    const uint32_t slot = base + t;
    q.o[slot] = make_float4(jc.cam_pos[0], jc.cam_pos[1], jc.cam_pos[2], 0.f);
    // A cancelled job's new paths get an empty ray interval (nothing to trace).
    q.d[slot] = make_float4(d.x, d.y, d.z, J.canceled ? 0.f : jc.max_trace);
    q.thr[slot] = make_float4(1.f, 1.f, 1.f, 1.f);
    q.rad[slot] = make_float4(0.f, 0.f, 0.f, 1.f);
    q.meta[slot] = make_uint4(0u, job, uint32_t(g), uint32_t(g >> 32));
    J.jit[g] = j;
  }
}

template <int STACK, int PER>
__global__ void __launch_bounds__(kTraceBlock, SNOG_TRACE_MINBLOCKS) k_e_closest(EngineCtl *ctl, uint32_t cur, const EngineJobDev *jobs,
                                                      const DevScene *scenes, EQ q, uint32_t *hit_ref,
                                                      float *hit_t) {
  const uint32_t n = ctl->qcount[cur];
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->rays_closest += n;
  TraceCounters c{0, 0, 0};
  trace_loop<STACK, kClosestOnly, PER>(
      &ctl->disp_closest, n, c,
      [&](uint32_t ray, Traversal<STACK> &tr, bool &any) {
        const float4 o = q.o[ray], d = q.d[ray];
        tr.init(scenes[jobs[q.meta[ray].y].scene], xyz(o), xyz(d), o.w, d.w);
        any = false;
      },
      [&](uint32_t ray, Traversal<STACK> &tr, bool) {
        hit_ref[ray] = tr.hit_ref;
        hit_t[ray] = tr.t1;
      });
  if (c.overflow) atomicOr(&ctl->err, 1u);
}

template <int STACK>
__global__ void __launch_bounds__(kTraceBlock, SNOG_TRACE_MINBLOCKS) k_e_shadow(EngineCtl *ctl, const DevScene *scenes, ESQ q) {
  const uint32_t n = ctl->scount;
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->rays_shadow += n;
  TraceCounters c{0, 0, 0};
  trace_loop<STACK, kAnyOnly>(
      &ctl->disp_shadow, n, c,
      [&](uint32_t ray, Traversal<STACK> &tr, bool &any) {
        const float4 o = q.o[ray], d = q.d[ray];
        tr.init(scenes[__float_as_uint(q.c[ray].w)], xyz(o), xyz(d), o.w, d.w);
        any = true;
      },
      [&](uint32_t ray, Traversal<STACK> &tr, bool) {
        if (tr.hit_ref != PREF_END) return;
        const float4 cc = q.c[ray];
        float *dst = reinterpret_cast<float *>(q.tgt[ray]);
        atomicAdd(dst, cc.x);
        atomicAdd(dst + 1, cc.y);
        atomicAdd(dst + 2, cc.z);
      });
  if (c.overflow) atomicOr(&ctl->err, 1u);
}

// Shading, first half: emission, the continuation sample and roulette; the
// vertices to light go to a list for k_e_direct.  6 blocks of 128 per SM (80
// registers) for both halves: the bodies are long and divergent, and more
// resident warps hide their instruction-fetch stalls (4 or 5 blocks for
// k_e_direct, 8 for k_e_shade measured 0.6-2 % slower on the terrain frame).
// DIRECT: the direct integrator's code is compiled in (launched while a job
// of that integrator is active; the path integrator's kernel stays smaller).
#ifndef SNOG_SHADE_MINBLOCKS
#define SNOG_SHADE_MINBLOCKS 6
#endif
#ifndef SNOG_DIRECT_MINBLOCKS
#define SNOG_DIRECT_MINBLOCKS 6
#endif
template <bool DIRECT>
__global__ void __launch_bounds__(128, SNOG_SHADE_MINBLOCKS) k_e_shade(EngineCtl *ctl, uint32_t cur, const EngineJobDev *jobs,
                                                 const DevScene *scenes, EQ qin, const uint32_t *hit_ref,
                                                 const float *hit_t, EQ qout, EDL dl,
                                                 unsigned long long *job_done, unsigned long long *job_spawned,
                                                 EQ sp, uint32_t sp_cap) {
  const uint32_t n = ctl->qcount[cur];
  uint32_t *count_out = &ctl->qcount[cur ^ 1u];
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;

  for (uint32_t wb = warp * 32; wb < n; wb += nwarps * 32) {
    const uint32_t i = wb + lane;
    const bool active = i < n;
    uint32_t ps = 0, ref = PREF_END, job = 0, scene = 0, bounce = 0;
    unsigned long long g = 0;
    float4 o4 = make_float4(0, 0, 0, 0), d4 = o4;
    float3 thr = f3(0, 0, 0), rad = f3(0, 0, 0);
    float rr_ratio = 1.f, alpha = 1.f;
    bool alive = false;
    Isec I;
    BsdfCtx B{nullptr, 1.f, 1.f};
    DevMedium med{1.f, {0, 0, 0}};
    const EngineJobDev *J = jobs;
    const DevScene *s = scenes;
    Rng rng{0, 0, 0, 0};
    uint32_t pixel = 0, sidx = 0;
    if (active) {
      const uint4 meta = qin.meta[i];
      ps = meta.x;
      job = meta.y;
      g = (unsigned long long)meta.z | ((unsigned long long)meta.w << 32);
      J = jobs + job;
      scene = J->scene;
      s = scenes + scene;
    }
    const bool retire = active && J->canceled;   // cancelled job: the path ends here, unshaded
    if (active && !retire) {
      o4 = qin.o[i];
      d4 = qin.d[i];
      ref = hit_ref[i];
      const float t = hit_t[i];
      const float4 t4 = qin.thr[i], r4 = qin.rad[i];
      thr = xyz(t4);
      rr_ratio = t4.w;
      rad = xyz(r4);
      alpha = r4.w;
      const JobConsts &jc = J->jc;
      rng = Rng{jc.seed_lo, jc.seed_hi, uint32_t(g), uint32_t(g >> 32)};
      pixel = uint32_t(g / jc.S);
      sidx = uint32_t(g % jc.S);
      bounce = ps_len(ps);
      const uint32_t depth = ps_depth(ps);
      med = s->media[depth ? ps_medium(ps, depth - 1) : 0u];
      const float t1 = ref == PREF_END ? d4.w : t;
      thr = mul3(thr, medium_transmittance(med, length(xyz(d4)) * (t1 - o4.w)));
      // The direct integrator adds every surface's own emission
      // (RecursiveInteg::Lo, render/recursive-integ.cc:28-36).
      const bool include_emitters =
          (DIRECT && jc.integ == SNOG_INTEG_DIRECT) || bounce == 0 || ps_spec(ps) || jc.direct_samples == 0;
      if (ref == PREF_END) {
        if (include_emitters) rad = add(rad, mul3(background(*s, xyz(d4)), thr));
        if (bounce == 0 && rad.x == 0.f && rad.y == 0.f && rad.z == 0.f) alpha = jc.bg_alpha;
      } else {
        I = make_isec(*s, ref, xyz(o4), xyz(d4), t);
        const DevMaterial &M = s->mats[I.mat];
        if (include_emitters && M.type == MAT_GLOW && !I.back) rad = add(rad, mul3(load3(M.color), thr));
        const DevMaterial *bm = bsdf_material(*s, I.mat);
        if (bm) {
          B.m = bm;
          B.medium_ior = med.ior;
          B.enclosing_ior = depth >= 2 ? s->media[ps_medium(ps, depth - 2)].ior : 1.f;
          alive = true;
        }
      }
    }

    // ---- continuation first, so shadow rays know where their path lives --
    // Path integrator: one BSDF sample over all lobes, roulette beyond
    // min_path_len (render/path-integ.cc:309-385).  Direct integrator: the
    // specular reflection and the specular transmission each continue with
    // weight val |cos|, with roulette (survive 1/2 at weight 2) for rays
    // deeper than 5 (render/recursive-integ.cc:28-116).  Both run through
    // one bsdf_sample call site, so the BSDF code is inlined once.
    bool cont = false, spawn = false;
    float3 thr_next = thr, next_d = f3(0, 0, 0), thr_sp = f3(0, 0, 0), dir_sp = f3(0, 0, 0);
    float rr_next = rr_ratio;
    uint32_t ps_next = ps, ps_sp = 0;
    if (alive) {
      const JobConsts &jc = J->jc;
      const bool direct = (DIRECT && jc.integ == SNOG_INTEG_DIRECT);
      const uint32_t n_smp = direct ? 2u : 1u;
      for (uint32_t k = 0; k < n_smp; k++) {
        float2 prm = make_float2(0.f, 0.f);
        uint32_t flags = B_SPECULAR | (k ? B_TRANSMISSIVE : B_REFLECTIVE);
        if (!direct) {
          prm = bounce < jc.min_len ? strat_uv(strata_for(jc.S), rng, pixel, sidx, dim_of(bounce, K_BSDF))
                                    : rng.uv(dim_of(bounce, K_BSDF));
          flags = B_ALL;
        }
        BSample bs = bsdf_sample(B, I, prm, flags);
        float3 w;
        bool go;
        if (direct) {
          go = csum(bs.val) > 0.f && bounce + 1u < kMaxBounce;
          w = mul3(thr, mul(bs.val, fabsf(I.cos_n(bs.dir))));
          if (go && bounce + 1u > 5u) {
            if (rng.u(dim_of(bounce, K_RR) ^ (k << 20)) < 0.5f) go = false;
            else w = mul(w, 2.f);
          }
        } else {
          go = bs.pdf != 0.f && !(bs.val.x == 0.f && bs.val.y == 0.f && bs.val.z == 0.f);
          w = mul3(thr, mul(bs.val, fabsf(I.cos_n(bs.dir)) / bs.pdf));
          if (go && bounce > jc.min_len) {
            float p = fminf(intensity(w) * rr_ratio, 1.f);
            if (rng.u(dim_of(bounce, K_RR)) > p) {
              go = false;
            } else {
              w = mul(w, 1.f / p);
              rr_next = rr_ratio * p;
            }
          }
          go = go && bounce != jc.max_len;
        }
        if (!go) continue;
        uint32_t nps = (ps & ~0x1ffu) | (bounce + 1) | ((bs.flags & B_SPECULAR) ? 0x100u : 0u);
        if (bs.flags & B_TRANSMISSIVE) {
          const uint32_t mid = s->mats[I.mat].medium_id;
          if (mid && I.back) {
            nps = ps_pop(nps);
          } else if (mid && !ps_push(nps, mid)) {
            atomicOr(&ctl->err, 2u);   // a fifth nested medium: the path ends here
            continue;
          }
        }
        if (!cont) {
          cont = true;
          thr_next = w;
          next_d = I.nf.from(bs.dir);
          ps_next = nps;
        } else {
          spawn = true;
          thr_sp = w;
          dir_sp = I.nf.from(bs.dir);
          ps_sp = nps;
        }
      }
    }
    // A second ray waits in the spawn ring for a queue slot.  When the ring
    // is full, one of the two rays continues, chosen with probability 1/2,
    // at twice its weight -- an unbiased estimate of the pair's sum.
    {
      const uint32_t sslot = warp_append(&ctl->spawn_n, spawn);
      if (spawn) {
        if (sslot < ctl->spawn_room) {
          const JobConsts &jc = J->jc;
          const uint32_t at = uint32_t((ctl->spawn_tail + sslot) % sp_cap);
          sp.o[at] = make_float4(I.pos.x, I.pos.y, I.pos.z, jc.min_trace);
          sp.d[at] = make_float4(dir_sp.x, dir_sp.y, dir_sp.z, jc.horizon);
          sp.thr[at] = make_float4(thr_sp.x, thr_sp.y, thr_sp.z, 1.f);
          sp.rad[at] = make_float4(0.f, 0.f, 0.f, 0.f);
          sp.meta[at] = make_uint4(ps_sp, job, uint32_t(g), uint32_t(g >> 32));
        } else {
          if (rng.u(dim_of(bounce, K_RR) ^ (3u << 20)) < 0.5f) {
            thr_next = thr_sp;
            next_d = dir_sp;
            ps_next = ps_sp;
          }
          thr_next = mul(thr_next, 2.f);
          spawn = false;
        }
      }
      // Spawned rays per job: a job is finished when its finished rays
      // reach its paths plus its spawned rays.
      const uint32_t key = spawn ? job : 0xffffffffu;
      const unsigned m = __match_any_sync(0xffffffffu, key);
      if (spawn && lane == uint32_t(__ffs(m) - 1)) atomicAdd(job_spawned + job, (unsigned long long)__popc(m));
    }
    const uint32_t slot = warp_append(count_out, cont);
    float4 *target = nullptr;
    if (active && !retire) {
      if (cont) {
        const JobConsts &jc = J->jc;
        qout.o[slot] = make_float4(I.pos.x, I.pos.y, I.pos.z, jc.min_trace);
        qout.d[slot] = make_float4(next_d.x, next_d.y, next_d.z, jc.horizon);
        qout.thr[slot] = make_float4(thr_next.x, thr_next.y, thr_next.z, rr_next);
        qout.rad[slot] = make_float4(rad.x, rad.y, rad.z, alpha);
        qout.meta[slot] = make_uint4(ps_next, job, uint32_t(g), uint32_t(g >> 32));
        target = qout.rad + slot;
      } else {
        float4 *res = J->result + g;
        if (DIRECT && J->jc.integ == SNOG_INTEG_DIRECT) {
          // several rays of one path end here: their radiance adds up
          atomicAdd(&res->x, rad.x);
          atomicAdd(&res->y, rad.y);
          atomicAdd(&res->z, rad.z);
          if (alpha != 0.f) atomicAdd(&res->w, alpha);
        } else {
          *res = make_float4(rad.x, rad.y, rad.z, alpha);
        }
        target = res;
      }
    }
    // Count finished paths per job, one atomic per group of lanes sharing a job.
    {
      const bool fin = active && !cont;
      const uint32_t key = fin ? job : 0xffffffffu;
      const unsigned m = __match_any_sync(0xffffffffu, key);
      if (fin && lane == uint32_t(__ffs(m) - 1)) atomicAdd(job_done + job, (unsigned long long)__popc(m));
    }

    // Vertices with lights to sample go to the direct-lighting list.
    const bool lit = alive && J->jc.direct_samples != 0u && s->n_lights != 0u;
    const uint32_t dslot = warp_append(&ctl->dcount, lit);
    if (lit) {
      dl.idx[dslot] = i;
      dl.tgt[dslot] = reinterpret_cast<unsigned long long>(target);
    }
  }
}

// Direct lighting of the vertices the shading kernel listed, one list entry
// per thread: the vertex is rebuilt from its queue entry (the same arithmetic
// as in k_e_shade, so the same bits), then every light is sampled.  Kept out
// of k_e_shade so neither kernel's body outgrows the instruction cache, and
// run over a compacted list so escaped and absorbed paths leave no idle lanes.
template <bool DIRECT>
__global__ void __launch_bounds__(128, SNOG_DIRECT_MINBLOCKS) k_e_direct(EngineCtl *ctl, const EngineJobDev *jobs,
                                                  const DevScene *scenes, EQ qin, const uint32_t *hit_ref,
                                                  const float *hit_t, EDL dl, ESQ sq) {
  const uint32_t n = ctl->dcount;
  uint32_t *count_sq = &ctl->scount;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;

  for (uint32_t wb = warp * 32; wb < n; wb += nwarps * 32) {
    const uint32_t k = wb + lane;
    const bool alive = k < n;
    uint32_t scene = 0, bounce = 0, pixel = 0, sidx = 0;
    float3 thr = f3(0, 0, 0);
    Isec I;
    BsdfCtx B{nullptr, 1.f, 1.f};
    DevMedium med{1.f, {0, 0, 0}};
    const EngineJobDev *J = jobs;
    const DevScene *s = scenes;
    Rng rng{0, 0, 0, 0};
    float4 *target = nullptr;
    if (alive) {
      const uint32_t i = dl.idx[k];
      target = reinterpret_cast<float4 *>(dl.tgt[k]);
      const uint4 meta = qin.meta[i];
      const uint32_t ps = meta.x;
      const unsigned long long g = (unsigned long long)meta.z | ((unsigned long long)meta.w << 32);
      J = jobs + meta.y;
      scene = J->scene;
      s = scenes + scene;
      const JobConsts &jc = J->jc;
      const float4 o4 = qin.o[i], d4 = qin.d[i];
      const float t = hit_t[i];
      rng = Rng{jc.seed_lo, jc.seed_hi, uint32_t(g), uint32_t(g >> 32)};
      pixel = uint32_t(g / jc.S);
      sidx = uint32_t(g % jc.S);
      bounce = ps_len(ps);
      const uint32_t depth = ps_depth(ps);
      med = s->media[depth ? ps_medium(ps, depth - 1) : 0u];
      thr = mul3(xyz(qin.thr[i]), medium_transmittance(med, length(xyz(d4)) * (t - o4.w)));
      I = make_isec(*s, hit_ref[i], xyz(o4), xyz(d4), t);
      B.m = bsdf_material(*s, I.mat);
      B.medium_ior = med.ior;
      B.enclosing_ior = depth >= 2 ? s->media[ps_medium(ps, depth - 2)].ior : 1.f;
    }

    // ---- direct lighting (render/direct-illum.cc:83-255) ----------------
    // The light loop bound is the largest in the warp, so shadow-ray appends
    // stay warp-synchronous.
    uint32_t nl = (alive && J->jc.direct_samples) ? s->n_lights : 0u;
    uint32_t ns = alive ? J->jc.direct_samples : 0u;
    for (int off = 16; off > 0; off >>= 1) {
      nl = max(nl, __shfl_xor_sync(0xffffffffu, nl, off));
      ns = max(ns, __shfl_xor_sync(0xffffffffu, ns, off));
    }
    for (uint32_t l = 0; l < nl; l++) {
      for (uint32_t jn = 0; jn < ns; jn++) {
        bool emit_l = false, emit_b = false;
        float3 c_l = f3(0, 0, 0), c_b = f3(0, 0, 0), dir_l = c_l, dir_b = c_l;
        float dist_l = 0.f, dist_b = 0.f;
        const JobConsts &jc = J->jc;
        if (alive && l < s->n_lights && jn < jc.direct_samples) {
          const DevLight &L = s->lights[l];
          const bool point = is_point_light(L);
          const uint32_t flags = B_ALL & ~B_SPECULAR;
          const float inv_ns = 1.f / float(jc.direct_samples);
          const uint32_t kl = K_LIGHT0 + 3 * l;
          float2 pl, pb;
          // The direct integrator draws every depth's light samples from the
          // pixel's stratified set, as its sample channels are shared down
          // the recursion (render/recursive-integ.cc:28-36).
          if (bounce < jc.min_len || (DIRECT && jc.integ == SNOG_INTEG_DIRECT)) {
            const Strata st_direct = strata_for(jc.S * jc.direct_samples);
            pl = strat_uv(st_direct, rng, pixel, sidx * jc.direct_samples + jn, dim_of(bounce, kl));
            pb = strat_uv(st_direct, rng, pixel, sidx * jc.direct_samples + jn, dim_of(bounce, kl + 1));
          } else {
            const Strata st_rand = strata_for(jc.direct_samples);
            pl = strat_uv(st_rand, rng, uint32_t(rng.path_lo ^ (bounce << 24)), jn, dim_of(bounce, kl));
            pb = strat_uv(st_rand, rng, uint32_t(rng.path_lo ^ (bounce << 24)), jn, dim_of(bounce, kl + 1));
          }
          const float extra = rng.u(dim_of(bounce, kl + 2) ^ (jn << 20));
          LSample ls = light_sample(*s, L, I, pl, extra);
          if (ls.pdf > 0.f && csum(ls.val) > 0.f) {
            float bpdf;
            float3 bv = bsdf_eval(B, I, ls.dir, flags, bpdf);
            if (csum(bv) > 0.f) {
              float3 c = ls.val;
              c = mul3(c, medium_transmittance(med, (ls.dist == 0.f ? jc.horizon : ls.dist) - 2.f * jc.min_trace));
              if (!point) c = mul(c, mis_weight(ls.pdf, bpdf));
              c = mul(mul3(c, bv), fabsf(I.cos_n(ls.dir)) / ls.pdf);
              c_l = mul(mul3(c, thr), inv_ns);
              dir_l = ls.dir;
              dist_l = ls.dist;
              emit_l = true;
            }
          }
          if (!point) {
            BSample bs = bsdf_sample(B, I, pb, flags);
            if (bs.pdf > 0.f && csum(bs.val) > 0.f) {
              LSample lv = light_eval(*s, L, I, bs.dir);
              if (lv.pdf > 0.f && csum(lv.val) > 0.f) {
                float3 c = lv.val;
                c = mul3(c, medium_transmittance(med, (lv.dist == 0.f ? jc.horizon : lv.dist) - 2.f * jc.min_trace));
                c = mul(c, mis_weight(bs.pdf, lv.pdf));
                c = mul(mul3(c, bs.val), fabsf(I.cos_n(bs.dir)) / bs.pdf);
                c_b = mul(mul3(c, thr), inv_ns);
                dir_b = bs.dir;
                dist_b = lv.dist;
                emit_b = true;
              }
            }
          }
        }
        uint32_t sl = warp_append(count_sq, emit_l);
        if (emit_l) {
          const float3 wd = I.nf.from(dir_l);
          sq.o[sl] = make_float4(I.pos.x, I.pos.y, I.pos.z, jc.min_trace);
          sq.d[sl] = make_float4(wd.x, wd.y, wd.z, (dist_l == 0.f ? jc.horizon : dist_l) - jc.min_trace);
          sq.c[sl] = make_float4(c_l.x, c_l.y, c_l.z, __uint_as_float(scene));
          sq.tgt[sl] = reinterpret_cast<unsigned long long>(target);
        }
        sl = warp_append(count_sq, emit_b);
        if (emit_b) {
          const float3 wd = I.nf.from(dir_b);
          sq.o[sl] = make_float4(I.pos.x, I.pos.y, I.pos.z, jc.min_trace);
          sq.d[sl] = make_float4(wd.x, wd.y, wd.z, (dist_b == 0.f ? jc.horizon : dist_b) - jc.min_trace);
          sq.c[sl] = make_float4(c_b.x, c_b.y, c_b.z, __uint_as_float(scene));
          sq.tgt[sl] = reinterpret_cast<unsigned long long>(target);
        }
      }
    }
  }
}

// One iteration's kernel sequence on ST.  EV (null while capturing a graph)
// receives five events: before plan, before closest, before shade (shading and
// direct lighting), before shadow, after shadow.
template <int STACK, int PER>
void launch_iteration(cudaStream_t st, EngineCtl *ctl, const WorkItem *ring, uint32_t R, uint32_t N,
                      uint32_t cur, const EngineJobDev *jobs, const DevScene *scenes, EQ qc, EQ qn,
                      uint32_t *hit_ref, float *hit_t, EDL dl, ESQ sq, unsigned long long *job_done,
                      unsigned long long *job_spawned, EQ sp, uint32_t sp_cap, bool direct,
                      const cudaEvent_t *ev) {
  const uint32_t sms = uint32_t(num_sms());
  if (ev) cudaEventRecord(ev[0], st);
  k_e_plan<<<1, 1, 0, st>>>(ctl, ring, R, N, cur, sp_cap);
  k_e_regen<<<sms * 8, 256, 0, st>>>(ctl, ring, R, jobs, qc, sp, sp_cap);
  if (ev) cudaEventRecord(ev[1], st);
  k_e_closest<STACK, PER><<<resident_grid(k_e_closest<STACK, PER>, kTraceBlock), kTraceBlock, 0, st>>>(
      ctl, cur, jobs, scenes, qc, hit_ref, hit_t);
  if (ev) cudaEventRecord(ev[2], st);
  if (direct) {
    k_e_shade<true><<<sms * 12, 128, 0, st>>>(ctl, cur, jobs, scenes, qc, hit_ref, hit_t, qn, dl, job_done,
                                              job_spawned, sp, sp_cap);
    k_e_direct<true><<<sms * 12, 128, 0, st>>>(ctl, jobs, scenes, qc, hit_ref, hit_t, dl, sq);
  } else {
    k_e_shade<false><<<sms * 12, 128, 0, st>>>(ctl, cur, jobs, scenes, qc, hit_ref, hit_t, qn, dl, job_done,
                                               job_spawned, sp, sp_cap);
    k_e_direct<false><<<sms * 12, 128, 0, st>>>(ctl, jobs, scenes, qc, hit_ref, hit_t, dl, sq);
  }
  if (ev) cudaEventRecord(ev[3], st);
  k_e_shadow<STACK><<<resident_grid(k_e_shadow<STACK>, kTraceBlock), kTraceBlock, 0, st>>>(ctl, scenes, sq);
  if (ev) cudaEventRecord(ev[4], st);
}

}  // namespace

size_t BlockCache::round_up(size_t n) {
  if (n <= 4096) return 4096;
  size_t p = 1;
  while (p <= n / 2) p <<= 1;     // largest power of two <= n
  const size_t step = p / 8;
  return (n + step - 1) / step * step;
}

void *BlockCache::get(size_t n) {
  const size_t r = round_up(n);
  auto it = free_.lower_bound(r);
  if (it != free_.end() && it->first <= r + r / 4) {
    void *p = it->second;
    free_.erase(it);
    return p;
  }
  void *p = nullptr;
  if (cudaMalloc(&p, r) != cudaSuccess) {
    cudaGetLastError();
    trim();
    if (cudaMalloc(&p, r) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
  }
  size_of_[p] = r;
  held_ += r;
  return p;
}

void BlockCache::put(void *p) {
  if (!p) return;
  auto it = size_of_.find(p);
  if (it != size_of_.end()) free_.insert({it->second, p});
}

void BlockCache::trim() {
  for (auto &kv : free_) {
    cudaFree(kv.second);
    held_ -= size_of_[kv.second];
    size_of_.erase(kv.second);
  }
  free_.clear();
}

Engine::Engine(const EngineConfigHost &cfg, cudaStream_t stream) : cfg_(cfg) {
  t0_ = std::chrono::steady_clock::now();
  if (cfg_.slots < 1024 || cfg_.slots > (1u << 30) || cfg_.item_paths == 0 || cfg_.ring_items < 16 ||
      cfg_.max_jobs == 0 || cfg_.iters_per_launch == 0 || cfg_.iters_per_launch > 64 || cfg_.max_scenes == 0 ||
      cfg_.max_lights > 256)
    throw Error{SNOG_EINVAL, "engine config out of range"};
  max_scenes_ = cfg_.max_scenes;
  if (stream) {
    stream_ = stream;
  } else {
    check_cuda(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
    own_stream_ = true;
  }
  const size_t N = cfg_.slots, L = cfg_.max_lights ? cfg_.max_lights : 1;
  size_t off = 0;
  auto take = [&](size_t b) {
    size_t o = off;
    off += (b + 255) & ~size_t(255);
    return o;
  };
  size_t o_q[2][5];
  for (int k = 0; k < 2; k++)
    for (int a = 0; a < 5; a++) o_q[k][a] = take(16 * N);
  size_t o_href = take(4 * N), o_ht = take(4 * N), o_didx = take(4 * N), o_dtgt = take(8 * N);
  size_t o_so = take(16 * N * 2 * L), o_sd = take(16 * N * 2 * L), o_sc = take(16 * N * 2 * L),
         o_st = take(8 * N * 2 * L);
  // Spawn ring for the direct integrator's second rays: a quarter of the
  // queue (a full ring makes a vertex pick one of its two rays instead).
  sp_cap_ = std::max<uint32_t>(cfg_.slots / 4, 1024);
  size_t o_sp[5];
  for (int a = 0; a < 5; a++) o_sp[a] = take(16 * size_t(sp_cap_));
  size_t o_ctl = take(sizeof(EngineCtl)), o_ring = take(sizeof(WorkItem) * cfg_.ring_items);
  size_t o_jobs = take(sizeof(EngineJobDev) * cfg_.max_jobs), o_done = take(16 * size_t(cfg_.max_jobs));
  size_t o_sc2 = take(sizeof(DevScene) * max_scenes_);
  check_cuda(cudaMalloc(&block_, off), "engine buffers");
  char *b = static_cast<char *>(block_);
  for (int k = 0; k < 2; k++) {
    q_o_[k] = reinterpret_cast<float4 *>(b + o_q[k][0]);
    q_d_[k] = reinterpret_cast<float4 *>(b + o_q[k][1]);
    q_thr_[k] = reinterpret_cast<float4 *>(b + o_q[k][2]);
    q_rad_[k] = reinterpret_cast<float4 *>(b + o_q[k][3]);
    q_meta_[k] = reinterpret_cast<uint4 *>(b + o_q[k][4]);
  }
  sp_o_ = reinterpret_cast<float4 *>(b + o_sp[0]);
  sp_d_ = reinterpret_cast<float4 *>(b + o_sp[1]);
  sp_thr_ = reinterpret_cast<float4 *>(b + o_sp[2]);
  sp_rad_ = reinterpret_cast<float4 *>(b + o_sp[3]);
  sp_meta_ = reinterpret_cast<uint4 *>(b + o_sp[4]);
  hit_ref_ = reinterpret_cast<uint32_t *>(b + o_href);
  hit_t_ = reinterpret_cast<float *>(b + o_ht);
  d_idx_ = reinterpret_cast<uint32_t *>(b + o_didx);
  d_tgt_ = reinterpret_cast<unsigned long long *>(b + o_dtgt);
  s_o_ = reinterpret_cast<float4 *>(b + o_so);
  s_d_ = reinterpret_cast<float4 *>(b + o_sd);
  s_c_ = reinterpret_cast<float4 *>(b + o_sc);
  s_tgt_ = reinterpret_cast<unsigned long long *>(b + o_st);
  ctl_ = reinterpret_cast<EngineCtl *>(b + o_ctl);
  ring_ = reinterpret_cast<WorkItem *>(b + o_ring);
  jobs_dev_ = reinterpret_cast<EngineJobDev *>(b + o_jobs);
  job_done_ = reinterpret_cast<unsigned long long *>(b + o_done);
  scenes_dev_ = reinterpret_cast<DevScene *>(b + o_sc2);
  check_cuda(cudaMemsetAsync(ctl_, 0, sizeof(EngineCtl), stream_), "memset");
  check_cuda(cudaMemsetAsync(job_done_, 0, 16 * size_t(cfg_.max_jobs), stream_), "memset");
  check_cuda(cudaMallocHost(&ctl_host_, sizeof(EngineCtl)), "pinned");
  check_cuda(cudaMallocHost(&done_host_, 16 * size_t(cfg_.max_jobs)), "pinned");
  staging_cap_ = size_t(cfg_.max_jobs) * sizeof(EngineJobDev) + size_t(cfg_.ring_items) * sizeof(WorkItem) + 4096;
  check_cuda(cudaMallocHost(&staging_, staging_cap_), "pinned staging");
  std::memset(done_host_, 0, 16 * size_t(cfg_.max_jobs));
  for (uint32_t k = cfg_.max_jobs; k > 0; k--) free_slots_.push_back(k - 1);
  check_cuda(cudaStreamSynchronize(stream_), "engine init");
}

Engine::~Engine() {
  if (stream_) cudaStreamSynchronize(stream_);
  for (auto &kv : jobs_) release_job(kv.second);
  for (auto &row : graph_)
    for (cudaGraphExec_t &gx : row)
      if (gx) cudaGraphExecDestroy(gx);
  cache_.trim();
  cudaFree(block_);
  cudaFreeHost(ctl_host_);
  cudaFreeHost(done_host_);
  cudaFreeHost(staging_);
  for (cudaEvent_t e : events_) cudaEventDestroy(e);
  if (own_stream_) cudaStreamDestroy(stream_);
}

void Engine::reset_scenes() {
  if (!jobs_.empty()) throw Error{SNOG_EBUSY, "engine has jobs in flight"};
  scenes_.clear();
}

void Engine::clear_counters() {
  prof_ = Profile{};
  kernel_launches_ = 0;
  base_closest_ = last_ctl_.rays_closest;
  base_shadow_ = last_ctl_.rays_shadow;
}

double Engine::now_ms() const {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0_).count();
}

uint32_t Engine::add_scene(SceneImpl *scene) {
  if (!scene->on_device) throw Error{SNOG_EINVAL, "scene was built host-only"};
  if (scenes_.size() >= max_scenes_) throw Error{SNOG_EINVAL, "engine scene table full"};
  if (!stack_class_for_depth(scene->dev.max_depth))
    throw Error{SNOG_EINVAL, "octree deeper than the traversal kernels support"};
  if (scene->dev.n_lights > cfg_.max_lights)
    throw Error{SNOG_EINVAL, "scene has more lights than the engine's max_lights"};
  const uint32_t slot = uint32_t(scenes_.size());
  scenes_.push_back(scene);
  check_cuda(cudaMemcpyAsync(scenes_dev_ + slot, &scene->dev, sizeof(DevScene), cudaMemcpyHostToDevice, stream_),
             "scene table");
  check_cuda(cudaStreamSynchronize(stream_), "scene table");
  const int sc = stack_class_for_depth(scene->dev.max_depth);
  if (sc > graph_stack_) {
    for (auto &row : graph_)
      for (cudaGraphExec_t &gx : row) {
        if (gx) cudaGraphExecDestroy(gx);
        gx = nullptr;
      }
    graph_stack_ = sc;
  }
  return slot;
}

// Every iteration of one launch (iters_per_launch pairs, queue 0 -> 1 -> 0),
// with events around the kernels while profiling.
void Engine::launch_iterations(bool direct, bool pair) {
  EQ q[2];
  for (int k = 0; k < 2; k++) q[k] = EQ{q_o_[k], q_d_[k], q_thr_[k], q_rad_[k], q_meta_[k]};
  ESQ sq{s_o_, s_d_, s_c_, s_tgt_};
  const uint32_t n_iter = 2 * cfg_.iters_per_launch;
  if (profile_on_ && events_.size() < 5 * size_t(n_iter)) {
    while (events_.size() < 5 * size_t(n_iter)) {
      cudaEvent_t e;
      check_cuda(cudaEventCreate(&e), "event");
      events_.push_back(e);
    }
  }
  for (uint32_t it = 0; it < n_iter; it++) {
    const uint32_t cur = it & 1u;
    const cudaEvent_t *ev = profile_on_ ? &events_[5 * it] : nullptr;
#define SNOG_ITER(S, P)                                                                                     \
  launch_iteration<S, P>(stream_, ctl_, ring_, cfg_.ring_items, cfg_.slots, cur, jobs_dev_, scenes_dev_, q[cur], \
                         q[cur ^ 1], hit_ref_, hit_t_, EDL{d_idx_, d_tgt_}, sq, job_done_,                      \
                         job_done_ + cfg_.max_jobs, EQ{sp_o_, sp_d_, sp_thr_, sp_rad_, sp_meta_}, sp_cap_,     \
                         direct, ev)
    switch (graph_stack_ * 2 + (pair ? 1 : 0)) {
      case 64: SNOG_ITER(32, 1); break;
      case 65: SNOG_ITER(32, 2); break;
      case 128: SNOG_ITER(64, 1); break;
      case 129: SNOG_ITER(64, 2); break;
      case 256: SNOG_ITER(128, 1); break;
      case 257: SNOG_ITER(128, 2); break;
      case 513: SNOG_ITER(256, 2); break;
      default: SNOG_ITER(256, 1); break;
    }
#undef SNOG_ITER
  }
}

void Engine::build_graph(bool direct, bool pair) {
  cudaGraph_t g;
  const bool prof = profile_on_;
  profile_on_ = false;
  check_cuda(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capture");
  launch_iterations(direct, pair);
  profile_on_ = prof;
  cudaError_t e = cudaStreamEndCapture(stream_, &g);
  check_cuda(e, "end capture");
  e = cudaGraphInstantiate(&graph_[direct][pair], g, 0);
  cudaGraphDestroy(g);
  check_cuda(e, "graph instantiate");
}

uint64_t Engine::scene_check(uint32_t scene_slot) const {
  const DevScene &d = scenes_.at(scene_slot)->dev;
  return uint64_t(d.n_tri + d.n_sph + d.n_tpar) | (uint64_t(d.n_nodes) << 32);
}

uint64_t Engine::submit(uint32_t scene_slot, const SnogCamera &cam, const SnogRenderParams &p, float *out,
                        bool out_on_device, double submit_ms, Checkpoint *resume, const SnogRenderWindow *win) {
  if (scene_slot >= scenes_.size()) throw Error{SNOG_ENOTFOUND, "unknown scene slot"};
  if (p.width == 0 || p.height == 0 || p.spp == 0) throw Error{SNOG_EINVAL, "width, height, spp must be > 0"};
  if (p.max_path_len > 255) throw Error{SNOG_EINVAL, "max_path_len must be <= 255"};
  if (p.integrator > SNOG_INTEG_DIRECT) throw Error{SNOG_EINVAL, "unknown integrator"};
  if (p.direct_samples > 64) throw Error{SNOG_EINVAL, "direct_samples must be <= 64"};
  if (win) {
    check_window(p, *win);
    if (resume) throw Error{SNOG_EINVAL, "a windowed job cannot resume a checkpoint"};
  }
  const uint64_t pat_pixels =
      win ? uint64_t(win->pat_width) * win->pat_height : uint64_t(p.width + 4) * (p.height + 4);
  if (pat_pixels * p.spp >= (1ull << 32)) throw Error{SNOG_EINVAL, "a job is limited to 2^32 paths"};
  if (scenes_[scene_slot]->dev.n_lights * p.direct_samples > cfg_.max_lights)
    throw Error{SNOG_EINVAL, "lights x direct_samples exceeds the engine's max_lights"};
  HostJob j;
  j.id = next_id_++;
  j.scene_slot = scene_slot;
  j.jc = make_job(scenes_[scene_slot]->dev, cam, p, win);
  j.total = job_total(j.jc);
  j.npix = size_t(j.jc.W) * j.jc.H;
  j.out = out;
  j.out_on_device = out_on_device;
  j.bytes = j.total * 24 + j.npix * (20 + (out_on_device ? 0 : 12)) + 4096;
  if (j.bytes > cfg_.mem_budget) throw Error{SNOG_ENOMEM, "job larger than the engine's memory budget"};
  j.st.submit_ms = submit_ms >= 0 ? submit_ms : now_ms();
  j.st.paths = uint64_t(j.jc.W) * j.jc.H * p.spp;
  j.cam = cam;
  j.params = p;
  if (resume) {
    if (resume->total != j.total || resume->done > j.total || resume->result.size() != resume->done ||
        resume->jit.size() != resume->done)
      throw Error{SNOG_EINVAL, "checkpoint does not match the job's size"};
    if (resume->scene_check != scene_check(scene_slot))
      throw Error{SNOG_EINVAL, "checkpoint was taken on a different scene"};
    j.resume.reset(new Checkpoint(std::move(*resume)));
  }
  const uint64_t id = j.id;
  jobs_.emplace(id, std::move(j));
  pending_.push_back(id);
  return id;
}

bool Engine::pause(uint64_t id, bool on) {
  auto it = jobs_.find(id);
  if (it == jobs_.end()) return false;
  it->second.paused = on;
  return true;
}

bool Engine::drained(uint64_t id) const {
  auto it = jobs_.find(id);
  if (it == jobs_.end()) return false;
  const HostJob &j = it->second;
  return j.paused && j.table_slot != ~0u && rays_done(j) >= j.pushed + rays_spawned(j);
}

void Engine::checkpoint(uint64_t id, Checkpoint &out) {
  if (!drained(id)) throw Error{SNOG_EBUSY, "job is not paused with its paths finished"};
  HostJob &j = jobs_.at(id);
  out.cam = j.cam;
  out.params = j.params;
  out.total = j.total;
  out.done = j.pushed;
  out.scene_check = scene_check(j.scene_slot);
  out.result.resize(j.pushed);
  out.jit.resize(j.pushed);
  if (j.pushed) {
    check_cuda(cudaMemcpyAsync(out.result.data(), j.result, j.pushed * sizeof(float4), cudaMemcpyDeviceToHost,
                               stream_),
               "checkpoint");
    check_cuda(cudaMemcpyAsync(out.jit.data(), j.jit, j.pushed * sizeof(float2), cudaMemcpyDeviceToHost, stream_),
               "checkpoint");
  }
  check_cuda(cudaStreamSynchronize(stream_), "checkpoint");
}

bool Engine::cancel(uint64_t id) {
  auto it = jobs_.find(id);
  if (it == jobs_.end()) return false;
  it->second.canceled = true;
  return true;
}

void Engine::release_job(HostJob &j) {
  cache_.put(j.result);
  cache_.put(j.jit);
  cache_.put(j.accum);
  cache_.put(j.wsum);
  if (!j.out_on_device) cache_.put(j.dev_out);
  j.result = nullptr;
  j.jit = nullptr;
  j.accum = nullptr;
  j.wsum = nullptr;
  j.dev_out = nullptr;
}

void *Engine::stage(const void *src, size_t n) {
  const size_t need = (n + 15) & ~size_t(15);
  if (staging_used_ + need > staging_cap_) {
    // Everything staged so far must have been copied before the area is reused.
    check_cuda(cudaStreamSynchronize(stream_), "staging");
    staging_used_ = 0;
  }
  char *p = staging_ + staging_used_;
  std::memcpy(p, src, n);
  staging_used_ += need;
  return p;
}

// Admit pending jobs in arrival order while the memory budget and the job
// table allow.
void Engine::admit() {
  while (!pending_.empty()) {
    HostJob &j = jobs_.at(pending_.front());
    if (j.canceled) {
      j.st.status = SNOG_ECANCELED;
      finished_[j.id] = j.st;
      jobs_.erase(j.id);
      pending_.pop_front();
      continue;
    }
    if (free_slots_.empty() || budget_used_ + j.bytes > cfg_.mem_budget) break;
    auto alloc = [&](void **p, size_t n) {
      *p = cache_.get(n);
      return *p != nullptr;
    };
    bool ok = alloc(reinterpret_cast<void **>(&j.result), j.total * 16) &&
              alloc(reinterpret_cast<void **>(&j.jit), j.total * 8) &&
              alloc(reinterpret_cast<void **>(&j.accum), j.npix * 16) &&
              alloc(reinterpret_cast<void **>(&j.wsum), j.npix * 4);
    if (ok && !j.out_on_device) ok = alloc(reinterpret_cast<void **>(&j.dev_out), j.npix * 12);
    if (!ok) {
      release_job(j);
      if (!active_.empty()) break;   // device full: retry once running jobs have freed memory
      // Nothing running will free memory: this job cannot be admitted.
      j.st.status = SNOG_ENOMEM;
      j.st.finish_ms = now_ms();
      finished_[j.id] = j.st;
      jobs_.erase(j.id);
      pending_.pop_front();
      continue;
    }
    if (j.out_on_device) j.dev_out = j.out;
    j.table_slot = free_slots_.back();
    free_slots_.pop_back();
    budget_used_ += j.bytes;
    EngineJobDev rec;
    std::memset(&rec, 0, sizeof rec);
    rec.jc = j.jc;
    rec.scene = j.scene_slot;
    rec.total = j.total;
    rec.result = j.result;
    rec.jit = j.jit;
    check_cuda(cudaMemcpyAsync(jobs_dev_ + j.table_slot, stage(&rec, sizeof rec), sizeof rec,
                               cudaMemcpyHostToDevice, stream_),
               "job record");
    check_cuda(cudaMemsetAsync(job_done_ + j.table_slot, 0, 8, stream_), "job counter");
    check_cuda(cudaMemsetAsync(job_done_ + cfg_.max_jobs + j.table_slot, 0, 8, stream_), "job counter");
    done_host_[j.table_slot] = 0;
    done_host_[cfg_.max_jobs + j.table_slot] = 0;
    // The direct integrator's rays of one path add into its result.
    if (j.jc.integ == SNOG_INTEG_DIRECT)
      check_cuda(cudaMemsetAsync(j.result, 0, j.total * sizeof(float4), stream_), "result");
    if (j.resume) {
      // A resumed job: its finished paths come from the checkpoint and
      // count as done; work items start after them.
      const Checkpoint &c = *j.resume;
      if (c.done) {
        check_cuda(cudaMemcpyAsync(j.result, c.result.data(), c.done * sizeof(float4), cudaMemcpyHostToDevice,
                                   stream_),
                   "resume");
        check_cuda(cudaMemcpyAsync(j.jit, c.jit.data(), c.done * sizeof(float2), cudaMemcpyHostToDevice, stream_),
                   "resume");
        const unsigned long long done = c.done;
        check_cuda(cudaMemcpyAsync(job_done_ + j.table_slot, &done, 8, cudaMemcpyHostToDevice, stream_), "resume");
        check_cuda(cudaStreamSynchronize(stream_), "resume");
      }
      j.pushed = c.done;
      done_host_[j.table_slot] = c.done;
      j.resume.reset();
    }
    j.st.admit_ms = now_ms();
    active_.push_back(j.id);
    pending_.pop_front();
  }
}

// Push work items while the ring has room, at most about four queues' worth
// of paths ahead of what the device has taken, in arrival order: the oldest
// admitted job with work left goes first, so the job that waited longest
// finishes first (arrival order minimises the largest latency on one
// device), except that small jobs -- at most a quarter of the queue -- go
// ahead of large ones: they cost the large ones little and finish within a
// launch.  The window keeps that possible for small jobs that arrive while
// large ones run; it still covers more than one launch of iterations.
void Engine::push_items() {
  const uint64_t R = cfg_.ring_items;
  const uint64_t small = std::max<uint64_t>(cfg_.slots / 4, 1);
  const uint64_t window = 4 * uint64_t(cfg_.slots);
  std::vector<WorkItem> batch;
  const uint64_t head = last_ctl_.item_head;
  auto room = [&] {
    return pushed_tail_ + batch.size() - head < R - 1 && pushed_cum_ - last_ctl_.ticket < window;
  };
  auto push_from = [&](HostJob &j) {
    WorkItem w;
    w.job = j.table_slot;
    w.pad = 0;
    w.begin = j.pushed;
    w.count = std::min<uint64_t>(cfg_.item_paths, j.total - j.pushed);
    w.cum = pushed_cum_;
    pushed_cum_ += w.count;
    j.pushed += w.count;
    if (j.st.start_ms == 0) j.st.start_ms = now_ms();
    batch.push_back(w);
  };
  for (int pass = 0; pass < 2; pass++) {   // small jobs, then all jobs, each in arrival order
    for (size_t k = 0; k < active_.size() && room(); k++) {
      HostJob &j = jobs_.at(active_[k]);
      if (j.canceled || j.paused || (pass == 0 && j.total > small)) continue;
      while (j.pushed < j.total && room()) push_from(j);
    }
  }
  if (batch.empty()) return;
  // Copy into the ring (possibly wrapping), then publish tail and avail_end.
  uint64_t pos = pushed_tail_;
  size_t k = 0;
  while (k < batch.size()) {
    const uint64_t slot = pos % R;
    const size_t run = std::min<size_t>(batch.size() - k, size_t(R - slot));
    check_cuda(cudaMemcpyAsync(ring_ + slot, stage(batch.data() + k, run * sizeof(WorkItem)),
                               run * sizeof(WorkItem), cudaMemcpyHostToDevice, stream_),
               "ring push");
    k += run;
    pos += run;
  }
  pushed_tail_ = pos;
  // tail and avail_end are adjacent fields of the control block
  unsigned long long pub[2] = {pushed_tail_, pushed_cum_};
  check_cuda(cudaMemcpyAsync(&ctl_->item_tail, stage(pub, sizeof pub), sizeof pub, cudaMemcpyHostToDevice, stream_),
             "ring tail");
}

bool Engine::step() {
  if (staging_used_) {
    check_cuda(cudaStreamSynchronize(stream_), "staging");   // earlier staged copies done
    staging_used_ = 0;
  }
  admit();
  // Tell the device about cancellations: the job's queued paths retire.
  for (uint64_t id : active_) {
    HostJob &j = jobs_.at(id);
    if (j.canceled && !j.cancel_sent) {
      const uint32_t one = 1;
      check_cuda(cudaMemcpyAsync(&jobs_dev_[j.table_slot].canceled, stage(&one, sizeof one), sizeof one,
                                 cudaMemcpyHostToDevice, stream_),
                 "cancel flag");
      j.cancel_sent = true;
    }
  }
  push_items();
  // After a launch (an even number of iterations) the live rays are in queue 0.
  const bool inflight = last_ctl_.qcount[0] > 0 || last_ctl_.ticket < pushed_cum_ ||
                        last_ctl_.spawn_tail > last_ctl_.spawn_head || last_ctl_.spawn_n > 0;
  if (!inflight && active_.empty() && pending_.empty()) return false;
  // Launch while paths are in flight or an active job has work to push; a
  // job complete on the device is finished below either way.
  bool work = inflight;
  for (size_t k = 0; k < active_.size() && !work; k++) {
    const HostJob &j = jobs_.at(active_[k]);
    work = !j.paused && !j.canceled && j.pushed < j.total;
  }
  bool finishing = false;
  for (size_t k = 0; k < active_.size() && !finishing; k++) {
    const HostJob &j = jobs_.at(active_[k]);
    finishing = rays_done(j) >= j.total + rays_spawned(j) ||
                (j.canceled && rays_done(j) >= j.pushed + rays_spawned(j));
  }
  // Nothing to launch or finish: every remaining job is paused (or waits
  // for memory a paused job holds).  The caller waits for a command.
  if (!work && !finishing) return false;
  // The shading kernel with the direct integrator's code while a job of that
  // integrator is active (spawned rays belong to such jobs).
  bool direct = false;
  for (size_t k = 0; k < active_.size() && !direct; k++)
    direct = jobs_.at(active_[k]).jc.integ == SNOG_INTEG_DIRECT;
  // Closest-hit rounds deal list entries in pairs while most of the active
  // jobs' remaining paths are in scenes with long lists along rays.
  uint64_t paired = 0, single = 0;
  for (size_t k = 0; k < active_.size(); k++) {
    const HostJob &j = jobs_.at(active_[k]);
    const uint64_t left = j.total > rays_done(j) ? j.total - rays_done(j) : 0;
    (scenes_[j.scene_slot]->dev.pair_lists ? paired : single) += left;
  }
  const bool pair = paired > single;
  if (work) {
    if (profile_on_) {
      launch_iterations(direct, pair);
    } else {
      if (!graph_[direct][pair]) build_graph(direct, pair);
      check_cuda(cudaGraphLaunch(graph_[direct][pair], stream_), "graph launch");
    }
    kernel_launches_ += 6 * 2 * cfg_.iters_per_launch;
    check_cuda(cudaMemcpyAsync(ctl_host_, ctl_, sizeof(EngineCtl), cudaMemcpyDeviceToHost, stream_), "ctl");
    check_cuda(cudaMemcpyAsync(done_host_, job_done_, 16 * size_t(cfg_.max_jobs), cudaMemcpyDeviceToHost, stream_),
               "done");
    check_cuda(cudaStreamSynchronize(stream_), "iteration");
    staging_used_ = 0;
    last_ctl_ = *ctl_host_;
    check_render_flags(last_ctl_.err);
    if (profile_on_) {
      for (uint32_t it = 0; it < 2 * cfg_.iters_per_launch; it++) {
        const cudaEvent_t *ev = &events_[5 * it];
        float ms[4];
        for (int k = 0; k < 4; k++) check_cuda(cudaEventElapsedTime(&ms[k], ev[k], ev[k + 1]), "event time");
        prof_.other_ms += ms[0];
        prof_.closest_ms += ms[1];
        prof_.shade_ms += ms[2];
        prof_.shadow_ms += ms[3];
      }
      prof_.iterations += 2 * cfg_.iters_per_launch;
    }
  }
  // Completed (or cancelled and drained) jobs: filter every finished job's
  // samples into its image (and copy host images back), one sync for all.
  std::vector<size_t> done_idx;
  bool copies = false;
  for (size_t k = 0; k < active_.size(); k++) {
    HostJob &j = jobs_.at(active_[k]);
    const uint64_t done = rays_done(j), spawned = rays_spawned(j);
    if (done >= j.total + spawned || (j.canceled && done >= j.pushed + spawned)) {
      done_idx.push_back(k);
      if (done >= j.total + spawned && !j.cancel_sent) {   // complete before any cancel reached the device
        check_cuda(splat_job(j.jc, j.result, j.jit, j.total, j.accum, j.wsum, j.dev_out, stream_), "splat");
        kernel_launches_ += 2;
        if (!j.out_on_device)
          check_cuda(cudaMemcpyAsync(j.out, j.dev_out, j.npix * 12, cudaMemcpyDeviceToHost, stream_), "image D2H");
        copies = true;
      }
    }
  }
  if (copies) check_cuda(cudaStreamSynchronize(stream_), "finish");
  const double t_fin = now_ms();
  for (size_t r = done_idx.size(); r-- > 0;) {
    const size_t k = done_idx[r];
    HostJob &j = jobs_.at(active_[k]);
    j.st.status = (rays_done(j) >= j.total + rays_spawned(j) && !j.cancel_sent) ? SNOG_OK : SNOG_ECANCELED;
    j.st.finish_ms = t_fin;
    budget_used_ -= j.bytes;
    release_job(j);
    free_slots_.push_back(j.table_slot);
    finished_[j.id] = j.st;
    jobs_.erase(j.id);
    active_.erase(active_.begin() + long(k));
  }
  return true;
}

void Engine::run_to_completion() {
  while (step()) {
  }
}

JobStatsHost Engine::stats(uint64_t id) {
  auto f = finished_.find(id);
  if (f != finished_.end()) return f->second;
  auto j = jobs_.find(id);
  if (j != jobs_.end()) return j->second.st;
  JobStatsHost none;
  none.status = SNOG_ENOTFOUND;
  return none;
}

}  // namespace snog
