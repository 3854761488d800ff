// probe.cu -- snog_sample_probe: the shading functions of the path evaluated
// at given parameters, for per-sample comparison with the reference.
//
// The renderers draw their sample parameters from a counter-based generator,
// the reference from per-thread mt19937 streams, so whole images agree only
// statistically.  This entry point takes the parameters as input instead:
// for each probe (a ray and two 2-D parameters) it finds the closest hit from
// the scene's default medium and evaluates, at that hit, the same device
// functions the shading kernels call -- Bsdf::sample (material/bsdf.h:158-161)
// at the BSDF parameter, every light sampler's sample
// (light/light-sampler.h) at the light parameter, Bsdf::eval at each light
// sample's direction and each light sampler's eval at the BSDF sample's
// direction -- so each can be compared, sample by sample, with the
// reference's functions at the same parameters.

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "launch.h"
#include "scene.h"
#include "shade.cuh"

namespace snog {

int set_error(int code, const std::string &msg);
extern thread_local std::string g_last_error;

namespace {

// Output layout per probe (floats): kProbeHead, then kProbeLight per light.
constexpr int kProbeHead = 9;    // hit, BSDF sample val[3] pdf dir[3] flags
constexpr int kProbeLight = 18;  // light sample val[3] pdf dir[3] dist extra; BSDF eval
                                 // there val[3] pdf; light eval at the BSDF sample's
                                 // dir val[3] pdf dist

// One thread per probe.  PR: 12 floats per probe (origin, t0, direction,
// t1, BSDF u v, light u v); EXTRA: n_lights numbers per probe for samplers
// that draw one more (the sphere light).
__global__ void k_probe_shade(DevScene s, const float *__restrict__ pr, const float *__restrict__ extra,
                              const int32_t *__restrict__ prim, const float *__restrict__ hit_t, uint32_t n,
                              float *__restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t nl = s.n_lights;
  float *r = out + size_t(i) * (kProbeHead + size_t(kProbeLight) * nl);
  for (uint32_t k = 0; k < kProbeHead + kProbeLight * nl; k++) r[k] = 0.f;
  if (prim[i] < 0) return;
  const float *q = pr + size_t(i) * 12;
  const Isec I = make_isec(s, uint32_t(prim[i]), f3(q[0], q[1], q[2]), f3(q[4], q[5], q[6]), hit_t[i]);
  r[0] = 1.f;
  const DevMaterial *bm = bsdf_material(s, I.mat);
  // A ray from the default medium (media[0]), which no medium encloses.
  const BsdfCtx B{bm, s.media[0].ior, 1.f};
  BSample bs{f3(0.f, 0.f, 0.f), 0.f, f3(0.f, 0.f, 0.f), 0u};
  if (bm) bs = bsdf_sample(B, I, make_float2(q[8], q[9]), B_ALL);
  r[1] = bs.val.x; r[2] = bs.val.y; r[3] = bs.val.z;
  r[4] = bs.pdf;
  r[5] = bs.dir.x; r[6] = bs.dir.y; r[7] = bs.dir.z;
  r[8] = float(bs.flags);
  for (uint32_t k = 0; k < nl; k++) {
    float *l = r + kProbeHead + size_t(kProbeLight) * k;
    const DevLight &L = s.lights[k];
    const float ex = extra ? extra[size_t(i) * nl + k] : 0.5f;
    const LSample ls = light_sample(s, L, I, make_float2(q[10], q[11]), ex);
    l[0] = ls.val.x; l[1] = ls.val.y; l[2] = ls.val.z;
    l[3] = ls.pdf;
    l[4] = ls.dir.x; l[5] = ls.dir.y; l[6] = ls.dir.z;
    l[7] = ls.dist;
    l[8] = ex;
    if (bm && ls.pdf != 0.f) {
      float pdf = 0.f;
      const float3 v = bsdf_eval(B, I, ls.dir, B_ALL, pdf);
      l[9] = v.x; l[10] = v.y; l[11] = v.z;
      l[12] = pdf;
    }
    if (bm && bs.pdf != 0.f) {
      const LSample le = light_eval(s, L, I, bs.dir);
      l[13] = le.val.x; l[14] = le.val.y; l[15] = le.val.z;
      l[16] = le.pdf;
      l[17] = le.dist;
    }
  }
}

}  // namespace
}  // namespace snog

using namespace snog;

extern "C" int snog_sample_probe(SnogScene *scene, const float *probes, const float *extra, uint32_t n,
                                 float *out) {
  try {
    g_last_error.clear();
    if (!scene || (n && (!probes || !out))) throw Error{SNOG_EINVAL, "null argument"};
    SceneImpl &S = *scene->impl;
    if (!S.on_device) throw Error{SNOG_EINVAL, "scene was built host-only"};
    if (!stack_class_for_depth(S.dev.max_depth))
      throw Error{SNOG_EINVAL, "octree deeper than the traversal kernels support (84 levels)"};
    if (n == 0) return SNOG_OK;
    std::lock_guard<std::mutex> lk(S.mu);
    const uint32_t nl = S.dev.n_lights;
    const size_t stride = kProbeHead + size_t(kProbeLight) * nl;
    // The closest hits, through the ray-batch traversal (SoA rays, t0 = 0).
    std::vector<float> soa(size_t(n) * 7);
    for (uint32_t i = 0; i < n; i++) {
      const float *q = probes + size_t(i) * 12;
      if (q[3] != 0.f) throw Error{SNOG_EINVAL, "probe rays must start at t0 = 0"};
      const float v[7] = {q[0], q[1], q[2], q[4], q[5], q[6], q[7]};
      for (int a = 0; a < 7; a++) soa[size_t(a) * n + i] = v[a];
    }
    DevBuf d_soa(soa.size() * 4), d_pr(size_t(n) * 48), d_ex(extra ? size_t(n) * nl * 4 : 0),
        d_prim(size_t(n) * 4), d_t(size_t(n) * 4), d_cnt(64), d_out(size_t(n) * stride * 4);
    check_cuda(cudaMemcpy(d_soa.p, soa.data(), soa.size() * 4, cudaMemcpyHostToDevice), "probe rays H2D");
    check_cuda(cudaMemcpy(d_pr.p, probes, size_t(n) * 48, cudaMemcpyHostToDevice), "probes H2D");
    if (extra && nl)
      check_cuda(cudaMemcpy(d_ex.p, extra, size_t(n) * nl * 4, cudaMemcpyHostToDevice), "extra H2D");
    check_cuda(cudaMemset(d_cnt.p, 0, 64), "memset");
    check_cuda(launch_trace_batch(S.dev, d_soa.as<float>(), n, n, d_prim.as<int32_t>(), d_t.as<float>(), nullptr,
                                  d_cnt.as<unsigned long long>(), d_cnt.as<uint32_t>() + 8,
                                  d_cnt.as<uint32_t>() + 9, nullptr, nullptr),
               "probe trace launch");
    k_probe_shade<<<(n + 127) / 128, 128>>>(S.dev, d_pr.as<float>(), extra && nl ? d_ex.as<float>() : nullptr,
                                             d_prim.as<int32_t>(), d_t.as<float>(), n, d_out.as<float>());
    check_cuda(cudaGetLastError(), "probe shade launch");
    check_cuda(cudaMemcpy(out, d_out.p, size_t(n) * stride * 4, cudaMemcpyDeviceToHost), "probe D2H");
    uint32_t flags[2];
    check_cuda(cudaMemcpy(flags, d_cnt.as<uint32_t>() + 8, 8, cudaMemcpyDeviceToHost), "flags D2H");
    if (flags[0]) throw Error{SNOG_EINVAL, "traversal stack overflow (non-finite ray?)"};
    return SNOG_OK;
  } catch (const Error &e) {
    return set_error(e.code, e.msg);
  } catch (const std::exception &e) {
    return set_error(SNOG_EINVAL, e.what());
  }
}
