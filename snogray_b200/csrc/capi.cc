// capi.cc -- the extern "C" entry points of include/snogray_b200.h for
// scenes and ray batches.  No exception crosses this boundary: every entry
// catches snog::Error / std::exception and returns a status, with the message
// kept per thread for snog_last_error().

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "launch.h"
#include "ply.h"
#include "scene.h"

namespace snog {

thread_local std::string g_last_error;

int set_error(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

int num_sms() {
  static int cached[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (!cached[dev]) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    cached[dev] = v > 0 ? v : 148;
  }
  return cached[dev];
}

int blocks_per_sm_cached(const void *kernel, int threads, int (*query)(const void *, int)) {
  static std::mutex mu;
  static std::vector<std::pair<std::pair<const void *, int>, int>> cache;
  std::lock_guard<std::mutex> lk(mu);
  for (auto &e : cache)
    if (e.first.first == kernel && e.first.second == threads) return e.second;
  int v = query(kernel, threads);
  cache.push_back({{kernel, threads}, v});
  return v;
}

template <class F>
int guarded(F &&f) {
  try {
    g_last_error.clear();
    return f();
  } catch (const Error &e) {
    return set_error(e.code, e.msg);
  } catch (const std::bad_alloc &) {
    return set_error(SNOG_ENOMEM, "host allocation failed");
  } catch (const std::exception &e) {
    return set_error(SNOG_EINVAL, e.what());
  } catch (...) {
    return set_error(SNOG_EINVAL, "unknown error");
  }
}

void RenderCache::release() {
  wave_free(wb);
  cudaFree(accum);
  cudaFree(wsum);
  cudaFree(out);
  accum = nullptr;
  wsum = nullptr;
  out = nullptr;
  npix_cap = 0;
}

// Paths per wave: SNOG_WAVE_PATHS if set, else 16M, limited to what fits in
// a quarter of the free device memory and to the job's own path count.
static uint64_t choose_wave_cap(uint64_t total_paths, uint32_t spp, uint32_t n_lights) {
  uint64_t cap = 1ull << 24;
  if (const char *e = getenv("SNOG_WAVE_PATHS")) cap = strtoull(e, nullptr, 10);
  size_t free_b = 0, tot_b = 0;
  if (cudaMemGetInfo(&free_b, &tot_b) == cudaSuccess) {
    uint64_t fit = (free_b / 4) / wave_bytes_per_path(n_lights);
    if (cap > fit) cap = fit;
  }
  if (cap > total_paths) cap = total_paths;
  cap = (cap / spp) * spp;
  if (cap < spp) cap = spp;
  return (cap + 255) & ~uint64_t(255);
}

static void check_params(const SnogRenderParams &p) {
  if (p.width == 0 || p.height == 0 || p.spp == 0)
    throw Error{SNOG_EINVAL, "width, height and spp must be positive"};
  if (p.width > 65536 || p.height > 65536) throw Error{SNOG_EINVAL, "image too large"};
  if (p.max_path_len > 255) throw Error{SNOG_EINVAL, "max_path_len must be <= 255"};
  if (p.direct_samples > 64) throw Error{SNOG_EINVAL, "direct_samples must be <= 64"};
  if (p.integrator > SNOG_INTEG_DIRECT) throw Error{SNOG_EINVAL, "unknown integrator"};
  if (uint64_t(p.width + 4) * (p.height + 4) * p.spp >= (1ull << 40))
    throw Error{SNOG_EINVAL, "too many paths in one job"};
  if (uint64_t(p.width + 4) * (p.height + 4) >= (1ull << 32))
    throw Error{SNOG_EINVAL, "render pattern too large"};
}

RenderPool &render_pool(int device) {
  static std::mutex mu;
  static std::map<int, std::unique_ptr<RenderPool>> pools;
  std::lock_guard<std::mutex> lk(mu);
  auto &p = pools[device];
  if (!p) p.reset(new RenderPool);
  return *p;
}

// Render with the device's pooled working memory; the resolved image goes to
// d_out (device) or, if null, to h_out (host, copied before returning).
static void render_into(SceneImpl &S, const SnogCamera &cam, const SnogRenderParams &p, float *d_out,
                        float *h_out, cudaStream_t st, SnogRenderStats *stats,
                        const SnogRenderWindow *win = nullptr) {
  check_params(p);
  if (win) check_window(p, *win);
  if (p.integrator == SNOG_INTEG_DIRECT) {   // the streaming engine carries its spawned rays
    render_on_engine(S, cam, p, d_out, h_out, st, stats, win);
    return;
  }
  if (!stack_class_for_depth(S.dev.max_depth))
    throw Error{SNOG_EINVAL, "octree deeper than the traversal kernels support (84 levels)"};
  RenderPool &pool = render_pool(S.device);
  std::lock_guard<std::mutex> plk(pool.mu);
  if (!pool.done) check_cuda(cudaEventCreateWithFlags(&pool.done, cudaEventDisableTiming), "event");
  RenderCache &rc = pool.rc;
  JobConsts jc = make_job(S.dev, cam, p, win);
  const uint64_t total = job_total(jc);
  // Shadow-queue entries a vertex may need: two per light sample.
  const uint32_t ls = std::max(1u, S.dev.n_lights) * std::max(1u, p.direct_samples);
  uint64_t cap = choose_wave_cap(total, p.spp, ls);
  const size_t npix = size_t(jc.W) * jc.H;
  const bool grow = rc.wb.wave_cap < cap || rc.wb.n_lights < ls || rc.npix_cap < npix;
  // Buffers about to be replaced may still be in use by a render on another stream.
  if (grow) check_cuda(cudaEventSynchronize(pool.done), "pool wait");
  check_cuda(cudaStreamWaitEvent(st, pool.done, 0), "pool order");
  if (rc.wb.wave_cap < cap || rc.wb.n_lights < ls) {
    cudaError_t e = wave_alloc(rc.wb, std::max<uint64_t>(cap, rc.wb.wave_cap), std::max(ls, rc.wb.n_lights));
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw Error{SNOG_ENOMEM, std::string("wave buffers: ") + cudaGetErrorString(e)};
    }
  }
  if (rc.npix_cap < npix) {
    cudaFree(rc.accum);
    cudaFree(rc.wsum);
    cudaFree(rc.out);
    rc.accum = nullptr;
    rc.wsum = nullptr;
    rc.out = nullptr;
    rc.npix_cap = 0;
    check_cuda(cudaMalloc(&rc.accum, npix * sizeof(float4)), "accum");
    check_cuda(cudaMalloc(&rc.wsum, npix * sizeof(float)), "wsum");
    check_cuda(cudaMalloc(&rc.out, npix * 3 * sizeof(float)), "out");
    rc.npix_cap = npix;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (stats) {
    check_cuda(cudaEventCreate(&e0), "event");
    check_cuda(cudaEventCreate(&e1), "event");
    check_cuda(cudaEventRecord(e0, st), "event record");
  }
  uint32_t waves = 0, launches = 0;
  const char *pe = getenv("SNOG_PROFILE_KERNELS");
  const bool profile = stats && pe && pe[0] == '1';
  const bool count = stats && (profile || (p.flags & SNOG_RENDER_COUNT_TRAVERSAL));
  RenderProfile prof;
  WaveBuffers wave = rc.wb;   // the pool may be larger than this job's wave
  wave.wave_cap = cap;
  cudaError_t e = render_job(S.dev, jc, wave, rc.accum, rc.wsum, d_out ? d_out : rc.out, st, &waves,
                             &launches, profile ? &prof : nullptr, count);
  if (e == cudaSuccess && !d_out)
    e = cudaMemcpyAsync(h_out, rc.out, npix * 3 * sizeof(float), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaEventRecord(pool.done, st);
  if (e == cudaSuccess && !d_out) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    throw Error{SNOG_ECUDA, std::string("render: ") + cudaGetErrorString(e)};
  }
  if (stats) {
    check_cuda(cudaEventRecord(e1, st), "event record");
    check_cuda(cudaEventSynchronize(e1), "render sync");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    unsigned long long hs[7] = {0, 0, 0, 0, 0, 0, 0};
    uint32_t flags[4] = {0, 0, 0, 0};
    check_cuda(cudaMemcpy(hs, rc.wb.stats, sizeof hs, cudaMemcpyDeviceToHost), "stats");
    check_cuda(cudaMemcpy(flags, rc.wb.counters, 16, cudaMemcpyDeviceToHost), "flags");
    check_render_flags(flags[3]);
    stats->paths = total;
    stats->closest_rays = hs[0];
    stats->shadow_rays = hs[1];
    stats->device_ms = ms;
    stats->waves = waves;
    stats->kernel_launches = launches;
    stats->illum_calls = hs[6];
    if (profile) {
      check_cuda(prof.collect(), "profile events");
      stats->closest_ms = prof.ms[RenderProfile::CLOSEST];
      stats->shadow_ms = prof.ms[RenderProfile::SHADOW];
      stats->shade_ms = prof.ms[RenderProfile::SHADE];
      stats->other_ms = prof.ms[RenderProfile::OTHER];
      stats->closest_launches = prof.launches[RenderProfile::CLOSEST];
      stats->shadow_launches = prof.launches[RenderProfile::SHADOW];
    }
    if (count) {
      stats->closest_nodes = hs[2];
      stats->closest_tests = hs[3];
      stats->shadow_nodes = hs[4];
      stats->shadow_tests = hs[5];
    }
  }
}

}  // namespace snog

using namespace snog;

extern "C" {

int snog_render(SnogScene *scene, const SnogCamera *camera, const SnogRenderParams *params, float *out_rgb,
                SnogRenderStats *stats) {
  return guarded([&] {
    if (!scene || !camera || !params || !out_rgb) throw Error{SNOG_EINVAL, "null argument"};
    SceneImpl &S = *scene->impl;
    if (!S.on_device) throw Error{SNOG_EINVAL, "scene was built host-only"};
    std::lock_guard<std::mutex> lk(S.mu);
    render_into(S, *camera, *params, nullptr, out_rgb, nullptr, stats);
    return int(SNOG_OK);
  });
}

int snog_render_device(SnogScene *scene, const SnogCamera *camera, const SnogRenderParams *params,
                       float *d_out_rgb, void *stream, SnogRenderStats *stats) {
  return guarded([&] {
    if (!scene || !camera || !params || !d_out_rgb) throw Error{SNOG_EINVAL, "null argument"};
    SceneImpl &S = *scene->impl;
    if (!S.on_device) throw Error{SNOG_EINVAL, "scene was built host-only"};
    std::lock_guard<std::mutex> lk(S.mu);
    render_into(S, *camera, *params, d_out_rgb, nullptr, cudaStream_t(stream), stats);
    return int(SNOG_OK);
  });
}

int snog_render_window(SnogScene *scene, const SnogCamera *camera, const SnogRenderParams *params,
                       const SnogRenderWindow *window, float *out_rgb, SnogRenderStats *stats) {
  return guarded([&] {
    if (!scene || !camera || !params || !out_rgb) throw Error{SNOG_EINVAL, "null argument"};
    SceneImpl &S = *scene->impl;
    if (!S.on_device) throw Error{SNOG_EINVAL, "scene was built host-only"};
    std::lock_guard<std::mutex> lk(S.mu);
    render_into(S, *camera, *params, nullptr, out_rgb, nullptr, stats, window);
    return int(SNOG_OK);
  });
}

const char *snog_version(void) { return "snogray_b200 0.2 (sm_100a)"; }

const char *snog_last_error(void) { return g_last_error.c_str(); }

int snog_init(int device) {
  return guarded([&] {
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    check_cuda(cudaFree(nullptr), "context init");
    return int(SNOG_OK);
  });
}

int snog_scene_create(const SnogSceneDesc *desc, SnogScene **out) {
  return snog_scene_create_ex(desc, SNOG_OCTREE_AUTO, out);
}

int snog_scene_create_ex(const SnogSceneDesc *desc, uint32_t octree_mode, SnogScene **out) {
  return guarded([&] {
    if (!desc || !out) throw Error{SNOG_EINVAL, "null argument"};
    if ((octree_mode & 0xffu) > SNOG_OCTREE_DEVICE || (octree_mode >> 8) > 2u)
      throw Error{SNOG_EINVAL, "unknown octree mode"};
    *out = nullptr;
    SceneImpl *impl = build_scene(*desc, true, octree_mode);
    *out = new SnogScene{impl};
    return int(SNOG_OK);
  });
}

int snog_scene_build_host(const SnogSceneDesc *desc, SnogScene **out) {
  return guarded([&] {
    if (!desc || !out) throw Error{SNOG_EINVAL, "null argument"};
    *out = nullptr;
    SceneImpl *impl = build_scene(*desc, false);
    *out = new SnogScene{impl};
    return int(SNOG_OK);
  });
}

int snog_scene_destroy(SnogScene *scene) {
  return guarded([&] {
    if (!scene) return int(SNOG_OK);
    {
      std::lock_guard<std::mutex> lk(scene->impl->mu);
      cudaFree(scene->impl->trace_scratch);
      scene->impl->arena.release();
    }
    delete scene->impl;
    delete scene;
    return int(SNOG_OK);
  });
}

int snog_ply_load(const char *path, SnogPlyMesh *out) {
  return guarded([&] {
    if (!path || !out) throw Error{SNOG_EINVAL, "null argument"};
    std::memset(out, 0, sizeof *out);
    PlyMeshHost m = read_ply(path);
    auto copy = [](const auto &v) {
      using T = typename std::decay_t<decltype(v)>::value_type;
      T *p = static_cast<T *>(std::malloc(v.empty() ? 1 : v.size() * sizeof(T)));
      if (!p) throw std::bad_alloc();
      if (!v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
      return p;
    };
    SnogPlyMesh r{};
    r.n_vertices = uint32_t(m.vertices.size() / 3);
    r.n_triangles = uint32_t(m.triangles.size() / 3);
    r.vertices = copy(m.vertices);
    r.normals = m.normals.empty() ? nullptr : copy(m.normals);
    r.triangles = copy(m.triangles);
    *out = r;
    return int(SNOG_OK);
  });
}

int snog_ply_free(SnogPlyMesh *mesh) {
  return guarded([&] {
    if (!mesh) throw Error{SNOG_EINVAL, "null argument"};
    std::free(mesh->vertices);
    std::free(mesh->normals);
    std::free(mesh->triangles);
    std::memset(mesh, 0, sizeof *mesh);
    return int(SNOG_OK);
  });
}

int snog_scene_info(const SnogScene *scene, SnogSceneInfo *info) {
  return guarded([&] {
    if (!scene || !info) throw Error{SNOG_EINVAL, "null argument"};
    *info = scene->impl->info;
    return int(SNOG_OK);
  });
}

int snog_scene_octree(const SnogScene *scene, uint32_t *children, uint32_t *heads, int32_t *plist) {
  return guarded([&] {
    if (!scene) throw Error{SNOG_EINVAL, "null argument"};
    const OctreeArrays &o = host_octree(*scene->impl);
    if (children) std::memcpy(children, o.children.data(), o.children.size() * 4);
    if (heads) std::memcpy(heads, o.heads.data(), o.heads.size() * 4);
    if (plist) {
      for (size_t i = 0; i < o.plist.size(); i++) {
        uint32_t r = o.plist[i];
        plist[i] = r == PREF_END ? -1 : int32_t(r);
      }
    }
    return int(SNOG_OK);
  });
}

int snog_trace_device(SnogScene *scene, const float *d_rays, uint32_t n, uint32_t n_closest,
                      int32_t *d_prim, float *d_t, float *d_normal, void *stream) {
  return guarded([&] {
    if (!scene || (n && (!d_rays || !d_prim))) throw Error{SNOG_EINVAL, "null argument"};
    if (n_closest > n) throw Error{SNOG_EINVAL, "n_closest > n"};
    SceneImpl &S = *scene->impl;
    if (!S.on_device) throw Error{SNOG_EINVAL, "scene was built host-only"};
    if (!stack_class_for_depth(S.dev.max_depth))
      throw Error{SNOG_EINVAL, "octree deeper than the traversal kernels support (84 levels)"};
    std::lock_guard<std::mutex> lk(S.mu);
    if (!S.trace_scratch) check_cuda(cudaMalloc(&S.trace_scratch, 64), "trace scratch");
    check_cuda(cudaMemsetAsync(S.trace_scratch, 0, 64, cudaStream_t(stream)), "memset");
    check_cuda(launch_trace_batch(S.dev, d_rays, n, n_closest, d_prim, d_t, d_normal, nullptr,
                                  S.trace_scratch + 1, S.trace_scratch, cudaStream_t(stream), nullptr),
               "trace launch");
    return int(SNOG_OK);
  });
}

int snog_trace(SnogScene *scene, const float *rays, uint32_t n, uint32_t n_closest, int32_t *prim,
               float *t, float *normal, uint64_t *counters4) {
  return guarded([&] {
    if (!scene || (n && (!rays || !prim))) throw Error{SNOG_EINVAL, "null argument"};
    if (n_closest > n) throw Error{SNOG_EINVAL, "n_closest > n"};
    SceneImpl &S = *scene->impl;
    if (!S.on_device) throw Error{SNOG_EINVAL, "scene was built host-only"};
    if (!stack_class_for_depth(S.dev.max_depth))
      throw Error{SNOG_EINVAL, "octree deeper than the traversal kernels support (84 levels)"};
    std::lock_guard<std::mutex> lk(S.mu);
    if (n == 0) {
      if (counters4) std::memset(counters4, 0, 32);
      return int(SNOG_OK);
    }
    DevBuf d_rays(size_t(n) * 7 * 4), d_prim(size_t(n) * 4), d_t(t ? size_t(n) * 4 : 0),
        d_nrm(normal ? size_t(n) * 12 : 0), d_cnt(64);
    check_cuda(cudaMemcpy(d_rays.p, rays, size_t(n) * 7 * 4, cudaMemcpyHostToDevice), "rays H2D");
    check_cuda(cudaMemset(d_cnt.p, 0, 64), "memset");
    check_cuda(launch_trace_batch(S.dev, d_rays.as<float>(), n, n_closest, d_prim.as<int32_t>(),
                                  t ? d_t.as<float>() : nullptr, normal ? d_nrm.as<float>() : nullptr,
                                  d_cnt.as<unsigned long long>(), d_cnt.as<uint32_t>() + 8,
                                  d_cnt.as<uint32_t>() + 9, nullptr, nullptr),
               "trace launch");
    check_cuda(cudaMemcpy(prim, d_prim.p, size_t(n) * 4, cudaMemcpyDeviceToHost), "prim D2H");
    if (t) check_cuda(cudaMemcpy(t, d_t.p, size_t(n) * 4, cudaMemcpyDeviceToHost), "t D2H");
    if (normal) check_cuda(cudaMemcpy(normal, d_nrm.p, size_t(n) * 12, cudaMemcpyDeviceToHost), "n D2H");
    uint64_t cnt[8];
    check_cuda(cudaMemcpy(cnt, d_cnt.p, 64, cudaMemcpyDeviceToHost), "counters D2H");
    if (counters4) std::memcpy(counters4, cnt, 32);
    if (reinterpret_cast<uint32_t *>(cnt)[8])
      throw Error{SNOG_EINVAL, "traversal stack overflow (non-finite ray?)"};
    return int(SNOG_OK);
  });
}

}  // extern "C"
