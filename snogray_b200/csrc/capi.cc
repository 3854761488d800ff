// capi.cc -- the extern "C" entry points of include/snogray_b200.h for
// scenes and ray batches.  No exception crosses this boundary: every entry
// catches snog::Error / std::exception and returns a status, with the message
// kept per thread for snog_last_error().

#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "launch.h"
#include "scene.h"

struct SnogScene {
  snog::SceneImpl *impl;
};

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

// RAII device buffer for per-call temporaries.
struct DevBuf {
  void *p = nullptr;
  explicit DevBuf(size_t n) {
    if (n == 0) n = 16;
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw Error{e == cudaErrorMemoryAllocation ? SNOG_ENOMEM : SNOG_ECUDA,
                  std::string("cudaMalloc: ") + cudaGetErrorString(e)};
    }
  }
  ~DevBuf() { cudaFree(p); }
  template <class T>
  T *as() const { return static_cast<T *>(p); }
};

}  // namespace snog

using namespace snog;

extern "C" {

const char *snog_version(void) { return "snogray_b200 0.1 (sm_100a)"; }

const char *snog_last_error(void) { return g_last_error.c_str(); }

int snog_init(int device) {
  return guarded([&] {
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    check_cuda(cudaFree(nullptr), "context init");
    return int(SNOG_OK);
  });
}

int snog_scene_create(const SnogSceneDesc *desc, SnogScene **out) {
  return guarded([&] {
    if (!desc || !out) throw Error{SNOG_EINVAL, "null argument"};
    *out = nullptr;
    SceneImpl *impl = build_scene(*desc);
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
      scene->impl->arena.release();
    }
    delete scene->impl;
    delete scene;
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
    const SceneImpl &S = *scene->impl;
    const OctreeArrays &o = S.oct;
    if (children) std::memcpy(children, o.children.data(), o.children.size() * 4);
    if (heads) std::memcpy(heads, o.heads.data(), o.heads.size() * 4);
    if (plist) {
      for (size_t i = 0; i < o.plist.size(); i++) {
        uint32_t r = o.plist[i];
        if (r == PREF_END) {
          plist[i] = -1;
          continue;
        }
        uint32_t kind = r >> 30, idx = r & PREF_INDEX_MASK;
        plist[i] = int32_t(kind == PK_TRI ? idx : kind == PK_SPHERE ? S.n_tri + idx
                                                                     : S.n_tri + S.n_sph + idx);
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
    check_cuda(launch_trace_batch(S.dev, d_rays, n, n_closest, d_prim, d_t, d_normal, nullptr,
                                  nullptr, cudaStream_t(stream), nullptr),
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
                                  d_cnt.as<unsigned long long>(), d_cnt.as<uint32_t>() + 8, nullptr,
                                  nullptr),
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
