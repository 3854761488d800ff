// scene.h -- the library-side scene object behind the SnogScene handle.

#ifndef SNOG_SCENE_H
#define SNOG_SCENE_H

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/snogray_b200.h"
#include "octree_build.h"
#include "snog_common.h"
#include "wavefront.h"

namespace snog {

// Device working memory of the render calls on one scene, kept between
// calls and grown on demand.
struct RenderCache {
  WaveBuffers wb;
  float4 *accum = nullptr;     // W*H colour*weight sums (+ alpha)
  float *wsum = nullptr;       // W*H filter weight sums
  float *out = nullptr;        // W*H*3 resolved image (host-output calls)
  size_t npix_cap = 0;
  void release();
};

// Device allocations owned by one scene.
struct DeviceArena {
  std::vector<void *> blocks;
  uint64_t bytes = 0;
  void *alloc(size_t n);           // throws CudaError on failure
  void *upload(const void *src, size_t n);
  void release();
};

struct SceneImpl {
  std::mutex mu;
  int device = 0;
  OctreeArrays oct;                 // host copy (export, stats); for a device-built
                                    // tree only origin/size/statistics until exported
  bool oct_device = false;          // the octree was built on the device
  uint32_t oct_nodes = 0, oct_plist4 = 0, oct_plist_host = 0;
  DevScene dev{};                   // device view passed to kernels
  DeviceArena arena;
  SnogSceneInfo info{};
  uint32_t n_tri = 0, n_sph = 0, n_tpar = 0;
  // host copies needed by the host side of rendering
  float bbox_min[3], bbox_max[3];
  bool on_device = false;
  uint32_t *trace_scratch = nullptr;   // ray-batch dispenser counter (+ flags)
};

// Working memory of the plain renderer, one per device, shared by every
// scene: renders on any stream take it in turn, each waiting (on the device)
// for the event the previous one recorded after its last use.
struct RenderPool {
  std::mutex mu;
  RenderCache rc;
  cudaEvent_t done = nullptr;
};
RenderPool &render_pool(int device);

// Scenes with at least this many surfaces build their octree on the device
// unless the caller asks for the host builder.
constexpr size_t kDeviceOctreeMinSurfaces = 65536;

// Build and upload; throws snog::Error on failure.  OCTREE_MODE is one of
// SNOG_OCTREE_AUTO / _HOST / _DEVICE (a host-only scene always uses the host
// builder).
SceneImpl *build_scene(const SnogSceneDesc &desc, bool upload = true, uint32_t octree_mode = SNOG_OCTREE_AUTO);

// The octree in the host layout, downloaded on first use for a device-built
// tree.
const OctreeArrays &host_octree(SceneImpl &S);

// One job rendered on a streaming engine kept per device (engine_api.cc):
// the plain render calls use it for the direct integrator.  Synchronous;
// D_OUT (device) or H_OUT (host) receives the image.
void render_on_engine(SceneImpl &S, const SnogCamera &cam, const SnogRenderParams &p, float *d_out,
                      float *h_out, cudaStream_t st, SnogRenderStats *stats,
                      const SnogRenderWindow *win = nullptr);

struct Error {
  int code;
  std::string msg;
};

void check_cuda(int err, const char *what);   // throws Error{SNOG_ECUDA}

// RAII device buffer for per-call temporaries (at least 16 bytes, so a
// zero-length request still yields a valid pointer).
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
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  template <class T>
  T *as() const { return static_cast<T *>(p); }
};

// Error flags the render kernels raise in their flag word: bit 0, a
// traversal stack overflowed (a non-finite ray); bit 1, a path entered a
// fifth nested medium (the path state holds four; the reference's media
// list is unbounded, material/media.cc:76-118).  Throws for any set flag.
void check_render_flags(uint32_t flags);

}  // namespace snog

// The opaque handle of the C ABI.
struct SnogScene {
  snog::SceneImpl *impl;
};

#endif
