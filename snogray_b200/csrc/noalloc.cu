// noalloc.cu -- snog_render_device_noalloc: the device-output render without
// any device allocation.
//
// Who needs it: hosts that own every byte of device memory through their own
// allocator or a fixed budget (an engine or server that pre-reserves the GPU
// and forbids libraries from calling cudaMalloc), and hosts that cannot
// tolerate cudaMalloc / cudaFree stalling the device -- cudaFree synchronises
// the whole device, which a render loop interleaving work on several streams
// cannot afford.  snog_render_device grows per-scene working memory with
// cudaMalloc on demand; this entry point takes all of it from one fixed,
// file-scope device array instead.
//
// The array (kScratchBytes, 64 MiB) is a static __device__ object: every GPU
// that loads the library holds it until the process exits.  It bounds what
// one call can do: at most kMaxPixels output pixels (the accumulator lives in
// it), and the rest is the wavefront's path state, so a call is refused if a
// wave could not hold even one pixel's samples.  Larger jobs must use
// snog_render_device.
//
// Host code cannot use the array's name as a device address (in host code it
// names a host-side stand-in), so its address is fetched per device with
// cudaGetSymbolAddress, with that device current, the first time a call runs
// on that device -- that first call should come before any stream capture.
// All calls share the array and it keeps the last call's contents; the render
// clears what must start at zero (accumulators, counters).  Calls whose work
// overlaps on the GPU (different streams, or different host threads) race on
// the array: callers must order them, e.g. on one stream.

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "launch.h"
#include "scene.h"
#include "wavefront.h"

namespace snog {

int set_error(int code, const std::string &msg);
extern thread_local std::string g_last_error;

namespace {

constexpr size_t kScratchBytes = size_t(64) << 20;
constexpr size_t kMaxPixels = size_t(1) << 20;     // accumulator: 20 bytes per pixel
constexpr size_t kAccumBytes = kMaxPixels * 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_addr_mu;
void *g_addr[kMaxDevices] = {nullptr};

// Device address of g_scratch on the current device (set up once per device).
void *scratch_address() {
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) throw Error{SNOG_EINVAL, "device index out of range"};
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    check_cuda(cudaGetSymbolAddress(&p, g_scratch), "cudaGetSymbolAddress(scratch)");
    g_addr[dev] = p;
  }
  return g_addr[dev];
}

// Lay the wavefront's buffers out in [base, base + bytes) for CAP paths (the
// same arrays wave_alloc allocates).
void carve_waves(WaveBuffers &wb, char *base, size_t bytes, uint64_t cap, uint32_t n_lights) {
  const uint64_t nl = n_lights ? n_lights : 1;
  size_t off = 0;
  auto take = [&](size_t b) {
    char *p = base + off;
    off += (b + 255) & ~size_t(255);
    return p;
  };
  wb = WaveBuffers{};
  wb.wave_cap = cap;
  wb.n_lights = n_lights;
  wb.thr = reinterpret_cast<float4 *>(take(16 * cap));
  wb.rad = reinterpret_cast<float4 *>(take(16 * cap));
  wb.pstate = reinterpret_cast<uint32_t *>(take(4 * cap));
  for (int k = 0; k < 2; k++) {
    wb.q_o[k] = reinterpret_cast<float4 *>(take(16 * cap));
    wb.q_d[k] = reinterpret_cast<float4 *>(take(16 * cap));
    wb.q_path[k] = reinterpret_cast<uint32_t *>(take(4 * cap));
  }
  wb.hit_ref = reinterpret_cast<uint32_t *>(take(4 * cap));
  wb.hit_t = reinterpret_cast<float *>(take(4 * cap));
  wb.jit = reinterpret_cast<float2 *>(take(8 * cap));
  wb.d_idx = reinterpret_cast<uint32_t *>(take(4 * cap));
  wb.d_thr = reinterpret_cast<float4 *>(take(16 * cap));
  wb.s_o = reinterpret_cast<float4 *>(take(16 * cap * 2 * nl));
  wb.s_d = reinterpret_cast<float4 *>(take(16 * cap * 2 * nl));
  wb.s_c = reinterpret_cast<float4 *>(take(16 * cap * 2 * nl));
  wb.counters = reinterpret_cast<uint32_t *>(take(64));
  wb.stats = reinterpret_cast<unsigned long long *>(take(64));
  if (off > bytes) throw Error{SNOG_EINVAL, "no-alloc scratch layout overflow"};
  wb.bytes = off;
  wb.block = nullptr;   // not owned: nothing to free
}

}  // namespace
}  // namespace snog

using namespace snog;

extern "C" int snog_render_device_noalloc(SnogScene *scene, const SnogCamera *camera,
                                          const SnogRenderParams *params, float *d_out_rgb, void *stream) {
  try {
    g_last_error.clear();
    if (!scene || !camera || !params || !d_out_rgb) throw Error{SNOG_EINVAL, "null argument"};
    SceneImpl &S = *scene->impl;
    if (!S.on_device) throw Error{SNOG_EINVAL, "scene was built host-only"};
    // The scratch address and the scene's arrays must belong to one device:
    // the scene's device has to be the current one.
    int cur = -1;
    check_cuda(cudaGetDevice(&cur), "cudaGetDevice");
    if (cur != S.device)
      throw Error{SNOG_EINVAL, "the scene was created on device " + std::to_string(S.device) +
                                   " but device " + std::to_string(cur) + " is current"};
    const SnogRenderParams &p = *params;
    if (p.integrator != SNOG_INTEG_PATH)
      throw Error{SNOG_EINVAL, "the no-alloc render runs the path integrator only"};
    if (p.width == 0 || p.height == 0 || p.spp == 0)
      throw Error{SNOG_EINVAL, "width, height and spp must be positive"};
    if (p.max_path_len > 255) throw Error{SNOG_EINVAL, "max_path_len must be <= 255"};
    const size_t npix = size_t(p.width) * p.height;
    if (npix > kMaxPixels)
      throw Error{SNOG_EINVAL, "image of " + std::to_string(npix) + " pixels exceeds the no-alloc limit of " +
                                   std::to_string(kMaxPixels) + " pixels; use snog_render_device"};
    if (!stack_class_for_depth(S.dev.max_depth))
      throw Error{SNOG_EINVAL, "octree deeper than the traversal kernels support (84 levels)"};
    // Path capacity of the wave region, in whole pixels' worth of samples.
    const size_t wave_bytes = kScratchBytes - kAccumBytes - 32 * 256;   // per-array alignment slack
    if (p.direct_samples > 64) throw Error{SNOG_EINVAL, "direct_samples must be <= 64"};
    // Shadow-queue entries a vertex may need: two per light sample.
    const uint32_t ls = (S.dev.n_lights ? S.dev.n_lights : 1u) * (p.direct_samples ? p.direct_samples : 1u);
    uint64_t cap = wave_bytes / wave_bytes_per_path(ls);
    cap = (cap / p.spp) * p.spp;
    if (cap < p.spp)
      throw Error{SNOG_EINVAL, std::to_string(p.spp) + " samples per pixel do not fit the no-alloc scratch "
                                   "for this scene's " + std::to_string(ls) +
                                   " light samples per vertex; use snog_render_device"};
    const uint64_t total = uint64_t(p.width + 4) * (p.height + 4) * p.spp;
    if (cap > total) cap = total;

    std::lock_guard<std::mutex> lk(S.mu);
    char *base = static_cast<char *>(scratch_address());
    float4 *accum = reinterpret_cast<float4 *>(base);
    float *wsum = reinterpret_cast<float *>(base + kMaxPixels * 16);
    WaveBuffers wb;
    carve_waves(wb, base + kAccumBytes, kScratchBytes - kAccumBytes, cap, ls);
    JobConsts jc = make_job(S.dev, *camera, p);
    uint32_t waves = 0, launches = 0;
    cudaError_t e = render_job(S.dev, jc, wb, accum, wsum, d_out_rgb, cudaStream_t(stream), &waves, &launches);
    if (e != cudaSuccess) throw Error{SNOG_ECUDA, std::string("render: ") + cudaGetErrorString(e)};
    return SNOG_OK;
  } catch (const Error &e) {
    return set_error(e.code, e.msg);
  } catch (const std::exception &e) {
    return set_error(SNOG_EINVAL, e.what());
  }
}
