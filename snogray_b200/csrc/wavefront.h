// wavefront.h -- host interface of the wavefront path tracer (wavefront.cu).

#ifndef SNOG_WAVEFRONT_H
#define SNOG_WAVEFRONT_H

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/snogray_b200.h"
#include "snog_common.h"

namespace snog {

// Constants of one render job, passed by value to every kernel.
struct JobConsts {
  uint32_t W, H;            // output image
  uint32_t PW, PH;          // render pattern incl. the filter margin
  int32_t PX, PY;           // film pixel of the pattern's top-left corner (-2, -2 for a whole image)
  int32_t OX, OY;           // film pixel of the output's top-left corner (0, 0 for a whole image)
  uint32_t FW, FH;          // film (camera) size, RenderMgr's width x height
  uint32_t S;               // samples per pixel
  uint32_t min_len, max_len, direct_samples;
  float min_trace, bg_alpha, max_trace, horizon;
  float cam_pos[3], cam_fwd[3], cam_right[3], cam_up[3];
  float tan_x, tan_y;
  uint32_t u_steps, v_steps, cells;
  uint32_t seed_lo, seed_hi;
  uint32_t integ;           // SNOG_INTEG_PATH or SNOG_INTEG_DIRECT
};

// Device buffers for one wave of paths (sized for wave_cap paths).
struct WaveBuffers {
  uint64_t wave_cap = 0;
  uint32_t n_lights = 0;                     // light samples per vertex the shadow queue is sized for
  float4 *thr = nullptr, *rad = nullptr;     // per path: throughput+rr, radiance+alpha
  uint32_t *pstate = nullptr;                // per path: length, flags, media stack
  float4 *q_o[2] = {nullptr, nullptr};       // ray queues: origin + t0
  float4 *q_d[2] = {nullptr, nullptr};       //             dir + t1
  uint32_t *q_path[2] = {nullptr, nullptr};
  uint32_t *hit_ref = nullptr;               // per queue slot
  float *hit_t = nullptr;
  float2 *jit = nullptr;                     // per path: camera jitter (splat reuses it)
  uint32_t *d_idx = nullptr;                 // direct-lighting list: queue index,
  float4 *d_thr = nullptr;                   //   throughput and path state of each lit vertex
  float4 *s_o = nullptr, *s_d = nullptr, *s_c = nullptr;   // shadow queue (c.w = path id)
  uint32_t *counters = nullptr;              // [0,1] ray queues, [2] shadow queue, [3] error flags,
                                             // [4,5] trace dispensers, [6] direct-lighting list
  unsigned long long *stats = nullptr;       // [0] closest rays, [1] shadow rays
  uint64_t bytes = 0;
  void *block = nullptr;
};

// Bytes needed per path of wave capacity when a vertex takes N_LIGHTS light
// samples (lights x direct_samples; the shadow queue holds two rays each).
uint64_t wave_bytes_per_path(uint32_t n_lights);
// Allocate / free (cudaMalloc of one block).
cudaError_t wave_alloc(WaveBuffers &wb, uint64_t cap, uint32_t n_lights);
void wave_free(WaveBuffers &wb);

// A job's constants.  WIN (may be null: the whole image with the filter
// margin, as snogray.lua:543-550 builds the pattern) sets the pattern and the
// output window of a partial render; check_window validates it.
JobConsts make_job(const DevScene &s, const SnogCamera &cam, const SnogRenderParams &p,
                   const SnogRenderWindow *win = nullptr);
void check_window(const SnogRenderParams &p, const SnogRenderWindow &win);
// Paths a job traces: pattern pixels x samples.
inline uint64_t job_total(const JobConsts &jc) { return uint64_t(jc.PW) * jc.PH * jc.S; }

// Optional per-kernel timing: CUDA events around every launch of the render,
// grouped by kernel kind, read back after the render completes.
struct RenderProfile {
  enum Kind { CLOSEST = 0, SHADOW = 1, SHADE = 2, OTHER = 3 };
  struct Mark { int kind; cudaEvent_t a, b; };
  Mark *marks = nullptr;
  uint32_t n = 0, cap = 0;
  double ms[4] = {0, 0, 0, 0};
  uint32_t launches[4] = {0, 0, 0, 0};
  cudaError_t begin(cudaStream_t st, int kind);   // records the start event
  cudaError_t end(cudaStream_t st);               // records the end event
  cudaError_t collect();                          // after sync: sums, frees events
  ~RenderProfile();
};

// Render a whole job on STREAM into accum (float4 colour*weight sums + float
// weight, W*H each; zeroed here) and resolve it to out_rgb (W*H*3 floats,
// device).  Paths are processed in waves of at most wb.wave_cap.  With PROF,
// every launch is bracketed by events; with COUNT (or PROF) the traversal
// counts its node visits and primitive tests into wb.stats[2..5].
// Mitchell-filter all TOTAL samples of a finished job (radiance + alpha and
// camera jitter per path, pattern-pixel-major) into its image: clears
// accum/wsum, gathers, resolves into out_rgb.
cudaError_t splat_job(const JobConsts &jc, const float4 *rad, const float2 *jit, uint64_t total, float4 *accum,
                      float *wsum, float *out_rgb, cudaStream_t st);

cudaError_t render_job(const DevScene &s, const JobConsts &jc, WaveBuffers &wb, float4 *accum,
                       float *wsum, float *out_rgb, cudaStream_t st, uint32_t *waves, uint32_t *launches,
                       RenderProfile *prof = nullptr, bool count = false);

}  // namespace snog

#endif
