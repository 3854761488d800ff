// engine.h -- the streaming render engine: many jobs (scene, camera, image
// size, samples) traced together by one persistent wavefront with path
// regeneration, fed by a device work ring of (job, path-range) items.
//
// Per iteration (captured once in a CUDA graph, replayed K times per launch):
//   k_e_plan     one thread: how many queue slots are free, how many paths
//                the ring still offers; reserves that many path tickets
//   k_e_regen    new camera paths for the free slots, from the ring items
//   k_e_closest  octree closest hit for every queued ray (any scene)
//   k_e_shade    emission, direct lighting (shadow rays), BSDF continuation
//                and roulette; surviving paths go to the other queue,
//                finished ones write their radiance to their job's result
//   k_e_shadow   any-hit for the shadow rays; unoccluded ones add their
//                contribution to the path's next-queue entry or result
// The host admits jobs (device-memory budget), pushes their items into the
// ring round-robin across jobs (so jobs that arrive later interleave with
// running ones), launches the graph, and gathers-and-filters each job's
// samples into its image once all its paths are done.

#ifndef SNOG_ENGINE_H
#define SNOG_ENGINE_H

#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/snogray_b200.h"
#include "scene.h"
#include "wavefront.h"

namespace snog {

// Device-side job record.
struct EngineJobDev {
  JobConsts jc;
  uint32_t scene;          // index into the engine's scene table
  uint32_t canceled;       // set by the host: remaining paths retire unshaded
  unsigned long long total;
  float4 *result;          // per path: radiance rgb, alpha
  float2 *jit;             // per path: camera jitter in the pixel
};

// One work item: paths [begin, begin + count) of a job; `cum` is the number of
// paths of all items pushed before it (tickets are global over the ring).
struct WorkItem {
  uint32_t job, pad;
  unsigned long long begin, count, cum;
};

// Engine control block (device).
struct EngineCtl {
  uint32_t qcount[2];      // live rays in each queue
  uint32_t scount;         // shadow rays queued this iteration
  uint32_t err;            // traversal stack overflow
  uint32_t disp_closest, disp_shadow;
  uint32_t regen_n, regen_base;
  unsigned long long ticket;       // next path ticket
  unsigned long long regen_start;
  unsigned long long item_head;    // first ring item not fully consumed
  unsigned long long item_tail;    // one past the last pushed item (host-written)
  unsigned long long avail_end;    // cum + count of the last pushed item (host-written)
  unsigned long long rays_closest, rays_shadow, paths_started;
  // Spawn ring: second specular rays of the direct integrator waiting for a
  // queue slot.  Shade appends (spawn_n, up to spawn_room), plan publishes
  // them and hands regen the oldest (regen_spawn from regen_spawn_head).
  unsigned long long spawn_head, spawn_tail, regen_spawn_head;
  uint32_t spawn_n, spawn_room, regen_spawn;
  uint32_t dcount;          // vertices queued for direct lighting this iteration
};

struct EngineConfigHost {
  uint32_t slots = 1u << 24;       // paths in flight
  uint32_t item_paths = 1u << 16;  // paths per work item
  uint32_t ring_items = 1u << 14;
  uint32_t max_jobs = 4096;
  uint32_t max_lights = 4;         // light samples per vertex the shadow queue holds
  uint32_t iters_per_launch = 4;
  uint32_t max_scenes = 1024;      // scene table entries
  uint64_t mem_budget = 120ull << 30;
};

struct JobStatsHost {
  double submit_ms = 0, admit_ms = 0, start_ms = 0, finish_ms = 0;   // since engine start
  uint64_t paths = 0;
  int status = SNOG_EBUSY;         // SNOG_OK done, SNOG_EBUSY pending, SNOG_ECANCELED
};

// Device blocks for per-job buffers, kept for reuse instead of a cudaMalloc
// and cudaFree per job.  Sizes are rounded up to an eighth of their power of
// two, so a freed block serves any later request of the same class.
class BlockCache {
 public:
  ~BlockCache() { trim(); }
  void *get(size_t n);     // null if the device has no room even after trim()
  void put(void *p);
  void trim();             // free every cached block that is not in use
  uint64_t held() const { return held_; }

 private:
  static size_t round_up(size_t n);
  std::multimap<size_t, void *> free_;
  std::map<void *, size_t> size_of_;
  uint64_t held_ = 0;
};

class Engine {
 public:
  // STREAM: the caller's stream, or null for a stream of the engine's own.
  explicit Engine(const EngineConfigHost &cfg, cudaStream_t stream = nullptr);
  ~Engine();

  uint32_t add_scene(SceneImpl *scene);                 // returns slot; throws
  // Forget every scene (slots restart at 0).  Only while nothing is in flight.
  void reset_scenes();
  bool idle() const { return jobs_.empty(); }
  cudaStream_t stream() const { return stream_; }
  const EngineConfigHost &config() const { return cfg_; }
  // Per-kernel device time (CUDA events around each kernel instead of graph
  // launches) while profiling is on.
  struct Profile {
    double closest_ms = 0, shadow_ms = 0, shade_ms = 0, other_ms = 0;
    uint64_t iterations = 0;
  };
  void set_profile(bool on) { profile_on_ = on; }
  const Profile &profile() const { return prof_; }
  void clear_counters();
  // A job's finished paths [0, done): per-path radiance + alpha and film
  // jitter, with the job's camera and parameters -- what a resumed job needs.
  struct Checkpoint {
    SnogCamera cam{};
    SnogRenderParams params{};
    uint64_t total = 0, done = 0;
    uint64_t scene_check = 0;           // primitive and octree node counts of the scene
    std::vector<float4> result;
    std::vector<float2> jit;
  };
  // Queue a job; OUT is a host (on_device = false) or device image buffer.
  // SUBMIT_MS (engine clock) overrides the submission time recorded.
  // RESUME (optional): continue from a checkpoint of the same camera and
  // parameters on the same scene; its paths are not traced again.
  // WIN (may be null) renders a pattern into an output window (make_job);
  // such a job cannot be resumed from a checkpoint.
  uint64_t submit(uint32_t scene_slot, const SnogCamera &cam, const SnogRenderParams &p, float *out,
                  bool out_on_device, double submit_ms = -1, Checkpoint *resume = nullptr,
                  const SnogRenderWindow *win = nullptr);
  bool cancel(uint64_t job);
  // Stop (PAUSE) or restart pushing a job's work; paths already pushed finish.
  bool pause(uint64_t job, bool pause);
  bool is_paused(uint64_t job) const {
    auto it = jobs_.find(job);
    return it != jobs_.end() && it->second.paused;
  }
  // True when JOB is paused, admitted and has no path in flight.
  bool drained(uint64_t job) const;
  // Copy a drained job's finished paths out (throws if not drained).
  void checkpoint(uint64_t job, Checkpoint &out);
  // Scene fingerprint recorded in checkpoints.
  uint64_t scene_check(uint32_t scene_slot) const;
  // Drive the engine until every submitted job is finished (batch mode).
  void run_to_completion();
  // One scheduling round: admit, push items, one graph launch, completions.
  // Returns false when there is nothing in flight and nothing pending.
  bool step();
  JobStatsHost stats(uint64_t job);
  uint64_t rays_closest() const { return last_ctl_.rays_closest - base_closest_; }
  uint64_t rays_shadow() const { return last_ctl_.rays_shadow - base_shadow_; }
  double now_ms() const;
  uint32_t launches() const { return kernel_launches_; }

  std::mutex mu;   // guards the host job tables (server threads)

 private:
  struct HostJob {
    uint64_t id;
    uint32_t scene_slot, table_slot = ~0u;
    JobConsts jc;
    uint64_t total, pushed = 0;
    size_t npix;
    float *out;
    bool out_on_device;
    float4 *result = nullptr;
    float2 *jit = nullptr;
    float4 *accum = nullptr;
    float *wsum = nullptr;
    float *dev_out = nullptr;
    uint64_t bytes = 0;
    bool canceled = false, cancel_sent = false;
    bool paused = false;
    SnogCamera cam{};
    SnogRenderParams params{};
    std::unique_ptr<Checkpoint> resume;   // uploaded at admission, then dropped
    JobStatsHost st;
  };

  // Rays of job J finished / spawned as of the last step (a job is done
  // when every path and every spawned ray has finished).
  uint64_t rays_done(const HostJob &j) const { return done_host_[j.table_slot]; }
  uint64_t rays_spawned(const HostJob &j) const { return done_host_[cfg_.max_jobs + j.table_slot]; }
  void build_graph(bool direct, bool pair);
  void launch_iterations(bool direct, bool pair);
  void admit();
  void push_items();
  void release_job(HostJob &j);
  void *stage(const void *src, size_t n);   // copy into this step's pinned staging area

  EngineConfigHost cfg_;
  cudaStream_t stream_ = nullptr;
  bool own_stream_ = false;
  bool profile_on_ = false;
  Profile prof_;
  std::vector<cudaEvent_t> events_;
  // [with the direct integrator's shading][closest-hit rounds in pairs]
  cudaGraphExec_t graph_[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  int graph_stack_ = 0;
  // device buffers
  void *block_ = nullptr;
  float4 *q_o_[2], *q_d_[2], *q_thr_[2], *q_rad_[2];
  uint4 *q_meta_[2];
  uint32_t *hit_ref_;
  float *hit_t_;
  float4 *s_o_, *s_d_, *s_c_;
  unsigned long long *s_tgt_;
  uint32_t *d_idx_;                           // direct-lighting list: queue index of the vertex
  unsigned long long *d_tgt_;                 //   and the radiance its light adds to
  EngineCtl *ctl_;
  WorkItem *ring_;
  EngineJobDev *jobs_dev_;
  unsigned long long *job_done_;              // [max_jobs] finished rays, [max_jobs] spawned rays
  float4 *sp_o_, *sp_d_, *sp_thr_, *sp_rad_;   // spawn ring, sp_cap_ entries
  uint4 *sp_meta_;
  uint32_t sp_cap_ = 0;
  DevScene *scenes_dev_;
  uint32_t max_scenes_ = 0;
  // host mirrors
  BlockCache cache_;
  char *staging_ = nullptr;                    // pinned, reused every step
  size_t staging_cap_ = 0, staging_used_ = 0;
  EngineCtl *ctl_host_ = nullptr;              // pinned
  unsigned long long *done_host_ = nullptr;    // pinned
  EngineCtl last_ctl_{};
  std::vector<SceneImpl *> scenes_;
  std::vector<uint32_t> free_slots_;
  std::deque<uint64_t> pending_;
  std::vector<uint64_t> active_;
  std::map<uint64_t, HostJob> jobs_;
  std::map<uint64_t, JobStatsHost> finished_;
  uint64_t next_id_ = 1;
  uint64_t pushed_tail_ = 0, pushed_cum_ = 0;
  uint64_t budget_used_ = 0;
  uint32_t kernel_launches_ = 0;
  uint64_t base_closest_ = 0, base_shadow_ = 0;
  std::chrono::steady_clock::time_point t0_;
};

}  // namespace snog

#endif
