// engine_api.cc -- extern "C" entry points for batched and served rendering
// (include/snogray_b200.h): snog_render_batch drives the streaming engine to
// completion on the calling thread; a SnogServer runs it on a background
// thread and accepts jobs at any time.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"

namespace snog {
int set_error(int code, const std::string &msg);
extern thread_local std::string g_last_error;
}  // namespace snog

using namespace snog;

namespace snog {

void render_on_engine(SceneImpl &S, const SnogCamera &cam, const SnogRenderParams &p, float *d_out,
                      float *h_out, cudaStream_t st, SnogRenderStats *stats, const SnogRenderWindow *win) {
  static std::mutex mu;
  static std::map<int, std::unique_ptr<Engine>> engines;
  std::lock_guard<std::mutex> lk(mu);
  // Queue sized so the shadow queue (two rays of 56 bytes per light sample
  // per slot) stays near 2 GB.
  const uint32_t ls = std::max(1u, S.dev.n_lights) * std::max(1u, p.direct_samples);
  std::unique_ptr<Engine> &e = engines[S.device];
  if (!e || e->config().max_lights < ls) {
    e.reset();
    EngineConfigHost c;
    c.max_lights = std::max(4u, ls);
    uint64_t slots = (2ull << 30) / (112ull * c.max_lights);
    slots = std::min<uint64_t>(std::max<uint64_t>(slots, 1u << 16), 1u << 22);
    c.slots = uint32_t(slots);
    e.reset(new Engine(c));
  }
  check_cuda(cudaStreamSynchronize(st), "caller stream");   // the output buffer's earlier users
  e->reset_scenes();
  const uint32_t slot = e->add_scene(&S);
  e->clear_counters();
  const auto t0 = std::chrono::steady_clock::now();
  const uint64_t id = e->submit(slot, cam, p, d_out ? d_out : h_out, d_out != nullptr, -1, nullptr, win);
  e->run_to_completion();
  const JobStatsHost js = e->stats(id);
  if (js.status != SNOG_OK) throw Error{js.status, "render did not complete"};
  if (stats) {
    std::memset(stats, 0, sizeof *stats);
    stats->paths = win ? uint64_t(win->pat_width) * win->pat_height * p.spp
                       : uint64_t(p.width + 4) * (p.height + 4) * p.spp;
    stats->closest_rays = e->rays_closest();
    stats->shadow_rays = e->rays_shadow();
    stats->device_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    stats->waves = 1;
    stats->kernel_launches = e->launches();
  }
}

}  // namespace snog

namespace {

template <class F>
int api_call(F &&f) {
  try {
    g_last_error.clear();
    return f();
  } catch (const Error &e) {
    return set_error(e.code, e.msg);
  } catch (const std::bad_alloc &) {
    return set_error(SNOG_ENOMEM, "host allocation failed");
  } catch (const std::exception &e) {
    return set_error(SNOG_EINVAL, e.what());
  }
}

EngineConfigHost to_host(const SnogEngineConfig *c) {
  EngineConfigHost h;
  if (!c) return h;
  h.slots = c->slots;
  h.item_paths = c->item_paths;
  h.ring_items = c->ring_items;
  h.max_jobs = c->max_jobs;
  h.max_lights = c->max_lights;
  h.iters_per_launch = c->iters_per_launch;
  h.max_scenes = c->max_scenes;
  h.mem_budget = c->mem_budget;
  return h;
}

void to_abi(const EngineConfigHost &h, SnogEngineConfig *c) {
  c->slots = h.slots;
  c->item_paths = h.item_paths;
  c->ring_items = h.ring_items;
  c->max_jobs = h.max_jobs;
  c->max_lights = h.max_lights;
  c->iters_per_launch = h.iters_per_launch;
  c->max_scenes = h.max_scenes;
  c->reserved = 0;
  c->mem_budget = h.mem_budget;
}

void check_jobs(SnogScene *const *scenes, const SnogCamera *cameras, const SnogRenderParams *params,
                uint32_t n_jobs, float *const *outs) {
  if (n_jobs && (!scenes || !cameras || !params)) throw Error{SNOG_EINVAL, "null argument"};
  for (uint32_t i = 0; i < n_jobs; i++) {
    if (!scenes[i]) throw Error{SNOG_EINVAL, "null scene"};
    if (outs && !outs[i]) throw Error{SNOG_EINVAL, "null output buffer"};
  }
}

uint64_t job_paths(const SnogRenderParams &p) { return uint64_t(p.width + 4) * (p.height + 4) * p.spp; }

// Defaults sized to a batch: no more queue slots than the batch has paths,
// shadow queue for the most light samples any job takes, a job slot per job.
EngineConfigHost auto_config(SnogScene *const *scenes, const SnogRenderParams *params, uint32_t n_jobs) {
  EngineConfigHost h;
  uint64_t total = 0;
  for (uint32_t i = 0; i < n_jobs; i++) total += job_paths(params[i]);
  while (h.slots > 65536 && uint64_t(h.slots) / 2 >= total) h.slots /= 2;
  uint32_t ml = 1;
  std::unordered_map<SceneImpl *, int> distinct;
  for (uint32_t i = 0; i < n_jobs; i++) {
    ml = std::max(ml, scenes[i]->impl->dev.n_lights * std::max(1u, params[i].direct_samples));
    distinct[scenes[i]->impl] = 1;
  }
  h.max_lights = ml;
  h.max_jobs = std::max<uint32_t>(h.max_jobs, std::min<uint32_t>(n_jobs, 1u << 16));
  h.max_scenes = std::max<uint32_t>(h.max_scenes, uint32_t(distinct.size()));
  return h;
}

bool profile_requested() {
  const char *e = std::getenv("SNOG_PROFILE_KERNELS");
  return e && e[0] == '1';
}

// Render a batch to completion on an idle engine.
void render_on(Engine &eng, SnogScene *const *scenes, const SnogCamera *cameras, const SnogRenderParams *params,
               uint32_t n_jobs, float *const *outs, bool outs_on_device, SnogBatchStats *stats) {
  if (!eng.idle()) throw Error{SNOG_EBUSY, "engine has jobs in flight"};
  eng.reset_scenes();
  eng.clear_counters();
  eng.set_profile(profile_requested());
  std::unordered_map<SceneImpl *, uint32_t> slot_of;
  for (uint32_t i = 0; i < n_jobs; i++) {
    SceneImpl *si = scenes[i]->impl;
    if (!slot_of.count(si)) slot_of[si] = eng.add_scene(si);
  }
  const double t0 = eng.now_ms();
  uint64_t paths = 0;
  std::vector<uint64_t> ids(n_jobs);
  for (uint32_t i = 0; i < n_jobs; i++) {
    ids[i] = eng.submit(slot_of[scenes[i]->impl], cameras[i], params[i], outs ? outs[i] : nullptr,
                        outs ? outs_on_device : false);
    paths += uint64_t(params[i].width) * params[i].height * params[i].spp;
  }
  eng.run_to_completion();
  for (uint32_t i = 0; i < n_jobs; i++)
    if (eng.stats(ids[i]).status != SNOG_OK)
      throw Error{eng.stats(ids[i]).status, "job " + std::to_string(i) + " could not be rendered (device memory)"};
  if (stats) {
    std::memset(stats, 0, sizeof *stats);
    stats->paths = paths;
    stats->closest_rays = eng.rays_closest();
    stats->shadow_rays = eng.rays_shadow();
    stats->wall_ms = eng.now_ms() - t0;
    stats->kernel_launches = eng.launches();
    const Engine::Profile &pr = eng.profile();
    stats->iterations = uint32_t(pr.iterations);
    stats->closest_ms = pr.closest_ms;
    stats->shadow_ms = pr.shadow_ms;
    stats->shade_ms = pr.shade_ms;
    stats->other_ms = pr.other_ms;
  }
  eng.set_profile(false);
}

void fill(SnogJobStats *o, const JobStatsHost &s) {
  o->submit_ms = s.submit_ms;
  o->admit_ms = s.admit_ms;
  o->start_ms = s.start_ms;
  o->finish_ms = s.finish_ms;
  o->paths = s.paths;
  o->status = s.status;
}

}  // namespace

struct SnogEngine {
  std::unique_ptr<Engine> engine;
  std::mutex mu;
};

struct SnogServer {
  std::unique_ptr<Engine> engine;
  std::mutex engine_mu;                 // held while the engine is driven
  std::mutex mu;                        // inbox, results
  std::condition_variable cv_work, cv_done;
  std::thread worker;
  bool stop = false;
  std::string thread_error;
  struct Inbox {
    uint64_t id;
    uint32_t slot;
    SnogCamera cam;
    SnogRenderParams p;
    float *out;
    double submit_ms;
  };
  std::deque<Inbox> inbox;
  std::vector<uint64_t> cancels;
  std::vector<std::pair<uint64_t, bool>> pauses;      // (server id, pause) requests
  std::set<uint64_t> pause_requested;                  // server ids paused by the caller
  // Checkpoint requests, filled by the worker between scheduling rounds once
  // the job has no path in flight (API threads never take engine_mu while
  // the worker runs: it would re-take the mutex first every round).
  struct CkpReq {
    uint64_t job;
    bool done = false;
    std::string error;
    Engine::Checkpoint data;
  };
  std::vector<std::shared_ptr<CkpReq>> ckp_reqs;
  bool ckp_new = false;
  std::map<uint64_t, std::unique_ptr<Engine::Checkpoint>> resumes;   // inbox id -> checkpoint
  bool idle = false;                                   // last step found nothing to run
  std::unordered_map<uint64_t, uint64_t> to_engine;   // server id -> engine id
  std::map<uint64_t, JobStatsHost> results;           // finished
  std::map<uint64_t, std::string> failed;             // refused at admission
  uint64_t next_id = 1;

  void run() {
    for (;;) {
      std::vector<Inbox> take;
      std::vector<uint64_t> cancel_now;
      std::vector<std::pair<uint64_t, bool>> pause_now;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] {
          return stop || !inbox.empty() || !cancels.empty() || !pauses.empty() || ckp_new ||
                 (!to_engine.empty() && !idle);
        });
        ckp_new = false;
        if (stop) return;
        take.assign(inbox.begin(), inbox.end());
        inbox.clear();
        cancel_now.swap(cancels);
        pause_now.swap(pauses);
      }
      std::vector<std::pair<uint64_t, JobStatsHost>> finished;
      try {
        std::lock_guard<std::mutex> elk(engine_mu);
        for (auto &in : take) {
          try {
            std::unique_ptr<Engine::Checkpoint> ck;
            {
              std::lock_guard<std::mutex> lk(mu);
              auto r = resumes.find(in.id);
              if (r != resumes.end()) {
                ck = std::move(r->second);
                resumes.erase(r);
              }
            }
            uint64_t eid = engine->submit(in.slot, in.cam, in.p, in.out, false, in.submit_ms, ck.get());
            std::lock_guard<std::mutex> lk(mu);
            to_engine[in.id] = eid;
          } catch (const Error &e) {
            std::lock_guard<std::mutex> lk(mu);
            failed[in.id] = e.msg;
          }
        }
        for (uint64_t id : cancel_now) {
          std::lock_guard<std::mutex> lk(mu);
          auto it = to_engine.find(id);
          if (it != to_engine.end()) engine->cancel(it->second);
        }
        for (auto &pr : pause_now) {
          std::lock_guard<std::mutex> lk(mu);
          auto it = to_engine.find(pr.first);
          if (it != to_engine.end()) engine->pause(it->second, pr.second);
        }
        const bool ran = engine->step();
        std::lock_guard<std::mutex> lk(mu);
        idle = !ran;
        for (auto r = ckp_reqs.begin(); r != ckp_reqs.end();) {
          auto t = to_engine.find((*r)->job);
          if (t == to_engine.end()) {
            (*r)->error = "job is over; nothing to checkpoint";
          } else if (engine->drained(t->second)) {
            engine->checkpoint(t->second, (*r)->data);
          } else {
            ++r;
            continue;
          }
          (*r)->done = true;
          r = ckp_reqs.erase(r);
        }
        for (auto it = to_engine.begin(); it != to_engine.end();) {
          JobStatsHost s = engine->stats(it->second);
          if (s.status != SNOG_EBUSY) {
            finished.push_back({it->first, s});
            it = to_engine.erase(it);
          } else {
            ++it;
          }
        }
      } catch (const std::exception &e) {
        std::lock_guard<std::mutex> lk(mu);
        thread_error = e.what();
        for (auto &kv : to_engine) failed[kv.first] = thread_error;
        to_engine.clear();
      } catch (const Error &e) {
        std::lock_guard<std::mutex> lk(mu);
        thread_error = e.msg;
        for (auto &kv : to_engine) failed[kv.first] = thread_error;
        to_engine.clear();
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        for (auto &f : finished) results[f.first] = f.second;
      }
      cv_done.notify_all();
    }
  }
};

extern "C" {

int snog_engine_default_config(SnogEngineConfig *cfg) {
  return api_call([&] {
    if (!cfg) throw Error{SNOG_EINVAL, "null argument"};
    to_abi(EngineConfigHost{}, cfg);
    return int(SNOG_OK);
  });
}

int snog_engine_create(const SnogEngineConfig *cfg, void *stream, SnogEngine **out) {
  return api_call([&] {
    if (!out) throw Error{SNOG_EINVAL, "null argument"};
    std::unique_ptr<SnogEngine> e(new SnogEngine);
    e->engine.reset(new Engine(to_host(cfg), static_cast<cudaStream_t>(stream)));
    *out = e.release();
    return int(SNOG_OK);
  });
}

int snog_engine_render(SnogEngine *engine, SnogScene *const *scenes, const SnogCamera *cameras,
                       const SnogRenderParams *params, uint32_t n_jobs, float *const *outs, int outs_on_device,
                       SnogBatchStats *stats) {
  return api_call([&] {
    if (!engine) throw Error{SNOG_EINVAL, "null argument"};
    check_jobs(scenes, cameras, params, n_jobs, outs);
    if (!outs && n_jobs) throw Error{SNOG_EINVAL, "null argument"};
    std::lock_guard<std::mutex> lk(engine->mu);
    render_on(*engine->engine, scenes, cameras, params, n_jobs, outs, outs_on_device != 0, stats);
    return int(SNOG_OK);
  });
}

int snog_engine_destroy(SnogEngine *engine) {
  return api_call([&] {
    delete engine;
    return int(SNOG_OK);
  });
}

int snog_render_batch(SnogScene *const *scenes, const SnogCamera *cameras, const SnogRenderParams *params,
                      uint32_t n_jobs, float *const *outs, int outs_on_device, const SnogEngineConfig *cfg,
                      SnogBatchStats *stats) {
  return api_call([&] {
    check_jobs(scenes, cameras, params, n_jobs, outs);
    if (!outs && n_jobs) throw Error{SNOG_EINVAL, "null argument"};
    Engine eng(cfg ? to_host(cfg) : auto_config(scenes, params, n_jobs));
    render_on(eng, scenes, cameras, params, n_jobs, outs, outs_on_device != 0, stats);
    return int(SNOG_OK);
  });
}

// Coordinate descent over (slots, item_paths, iters_per_launch) on a sample
// of the batch: up to SAMPLE_JOBS jobs, evenly spaced, at reduced spp so the
// sample is a few queue-fulls of paths.  Results are discarded.
int snog_engine_autotune(SnogScene *const *scenes, const SnogCamera *cameras, const SnogRenderParams *params,
                         uint32_t n_jobs, uint32_t sample_jobs, const SnogEngineConfig *base,
                         SnogEngineConfig *best, double *best_mpaths) {
  return api_call([&] {
    check_jobs(scenes, cameras, params, n_jobs, nullptr);
    if (!best || n_jobs == 0) throw Error{SNOG_EINVAL, "null argument or empty batch"};
    if (sample_jobs == 0) sample_jobs = 64;
    const uint32_t ns = std::min(n_jobs, sample_jobs);
    std::vector<SnogScene *> sc(ns);
    std::vector<SnogCamera> cam(ns);
    std::vector<SnogRenderParams> prm(ns);
    uint64_t sample_paths = 0;
    for (uint32_t k = 0; k < ns; k++) {
      const uint32_t i = uint32_t(uint64_t(k) * n_jobs / ns);
      sc[k] = scenes[i];
      cam[k] = cameras[i];
      prm[k] = params[i];
      sample_paths += job_paths(prm[k]);
    }
    // Aim for ~128M sample paths: two fills of the largest queue tried, so
    // each queue size is timed through its steady state and its drain.
    const double target = 128.0 * (1 << 20);
    if (sample_paths > target) {
      const double f = target / double(sample_paths);
      sample_paths = 0;
      for (auto &p : prm) {
        p.spp = std::max(1u, uint32_t(p.spp * f));
        sample_paths += job_paths(p);
      }
    }
    EngineConfigHost cur = base ? to_host(base) : auto_config(scenes, params, n_jobs);
    {
      EngineConfigHost need = auto_config(scenes, params, n_jobs);
      cur.max_lights = std::max(cur.max_lights, need.max_lights);
      cur.max_scenes = std::max(cur.max_scenes, need.max_scenes);
      cur.max_jobs = std::max(cur.max_jobs, ns);
    }
    uint64_t paths = 0;
    for (auto &p : prm) paths += uint64_t(p.width) * p.height * p.spp;
    std::vector<std::vector<float>> imgs(ns);
    std::vector<float *> outs(ns);
    for (uint32_t k = 0; k < ns; k++) {
      imgs[k].resize(size_t(prm[k].width) * prm[k].height * 3);
      outs[k] = imgs[k].data();
    }
    auto measure = [&](const EngineConfigHost &h) {
      Engine eng(h);
      SnogBatchStats st;
      render_on(eng, sc.data(), cam.data(), prm.data(), ns, outs.data(), false, &st);   // warm (graph, caches)
      render_on(eng, sc.data(), cam.data(), prm.data(), ns, outs.data(), false, &st);
      return double(paths) / (st.wall_ms * 1e3);
    };
    double best_rate = measure(cur);
    auto try_values = [&](uint32_t EngineConfigHost::*field, std::initializer_list<uint32_t> values) {
      const uint32_t keep = cur.*field;
      uint32_t best_v = keep;
      for (uint32_t v : values) {
        if (v == keep) continue;
        EngineConfigHost h = cur;
        h.*field = v;
        if (field == &EngineConfigHost::slots && v / 2 > sample_paths) continue;
        double r;
        try {
          r = measure(h);
        } catch (const Error &e) {
          if (e.code == SNOG_ENOMEM) continue;
          throw;
        }
        if (r > best_rate * 1.02) {
          best_rate = r;
          best_v = v;
        }
      }
      cur.*field = best_v;
    };
    // Larger queues mean fewer, longer trace launches, each ending in one
    // tail where SMs run out of rays (the 1920x1080 64-spp terrain frame:
    // 16M slots 279.8 ms, 32M 273.6 ms, 64M 271.5 ms).
    try_values(&EngineConfigHost::slots, {1u << 21, 1u << 22, 1u << 23, 1u << 24, 1u << 25, 1u << 26});
    try_values(&EngineConfigHost::item_paths, {1u << 12, 1u << 14, 1u << 16, 1u << 18});
    try_values(&EngineConfigHost::iters_per_launch, {1u, 2u, 4u, 8u});
    to_abi(cur, best);
    if (best_mpaths) *best_mpaths = best_rate;
    return int(SNOG_OK);
  });
}

int snog_server_create(const SnogEngineConfig *cfg, SnogServer **out) {
  return api_call([&] {
    if (!out) throw Error{SNOG_EINVAL, "null argument"};
    std::unique_ptr<SnogServer> s(new SnogServer);
    s->engine.reset(new Engine(to_host(cfg)));
    SnogServer *raw = s.get();
    s->worker = std::thread([raw] { raw->run(); });
    *out = s.release();
    return int(SNOG_OK);
  });
}

int snog_server_add_scene(SnogServer *server, SnogScene *scene, uint32_t *slot) {
  return api_call([&] {
    if (!server || !scene || !slot) throw Error{SNOG_EINVAL, "null argument"};
    std::lock_guard<std::mutex> elk(server->engine_mu);
    *slot = server->engine->add_scene(scene->impl);
    return int(SNOG_OK);
  });
}

int snog_server_submit(SnogServer *server, uint32_t slot, const SnogCamera *camera,
                       const SnogRenderParams *params, float *host_out, uint64_t *job_id) {
  return api_call([&] {
    if (!server || !camera || !params || !host_out || !job_id) throw Error{SNOG_EINVAL, "null argument"};
    {
      std::lock_guard<std::mutex> lk(server->mu);
      if (!server->thread_error.empty()) throw Error{SNOG_ECUDA, "server stopped: " + server->thread_error};
      const uint64_t id = server->next_id++;
      server->inbox.push_back(SnogServer::Inbox{id, slot, *camera, *params, host_out,
                                                server->engine->now_ms()});
      *job_id = id;
    }
    server->cv_work.notify_one();
    return int(SNOG_OK);
  });
}

// Pause / resume requests go to the worker, which applies them between
// scheduling rounds.
static int server_pause(SnogServer *server, uint64_t job_id, bool on) {
  return api_call([&] {
    if (!server) throw Error{SNOG_EINVAL, "null argument"};
    {
      std::lock_guard<std::mutex> lk(server->mu);
      if (job_id == 0 || job_id >= server->next_id) throw Error{SNOG_ENOTFOUND, "unknown job"};
      if (server->results.count(job_id) || server->failed.count(job_id))
        throw Error{SNOG_EINVAL, "job is over"};
      if (on) server->pause_requested.insert(job_id);
      else server->pause_requested.erase(job_id);
      server->pauses.push_back({job_id, on});
    }
    server->cv_work.notify_one();
    return int(SNOG_OK);
  });
}

// Checkpoint file: "SNOGCKP1", the job's SnogCamera and SnogRenderParams,
// uint64 total paths, finished paths D, scene fingerprint, then D float4
// (radiance, alpha) and D float2 (film jitter), little-endian.
static void write_checkpoint(const char *path, const Engine::Checkpoint &c) {
  FILE *f = std::fopen(path, "wb");
  if (!f) throw Error{SNOG_EINVAL, std::string("cannot write ") + path};
  bool ok = std::fwrite("SNOGCKP1", 1, 8, f) == 8 && std::fwrite(&c.cam, sizeof c.cam, 1, f) == 1 &&
            std::fwrite(&c.params, sizeof c.params, 1, f) == 1 && std::fwrite(&c.total, 8, 1, f) == 1 &&
            std::fwrite(&c.done, 8, 1, f) == 1 && std::fwrite(&c.scene_check, 8, 1, f) == 1 &&
            std::fwrite(c.result.data(), sizeof(float4), c.done, f) == c.done &&
            std::fwrite(c.jit.data(), sizeof(float2), c.done, f) == c.done;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) throw Error{SNOG_EINVAL, std::string("writing ") + path + " failed"};
}

static Engine::Checkpoint read_checkpoint(const char *path) {
  FILE *f = std::fopen(path, "rb");
  if (!f) throw Error{SNOG_EINVAL, std::string("cannot read ") + path};
  Engine::Checkpoint c;
  char magic[8];
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "SNOGCKP1", 8) == 0 &&
            std::fread(&c.cam, sizeof c.cam, 1, f) == 1 && std::fread(&c.params, sizeof c.params, 1, f) == 1 &&
            std::fread(&c.total, 8, 1, f) == 1 && std::fread(&c.done, 8, 1, f) == 1 &&
            std::fread(&c.scene_check, 8, 1, f) == 1 && c.done <= c.total && c.done <= (1ull << 32);
  // The header is untrusted: its path counts must agree with the job's size
  // and with the bytes that follow before anything is sized from them.
  if (ok) ok = c.total == job_paths(c.params);
  if (ok) {
    const long here = std::ftell(f);
    ok = here >= 0 && std::fseek(f, 0, SEEK_END) == 0;
    const long end = ok ? std::ftell(f) : -1;
    ok = ok && end >= here && uint64_t(end - here) == c.done * (sizeof(float4) + sizeof(float2)) &&
         std::fseek(f, here, SEEK_SET) == 0;
  }
  if (ok) {
    c.result.resize(c.done);
    c.jit.resize(c.done);
    ok = std::fread(c.result.data(), sizeof(float4), c.done, f) == c.done &&
         std::fread(c.jit.data(), sizeof(float2), c.done, f) == c.done;
  }
  std::fclose(f);
  if (!ok) throw Error{SNOG_EINVAL, std::string(path) + " is not a complete snogray_b200 checkpoint"};
  return c;
}

static int server_status(SnogServer *server, uint64_t job_id, SnogJobStats *stats) {
  auto r = server->results.find(job_id);
  if (r != server->results.end()) {
    if (stats) fill(stats, r->second);
    if (r->second.status == SNOG_OK) return int(SNOG_OK);
    return set_error(r->second.status, r->second.status == SNOG_ECANCELED ? "job was cancelled"
                                                                          : "job could not be admitted (device memory)");
  }
  auto f = server->failed.find(job_id);
  if (f != server->failed.end()) return set_error(SNOG_EINVAL, f->second);
  if (job_id == 0 || job_id >= server->next_id) return set_error(SNOG_ENOTFOUND, "unknown job");
  return int(SNOG_EBUSY);
}

int snog_server_poll(SnogServer *server, uint64_t job_id, SnogJobStats *stats) {
  return api_call([&] {
    if (!server) throw Error{SNOG_EINVAL, "null argument"};
    std::lock_guard<std::mutex> lk(server->mu);
    return server_status(server, job_id, stats);
  });
}

int snog_server_wait(SnogServer *server, uint64_t job_id, uint32_t timeout_ms, SnogJobStats *stats) {
  return api_call([&] {
    if (!server) throw Error{SNOG_EINVAL, "null argument"};
    std::unique_lock<std::mutex> lk(server->mu);
    int rc = server_status(server, job_id, stats);
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms);
    while (rc == SNOG_EBUSY) {
      if (server->cv_done.wait_until(lk, deadline) == std::cv_status::timeout) {
        rc = server_status(server, job_id, stats);
        if (rc == SNOG_EBUSY) return set_error(SNOG_ETIMEOUT, "job still running");
        break;
      }
      rc = server_status(server, job_id, stats);
    }
    return rc;
  });
}

int snog_server_cancel(SnogServer *server, uint64_t job_id) {
  return api_call([&] {
    if (!server) throw Error{SNOG_EINVAL, "null argument"};
    {
      std::lock_guard<std::mutex> lk(server->mu);
      for (auto it = server->inbox.begin(); it != server->inbox.end(); ++it)
        if (it->id == job_id) {
          JobStatsHost s;
          s.status = SNOG_ECANCELED;
          s.submit_ms = it->submit_ms;
          server->results[job_id] = s;
          server->inbox.erase(it);
          return int(SNOG_OK);
        }
      if (job_id == 0 || job_id >= server->next_id) return set_error(SNOG_ENOTFOUND, "unknown job");
      if (server->results.count(job_id) || server->failed.count(job_id)) return int(SNOG_OK);   // already over
      // Running, or taken by the worker and about to be: the worker applies
      // cancels after the submissions it has taken.
      server->cancels.push_back(job_id);
    }
    server->cv_work.notify_one();
    return int(SNOG_OK);
  });
}

int snog_server_pause(SnogServer *server, uint64_t job_id) { return server_pause(server, job_id, true); }

int snog_server_resume(SnogServer *server, uint64_t job_id) { return server_pause(server, job_id, false); }

int snog_server_checkpoint(SnogServer *server, uint64_t job_id, const char *path, uint32_t timeout_ms) {
  return api_call([&] {
    if (!server || !path) throw Error{SNOG_EINVAL, "null argument"};
    auto req = std::make_shared<SnogServer::CkpReq>();
    req->job = job_id;
    {
      std::lock_guard<std::mutex> lk(server->mu);
      auto fin = server->results.find(job_id);
      if (fin != server->results.end())
        throw Error{SNOG_EINVAL, fin->second.status == SNOG_OK ? "job is finished; nothing to checkpoint"
                                                               : "job was cancelled or refused; nothing to checkpoint"};
      auto bad = server->failed.find(job_id);
      if (bad != server->failed.end()) throw Error{SNOG_EINVAL, "job failed: " + bad->second};
      if (job_id == 0 || job_id >= server->next_id) throw Error{SNOG_ENOTFOUND, "unknown job"};
      if (!server->pause_requested.count(job_id)) throw Error{SNOG_EINVAL, "job is not paused (snog_server_pause)"};
      server->ckp_reqs.push_back(req);
      server->ckp_new = true;
    }
    server->cv_work.notify_one();
    {
      std::unique_lock<std::mutex> lk(server->mu);
      const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms);
      while (!req->done) {
        if (server->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && !req->done) {
          auto &v = server->ckp_reqs;
          v.erase(std::remove(v.begin(), v.end(), req), v.end());
          throw Error{SNOG_ETIMEOUT, "job still has paths in flight"};
        }
      }
    }
    if (!req->error.empty()) throw Error{SNOG_EINVAL, req->error};
    write_checkpoint(path, req->data);
    return int(SNOG_OK);
  });
}

int snog_server_submit_resume(SnogServer *server, uint32_t slot, const char *path, float *host_out,
                              uint64_t *job_id) {
  return api_call([&] {
    if (!server || !path || !host_out || !job_id) throw Error{SNOG_EINVAL, "null argument"};
    std::unique_ptr<Engine::Checkpoint> c(new Engine::Checkpoint(read_checkpoint(path)));
    {
      std::lock_guard<std::mutex> lk(server->mu);
      if (!server->thread_error.empty()) throw Error{SNOG_ECUDA, "server stopped: " + server->thread_error};
      const uint64_t id = server->next_id++;
      server->inbox.push_back(SnogServer::Inbox{id, slot, c->cam, c->params, host_out, server->engine->now_ms()});
      server->resumes[id] = std::move(c);
      *job_id = id;
    }
    server->cv_work.notify_one();
    return int(SNOG_OK);
  });
}

int snog_server_destroy(SnogServer *server) {
  return api_call([&] {
    if (!server) return int(SNOG_OK);
    {
      std::lock_guard<std::mutex> lk(server->mu);
      server->stop = true;
    }
    server->cv_work.notify_all();
    if (server->worker.joinable()) server->worker.join();
    delete server;
    return int(SNOG_OK);
  });
}

}  // extern "C"
