/* snogray_b200.h -- C ABI of the B200 path-tracing backend.
 *
 * This is the drop-in boundary for snogray's render path: plain C types,
 * host or device pointers with sizes, opaque handles, int status codes.  A
 * host program (the reference-shaped C++ classes in snogray_b200.hpp, the
 * Python package snogray_b200, or a binding generated from this header)
 * describes a scene once, then renders it or traces ray batches through it.
 *
 * Each entry point names the reference interface it replaces (paths are
 * relative to the snogray source tree).
 *
 * Errors: every function returns SNOG_OK (0) or a positive SNOG_E* code and
 * never throws or aborts; snog_last_error() gives a message for the calling
 * thread's most recent failure.  The reference reports the same conditions
 * with std::runtime_error (render/global-render-state.cc:73-74,90,
 * light/surface-light-sampler.cc:30-36).
 *
 * Threading: functions taking a SnogScene may be called from several threads
 * for different scenes; calls on one scene are serialised by the library.
 */
#ifndef SNOGRAY_B200_H
#define SNOGRAY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum SnogStatus {
  SNOG_OK = 0,
  SNOG_EINVAL = 1,      /* bad argument or scene description */
  SNOG_ENOMEM = 2,      /* device or host allocation failed / over budget */
  SNOG_ECUDA = 3,       /* CUDA runtime error */
  SNOG_ETIMEOUT = 4,    /* a bounded device wait ran out */
  SNOG_EBUSY = 5,       /* result not ready yet */
  SNOG_ENOTFOUND = 6,   /* unknown handle / job id */
  SNOG_ECANCELED = 7    /* job was cancelled */
};

/* Material kinds; the records mirror the reference constructors. */
enum SnogMaterialType {
  SNOG_LAMBERT = 0,        /* Lambert (color)                  material/lambert.h */
  SNOG_COOK_TORRANCE = 1,  /* CookTorrance (color, gloss, m, Ior) material/cook-torrance.h:27-30 */
  SNOG_MIRROR = 2,         /* Mirror (Ior, reflectance, color) material/mirror.h:47-49 */
  SNOG_GLASS = 3,          /* Glass (Medium (ior, absorb))     material/glass.h:27 */
  SNOG_GLOW = 4            /* Glow (color [, underlying])      material/glow.h:28-30 */
};

typedef struct SnogMaterial {
  uint32_t type;
  float color[3];      /* Lambert colour, CT diffuse, Mirror underlying, Glow emission */
  float gloss[3];      /* CT gloss colour, Mirror reflectance */
  float m;             /* CT rms microfacet slope */
  float ior_n, ior_k;  /* CT/Mirror Ior (n + ik); Glass medium ior (n) */
  float absorb[3];     /* Glass medium absorption */
  int32_t underlying;  /* Glow: index of an earlier material, or -1 */
} SnogMaterial;

typedef struct SnogSphere { float center[3]; float radius; uint32_t material; } SnogSphere;

/* Tripar (surface/tripar.h): corner v0, edges e1, e2; normal = e2 x e1. */
typedef struct SnogTripar {
  float v0[3], e1[3], e2[3];
  uint32_t parallelogram;
  uint32_t material;
} SnogTripar;

/* PointLight (light/point-light.h:32-47); angle >= 2*pi means omni. */
typedef struct SnogPointLight {
  float pos[3]; float color[3]; float angle; float fringe_angle; float dir[3];
} SnogPointLight;

/* FarLight (light/far-light.h:39-45). */
typedef struct SnogFarLight { float dir[3]; float angle; float color[3]; } SnogFarLight;

/* A scene, as the reference's SurfaceGroup holds it: one triangle mesh whose
 * parts are runs of equal tri_material (non-decreasing), spheres, tripars,
 * explicit lights and at most one lat-long envmap light (light/envmap-light.h,
 * texture/spheremap.h).  Surfaces whose material is a Glow become area
 * lights, as Primitive::add_light_samplers does (surface/primitive.cc:48-54).
 * Primitive ids: triangles [0,nt), spheres [nt,nt+ns), tripars after.
 * All arrays are host memory, read during snog_scene_create only. */
typedef struct SnogSceneDesc {
  uint32_t n_materials; const SnogMaterial *materials;
  uint32_t n_vertices; const float *vertices;          /* 3 floats each */
  uint32_t n_triangles; const uint32_t *triangles;     /* 3 indices each */
  const uint32_t *tri_material;
  uint32_t n_spheres; const SnogSphere *spheres;
  uint32_t n_tripars; const SnogTripar *tripars;
  uint32_t n_point_lights; const SnogPointLight *point_lights;
  uint32_t n_far_lights; const SnogFarLight *far_lights;
  uint32_t env_width, env_height;                      /* 0 = none; width = 2*height */
  const float *env_rgb;                                /* env_height rows of env_width RGB, top row first */
  float env_frame[9];                                  /* envmap light frame axes x, y, z */
  /* Optional vertex normals, 3 floats per vertex (NULL: none).  With them
   * triangles shade with the interpolated normal and the geometric normal
   * turned to agree with it (surface/mesh.cc:607-641, Mesh::add_normals
   * mesh.h:95-111). */
  const float *vertex_normals;
  /* Nonzero for a right-handed mesh: geometric normal e1 x e2 instead of
   * e2 x e1 (Mesh::left_handed, surface/mesh.cc:270; PLY meshes are
   * right-handed, load/mesh/load-ply.cc). */
  uint32_t mesh_right_handed;
} SnogSceneDesc;

/* Camera as the reference holds it after move/point/set_fov
 * (camera/camera.h:84-128, 231-242, 384-389). */
typedef struct SnogCamera {
  float pos[3], forward[3], right[3], up[3];
  float tan_half_fov_x, tan_half_fov_y;
} SnogCamera;

/* Render parameters: the reference's ValTable keys in brackets. */
typedef struct SnogRenderParams {
  uint32_t width, height;
  uint32_t spp;              /* [samples] */
  uint32_t min_path_len;     /* [surface_integ.min_path_len], default 3 */
  uint32_t max_path_len;     /* [surface_integ.max_path_len], default 25 */
  uint32_t direct_samples;   /* [surface_integ.direct_samples], default 1; with the
                                direct integrator [surface_integ.light_samples],
                                the reference's default 16 */
  float min_trace;           /* [min_trace], default 1e-3 */
  float bg_alpha;            /* [background_alpha], default 1 */
  uint64_t seed;             /* stream selector for the GPU's counter-based RNG */
  uint32_t integrator;       /* [surface_integ.type]: SNOG_INTEG_PATH or SNOG_INTEG_DIRECT */
  uint32_t flags;            /* SNOG_RENDER_* bits, 0 by default */
} SnogRenderParams;

/* SnogRenderParams::flags.  COUNT_TRAVERSAL: the path integrator's traversal
 * kernels count their node visits and primitive tests into SnogRenderStats
 * (closest_nodes ...), the counts behind the reference's
 * RenderStats::IsecStats (render/render-stats.h:30-52); it costs one
 * warp-reduced atomic per warp per launch. */
enum { SNOG_RENDER_COUNT_TRAVERSAL = 1 };

/* The pixels to render and the output window of a partial render, as the
 * reference's --limit option sets them up (snogray.lua:442-454, 543-550).
 * The film is params->width x params->height pixels (the RenderMgr's size,
 * render-mgr/render-mgr.h:39-40); film pixel (0, 0) is the top-left one.
 *   pattern: the film rectangle [pat_x, pat_x + pat_width) x
 *            [pat_y, pat_y + pat_height) whose pixels get samples
 *            (RenderPattern (left_x, top_y, width, height),
 *            render-mgr/render-pattern.h:105-108); it may extend beyond the
 *            film, as the filter margin does;
 *   output:  out_width x out_height pixels whose top-left is film pixel
 *            (out_x, out_y) (ImageSampledOutput's sample_base_x/y and size,
 *            snogray.lua:451-454).
 * Every sample adds to the output pixels its Mitchell filter reaches. */
typedef struct SnogRenderWindow {
  int32_t pat_x, pat_y;
  uint32_t pat_width, pat_height;
  int32_t out_x, out_y;
  uint32_t out_width, out_height;
} SnogRenderWindow;

/* Surface integrators: PathInteg (render/path-integ.cc:134-407) and
 * DirectInteg, direct lighting plus specular recursion with roulette beyond
 * depth 5 (render/direct-integ.h:29-104, render/recursive-integ.cc:28-212).
 * The direct integrator runs on the streaming engine (snog_render uses one
 * internally); a surface that both reflects and transmits specularly starts
 * a second ray, as the reference's recursion does.  min_path_len and
 * max_path_len do not apply to it. */
enum { SNOG_INTEG_PATH = 0, SNOG_INTEG_DIRECT = 1 };

typedef struct SnogSceneInfo {
  uint32_t n_nodes, n_plist, max_depth, n_leaf_nodes;
  uint32_t n_triangles, n_spheres, n_tripars, n_lights;
  uint64_t n_list_surfaces;       /* surface references in all node lists */
  float origin[3], size;          /* octree root cube */
  float bbox_min[3], bbox_max[3];
  float horizon;
  uint64_t device_bytes;
  double build_ms;
  /* 1 when the closest-hit traversal deals list entries to lanes in pairs
   * for this scene: random rays through it test more than 2.5 primitives per
   * node visit (long lists along rays); decided when the scene is created. */
  uint32_t pair_lists;
  uint32_t reserved;
} SnogSceneInfo;

typedef struct SnogRenderStats {
  uint64_t paths;            /* camera samples traced (pattern incl. filter margin) */
  uint64_t closest_rays;     /* closest-hit queries (Scene::intersect) */
  uint64_t shadow_rays;      /* any-hit queries (Scene::occludes) */
  double device_ms;          /* device time of the render, CUDA events */
  uint32_t waves;            /* wavefront batches the render was split into */
  uint32_t kernel_launches;
  /* Filled only when the environment variable SNOG_PROFILE_KERNELS=1: device
   * time of each kernel kind summed over its launches (CUDA events on the
   * render stream). */
  double closest_ms, shadow_ms, shade_ms, other_ms;
  uint32_t closest_launches, shadow_launches;
  /* Node visits and primitive tests of the closest-hit and shadow queries
   * (space_node_intersect_calls and surface_intersects_tests of the
   * reference's IsecStats, without its negative cache), filled by the path
   * integrator when params->flags has SNOG_RENDER_COUNT_TRAVERSAL or
   * SNOG_PROFILE_KERNELS=1. */
  uint64_t closest_nodes, closest_tests, shadow_nodes, shadow_tests;
  /* Vertices lit by direct illumination (the reference's
   * RenderStats::illum_calls), path integrator. */
  uint64_t illum_calls;
} SnogRenderStats;

typedef struct SnogScene SnogScene;

/* Library version string. */
const char *snog_version(void);

/* Message for the calling thread's last failing call ("" if none). */
const char *snog_last_error(void);

/* Select the CUDA device used by subsequent calls from this process. */
int snog_init(int device);

/* Build the acceleration structure and upload the scene.  Replaces
 * GlobalRenderState (render/global-render-state.cc:28-49) -> Scene
 * (render/scene.cc:26-44) -> Octree::Builder (space/octree-builder.cc:173-650),
 * Scene::light_samplers and EnvmapLight::Sampler's Hist2dDist
 * (light/envmap-light.cc:103-140, geometry/hist-2d-dist.cc:65-120). */
int snog_scene_create(const SnogSceneDesc *desc, SnogScene **out);

/* A triangle mesh read from a PLY file (ASCII, binary little- or
 * big-endian), with the reference's rules (load/mesh/load-ply.cc:41-214):
 * vertex x, y, z and optional nx, ny, nz properties, face vertex_indices
 * lists of exactly 3 entries (faces with fewer are skipped, more are an
 * error); a normal is kept only if some component exceeds 1e-15, and a later
 * normal after a skipped one is an error ("Normal consistency error"); a
 * face index goes through single precision as the reference's does.  The
 * mesh is right-handed (set SnogSceneDesc::mesh_right_handed).  Arrays are
 * owned by the library: release them with snog_ply_free. */
typedef struct SnogPlyMesh {
  uint32_t n_vertices;
  float *vertices;           /* 3 per vertex */
  float *normals;            /* 3 per vertex, or NULL */
  uint32_t n_triangles;
  uint32_t *triangles;       /* 3 per triangle */
} SnogPlyMesh;

/* Replaces load_ply_file (load/mesh/load-ply.cc:163-214). */
int snog_ply_load(const char *path, SnogPlyMesh *out);
int snog_ply_free(SnogPlyMesh *mesh);

/* Octree builders for snog_scene_create_ex.  Both give the same tree (node
 * arrays and list order identical to Octree::Builder's); the device builder
 * replays the root's growth on the host and places the surfaces in parallel
 * (octree_gpu.cu).  AUTO, snog_scene_create's choice, uses the device for
 * scenes of 65536 surfaces or more. */
enum { SNOG_OCTREE_AUTO = 0, SNOG_OCTREE_HOST = 1, SNOG_OCTREE_DEVICE = 2 };

/* How the closest-hit traversal deals a node's surface list to the lanes of
 * a warp, ORed into snog_scene_create_ex's OCTREE_MODE.  Hits, t values and
 * traversal counts are the same in every mode; only the speed differs.
 * PROBE (the default): pairs when random rays through the scene test more
 * than 2.5 primitives per node visit (SnogSceneInfo::pair_lists); SINGLE:
 * one entry per lane (up to 32 per round); PAIRED: two consecutive entries
 * per lane (up to 64 per round). */
enum { SNOG_LISTS_PROBE = 0, SNOG_LISTS_SINGLE = 1 << 8, SNOG_LISTS_PAIRED = 2 << 8 };

/* snog_scene_create with the octree builder chosen by OCTREE_MODE (one
 * SNOG_OCTREE_* value, optionally ORed with one SNOG_LISTS_* value); replaces
 * the same reference path (space/octree-builder.cc:173-650). */
int snog_scene_create_ex(const SnogSceneDesc *desc, uint32_t octree_mode, SnogScene **out);

/* Build the acceleration structure on the host only, without touching the
 * device (no CUDA context needed): the handle serves snog_scene_info and
 * snog_scene_octree, and is refused by the tracing and rendering calls. */
int snog_scene_build_host(const SnogSceneDesc *desc, SnogScene **out);

int snog_scene_destroy(SnogScene *scene);

/* Octree statistics and sizes; replaces Octree::stats (space/octree.cc:308-367). */
int snog_scene_info(const SnogScene *scene, SnogSceneInfo *info);

/* Copy the octree out: children (8*n_nodes), heads (n_nodes), and the packed
 * surface lists as primitive ids with -1 ending each list (n_plist).  This is
 * the reference's Octree::nodes / surface_ptrs (space/octree.h:111-121). */
int snog_scene_octree(const SnogScene *scene, uint32_t *children, uint32_t *heads,
                      int32_t *plist);

/* Closest-hit / any-hit queries for a ray batch in HOST memory, SoA:
 * rays = ox[n] oy[n] oz[n] dx[n] dy[n] dz[n] tmax[n], t0 = 0.  Rays [0,
 * n_closest) are closest-hit queries (Space::intersect, space/space.cc:72-84),
 * the rest any-hit queries (Space::intersects, space/space.cc:120-129).
 * prim[i] = id of the hit primitive or -1; for an any-hit query it is the
 * primitive that stopped the search.  t[i] = hit distance (closest queries),
 * normal = world-space geometric normal (3 per ray, may be NULL).  Counters
 * (may be NULL): node visits and primitive tests per query kind, in the
 * reference's RenderStats::IsecStats sense without the negative cache. */
int snog_trace(SnogScene *scene, const float *rays, uint32_t n, uint32_t n_closest,
               int32_t *prim, float *t, float *normal, uint64_t *counters4);

/* The same with DEVICE pointers, asynchronous on STREAM (a cudaStream_t,
 * NULL = default stream). */
int snog_trace_device(SnogScene *scene, const float *d_rays, uint32_t n, uint32_t n_closest,
                      int32_t *d_prim, float *d_t, float *d_normal, void *stream);

/* The path's shading functions at given sample parameters, for per-sample
 * comparison with the reference's (material/bsdf.h:158-168,
 * light/light-sampler.h): PROBES (HOST, 12 floats each: ray origin, t0 = 0,
 * unit direction, t1, BSDF parameter u v, light parameter u v).  For each
 * probe, the closest hit from the scene's default medium and there:
 * Bsdf::sample at the BSDF parameter (all flags); for every light sampler,
 * in the reference's order, its sample at the light parameter, Bsdf::eval
 * at that sample's direction and the sampler's eval at the BSDF sample's
 * direction.  EXTRA (HOST, may be NULL = 0.5): n x n_lights numbers for
 * samplers that draw one more (the sphere light's, sphere-light-sampler.cc:90).
 * OUT (HOST): n x (9 + 18 x n_lights) floats per probe: hit; BSDF sample val
 * r g b, pdf, dir x y z (normal frame), flags; then per light: sample val
 * r g b, pdf, dir x y z, dist, the extra number used; BSDF eval val r g b,
 * pdf; light eval val r g b, pdf, dist.  Evaluations whose sample had pdf 0
 * are left 0. */
int snog_sample_probe(SnogScene *scene, const float *probes, const float *extra, uint32_t n, float *out);

/* Render the whole image with the path integrator and the Mitchell-filtered
 * sampled output, into HOST memory out_rgb (height rows of width RGB floats,
 * top row first; the flushed values of ImageSampledOutput,
 * image/image-sampled-output.cc:79-123).  Replaces RenderMgr::render
 * (render-mgr/render-mgr.cc:50-74) with PathInteg (render/path-integ.cc:134-407).
 * The rendered pattern includes the filter margin, as snogray.lua:543-550. */
int snog_render(SnogScene *scene, const SnogCamera *camera, const SnogRenderParams *params,
                float *out_rgb, SnogRenderStats *stats);

/* The same with a DEVICE output buffer, asynchronous on STREAM; stats (may
 * be NULL) are filled after an internal synchronisation only if non-NULL. */
int snog_render_device(SnogScene *scene, const SnogCamera *camera,
                       const SnogRenderParams *params, float *d_out_rgb, void *stream,
                       SnogRenderStats *stats);

/* Render the pattern of WINDOW into its output window (HOST memory out_rgb:
 * window->out_height rows of window->out_width RGB floats, top row first).
 * Replaces RenderMgr::render (unsigned num_threads, RenderPattern &,
 * ImageSampledOutput &, Progress &, RenderStats &)
 * (render-mgr/render-mgr.h:45-50, render-mgr.cc:50-74) for partial renders;
 * WINDOW NULL is snog_render.  stats->paths counts the pattern's samples. */
int snog_render_window(SnogScene *scene, const SnogCamera *camera, const SnogRenderParams *params,
                       const SnogRenderWindow *window, float *out_rgb, SnogRenderStats *stats);

/* ---- Batched and served rendering ---------------------------------------
 * The streaming engine traces many jobs (scene, camera, size, samples) in one
 * persistent wavefront with path regeneration: paths of all admitted jobs
 * share the ray queues, finished paths are replaced at once by new camera
 * paths from a device work ring of (job, path range) items, and each
 * iteration's kernel sequence is a CUDA graph.  It replaces RenderMgr's
 * packet queue and render threads (render-mgr/render-mgr.cc:126-256) for many
 * renders at once; each job's image equals its plain render (snog_render) up
 * to float summation order. */
typedef struct SnogEngineConfig {
  uint32_t slots;             /* paths in flight (ray queue capacity) */
  uint32_t item_paths;        /* paths per work item (the scheduling grain) */
  uint32_t ring_items;        /* work ring capacity, items */
  uint32_t max_jobs;          /* jobs admitted at once */
  uint32_t max_lights;        /* light samples per vertex (lights x direct_samples) */
  uint32_t iters_per_launch;  /* iteration pairs per graph launch */
  uint32_t max_scenes;        /* scene table entries */
  uint32_t reserved;          /* 0 */
  uint64_t mem_budget;        /* device bytes for per-job buffers (admission) */
} SnogEngineConfig;

typedef struct SnogJobStats {
  double submit_ms, admit_ms, start_ms, finish_ms;   /* engine clock */
  uint64_t paths;                                    /* width x height x spp */
  int32_t status;                                    /* SNOG_OK, SNOG_EBUSY, SNOG_ECANCELED */
} SnogJobStats;

typedef struct SnogBatchStats {
  uint64_t paths, closest_rays, shadow_rays;
  double wall_ms;
  uint32_t kernel_launches;
  uint32_t iterations;        /* the rest only with SNOG_PROFILE_KERNELS=1 */
  double closest_ms, shadow_ms, shade_ms, other_ms;   /* device time per kernel kind */
} SnogBatchStats;

/* Defaults: 16M slots, 64K-path items, 16K-item ring, 4096 jobs, 4 light
 * samples, 4 iteration pairs per launch, 1024 scenes, 120 GB budget. */
int snog_engine_default_config(SnogEngineConfig *cfg);

/* A persistent engine: its queues (the bulk of its memory) and CUDA graph
 * stay allocated between renders.  STREAM is the caller's cudaStream_t or
 * NULL for a stream of its own; all its work is ordered on that stream. */
typedef struct SnogEngine SnogEngine;
int snog_engine_create(const SnogEngineConfig *cfg, void *stream, SnogEngine **out);
/* Render N_JOBS jobs to completion (as snog_render_batch). */
int snog_engine_render(SnogEngine *engine, SnogScene *const *scenes, const SnogCamera *cameras,
                       const SnogRenderParams *params, uint32_t n_jobs, float *const *outs, int outs_on_device,
                       SnogBatchStats *stats);
int snog_engine_destroy(SnogEngine *engine);

/* Pick slots (queue depth), item_paths (scheduling grain) and
 * iters_per_launch for a batch by timing candidates on a sample of it (each
 * job at 1 spp, at most SAMPLE_JOBS jobs evenly spaced, 0 = 64); the rest of
 * BASE is kept.  best_mpaths (may be NULL) receives the winner's rate on the
 * sample. */
int snog_engine_autotune(SnogScene *const *scenes, const SnogCamera *cameras, const SnogRenderParams *params,
                         uint32_t n_jobs, uint32_t sample_jobs, const SnogEngineConfig *base,
                         SnogEngineConfig *best, double *best_mpaths);

/* Render N_JOBS jobs together to completion.  outs[i] receives job i's image
 * (height x width RGB floats, top row first) in host memory, or device memory
 * if outs_on_device.  cfg may be NULL for defaults. */
int snog_render_batch(SnogScene *const *scenes, const SnogCamera *cameras, const SnogRenderParams *params,
                      uint32_t n_jobs, float *const *outs, int outs_on_device, const SnogEngineConfig *cfg,
                      SnogBatchStats *stats);

/* A render server: a background thread drives the engine; jobs submitted
 * while others run are admitted as job slots and the memory budget allow and
 * interleave with them (continuous batching).  No counterpart in the
 * reference (which renders one image per process). */
typedef struct SnogServer SnogServer;
int snog_server_create(const SnogEngineConfig *cfg, SnogServer **out);
/* Make SCENE resident in the server; jobs name it by the returned slot. */
int snog_server_add_scene(SnogServer *server, SnogScene *scene, uint32_t *slot);
/* Queue a job; its image goes to HOST_OUT (height x width RGB floats) when done. */
int snog_server_submit(SnogServer *server, uint32_t slot, const SnogCamera *camera,
                       const SnogRenderParams *params, float *host_out, uint64_t *job_id);
/* SNOG_OK when the job is finished (stats filled), SNOG_EBUSY while it is not,
 * SNOG_ECANCELED / SNOG_ENOTFOUND. */
int snog_server_poll(SnogServer *server, uint64_t job_id, SnogJobStats *stats);
/* Wait up to timeout_ms; SNOG_ETIMEOUT if the job is still running. */
int snog_server_wait(SnogServer *server, uint64_t job_id, uint32_t timeout_ms, SnogJobStats *stats);
int snog_server_cancel(SnogServer *server, uint64_t job_id);

/* Preemption and checkpoints of resident jobs; replaces the reference's
 * recovery of an interrupted render (--continue: image/recover-image.cc:32-88,
 * snogray.lua:466-486), at path granularity.
 * snog_server_pause stops starting a job's paths (those started finish) and
 * frees the device for other jobs; snog_server_resume continues it.  A job
 * stays SNOG_EBUSY while paused and keeps its per-job device memory. */
int snog_server_pause(SnogServer *server, uint64_t job_id);
int snog_server_resume(SnogServer *server, uint64_t job_id);
/* Write a paused job's finished paths (per-path radiance and film jitter,
 * with its camera and parameters) to PATH, once none is in flight (waits up
 * to TIMEOUT_MS: SNOG_ETIMEOUT).  The job stays paused. */
int snog_server_checkpoint(SnogServer *server, uint64_t job_id, const char *path, uint32_t timeout_ms);
/* Submit a job continuing the checkpoint in PATH on the scene in SLOT (the
 * scene it was taken on; SNOG_EINVAL otherwise): only the remaining paths
 * are traced, and the image is the one an uninterrupted render of the job
 * gives (path streams are keyed by job seed and path index). */
int snog_server_submit_resume(SnogServer *server, uint32_t slot, const char *path, float *host_out,
                              uint64_t *job_id);
/* Stops the server thread (finishing nothing further) and frees it. */
int snog_server_destroy(SnogServer *server);

/* The same render as snog_render_device, but the library allocates no device
 * memory: all working memory comes from one fixed 64 MiB device array that
 * the library holds (per GPU) until the process exits.  No counterpart in the
 * reference, which renders on the CPU.  For hosts that manage every byte of
 * device memory themselves, or cannot let cudaMalloc/cudaFree stall the
 * device mid-loop.  Limits: at most 1048576 output pixels, and a wave of the
 * scratch must hold one pixel's samples; larger jobs return SNOG_EINVAL.  The
 * first call on a device looks up the array's address and should come before
 * any stream capture.  The scene's device must be the current device
 * (SNOG_EINVAL otherwise).  Calls share the array: calls whose work overlaps
 * on the GPU race and must be ordered by the caller (e.g. one stream). */
int snog_render_device_noalloc(SnogScene *scene, const SnogCamera *camera,
                               const SnogRenderParams *params, float *d_out_rgb, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* SNOGRAY_B200_H */
