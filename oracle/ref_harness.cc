// ref_harness.cc -- drives the snogray reference renderer through its own C++
// API, for golden data and CPU timing.
//
// TEST INFRASTRUCTURE ONLY.  Linked against the reference's sources compiled
// in place (oracle/Makefile); only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline / reference legs run it, as the checker or as the
// measured reference, never as part of the product.
//
// Modes:
//   octree SPEC OUT                 dump the reference octree (node array in
//                                   BFS order and the packed surface lists as
//                                   primitive ids) -- space/octree-builder.cc
//   trace SPEC RAYS OUT [threads]   closest-hit / any-hit queries through
//                                   Octree::for_each_possible_intersector
//                                   with the reference's own callbacks
//                                   (space/space.cc:36-129)
//   ply FILE OUT                    load a PLY mesh with load_ply_file
//                                   (load/mesh/load-ply.cc) and dump its
//                                   vertices, normals and triangles; a load
//                                   error is written to OUT as its message
//   render SPEC OUT.pfm [threads] [seed_skip] [spp] [row0] [rows] [repeat] [keep]
//                                   RenderMgr::render of the whole image
//                                   (render-mgr/render-mgr.cc:50-74), or of
//                                   a band of rows for a bounded CPU sample;
//                                   with KEEP nonzero, repetition r writes
//                                   OUT.pfm.r.pfm instead of overwriting OUT.pfm
//   camera SPEC IN OUT              Camera::eye_ray directions of the
//                                   spec's camera at IN's film locations
//                                   (camera/camera.h:322-389)
//   filter IN OUT                   the image output's default filter,
//                                   ImageMitchellFilt::val (x, y)
//                                   (image/image-mitchell-filt.h:45-65), at
//                                   IN's offsets (uint32 n, n x 2 floats)
//   samples SPEC PROBES OUT         per probe (a ray and four parameters),
//                                   Scene::intersect and make_intersect
//                                   from the default medium, then the hit's
//                                   Bsdf::sample / Bsdf::eval and every light
//                                   sampler's sample / eval at the given
//                                   parameters (render/intersect.h,
//                                   material/bsdf.h:158-168,
//                                   light/light-sampler.h)
//
// The reference keeps octree nodes, surface lists and camera fields private;
// this program (and only this program) reads them by compiling the
// reference headers with `private`/`protected` opened.  Nothing in the
// reference is modified.

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <deque>
#include <fstream>
#include <functional>
#include <iostream>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "scene_spec.h"

#define private public
#define protected public
#include "util/val-table.h"
#include "geometry/pos.h"
#include "geometry/vec.h"
#include "geometry/frame.h"
#include "color/color.h"
#include "surface/surface-group.h"
#include "surface/mesh.h"
// Mesh::Part and Mesh::Part::Triangle are defined in mesh.cc; compiling it
// here (instead of linking the archive's copy) makes them complete types so
// triangle pointers can be mapped back to triangle indices.
#include "surface/mesh.cc"
#include "surface/sphere.h"
#include "surface/tripar.h"
#include "material/lambert.h"
#include "material/cook-torrance.h"
#include "material/mirror.h"
#include "material/glass.h"
#include "material/glow.h"
#include "material/medium.h"
#include "light/point-light.h"
#include "light/far-light.h"
#include "light/envmap-light.h"
#include "texture/envmap.h"
#include "load/load-envmap.h"
#include "load/mesh/load-ply.h"
#include "image/image.h"
#include "image/image-sampled-output.h"
#include "image/image-mitchell-filt.h"
#include "camera/camera.h"
#include "render/global-render-state.h"
#include "render/render-context.h"
#include "render/render-stats.h"
#include "render/intersect.h"
#include "material/media.h"
#include "material/bsdf.h"
#include "light/light-sampler.h"
#include "render-mgr/render-mgr.h"
#include "render-mgr/render-pattern.h"
#include "space/octree.h"
#include "space/octree-node.h"
#include "util/progress.h"
#include "cli/build-info.h"
#undef private
#undef protected

using namespace snogray;

// The reference's CLI defines this table in a generated file.
namespace snogray { const ValTable build_info; }

namespace {

struct NullProgress : Progress {
  void set_start(int) override {}
  void set_size(unsigned) override {}
  void start() override {}
  void update(int) override {}
  void end() override {}
};

// A reference scene built from a spec, plus the map from the reference's
// renderable pointers back to primitive ids (triangles, then spheres, then
// tripars, in insertion order).
struct RefScene {
  snogspec::Scene spec;
  SurfaceGroup *root = nullptr;
  std::unordered_map<const void *, int32_t> prim_id;
  std::unique_ptr<GlobalRenderState> grs;
  ValTable params;
};

Ref<const Material> make_material(const snogspec::Scene &s, uint32_t i,
                                  std::vector<Ref<const Material>> &built) {
  const snogspec::MatRec &m = s.mats[i];
  Color col(m.color[0], m.color[1], m.color[2]);
  Color gloss(m.gloss[0], m.gloss[1], m.gloss[2]);
  switch (m.type) {
    case snogspec::MAT_LAMBERT:
      return new Lambert(col);
    case snogspec::MAT_COOK_TORRANCE:
      return new CookTorrance(col, gloss, m.m, Ior(m.ior_n, m.ior_k));
    case snogspec::MAT_MIRROR:
      return new Mirror(Ior(m.ior_n, m.ior_k), gloss, col);
    case snogspec::MAT_GLASS:
      return new Glass(Medium(m.ior_n, Color(m.absorb[0], m.absorb[1], m.absorb[2])));
    case snogspec::MAT_GLOW:
      if (m.underlying >= 0) return new Glow(col, built[m.underlying]);
      return new Glow(col);
  }
  throw std::runtime_error("unknown material type");
}

void build_scene(RefScene &rs, const std::string &spec_path) {
  rs.spec = snogspec::load(spec_path);
  const snogspec::Scene &s = rs.spec;
  const snogspec::SpecHeader &h = s.h;

  std::vector<Ref<const Material>> mats;
  for (uint32_t i = 0; i < h.n_materials; i++) mats.push_back(make_material(s, i, mats));

  rs.root = new SurfaceGroup;
  int32_t next_id = 0;

  if (h.n_triangles) {
    Mesh *mesh = new Mesh();
    std::vector<scoord_t> vcoords(s.verts.begin(), s.verts.end());
    mesh->add_vertices(vcoords);
    if (h.has_normals) mesh->add_normals(std::vector<sdist_t>(s.normals.begin(), s.normals.end()), 0);
    mesh->left_handed = h.right_handed == 0;
    uint32_t t = 0;
    while (t < h.n_triangles) {
      uint32_t mat = s.tri_mat[t], t_end = t;
      std::vector<Mesh::vert_index_t> idx;
      while (t_end < h.n_triangles && s.tri_mat[t_end] == mat) {
        for (int k = 0; k < 3; k++) idx.push_back(s.tris[3 * t_end + k]);
        t_end++;
      }
      Mesh::part_index_t part = mesh->add_part(mats[mat]);
      mesh->add_triangles(part, idx);
      t = t_end;
    }
    for (Mesh::Part *part : mesh->parts)
      for (auto &tri : part->triangles) rs.prim_id[&tri] = next_id++;
    rs.root->add(mesh);
  }
  for (const auto &sp : s.spheres) {
    Sphere *sph = new Sphere(mats[sp.mat], Pos(sp.center[0], sp.center[1], sp.center[2]), sp.radius);
    rs.prim_id[static_cast<const Surface::Renderable *>(sph)] = next_id++;
    rs.root->add(sph);
  }
  for (const auto &tp : s.tripars) {
    Tripar *tri = new Tripar(mats[tp.mat], Pos(tp.v0[0], tp.v0[1], tp.v0[2]),
                             Vec(tp.e1[0], tp.e1[1], tp.e1[2]), Vec(tp.e2[0], tp.e2[1], tp.e2[2]),
                             tp.parallelogram != 0);
    rs.prim_id[static_cast<const Surface::Renderable *>(tri)] = next_id++;
    rs.root->add(tri);
  }
  for (const auto &pl : s.plights) {
    Pos pos(pl.pos[0], pl.pos[1], pl.pos[2]);
    Color col(pl.color[0], pl.color[1], pl.color[2]);
    if (pl.angle >= 2 * PIf)
      rs.root->add(new PointLight(pos, col));
    else
      rs.root->add(new PointLight(pos, col, pl.angle, Vec(pl.dir[0], pl.dir[1], pl.dir[2]),
                                  pl.fringe_angle));
  }
  for (const auto &fl : s.flights)
    rs.root->add(new FarLight(Vec(fl.dir[0], fl.dir[1], fl.dir[2]), fl.angle,
                              Color(fl.color[0], fl.color[1], fl.color[2])));
  if (h.env_w) {
    Ref<Image> img = new Image(h.env_w, h.env_h);
    for (uint32_t y = 0; y < h.env_h; y++)
      for (uint32_t x = 0; x < h.env_w; x++) {
        const float *p = &s.env[(size_t(y) * h.env_w + x) * 3];
        (*img)(x, y) = Color(p[0], p[1], p[2]);
      }
    Ref<Envmap> em = make_envmap(img, "latlong");
    const float *f = h.env_frame;
    Frame frame(Vec(f[0], f[1], f[2]), Vec(f[3], f[4], f[5]), Vec(f[6], f[7], f[8]));
    rs.root->add(new EnvmapLight(em, frame));
  }

  rs.params.set("samples", unsigned(h.spp));
  if (h.integrator == 1) {
    // DirectInteg: direct lighting with light_samples per light, specular
    // recursion (render/direct-integ.h:77-86)
    rs.params.set("surface_integ.type", std::string("direct"));
    rs.params.set("surface_integ.light_samples", unsigned(h.direct_samples));
  } else {
    rs.params.set("surface_integ.type", std::string("path"));
    rs.params.set("surface_integ.min_path_len", unsigned(h.min_path_len));
    rs.params.set("surface_integ.max_path_len", unsigned(h.max_path_len));
    rs.params.set("surface_integ.direct_samples", unsigned(h.direct_samples));
  }
  rs.params.set("min_trace", float(h.min_trace));
  rs.params.set("background_alpha", float(h.bg_alpha));
  rs.grs.reset(new GlobalRenderState(*rs.root, rs.params));
}

const Octree &octree_of(const RefScene &rs) {
  const Octree *oct = dynamic_cast<const Octree *>(&*rs.grs->scene.space);
  if (!oct) throw std::runtime_error("scene space is not an octree");
  return *oct;
}

int mode_octree(const std::string &spec, const std::string &out) {
  RefScene rs;
  build_scene(rs, spec);
  const Octree &oct = octree_of(rs);
  FILE *f = fopen(out.c_str(), "wb");
  float hdr_f[4] = {oct.origin.x, oct.origin.y, oct.origin.z, oct.size};
  uint32_t n_nodes = oct.nodes.size(), n_list = oct.surface_ptrs.size();
  fwrite(hdr_f, 4, 4, f);
  fwrite(&n_nodes, 4, 1, f);
  fwrite(&n_list, 4, 1, f);
  for (const auto &n : oct.nodes) {
    fwrite(n.child_node_indices, 4, 8, f);
    fwrite(&n.surface_ptrs_head_index, 4, 1, f);
  }
  for (const Surface::Renderable *p : oct.surface_ptrs) {
    int32_t id = p ? rs.prim_id.at(p) : -1;
    fwrite(&id, 4, 1, f);
  }
  fclose(f);
  Octree::Stats st = oct.stats();
  printf("{\"nodes\": %lu, \"leaf_nodes\": %lu, \"surfaces\": %lu, \"dup_surfaces\": %lu, "
         "\"max_depth\": %u, \"avg_depth\": %.6f}\n",
         st.num_nodes, st.num_leaf_nodes, st.num_surfaces, st.num_dup_surfaces, st.max_depth,
         st.avg_depth);
  return 0;
}

// The reference's closest-hit callback (space/space.cc:36-63), recording the
// renderable that produced the surviving hit.
struct ClosestCb : Space::IntersectCallback {
  ClosestCb(Ray &r, RenderContext &c) : ray(r), context(c) {}
  bool operator()(const Surface::Renderable *surf) override {
    const Surface::Renderable::IsecInfo *ii = surf->intersect(ray, context);
    if (ii) {
      closest = ii;
      closest_surf = surf;
      return true;
    }
    return false;
  }
  Ray &ray;
  RenderContext &context;
  const Surface::Renderable::IsecInfo *closest = nullptr;
  const Surface::Renderable *closest_surf = nullptr;
};

// The reference's any-hit callback (space/space.cc:90-115), recording the
// renderable that stopped the search.
struct AnyCb : Space::IntersectCallback {
  AnyCb(const Ray &r, RenderContext &c) : ray(r), context(c) {}
  bool operator()(const Surface::Renderable *surf) override {
    bool hit = surf->intersects(ray, context);
    if (hit) {
      hit_surf = surf;
      stop_iteration();
    }
    return hit;
  }
  const Ray &ray;
  RenderContext &context;
  const Surface::Renderable *hit_surf = nullptr;
};

int mode_trace(const std::string &spec, const std::string &rays_path, const std::string &out,
               unsigned threads) {
  RefScene rs;
  build_scene(rs, spec);
  const Octree &oct = octree_of(rs);
  snogspec::RayBatch rb = snogspec::load_rays(rays_path);
  const uint32_t n = rb.n;
  std::vector<int32_t> prim(n, -1);
  std::vector<float> tout(n, 0.f), nrm(size_t(n) * 3, 0.f);
  std::vector<RenderStats> stats(threads);
  std::atomic<uint32_t> next(0);
  const uint32_t chunk = 4096;

  auto worker = [&](unsigned tid) {
    RenderContext ctx(*rs.grs);
    for (;;) {
      uint32_t b = next.fetch_add(chunk);
      if (b >= n) break;
      uint32_t e = std::min(n, b + chunk);
      for (uint32_t i = b; i < e; i++) {
        Ray ray(Pos(rb.ox()[i], rb.oy()[i], rb.oz()[i]), Vec(rb.dx()[i], rb.dy()[i], rb.dz()[i]),
                rb.tmax()[i]);
        if (i < rb.n_closest) {
          ClosestCb cb(ray, ctx);
          oct.for_each_possible_intersector(ray, cb, ctx, ctx.stats.intersect);
          if (cb.closest_surf) {
            prim[i] = rs.prim_id.at(cb.closest_surf);
            tout[i] = ray.t1;
            Vec nv = cb.closest->normal();
            nrm[3 * size_t(i)] = nv.x;
            nrm[3 * size_t(i) + 1] = nv.y;
            nrm[3 * size_t(i) + 2] = nv.z;
          }
          ctx.mempool.reset();
        } else {
          AnyCb cb(ray, ctx);
          oct.for_each_possible_intersector(ray, cb, ctx, ctx.stats.shadow);
          if (cb.hit_surf) prim[i] = rs.prim_id.at(cb.hit_surf);
        }
      }
    }
    stats[tid] += ctx.stats;
  };

  auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < threads; t++) pool.emplace_back(worker, t);
  for (auto &th : pool) th.join();
  double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

  RenderStats tot;
  for (auto &s : stats) tot += s;
  FILE *f = fopen(out.c_str(), "wb");
  fwrite(prim.data(), 4, n, f);
  fwrite(tout.data(), 4, n, f);
  fwrite(nrm.data(), 4, size_t(n) * 3, f);
  const RenderStats::IsecStats *is[2] = {&tot.intersect, &tot.shadow};
  for (auto *s : is) {
    unsigned long long v[5] = {s->surface_intersects_tests, s->surface_intersects_hits,
                               s->neg_cache_hits, s->neg_cache_collisions,
                               s->space_node_intersect_calls};
    fwrite(v, 8, 5, f);
  }
  fclose(f);
  printf("{\"rays\": %u, \"seconds\": %.6f, \"threads\": %u, \"mrays_per_s\": %.4f}\n", n, secs,
         threads, n / secs * 1e-6);
  return 0;
}

// The spec's pinhole camera, set field by field (camera/camera.h:322-389).
Camera camera_of(const snogspec::SpecHeader &h) {
  Camera camera;
  camera.pos = Pos(h.cam_pos[0], h.cam_pos[1], h.cam_pos[2]);
  camera.forward = Vec(h.cam_forward[0], h.cam_forward[1], h.cam_forward[2]);
  camera.right = Vec(h.cam_right[0], h.cam_right[1], h.cam_right[2]);
  camera.up = Vec(h.cam_up[0], h.cam_up[1], h.cam_up[2]);
  camera.tan_half_fov_x = h.tan_half_fov_x;
  camera.tan_half_fov_y = h.tan_half_fov_y;
  return camera;
}

// Film locations (uint32 n, n x 2 floats u v) to Camera::eye_ray directions
// (n x 3 floats; the direction is eye_vec, not normalised).
int mode_camera(const std::string &spec, const std::string &in_path, const std::string &out) {
  RefScene rs;
  build_scene(rs, spec);
  const Camera camera = camera_of(rs.spec.h);
  std::ifstream in(in_path, std::ios::binary);
  uint32_t n = 0;
  in.read(reinterpret_cast<char *>(&n), 4);
  std::vector<float> uv(size_t(n) * 2), d(size_t(n) * 3);
  in.read(reinterpret_cast<char *>(uv.data()), std::streamsize(uv.size() * 4));
  if (!in) throw std::runtime_error("short film-location file");
  for (uint32_t i = 0; i < n; i++) {
    const Ray r = camera.eye_ray(UV(uv[2 * size_t(i)], uv[2 * size_t(i) + 1]), 1.f);
    d[3 * size_t(i)] = r.dir.x;
    d[3 * size_t(i) + 1] = r.dir.y;
    d[3 * size_t(i) + 2] = r.dir.z;
  }
  FILE *f = fopen(out.c_str(), "wb");
  if (!f) throw std::runtime_error("cannot write " + out);
  fwrite(d.data(), 4, d.size(), f);
  fclose(f);
  printf("{\"rays\": %u}\n", n);
  return 0;
}

int mode_render(const std::string &spec, const std::string &out, unsigned threads,
                unsigned seed_skip, unsigned spp_override, int row0, int rows, unsigned repeat,
                bool keep) {
  RefScene rs;
  snogspec::Scene peek = snogspec::load(spec);
  (void)peek;
  build_scene(rs, spec);
  if (spp_override) {
    rs.params.set("samples", spp_override);
    rs.grs.reset(new GlobalRenderState(*rs.root, rs.params));
  }
  const snogspec::SpecHeader &h = rs.spec.h;

  // Each RenderContext draws the next seed from a process-wide counter
  // (render/render-context.cc:27-40); skipping SEED_SKIP contexts gives an
  // independent, reproducible stream for a single-threaded render.
  for (unsigned i = 0; i < seed_skip; i++) RenderContext skip(*rs.grs);

  Camera camera = camera_of(h);

  unsigned w = h.width, hgt = h.height;
  int y0 = 0, nrows = int(hgt);
  if (rows > 0) {
    y0 = row0;
    nrows = rows;
  }
  // Each repetition is an independent render of the same job into a fresh
  // output; the scene (and its octree) is built once.
  for (unsigned rep = 0; rep < repeat; rep++) {
    ValTable out_params;
    ImageSampledOutput output(keep ? out + "." + std::to_string(rep) + ".pfm" : out, w, hgt, out_params);
    int xm = int(output.filter_x_radius()), ym = int(output.filter_y_radius());
    RenderPattern pattern(0 - xm, y0 - ym, int(w) + 2 * xm, nrows + 2 * ym);
    RenderMgr mgr(*rs.grs, camera, w, hgt);
    NullProgress prog;
    RenderStats stats;
    auto t0 = std::chrono::steady_clock::now();
    mgr.render(threads, pattern, output, prog, stats);
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    unsigned spp = rs.grs->num_samples;
    double paths = double(w) * nrows * spp;
    printf("{\"rep\": %u, \"seconds\": %.6f, \"threads\": %u, \"spp\": %u, \"rows\": %d, \"paths\": %.0f, "
           "\"mpaths_per_s\": %.6f, \"scene_intersect_calls\": %llu, \"scene_shadow_tests\": %llu, "
           "\"mrays_per_s\": %.6f, \"node_calls\": %llu, \"shadow_node_calls\": %llu, "
           "\"surface_tests\": %llu, \"shadow_surface_tests\": %llu, \"neg_cache_hits\": %llu, "
           "\"shadow_neg_cache_hits\": %llu}\n",
           rep, secs, threads, spp, nrows, paths, paths / secs * 1e-6, stats.scene_intersect_calls,
           stats.scene_shadow_tests,
           double(stats.scene_intersect_calls + stats.scene_shadow_tests) / secs * 1e-6,
           stats.intersect.space_node_intersect_calls, stats.shadow.space_node_intersect_calls,
           stats.intersect.surface_intersects_tests, stats.shadow.surface_intersects_tests,
           stats.intersect.neg_cache_hits, stats.shadow.neg_cache_hits);
    fflush(stdout);
  }
  return 0;
}

// OUT: "OK" or "ERR" + message line; for OK then uint32 n_vertices,
// n_normals, n_triangles and the float / uint32 arrays.
// Probe file: uint32 n, then n x 12 floats (origin, t0, direction, t1,
// BSDF parameter u v, light parameter u v).  Output: uint32 n, uint32
// n_lights, then per probe kProbeOut floats: hit, BSDF sample (val[3], pdf,
// dir[3] in the normal frame, flags), BSDF eval at the light sample's
// direction (val[3], pdf, per light), light samples and evals -- the layout
// below.  The sphere light sampler draws one extra number from the
// context's generator (light/sphere-light-sampler.cc:90): the generator is
// reseeded before each light's sample, and the number it will draw is
// written out so a caller can feed the same value.
constexpr int kProbeHead = 9;    // hit, bsdf sample val[3] pdf dir[3] flags
constexpr int kProbeLight = 18;  // per light: sample val[3] pdf dir[3] dist extra;
                                 // bsdf eval at it val[3] pdf; light eval at the
                                 // bsdf sample's dir val[3] pdf

int mode_samples(const std::string &spec, const std::string &probes_path, const std::string &out) {
  RefScene rs;
  build_scene(rs, spec);
  std::ifstream in(probes_path, std::ios::binary);
  uint32_t n = 0;
  in.read(reinterpret_cast<char *>(&n), 4);
  std::vector<float> pr(size_t(n) * 12);
  in.read(reinterpret_cast<char *>(pr.data()), std::streamsize(pr.size() * 4));
  if (!in) throw std::runtime_error("short probe file");
  const Scene &scene = rs.grs->scene;
  const uint32_t nl = scene.num_light_samplers();
  const size_t stride = kProbeHead + size_t(kProbeLight) * nl;
  std::vector<float> res(size_t(n) * stride, 0.f);
  RenderContext ctx(*rs.grs);
  for (uint32_t i = 0; i < n; i++) {
    const float *q = &pr[size_t(i) * 12];
    float *r = &res[size_t(i) * stride];
    Ray ray(Pos(q[0], q[1], q[2]), Vec(q[4], q[5], q[6]), q[3], q[7]);
    const Surface::Renderable::IsecInfo *ii = scene.intersect(ray, ctx);
    if (!ii) continue;
    Media media(ctx.default_medium);
    Intersect isec = ii->make_intersect(media, ctx);
    r[0] = 1.f;
    const Bsdf *bsdf = isec.bsdf;
    Bsdf::Sample bs;
    if (bsdf) bs = bsdf->sample(UV(q[8], q[9]), Bsdf::ALL);
    for (int c = 0; c < 3; c++) r[1 + c] = bs.val[c];
    r[4] = bs.pdf;
    r[5] = bs.dir.x; r[6] = bs.dir.y; r[7] = bs.dir.z;
    r[8] = float(bs.flags);
    for (uint32_t k = 0; k < nl; k++) {
      float *l = r + kProbeHead + size_t(kProbeLight) * k;
      const unsigned seed = 7919u * i + 104729u * k + 1u;
      l[8] = Random(seed)();
      ctx.random.seed(seed);
      const Light::Sampler *ls = scene.light_samplers[k];
      Light::Sampler::Sample s = ls->sample(isec, UV(q[10], q[11]));
      for (int c = 0; c < 3; c++) l[c] = s.val[c];
      l[3] = s.pdf;
      l[4] = s.dir.x; l[5] = s.dir.y; l[6] = s.dir.z;
      l[7] = float(s.dist);
      if (bsdf && s.pdf != 0.f) {
        Bsdf::Value bv = bsdf->eval(s.dir, Bsdf::ALL);
        for (int c = 0; c < 3; c++) l[9 + c] = bv.val[c];
        l[12] = bv.pdf;
      }
      if (bsdf && bs.pdf != 0.f) {
        Light::Sampler::Value lv = ls->eval(isec, bs.dir);
        for (int c = 0; c < 3; c++) l[13 + c] = lv.val[c];
        l[16] = lv.pdf;
        l[17] = float(lv.dist);
      }
    }
    ctx.mempool.reset();
  }
  FILE *f = fopen(out.c_str(), "wb");
  if (!f) throw std::runtime_error("cannot write " + out);
  fwrite(&n, 4, 1, f);
  fwrite(&nl, 4, 1, f);
  fwrite(res.data(), 4, res.size(), f);
  fclose(f);
  printf("{\"probes\": %u, \"lights\": %u}\n", n, nl);
  return 0;
}

int mode_filter(const std::string &in_path, const std::string &out) {
  std::ifstream in(in_path, std::ios::binary);
  uint32_t n = 0;
  in.read(reinterpret_cast<char *>(&n), 4);
  std::vector<float> xy(size_t(n) * 2), v(n);
  in.read(reinterpret_cast<char *>(xy.data()), std::streamsize(xy.size() * 4));
  if (!in) throw std::runtime_error("short offsets file");
  const ImageMitchellFilt filt;
  for (uint32_t i = 0; i < n; i++) v[i] = filt.val(xy[2 * size_t(i)], xy[2 * size_t(i) + 1]);
  FILE *f = fopen(out.c_str(), "wb");
  if (!f) throw std::runtime_error("cannot write " + out);
  fwrite(v.data(), 4, n, f);
  fclose(f);
  printf("{\"b\": %.9g, \"c\": %.9g, \"x_radius\": %.9g, \"y_radius\": %.9g}\n", filt.b, filt.c, filt.x_radius,
         filt.y_radius);
  return 0;
}

int mode_ply(const char *file, const char *out_path) {
  Mesh mesh;
  Mesh::part_index_t part = mesh.add_part(new Lambert(Color(0.5f)));
  FILE *o = fopen(out_path, "wb");
  if (!o) throw std::runtime_error("cannot write output");
  try {
    load_ply_file(file, mesh, part, ValTable());
  } catch (std::exception &e) {
    fprintf(o, "ERR %s\n", e.what());
    fclose(o);
    return 0;
  }
  fprintf(o, "OK\n");
  const Mesh::Part &p = *mesh.parts[part];
  uint32_t nv = uint32_t(mesh.vertices.size()), nn = uint32_t(mesh.vertex_normals.size()),
           nt = uint32_t(p.triangles.size());
  fwrite(&nv, 4, 1, o);
  fwrite(&nn, 4, 1, o);
  fwrite(&nt, 4, 1, o);
  for (const auto &v : mesh.vertices) {
    float c[3] = {float(v.x), float(v.y), float(v.z)};
    fwrite(c, 4, 3, o);
  }
  for (const auto &v : mesh.vertex_normals) {
    float c[3] = {float(v.x), float(v.y), float(v.z)};
    fwrite(c, 4, 3, o);
  }
  for (const auto &t : p.triangles) {
    uint32_t vi[3] = {uint32_t(t.vi[0]), uint32_t(t.vi[1]), uint32_t(t.vi[2])};
    fwrite(vi, 4, 3, o);
  }
  fclose(o);
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  try {
    if (argc < 2) throw std::runtime_error("usage: snog_ref MODE ...");
    std::string mode = argv[1];
    if (mode == "octree" && argc == 4) return mode_octree(argv[2], argv[3]);
    if (mode == "ply" && argc == 4) return mode_ply(argv[2], argv[3]);
    if (mode == "trace" && argc >= 5)
      return mode_trace(argv[2], argv[3], argv[4], argc > 5 ? atoi(argv[5]) : 1);
    if (mode == "samples" && argc == 5) return mode_samples(argv[2], argv[3], argv[4]);
    if (mode == "filter" && argc == 4) return mode_filter(argv[2], argv[3]);
    if (mode == "camera" && argc == 5) return mode_camera(argv[2], argv[3], argv[4]);
    if (mode == "render" && argc >= 4)
      return mode_render(argv[2], argv[3], argc > 4 ? atoi(argv[4]) : 1,
                         argc > 5 ? atoi(argv[5]) : 0, argc > 6 ? atoi(argv[6]) : 0,
                         argc > 7 ? atoi(argv[7]) : 0, argc > 8 ? atoi(argv[8]) : 0,
                         argc > 9 ? unsigned(atoi(argv[9])) : 1u, argc > 10 && atoi(argv[10]) != 0);
    throw std::runtime_error("bad arguments");
  } catch (std::exception &e) {
    fprintf(stderr, "snog_ref: %s\n", e.what());
    return 1;
  }
}
