// snogray_b200.hpp -- the reference's scene/render classes, header-only, over
// the C ABI in snogray_b200.h.
//
// A program written against snogray's C++ API for this path builds its scene
// with the same class names and constructor arguments and renders it with a
// RenderMgr-shaped call; the scene is flattened once into a SnogSceneDesc and
// uploaded (snog_scene_create), and RenderMgr::render runs the B200 wavefront
// renderer (snog_render).  Errors from the library are rethrown as
// std::runtime_error, the reference's convention for scene and parameter
// errors (render/global-render-state.cc:73-74, 90).
//
// Mirrors (reference file:line):
//   Color, Pos, Vec                  color/color.h, geometry/pos.h, geometry/vec.h
//   Medium (ior, absorb)             material/medium.h:30-32
//   Ior (n, k)                       material/ior.h
//   Lambert (color)                  material/lambert.h:29
//   CookTorrance (col, gloss, m, ior) material/cook-torrance.h:27-30
//   Mirror (ior, reflectance, col)   material/mirror.h:47-49
//   Glass (medium)                   material/glass.h:27
//   Glow (col [, underlying])        material/glow.h:28-30
//   Sphere (mat, center, radius)     surface/sphere.h:32
//   Tripar (mat, v0, e1, e2, par)    surface/tripar.h:28-30
//   Mesh: add_part, add_vertex, add_triangle(s)  surface/mesh.h:62, 188, 197
//   PointLight (pos, col [, angle, dir, fringe]) light/point-light.h:32-47
//   FarLight (dir, angle, intensity) light/far-light.h:39
//   EnvmapLight (envmap, frame)      light/envmap-light.h:29
//   SurfaceGroup::add (surface | light)          surface/surface-group.h:36-40
//   Camera: move, point, set_vert_fov, set_horiz_fov  camera/camera.h:84-128, 231-247
//   GlobalRenderState (scene, params)            render/global-render-state.cc:28-49
//   RenderMgr (state, camera, w, h); render (num_threads, pattern, output,
//                                    progress, stats)  render-mgr/render-mgr.h:39-50
//   RenderPattern (left_x, top_y, width, height)  render-mgr/render-pattern.h:105-108
//   Progress (set_start, set_size, start, update, end)  util/progress.h
//   RenderStats, RenderStats::IsecStats  render/render-stats.h:24-71
//   ImageSampledOutput (w, h [, sample_base_x, sample_base_y])
//                                    image/image-sampled-output.h:54-56
//
// Differences: one CUDA device per process (snog_init); surfaces are owned by
// shared pointers rather than the reference's raw-pointer ownership by the
// group; primitive ids follow "all mesh triangles (mesh by mesh, part by
// part), then spheres, then tripars" whatever order they were added in (ids
// only matter to the trace API and to ties between equal hit distances).

#ifndef SNOGRAY_B200_HPP
#define SNOGRAY_B200_HPP

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "snogray_b200.h"

namespace snogray_b200 {

inline void check(int rc, const char *what) {
  if (rc != SNOG_OK)
    throw std::runtime_error(std::string(what) + ": " + snog_last_error() + " (status " + std::to_string(rc) + ")");
}

struct Color {
  float r = 0, g = 0, b = 0;
  Color() = default;
  Color(float v) : r(v), g(v), b(v) {}
  Color(float r_, float g_, float b_) : r(r_), g(g_), b(b_) {}
};

struct Vec {
  float x = 0, y = 0, z = 0;
  Vec() = default;
  Vec(float x_, float y_, float z_) : x(x_), y(y_), z(z_) {}
};
inline Vec operator-(const Vec &a, const Vec &b) { return Vec(a.x - b.x, a.y - b.y, a.z - b.z); }
inline Vec cross(const Vec &a, const Vec &b) {
  return Vec(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float dot(const Vec &a, const Vec &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Vec unit(const Vec &v) {
  const float inv = 1.0f / std::sqrt(dot(v, v));
  return Vec(v.x * inv, v.y * inv, v.z * inv);
}
using Pos = Vec;

// A coordinate frame (its axes; the origin is unused by the envmap light).
struct Frame {
  Vec x{1, 0, 0}, y{0, 1, 0}, z{0, 0, 1};
};

struct Ior {
  float n = 1.5f, k = 0.f;
  Ior(float n_ = 1.5f, float k_ = 0.f) : n(n_), k(k_) {}
};

struct Medium {
  float ior = 1.f;
  Color absorption;
  Medium(float ior_ = 1.f, const Color &absorb = Color(0.f)) : ior(ior_), absorption(absorb) {}
};

// ---- materials -------------------------------------------------------------

class Material {
 public:
  virtual ~Material() = default;
  // The C record; UNDERLYING is the flattened index of the underlying material.
  virtual SnogMaterial record(int32_t underlying) const = 0;
  virtual std::shared_ptr<const Material> underlying() const { return nullptr; }

 protected:
  static SnogMaterial blank(uint32_t type) {
    SnogMaterial m{};
    m.type = type;
    m.gloss[0] = m.gloss[1] = m.gloss[2] = 1.f;
    m.ior_n = 1.5f;
    m.underlying = -1;
    return m;
  }
  static void set3(float *d, const Color &c) {
    d[0] = c.r;
    d[1] = c.g;
    d[2] = c.b;
  }
};
using MaterialRef = std::shared_ptr<const Material>;

class Lambert : public Material {
 public:
  explicit Lambert(const Color &col) : color(col) {}
  SnogMaterial record(int32_t) const override {
    SnogMaterial m = blank(SNOG_LAMBERT);
    set3(m.color, color);
    return m;
  }
  Color color;
};

class CookTorrance : public Material {
 public:
  CookTorrance(const Color &col, const Color &gloss_col, float m_, const Ior &ior_ = Ior(1.5f))
      : color(col), gloss_color(gloss_col), m(m_), ior(ior_) {}
  SnogMaterial record(int32_t) const override {
    SnogMaterial r = blank(SNOG_COOK_TORRANCE);
    set3(r.color, color);
    set3(r.gloss, gloss_color);
    r.m = m;
    r.ior_n = ior.n;
    r.ior_k = ior.k;
    return r;
  }
  Color color, gloss_color;
  float m;
  Ior ior;
};

// A mirror with a Lambertian underlying material of colour COL.
class Mirror : public Material {
 public:
  Mirror(const Ior &ior_, const Color &reflectance_, const Color &col = Color(0.f))
      : ior(ior_), reflectance(reflectance_), color(col) {}
  SnogMaterial record(int32_t) const override {
    SnogMaterial r = blank(SNOG_MIRROR);
    set3(r.color, color);
    set3(r.gloss, reflectance);
    r.ior_n = ior.n;
    r.ior_k = ior.k;
    return r;
  }
  Ior ior;
  Color reflectance, color;
};

class Glass : public Material {
 public:
  explicit Glass(const Medium &medium) : medium_(medium) {}
  SnogMaterial record(int32_t) const override {
    SnogMaterial r = blank(SNOG_GLASS);
    r.ior_n = medium_.ior;
    r.ior_k = 0.f;
    set3(r.absorb, medium_.absorption);
    return r;
  }
  Medium medium_;
};

class Glow : public Material {
 public:
  explicit Glow(const Color &col) : color(col) {}
  Glow(const Color &col, const MaterialRef &underlying_material) : color(col), under(underlying_material) {}
  SnogMaterial record(int32_t underlying_index) const override {
    SnogMaterial r = blank(SNOG_GLOW);
    set3(r.color, color);
    r.underlying = under ? underlying_index : -1;
    return r;
  }
  MaterialRef underlying() const override { return under; }
  Color color;
  MaterialRef under;
};

// ---- surfaces --------------------------------------------------------------

class Surface {
 public:
  virtual ~Surface() = default;
};

class Sphere : public Surface {
 public:
  Sphere(const MaterialRef &mat, const Pos &center_, float radius_) : material(mat), center(center_), radius(radius_) {}
  MaterialRef material;
  Pos center;
  float radius;
};

// Triangle (parallelogram = false) or parallelogram with corner V0 and edges
// E1, E2; its normal is E2 x E1.
class Tripar : public Surface {
 public:
  Tripar(const MaterialRef &mat, const Pos &v0_, const Vec &e1_, const Vec &e2_, bool parallelogram_ = false)
      : material(mat), v0(v0_), e1(e1_), e2(e2_), parallelogram(parallelogram_) {}
  MaterialRef material;
  Pos v0;
  Vec e1, e2;
  bool parallelogram;
};

class Mesh : public Surface {
 public:
  using vert_index_t = uint32_t;
  using part_index_t = uint32_t;
  part_index_t add_part(const MaterialRef &mat) {
    parts.push_back(Part{mat, {}});
    return part_index_t(parts.size() - 1);
  }
  vert_index_t add_vertex(const Pos &pos) {
    vertices.push_back(pos);
    return vert_index_t(vertices.size() - 1);
  }
  // A vertex with its normal (Mesh::add_vertex (pos, normal), mesh.h:65-67);
  // a mesh with normals shades with interpolated normals.
  vert_index_t add_vertex(const Pos &pos, const Vec &normal) {
    if (normals.size() != vertices.size()) throw std::runtime_error("Mesh: every vertex needs a normal");
    normals.push_back(normal);
    return add_vertex(pos);
  }
  // Normals for the vertices from BASE_VERT on (Mesh::add_normals, mesh.h:95-111).
  void add_normals(const std::vector<Vec> &new_normals, vert_index_t base_vert) {
    if (base_vert != normals.size()) throw std::runtime_error("Mesh::add_normals: normals out of step with vertices");
    normals.insert(normals.end(), new_normals.begin(), new_normals.end());
  }
  void add_triangle(part_index_t part, vert_index_t a, vert_index_t b, vert_index_t c) {
    at(part).tris.insert(at(part).tris.end(), {a, b, c});
  }
  void add_triangles(part_index_t part, const std::vector<vert_index_t> &tri_vert_indices,
                     vert_index_t base_vert = 0) {
    if (tri_vert_indices.size() % 3) throw std::runtime_error("Mesh::add_triangles: index count not a multiple of 3");
    for (vert_index_t v : tri_vert_indices) at(part).tris.push_back(base_vert + v);
  }
  struct Part {
    MaterialRef material;
    std::vector<vert_index_t> tris;
  };
  std::vector<Pos> vertices;
  std::vector<Vec> normals;        // empty, or one per vertex
  std::vector<Part> parts;
  bool left_handed = true;         // geometric normal e2 x e1 (false: e1 x e2)

 private:
  Part &at(part_index_t p) {
    if (p >= parts.size()) throw std::runtime_error("Mesh: no part " + std::to_string(p));
    return parts[p];
  }
};

// load_ply_file (load/mesh/load-ply.cc:163-214): adds the PLY file's
// vertices, normals and triangles (into PART) to MESH and makes it
// right-handed, as the reference does.
inline void load_ply_file(const std::string &filename, Mesh &mesh, Mesh::part_index_t part) {
  SnogPlyMesh m{};
  if (snog_ply_load(filename.c_str(), &m) != SNOG_OK) throw std::runtime_error(snog_last_error());
  const Mesh::vert_index_t base = Mesh::vert_index_t(mesh.vertices.size());
  const bool with_normals = m.normals != nullptr;
  if (with_normals && mesh.normals.size() != mesh.vertices.size()) {
    snog_ply_free(&m);
    throw std::runtime_error("load_ply_file: the mesh's earlier vertices have no normals");
  }
  for (uint32_t v = 0; v < m.n_vertices; v++) {
    mesh.vertices.push_back(Pos(m.vertices[3 * v], m.vertices[3 * v + 1], m.vertices[3 * v + 2]));
    if (with_normals) mesh.normals.push_back(Vec(m.normals[3 * v], m.normals[3 * v + 1], m.normals[3 * v + 2]));
  }
  std::vector<Mesh::vert_index_t> idx(m.triangles, m.triangles + 3 * size_t(m.n_triangles));
  snog_ply_free(&m);
  mesh.add_triangles(part, idx, base);
  mesh.left_handed = false;
}

// ---- lights ----------------------------------------------------------------

class Light {
 public:
  virtual ~Light() = default;
};

class PointLight : public Light {
 public:
  PointLight(const Pos &pos_, const Color &col) : pos(pos_), color(col) {}
  PointLight(const Pos &pos_, const Color &col, float angle_, const Vec &dir_, float fringe_angle_ = 0.f)
      : pos(pos_), color(col), angle(angle_), dir(dir_), fringe_angle(fringe_angle_) {}
  Pos pos;
  Color color;
  float angle = 8.f * std::atan(1.f);   // 2 pi: omnidirectional
  Vec dir{0, 0, 1};
  float fringe_angle = 0.f;
};

class FarLight : public Light {
 public:
  FarLight(const Vec &dir_, float angle_, const Color &intensity_) : dir(dir_), angle(angle_), intensity(intensity_) {}
  Vec dir;
  float angle;
  Color intensity;
};

// A lat-long environment map: HEIGHT rows of WIDTH RGB floats, top row first,
// WIDTH = 2 * HEIGHT.
struct Envmap {
  uint32_t width = 0, height = 0;
  std::vector<float> rgb;
};

class EnvmapLight : public Light {
 public:
  explicit EnvmapLight(std::shared_ptr<const Envmap> envmap_, const Frame &frame_ = Frame())
      : envmap(std::move(envmap_)), frame(frame_) {}
  std::shared_ptr<const Envmap> envmap;
  Frame frame;
};

// ---- scene -----------------------------------------------------------------

class SurfaceGroup {
 public:
  void add(std::shared_ptr<Surface> surface) { surfaces.push_back(std::move(surface)); }
  void add(std::shared_ptr<Light> light) { lights.push_back(std::move(light)); }
  std::vector<std::shared_ptr<Surface>> surfaces;
  std::vector<std::shared_ptr<Light>> lights;
};

// ValTable keys of the path integrator and output (render-params.h:32-36,
// render/path-integ.cc:64-68, global-render-state.cc:37-38).
struct RenderParams {
  uint32_t samples = 16;
  uint32_t min_path_len = 3, max_path_len = 25, direct_samples = 1;
  float min_trace = 1e-3f;
  float background_alpha = 1.f;
  uint64_t seed = 0;
  // [surface_integ.type]: "path" (SNOG_INTEG_PATH) or "direct"; the direct
  // integrator takes its light samples per light from light_samples.
  uint32_t integrator = SNOG_INTEG_PATH;
  uint32_t light_samples = 16;
};

// The flattened scene uploaded to the device (Scene + Octree + light
// samplers); like the reference's GlobalRenderState it is built once and read
// by every render.
class GlobalRenderState {
 public:
  // ON_DEVICE = false builds the octree on the host only (snog_scene_build_host):
  // info() works, rendering is refused.
  GlobalRenderState(const SurfaceGroup &scene, const RenderParams &params_ = RenderParams(), bool on_device = true)
      : params(params_) {
    Flat f;
    f.flatten(scene);
    SnogSceneDesc d{};
    d.n_materials = uint32_t(f.mats.size());
    d.materials = f.mats.data();
    d.n_vertices = uint32_t(f.verts.size() / 3);
    d.vertices = f.verts.data();
    d.n_triangles = uint32_t(f.tris.size() / 3);
    d.triangles = f.tris.data();
    d.tri_material = f.tri_mat.data();
    d.n_spheres = uint32_t(f.spheres.size());
    d.spheres = f.spheres.data();
    d.n_tripars = uint32_t(f.tripars.size());
    d.tripars = f.tripars.data();
    d.n_point_lights = uint32_t(f.plights.size());
    d.point_lights = f.plights.data();
    d.n_far_lights = uint32_t(f.flights.size());
    d.far_lights = f.flights.data();
    d.vertex_normals = f.with_normals ? f.normals.data() : nullptr;
    d.mesh_right_handed = f.left_handed ? 0u : 1u;
    if (f.env) {
      d.env_width = f.env->envmap->width;
      d.env_height = f.env->envmap->height;
      d.env_rgb = f.env->envmap->rgb.data();
      const Vec ax[3] = {f.env->frame.x, f.env->frame.y, f.env->frame.z};
      for (int k = 0; k < 3; k++) {
        d.env_frame[3 * k] = ax[k].x;
        d.env_frame[3 * k + 1] = ax[k].y;
        d.env_frame[3 * k + 2] = ax[k].z;
      }
    } else {
      d.env_frame[0] = d.env_frame[4] = d.env_frame[8] = 1.f;
    }
    check(on_device ? snog_scene_create(&d, &scene_) : snog_scene_build_host(&d, &scene_), "GlobalRenderState");
  }
  ~GlobalRenderState() { snog_scene_destroy(scene_); }
  GlobalRenderState(const GlobalRenderState &) = delete;
  GlobalRenderState &operator=(const GlobalRenderState &) = delete;

  SnogScene *handle() const { return scene_; }
  SnogSceneInfo info() const {
    SnogSceneInfo i{};
    check(snog_scene_info(scene_, &i), "GlobalRenderState::info");
    return i;
  }
  RenderParams params;

 private:
  // Flattening: materials get indices in order of first use (a Glow's
  // underlying material first); a mesh part whose material index would fall
  // below the previous part's gets a copy of the record, so triangle
  // materials stay non-decreasing as SnogSceneDesc requires.
  struct Flat {
    std::vector<SnogMaterial> mats;
    std::map<const Material *, uint32_t> index;
    std::vector<float> verts, normals;
    std::vector<uint32_t> tris, tri_mat;
    uint32_t n_meshes = 0;
    bool with_normals = false, left_handed = true;
    std::vector<SnogSphere> spheres;
    std::vector<SnogTripar> tripars;
    std::vector<SnogPointLight> plights;
    std::vector<SnogFarLight> flights;
    const EnvmapLight *env = nullptr;

    uint32_t mat(const MaterialRef &m) {
      if (!m) throw std::runtime_error("surface without a material");
      auto it = index.find(m.get());
      if (it != index.end()) return it->second;
      int32_t under = -1;
      if (m->underlying()) under = int32_t(mat(m->underlying()));
      const uint32_t k = uint32_t(mats.size());
      mats.push_back(m->record(under));
      index[m.get()] = k;
      return k;
    }
    static void put3(float *d, const Vec &v) {
      d[0] = v.x;
      d[1] = v.y;
      d[2] = v.z;
    }
    void flatten(const SurfaceGroup &g) {
      uint32_t last = 0;
      for (auto &s : g.surfaces)
        if (auto *mesh = dynamic_cast<const Mesh *>(s.get())) {
          const uint32_t base = uint32_t(verts.size() / 3);
          // One mesh record per scene: every mesh must agree on handedness and
          // on having vertex normals.
          const bool has_n = !mesh->normals.empty();
          if (n_meshes++ && (has_n != with_normals || mesh->left_handed != left_handed))
            throw std::runtime_error("meshes of one scene must agree on handedness and vertex normals");
          with_normals = has_n;
          left_handed = mesh->left_handed;
          if (has_n && mesh->normals.size() != mesh->vertices.size())
            throw std::runtime_error("Mesh: normals for only some vertices");
          for (const Pos &p : mesh->vertices) verts.insert(verts.end(), {p.x, p.y, p.z});
          for (const Vec &n : mesh->normals) normals.insert(normals.end(), {n.x, n.y, n.z});
          for (auto &part : mesh->parts) {
            uint32_t mi = mat(part.material);
            if (mi < last) {   // keep runs non-decreasing: a private copy of the record
              mi = uint32_t(mats.size());
              mats.push_back(mats[index[part.material.get()]]);
            }
            last = mi;
            for (uint32_t v : part.tris) {
              if (v >= mesh->vertices.size()) throw std::runtime_error("Mesh: vertex index out of range");
              tris.push_back(base + v);
            }
            tri_mat.insert(tri_mat.end(), part.tris.size() / 3, mi);
          }
        }
      for (auto &s : g.surfaces)
        if (auto *sp = dynamic_cast<const Sphere *>(s.get())) {
          SnogSphere r{};
          put3(r.center, sp->center);
          r.radius = sp->radius;
          r.material = mat(sp->material);
          spheres.push_back(r);
        }
      for (auto &s : g.surfaces)
        if (auto *tp = dynamic_cast<const Tripar *>(s.get())) {
          SnogTripar r{};
          put3(r.v0, tp->v0);
          put3(r.e1, tp->e1);
          put3(r.e2, tp->e2);
          r.parallelogram = tp->parallelogram ? 1u : 0u;
          r.material = mat(tp->material);
          tripars.push_back(r);
        }
      for (auto &l : g.lights) {
        if (auto *pl = dynamic_cast<const PointLight *>(l.get())) {
          SnogPointLight r{};
          put3(r.pos, pl->pos);
          r.color[0] = pl->color.r;
          r.color[1] = pl->color.g;
          r.color[2] = pl->color.b;
          r.angle = pl->angle;
          r.fringe_angle = pl->fringe_angle;
          put3(r.dir, pl->dir);
          plights.push_back(r);
        } else if (auto *fl = dynamic_cast<const FarLight *>(l.get())) {
          SnogFarLight r{};
          put3(r.dir, fl->dir);
          r.angle = fl->angle;
          r.color[0] = fl->intensity.r;
          r.color[1] = fl->intensity.g;
          r.color[2] = fl->intensity.b;
          flights.push_back(r);
        } else if (auto *el = dynamic_cast<const EnvmapLight *>(l.get())) {
          if (env) throw std::runtime_error("at most one envmap light");
          if (!el->envmap) throw std::runtime_error("envmap light without an envmap");
          env = el;
        }
      }
    }
  };
  SnogScene *scene_ = nullptr;
};

// Pinhole camera in the reference's representation: move, point at a target
// with an up vector, field of view (camera/camera.h:84-128, 231-247).
class Camera {
 public:
  void move(const Pos &p) { pos = p; }
  void point(const Pos &targ, const Vec &user_up) {
    forward = unit(targ - pos);
    right = unit(cross(user_up, forward));
    up = unit(cross(forward, right));
  }
  // Field of view for an image of aspect ratio ASPECT (width / height).
  void set_vert_fov(float fov, float aspect) {
    const float t = std::tan(fov / 2);
    tan_y = t;
    tan_x = t * aspect;
  }
  void set_horiz_fov(float fov, float aspect) {
    const float t = std::tan(fov / 2);
    tan_x = t;
    tan_y = t / aspect;
  }
  SnogCamera c_struct() const {
    SnogCamera c{};
    const Vec v[4] = {pos, forward, right, up};
    float *dst[4] = {c.pos, c.forward, c.right, c.up};
    for (int k = 0; k < 4; k++) {
      dst[k][0] = v[k].x;
      dst[k][1] = v[k].y;
      dst[k][2] = v[k].z;
    }
    c.tan_half_fov_x = tan_x;
    c.tan_half_fov_y = tan_y;
    return c;
  }
  Pos pos{0, 0, 0};
  Vec forward{0, 0, 1}, right{1, 0, 0}, up{0, 1, 0};
  float tan_x = 0.f, tan_y = 0.f;
};

// The finished image: HEIGHT rows of WIDTH RGB floats, top row first (the
// flushed values of the reference's ImageSampledOutput).  Its top-left pixel
// is film pixel (sample_base_x, sample_base_y), the offset a --limit render
// gives its output (snogray.lua:451-452); 0, 0 for a whole image.
class ImageSampledOutput {
 public:
  ImageSampledOutput(uint32_t w, uint32_t h, int32_t base_x = 0, int32_t base_y = 0)
      : width(w), height(h), sample_base_x(base_x), sample_base_y(base_y), rgb(size_t(w) * h * 3) {}
  // The Mitchell filter's reach in pixels, the margin the reference's driver
  // adds around a render pattern (image/image-filter-conv.h:39-40,
  // snogray.lua:543-550).
  int filter_x_radius() const { return 2; }
  int filter_y_radius() const { return 2; }
  // Portable float map (little-endian), bottom row first as PFM stores it.
  void write_pfm(const std::string &path) const {
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write " + path);
    std::fprintf(f, "PF\n%u %u\n-1.0\n", width, height);
    for (uint32_t y = height; y-- > 0;) std::fwrite(&rgb[size_t(y) * width * 3], sizeof(float), size_t(width) * 3, f);
    std::fclose(f);
  }
  uint32_t width, height;
  int32_t sample_base_x, sample_base_y;
  std::vector<float> rgb;
};

// The pixels to render: the film rectangle [left_x, left_x + width) x
// [top_y, top_y + height) (render-mgr/render-pattern.h:105-108).
class RenderPattern {
 public:
  RenderPattern(int left_x, int top_y, int width, int height)
      : x_beg(left_x), y_beg(top_y), x_end(left_x + width), y_end(top_y + height) {}
  int left_x() const { return x_beg; }
  int top_y() const { return y_beg; }
  int width() const { return x_end - x_beg; }
  int height() const { return y_end - y_beg; }

 private:
  int x_beg, y_beg, x_end, y_end;
};

// Progress reports (util/progress.h): the render calls set_start and
// set_size with the pattern's position range, start, one update at the end
// of the device work, and end.
class Progress {
 public:
  virtual ~Progress() = default;
  virtual void set_start(int) {}
  virtual void set_size(unsigned) {}
  virtual void start() {}
  virtual void update(int) {}
  virtual void end() {}
};

// The reference's render statistics (render/render-stats.h:24-71):
// scene_intersect_calls and scene_shadow_tests count closest-hit and shadow
// queries; IsecStats counts the traversal's node visits and primitive tests
// (the path integrator's; the negative cache the reference keeps is not used
// here, so neg_cache_* stay 0 and a primitive met twice by one ray is tested
// twice).  illum_calls counts vertices lit (path integrator).  paths and
// device_ms are this library's additions.
struct RenderStats {
  struct IsecStats {
    unsigned long long surface_intersects_tests = 0, surface_intersects_hits = 0;
    unsigned long long neg_cache_hits = 0, neg_cache_collisions = 0;
    unsigned long long space_node_intersect_calls = 0;
  };
  unsigned long long scene_intersect_calls = 0, scene_shadow_tests = 0, illum_calls = 0;
  IsecStats intersect, shadow;
  uint64_t paths = 0;
  double device_ms = 0;
  // Names this library used before the reference's fields were added.
  uint64_t closest_rays = 0, shadow_rays = 0;
};

class RenderMgr {
 public:
  RenderMgr(const GlobalRenderState &state, const Camera &camera, unsigned width, unsigned height)
      : state_(state), camera_(camera), width_(width), height_(height) {}

  // Render the pixels of PATTERN into OUTPUT, as the reference's
  // RenderMgr::render (render-mgr/render-mgr.h:45-50): the film is the
  // renderer's width x height, OUTPUT covers the film pixels from its
  // sample base, and every sample adds to the output pixels its filter
  // reaches.  NUM_THREADS is accepted for the signature's sake: the work runs
  // on the GPU.  STATS is added to, as the reference's is.
  void render(unsigned num_threads, RenderPattern &pattern, ImageSampledOutput &output, Progress &prog,
              RenderStats &stats) {
    (void)num_threads;
    SnogRenderWindow win{};
    win.pat_x = pattern.left_x();
    win.pat_y = pattern.top_y();
    if (pattern.width() <= 0 || pattern.height() <= 0)
      throw std::runtime_error("RenderMgr::render: empty render pattern");
    win.pat_width = uint32_t(pattern.width());
    win.pat_height = uint32_t(pattern.height());
    win.out_x = output.sample_base_x;
    win.out_y = output.sample_base_y;
    win.out_width = output.width;
    win.out_height = output.height;
    const SnogCamera cam = camera_.c_struct();
    SnogRenderParams p = params();
    p.flags |= SNOG_RENDER_COUNT_TRAVERSAL;
    const unsigned npos = unsigned(pattern.width()) * unsigned(pattern.height());
    prog.set_start(0);
    prog.set_size(npos);
    prog.start();
    SnogRenderStats st{};
    check(snog_render_window(state_.handle(), &cam, &p, &win, output.rgb.data(), &st), "RenderMgr::render");
    prog.update(int(npos));
    prog.end();
    add(stats, st);
  }

  // The whole image (the pattern with the filter margin, snogray.lua:543-550)
  // into OUTPUT, whose size must be the renderer's.
  void render(ImageSampledOutput &output, RenderStats &stats) {
    if (output.width != width_ || output.height != height_)
      throw std::runtime_error("RenderMgr::render: output size differs from the renderer's");
    const SnogCamera cam = camera_.c_struct();
    SnogRenderParams p = params();
    SnogRenderStats st{};
    check(snog_render(state_.handle(), &cam, &p, output.rgb.data(), &st), "RenderMgr::render");
    add(stats, st);
  }

 private:
  SnogRenderParams params() const {
    SnogRenderParams p{};
    p.width = width_;
    p.height = height_;
    p.spp = state_.params.samples;
    p.min_path_len = state_.params.min_path_len;
    p.max_path_len = state_.params.max_path_len;
    p.integrator = state_.params.integrator;
    p.direct_samples =
        p.integrator == SNOG_INTEG_DIRECT ? state_.params.light_samples : state_.params.direct_samples;
    p.min_trace = state_.params.min_trace;
    p.bg_alpha = state_.params.background_alpha;
    p.seed = state_.params.seed;
    return p;
  }
  static void add(RenderStats &stats, const SnogRenderStats &st) {
    stats.scene_intersect_calls += st.closest_rays;
    stats.scene_shadow_tests += st.shadow_rays;
    stats.intersect.space_node_intersect_calls += st.closest_nodes;
    stats.intersect.surface_intersects_tests += st.closest_tests;
    stats.shadow.space_node_intersect_calls += st.shadow_nodes;
    stats.shadow.surface_intersects_tests += st.shadow_tests;
    stats.illum_calls += st.illum_calls;
    stats.paths += st.paths;
    stats.closest_rays += st.closest_rays;
    stats.shadow_rays += st.shadow_rays;
    stats.device_ms += st.device_ms;
  }

  const GlobalRenderState &state_;
  Camera camera_;
  unsigned width_, height_;
};

}  // namespace snogray_b200

#endif
