// scene_spec.h -- on-disk scene specification read by the oracle programs.
//
// TEST INFRASTRUCTURE: this file belongs to the oracle (the CPU checker).  The
// product library never reads it; it receives the same scene through the
// SnogSceneDesc struct of the C ABI.  tests/ and bench.py write spec files
// with oracle/spec.py from the very numpy arrays they pass to the C ABI, so
// the reference renderer, the restatement and the CUDA path see one scene.
//
// Layout (little-endian): SpecHeader, then the arrays in the order of the
// header's counts.  Every record is a flat struct of 32-bit fields.

#ifndef SNOG_ORACLE_SCENE_SPEC_H
#define SNOG_ORACLE_SCENE_SPEC_H

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace snogspec {

enum MatType : uint32_t {
  MAT_LAMBERT = 0,       // Lambert (color)                     material/lambert.h
  MAT_COOK_TORRANCE = 1, // CookTorrance (color, gloss, m, ior) material/cook-torrance.h:27
  MAT_MIRROR = 2,        // Mirror (ior, reflectance, color)    material/mirror.h:47
  MAT_GLASS = 3,         // Glass (Medium (ior, absorb))        material/glass.h:27
  MAT_GLOW = 4,          // Glow (color [, underlying])         material/glow.h:28
};

struct MatRec {
  uint32_t type;
  float color[3];        // Lambert/CT diffuse/Mirror underlying/Glow emission
  float gloss[3];        // CT gloss colour, Mirror reflectance
  float m;               // CT rms slope
  float ior_n, ior_k;    // CT / Mirror Ior, Glass medium ior (n)
  float absorb[3];       // Glass medium absorption
  int32_t underlying;    // Glow underlying material index, or -1
};

struct SphereRec { float center[3]; float radius; uint32_t mat; };
struct TriparRec { float v0[3]; float e1[3]; float e2[3]; uint32_t parallelogram; uint32_t mat; };
struct PointLightRec { float pos[3]; float color[3]; float angle; float fringe_angle; float dir[3]; };
struct FarLightRec { float dir[3]; float angle; float color[3]; };

struct SpecHeader {
  char magic[8];                 // "SNOGSPC1"
  uint32_t n_materials, n_vertices, n_triangles, n_spheres, n_tripars;
  uint32_t n_point_lights, n_far_lights;
  uint32_t env_w, env_h;         // 0 = no envmap light
  float env_frame[9];            // envmap light frame axes x, y, z
  // Camera, as the reference Camera holds it after move/point/set_fov
  // (camera/camera.h:114-128, 231-242).
  float cam_pos[3], cam_forward[3], cam_right[3], cam_up[3];
  float tan_half_fov_x, tan_half_fov_y;
  // Render parameters (ValTable keys in brackets).
  uint32_t width, height;        // output image size
  uint32_t spp;                  // [samples]
  uint32_t min_path_len;         // [surface_integ.min_path_len]
  uint32_t max_path_len;         // [surface_integ.max_path_len]
  uint32_t direct_samples;       // [surface_integ.direct_samples]
  float min_trace;               // [min_trace]
  float bg_alpha;                // [background_alpha]
  uint32_t has_normals;          // vertex normals follow the envmap (3 floats each)
  uint32_t right_handed;         // the mesh is right-handed (Mesh::left_handed false)
  uint32_t integrator;           // [surface_integ.type]: 0 path, 1 direct (direct_samples
                                 // is then [surface_integ.light_samples])
  uint32_t reserved[5];
};

struct Scene {
  SpecHeader h;
  std::vector<MatRec> mats;
  std::vector<float> verts;        // 3 per vertex
  std::vector<uint32_t> tris;      // 3 per triangle
  std::vector<uint32_t> tri_mat;   // per triangle, non-decreasing (mesh part)
  std::vector<SphereRec> spheres;
  std::vector<TriparRec> tripars;
  std::vector<PointLightRec> plights;
  std::vector<FarLightRec> flights;
  std::vector<float> env;          // env_w*env_h*3, row 0 = top row of image
  std::vector<float> normals;      // 3 per vertex when h.has_normals
};

template <class T>
static void read_vec(FILE *f, std::vector<T> &v, size_t n) {
  v.resize(n);
  if (n && fread(v.data(), sizeof(T), n, f) != n)
    throw std::runtime_error("scene spec: truncated file");
}

static inline Scene load(const std::string &path) {
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) throw std::runtime_error("scene spec: cannot open " + path);
  Scene s;
  if (fread(&s.h, sizeof(s.h), 1, f) != 1 || memcmp(s.h.magic, "SNOGSPC1", 8) != 0) {
    fclose(f);
    throw std::runtime_error("scene spec: bad header in " + path);
  }
  read_vec(f, s.mats, s.h.n_materials);
  read_vec(f, s.verts, size_t(s.h.n_vertices) * 3);
  read_vec(f, s.tris, size_t(s.h.n_triangles) * 3);
  read_vec(f, s.tri_mat, s.h.n_triangles);
  read_vec(f, s.spheres, s.h.n_spheres);
  read_vec(f, s.tripars, s.h.n_tripars);
  read_vec(f, s.plights, s.h.n_point_lights);
  read_vec(f, s.flights, s.h.n_far_lights);
  read_vec(f, s.env, size_t(s.h.env_w) * s.h.env_h * 3);
  if (s.h.has_normals) read_vec(f, s.normals, size_t(s.h.n_vertices) * 3);
  fclose(f);
  return s;
}

// Ray batch file: uint32 n, uint32 n_closest, then n*7 floats as SoA
// (ox[n] oy[n] oz[n] dx[n] dy[n] dz[n] tmax[n]).  Rays [0, n_closest) are
// closest-hit queries, the rest any-hit queries.  t0 is 0 for all of them.
struct RayBatch {
  uint32_t n = 0, n_closest = 0;
  std::vector<float> soa;
  const float *ox() const { return soa.data(); }
  const float *oy() const { return soa.data() + n; }
  const float *oz() const { return soa.data() + 2 * size_t(n); }
  const float *dx() const { return soa.data() + 3 * size_t(n); }
  const float *dy() const { return soa.data() + 4 * size_t(n); }
  const float *dz() const { return soa.data() + 5 * size_t(n); }
  const float *tmax() const { return soa.data() + 6 * size_t(n); }
};

static inline RayBatch load_rays(const std::string &path) {
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) throw std::runtime_error("rays: cannot open " + path);
  RayBatch r;
  if (fread(&r.n, 4, 1, f) != 1 || fread(&r.n_closest, 4, 1, f) != 1) {
    fclose(f);
    throw std::runtime_error("rays: bad header");
  }
  read_vec(f, r.soa, size_t(r.n) * 7);
  fclose(f);
  return r;
}

}  // namespace snogspec

#endif
