// scene.cc -- validate a SnogSceneDesc, build the octree, derive the light
// samplers and the envmap sampling tables, and upload everything in the
// device layout described in snog_common.h.
//
// Compiled with -ffp-contract=off: bounding boxes, edges and midpoints must
// round exactly as the reference's float code does.

#include "launch.h"
#include "scene.h"

#include "octree_gpu.h"

#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>

namespace snog {

void check_cuda(int err, const char *what) {
  if (err != cudaSuccess)
    throw Error{SNOG_ECUDA, std::string(what) + ": " + cudaGetErrorString(cudaError_t(err))};
}

void check_render_flags(uint32_t flags) {
  if (flags & 1u) throw Error{SNOG_EINVAL, "traversal stack overflow (non-finite ray?)"};
  if (flags & 2u)
    throw Error{SNOG_EINVAL, "a path entered a fifth nested medium; the media stack holds four"};
}

void *DeviceArena::alloc(size_t n) {
  void *p = nullptr;
  size_t sz = n ? (n + 255) & ~size_t(255) : 256;
  cudaError_t e = cudaMalloc(&p, sz);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error{e == cudaErrorMemoryAllocation ? SNOG_ENOMEM : SNOG_ECUDA,
                std::string("cudaMalloc: ") + cudaGetErrorString(e)};
  }
  blocks.push_back(p);
  bytes += sz;
  return p;
}

void *DeviceArena::upload(const void *src, size_t n) {
  void *p = alloc(n);
  if (n) check_cuda(cudaMemcpy(p, src, n, cudaMemcpyHostToDevice), "upload");
  return p;
}

void DeviceArena::release() {
  for (void *p : blocks) cudaFree(p);
  blocks.clear();
  bytes = 0;
}

namespace {

struct V3 {
  float x, y, z;
};
inline V3 v3(const float *p) { return V3{p[0], p[1], p[2]}; }
inline V3 vsub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 vadd(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 vcross(V3 a, V3 b) {
  return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline float vlen2(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
inline V3 vunit(V3 a) {
  float l = std::sqrt(vlen2(a));
  float s = 1 / l;
  return V3{a.x * s, a.y * s, a.z * s};
}
inline V3 vperp(V3 v) {   // geometry/vec.h:122-129
  float nz = (v.x == v.z) ? v.z : -v.z;
  return V3{v.y * v.y + v.x * nz, -nz * nz - v.x * v.y, v.x * v.x - v.y * nz};
}

struct BoxAcc {
  float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  bool empty = true;
  void add(V3 p) {   // BBox += Pos with snogray::min/max (geometry/bbox.h:58-63)
    float c[3] = {p.x, p.y, p.z};
    if (empty) {
      for (int k = 0; k < 3; k++) lo[k] = hi[k] = c[k];
      empty = false;
      return;
    }
    for (int k = 0; k < 3; k++) {
      lo[k] = lo[k] < c[k] ? lo[k] : c[k];
      hi[k] = hi[k] > c[k] ? hi[k] : c[k];
    }
  }
  void add(const Box3 &b) {
    add(V3{b.lo[0], b.lo[1], b.lo[2]});
    add(V3{b.hi[0], b.hi[1], b.hi[2]});
  }
};

Box3 box_of_points(std::initializer_list<V3> pts) {
  BoxAcc a;
  for (V3 p : pts) a.add(p);
  Box3 b;
  for (int k = 0; k < 3; k++) {
    b.lo[k] = a.lo[k];
    b.hi[k] = a.hi[k];
  }
  return b;
}

void fail(const std::string &m) { throw Error{SNOG_EINVAL, m}; }

// The 16-byte device node (snog_common.h): breadth-first numbering gives the
// children of a node consecutive ids in octant order, checked here.  The
// surface lists are copied to PLIST4 with every list starting at a multiple
// of 4 entries and padded with PREF_END to one.
std::vector<uint4> compact_nodes(const OctreeArrays &o, std::vector<uint32_t> &plist4) {
  const size_t n = o.heads.size();
  std::vector<uint4> out(n);
  plist4.assign(4, PREF_END);
  for (size_t i = 0; i < n; i++) {
    const uint32_t *k = &o.children[8 * i];
    uint4 r{0, 0, o.heads[i], 0};
    const bool leaf = k[0] == 1 && k[1] == 1;
    if (!leaf) {
      uint32_t expect = 0;
      for (uint32_t s = 0; s < 8; s++) {
        if (!k[s]) continue;
        if (r.y == 0) {
          r.x = k[s];
          expect = k[s];
        }
        if (k[s] != expect) throw Error{SNOG_EINVAL, "octree children not consecutive"};
        expect++;
        r.y |= 1u << s;
      }
    }
    if (r.z) {
      const uint32_t start = uint32_t(plist4.size());
      for (uint32_t e = r.z; o.plist[e] != PREF_END; e++) {
        plist4.push_back(o.plist[e]);
        r.w++;
      }
      while (plist4.size() % 4) plist4.push_back(PREF_END);
      r.z = start;
    }
    out[i] = r;
  }
  return out;
}

template <class T>
T *dev_upload(DeviceArena &a, const std::vector<T> &v) {
  return static_cast<T *>(a.upload(v.data(), v.size() * sizeof(T)));
}

}  // namespace

SceneImpl *build_scene(const SnogSceneDesc &d, bool upload, uint32_t octree_mode) {
  auto t_start = std::chrono::steady_clock::now();
  // Bits 8-9: the SNOG_LISTS_* dealing; the low byte: the octree builder.
  const uint32_t lists_mode = octree_mode & 0x300u;
  octree_mode &= 0xffu;
  // ---- validation --------------------------------------------------------
  if (d.n_materials == 0 || !d.materials) fail("scene has no materials");
  for (uint32_t i = 0; i < d.n_materials; i++) {
    const SnogMaterial &m = d.materials[i];
    if (m.type > SNOG_GLOW) fail("material " + std::to_string(i) + ": unknown type");
    if (m.type == SNOG_GLOW && m.underlying >= int32_t(i))
      fail("material " + std::to_string(i) + ": underlying must be an earlier material");
  }
  if (d.n_triangles && (!d.triangles || !d.tri_material || !d.vertices))
    fail("triangles given without vertex/index/material arrays");
  for (uint32_t t = 0; t < d.n_triangles; t++) {
    for (int k = 0; k < 3; k++)
      if (d.triangles[3 * size_t(t) + k] >= d.n_vertices)
        fail("triangle " + std::to_string(t) + ": vertex index out of range");
    if (d.tri_material[t] >= d.n_materials) fail("triangle material out of range");
    if (t && d.tri_material[t] < d.tri_material[t - 1])
      fail("tri_material must be non-decreasing (mesh parts are contiguous runs)");
  }
  for (uint32_t i = 0; i < d.n_spheres; i++)
    if (d.spheres[i].material >= d.n_materials) fail("sphere material out of range");
  for (uint32_t i = 0; i < d.n_tripars; i++)
    if (d.tripars[i].material >= d.n_materials) fail("tripar material out of range");
  if (d.env_width || d.env_height) {
    if (!d.env_rgb || d.env_width != 2 * d.env_height || d.env_height == 0)
      fail("envmap must be a lat-long image with width == 2 * height");
  }
  if (d.n_triangles + d.n_spheres + d.n_tripars == 0) fail("scene has no surfaces");
  if (d.vertex_normals)
    for (uint32_t v = 0; v < 3 * d.n_vertices; v++)
      if (!std::isfinite(d.vertex_normals[v])) fail("vertex normal " + std::to_string(v / 3) + " is not finite");
  if (uint64_t(d.n_triangles) + d.n_spheres + d.n_tripars >= (1ull << 31))
    fail("too many primitives (limit 2^31)");

  std::unique_ptr<SceneImpl> sc(new SceneImpl);
  if (upload) check_cuda(cudaGetDevice(&sc->device), "cudaGetDevice");
  SceneImpl &S = *sc;
  S.n_tri = d.n_triangles;
  S.n_sph = d.n_spheres;
  S.n_tpar = d.n_tripars;

  // ---- materials and media ---------------------------------------------
  std::vector<DevMaterial> mats(d.n_materials);
  std::vector<DevMedium> media(1, DevMedium{1.0f, {0, 0, 0}});   // default medium
  for (uint32_t i = 0; i < d.n_materials; i++) {
    const SnogMaterial &m = d.materials[i];
    DevMaterial &o = mats[i];
    std::memset(&o, 0, sizeof(o));
    o.type = m.type;
    o.underlying = m.type == SNOG_GLOW ? m.underlying : -1;
    for (int k = 0; k < 3; k++) {
      o.color[k] = m.color[k];
      o.gloss[k] = m.gloss[k];
      o.absorb[k] = m.absorb[k];
    }
    o.m = m.m;
    o.ior_n = m.ior_n;
    o.ior_k = m.ior_k;
    if (m.type == SNOG_MIRROR) {
      // Mirror's underlying Lambert exists unless the colour is (summed)
      // below Eps (material/mirror.cc:28-31, color.h:256-264).
      float sum = m.color[0] + m.color[1] + m.color[2];
      o.has_lambert = !(sum < 3 * 1e-15f);
    }
    if (m.type == SNOG_GLASS) {
      // A medium is its ior and absorption (material/medium.h:23-58), so
      // glass materials with equal ones share a medium id.  The path state
      // holds 5-bit ids: at most 31 distinct media besides the default.
      const DevMedium md{m.ior_n, {m.absorb[0], m.absorb[1], m.absorb[2]}};
      uint32_t id = 1;
      while (id < media.size() && !(media[id].ior == md.ior && media[id].absorb[0] == md.absorb[0] &&
                                    media[id].absorb[1] == md.absorb[1] && media[id].absorb[2] == md.absorb[2]))
        id++;
      if (id == media.size()) {
        if (media.size() == 32) throw Error{SNOG_EINVAL, "more than 31 distinct glass media (ior, absorb)"};
        media.push_back(md);
      }
      o.medium_id = id;
    }
    if (m.type == SNOG_GLOW && m.underlying >= 0) o.medium_id = mats[m.underlying].medium_id;
  }

  // ---- primitives, bounding boxes, octree -------------------------------
  // One 48-byte record per primitive, indexed by primitive id; the octree
  // lists hold those ids (snog_common.h).
  BoxAcc scene_box, mesh_box;
  const size_t n_prims = size_t(d.n_triangles) + d.n_spheres + d.n_tripars;
  std::vector<float4> prims(3 * n_prims, make_float4(0.f, 0.f, 0.f, 0.f));
  std::vector<uint32_t> prim_mat(n_prims);
  auto put = [&](size_t id, float4 a, float4 b, float4 c, uint32_t mat) {
    prims[3 * id] = a;
    prims[3 * id + 1] = b;
    prims[3 * id + 2] = c;
    prim_mat[id] = mat;
  };
  // The octree is built on the host (OctreeBuilder, surface by surface) or
  // on the device (build_octree_device, the same tree from the surfaces'
  // boxes in insertion order).
  const bool dev_oct = upload && (octree_mode == SNOG_OCTREE_DEVICE ||
                                  (octree_mode == SNOG_OCTREE_AUTO && n_prims >= kDeviceOctreeMinSurfaces));
  OctreeBuilder ob;
  std::vector<Box3> oct_boxes;
  std::vector<uint32_t> oct_refs;
  if (dev_oct) {
    oct_boxes.reserve(n_prims);
    oct_refs.reserve(n_prims);
  }
  auto oct_add = [&](uint32_t ref, const Box3 &b) {
    if (dev_oct) {
      oct_boxes.push_back(b);
      oct_refs.push_back(ref);
    } else {
      ob.add(ref, b);
    }
  };
  for (uint32_t v = 0; v < d.n_vertices; v++) mesh_box.add(v3(d.vertices + 3 * size_t(v)));
  for (uint32_t t = 0; t < d.n_triangles; t++) {
    const uint32_t *ix = d.triangles + 3 * size_t(t);
    V3 p0 = v3(d.vertices + 3 * size_t(ix[0])), p1 = v3(d.vertices + 3 * size_t(ix[1])),
       p2 = v3(d.vertices + 3 * size_t(ix[2]));
    V3 e1 = vsub(p1, p0), e2 = vsub(p2, p0);
    put(t, make_float4(p0.x, p0.y, p0.z, float(PRIM_TRI)), make_float4(e1.x, e1.y, e1.z, 0.f),
        make_float4(e2.x, e2.y, e2.z, 0.f), d.tri_material[t]);
    // Degenerate triangles are left out of the space (surface/mesh.cc:833-846);
    // the mesh is left-handed, normal = e2 x e1 (surface/mesh.h:55).
    if (vlen2(vcross(e2, e1)) > 0) oct_add(t, box_of_points({p0, p1, p2}));
  }
  if (d.n_triangles) scene_box.add(Box3{{mesh_box.lo[0], mesh_box.lo[1], mesh_box.lo[2]},
                                       {mesh_box.hi[0], mesh_box.hi[1], mesh_box.hi[2]}});
  for (uint32_t i = 0; i < d.n_spheres; i++) {
    const SnogSphere &s = d.spheres[i];
    const uint32_t id = d.n_triangles + i;
    put(id, make_float4(s.center[0], s.center[1], s.center[2], float(PRIM_SPHERE)),
        make_float4(s.radius, 0.f, 0.f, 0.f), make_float4(0.f, 0.f, 0.f, 0.f), s.material);
    float r = s.radius;
    Box3 b{{s.center[0] - r, s.center[1] - r, s.center[2] - r},
           {s.center[0] + r, s.center[1] + r, s.center[2] + r}};   // surface/sphere.cc:164-170
    scene_box.add(b);
    oct_add(id, b);
  }
  for (uint32_t i = 0; i < d.n_tripars; i++) {
    const SnogTripar &p = d.tripars[i];
    const uint32_t id = d.n_triangles + d.n_spheres + i;
    V3 v0 = v3(p.v0), e1 = v3(p.e1), e2 = v3(p.e2);
    put(id, make_float4(v0.x, v0.y, v0.z, float(p.parallelogram ? PRIM_PARALLELOGRAM : PRIM_TRIPAR)),
        make_float4(e1.x, e1.y, e1.z, 0.f), make_float4(e2.x, e2.y, e2.z, 0.f), p.material);
    Box3 b = p.parallelogram ? box_of_points({v0, vadd(v0, e1), vadd(v0, e2), vadd(vadd(v0, e1), e2)})
                             : box_of_points({v0, vadd(v0, e1), vadd(v0, e2)});   // surface/tripar.cc:188-197
    scene_box.add(b);
    oct_add(id, b);
  }
  if (!dev_oct) S.oct = ob.finish();

  // ---- light samplers, in the reference's order -------------------------
  std::vector<DevLight> lights;
  auto glow_color = [&](uint32_t mi, float out[3]) {
    for (int k = 0; k < 3; k++) out[k] = d.materials[mi].color[k];
  };
  for (uint32_t i = 0; i < d.n_spheres; i++)
    if (d.materials[d.spheres[i].material].type == SNOG_GLOW) {
      DevLight L{};
      L.type = LS_SPHERE;
      for (int k = 0; k < 3; k++) L.p[k] = d.spheres[i].center[k];
      L.p[3] = d.spheres[i].radius;
      glow_color(d.spheres[i].material, L.intensity);
      lights.push_back(L);
    }
  for (uint32_t i = 0; i < d.n_tripars; i++)
    if (d.materials[d.tripars[i].material].type == SNOG_GLOW) {
      DevLight L{};
      L.type = LS_TRIPAR;
      L.flags = d.tripars[i].parallelogram ? 1 : 0;
      for (int k = 0; k < 3; k++) {
        L.p[k] = d.tripars[i].v0[k];
        L.p[3 + k] = d.tripars[i].e1[k];
        L.p[6 + k] = d.tripars[i].e2[k];
      }
      glow_color(d.tripars[i].material, L.intensity);
      lights.push_back(L);
    }
  for (uint32_t i = 0; i < d.n_point_lights; i++) {
    const SnogPointLight &pl = d.point_lights[i];
    DevLight L{};
    L.type = LS_POINT;
    for (int k = 0; k < 3; k++) {
      L.p[k] = pl.pos[k];
      L.intensity[k] = pl.color[k];
    }
    if (pl.angle >= 2 * 3.14159265f) {   // PointLight (pos, col): omni (light/point-light.h:32-34)
      L.p[3] = 0; L.p[4] = 0; L.p[5] = 1;
      L.a = -1;
      L.b = -1;
    } else {                             // light/point-light.h:42-47
      for (int k = 0; k < 3; k++) L.p[3 + k] = pl.dir[k];
      L.a = std::cos(pl.angle / 2);
      L.b = std::cos((pl.angle - pl.fringe_angle) / 2);
    }
    lights.push_back(L);
  }
  for (uint32_t i = 0; i < d.n_far_lights; i++) {
    const SnogFarLight &fl = d.far_lights[i];
    DevLight L{};
    L.type = LS_FAR;
    V3 z = vunit(v3(fl.dir));            // Frame (dir.unit ()) (geometry/frame.h:50-55)
    V3 x = vunit(vperp(z));
    V3 y = vunit(vcross(z, x));
    float f[9] = {x.x, x.y, x.z, y.x, y.y, y.z, z.x, z.y, z.z};
    std::memcpy(L.p, f, sizeof f);
    for (int k = 0; k < 3; k++) L.intensity[k] = fl.color[k];
    L.a = fl.angle == 0 ? 1.0f : std::cos(fl.angle / 2);   // light/far-light.h:39-45
    lights.push_back(L);
  }
  uint32_t env_light = ~0u;
  std::vector<float4> texels;
  std::vector<float> row_cdf, col_cdf;
  uint32_t lw = 0, lh = 0;
  if (d.env_width) {
    DevLight L{};
    L.type = LS_ENV;
    env_light = uint32_t(lights.size());
    lights.push_back(L);
    const uint32_t w = d.env_width, h = d.env_height;
    texels.resize(size_t(w) * h);
    for (size_t i = 0; i < size_t(w) * h; i++)
      texels[i] = make_float4(d.env_rgb[3 * i], d.env_rgb[3 * i + 1], d.env_rgb[3 * i + 2], 0.f);
    // Light map: box-downsampled to at most 1024 on a side, rows flipped
    // (texture/spheremap.cc:32-71).
    uint32_t div = 1;
    while (w / div > 1024 || h / div > 1024) div++;
    lw = w / div;
    lh = h / div;
    const float avg_scale = 1.f / float(div * div);
    std::vector<float> lmap(size_t(lw) * lh * 3, 0.f);
    for (uint32_t y = 0; y < h; y++)
      for (uint32_t x = 0; x < w; x++) {
        uint32_t lx = x / div, ly = lh - y / div - 1;
        if (lx >= lw || ly >= lh) continue;
        const float *c = d.env_rgb + 3 * (size_t(y) * w + x);
        float *o = &lmap[3 * (size_t(ly) * lw + lx)];
        for (int k = 0; k < 3; k++) o[k] = o[k] + c[k] * avg_scale;
      }
    // Histogram of intensity x cos(latitude), then the double-precision
    // cumulative sums of Hist2dDist (light/envmap-light.cc:103-140,
    // geometry/hist-2d-dist.cc:65-120).
    std::vector<float> bins(size_t(lw) * lh, 0.f);
    const double kPi = 3.14159265358979323846;
    double row_lat_inc = kPi / lh;
    double row_lat = -kPi / 2 + row_lat_inc / 2;
    for (uint32_t row = 0; row < lh; row++) {
      double row_scale = std::cos(row_lat);
      for (uint32_t col = 0; col < lw; col++) {
        const float *c = &lmap[3 * (size_t(row) * lw + col)];
        float inten = (c[0] + c[1] + c[2]) / 3;
        bins[size_t(row) * lw + col] += float(double(inten) * row_scale);
      }
      row_lat += row_lat_inc;
    }
    double bin_sum = 0;
    for (size_t i = 0; i < bins.size(); i++) bin_sum += double(bins[i]);
    double inv_bin_sum = bin_sum == 0 ? 0 : 1 / bin_sum;
    row_cdf.resize(lh);
    col_cdf.resize(size_t(lw) * lh);
    double norm_sum = 0;
    for (uint32_t row = 0; row < lh; row++) {
      for (uint32_t col = 0; col < lw; col++) norm_sum += double(bins[size_t(row) * lw + col]) * inv_bin_sum;
      row_cdf[row] = float(norm_sum);
    }
    for (uint32_t row = 0; row < lh; row++) {
      double row_sum = 0;
      for (uint32_t col = 0; col < lw; col++) row_sum += double(bins[size_t(row) * lw + col]);
      double inv_row_sum = row_sum == 0 ? 0 : 1 / row_sum;
      double acc = 0;
      for (uint32_t col = 0; col < lw; col++) {
        acc += double(bins[size_t(row) * lw + col]) * inv_row_sum;
        col_cdf[size_t(row) * lw + col] = float(acc);
      }
    }
  }

  // ---- scene scalars ------------------------------------------------------
  for (int k = 0; k < 3; k++) {
    S.bbox_min[k] = scene_box.lo[k];
    S.bbox_max[k] = scene_box.hi[k];
  }
  V3 ext{scene_box.hi[0] - scene_box.lo[0], scene_box.hi[1] - scene_box.lo[1],
         scene_box.hi[2] - scene_box.lo[2]};
  float horizon = std::sqrt(vlen2(ext));   // render/scene.cc:28, geometry/bbox.h:102-105

  // ---- upload ------------------------------------------------------------
  DevScene &D = S.dev;
  std::memset(&D, 0, sizeof(D));
  DeviceArena &A = S.arena;
  if (upload) try {
    DeviceOctree dov;
    bool built = false;
    if (dev_oct) {
      try {
        build_octree_device(oct_boxes, oct_refs, A, dov);
        built = true;
      } catch (const Error &e) {
        // Trees the device builder does not take (root grown more than 40
        // times, deeper than 40 levels, or a descent wider than its stack)
        // go to the host builder in AUTO mode.  The device builder finds
        // these before it allocates its outputs in the scene's arena.
        if (octree_mode != SNOG_OCTREE_AUTO || e.code != SNOG_EINVAL) throw;
        for (size_t i = 0; i < oct_boxes.size(); i++) ob.add(oct_refs[i], oct_boxes[i]);
        S.oct = ob.finish();
      }
    }
    if (built) {
      D.nodes = dov.nodes;
      D.plist = dov.plist;
      S.oct_device = true;
      S.oct_nodes = dov.n_nodes;
      S.oct_plist4 = dov.n_plist4;
      S.oct.origin[0] = dov.origin[0];
      S.oct.origin[1] = dov.origin[1];
      S.oct.origin[2] = dov.origin[2];
      S.oct.size = dov.size;
      S.oct.max_depth = dov.max_depth;
      S.oct.n_leaf = dov.n_leaf;
      S.oct.n_list_surfaces = dov.n_list_surfaces;
      S.oct_plist_host = dov.n_plist_host;
    } else {
      std::vector<uint32_t> plist4;
      std::vector<uint4> nodes = compact_nodes(S.oct, plist4);
      D.nodes = dev_upload(A, nodes);
      D.plist = dev_upload(A, plist4);
      S.oct_plist4 = uint32_t(plist4.size());
    }
    D.prims = dev_upload(A, prims);
    {
      float4 *lrec = static_cast<float4 *>(A.alloc(size_t(S.oct_plist4) * 48));
      check_cuda(build_list_records(D.plist, S.oct_plist4, D.prims, lrec, nullptr), "list records");
      check_cuda(cudaStreamSynchronize(nullptr), "list records");
      D.lrec = lrec;
    }
    D.prim_mat = dev_upload(A, prim_mat);
    if (d.vertex_normals && d.n_triangles) {
      std::vector<float4> vn(d.n_vertices);
      for (uint32_t v = 0; v < d.n_vertices; v++)
        vn[v] = make_float4(d.vertex_normals[3 * size_t(v)], d.vertex_normals[3 * size_t(v) + 1],
                            d.vertex_normals[3 * size_t(v) + 2], 0.f);
      std::vector<uint4> vi(d.n_triangles);
      for (uint32_t t = 0; t < d.n_triangles; t++)
        vi[t] = make_uint4(d.triangles[3 * size_t(t)], d.triangles[3 * size_t(t) + 1], d.triangles[3 * size_t(t) + 2], 0u);
      D.vnormals = dev_upload(A, vn);
      D.tri_vidx = dev_upload(A, vi);
    }
    D.mats = dev_upload(A, mats);
    D.lights = dev_upload(A, lights);
    D.media = dev_upload(A, media);
    D.env_texels = dev_upload(A, texels);
    D.env_row_cdf = dev_upload(A, row_cdf);
    D.env_col_cdf = dev_upload(A, col_cdf);
  } catch (...) {
    A.release();
    throw;
  }
  S.on_device = upload;
  D.n_nodes = S.oct_device ? S.oct_nodes : uint32_t(S.oct.heads.size());
  D.n_tri = d.n_triangles;
  D.n_sph = d.n_spheres;
  D.n_tpar = d.n_tripars;
  D.n_mats = d.n_materials;
  D.n_lights = uint32_t(lights.size());
  D.n_media = uint32_t(media.size());
  D.env_light = env_light;
  D.env_w = d.env_width;
  D.env_h = d.env_height;
  D.lmap_w = lw;
  D.lmap_h = lh;
  std::memcpy(D.env_frame, d.env_frame, sizeof D.env_frame);
  for (int k = 0; k < 3; k++) {
    D.origin[k] = S.oct.origin[k];
    D.bbox_min[k] = scene_box.lo[k];
    D.bbox_max[k] = scene_box.hi[k];
    // midpoint (mesh._bbox.min, mesh._bbox.max), used by the triangle
    // tangent-frame fallback (surface/mesh.cc:577-594).
    D.mesh_center[k] = mesh_box.lo[k] + (mesh_box.hi[k] - mesh_box.lo[k]) / 2;
  }
  D.size = S.oct.size;
  D.horizon = horizon;
  D.max_depth = S.oct.max_depth;
  D.right_handed = d.mesh_right_handed ? 1u : 0u;
  D.pair_lists = !upload                             ? 0u
                 : lists_mode == SNOG_LISTS_SINGLE ? 0u
                 : lists_mode == SNOG_LISTS_PAIRED ? 1u
                                                   : probe_pair_lists(D);

  SnogSceneInfo &I = S.info;
  std::memset(&I, 0, sizeof(I));
  I.n_nodes = D.n_nodes;
  I.n_plist = S.oct_device ? S.oct_plist_host : uint32_t(S.oct.plist.size());
  I.max_depth = S.oct.max_depth;
  I.n_leaf_nodes = S.oct.n_leaf;
  I.n_triangles = D.n_tri;
  I.n_spheres = D.n_sph;
  I.n_tripars = D.n_tpar;
  I.n_lights = D.n_lights;
  I.n_list_surfaces = S.oct.n_list_surfaces;
  for (int k = 0; k < 3; k++) {
    I.origin[k] = D.origin[k];
    I.bbox_min[k] = D.bbox_min[k];
    I.bbox_max[k] = D.bbox_max[k];
  }
  I.size = D.size;
  I.horizon = horizon;
  I.device_bytes = A.bytes;
  I.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
  I.pair_lists = D.pair_lists;
  return sc.release();
}

const OctreeArrays &host_octree(SceneImpl &S) {
  std::lock_guard<std::mutex> lk(S.mu);
  if (S.oct_device && S.oct.heads.empty() && S.oct_nodes) {
    check_cuda(cudaSetDevice(S.device), "cudaSetDevice");
    S.oct = octree_from_device(S.dev.nodes, S.oct_nodes, S.dev.plist, S.oct_plist4, S.oct.origin, S.oct.size,
                               S.oct.max_depth);
  }
  return S.oct;
}

}  // namespace snog
