// snog_common.h -- data layout shared by the host library and the sm_100a
// kernels: the flattened scene in HBM, the wavefront's path/ray records and
// the small float3 helpers both sides use.
//
// Layout of one scene in device memory (all arrays 16-byte aligned):
//   nodes          uint4[n_nodes]         BFS order: first child, child mask,
//                                         list start, list length (below)
//   plist          uint32[n_plist]        surface lists of primitive ids; each
//                                         list starts at a multiple of 4 and
//                                         is padded with PREF_END to one
//   lrec           float4[3 * n_plist]    the surface lists again, as the
//                                         primitives' 48-byte records in list
//                                         order with the id in c.w: a list
//                                         test reads one record, not an id
//                                         and then a record
//   prims          float4[3 * n_prims]    one 48-byte record per primitive,
//                                         indexed by primitive id (triangles,
//                                         then spheres, then tripars):
//                     triangle  a = corner, b = edge1, c = edge2 (edges
//                               precomputed with the same IEEE subtraction the
//                               reference does per test, surface/mesh.cc:735-736)
//                     sphere    a = centre, b.x = radius
//                     tripar    a = corner, b = edge1, c = edge2
//                               a.w holds the kind (PRIM_* below, as a float)
//   prim_mat       uint32[n_prims]        material index per primitive
//   vnormals       float4[n_vertices]     vertex normals (optional), with
//   tri_vidx       uint4[n_triangles]     each triangle's vertex indices
//   mats, lights, envmap texels and Hist2dDist cumulative sums

#ifndef SNOG_COMMON_H
#define SNOG_COMMON_H

#include <cstdint>

#include <cuda_runtime.h>   // vector types (float3, float4, uint4) on both sides

#ifdef __CUDACC__
#define SNOG_HD __host__ __device__ __forceinline__
#else
#define SNOG_HD inline
#include <cmath>
#endif

namespace snog {

// Primitive kinds, stored in the w component of a primitive record's first
// float4.
enum : uint32_t { PRIM_TRI = 0, PRIM_SPHERE = 1, PRIM_TRIPAR = 2, PRIM_PARALLELOGRAM = 3 };
constexpr uint32_t PREF_END = 0xffffffffu;   // ends a surface list

// Material kinds (same numbering as SnogMaterial::type in the C ABI).
enum : uint32_t { MAT_LAMBERT = 0, MAT_COOK_TORRANCE = 1, MAT_MIRROR = 2, MAT_GLASS = 3, MAT_GLOW = 4 };

// Light-sampler kinds, in the reference's sampler order: surface lights of
// glowing spheres and tripars in surface order, then explicit lights
// (surface/surface-group.cc:80-92).
enum : uint32_t { LS_TRIPAR = 0, LS_SPHERE = 1, LS_POINT = 2, LS_FAR = 3, LS_ENV = 4 };

struct DevMaterial {
  uint32_t type;
  int32_t underlying;      // Glow: index of the underlying material, or -1
  uint32_t has_lambert;    // Mirror: underlying Lambert present (mirror.cc:28-31)
  uint32_t medium_id;      // Glass: medium id (index into media table), else 0
  float color[3];          // Lambert / CT diffuse / Mirror underlying / Glow emission
  float gloss[3];          // CT gloss colour / Mirror reflectance
  float m;                 // CT rms slope
  float ior_n, ior_k;      // CT and Mirror surface Ior; Glass medium ior
  float absorb[3];         // Glass medium absorption
};

struct DevLight {
  uint32_t type;
  uint32_t flags;          // LS_TRIPAR: parallelogram
  float p[9];              // tripar v0,e1,e2 | sphere centre,r | point pos,dir |
                           // far frame x,y,z (9 floats)
  float intensity[3];
  float a, b;              // point: cos_half_angle, cos_half_core_angle;
                           // far: cos_half_angle
};

// Medium table entry (material/medium.h:30-58).  Entry 0 is the default
// medium (ior 1, no absorption) the camera starts in.
struct DevMedium {
  float ior;
  float absorb[3];
};

// One octree node in the device layout, 16 bytes (one 128-bit load).
// Breadth-first numbering gives a node's children consecutive ids in octant
// order, so the eight child ids of the reference's node
// (space/octree-node.h:27-86) reduce to the first child's id and an 8-bit
// mask: child(slot) = first + popc(mask & ((1 << slot) - 1)).
//   x = first child id, y = child mask (0 = leaf),
//   z = first entry of the surface list in plist, w = list length
struct DevScene {
  const uint4 *nodes;
  const uint32_t *plist;
  const float4 *lrec;         // 3 per plist slot: the primitive record of the slot's id, id in c.w
  const float4 *prims;
  const uint32_t *prim_mat;
  const DevMaterial *mats;
  const DevLight *lights;
  const DevMedium *media;
  const float4 *env_texels;   // env_w * env_h, row 0 = top image row
  const float *env_row_cdf;   // lmap_h
  const float *env_col_cdf;   // lmap_w * lmap_h
  uint32_t n_nodes, n_tri, n_sph, n_tpar;
  uint32_t n_mats, n_lights, n_media, env_light;   // env_light: light index or ~0u
  uint32_t env_w, env_h, lmap_w, lmap_h;
  float env_frame[9];
  float origin[3], size;      // octree root cube
  float bbox_min[3], bbox_max[3];
  float mesh_center[3];       // midpoint of the mesh bounding box (mesh.cc:581)
  float horizon;              // scene bbox diameter (render/scene.cc:28)
  uint32_t max_depth;         // octree depth, sizes the traversal stack
  uint32_t pair_lists;        // closest-hit rounds deal list entries in pairs (long lists along rays)
  uint32_t right_handed;      // mesh geometric normal e1 x e2 (else e2 x e1)
  const float4 *vnormals;     // per vertex, or null: no interpolated normals
  const uint4 *tri_vidx;      // per triangle, its vertex indices (with vnormals)
};

// -- float3 helpers --------------------------------------------------------
// Written as explicit single operations so that, in the files compiled with
// --fmad=false, every expression rounds exactly like the reference's
// TVec/TPos code evaluated left to right.

SNOG_HD float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
SNOG_HD float3 add(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
SNOG_HD float3 sub(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
SNOG_HD float3 mul(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
SNOG_HD float3 mul3(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
SNOG_HD float3 neg(float3 a) { return f3(-a.x, -a.y, -a.z); }
SNOG_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
SNOG_HD float3 cross(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
SNOG_HD float length_sq(float3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
SNOG_HD float length(float3 a) { return sqrtf(length_sq(a)); }
SNOG_HD float3 unit(float3 a) { return mul(a, 1.0f / length(a)); }
// TVec::perpendicular (geometry/vec.h:122-129).
SNOG_HD float3 perpendicular(float3 v) {
  float nz = (v.x == v.z) ? v.z : -v.z;
  return f3(v.y * v.y + v.x * nz, -nz * nz - v.x * v.y, v.x * v.x - v.y * nz);
}
SNOG_HD float3 load3(const float *p) { return f3(p[0], p[1], p[2]); }
SNOG_HD float3 xyz(float4 v) { return f3(v.x, v.y, v.z); }
SNOG_HD float fmin_ref(float a, float b) { return a < b ? a : b; }   // util/snogmath.h:43
SNOG_HD float fmax_ref(float a, float b) { return a > b ? a : b; }   // util/snogmath.h:48
SNOG_HD float csum(float3 c) { return c.x + c.y + c.z; }
SNOG_HD float intensity(float3 c) { return (c.x + c.y + c.z) / 3.0f; }  // color.h:160-165

}  // namespace snog

#endif
