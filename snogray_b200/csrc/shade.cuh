// shade.cuh -- per-vertex shading on the device: intersection frames, the
// four BSDFs, Fresnel, the light samplers (area tripar/sphere, point, far,
// lat-long envmap through Hist2dDist), MIS weights and the counter-based
// random numbers.
//
// Everything here follows the reference's formulas and branch structure
// (files cited per function), in single precision with every operation
// rounded on its own: the library is compiled with -fmad=false, so the same
// shading code inlined into the wave renderer and into the streaming engine
// gives the same bits and a job's image is the same on either.  Images are
// compared with the reference's statistically, not bit for bit.
//
// Vectors in "normal space" are expressed in the intersection's shading
// frame, whose z axis is the (possibly flipped) surface normal, as the
// reference's Bsdf and Light::Sampler interfaces use them.

#ifndef SNOG_SHADE_CUH
#define SNOG_SHADE_CUH

#include "snog_common.h"
#include "trace.cuh"

namespace snog {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.31830988618379067154f;

// Bsdf::Flags (material/bsdf.h:50-99).
enum : uint32_t {
  B_SPECULAR = 0x01, B_GLOSSY = 0x02, B_DIFFUSE = 0x04,
  B_REFLECTIVE = 0x10, B_TRANSMISSIVE = 0x20,
  B_ALL_LAYERS = 0x07, B_ALL_DIRECTIONS = 0x30, B_ALL = 0x37
};

// ---------------------------------------------------------------------------
// Counter-based random numbers.  A stream value is a hash of (seed, path,
// dimension); no state is carried between kernels.  The mixer is a
// multiply-xorshift permutation applied over the four 32-bit words (after
// the "pcg4d" construction of Jarzynski & Olano, "Hash Functions for GPU
// Rendering", JCGT 9(3), 2020).

__device__ __forceinline__ uint4 pcg4(uint4 v) {
  v.x = v.x * 1664525u + 1013904223u;
  v.y = v.y * 1664525u + 1013904223u;
  v.z = v.z * 1664525u + 1013904223u;
  v.w = v.w * 1664525u + 1013904223u;
  v.x += v.y * v.w; v.y += v.z * v.x; v.z += v.x * v.y; v.w += v.y * v.z;
  v.x ^= v.x >> 16; v.y ^= v.y >> 16; v.z ^= v.z >> 16; v.w ^= v.w >> 16;
  v.x += v.y * v.w; v.y += v.z * v.x; v.z += v.x * v.y; v.w += v.y * v.z;
  return v;
}

__device__ __forceinline__ float u01(uint32_t h) { return float(h >> 8) * (1.0f / 16777216.0f); }

struct Rng {
  uint32_t seed_lo, seed_hi, path_lo, path_hi;
  // Two independent uniforms in [0,1) for dimension DIM.
  __device__ __forceinline__ float2 uv(uint32_t dim) const {
    uint4 h = pcg4(make_uint4(path_lo, path_hi ^ (dim * 0x9E3779B9u), seed_lo ^ dim, seed_hi));
    return make_float2(u01(h.x), u01(h.y));
  }
  __device__ __forceinline__ float u(uint32_t dim) const { return uv(dim).x; }
};

// A bijection of [0, n) selected by KEY: invertible mixing steps on the
// smallest power-of-two domain covering n, cycle-walked until the value lands
// below n (the permutation construction of Kensler, "Correlated Multi-Jittered
// Sampling", Pixar Technical Memo 13-01, 2013; our own choice of steps).
__device__ __forceinline__ uint32_t permute(uint32_t i, uint32_t n, uint32_t key) {
  if (n <= 1) return 0;
  uint32_t w = n - 1;
  w |= w >> 1; w |= w >> 2; w |= w >> 4; w |= w >> 8; w |= w >> 16;
  do {
    i ^= key;
    i *= 0xe170893du;
    i ^= key >> 16;
    i ^= (i & w) >> 4;
    i ^= key >> 8;
    i *= 0x0929eb3fu;
    i ^= key >> 23;
    i ^= (i & w) >> 1;
    i *= 1u | key >> 27;
    i *= 0x6935fa69u;
    i ^= (i & w) >> 11;
    i *= 0x74dcb303u;
    i ^= (i & w) >> 2;
    i *= 0x9e501cc3u;
    i ^= (i & w) >> 2;
    i *= 0xc860a3dfu;
    i &= w;
    i ^= i >> 5;
  } while (i >= n);
  return i;
}

// A stratified UV for sample S of a pixel's N samples on channel CH: the
// reference's Grid generator jitters within a ceil(sqrt N) x round(sqrt N)
// grid and shuffles each channel independently per pixel
// (render/grid.cc:24-67, render/sample-set.cc:37-56); here the shuffle is a
// keyed permutation and the jitter a hash.
struct Strata {
  uint32_t n, u_steps, v_steps, cells;
};

__device__ __forceinline__ float2 strat_uv(const Strata &st, const Rng &rng, uint32_t pixel_key,
                                           uint32_t s, uint32_t ch) {
  uint32_t key = pcg4(make_uint4(pixel_key, ch, rng.seed_lo, rng.seed_hi ^ 0x5bd1e995u)).x;
  uint32_t cell = permute(s, st.cells, key);
  float2 j = rng.uv(ch ^ 0x40000000u);
  uint32_t cu = cell % st.u_steps, cv = cell / st.u_steps;
  float u = (float(cu) + j.x) / float(st.u_steps);
  float v = (float(cv) + j.y) / float(st.v_steps);
  return make_float2(fminf(u, 0.99999994f), fminf(v, 0.99999994f));
}

// ---------------------------------------------------------------------------
// Frames.

struct Frame3 {
  float3 x, y, z;
  __device__ __forceinline__ float3 to(float3 v) const { return f3(dot(v, x), dot(v, y), dot(v, z)); }
  __device__ __forceinline__ float3 from(float3 v) const {
    return f3(x.x * v.x + y.x * v.y + z.x * v.z, x.y * v.x + y.y * v.y + z.y * v.z,
              x.z * v.x + y.z * v.y + z.z * v.z);
  }
};

// Everything the reference's Intersect carries that shading reads
// (render/intersect.h, render/intersect.cc:87-136).
struct Isec {
  float3 pos;          // normal_frame.origin
  Frame3 nf;           // normal frame (z flipped for back-face hits)
  float3 v;            // eye vector in the normal frame, v.z >= 0
  float3 geom_n;       // geometric normal in the normal frame, z >= 0
  bool back;
  uint32_t mat;        // material index
  __device__ __forceinline__ float cos_n(float3 d) const { return d.z; }
  __device__ __forceinline__ float cos_geom_n(float3 d) const { return dot(d, geom_n); }
};

// Triangle tangent frame (surface/mesh.cc:563-603), mesh axis (0,0,1).
__device__ __forceinline__ Frame3 tri_frame(const DevScene &s, float3 pos, float3 n) {
  float3 t = cross(n, f3(0.f, 0.f, 1.f));
  if (length_sq(t) < 1e-15f) {
    float3 cent = sub(load3(s.mesh_center), pos);
    t = cross(n, cent);
    if (length_sq(t) < 1e-15f) t = perpendicular(n);
  }
  t = unit(t);
  return Frame3{t, cross(t, n), n};
}

// IsecInfo::make_intersect + Intersect::finish_init for the three kinds
// (surface/mesh.cc:607-709, surface/sphere.cc:48-90, surface/tripar.cc:45-73).
__device__ __forceinline__ Isec make_isec(const DevScene &s, uint32_t ref, float3 o, float3 d, float t) {
  Isec I;
  I.pos = add(o, mul(d, t));
  const PrimRec r = load_prim(s, ref);
  I.mat = __ldg(s.prim_mat + ref);
  Frame3 f, nf;
  if (r.a.w == float(PRIM_TRI)) {
    // Triangle::raw_normal: e2 x e1 for a left-handed mesh, e1 x e2 for a
    // right-handed one (surface/mesh.cc:264-271), each in its own operand
    // order (negating the other would flip the sign of zero components).
    const float3 gn = unit(s.right_handed ? cross(xyz(r.b), xyz(r.c)) : cross(xyz(r.c), xyz(r.b)));
    f = tri_frame(s, I.pos, gn);
    nf = f;
    if (s.vnormals) {
      // Interpolated vertex normal at the hit's barycentrics (the same u, v
      // the intersection test computed; they do not depend on the ray's
      // extent), and the geometric normal turned to agree with it
      // (surface/mesh.cc:616-637).
      float th, u = 0.f, v = 0.f;
      tripar_hit(xyz(r.a), xyz(r.b), xyz(r.c), false, o, d, -INFINITY, INFINITY, th, u, v);
      const uint4 vi = __ldg(s.tri_vidx + ref);
      float3 n = mul(xyz(__ldg(s.vnormals + vi.x)), 1.f - u - v);
      n = add(n, mul(xyz(__ldg(s.vnormals + vi.y)), u));
      n = add(n, mul(xyz(__ldg(s.vnormals + vi.z)), v));
      n = unit(n);
      if (dot(n, f.z) < 0.f) f.z = neg(f.z);
      nf = tri_frame(s, I.pos, n);
    }
  } else if (r.a.w == float(PRIM_SPHERE)) {
    float3 n = unit(sub(I.pos, xyz(r.a)));
    float3 tt = cross(n, f3(0.f, 0.f, 1.f));
    if (length_sq(tt) < 1e-15f) tt = perpendicular(n);
    tt = unit(tt);
    f = Frame3{tt, cross(tt, n), n};
    nf = f;
  } else {
    float3 e1 = xyz(r.b), e2 = xyz(r.c);
    float3 n = unit(cross(e2, e1));
    float3 sx = mul(e1, 1.0f / length(e1));
    f = Frame3{sx, cross(sx, n), n};
    nf = f;
  }
  // Intersect::finish_init (render/intersect.cc:84-136); no bump maps.
  float3 wv = neg(unit(d));
  I.nf = nf;
  I.v = nf.to(wv);
  float gvz = dot(wv, f.z);
  I.back = gvz < 0.f;
  if (I.back) {
    I.v.z = -I.v.z;
    I.nf.z = neg(I.nf.z);
  }
  I.geom_n = I.nf.to(f.z);
  I.geom_n.z = fabsf(I.geom_n.z);
  return I;
}

// ---------------------------------------------------------------------------
// Sampling helpers.

// z_axis_cos_spherical_to_vec (geometry/spherical-coords.h:157-168).
__device__ __forceinline__ float3 cos_sph_to_vec(float cos_colat, float lng) {
  float sin_lat = cos_colat;
  float cos_lat = sqrtf(fmaxf(0.f, 1.f - sin_lat * sin_lat));
  float cos_lng = cosf(lng);
  float sin_lng = sqrtf(fmaxf(0.f, 1.f - cos_lng * cos_lng));
  if (lng < 0.f || lng > kPi) sin_lng = -sin_lng;
  return f3(cos_lng * cos_lat, -sin_lng * cos_lat, sin_lat);
}

// Dist::z_normal_symm_vec (material/dist.h).
__device__ __forceinline__ float3 z_symm_vec(float cos_theta, float v) {
  return cos_sph_to_vec(cos_theta, v * 2.f * kPi);
}

// Fresnel::reflectance (material/fresnel.h:75-166) for relative ior n + ik.
__device__ __forceinline__ float fresnel(float n, float k, float cos_refl) {
  cos_refl = fabsf(fminf(fmaxf(cos_refl, -1.f), 1.f));
  float refl_angle = acosf(cos_refl);
  float Rs, Rp;
  if (k == 0.f) {
    float sin_t = fminf(fmaxf(sinf(refl_angle) / n, -1.f), 1.f);
    float cos_t = sqrtf(1.f - sin_t * sin_t);
    float nc1 = n * cos_refl, nc2 = n * cos_t;
    float Fs = (nc1 - cos_t) / (nc1 + cos_t);
    float Fp = (cos_refl - nc2) / (cos_refl + nc2);
    Rs = Fs * Fs;
    Rp = Fp * Fp;
  } else {
    float n2k2 = n * n * k * k, n2_m_k2 = n * n - k * k;
    float sin_r = sinf(refl_angle);
    float q = n2_m_k2 - sin_r * sin_r;
    float sin_tan = sin_r * tanf(refl_angle);
    float common = sqrtf(q * q + 4.f * n2k2);
    float a2 = (common + q) / 2.f, b2 = (common - q) / 2.f;
    float a2pb2 = a2 + b2, a = sqrtf(a2);
    float t1 = a2pb2 + cos_refl * cos_refl, t2 = 2.f * a * cos_refl;
    Rs = (t1 - t2) / (t1 + t2);
    float p1 = a2pb2 + sin_tan * sin_tan, p2 = 2.f * a * sin_tan;
    Rp = Rs * ((p1 - p2) / (p1 + p2));
  }
  float r = (Rs + Rp) / 2.f;
  return fminf(fmaxf(r, 0.f), 1.f);
}

// Vec::refraction (geometry/vec.h:165-186).
__device__ __forceinline__ float3 refraction(float3 v, float3 n, float ior_in, float ior_out) {
  float ratio = ior_in / ior_out;
  float c1 = -dot(v, n);
  float c2_sq = 1.f - (ratio * ratio) * (1.f - c1 * c1);
  if (c2_sq < -1e-15f) return f3(0.f, 0.f, 0.f);
  if (c2_sq < 0.f) c2_sq = 0.f;
  return add(mul(v, ratio), mul(n, ratio * c1 - sqrtf(c2_sq)));
}

// mis_sample_weight, power heuristic (render/mis-sample-weight.h:46-77).
__device__ __forceinline__ float mis_weight(float pdf, float other_pdf) {
  float term = pdf, other = other_pdf;
  if (term > 1e10f) return 1.f;
  if (other > 1e10f) return 0.f;
  return (term * pdf) / (term * term + other * other);
}

// ---------------------------------------------------------------------------
// BSDFs (samples and values in normal space).

struct BSample {
  float3 val;
  float pdf;
  float3 dir;
  uint32_t flags;
};

struct BsdfCtx {
  const DevMaterial *m;     // the material whose BSDF this is (Glow resolved)
  float medium_ior;         // ior of the medium the ray travels in
  float enclosing_ior;      // ior of the medium enclosing that one
};

// Lambert (material/lambert.cc:28-86) with the CosDist (material/cos-dist.h).
__device__ __forceinline__ BSample lambert_sample(const Isec &I, float3 color, float2 prm, uint32_t flags) {
  BSample r{f3(0.f, 0.f, 0.f), 0.f, f3(0.f, 0.f, 1.f), 0u};
  if ((flags & (B_REFLECTIVE | B_DIFFUSE)) == (B_REFLECTIVE | B_DIFFUSE)) {
    float ct = sqrtf(prm.x);
    float pdf = ct * kInvPi;
    float3 dir = z_symm_vec(ct, prm.y);
    if (I.cos_n(dir) > 0.f && I.cos_geom_n(dir) > 0.f) {
      r.val = mul(color, kInvPi);
      r.pdf = pdf;
      r.dir = dir;
      r.flags = B_REFLECTIVE | B_DIFFUSE;
    }
  }
  return r;
}

// Ward isotropic distribution (material/ward-dist.h:22-81).
__device__ __forceinline__ float ward_pdf(float m, float cos_t) {
  if (cos_t == 0.f) return 0.f;
  float inv_m2 = m == 0.f ? 0.f : 1.f / (m * m);
  float ic = 1.f / cos_t, ic2 = ic * ic, ic3 = ic2 * ic;
  float tan2 = ic2 - 1.f;
  return inv_m2 * kInvPi * ic3 * expf(-tan2 * inv_m2);
}

struct CT {
  float m, diff_weight, inv_diff_weight, inv_gloss_weight, nv, inv_4_nv;
  float fn, fk;             // Fresnel (medium ior -> material ior)
  uint32_t gloss_layer, have_layers;
  float3 diff, gloss;
};

// CookTorranceBsdf construction (material/cook-torrance.cc:44-62).
__device__ __forceinline__ CT make_ct(const Isec &I, const DevMaterial &M, float medium_ior) {
  CT c;
  c.m = M.m;
  c.diff = load3(M.color);
  c.gloss = load3(M.gloss);
  float di = intensity(c.diff), gi = intensity(c.gloss);
  c.diff_weight = (di + gi) == 0.f ? 0.f : di / (di + gi);
  c.inv_diff_weight = c.diff_weight == 0.f ? 0.f : 1.f / c.diff_weight;
  c.inv_gloss_weight = c.diff_weight == 1.f ? 0.f : 1.f / (1.f - c.diff_weight);
  c.fn = M.ior_n / medium_ior;   // Fresnel (n1, Ior) (material/fresnel.h:55-61)
  c.fk = M.ior_k / medium_ior;
  c.nv = I.cos_n(I.v);
  c.inv_4_nv = c.nv != 0.f ? 1.f / (4.f * c.nv) : 0.f;
  c.gloss_layer = c.m < 0.5f ? B_GLOSSY : B_DIFFUSE;
  c.have_layers = (c.diff_weight > 0.f ? B_DIFFUSE : 0u) | (c.diff_weight < 1.f ? c.gloss_layer : 0u);
  return c;
}

// CookTorranceBsdf::val (material/cook-torrance.cc:292-340).
__device__ __forceinline__ float3 ct_val(const CT &c, const Isec &I, float3 l, float3 h, uint32_t flags,
                                         float ddw, float &pdf) {
  float nl = I.cos_n(l);
  float3 col = f3(0.f, 0.f, 0.f);
  pdf = 0.f;
  if (flags & B_DIFFUSE) {
    pdf += nl * kInvPi * ddw;
    col = add(col, mul(c.diff, kInvPi));
  }
  if (flags & c.gloss_layer) {
    float nh = I.cos_n(h);
    float inv_nl = nl != 0.f ? 1.f / nl : 0.f;
    float vh = fminf(dot(I.v, h), 1.f);
    float G = fminf(2.f * nh * ((c.nv > nl) ? nl : c.nv) / vh, 1.f);
    float D = ward_pdf(c.m, nh);
    float g = fresnel(c.fn, c.fk, vh) * D * G * c.inv_4_nv * inv_nl;
    pdf += D / (4.f * vh) * (1.f - ddw);
    col = add(col, mul(c.gloss, g));
  }
  return col;
}

__device__ __forceinline__ BSample ct_sample(const CT &c, const Isec &I, float2 prm, uint32_t desired) {
  BSample r{f3(0.f, 0.f, 0.f), 0.f, f3(0.f, 0.f, 1.f), 0u};
  if (!(desired & B_REFLECTIVE)) return r;
  desired &= c.have_layers;
  if (!desired) return r;
  if (I.v.z < 0.f) return r;
  float ddw, inv_ddw, inv_dgw;
  if (desired == (B_DIFFUSE | c.gloss_layer)) {
    ddw = c.diff_weight; inv_ddw = c.inv_diff_weight; inv_dgw = c.inv_gloss_weight;
  } else if (desired == B_DIFFUSE) {
    ddw = 1.f; inv_ddw = 1.f; inv_dgw = 0.f;
  } else {
    ddw = 0.f; inv_ddw = 0.f; inv_dgw = 1.f;
  }
  float u = prm.x, v = prm.y;
  float3 l, h;
  uint32_t fl = B_REFLECTIVE;
  if (u < ddw) {
    if (desired != B_DIFFUSE) u = u * inv_ddw;
    l = z_symm_vec(sqrtf(u), v);
    h = unit(add(I.v, l));
    fl |= B_DIFFUSE;
  } else {
    u = (u - ddw) * inv_dgw;
    float ct = u >= 1.f ? 0.f : 1.f / sqrtf(c.m * c.m * -logf(1.f - u) + 1.f);
    h = z_symm_vec(ct, v);
    if (fminf(dot(I.v, h), 1.f) < 0.f) h = neg(h);
    l = sub(mul(h, dot(I.v, h) * 2.f), I.v);   // v.mirror (h) (geometry/vec.h:154-159)
    fl |= c.gloss_layer;
  }
  if (I.cos_n(l) > 1e-15f && I.cos_geom_n(l) > 1e-15f) {
    float pdf;
    r.val = ct_val(c, I, l, h, desired, ddw, pdf);
    r.pdf = pdf;
    r.dir = l;
    r.flags = fl;
  }
  return r;
}

__device__ __forceinline__ float3 ct_eval(const CT &c, const Isec &I, float3 dir, uint32_t flags, float &pdf) {
  pdf = 0.f;
  float cn = I.cos_n(dir);
  if ((flags & B_REFLECTIVE) && cn > 0.f) {
    flags &= c.have_layers;
    float ddw = (flags == (B_DIFFUSE | c.gloss_layer)) ? c.diff_weight : (flags == B_DIFFUSE) ? 1.f : 0.f;
    float3 h = unit(add(I.v, dir));
    return ct_val(c, I, dir, h, flags, ddw, pdf);
  }
  return f3(0.f, 0.f, 0.f);
}

// Resolve a Glow to its underlying material (material/glow.cc:44-50); null
// if the surface has no BSDF.
__device__ __forceinline__ const DevMaterial *bsdf_material(const DevScene &s, uint32_t mi) {
  const DevMaterial *m = s.mats + mi;
  if (m->type == MAT_GLOW) {
    if (m->underlying < 0) return nullptr;
    m = s.mats + m->underlying;
  }
  return m;
}

// Bsdf::sample for the material M at I.  u01 draws are only needed by none.
__device__ __forceinline__ BSample bsdf_sample(const BsdfCtx &B, const Isec &I, float2 prm, uint32_t flags) {
  const DevMaterial &M = *B.m;
  BSample r{f3(0.f, 0.f, 0.f), 0.f, f3(0.f, 0.f, 1.f), 0u};
  switch (M.type) {
    case MAT_LAMBERT:
      return lambert_sample(I, load3(M.color), prm, flags);
    case MAT_COOK_TORRANCE: {
      CT c = make_ct(I, M, B.medium_ior);
      return ct_sample(c, I, prm, flags);
    }
    case MAT_MIRROR: {
      // MirrorBsdf::sample (material/mirror.cc:51-85)
      if ((flags & (B_SPECULAR | B_REFLECTIVE)) == (B_SPECULAR | B_REFLECTIVE)) {
        float cr = I.cos_n(I.v);
        if (cr != 0.f) {
          float fr = fresnel(M.ior_n / B.medium_ior, M.ior_k / B.medium_ior, cr);
          float3 refl = mul(load3(M.gloss), fr / cr);
          if (csum(refl) > 3e-15f && I.cos_geom_n(I.v) > 0.f) {
            r.val = refl;
            r.pdf = 1.f;
            r.dir = f3(-I.v.x, -I.v.y, I.v.z);
            r.flags = B_SPECULAR | B_REFLECTIVE;
          } else if (M.has_lambert) {
            r = lambert_sample(I, load3(M.color), prm, flags);
            float fr2 = fresnel(M.ior_n / B.medium_ior, M.ior_k / B.medium_ior, I.cos_n(r.dir));
            float3 rr = mul(load3(M.gloss), fr2);
            r.val = mul3(r.val, f3(1.f - rr.x, 1.f - rr.y, 1.f - rr.z));
          }
        }
      }
      return r;
    }
    case MAT_GLASS: {
      // GlassBsdf::sample (material/glass.cc:29-120)
      if (flags & B_SPECULAR) {
        flags &= B_ALL_DIRECTIONS;
        const bool entering = !I.back;
        float old_ior = entering ? B.medium_ior : M.ior_n;
        float new_ior = entering ? M.ior_n : B.enclosing_ior;
        float3 xdir = refraction(neg(I.v), f3(0.f, 0.f, 1.f), old_ior, new_ior);
        float cos_x = -I.cos_n(xdir);
        float cos_r = fabsf(I.cos_n(I.v));
        float xmit = cos_x == 0.f ? 0.f : 1.f - fresnel(old_ior / new_ior, 0.f, cos_x);
        float refl = cos_r == 0.f ? 0.f : fresnel(new_ior / old_ior, 0.f, cos_r);
        if (xmit + refl != 0.f) {
          float xp = flags == B_TRANSMISSIVE ? 1.f : flags == B_REFLECTIVE ? 0.f : xmit / (xmit + refl);
          if (prm.x < xp) {
            if (cos_x != 0.f) xmit /= cos_x;
            r.val = f3(xmit, xmit, xmit);
            r.pdf = xp;
            r.dir = xdir;
            r.flags = B_SPECULAR | B_TRANSMISSIVE;
          } else {
            if (cos_r != 0.f) refl /= cos_r;
            r.val = f3(refl, refl, refl);
            r.pdf = 1.f - xp;
            r.dir = f3(-I.v.x, -I.v.y, I.v.z);
            r.flags = B_SPECULAR | B_REFLECTIVE;
          }
        }
      }
      return r;
    }
  }
  return r;
}

// Bsdf::eval; specular BSDFs (Mirror, Glass) evaluate to zero.
__device__ __forceinline__ float3 bsdf_eval(const BsdfCtx &B, const Isec &I, float3 dir, uint32_t flags,
                                            float &pdf) {
  const DevMaterial &M = *B.m;
  pdf = 0.f;
  if (M.type == MAT_LAMBERT) {
    float cn = I.cos_n(dir);
    if ((flags & (B_DIFFUSE | B_REFLECTIVE)) == (B_DIFFUSE | B_REFLECTIVE) && cn > 0.f) {
      pdf = cn * kInvPi;
      return mul(load3(M.color), kInvPi);
    }
    return f3(0.f, 0.f, 0.f);
  }
  if (M.type == MAT_COOK_TORRANCE) {
    CT c = make_ct(I, M, B.medium_ior);
    return ct_eval(c, I, dir, flags, pdf);
  }
  return f3(0.f, 0.f, 0.f);
}

// ---------------------------------------------------------------------------
// Lights.

struct LSample {
  float3 val;
  float pdf;
  float3 dir;      // normal space
  float dist;      // 0 = "to the horizon"
};

__device__ __forceinline__ bool is_point_light(const DevLight &L) {
  return L.type == LS_POINT || (L.type == LS_FAR && L.a == 1.f);
}

// cone_sample / cone_sample_pdf (geometry/cone-sample.h:28-77).
__device__ __forceinline__ float3 cone_sample(float cos_half, float2 prm) {
  float z = cos_half + prm.y * (1.f - cos_half);
  float r = sqrtf(fabsf(1.f - z * z));
  float phi = prm.x * 2.f * kPi;
  return f3(r * cosf(phi), r * sinf(phi), z);
}
__device__ __forceinline__ float cone_pdf(float cos_half) { return 0.5f * kInvPi / (1.f - cos_half); }

// Tripar::Sampler::sample + AngularSample (surface/tripar.cc:210-240,
// surface/surface-sampler.cc:26-67): a point on the shape and its solid-angle
// pdf seen from VIEW.
__device__ __forceinline__ bool tripar_angular(const DevLight &L, float u, float v, float3 view, float3 &dir,
                                               float &dist, float &pdf) {
  float3 v0 = load3(L.p), e1 = load3(L.p + 3), e2 = load3(L.p + 6);
  float3 nrm = cross(e2, e1);
  float area = length(nrm);
  nrm = mul(nrm, 1.f / area);
  const bool par = L.flags & 1u;
  if (!par && u + v > 1.f) {
    u = 1.f - u;
    v = 1.f - v;
  }
  if (!par) area *= 0.5f;
  float3 pos = add(add(v0, mul(e1, u)), mul(e2, v));
  float apdf = 1.f / area;
  float3 vv = sub(pos, view);
  dist = length(vv);
  pdf = 0.f;
  if (dist > 0.f) {
    float inv = 1.f / dist;
    dir = mul(vv, inv);
    float cadj = -dot(nrm, dir);
    if (cadj > 0.f) pdf = apdf / (cadj * (inv * inv));
  }
  return pdf > 0.f;
}

__device__ __forceinline__ float sphere_solid_angle(float3 lc, float r) {
  float d = length(lc);
  if (d < r) return 4.f * kPi;
  return 2.f * kPi * (1.f - cosf(asinf(r / d)));
}

// EnvmapLight's lat-long image lookup (texture/spheremap.h:146-151,
// texture/matrix-linterp.h:41-80, texture/matrix-tex.tcc:47-63) of a
// direction in the light's frame.
__device__ __forceinline__ float3 env_map(const DevScene &s, float3 dir) {
  float lng = atan2f(-dir.y, dir.x);
  float lat = asinf(fminf(fmaxf(dir.z / sqrtf(dir.x * dir.x + dir.y * dir.y + dir.z * dir.z), -1.f), 1.f));
  float u = fminf(fmaxf(lng * kInvPi * 0.5f + 0.5f, 0.f), 1.f);
  float v = fminf(fmaxf(lat * kInvPi + 0.5f, 0.f), 1.f);
  u = u - floorf(u);
  v = v - floorf(v);
  const uint32_t w = s.env_w, h = s.env_h;
  float x = u * float(w) - 0.5f, y = v * float(h) - 0.5f;
  float xl = floorf(x), yl = floorf(y);
  float xh_fr = x - xl, yh_fr = y - yl, xl_fr = 1.f - xh_fr, yl_fr = 1.f - yh_fr;
  int xi_lo = int(xl), yi_lo = int(yl);
  uint32_t xi_hi = uint32_t(xi_lo + 1), yi_hi = uint32_t(yi_lo + 1);
  if (xi_lo < 0) xi_lo += int(w);
  if (yi_lo < 0) yi_lo += int(h);
  if (xi_hi >= w) xi_hi -= w;
  if (yi_hi >= h) yi_hi -= h;
  uint32_t ylo = h - uint32_t(yi_lo) - 1, yhi = h - yi_hi - 1;
  float4 a = __ldg(s.env_texels + size_t(ylo) * w + uint32_t(xi_lo));
  float4 b = __ldg(s.env_texels + size_t(yhi) * w + uint32_t(xi_lo));
  float4 c = __ldg(s.env_texels + size_t(ylo) * w + xi_hi);
  float4 e = __ldg(s.env_texels + size_t(yhi) * w + xi_hi);
  float wa = xl_fr * yl_fr, wb = xl_fr * yh_fr, wc = xh_fr * yl_fr, we = xh_fr * yh_fr;
  return f3(wa * a.x + wb * b.x + wc * c.x + we * e.x, wa * a.y + wb * b.y + wc * c.y + we * e.y,
            wa * a.z + wb * b.z + wc * c.z + we * e.z);
}

__device__ __forceinline__ float3 env_frame_to(const DevScene &s, float3 d) {
  return f3(d.x * s.env_frame[0] + d.y * s.env_frame[1] + d.z * s.env_frame[2],
            d.x * s.env_frame[3] + d.y * s.env_frame[4] + d.z * s.env_frame[5],
            d.x * s.env_frame[6] + d.y * s.env_frame[7] + d.z * s.env_frame[8]);
}
__device__ __forceinline__ float3 env_frame_from(const DevScene &s, float3 d) {
  return f3(s.env_frame[0] * d.x + s.env_frame[3] * d.y + s.env_frame[6] * d.z,
            s.env_frame[1] * d.x + s.env_frame[4] * d.y + s.env_frame[7] * d.z,
            s.env_frame[2] * d.x + s.env_frame[5] * d.y + s.env_frame[8] * d.z);
}

// lower_bound over a float array (geometry/hist-2d-dist.cc:127-143).
__device__ __forceinline__ uint32_t lower_bound_f(const float *a, uint32_t n, float v) {
  uint32_t lo = 0, len = n;
  while (len > 0) {
    uint32_t half = len >> 1;
    if (__ldg(a + lo + half) < v) {
      lo += half + 1;
      len -= half + 1;
    } else {
      len = half;
    }
  }
  return lo;
}

// Hist2dDist::pdf (geometry/hist-2d-dist.cc:226-280).
__device__ __forceinline__ float hist_pdf(const DevScene &s, uint32_t col, uint32_t row) {
  const float *rc = s.env_row_cdf, *cc = s.env_col_cdf + size_t(row) * s.lmap_w;
  float rp = __ldg(rc + row) - (row ? __ldg(rc + row - 1) : 0.f);
  float cp = __ldg(cc + col) - (col ? __ldg(cc + col - 1) : 0.f);
  return rp * cp * float(s.lmap_w * s.lmap_h);
}

// Hist2dDist::sample (geometry/hist-2d-dist.cc:151-205) -> uv and pdf.
__device__ __forceinline__ bool hist_sample(const DevScene &s, float2 prm, float2 &uv, float &pdf) {
  float u = fminf(prm.x, 1.f), v = fminf(prm.y, 1.f);
  const uint32_t w = s.lmap_w, h = s.lmap_h;
  uint32_t row = lower_bound_f(s.env_row_cdf, h, v);
  if (row == h) return false;
  uint32_t col = lower_bound_f(s.env_col_cdf + size_t(row) * w, w, u);
  if (col >= w) col = w - 1;
  pdf = hist_pdf(s, col, row);
  float cw = 1.f / float(w), rh = 1.f / float(h);
  uv = make_float2(float(col) * cw + fmodf(prm.x, cw), float(row) * rh + fmodf(prm.y, rh));
  return true;
}

// LatLongMapping::map (uv -> direction) (texture/spheremap.h:41-44,
// geometry/spherical-coords.h:193-229).
__device__ __forceinline__ float3 latlong_to_vec(float2 uv) {
  float lng = (uv.x - 0.5f) * kPi * 2.f;
  float lat = (uv.y - 0.5f) * kPi;
  return cos_sph_to_vec(cosf(kPi / 2.f - lat), lng);
}

__device__ __forceinline__ float2 vec_to_latlong(float3 d) {
  float lng = atan2f(-d.y, d.x);
  float lat = asinf(fminf(fmaxf(d.z / sqrtf(d.x * d.x + d.y * d.y + d.z * d.z), -1.f), 1.f));
  return make_float2(fminf(fmaxf(lng * kInvPi * 0.5f + 0.5f, 0.f), 1.f),
                     fminf(fmaxf(lat * kInvPi + 0.5f, 0.f), 1.f));
}

// Light::Sampler::sample (viewpoint form).  EXTRA is the one additional
// uniform the sphere sampler draws (light/sphere-light-sampler.cc:90).
__device__ __forceinline__ LSample light_sample(const DevScene &s, const DevLight &L, const Isec &I,
                                                float2 prm, float extra) {
  LSample r{f3(0.f, 0.f, 0.f), 0.f, f3(0.f, 0.f, 1.f), 0.f};
  switch (L.type) {
    case LS_TRIPAR: {   // SurfaceLightSampler (light/surface-light-sampler.cc:47-70)
      float3 wdir;
      float dist, pdf;
      if (tripar_angular(L, prm.x, prm.y, I.pos, wdir, dist, pdf)) {
        float3 dir = I.nf.to(wdir);
        if (dir.z > 0.f) r = LSample{load3(L.intensity), pdf, dir, dist};
      }
      return r;
    }
    case LS_SPHERE: {   // light/sphere-light-sampler.cc:56-116
      float rad = L.p[3];
      float3 lc = I.nf.to(sub(load3(L.p), I.pos));
      if (lc.z >= -rad) {
        float pdf = 1.f / sphere_solid_angle(lc, rad);
        float rs = rad * sqrtf(prm.x);
        float ang = prm.y * 2.f * kPi;
        float x = rs * cosf(ang), y = rs * sinf(ang);
        float z = sqrtf(fabsf(rad * rad - x * x - y * y)) * sinf(kPi * (extra - 0.5f));
        float3 sv = add(lc, f3(x, y, z));
        if (I.cos_n(sv) > 0.f && I.cos_geom_n(sv) > 0.f) {
          float3 sd = unit(sv);
          float dist;
          if (sphere_hit(f3(0.f, 0.f, 0.f), rad, neg(lc), sd, 0.f, INFINITY, dist))
            r = LSample{load3(L.intensity), pdf, sd, dist};
        }
      }
      return r;
    }
    case LS_POINT: {    // light/point-light.cc:78-107
      float3 lpos = load3(L.p);
      float3 lvec = I.nf.to(sub(lpos, I.pos));
      if (I.cos_n(lvec) > 0.f && I.cos_geom_n(lvec) > 0.f) {
        float dist = length(lvec), inv = 1.f / dist;
        float cos_dir = dot(mul(sub(I.pos, lpos), inv), load3(L.p + 3));
        if (cos_dir >= L.a) {
          float3 it = load3(L.intensity);
          if (cos_dir < L.b) {
            float dd = (cos_dir - L.a) / (L.b - L.a);
            it = mul(it, dd * dd * dd * dd);
          }
          r = LSample{mul(it, inv * inv), 1.f, mul(lvec, inv), dist};
        }
      }
      return r;
    }
    case LS_FAR: {      // light/far-light.cc:96-113
      float3 c = cone_sample(L.a, prm);
      float3 w = f3(L.p[0] * c.x + L.p[3] * c.y + L.p[6] * c.z, L.p[1] * c.x + L.p[4] * c.y + L.p[7] * c.z,
                    L.p[2] * c.x + L.p[5] * c.y + L.p[8] * c.z);
      float3 sd = I.nf.to(w);
      float pdf = L.a == 1.f ? 1.f : cone_pdf(L.a);
      if (I.cos_n(sd) > 0.f && I.cos_geom_n(sd) > 0.f) r = LSample{load3(L.intensity), pdf, sd, 0.f};
      return r;
    }
    case LS_ENV: {      // light/envmap-light.cc:148-180
      float2 uv;
      float pdf;
      if (!hist_sample(s, prm, uv, pdf)) pdf = 0.f, uv = make_float2(0.f, 0.f);
      float3 ldir = latlong_to_vec(uv);
      float3 dir = I.nf.to(env_frame_from(s, ldir));
      if (I.cos_n(dir) < 0.f || I.cos_geom_n(dir) < 0.f) return r;
      pdf *= 0.25f * kInvPi;
      r = LSample{env_map(s, ldir), pdf, dir, 0.f};
      return r;
    }
  }
  return r;
}

// Light::Sampler::eval in normal-space direction DIR.
__device__ __forceinline__ LSample light_eval(const DevScene &s, const DevLight &L, const Isec &I, float3 dir) {
  LSample r{f3(0.f, 0.f, 0.f), 0.f, dir, 0.f};
  switch (L.type) {
    case LS_TRIPAR: {   // surface-light-sampler.cc:112-129, tripar.cc:247-256
      float3 wdir = I.nf.from(dir);
      float t, u, v;
      float3 v0 = load3(L.p), e1 = load3(L.p + 3), e2 = load3(L.p + 6);
      if (tripar_hit(v0, e1, e2, (L.flags & 1u) != 0, I.pos, wdir, 0.f, INFINITY, t, u, v)) {
        float3 sdir;
        float dist, pdf;
        if (tripar_angular(L, u, v, I.pos, sdir, dist, pdf)) r = LSample{load3(L.intensity), pdf, dir, dist};
      }
      return r;
    }
    case LS_SPHERE: {   // sphere-light-sampler.cc:170-194
      float rad = L.p[3];
      float3 lc = I.nf.to(sub(load3(L.p), I.pos));
      if (lc.z >= -rad) {
        float dist;
        if (sphere_hit(f3(0.f, 0.f, 0.f), rad, neg(lc), dir, 0.f, INFINITY, dist))
          r = LSample{load3(L.intensity), 1.f / sphere_solid_angle(lc, rad), dir, dist};
      }
      return r;
    }
    case LS_FAR: {      // far-light.cc:141-156
      if (L.a < 1.f) {
        float3 lz = I.nf.to(load3(L.p + 6));
        if (dot(dir, lz) >= L.a) r = LSample{load3(L.intensity), cone_pdf(L.a), dir, 0.f};
      }
      return r;
    }
    case LS_ENV: {      // envmap-light.cc:237-263
      float3 ldir = env_frame_to(s, I.nf.from(dir));
      float2 mp = vec_to_latlong(ldir);
      uint32_t col = uint32_t(min(max(int(mp.x * float(s.lmap_w)), 0), int(s.lmap_w) - 1));
      uint32_t row = uint32_t(min(max(int(mp.y * float(s.lmap_h)), 0), int(s.lmap_h) - 1));
      r = LSample{env_map(s, ldir), hist_pdf(s, col, row) * 0.25f * kInvPi, dir, 0.f};
      return r;
    }
  }
  return r;   // point lights: a direction never hits them exactly
}

// Scene::background (render/scene.cc:63-73): environment lights seen along
// world direction D (as given, unnormalised).
__device__ __forceinline__ float3 background(const DevScene &s, float3 d) {
  float3 rad = f3(0.f, 0.f, 0.f);
  for (uint32_t i = 0; i < s.n_lights; i++) {
    const DevLight &L = s.lights[i];
    if (L.type == LS_ENV) {
      rad = add(rad, env_map(s, env_frame_to(s, d)));
    } else if (L.type == LS_FAR && L.a < 1.f) {
      if (dot(d, load3(L.p + 6)) > L.a) rad = add(rad, load3(L.intensity));
    }
  }
  return rad;
}

}  // namespace snog

#endif
