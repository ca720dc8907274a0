// Internal device-side definitions shared by the roxy CUDA translation units.
//
// The library is compiled with -fmad=false: every float expression rounds
// like a sequence of IEEE single operations, which is what lets the hit
// distances and barycentrics match the float32 restatement of the
// reference's Moller-Trumbore bit for bit.  Where a fused multiply-add is
// wanted (slab tests on padded boxes, where rounding cannot change a
// result) it is written explicitly with __fmaf_rn.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "../../include/roxy.h"

namespace rx {

__host__ __device__ __forceinline__ float int_bits_as_float(int i) {
  float f;
  memcpy(&f, &i, sizeof(f));
  return f;
}

// ---------------------------------------------------------------- float3 ops
__host__ __device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__host__ __device__ __forceinline__ float3 xyz(float4 a) { return make_float3(a.x, a.y, a.z); }
__host__ __device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
__host__ __device__ __forceinline__ float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__host__ __device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__host__ __device__ __forceinline__ float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
// left-to-right sum of products, as the reference's vector dot
__host__ __device__ __forceinline__ float dot(float3 a, float3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__host__ __device__ __forceinline__ float3 cross(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// v * (1 / |v|), the reference's normalized()
__device__ __forceinline__ float3 normalized(float3 a) {
  float inv = 1.0f / sqrtf(dot(a, a));
  return inv * a;
}
__host__ __device__ __forceinline__ float3 vmin(float3 a, float3 b) { return f3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
__host__ __device__ __forceinline__ float3 vmax(float3 a, float3 b) { return f3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
__host__ __device__ __forceinline__ float maxc(float3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }

// ------------------------------------------------------------------- layout
// BVH node (64 B, four float4): both children's boxes live in the parent, so
// one coalesced 64-byte fetch decides which children to visit.
//   n[0] = (L.min.x, L.max.x, L.min.y, L.max.y)
//   n[1] = (L.min.z, L.max.z, R.min.x, R.max.x)
//   n[2] = (R.min.y, R.max.y, R.min.z, R.max.z)
//   n[3] = (left word, right word, left count, right count) as int bits
// child word >= 0: internal node index; < 0: leaf, first primitive = ~word,
// primitive count in the matching count slot (0 = empty leaf).
struct Node4 {
  float4 a, b, c, d;
};

// Primitives in leaf order, three float4 each (48 B):
//   triangle: a = (v0, kind = 0), b = (v1 - v0, 0), c = (v2 - v0, 0)
//   sphere:   a = (centre, kind = 1), b = (radius, 0, 0, 0), c = 0
//   cube:     a = (centre, kind = 2), b = (half extents, 0), c = 0
enum PrimKind { PRIM_TRI = 0, PRIM_SPHERE = 1, PRIM_CUBE = 2 };

// Shading record per primitive in leaf order (three float4):
//   s0 = (n0, material index bits), s1 = (n1, source id bits), s2 = (n2, 0)
// source id: triangle index in the caller's order, or the object slot for
// spheres.

// Linear primitive slot, scanned before the BVH exactly like the reference's
// _obj_* fields (rendering/taichi/intersect.py:259-287).
struct ObjSlot {
  int type;        // 0 sphere, 1 plane, 2 cube, 4 triangle
  int mat;         // palette index
  float radius, offset;
  float3 center, normal, extra, v0, v1, v2;
};  // 88 B

// Explicit light (emissive sphere or emissive triangle).
struct Light {
  int kind;        // 0 sphere, 1 triangle
  float area;
  float pick_pdf;
  float emission;  // intensity; radiance = albedo * intensity
  float3 p0, p1, p2;
  float3 albedo;
};

// Albedo texture: RGB u8 texels, row-major, at byte `offset` of the scene's
// texel buffer (rendering/taichi/fields.py:82-87 keeps them in a fixed
// 8 x 2048 x 2048 field; here they are packed back to back).
struct TexInfo {
  long long offset;
  int w, h, flip_v, pad;
};

struct DevScene {
  const float4* nodes;     // n_nodes * 4
  int n_nodes;
  const float4* nodes4;    // n_nodes4 * 8: the same tree 4-wide (LBVH builds), or null
  int n_nodes4;
  float3 root_min, root_max;
  const float4* prims;     // n_prims * 3
  const float4* shade;     // n_prims * 3
  int n_prims;
  const float4* mat_a;     // (albedo, type bits)
  const float4* mat_b;     // (roughness, ior, emission, texture)
  int n_mats;
  const ObjSlot* objs;
  int n_objs;
  const Light* lights;
  const float* alias_prob;
  const int* alias_idx;
  int n_lights;
  int exact_slab;          // 1: slab test with the reference's operation order
  const float4* uvs;       // 2 per source triangle: (uv0, uv1), (uv2, has_uv, 0), or null
  const TexInfo* tex;
  const unsigned char* texels;
  int n_tex;
  // light index of each emitter (-1: not a light), for the MIS weight of a
  // BSDF ray that hits a light: by caller triangle, by object slot (BVH
  // spheres), by linear object index; null when the caller gave no sources
  const int* light_of_tri;
  const int* light_of_obj;
  const int* light_of_lin;
};

// _sample_texture (rendering/taichi/trace.py:96-126): repeat wrap, optional
// v flip, bilinear over texels / 255, in the reference's float32 order.
__device__ __forceinline__ float3 tex_sample(const DevScene& S, int ti, float uu, float vv) {
  float3 r = make_float3(1.0f, 1.0f, 1.0f);
  if (ti < 0 || ti >= S.n_tex) return r;
  TexInfo T = S.tex[ti];
  if (T.w > 0 && T.h > 0) {
    float u = uu - floorf(uu), v = vv - floorf(vv);
    if (T.flip_v != 0) v = 1.0f - v;
    float x = u * (float)(T.w - 1), y = v * (float)(T.h - 1);
    int x0 = (int)floorf(x), y0 = (int)floorf(y);
    float tx = x - (float)x0, ty = y - (float)y0;
    // finite uv keep x0, y0 inside the image; the clamp only guards memory
    x0 = min(max(x0, 0), T.w - 1);
    y0 = min(max(y0, 0), T.h - 1);
    int x1 = min(x0 + 1, T.w - 1), y1 = min(y0 + 1, T.h - 1);
    const unsigned char* px = S.texels + T.offset;
    auto texel = [&](int yy, int xx) {
      const unsigned char* q = px + 3 * ((size_t)yy * T.w + xx);
      return make_float3((float)q[0] / 255.0f, (float)q[1] / 255.0f, (float)q[2] / 255.0f);
    };
    float3 c00 = texel(y0, x0), c10 = texel(y0, x1), c01 = texel(y1, x0), c11 = texel(y1, x1);
    float3 c0 = c00 * (1.0f - tx) + c10 * tx;
    float3 c1 = c01 * (1.0f - tx) + c11 * tx;
    r = c0 * (1.0f - ty) + c1 * ty;
  }
  return r;
}

// _bvh_albedo (trace.py:129-136): base albedo times the texture at the
// barycentric uv of source triangle `src`, when it has uvs.
__device__ __forceinline__ float3 textured_albedo(const DevScene& S, int src, int ti, float bu, float bv, float3 base) {
  if (ti < 0 || !S.uvs) return base;
  float4 a = __ldg(S.uvs + 2 * (size_t)src), b = __ldg(S.uvs + 2 * (size_t)src + 1);
  if (__float_as_int(b.z) == 0) return base;
  float w = 1.0f - bu - bv;
  float u = (a.x * w + a.z * bu) + b.x * bv;
  float v = (a.y * w + a.w * bu) + b.y * bv;
  return base * tex_sample(S, ti, u, v);
}

// --------------------------------------------------------------------- RNG
// Philox4x32-10 (Salmon et al., SC'11): counter = (pixel, sample, bounce,
// block), key = (seed, constant).  Identical to the oracle's generator.
__host__ __device__ __forceinline__ void philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                                uint32_t k1, uint32_t out[4]) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
    uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
    uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
__host__ __device__ __forceinline__ float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

constexpr uint32_t kKeyHi = 0x5EEDC0DEu;

enum {
  SLOT_LIGHT_PICK = 0, SLOT_LIGHT_ACCEPT = 1, SLOT_LIGHT_U1 = 2, SLOT_LIGHT_U2 = 3,
  SLOT_BSDF_U1 = 4, SLOT_BSDF_U2 = 5, SLOT_LOBE = 6, SLOT_RR = 7,
  SLOT_FUZZ_U1 = 8, SLOT_FUZZ_U2 = 9,
  SLOT_ALL_LIGHTS = 16
};

// device error bits (set by kernels, read by the host after a launch)
enum {
  ERR_STACK_OVERFLOW = 1,
  ERR_QUEUE_OVERFLOW = 2,
  ERR_SHADOW_OVERFLOW = 4,
  ERR_BAD_NODE = 8
};

constexpr int kStack = 64;

// ------------------------------------------------------------ intersection
// rendering/taichi/intersect.py:17-25
__device__ __forceinline__ float3 make_inv_dir(float3 d) {
  return f3(fabsf(d.x) > 1e-10f ? 1.0f / d.x : 1e30f, fabsf(d.y) > 1e-10f ? 1.0f / d.y : 1e30f,
            fabsf(d.z) > 1e-10f ? 1.0f / d.z : 1e30f);
}

// Moller-Trumbore with the reference's operation order and thresholds
// (rendering/taichi/intersect.py:57-78).  v0 and the two edges are stored
// precomputed; e = v - v0 rounds exactly as the reference computes it.
__device__ __forceinline__ bool tri_hit(float3 o, float3 d, float4 a, float4 b, float4 c, float tmax, float& t,
                                        float& u, float& v) {
  float3 e1 = xyz(b), e2 = xyz(c);
  float3 h = cross(d, e2);
  float det = dot(e1, h);
  if (!(fabsf(det) > 1e-8f)) return false;
  float f = 1.0f / det;
  float3 s = o - xyz(a);
  float uu = f * dot(s, h);
  if (!(uu >= 0.0f && uu <= 1.0f)) return false;
  float3 q = cross(s, e1);
  float vv = f * dot(d, q);
  if (!(vv >= 0.0f && uu + vv <= 1.0f)) return false;
  float tt = f * dot(e2, q);
  if (!(tt > 0.001f && tt < tmax)) return false;
  t = tt;
  u = uu;
  v = vv;
  return true;
}

// scene/primitives.py:90-105 (assumes a unit direction)
__device__ __forceinline__ float sphere_t(float3 o, float3 d, float3 c, float r) {
  float3 oc = o - c;
  float h = dot(d, oc);
  float cc = dot(oc, oc) - r * r;
  float disc = h * h - cc;
  float t = -1.0f;
  if (disc >= 0.0f) {
    float sq = sqrtf(disc);
    t = -h - sq;
    if (t < 0.001f) t = -h + sq;
    if (t < 0.001f) t = -1.0f;
  }
  return t;
}

// scene/primitives.py:145-154
__device__ __forceinline__ float plane_t(float3 o, float3 d, float3 n, float off) {
  float denom = dot(n, d);
  float t = -1.0f;
  if (fabsf(denom) >= 1e-6f) {
    float tc = -(dot(n, o) + off) / denom;
    if (tc >= 0.001f) t = tc;
  }
  return t;
}

// scene/primitives.py:187-201
__device__ __forceinline__ float cube_t(float3 o, float3 d, float3 c, float3 he) {
  float3 bmin = c - he, bmax = c + he;
  float3 t0 = f3((bmin.x - o.x) / d.x, (bmin.y - o.y) / d.y, (bmin.z - o.z) / d.z);
  float3 t1 = f3((bmax.x - o.x) / d.x, (bmax.y - o.y) / d.y, (bmax.z - o.z) / d.z);
  float3 lo = vmin(t0, t1), hi = vmax(t0, t1);
  float te = fmaxf(lo.x, fmaxf(lo.y, lo.z));
  float tx = fminf(hi.x, fminf(hi.y, hi.z));
  float t = -1.0f;
  if (tx >= te && tx >= 0.001f) t = te >= 0.001f ? te : tx;
  return t;
}

// scene/primitives.py:203-215
__device__ __forceinline__ float3 cube_normal(float3 p, float3 c, float3 he) {
  float3 dd = p - c;
  dd = f3(dd.x / he.x, dd.y / he.y, dd.z / he.z);
  float ax = fabsf(dd.x), ay = fabsf(dd.y), az = fabsf(dd.z);
  if (ax >= ay && ax >= az) return f3(dd.x > 0.0f ? 1.0f : -1.0f, 0.0f, 0.0f);
  if (ay >= az) return f3(0.0f, dd.y > 0.0f ? 1.0f : -1.0f, 0.0f);
  return f3(0.0f, 0.0f, dd.z > 0.0f ? 1.0f : -1.0f);
}

// t of a BVH-resident analytic primitive (sphere or cube record a, b): the
// same tests as the object slots, so a sphere or cube moved into the BVH
// returns the same t
__device__ __forceinline__ float analytic_t(float3 o, float3 d, float4 a, float4 b) {
  return __float_as_int(a.w) == PRIM_SPHERE ? sphere_t(o, d, xyz(a), b.x) : cube_t(o, d, xyz(a), xyz(b));
}

// un-flipped normal at point p of a BVH-resident analytic primitive
__device__ __forceinline__ float3 analytic_normal(float3 p, float4 a, float4 b) {
  return __float_as_int(a.w) == PRIM_SPHERE ? normalized(p - xyz(a)) : cube_normal(p, xyz(a), xyz(b));
}

// Linear scan of the object slots (intersect.py:259-287): closest t and slot.
__device__ __forceinline__ float objs_closest(const DevScene& S, float3 o, float3 d, int& slot) {
  float best = 1e9f;
  slot = -1;
  for (int i = 0; i < S.n_objs; ++i) {
    const ObjSlot& ob = S.objs[i];
    float t = -1.0f;
    if (ob.type == 0) t = sphere_t(o, d, ob.center, ob.radius);
    else if (ob.type == 1) t = plane_t(o, d, ob.normal, ob.offset);
    else if (ob.type == 2) t = cube_t(o, d, ob.center, ob.extra);
    else if (ob.type == 4) {
      float uu, vv, tt;
      float4 a = make_float4(ob.v0.x, ob.v0.y, ob.v0.z, 0.0f);
      float4 b = make_float4(ob.v1.x - ob.v0.x, ob.v1.y - ob.v0.y, ob.v1.z - ob.v0.z, 0.0f);
      float4 c = make_float4(ob.v2.x - ob.v0.x, ob.v2.y - ob.v0.y, ob.v2.z - ob.v0.z, 0.0f);
      if (tri_hit(o, d, a, b, c, 3.0e38f, tt, uu, vv)) t = tt;
    }
    if (t > 0.001f && t < best) {
      best = t;
      slot = i;
    }
  }
  return best;
}

__device__ __forceinline__ bool objs_any(const DevScene& S, float3 o, float3 d, float max_t) {
  for (int i = 0; i < S.n_objs; ++i) {
    const ObjSlot& ob = S.objs[i];
    float t = -1.0f;
    if (ob.type == 0) t = sphere_t(o, d, ob.center, ob.radius);
    else if (ob.type == 1) t = plane_t(o, d, ob.normal, ob.offset);
    else if (ob.type == 2) t = cube_t(o, d, ob.center, ob.extra);
    else if (ob.type == 4) {
      float uu, vv, tt;
      float4 a = make_float4(ob.v0.x, ob.v0.y, ob.v0.z, 0.0f);
      float4 b = make_float4(ob.v1.x - ob.v0.x, ob.v1.y - ob.v0.y, ob.v1.z - ob.v0.z, 0.0f);
      float4 c = make_float4(ob.v2.x - ob.v0.x, ob.v2.y - ob.v0.y, ob.v2.z - ob.v0.z, 0.0f);
      if (tri_hit(o, d, a, b, c, 3.0e38f, tt, uu, vv)) t = tt;
    }
    if (0.001f < t && t < max_t) return true;
  }
  return false;
}

// Slab test of both children of a node against [0.001, tmax].
// exact = reference operation order (intersect.py:28-43); otherwise the
// FMA form t = b * inv - o * inv, safe because every box is padded by 1e-4.
template <bool EXACT>
__device__ __forceinline__ void slab2(const float4 n0, const float4 n1, const float4 n2, float3 o, float3 inv,
                                      float3 oinv, float tmax, bool& hl, bool& hr, float& tl, float& tr) {
  float lx0, lx1, ly0, ly1, lz0, lz1, rx0, rx1, ry0, ry1, rz0, rz1;
  if (EXACT) {
    lx0 = (n0.x - o.x) * inv.x; lx1 = (n0.y - o.x) * inv.x;
    ly0 = (n0.z - o.y) * inv.y; ly1 = (n0.w - o.y) * inv.y;
    lz0 = (n1.x - o.z) * inv.z; lz1 = (n1.y - o.z) * inv.z;
    rx0 = (n1.z - o.x) * inv.x; rx1 = (n1.w - o.x) * inv.x;
    ry0 = (n2.x - o.y) * inv.y; ry1 = (n2.y - o.y) * inv.y;
    rz0 = (n2.z - o.z) * inv.z; rz1 = (n2.w - o.z) * inv.z;
  } else {
    lx0 = __fmaf_rn(n0.x, inv.x, -oinv.x); lx1 = __fmaf_rn(n0.y, inv.x, -oinv.x);
    ly0 = __fmaf_rn(n0.z, inv.y, -oinv.y); ly1 = __fmaf_rn(n0.w, inv.y, -oinv.y);
    lz0 = __fmaf_rn(n1.x, inv.z, -oinv.z); lz1 = __fmaf_rn(n1.y, inv.z, -oinv.z);
    rx0 = __fmaf_rn(n1.z, inv.x, -oinv.x); rx1 = __fmaf_rn(n1.w, inv.x, -oinv.x);
    ry0 = __fmaf_rn(n2.x, inv.y, -oinv.y); ry1 = __fmaf_rn(n2.y, inv.y, -oinv.y);
    rz0 = __fmaf_rn(n2.z, inv.z, -oinv.z); rz1 = __fmaf_rn(n2.w, inv.z, -oinv.z);
  }
  float lte = fmaxf(fminf(lx0, lx1), fmaxf(fminf(ly0, ly1), fminf(lz0, lz1)));
  float ltx = fminf(fmaxf(lx0, lx1), fminf(fmaxf(ly0, ly1), fmaxf(lz0, lz1)));
  float rte = fmaxf(fminf(rx0, rx1), fmaxf(fminf(ry0, ry1), fminf(rz0, rz1)));
  float rtx = fminf(fmaxf(rx0, rx1), fminf(fmaxf(ry0, ry1), fmaxf(rz0, rz1)));
  hl = ltx >= lte && ltx >= 0.001f && lte <= tmax;
  hr = rtx >= rte && rtx >= 0.001f && rte <= tmax;
  tl = lte;
  tr = rte;
}

__device__ __forceinline__ bool slab1(float3 bmin, float3 bmax, float3 o, float3 inv, float tmax, float& te) {
  float3 a = (bmin - o) * inv, b = (bmax - o) * inv;
  float3 lo = vmin(a, b), hi = vmax(a, b);
  te = fmaxf(lo.x, fmaxf(lo.y, lo.z));
  float tx = fminf(hi.x, fminf(hi.y, hi.z));
  return tx >= te && tx >= 0.001f && te <= tmax;
}

// x / d rounded to nearest, the same float as the division, given r =
// RN(1 / d): Markstein's correction step (P. Markstein, "Computation of
// elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
// Dev. 34(1), 1990): q = RN(x r), the residual x - q d is exact in one FMA,
// and RN(q + residual * r) is the correctly rounded quotient; a zero
// residual means q * d = x exactly, so q is the quotient (this keeps the
// sign of a zero x).  Requires 2^-30 <= d <= 2^30; with 2^-96 <= |x| <=
// 2^90 every intermediate is then a normal float.  For other nonzero x
// (and non-finite x) it divides.  Used where many quotients share one
// divisor: the running means of a frame (d = frame + 1) and the edge-aware
// filter's range terms (d = 2 sigma^2) and normalisation.
__device__ __forceinline__ float div_by(float x, float d, float r) {
  const float ax = fabsf(x);
  if (!(ax <= 0x1p+90f) || (ax < 0x1p-96f && ax != 0.0f)) return x / d;
  const float q = x * r;
  const float res = __fmaf_rn(-q, d, x);
  return res == 0.0f ? q : __fmaf_rn(res, r, q);
}

// Packed child word: >= 0 internal node index; < 0 leaf with
// ~word = (first primitive << kLeafBits) | primitive count.
constexpr int kLeafBits = 5;
constexpr int kMaxLeafPrims = (1 << kLeafBits) - 1;
constexpr int kMaxPrims = 1 << (31 - kLeafBits);
constexpr int kSentinel = 0x7fffffff;

__host__ __device__ __forceinline__ int pack_leaf(int first, int count) { return ~((first << kLeafBits) | count); }
__device__ __forceinline__ int leaf_first(int w) { return (~w) >> kLeafBits; }
__device__ __forceinline__ int leaf_count(int w) { return (~w) & kMaxLeafPrims; }

// Closest hit over the BVH (intersect.py:81-152 semantics): nearer child
// first, ties to the right child, leaves tested in depth-first order, a hit
// replaces the current one only when strictly closer.  The loop is the
// while-while form with postponed leaves (Aila & Laine, "Understanding the
// efficiency of ray traversal on GPUs", HPG 2009): a lane that reaches a leaf
// parks it and keeps descending until every lane of the warp holds a leaf,
// so leaf tests run together.  Leaves still execute in DFS order, so the
// first hit found among equally distant ones is the reference's.
// tmax in: current best distance (the linear scan's), out: closest hit.
// Returns the leaf-order primitive index or -1.
template <bool EXACT>
__device__ __forceinline__ int bvh_closest_ww(const DevScene& S, float3 o, float3 d, float& tmax, float& hu,
                                              float& hv, int* err) {
  int stack[kStack];
  int sp = 0;
  stack[0] = kSentinel;
  float3 inv = make_inv_dir(d);
  float3 oinv = o * inv;
  int hit = -1;
  float te;
  if (S.n_nodes <= 0 || !slab1(S.root_min, S.root_max, o, inv, tmax, te)) return -1;
  int node = 0, leaf = 0;  // leaf >= 0: no leaf parked
  // each record is visited at most once per ray; the guard turns a
  // malformed tree into an error flag instead of an endless loop
  int guard = 4 * S.n_nodes + 64;
  while (node != kSentinel) {
    while ((unsigned)node < (unsigned)kSentinel) {
      if (--guard < 0 || node >= S.n_nodes) {
        if (err) atomicOr(err, ERR_BAD_NODE);
        return hit;
      }
      const float4* np = S.nodes + 4 * (size_t)node;
      float4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2), n3 = __ldg(np + 3);
      bool hl, hr;
      float tl, tr;
      slab2<EXACT>(n0, n1, n2, o, inv, oinv, tmax, hl, hr, tl, tr);
      int lw = __float_as_int(n3.x), rw = __float_as_int(n3.y);
      if (!hl && !hr) {
        node = stack[sp--];
      } else {
        bool left_first = hl && (!hr || tl < tr);
        node = left_first ? lw : rw;
        if (hl && hr) {
          if (sp + 1 < kStack) {
            stack[++sp] = left_first ? rw : lw;
          } else if (err) {
            atomicOr(err, ERR_STACK_OVERFLOW);
          }
        }
      }
      if (node < 0 && leaf >= 0) {
        leaf = node;
        node = stack[sp--];
      }
      if (!__any_sync(__activemask(), leaf >= 0)) break;
    }
    while (leaf < 0) {
      int first = leaf_first(leaf), cnt = leaf_count(leaf);
      if (first + cnt > S.n_prims) {
        if (err) atomicOr(err, ERR_BAD_NODE);
        return hit;
      }
      for (int k = first; k < first + cnt; ++k) {
        const float4* pp = S.prims + 3 * (size_t)k;
        float4 a = __ldg(pp);
        float t, u, v;
        if (__float_as_int(a.w) == PRIM_TRI) {
          float4 b = __ldg(pp + 1), c = __ldg(pp + 2);
          if (tri_hit(o, d, a, b, c, tmax, t, u, v)) {
            tmax = t; hu = u; hv = v; hit = k;
          }
        } else {
          float4 b = __ldg(pp + 1);
          t = analytic_t(o, d, a, b);
          if (t > 0.001f && t < tmax) {
            tmax = t; hu = 0.0f; hv = 0.0f; hit = k;
          }
        }
      }
      leaf = node;
      if (node < 0) node = stack[sp--];
    }
  }
  return hit;
}

// Leaf test shared by the closest-hit loops.
__device__ __forceinline__ void leaf_closest(const DevScene& S, float3 o, float3 d, int first, int cnt, float& tmax,
                                             float& hu, float& hv, int& hit) {
  for (int k = first; k < first + cnt; ++k) {
    const float4* pp = S.prims + 3 * (size_t)k;
    float4 a = __ldg(pp);
    float t, u, v;
    if (__float_as_int(a.w) == PRIM_TRI) {
      float4 b = __ldg(pp + 1), c = __ldg(pp + 2);
      if (tri_hit(o, d, a, b, c, tmax, t, u, v)) {
        tmax = t; hu = u; hv = v; hit = k;
      }
    } else {
      float4 b = __ldg(pp + 1);
      t = analytic_t(o, d, a, b);
      if (t > 0.001f && t < tmax) {
        tmax = t; hu = 0.0f; hv = 0.0f; hit = k;
      }
    }
  }
}

// Closest hit, depth-first with (child word, entry distance) on the stack:
// a popped entry farther than the current hit is skipped without a fetch.
template <bool EXACT>
__device__ __forceinline__ int bvh_closest_ii(const DevScene& S, float3 o, float3 d, float& tmax, float& hu,
                                              float& hv, int* err) {
  int stk_w[kStack];
  float stk_t[kStack];
  int sp = 0;
  float3 inv = make_inv_dir(d);
  float3 oinv = o * inv;
  int hit = -1;
  float te;
  if (S.n_nodes <= 0 || !slab1(S.root_min, S.root_max, o, inv, tmax, te)) return -1;
  int word = 0;
  float wt = te;
  int guard = 4 * S.n_nodes + 64;
  for (;;) {
    if (wt <= tmax) {
      if (--guard < 0 || word >= S.n_nodes) {
        if (err) atomicOr(err, ERR_BAD_NODE);
        return hit;
      }
      if (word >= 0) {
        const float4* np = S.nodes + 4 * (size_t)word;
        float4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2), n3 = __ldg(np + 3);
        bool hl, hr;
        float tl, tr;
        slab2<EXACT>(n0, n1, n2, o, inv, oinv, tmax, hl, hr, tl, tr);
        int lw = __float_as_int(n3.x), rw = __float_as_int(n3.y);
        if (hl || hr) {
          bool left_first = hl && (!hr || tl < tr);
          if (hl && hr) {
            if (sp < kStack) {
              stk_w[sp] = left_first ? rw : lw;
              stk_t[sp] = left_first ? tr : tl;
              ++sp;
            } else if (err) {
              atomicOr(err, ERR_STACK_OVERFLOW);
            }
          }
          word = left_first ? lw : rw;
          wt = left_first ? tl : tr;
          continue;
        }
      } else {
        int first = leaf_first(word), cnt = leaf_count(word);
        if (first + cnt > S.n_prims) {
          if (err) atomicOr(err, ERR_BAD_NODE);
          return hit;
        }
        leaf_closest(S, o, d, first, cnt, tmax, hu, hv, hit);
      }
    }
    if (sp == 0) break;
    --sp;
    word = stk_w[sp];
    wt = stk_t[sp];
  }
  return hit;
}

// While-while form with postponed leaves and pop culling.
template <bool EXACT>
__device__ __forceinline__ int bvh_closest_wwt(const DevScene& S, float3 o, float3 d, float& tmax, float& hu,
                                               float& hv, int* err) {
  int stk_w[kStack];
  float stk_t[kStack];
  int sp = 0;
  stk_w[0] = kSentinel;
  stk_t[0] = -INFINITY;
  float3 inv = make_inv_dir(d);
  float3 oinv = o * inv;
  int hit = -1;
  float te;
  if (S.n_nodes <= 0 || !slab1(S.root_min, S.root_max, o, inv, tmax, te)) return -1;
  int node = 0, leaf = 0;
  int guard = 4 * S.n_nodes + 64;
  auto pop = [&]() {
    int w;
    float t;
    do {
      w = stk_w[sp];
      t = stk_t[sp];
      --sp;
    } while (t > tmax);
    return w;
  };
  while (node != kSentinel) {
    while ((unsigned)node < (unsigned)kSentinel) {
      if (--guard < 0 || node >= S.n_nodes) {
        if (err) atomicOr(err, ERR_BAD_NODE);
        return hit;
      }
      const float4* np = S.nodes + 4 * (size_t)node;
      float4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2), n3 = __ldg(np + 3);
      bool hl, hr;
      float tl, tr;
      slab2<EXACT>(n0, n1, n2, o, inv, oinv, tmax, hl, hr, tl, tr);
      int lw = __float_as_int(n3.x), rw = __float_as_int(n3.y);
      if (!hl && !hr) {
        node = pop();
      } else {
        bool left_first = hl && (!hr || tl < tr);
        node = left_first ? lw : rw;
        if (hl && hr) {
          if (sp + 1 < kStack) {
            ++sp;
            stk_w[sp] = left_first ? rw : lw;
            stk_t[sp] = left_first ? tr : tl;
          } else if (err) {
            atomicOr(err, ERR_STACK_OVERFLOW);
          }
        }
      }
      if (node < 0 && leaf >= 0) {
        leaf = node;
        node = pop();
      }
      if (!__any_sync(__activemask(), leaf >= 0)) break;
    }
    while (leaf < 0) {
      int first = leaf_first(leaf), cnt = leaf_count(leaf);
      if (first + cnt > S.n_prims) {
        if (err) atomicOr(err, ERR_BAD_NODE);
        return hit;
      }
      leaf_closest(S, o, d, first, cnt, tmax, hu, hv, hit);
      leaf = node;
      if (node < 0) node = pop();
    }
  }
  return hit;
}

// ------------------------------------------------------------ 4-wide BVH
// Node of 8 float4 (128 B, two cache lines): the children's boxes as
// (min x, max x, min y, max y, min z, max z) each over the four children,
// then the child words (>= 0: 4-wide node, < 0: packed leaf) and the
// children's primitive counts.  An empty slot has a box at 1e30 (never
// entered) and count 0.  The 4-wide tree is built from the LBVH: a node
// starts from its binary children and, while it has fewer than four, opens
// the internal child of largest surface area (leaves stay leaves), so
// traversal needs about half the dependent node fetches.

// Three-input min / max (PTX ISA 8.8, sm_100): one instruction each.
__device__ __forceinline__ float max3f(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

// Entry distances of a 4-wide node's children (INFINITY where the ray
// misses a child box before tmax) and their child words.  Each axis's near
// and far planes are chosen once per ray: for a direction component >= 0
// (inv > 0) the children's minima are the near planes, else their maxima;
// `sx`, `sy`, `sz` (1 where inv < 0) select the float4 of each.  For a fixed
// inv the rounded fma(plane, inv, -o*inv) is monotonic in the plane, so the
// near plane's distance equals min(t_min_plane, t_max_plane) exactly and the
// test gives the entry and exit distances of the two-sided slab test bit
// for bit, at 6 FMA and 5 min/max/compare per child instead of 6 FMA and 13
// (on the 1080p benchmark frame `k_extend` 25.3 -> 24.5 ms).
__device__ __forceinline__ void slab4_oct(const float4* np, int sx, int sy, int sz, float3 inv, float3 oinv,
                                          float tmax, float (&t)[4], int (&w)[4]) {
  const float4 nx4 = __ldg(np + sx), fx4 = __ldg(np + (sx ^ 1));
  const float4 ny4 = __ldg(np + 2 + sy), fy4 = __ldg(np + 2 + (sy ^ 1));
  const float4 nz4 = __ldg(np + 4 + sz), fz4 = __ldg(np + 4 + (sz ^ 1));
  const float4 wd4 = __ldg(np + 6);
  const float nx[4] = {nx4.x, nx4.y, nx4.z, nx4.w}, fx[4] = {fx4.x, fx4.y, fx4.z, fx4.w};
  const float ny[4] = {ny4.x, ny4.y, ny4.z, ny4.w}, fy[4] = {fy4.x, fy4.y, fy4.z, fy4.w};
  const float nz[4] = {nz4.x, nz4.y, nz4.z, nz4.w}, fz[4] = {fz4.x, fz4.y, fz4.z, fz4.w};
  const int wd[4] = {__float_as_int(wd4.x), __float_as_int(wd4.y), __float_as_int(wd4.z), __float_as_int(wd4.w)};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float te = max3f(__fmaf_rn(nx[i], inv.x, -oinv.x), __fmaf_rn(ny[i], inv.y, -oinv.y),
                           __fmaf_rn(nz[i], inv.z, -oinv.z));
    const float tx = min3f(__fmaf_rn(fx[i], inv.x, -oinv.x), __fmaf_rn(fy[i], inv.y, -oinv.y),
                           fminf(__fmaf_rn(fz[i], inv.z, -oinv.z), tmax));
    t[i] = fmaxf(te, 0.001f) <= tx ? te : INFINITY;
    w[i] = wd[i];
  }
}

__device__ __forceinline__ void cswap(float (&t)[4], int (&w)[4], int a, int b) {
  if (t[b] < t[a]) {
    float tt = t[a];
    t[a] = t[b];
    t[b] = tt;
    int ww = w[a];
    w[a] = w[b];
    w[b] = ww;
  }
}

// Closest hit on the 4-wide tree: children entered nearest first (sorting
// network on entry distance), farther ones stacked with their distance and
// skipped on pop once the current hit is closer.  Returns the same closest
// primitive as the binary traversal (up to the order among exactly equal
// hit distances).
__device__ __forceinline__ int bvh4_closest(const DevScene& S, float3 o, float3 d, float& tmax, float& hu, float& hv,
                                            int* err) {
  int stk_w[kStack];
  float stk_t[kStack];
  int sp = 0;
  const float3 inv = make_inv_dir(d);
  const float3 oinv = o * inv;
  const int sx = inv.x < 0.0f, sy = inv.y < 0.0f, sz = inv.z < 0.0f;
  int hit = -1;
  float te;
  if (S.n_nodes4 <= 0 || !slab1(S.root_min, S.root_max, o, inv, tmax, te)) return -1;
  int word = 0;
  float wt = te;
  int guard = 4 * S.n_nodes4 + 64;
  for (;;) {
    if (wt <= tmax) {
      if (--guard < 0 || word >= S.n_nodes4) {
        if (err) atomicOr(err, ERR_BAD_NODE);
        return hit;
      }
      if (word >= 0) {
        const float4* np = S.nodes4 + 8 * (size_t)word;
        float t[4];
        int w[4];
        slab4_oct(np, sx, sy, sz, inv, oinv, tmax, t, w);
        cswap(t, w, 0, 1);
        cswap(t, w, 2, 3);
        cswap(t, w, 0, 2);
        cswap(t, w, 1, 3);
        cswap(t, w, 1, 2);
        if (t[0] < INFINITY) {
#pragma unroll
          for (int k = 3; k >= 1; --k)
            if (t[k] < INFINITY) {
              if (sp < kStack) {
                stk_w[sp] = w[k];
                stk_t[sp] = t[k];
                ++sp;
              } else if (err) {
                atomicOr(err, ERR_STACK_OVERFLOW);
              }
            }
          word = w[0];
          wt = t[0];
          continue;
        }
      } else {
        const int first = leaf_first(word), cnt = leaf_count(word);
        if (first + cnt > S.n_prims) {
          if (err) atomicOr(err, ERR_BAD_NODE);
          return hit;
        }
        leaf_closest(S, o, d, first, cnt, tmax, hu, hv, hit);
      }
    }
    if (sp == 0) break;
    --sp;
    word = stk_w[sp];
    wt = stk_t[sp];
  }
  return hit;
}

#ifndef RX_TRAV
#define RX_TRAV 0
#endif

template <bool EXACT>
__device__ __forceinline__ int bvh_closest(const DevScene& S, float3 o, float3 d, float& tmax, float& hu, float& hv,
                                           int* err) {
  if constexpr (!EXACT) {
    if (S.nodes4) return bvh4_closest(S, o, d, tmax, hu, hv, err);
  }
#if RX_TRAV == 1
  return bvh_closest_ww<EXACT>(S, o, d, tmax, hu, hv, err);
#elif RX_TRAV == 2
  return bvh_closest_wwt<EXACT>(S, o, d, tmax, hu, hv, err);
#else
  return bvh_closest_ii<EXACT>(S, o, d, tmax, hu, hv, err);
#endif
}

// Any hit before max_t on the 4-wide tree: every entered child is visited
// (nearest first, the rest stacked) until the first primitive hit.
__device__ __forceinline__ bool bvh4_any(const DevScene& S, float3 o, float3 d, float max_t, int* err) {
  int stack[kStack];
  int sp = 0;
  const float3 inv = make_inv_dir(d);
  const float3 oinv = o * inv;
  const int sx = inv.x < 0.0f, sy = inv.y < 0.0f, sz = inv.z < 0.0f;
  float te;
  if (S.n_nodes4 <= 0 || !slab1(S.root_min, S.root_max, o, inv, max_t, te)) return false;
  int word = 0;
  int guard = 4 * S.n_nodes4 + 64;
  for (;;) {
    if (--guard < 0 || word >= S.n_nodes4) {
      if (err) atomicOr(err, ERR_BAD_NODE);
      return false;
    }
    if (word >= 0) {
      const float4* np = S.nodes4 + 8 * (size_t)word;
      float t[4];
      int w[4];
      slab4_oct(np, sx, sy, sz, inv, oinv, max_t, t, w);
      cswap(t, w, 0, 1);
      cswap(t, w, 2, 3);
      cswap(t, w, 0, 2);
      cswap(t, w, 1, 3);
      cswap(t, w, 1, 2);
      int next = 0;
      bool any = false;
      // nearest next, the others stacked farthest first
#pragma unroll
      for (int k = 3; k >= 0; --k)
        if (t[k] < INFINITY) {
          if (any) {
            if (sp < kStack) stack[sp++] = next;
            else if (err) atomicOr(err, ERR_STACK_OVERFLOW);
          }
          next = w[k];
          any = true;
        }
      if (any) {
        word = next;
        continue;
      }
    } else {
      const int first = leaf_first(word), cnt = leaf_count(word);
      if (first + cnt > S.n_prims) {
        if (err) atomicOr(err, ERR_BAD_NODE);
        return false;
      }
      for (int k = first; k < first + cnt; ++k) {
        const float4* pp = S.prims + 3 * (size_t)k;
        float4 a = __ldg(pp);
        float t, u, v;
        if (__float_as_int(a.w) == PRIM_TRI) {
          float4 b = __ldg(pp + 1), c = __ldg(pp + 2);
          if (tri_hit(o, d, a, b, c, max_t, t, u, v)) return true;
        } else {
          float4 b = __ldg(pp + 1);
          t = analytic_t(o, d, a, b);
          if (0.001f < t && t < max_t) return true;
        }
      }
    }
    if (sp == 0) return false;
    word = stack[--sp];
  }
}

// Any hit before max_t (intersect.py:155-219): stops at the first hit.
template <bool EXACT>
__device__ __forceinline__ bool bvh_any(const DevScene& S, float3 o, float3 d, float max_t, int* err) {
  if constexpr (!EXACT) {
    if (S.nodes4) return bvh4_any(S, o, d, max_t, err);
  }
  int stack[kStack];
  int sp = 0;
  stack[0] = kSentinel;
  float3 inv = make_inv_dir(d);
  float3 oinv = o * inv;
  float te;
  if (S.n_nodes <= 0 || !slab1(S.root_min, S.root_max, o, inv, max_t, te)) return false;
  int node = 0;
  int guard = 4 * S.n_nodes + 64;
  while (node != kSentinel) {
    if (--guard < 0 || node >= S.n_nodes) {
      if (err) atomicOr(err, ERR_BAD_NODE);
      return false;
    }
    if (node >= 0) {
      const float4* np = S.nodes + 4 * (size_t)node;
      float4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2), n3 = __ldg(np + 3);
      bool hl, hr;
      float tl, tr;
      slab2<EXACT>(n0, n1, n2, o, inv, oinv, max_t, hl, hr, tl, tr);
      int lw = __float_as_int(n3.x), rw = __float_as_int(n3.y);
      if (hl || hr) {
        bool left_first = hl && (!hr || tl < tr);
        node = left_first ? lw : rw;
        if (hl && hr) {
          if (sp + 1 < kStack) {
            stack[++sp] = left_first ? rw : lw;
          } else if (err) {
            atomicOr(err, ERR_STACK_OVERFLOW);
          }
        }
        continue;
      }
    } else {
      int first = leaf_first(node), cnt = leaf_count(node);
      if (first + cnt > S.n_prims) {
        if (err) atomicOr(err, ERR_BAD_NODE);
        return false;
      }
      for (int k = first; k < first + cnt; ++k) {
        const float4* pp = S.prims + 3 * (size_t)k;
        float4 a = __ldg(pp);
        float t, u, v;
        if (__float_as_int(a.w) == PRIM_TRI) {
          float4 b = __ldg(pp + 1), c = __ldg(pp + 2);
          if (tri_hit(o, d, a, b, c, max_t, t, u, v)) return true;
        } else {
          float4 b = __ldg(pp + 1);
          t = analytic_t(o, d, a, b);
          if (0.001f < t && t < max_t) return true;
        }
      }
    }
    node = stack[sp--];
  }
  return false;
}


// Hit record from the full scene query (intersect.py:249-309): the linear
// object slots first, then the BVH, which wins only when strictly closer.
struct SceneHit {
  float t;
  int prim;   // leaf-order primitive, or -1
  int slot;   // object slot, or -1
  float u, v;
};

// WIDE: the caller guarantees a 4-wide tree (only that traversal is
// compiled in, which keeps the batch kernels within their registers).
template <bool EXACT, bool WIDE = false>
__device__ __forceinline__ SceneHit scene_closest(const DevScene& S, float3 o, float3 d, int* err) {
  SceneHit h;
  int slot;
  float t = objs_closest(S, o, d, slot);
  h.slot = slot;
  h.prim = -1;
  h.u = 0.0f;
  h.v = 0.0f;
  float u = 0.0f, v = 0.0f;
  int p = WIDE ? bvh4_closest(S, o, d, t, u, v, err) : bvh_closest<EXACT>(S, o, d, t, u, v, err);
  if (p >= 0) {
    h.prim = p;
    h.slot = -1;
    h.u = u;
    h.v = v;
  }
  h.t = t;
  return h;
}

template <bool EXACT, bool WIDE = false>
__device__ __forceinline__ bool scene_any(const DevScene& S, float3 o, float3 d, float max_t, int* err) {
  if (objs_any(S, o, d, max_t)) return true;
  return WIDE ? bvh4_any(S, o, d, max_t, err) : bvh_any<EXACT>(S, o, d, max_t, err);
}

}  // namespace rx
