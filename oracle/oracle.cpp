// ORACLE — test infrastructure only.
//
// A CPU restatement, in plain IEEE float32 (built with -ffp-contract=off, no
// fast-math), of roxy-dcc's Taichi path-tracing hot path.  It is the parity
// checker for the CUDA library and the timed CPU baseline; the product never
// links, imports or calls it.  Each function cites the reference source it
// follows (paths relative to the reference project root).
//
// Parity pins: the BVH build, traversal and trace loop are checked against
// golden vectors produced by running the reference's own Python/Taichi-func
// source (tests/golden/make_golden.py).
//
// Layout conventions follow the reference's global fields
// (rendering/taichi/fields.py:14-88): flat float32 xyz triples, int32 ids.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct V3 { float x, y, z; };

inline V3 mk(float x, float y, float z) { V3 r = {x, y, z}; return r; }
inline V3 ld3(const float* p, long i) { return mk(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
inline V3 operator+(V3 a, V3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator-(V3 a) { return mk(-a.x, -a.y, -a.z); }
inline V3 operator*(V3 a, V3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
inline V3 operator*(V3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
inline V3 operator*(float s, V3 a) { return mk(s * a.x, s * a.y, s * a.z); }
inline V3 operator/(V3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
// Taichi Matrix.sum() reduces left to right: ((x0 + x1) + x2).
inline float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// Taichi normalized(): invlen = 1 / norm; invlen * v.
inline V3 normalized(V3 a) {
  float inv = 1.0f / std::sqrt(dot(a, a));
  return inv * a;
}
inline V3 vmin(V3 a, V3 b) { return mk(std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)); }
inline V3 vmax(V3 a, V3 b) { return mk(std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)); }

const float kPi = 3.14159265358979323846f;
const float kTwoPi = 6.283185307179586f;  // f32(2.0 * math.pi), folded by Taichi

// ----------------------------------------------------------------------------
// Counter-based RNG: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel
// random numbers: as easy as 1, 2, 3", SC'11).  The CUDA library uses the same
// generator with the same counter layout, so for a given (pixel, sample,
// bounce, slot) both sides draw the same number.
// ----------------------------------------------------------------------------
inline void mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  hi = (uint32_t)(p >> 32);
  lo = (uint32_t)p;
}

inline void philox4x32_10(const uint32_t ctr_in[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo(0xD2511F53u, c0, hi0, lo0);
    mulhilo(0xCD9E8D57u, c2, hi1, lo1);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

inline float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

// Random-number slots.  Four slots share one Philox block (slot / 4).
enum {
  SLOT_LIGHT_PICK = 0, SLOT_LIGHT_ACCEPT = 1, SLOT_LIGHT_U1 = 2, SLOT_LIGHT_U2 = 3,
  SLOT_BSDF_U1 = 4, SLOT_BSDF_U2 = 5, SLOT_LOBE = 6, SLOT_RR = 7,
  SLOT_FUZZ_U1 = 8, SLOT_FUZZ_U2 = 9,
  SLOT_ALL_LIGHTS = 16  // "all" mode: light i uses slots 16 + 4 i + {0, 1}
};

struct Rng {
  // counter mode
  uint32_t key0, key1, pixel, sample;
  uint32_t cached_bounce, cached_block;
  uint32_t block[4];
  bool has_block;
  // scripted mode: numbers are consumed in call order (reference ti.random())
  const float* stream;
  int n_stream, pos;
  bool scripted;

  float get(uint32_t bounce, uint32_t slot) {
    if (scripted) {
      float v = pos < n_stream ? stream[pos] : 0.5f;
      ++pos;
      return v;
    }
    uint32_t blk = slot >> 2;
    if (!has_block || blk != cached_block || bounce != cached_bounce) {
      uint32_t ctr[4] = {pixel, sample, bounce, blk};
      philox4x32_10(ctr, key0, key1, block);
      cached_block = blk;
      cached_bounce = bounce;
      has_block = true;
    }
    return u01(block[slot & 3]);
  }
};

}  // namespace

extern "C" {

// Scene in the reference's flat layout (rendering/taichi/fields.py:22-79).
typedef struct {
  // BVH nodes (fields.py:50-56), DFS pre-order as GPUBVHBuilder emits them
  int n_nodes;
  const float* node_min;  // [n_nodes*3]
  const float* node_max;
  const int* node_left;
  const int* node_right;
  const int* node_tri_start;
  const int* node_tri_count;
  // BVH-order triangles (fields.py:59-69)
  int n_tris;
  const float* v0; const float* v1; const float* v2;
  const float* n0; const float* n1; const float* n2;
  const int* tri_mat;
  // material palette (fields.py:73-78)
  int n_mats;
  const int* mat_type; const float* mat_albedo; const float* mat_roughness;
  const float* mat_ior; const float* mat_emission;
  // primitive slots (fields.py:22-40)
  int n_objects;
  const int* obj_type; const float* obj_center; const float* obj_radius;
  const float* obj_normal; const float* obj_offset; const float* obj_extra;
  const float* obj_v0; const float* obj_v1; const float* obj_v2;
  const int* obj_mat_type; const float* obj_albedo; const float* obj_roughness;
  const float* obj_ior; const float* obj_emission;
  // explicit lights.  Reference-compatible mode uses only the sphere lights
  // (fields.py:43-47 / extractor.py:36-50).  The default mode samples the
  // combined list below (emissive spheres + emissive triangles) by its alias
  // table.
  int n_lights;
  const int* light_kind;        // 0 sphere, 1 triangle
  const float* light_p0;        // sphere centre | triangle v0
  const float* light_p1;        // triangle v1 | (radius, 0, 0)
  const float* light_p2;        // triangle v2
  const float* light_albedo;    // emitter albedo rgb
  const float* light_emission;  // emitter intensity (radiance = albedo * intensity)
  const float* light_area;      // triangle area | 0
  const float* light_pick_pdf;  // selection probability
  const float* alias_prob;      // alias table
  const int* alias_idx;
  const int* light_obj;         // sphere light: object slot | triangle light: -1
  // albedo textures (fields.py:64-66,80-87): BVH-order uvs, texture index per
  // material, RGB u8 images packed back to back
  const float* uv0; const float* uv1; const float* uv2;  // [n_tris*2] or null
  const int* has_uv;                                      // [n_tris] or null
  const int* mat_texture;                                 // [n_mats] or null
  int n_tex;
  const int* tex_w; const int* tex_h; const int* tex_flip;
  const long long* tex_off;
  const unsigned char* texels;
} orc_scene;

typedef struct {
  int width, height;
  float fov_tan, aspect;
  float cam_pos[3], cam_fwd[3], cam_right[3], cam_up[3];
  int max_depth;
  int use_sky;
  float bg[3];
  int direct_light_mode;       // 0 one, 1 all
  int direct_light_max_depth;
  float sample_clamp;
  int reference_compat;        // 1: sphere-light NEE only, emission double-count
  uint32_t seed;
} orc_params;

}  // extern "C"

namespace {

// intersect.py:17-25
inline V3 make_inv_dir(V3 rd) {
  V3 r;
  r.x = std::fabs(rd.x) > 1e-10f ? 1.0f / rd.x : 1e30f;
  r.y = std::fabs(rd.y) > 1e-10f ? 1.0f / rd.y : 1e30f;
  r.z = std::fabs(rd.z) > 1e-10f ? 1.0f / rd.z : 1e30f;
  return r;
}

// intersect.py:28-43
inline bool aabb_hit_tmax_inv(V3 ro, V3 inv_d, V3 bmin, V3 bmax, float limit, float& t_enter) {
  V3 t_min = (bmin - ro) * inv_d;
  V3 t_max = (bmax - ro) * inv_d;
  V3 t1 = vmin(t_min, t_max);
  V3 t2 = vmax(t_min, t_max);
  t_enter = std::max(t1.x, std::max(t1.y, t1.z));
  float t_exit = std::min(t2.x, std::min(t2.y, t2.z));
  return t_exit >= t_enter && t_exit >= 0.001f && t_enter <= limit;
}

// intersect.py:57-78 (Moller-Trumbore).  Returns t = -1 on miss.
inline float tri_intersect(V3 ro, V3 rd, V3 v0, V3 v1, V3 v2, float& u, float& v) {
  V3 e1 = v1 - v0;
  V3 e2 = v2 - v0;
  V3 h = cross(rd, e2);
  float a = dot(e1, h);
  float t = -1.0f;
  u = 0.0f;
  v = 0.0f;
  if (std::fabs(a) > 1e-8f) {
    float f = 1.0f / a;
    V3 s = ro - v0;
    u = f * dot(s, h);
    if (0.0f <= u && u <= 1.0f) {
      V3 q = cross(s, e1);
      v = f * dot(rd, q);
      if (v >= 0.0f && u + v <= 1.0f) {
        float tc = f * dot(e2, q);
        if (tc > 0.001f) t = tc;
      }
    }
  }
  return t;
}

// scene/primitives.py:90-105
inline float sphere_intersect(V3 ro, V3 rd, V3 c, float r) {
  V3 oc = ro - c;
  float h = dot(rd, oc);
  float cc = dot(oc, oc) - r * r;
  float disc = h * h - cc;
  float t = -1.0f;
  if (disc >= 0.0f) {
    float sq = std::sqrt(disc);
    t = -h - sq;
    if (t < 0.001f) t = -h + sq;
    if (t < 0.001f) t = -1.0f;
  }
  return t;
}

// scene/primitives.py:145-154
inline float plane_intersect(V3 ro, V3 rd, V3 n, float offset) {
  float denom = dot(n, rd);
  float t = -1.0f;
  if (std::fabs(denom) >= 1e-6f) {
    float tc = -(dot(n, ro) + offset) / denom;
    if (tc >= 0.001f) t = tc;
  }
  return t;
}

// scene/primitives.py:187-201
inline float cube_intersect(V3 ro, V3 rd, V3 c, V3 he) {
  V3 bmin = c - he, bmax = c + he;
  V3 t_min = mk((bmin.x - ro.x) / rd.x, (bmin.y - ro.y) / rd.y, (bmin.z - ro.z) / rd.z);
  V3 t_max = mk((bmax.x - ro.x) / rd.x, (bmax.y - ro.y) / rd.y, (bmax.z - ro.z) / rd.z);
  V3 t1 = vmin(t_min, t_max), t2 = vmax(t_min, t_max);
  float te = std::max(t1.x, std::max(t1.y, t1.z));
  float tx = std::min(t2.x, std::min(t2.y, t2.z));
  float t = -1.0f;
  if (tx >= te && tx >= 0.001f) t = te >= 0.001f ? te : tx;
  return t;
}

// scene/primitives.py:203-215
inline V3 cube_normal(V3 p, V3 c, V3 he) {
  V3 d = (p - c);
  d = mk(d.x / he.x, d.y / he.y, d.z / he.z);
  V3 a = mk(std::fabs(d.x), std::fabs(d.y), std::fabs(d.z));
  if (a.x >= a.y && a.x >= a.z) return mk(d.x > 0.0f ? 1.0f : -1.0f, 0.0f, 0.0f);
  if (a.y >= a.z) return mk(0.0f, d.y > 0.0f ? 1.0f : -1.0f, 0.0f);
  return mk(0.0f, 0.0f, d.z > 0.0f ? 1.0f : -1.0f);
}

// intersect.py:81-152 — closest hit, 64-entry stack, ordered child push.
inline float bvh_intersect(const orc_scene& s, V3 ro, V3 rd, int& idx, float& cu, float& cv) {
  int stack[64];
  float stack_t[64];
  int sp = -1;
  V3 inv_d = make_inv_dir(rd);
  float closest_t = 1e9f;
  idx = -1;
  cu = 0.0f;
  cv = 0.0f;
  float rt;
  if (aabb_hit_tmax_inv(ro, inv_d, ld3(s.node_min, 0), ld3(s.node_max, 0), closest_t, rt)) {
    stack[++sp] = 0;
    stack_t[sp] = rt;
  }
  while (sp >= 0) {
    int node = stack[sp];
    float node_t = stack_t[sp];
    --sp;
    if (node_t > closest_t) continue;
    int cnt = s.node_tri_count[node];
    if (cnt > 0) {
      int st = s.node_tri_start[node];
      for (int i = st; i < st + cnt; ++i) {
        float u, v;
        float t = tri_intersect(ro, rd, ld3(s.v0, i), ld3(s.v1, i), ld3(s.v2, i), u, v);
        if (0.001f < t && t < closest_t) {
          closest_t = t;
          idx = i;
          cu = u;
          cv = v;
        }
      }
    } else {
      int l = s.node_left[node], r = s.node_right[node];
      float lt, rtt;
      bool lh = aabb_hit_tmax_inv(ro, inv_d, ld3(s.node_min, l), ld3(s.node_max, l), closest_t, lt);
      bool rh = aabb_hit_tmax_inv(ro, inv_d, ld3(s.node_min, r), ld3(s.node_max, r), closest_t, rtt);
      if (lh && rh) {
        if (lt < rtt) {
          stack[++sp] = r; stack_t[sp] = rtt;
          stack[++sp] = l; stack_t[sp] = lt;
        } else {
          stack[++sp] = l; stack_t[sp] = lt;
          stack[++sp] = r; stack_t[sp] = rtt;
        }
      } else if (lh) {
        stack[++sp] = l; stack_t[sp] = lt;
      } else if (rh) {
        stack[++sp] = r; stack_t[sp] = rtt;
      }
    }
  }
  return closest_t;
}

// intersect.py:155-219 — any hit before max_t.
inline bool bvh_occluded(const orc_scene& s, V3 ro, V3 rd, float max_t) {
  int stack[64];
  float stack_t[64];
  int sp = -1;
  V3 inv_d = make_inv_dir(rd);
  float rt;
  if (aabb_hit_tmax_inv(ro, inv_d, ld3(s.node_min, 0), ld3(s.node_max, 0), max_t, rt)) {
    stack[++sp] = 0;
    stack_t[sp] = rt;
  }
  bool occluded = false;
  while (sp >= 0 && !occluded) {
    int node = stack[sp];
    float node_t = stack_t[sp];
    --sp;
    if (node_t > max_t) continue;
    int cnt = s.node_tri_count[node];
    if (cnt > 0) {
      int st = s.node_tri_start[node];
      for (int i = st; i < st + cnt; ++i) {
        float u, v;
        float t = tri_intersect(ro, rd, ld3(s.v0, i), ld3(s.v1, i), ld3(s.v2, i), u, v);
        if (0.001f < t && t < max_t) occluded = true;
      }
    } else {
      int l = s.node_left[node], r = s.node_right[node];
      float lt, rtt;
      bool lh = aabb_hit_tmax_inv(ro, inv_d, ld3(s.node_min, l), ld3(s.node_max, l), max_t, lt);
      bool rh = aabb_hit_tmax_inv(ro, inv_d, ld3(s.node_min, r), ld3(s.node_max, r), max_t, rtt);
      if (lh && rh) {
        if (lt < rtt) {
          stack[++sp] = r; stack_t[sp] = rtt;
          stack[++sp] = l; stack_t[sp] = lt;
        } else {
          stack[++sp] = l; stack_t[sp] = lt;
          stack[++sp] = r; stack_t[sp] = rtt;
        }
      } else if (lh) {
        stack[++sp] = l; stack_t[sp] = lt;
      } else if (rh) {
        stack[++sp] = r; stack_t[sp] = rtt;
      }
    }
  }
  return occluded;
}

struct Hit {
  float t;
  V3 normal;
  int idx;
  int is_bvh;
  int bvh_mat;
  float u, v;
};

// intersect.py:249-309 — linear primitive scan, then the BVH.
inline Hit scene_intersect(const orc_scene& s, V3 ro, V3 rd) {
  Hit h;
  h.t = 1e9f;
  h.normal = mk(0.0f, 1.0f, 0.0f);
  h.idx = -1;
  h.is_bvh = 0;
  h.bvh_mat = 0;
  h.u = 0.0f;
  h.v = 0.0f;
  for (int i = 0; i < s.n_objects; ++i) {
    float t = -1.0f;
    V3 nrm = mk(0.0f, 0.0f, 0.0f);
    int ty = s.obj_type[i];
    if (ty == 0) {
      V3 c = ld3(s.obj_center, i);
      t = sphere_intersect(ro, rd, c, s.obj_radius[i]);
      if (t > 0.001f) nrm = normalized((ro + rd * t) - c);
    } else if (ty == 1) {
      t = plane_intersect(ro, rd, ld3(s.obj_normal, i), s.obj_offset[i]);
      if (t > 0.001f) nrm = ld3(s.obj_normal, i);
    } else if (ty == 2) {
      V3 c = ld3(s.obj_center, i), he = ld3(s.obj_extra, i);
      t = cube_intersect(ro, rd, c, he);
      if (t > 0.001f) nrm = cube_normal(ro + rd * t, c, he);
    } else if (ty == 4) {
      V3 a = ld3(s.obj_v0, i), b = ld3(s.obj_v1, i), c = ld3(s.obj_v2, i);
      float uu, vv;
      t = tri_intersect(ro, rd, a, b, c, uu, vv);
      if (t > 0.001f) nrm = normalized(cross(b - a, c - a));
    }
    if (t > 0.001f && t < h.t) {
      h.t = t;
      h.normal = nrm;
      h.idx = i;
    }
  }
  if (s.n_tris > 0) {
    int ti;
    float u, v;
    float t = bvh_intersect(s, ro, rd, ti, u, v);
    if (0.001f < t && t < h.t) {
      h.t = t;
      h.idx = ti;
      h.is_bvh = 1;
      h.bvh_mat = s.tri_mat[ti];
      h.u = u;
      h.v = v;
      float w = 1.0f - u - v;
      h.normal = normalized((ld3(s.n0, ti) * w + ld3(s.n1, ti) * u) + ld3(s.n2, ti) * v);
    }
  }
  return h;
}

// intersect.py:222-246
inline bool scene_occluded(const orc_scene& s, V3 ro, V3 rd, float max_t) {
  bool occ = false;
  for (int i = 0; i < s.n_objects; ++i) {
    float t = -1.0f;
    int ty = s.obj_type[i];
    if (ty == 0) t = sphere_intersect(ro, rd, ld3(s.obj_center, i), s.obj_radius[i]);
    else if (ty == 1) t = plane_intersect(ro, rd, ld3(s.obj_normal, i), s.obj_offset[i]);
    else if (ty == 2) t = cube_intersect(ro, rd, ld3(s.obj_center, i), ld3(s.obj_extra, i));
    else if (ty == 4) {
      float uu, vv;
      t = tri_intersect(ro, rd, ld3(s.obj_v0, i), ld3(s.obj_v1, i), ld3(s.obj_v2, i), uu, vv);
    }
    if (0.001f < t && t < max_t) occ = true;
  }
  if (!occ && s.n_tris > 0) occ = bvh_occluded(s, ro, rd, max_t);
  return occ;
}

// scatter.py:14-30 — cosine hemisphere with the reference's helper basis.
inline V3 cosine_hemisphere(V3 n, float r1, float r2) {
  float phi = kTwoPi * r1;
  float r = std::sqrt(r2);
  float lx = std::cos(phi) * r;
  float ly = std::sin(phi) * r;
  float lz = std::sqrt(std::max(0.0f, 1.0f - r2));
  V3 helper = std::fabs(n.x) > 0.9f ? mk(0.0f, 1.0f, 0.0f) : mk(1.0f, 0.0f, 0.0f);
  V3 b = normalized(cross(n, helper));
  V3 t = cross(b, n);
  return normalized((t * lx + b * ly) + n * lz);
}

// scatter.py:33-38
inline V3 diffuse_scatter(V3 n, float r1, float r2) {
  V3 s = cosine_hemisphere(n, r1, r2);
  if (dot(s, s) < 1e-8f) s = n;
  return normalized(s);
}

// scatter.py:6-11 — theta = acos(1 - 2u), phi = 2 pi u'.
inline V3 random_unit_vector(float r1, float r2) {
  float theta = std::acos(1.0f - 2.0f * r1);
  float phi = kTwoPi * r2;
  float st = std::sin(theta);
  return mk(st * std::cos(phi), st * std::sin(phi), std::cos(theta));
}

// scatter.py:40-49
inline V3 reflect(V3 rd, V3 n) { return rd - (2.0f * dot(rd, n)) * n; }
inline V3 refract(V3 rd, V3 n, float eta) {
  float cos_t = std::min(-dot(rd, n), 1.0f);
  V3 perp = eta * (rd + cos_t * n);
  V3 par = -std::sqrt(std::fabs(1.0f - dot(perp, perp))) * n;
  return perp + par;
}

// scatter.py:57-60
inline float schlick(float c, float eta) {
  float r0 = std::pow((1.0f - eta) / (1.0f + eta), 2.0f);
  return r0 + (1.0f - r0) * std::pow(1.0f - c, 5.0f);
}

// trace.py:23-57 — uniform cone sampling of a sphere light.
inline void sphere_light_sample(V3 hit_p, V3 center, float radius, float ru1, float ru2,
                                V3& light_dir, float& t_light, float& solid_over_pi) {
  V3 to_c = center - hit_p;
  float dist2 = std::max(dot(to_c, to_c), 1e-6f);
  float dist = std::sqrt(dist2);
  V3 axis = to_c / dist;
  float sin2 = std::min(radius * radius / dist2, 1.0f);
  float cos_max = std::sqrt(std::max(0.0f, 1.0f - sin2));
  float cos_t = 1.0f - ru1 * (1.0f - cos_max);
  float sin_t = std::sqrt(std::max(0.0f, 1.0f - cos_t * cos_t));
  float phi = kTwoPi * ru2;
  V3 helper = std::fabs(axis.x) > 0.9f ? mk(0.0f, 1.0f, 0.0f) : mk(1.0f, 0.0f, 0.0f);
  V3 bt = normalized(cross(axis, helper));
  V3 tg = cross(bt, axis);
  light_dir = normalized((tg * (std::cos(phi) * sin_t) + bt * (std::sin(phi) * sin_t)) + axis * cos_t);
  V3 oc = hit_p - center;
  float half_b = dot(oc, light_dir);
  float c = dot(oc, oc) - radius * radius;
  float disc = std::max(half_b * half_b - c, 0.0f);
  t_light = -half_b - std::sqrt(disc);
  solid_over_pi = 2.0f * (1.0f - cos_max);
}

struct Counters {
  long rays;
};

// Reference-compatible direct lighting: trace.py:60-93 (sphere lights only,
// uniform pick weighted by the light count in "one" mode).
inline V3 direct_light_compat(const orc_scene& s, const orc_params& p, Rng& rng, uint32_t bounce,
                              V3 hit_p, V3 n, V3 albedo, Counters& cnt) {
  V3 direct = mk(0.0f, 0.0f, 0.0f);
  // sphere lights = entries of kind 0 in the light list, in slot order
  int count = 0;
  for (int i = 0; i < s.n_lights; ++i) count += s.light_kind[i] == 0;
  if (count > 0) {
    int sel = (int)(rng.get(bounce, SLOT_LIGHT_PICK) * (float)count);
    sel = std::min(sel, count - 1);
    int k = -1;
    for (int i = 0; i < s.n_lights; ++i) {
      if (s.light_kind[i] != 0) continue;
      ++k;
      if (!(p.direct_light_mode == 1 || k == sel)) continue;
      uint32_t su1 = p.direct_light_mode == 1 ? SLOT_ALL_LIGHTS + 4 * k : SLOT_LIGHT_U1;
      float ru1 = rng.get(bounce, su1);
      float ru2 = rng.get(bounce, su1 + 1);
      V3 ldir;
      float tl, sop;
      float radius = s.light_p1[3 * i];
      sphere_light_sample(hit_p, ld3(s.light_p0, i), radius, ru1, ru2, ldir, tl, sop);
      float ndotl = dot(n, ldir);
      if (ndotl > 0.0f) {
        float max_t = tl * 0.999f;
        if (max_t > 0.001f) {
          V3 so = hit_p + n * 1e-4f;
          cnt.rays++;
          if (!scene_occluded(s, so, ldir, max_t)) {
            float w = 1.0f;
            if (p.direct_light_mode == 0) w = (float)count;
            V3 base = (albedo * ld3(s.light_albedo, i)) * s.light_emission[i];
            direct = direct + ((base * ndotl) * sop) * w;
          }
        }
      }
    }
  }
  return direct;
}

// Next-event estimation over the combined light list (emissive spheres and
// emissive triangles).  "one" mode picks a light with the alias table and
// weights by 1/pdf; "all" mode samples every light once.
inline V3 direct_light_full(const orc_scene& s, const orc_params& p, Rng& rng, uint32_t bounce,
                            V3 hit_p, V3 n, V3 albedo, Counters& cnt) {
  V3 direct = mk(0.0f, 0.0f, 0.0f);
  int nl = s.n_lights;
  if (nl <= 0) return direct;
  // light samples are taken from the normal-offset point the shadow ray and
  // the continuation ray start from, so a grazing shadow ray cannot clip the
  // sampled emitter's own plane before max_t
  const V3 sp = hit_p + n * 1e-4f;
  int first = 0, last = nl;
  if (p.direct_light_mode == 0) {
    float r0 = rng.get(bounce, SLOT_LIGHT_PICK);
    int col = std::min((int)(r0 * (float)nl), nl - 1);
    float r1 = rng.get(bounce, SLOT_LIGHT_ACCEPT);
    int li = r1 < s.alias_prob[col] ? col : s.alias_idx[col];
    first = li;
    last = li + 1;
  }
  for (int i = first; i < last; ++i) {
    uint32_t su1 = p.direct_light_mode == 1 ? SLOT_ALL_LIGHTS + 4 * i : SLOT_LIGHT_U1;
    float ru1 = rng.get(bounce, su1);
    float ru2 = rng.get(bounce, su1 + 1);
    float inv_pick = p.direct_light_mode == 1 ? 1.0f : 1.0f / s.light_pick_pdf[i];
    V3 base = (albedo * ld3(s.light_albedo, i)) * s.light_emission[i];
    if (s.light_kind[i] == 0) {
      V3 ldir;
      float tl, sop;
      sphere_light_sample(sp, ld3(s.light_p0, i), s.light_p1[3 * i], ru1, ru2, ldir, tl, sop);
      float ndotl = dot(n, ldir);
      if (ndotl > 0.0f) {
        float max_t = tl * 0.999f;
        if (max_t > 0.001f) {
          V3 so = sp;
          cnt.rays++;
          if (!scene_occluded(s, so, ldir, max_t))
            direct = direct + ((base * ndotl) * sop) * inv_pick;
        }
      }
    } else {
      V3 a = ld3(s.light_p0, i), b = ld3(s.light_p1, i), c = ld3(s.light_p2, i);
      float su = std::sqrt(ru1);
      float b1 = su * (1.0f - ru2);
      float b2 = su * ru2;
      V3 e1 = b - a, e2 = c - a;
      V3 y = (a + e1 * b1) + e2 * b2;
      V3 to = y - sp;
      float d2 = dot(to, to);
      float d = std::sqrt(d2);
      V3 wi = to * (1.0f / d);
      float ndotl = dot(n, wi);
      if (ndotl > 0.0f) {
        V3 ln = normalized(cross(e1, e2));
        float cos_l = std::fabs(dot(ln, wi));
        float max_t = d * 0.999f;
        if (max_t > 0.001f) {
          V3 so = sp;
          cnt.rays++;
          if (!scene_occluded(s, so, wi, max_t)) {
            float g = (((ndotl * cos_l) * s.light_area[i]) / (kPi * d2)) * inv_pick;
            direct = direct + base * g;
          }
        }
      }
    }
  }
  return direct;
}

struct PathOut {
  V3 color, normal, albedo;
  float depth;
};

// trace.py:96-126 _sample_texture.
inline V3 sample_texture(const orc_scene& s, int ti, float uu, float vv) {
  V3 r = mk(1.0f, 1.0f, 1.0f);
  if (ti < 0 || ti >= s.n_tex) return r;
  int w = s.tex_w[ti], h = s.tex_h[ti];
  if (w > 0 && h > 0) {
    float u = uu - std::floor(uu);
    float v = vv - std::floor(vv);
    if (s.tex_flip[ti] != 0) v = 1.0f - v;
    float x = u * (float)(w - 1);
    float y = v * (float)(h - 1);
    int x0 = (int)std::floor(x), y0 = (int)std::floor(y);
    int x1 = std::min(x0 + 1, w - 1), y1 = std::min(y0 + 1, h - 1);
    float tx = x - (float)x0, ty = y - (float)y0;
    const unsigned char* px = s.texels + s.tex_off[ti];
    auto texel = [&](int yy, int xx) {
      const unsigned char* q = px + 3 * ((size_t)yy * w + xx);
      return mk((float)q[0] / 255.0f, (float)q[1] / 255.0f, (float)q[2] / 255.0f);
    };
    V3 c0 = texel(y0, x0) * (1.0f - tx) + texel(y0, x1) * tx;
    V3 c1 = texel(y1, x0) * (1.0f - tx) + texel(y1, x1) * tx;
    r = c0 * (1.0f - ty) + c1 * ty;
  }
  return r;
}

// trace.py:129-136 _bvh_albedo (tri = BVH-order triangle).
inline V3 bvh_albedo(const orc_scene& s, int tri, int mat, float bu, float bv, V3 base) {
  int ti = s.mat_texture ? s.mat_texture[mat] : -1;
  if (ti >= 0 && s.has_uv && s.has_uv[tri] != 0) {
    float w = 1.0f - bu - bv;
    float u = (s.uv0[2 * tri] * w + s.uv1[2 * tri] * bu) + s.uv2[2 * tri] * bv;
    float v = (s.uv0[2 * tri + 1] * w + s.uv1[2 * tri + 1] * bu) + s.uv2[2 * tri + 1] * bv;
    return base * sample_texture(s, ti, u, v);
  }
  return base;
}

// trace.py:139-236 — the per-path bounce loop.
inline PathOut trace(const orc_scene& s, const orc_params& p, Rng& rng, V3 ro, V3 rd, Counters& cnt) {
  V3 color = mk(0.0f, 0.0f, 0.0f);
  V3 thr = mk(1.0f, 1.0f, 1.0f);
  float cur_ior = 1.0f;
  PathOut o;
  o.normal = mk(0.0f, 0.0f, 0.0f);
  o.albedo = mk(0.0f, 0.0f, 0.0f);
  o.depth = 0.0f;
  bool prev_nee = false;
  for (int depth = 0; depth < p.max_depth; ++depth) {
    uint32_t b = (uint32_t)depth;
    cnt.rays++;
    Hit h = scene_intersect(s, ro, rd);
    if (h.t < 0.0f || h.t >= 1e9f) {
      if (p.use_sky) {
        float t = 0.5f * (rd.y + 1.0f);
        color = color + thr * (mk(1.0f, 1.0f, 1.0f) * (1.0f - t) + mk(0.5f, 0.7f, 1.0f) * t);
      } else {
        color = color + thr * mk(p.bg[0], p.bg[1], p.bg[2]);
      }
      break;
    }
    V3 n = h.normal;
    bool front = dot(n, rd) < 0.0f;
    if (!front) n = -n;
    V3 hit_p = ro + rd * h.t;
    int mt;
    V3 alb;
    float rough, ior, em;
    bool listed_light;
    if (h.is_bvh) {
      mt = s.mat_type[h.bvh_mat];
      alb = bvh_albedo(s, h.idx, h.bvh_mat, h.u, h.v, ld3(s.mat_albedo, h.bvh_mat));
      rough = s.mat_roughness[h.bvh_mat];
      ior = s.mat_ior[h.bvh_mat];
      em = s.mat_emission[h.bvh_mat];
      // every emissive BVH triangle is in the light list except textured ones
      listed_light = !(s.mat_texture && s.mat_texture[h.bvh_mat] >= 0);
    } else {
      mt = s.obj_mat_type[h.idx];
      alb = ld3(s.obj_albedo, h.idx);
      rough = s.obj_roughness[h.idx];
      ior = s.obj_ior[h.idx];
      em = s.obj_emission[h.idx];
      listed_light = s.obj_type[h.idx] == 0 && em > 0.0f;
    }
    if (depth == 0) {
      o.normal = n;
      o.albedo = alb;
      o.depth = h.t;
    }
    bool nee_here = false;
    if (mt == 3) {
      bool skip = !p.reference_compat && prev_nee && listed_light && em > 0.0f;
      if (!skip) color = color + (thr * alb) * em;
      break;
    } else if (mt == 0) {
      if (depth < p.direct_light_max_depth) {
        V3 d = p.reference_compat ? direct_light_compat(s, p, rng, b, hit_p, n, alb, cnt)
                                  : direct_light_full(s, p, rng, b, hit_p, n, alb, cnt);
        color = color + thr * d;
        nee_here = s.n_lights > 0;
      }
      float r1 = rng.get(b, SLOT_BSDF_U1);
      float r2 = rng.get(b, SLOT_BSDF_U2);
      rd = diffuse_scatter(n, r1, r2);
      thr = thr * alb;
    } else if (mt == 1) {
      float f1 = rng.get(b, SLOT_FUZZ_U1);
      float f2 = rng.get(b, SLOT_FUZZ_U2);
      rd = normalized(reflect(rd, n) + random_unit_vector(f1, f2) * rough);
      thr = thr * alb;
    } else if (mt == 4) {
      bool did = false;
      if (depth < p.direct_light_max_depth) {
        V3 d = p.reference_compat ? direct_light_compat(s, p, rng, b, hit_p, n, alb, cnt)
                                  : direct_light_full(s, p, rng, b, hit_p, n, alb, cnt);
        color = color + (thr * d) * rough;
        did = s.n_lights > 0;
      }
      float lobe = rng.get(b, SLOT_LOBE);
      if (lobe < rough) {
        float r1 = rng.get(b, SLOT_BSDF_U1);
        float r2 = rng.get(b, SLOT_BSDF_U2);
        rd = diffuse_scatter(n, r1, r2);
        nee_here = did;
      } else {
        float f1 = rng.get(b, SLOT_FUZZ_U1);
        float f2 = rng.get(b, SLOT_FUZZ_U2);
        rd = normalized(reflect(rd, n) + random_unit_vector(f1, f2) * rough);
      }
      thr = thr * alb;
    } else if (mt == 2) {
      float eta;
      if (front) {
        eta = cur_ior / ior;
        cur_ior = ior;
      } else {
        eta = cur_ior / 1.0f;
        cur_ior = 1.0f;
      }
      // scatter.py:71-81
      float cos_t = std::min(-dot(rd, n), 1.0f);
      float sin_t = std::sqrt(1.0f - cos_t * cos_t);
      bool cannot = eta * sin_t > 1.0f;
      bool refl = cannot;
      if (!cannot) refl = schlick(cos_t, eta) > rng.get(b, SLOT_LOBE);
      rd = refl ? reflect(rd, n) : refract(rd, n, eta);
      thr = thr * alb;
    }
    prev_nee = nee_here;
    // trace.py:227-232
    if (depth > 2) {
      float rr = std::max(thr.x, std::max(thr.y, thr.z));
      if (rng.get(b, SLOT_RR) > rr) break;
      thr = thr / rr;
    }
    ro = hit_p + n * 1e-4f;
  }
  o.color = color;
  return o;
}

inline float fractf(float x) { return x - std::floor(x); }

// camera.py:23-30 with the counter-based per-pixel phase in place of the
// sin-hash (camera.py:9-20): jitter = fract(phase + (frame + 1) * R2).
inline V3 camera_dir(const orc_params& p, int px, int py, int frame, uint32_t k0, uint32_t k1) {
  uint32_t ctr[4] = {(uint32_t)(py * p.width + px), 0xFFFFFFFFu, 0xFFFFFFFFu, 0u};
  uint32_t ph[4];
  philox4x32_10(ctr, k0, k1, ph);
  float i = (float)(frame + 1);
  float jx = fractf(u01(ph[0]) + i * 0.7548776662466927f);
  float jy = fractf(u01(ph[1]) + i * 0.5698402909980532f);
  float u = ((float)px + jx) / (float)p.width * 2.0f - 1.0f;
  float v = 1.0f - ((float)py + jy) / (float)p.height * 2.0f;
  float ndx = u * p.aspect * p.fov_tan;
  float ndy = v * p.fov_tan;
  V3 f = mk(p.cam_fwd[0], p.cam_fwd[1], p.cam_fwd[2]);
  V3 r = mk(p.cam_right[0], p.cam_right[1], p.cam_right[2]);
  V3 up = mk(p.cam_up[0], p.cam_up[1], p.cam_up[2]);
  return normalized((f + r * ndx) + up * ndy);
}

const uint32_t kKeyHi = 0x5EEDC0DEu;

}  // namespace

extern "C" {

int orc_version(void) { return 3; }

void orc_philox(const uint32_t* ctr, uint32_t k0, uint32_t k1, uint32_t* out) {
  philox4x32_10(ctr, k0, k1, out);
}

// Closest-hit traversal of the reference BVH (intersect.py:81-152) for n rays.
void orc_bvh_intersect(const orc_scene* s, long n, const float* ro, const float* rd,
                       float* out_t, int* out_idx, float* out_u, float* out_v) {
#pragma omp parallel for schedule(dynamic, 256)
  for (long i = 0; i < n; ++i) {
    int idx;
    float u, v;
    float t = s->n_tris > 0 ? bvh_intersect(*s, ld3(ro, i), ld3(rd, i), idx, u, v) : 1e9f;
    if (s->n_tris <= 0) { idx = -1; u = 0.0f; v = 0.0f; }
    out_t[i] = t;
    out_idx[i] = idx;
    out_u[i] = u;
    out_v[i] = v;
  }
}

// Any-hit of the reference BVH (intersect.py:155-219).
void orc_bvh_occluded(const orc_scene* s, long n, const float* ro, const float* rd,
                      const float* max_t, int* out) {
#pragma omp parallel for schedule(dynamic, 256)
  for (long i = 0; i < n; ++i)
    out[i] = s->n_tris > 0 ? (int)bvh_occluded(*s, ld3(ro, i), ld3(rd, i), max_t[i]) : 0;
}

// Full scene query (intersect.py:249-309): t, hit index, is_bvh, u, v, normal.
void orc_scene_intersect(const orc_scene* s, long n, const float* ro, const float* rd,
                         float* out_t, int* out_idx, int* out_is_bvh, float* out_u,
                         float* out_v, float* out_normal) {
#pragma omp parallel for schedule(dynamic, 256)
  for (long i = 0; i < n; ++i) {
    Hit h = scene_intersect(*s, ld3(ro, i), ld3(rd, i));
    out_t[i] = h.t;
    out_idx[i] = h.idx;
    out_is_bvh[i] = h.is_bvh;
    out_u[i] = h.u;
    out_v[i] = h.v;
    out_normal[3 * i] = h.normal.x;
    out_normal[3 * i + 1] = h.normal.y;
    out_normal[3 * i + 2] = h.normal.z;
  }
}

// Single-triangle Moller-Trumbore (intersect.py:57-78) for n (ray, tri) pairs.
void orc_tri_intersect(long n, const float* ro, const float* rd, const float* v0,
                       const float* v1, const float* v2, float* out_t, float* out_u,
                       float* out_v) {
  for (long i = 0; i < n; ++i) {
    float u, v;
    out_t[i] = tri_intersect(ld3(ro, i), ld3(rd, i), ld3(v0, i), ld3(v1, i), ld3(v2, i), u, v);
    out_u[i] = u;
    out_v[i] = v;
  }
}

// One path from (ro, rd) with the random numbers taken in call order from
// _sample_texture for n uvs of texture `ti` -> out[n*3].
void orc_sample_texture(const orc_scene* s, int ti, int n, const float* uv, float* out) {
  for (int i = 0; i < n; ++i) {
    V3 c = sample_texture(*s, ti, uv[2 * i], uv[2 * i + 1]);
    out[3 * i] = c.x; out[3 * i + 1] = c.y; out[3 * i + 2] = c.z;
  }
}

// _bvh_albedo of BVH-order triangles tri[i] with material mat[i] at
// barycentrics (u[i], v[i]) over base albedo base[i*3] -> out[n*3].
void orc_bvh_albedo(const orc_scene* s, int n, const int* tri, const int* mat, const float* u, const float* v,
                    const float* base, float* out) {
  for (int i = 0; i < n; ++i) {
    V3 c = bvh_albedo(*s, tri[i], mat[i], u[i], v[i], mk(base[3 * i], base[3 * i + 1], base[3 * i + 2]));
    out[3 * i] = c.x; out[3 * i + 1] = c.y; out[3 * i + 2] = c.z;
  }
}

// `stream` — the way the reference's trace() consumes ti.random().  Used to
// pin this restatement against the reference's own trace source.
int orc_trace_scripted(const orc_scene* s, const orc_params* p, const float* ro, const float* rd,
                       const float* stream, int n_stream, float* out_color, float* out_normal,
                       float* out_albedo, float* out_depth, long* out_rays) {
  Rng rng;
  std::memset(&rng, 0, sizeof(rng));
  rng.scripted = true;
  rng.stream = stream;
  rng.n_stream = n_stream;
  Counters cnt = {0};
  PathOut o = trace(*s, *p, rng, ld3(ro, 0), ld3(rd, 0), cnt);
  out_color[0] = o.color.x; out_color[1] = o.color.y; out_color[2] = o.color.z;
  out_normal[0] = o.normal.x; out_normal[1] = o.normal.y; out_normal[2] = o.normal.z;
  out_albedo[0] = o.albedo.x; out_albedo[1] = o.albedo.y; out_albedo[2] = o.albedo.z;
  out_depth[0] = o.depth;
  out_rays[0] = cnt.rays;
  return rng.pos;
}

// Progressive render of frames [frame0, frame1) over rows [y0, y1) with the
// counter-based RNG, accumulating running means exactly as render_kernel
// does (trace.py:262-283).  Accumulators are full-image (height x width).
// Returns the number of rays cast (trace iterations + shadow rays).
long orc_render(const orc_scene* s, const orc_params* p, int frame0, int frame1, int y0, int y1,
                float* acc, float* acc_normal, float* acc_albedo, float* acc_depth,
                float* pixels, int n_threads) {
  long total = 0;
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
  const int W = p->width;
  for (int frame = frame0; frame < frame1; ++frame) {
    long frame_rays = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : frame_rays)
    for (long pix = (long)y0 * W; pix < (long)y1 * W; ++pix) {
      int px = (int)(pix % W), py = (int)(pix / W);
      Rng rng;
      std::memset(&rng, 0, sizeof(rng));
      rng.key0 = p->seed;
      rng.key1 = kKeyHi;
      rng.pixel = (uint32_t)pix;
      rng.sample = (uint32_t)frame;
      Counters cnt = {0};
      V3 rd = camera_dir(*p, px, py, frame, p->seed, kKeyHi);
      V3 ro = mk(p->cam_pos[0], p->cam_pos[1], p->cam_pos[2]);
      PathOut o = trace(*s, *p, rng, ro, rd, cnt);
      frame_rays += cnt.rays;
      V3 smp = o.color;
      if (p->sample_clamp > 0.0f) {
        float c = p->sample_clamp;
        smp = mk(std::min(std::max(smp.x, 0.0f), c), std::min(std::max(smp.y, 0.0f), c),
                 std::min(std::max(smp.z, 0.0f), c));
      }
      float* a = acc + 3 * pix;
      float* an = acc_normal + 3 * pix;
      float* aa = acc_albedo + 3 * pix;
      if (frame == 0) {
        a[0] = smp.x; a[1] = smp.y; a[2] = smp.z;
        an[0] = o.normal.x; an[1] = o.normal.y; an[2] = o.normal.z;
        aa[0] = o.albedo.x; aa[1] = o.albedo.y; aa[2] = o.albedo.z;
        acc_depth[pix] = o.depth;
      } else {
        float f = (float)frame, f1 = (float)(frame + 1);
        a[0] = (a[0] * f + smp.x) / f1; a[1] = (a[1] * f + smp.y) / f1; a[2] = (a[2] * f + smp.z) / f1;
        an[0] = (an[0] * f + o.normal.x) / f1; an[1] = (an[1] * f + o.normal.y) / f1;
        an[2] = (an[2] * f + o.normal.z) / f1;
        aa[0] = (aa[0] * f + o.albedo.x) / f1; aa[1] = (aa[1] * f + o.albedo.y) / f1;
        aa[2] = (aa[2] * f + o.albedo.z) / f1;
        acc_depth[pix] = (acc_depth[pix] * f + o.depth) / f1;
      }
      for (int c = 0; c < 3; ++c) pixels[3 * pix + c] = std::sqrt(std::min(a[c], 1.0f));
    }
    total += frame_rays;
  }
  return total;
}

// Per-sample radiance (no accumulation) for frames [frame0, frame1), used by
// statistical image tests: out[(f - frame0) * H * W + pix] rgb.
long orc_render_samples(const orc_scene* s, const orc_params* p, int frame0, int frame1,
                        float* out, int n_threads) {
  long total = 0;
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
  const long P = (long)p->width * p->height;
  for (int frame = frame0; frame < frame1; ++frame) {
    long fr = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : fr)
    for (long pix = 0; pix < P; ++pix) {
      int px = (int)(pix % p->width), py = (int)(pix / p->width);
      Rng rng;
      std::memset(&rng, 0, sizeof(rng));
      rng.key0 = p->seed;
      rng.key1 = kKeyHi;
      rng.pixel = (uint32_t)pix;
      rng.sample = (uint32_t)frame;
      Counters cnt = {0};
      V3 rd = camera_dir(*p, px, py, frame, p->seed, kKeyHi);
      PathOut o = trace(*s, *p, rng, mk(p->cam_pos[0], p->cam_pos[1], p->cam_pos[2]), rd, cnt);
      fr += cnt.rays;
      V3 smp = o.color;
      if (p->sample_clamp > 0.0f) {
        float c = p->sample_clamp;
        smp = mk(std::min(std::max(smp.x, 0.0f), c), std::min(std::max(smp.y, 0.0f), c),
                 std::min(std::max(smp.z, 0.0f), c));
      }
      float* o3 = out + 3 * ((long)(frame - frame0) * P + pix);
      o3[0] = smp.x; o3[1] = smp.y; o3[2] = smp.z;
    }
    total += fr;
  }
  return total;
}

// ----------------------------------------------------------------------------
// BVH build restating GPUBVHBuilder's Morton method
// (rendering/taichi/bvh_builder.py:353-478): triangle AABBs padded by 1e-4,
// centroid Morton codes with 10 bits per axis, stable sort, recursive
// median-by-count split, DFS pre-order node numbering.
// Outputs are sized for the worst case (2n - 1 nodes).  Returns node count.
// ----------------------------------------------------------------------------
namespace {
inline uint32_t expand_bits(uint32_t v) {
  v &= 0x000003ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

struct BuildCtx {
  const float* bmin;
  const float* bmax;
  const int* order;
  int leaf;
  float* out_min;
  float* out_max;
  int* left;
  int* right;
  int* start;
  int* count;
  int n_nodes;
};

int build_node(BuildCtx& c, int s, int e) {
  int idx = c.n_nodes++;
  int cnt = e - s;
  if (cnt <= c.leaf) {
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = s; i < e; ++i) {
      int t = c.order[i];
      for (int k = 0; k < 3; ++k) {
        mn[k] = std::min(mn[k], c.bmin[3 * t + k]);
        mx[k] = std::max(mx[k], c.bmax[3 * t + k]);
      }
    }
    for (int k = 0; k < 3; ++k) {
      c.out_min[3 * idx + k] = mn[k];
      c.out_max[3 * idx + k] = mx[k];
    }
    c.left[idx] = -1;
    c.right[idx] = -1;
    c.start[idx] = s;
    c.count[idx] = cnt;
  } else {
    int mid = (s + e) / 2;
    int l = build_node(c, s, mid);
    int r = build_node(c, mid, e);
    for (int k = 0; k < 3; ++k) {
      c.out_min[3 * idx + k] = std::min(c.out_min[3 * l + k], c.out_min[3 * r + k]);
      c.out_max[3 * idx + k] = std::max(c.out_max[3 * l + k], c.out_max[3 * r + k]);
    }
    c.left[idx] = l;
    c.right[idx] = r;
    c.start[idx] = -1;
    c.count[idx] = 0;
  }
  return idx;
}
}  // namespace

int orc_bvh_build_morton(int n, const float* v0, const float* v1, const float* v2, int leaf_size,
                         float* out_min, float* out_max, int* out_left, int* out_right,
                         int* out_start, int* out_count, int* out_order) {
  if (n <= 0) return 0;
  std::vector<float> bmin(3 * (size_t)n), bmax(3 * (size_t)n), cen(3 * (size_t)n);
  const float eps = 1e-4f;
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) {
      float a = v0[3 * i + k], b = v1[3 * i + k], c = v2[3 * i + k];
      bmin[3 * i + k] = std::min(a, std::min(b, c)) - eps;
      bmax[3 * i + k] = std::max(a, std::max(b, c)) + eps;
      cen[3 * i + k] = ((a + b) + c) / 3.0f;
    }
  }
  float mins[3], ext[3];
  for (int k = 0; k < 3; ++k) {
    float lo = INFINITY, hi = -INFINITY;
    for (int i = 0; i < n; ++i) {
      lo = std::min(lo, cen[3 * i + k]);
      hi = std::max(hi, cen[3 * i + k]);
    }
    mins[k] = lo;
    ext[k] = hi - lo;
    if (ext[k] <= 1e-12f) ext[k] = 1.0f;
  }
  std::vector<uint32_t> codes(n);
  const float scale = 1023.0f;
  for (int i = 0; i < n; ++i) {
    uint32_t q[3];
    for (int k = 0; k < 3; ++k) {
      float x = (cen[3 * i + k] - mins[k]) / ext[k];
      x = std::min(std::max(x, 0.0f), 1.0f);
      q[k] = (uint32_t)(x * scale);
    }
    codes[i] = (expand_bits(q[0]) << 2) | (expand_bits(q[1]) << 1) | expand_bits(q[2]);
  }
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return codes[a] < codes[b]; });
  BuildCtx c;
  c.bmin = bmin.data();
  c.bmax = bmax.data();
  c.order = order.data();
  c.leaf = leaf_size;
  c.out_min = out_min;
  c.out_max = out_max;
  c.left = out_left;
  c.right = out_right;
  c.start = out_start;
  c.count = out_count;
  c.n_nodes = 0;
  build_node(c, 0, n);
  for (int i = 0; i < n; ++i) out_order[i] = order[i];
  return c.n_nodes;
}

}  // extern "C"
