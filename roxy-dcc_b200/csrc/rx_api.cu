// C ABI of libroxy_cuda.so (declared in include/roxy.h).  Thin wrappers:
// argument checks, host<->device copies, locking, error text.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "rx_internal.cuh"
#include "rx_runtime.h"

struct rx_ctx {
  rx::Ctx c;
};
struct rx_scene {
  rx::Scene s;
};
struct rx_accum {
  rx::Accum* a;
  rx::Ctx* ctx;
};
struct rx_batch {
  rx::Batch* b;
  rx::Ctx* ctx;
};
struct rx_server {
  rx::Server* s;
  rx::Ctx* ctx;
};
struct rx_obj {
  rx::ObjParse* o;
  rx::Ctx* ctx;
};

namespace rx {

static thread_local std::string g_err;

void set_error(Ctx* ctx, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx) ctx->err = buf;
  g_err = buf;
}

int Scene::upload_palette(Ctx* c) {
  std::vector<float4> a, b;
  auto push = [&](const HostMat& m) {
    a.push_back(make_float4(m.albedo[0], m.albedo[1], m.albedo[2], int_bits_as_float(m.type)));
    b.push_back(make_float4(m.roughness, m.ior, m.emission, int_bits_as_float(m.texture)));
  };
  for (auto& m : user_mats) push(m);
  for (auto& m : obj_mats) push(m);
  if (a.empty()) {
    HostMat d = {0, {0.8f, 0.8f, 0.8f}, 0.0f, 1.0f, 0.0f};
    push(d);
  }
  if ((int)a.size() != n_mats || !mat_a.p) {
    if (!mat_a.alloc(c, a.size()) || !mat_b.alloc(c, b.size()))
      return set_error(c, "out of device memory for the material palette"), RX_ERR_CAPACITY;
  }
  CUDA_TRY(c, cudaMemcpyAsync(mat_a.p, a.data(), sizeof(float4) * a.size(), cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(mat_b.p, b.data(), sizeof(float4) * b.size(), cudaMemcpyHostToDevice, c->stream));
  n_mats = (int)a.size();
  return RX_OK;
}

// The linear slots scanned before the BVH: all objects, or, when the BVH
// holds the bounded analytic objects (spheres and cubes), planes and slot
// triangles only.
int Scene::upload_linear_objects(Ctx* c, bool exclude_bvh_objects) {
  std::vector<ObjSlot> lin;
  lin_slot.clear();
  for (int i = 0; i < (int)objs.size(); ++i) {
    if (exclude_bvh_objects && (objs[i].type == 0 || objs[i].type == 2)) continue;
    lin.push_back(objs[i]);
    lin_slot.push_back(i);
  }
  n_lin = (int)lin.size();
  if (!d_objs.alloc(c, std::max<size_t>(lin.size(), 1))) return set_error(c, "out of device memory"), RX_ERR_CAPACITY;
  if (!lin.empty())
    CUDA_TRY(c, cudaMemcpyAsync(d_objs.p, lin.data(), sizeof(ObjSlot) * lin.size(), cudaMemcpyHostToDevice,
                                c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  ++version;
  return upload_light_maps(c);
}

// light index of every emitting triangle / object slot / linear object
int Scene::upload_light_maps(Ctx* c) {
  if (light_src.empty() || (int)light_src.size() != n_lights || (int)light_kind.size() != n_lights) return RX_OK;
  std::vector<int> lt(std::max(n_tris, 1), -1), lo(std::max<size_t>(objs.size(), 1), -1), ll(std::max(n_lin, 1), -1);
  for (int i = 0; i < n_lights; ++i) {
    const int s = light_src[i];
    if (light_kind[i] == 1 && s >= 0 && s < n_tris) lt[s] = i;
    if (light_kind[i] == 0 && s >= 0 && s < (int)objs.size()) lo[s] = i;
  }
  for (int j = 0; j < n_lin && j < (int)lin_slot.size(); ++j) ll[j] = lo[lin_slot[j]];
  auto up = [&](DevBuf<int>& d, const std::vector<int>& h) -> int {
    if (!d.alloc(c, h.size())) return set_error(c, "out of device memory"), RX_ERR_CAPACITY;
    CUDA_TRY(c, cudaMemcpyAsync(d.p, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice, c->stream));
    return RX_OK;
  };
  int rc;
  if ((rc = up(d_light_of_tri, lt)) || (rc = up(d_light_of_obj, lo)) || (rc = up(d_light_of_lin, ll))) return rc;
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  ++version;
  return RX_OK;
}

}  // namespace rx

using namespace rx;

#define LOCK(ctxp) std::lock_guard<std::recursive_mutex> _lk((ctxp)->mu)

// SAH costs of one node traversal step and one primitive test, used to decide
// which LBVH subtrees collapse into leaves.
#ifndef RX_SAH_CT
#define RX_SAH_CT 0.6f
#endif
#ifndef RX_SAH_CI
#define RX_SAH_CI 1.0f
#endif

extern "C" {

int rx_version(void) { return 1; }

int rx_device_count(int* out) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    set_error(nullptr, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
    if (out) *out = 0;
    return RX_ERR_CUDA;
  }
  if (out) *out = n;
  return RX_OK;
}

const char* rx_last_error(const rx_ctx* ctx) { return ctx ? ctx->c.err.c_str() : g_err.c_str(); }

int rx_ctx_create(int device, rx_ctx** out) {
  if (!out) return set_error(nullptr, "rx_ctx_create: out is NULL"), RX_ERR_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
    return set_error(nullptr, "no CUDA device is available"), RX_ERR_CUDA;
  if (device < 0 || device >= n) return set_error(nullptr, "device %d out of range [0, %d)", device, n), RX_ERR_ARG;
  rx_ctx* c = new rx_ctx();
  c->c.device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->c.stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->c.num_sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) {
    // stream-ordered allocations keep freed memory in the device pool, so
    // accumulators and wave state of later requests reuse it without new
    // mappings
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      unsigned long long keep = ~0ULL;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
  }
  if (e == cudaSuccess) e = cudaMalloc(&c->c.d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(c->c.d_err, 0, sizeof(int));
  if (e != cudaSuccess) {
    set_error(nullptr, "context creation failed: %s", cudaGetErrorString(e));
    delete c;
    return RX_ERR_CUDA;
  }
  *out = c;
  return RX_OK;
}

int rx_ctx_destroy(rx_ctx* ctx) {
  if (!ctx) return RX_OK;
  cudaSetDevice(ctx->c.device);
  cudaStreamSynchronize(ctx->c.stream);
  host_stage_free(&ctx->c);
  cudaFree(ctx->c.d_err);
  cudaStreamDestroy(ctx->c.stream);
  delete ctx;
  return RX_OK;
}

int rx_ctx_hold(rx_ctx* ctx) {
  if (!ctx) return RX_ERR_ARG;
  ctx->c.hold_waiters.fetch_add(1);
  ctx->c.mu.lock();
  ctx->c.hold_waiters.fetch_sub(1);
  return RX_OK;
}

int rx_ctx_release(rx_ctx* ctx) {
  if (!ctx) return RX_ERR_ARG;
  ctx->c.mu.unlock();
  return RX_OK;
}

int rx_ctx_sync(rx_ctx* ctx) {
  if (!ctx) return RX_ERR_ARG;
  LOCK(&ctx->c);
  cudaSetDevice(ctx->c.device);
  CUDA_TRY(&ctx->c, cudaDeviceSynchronize());
  // error bits a kernel raised (a bounded wait that ran out, an overflow)
  int e = 0;
  CUDA_TRY(&ctx->c, cudaMemcpy(&e, ctx->c.d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    CUDA_TRY(&ctx->c, cudaMemset(ctx->c.d_err, 0, sizeof(int)));
    return set_error(&ctx->c, "device error flags 0x%x", e), RX_ERR_DEVICE;
  }
  return RX_OK;
}

int rx_conv_set_impl(rx_ctx* ctx, int impl) {
  if (!ctx || impl < 0 || impl > 2) return set_error(ctx ? &ctx->c : nullptr, "rx_conv_set_impl: 0, 1 or 2"), RX_ERR_ARG;
  ctx->c.conv_impl = impl;
  return RX_OK;
}

void* rx_ctx_stream(rx_ctx* ctx) { return ctx ? (void*)ctx->c.stream : nullptr; }

int rx_scene_create(rx_ctx* ctx, rx_scene** out) {
  if (!ctx || !out) return set_error(nullptr, "rx_scene_create: NULL argument"), RX_ERR_ARG;
  LOCK(&ctx->c);
  rx_scene* s = new rx_scene();
  s->s.ctx = &ctx->c;
  *out = s;
  return RX_OK;
}

int rx_scene_destroy(rx_scene* scene) {
  if (!scene) return RX_OK;
  Ctx* c = scene->s.ctx;
  {
    LOCK(c);
    cudaSetDevice(c->device);
    delete scene;
    cudaStreamSynchronize(c->stream);
  }
  return RX_OK;
}

}  // extern "C"

template <class T>
static int upload(Ctx* c, DevBuf<T>& buf, const T* host, size_t n) {
  if (!buf.alloc(c, std::max<size_t>(n, 1))) return set_error(c, "out of device memory (%zu elements)", n), RX_ERR_CAPACITY;
  if (n && host) CUDA_TRY(c, cudaMemcpyAsync(buf.p, host, sizeof(T) * n, cudaMemcpyHostToDevice, c->stream));
  return RX_OK;
}

extern "C" {

int rx_scene_set_triangles(rx_scene* scene, int n, const float* v0, const float* v1, const float* v2,
                           const float* n0, const float* n1, const float* n2, const int* mat_idx) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  cudaSetDevice(c->device);
  if (n < 0 || (n > 0 && (!v0 || !v1 || !v2))) return set_error(c, "set_triangles: bad arguments"), RX_ERR_ARG;
  if (n >= (1 << 30)) return set_error(c, "set_triangles: %d triangles exceed the limit", n), RX_ERR_CAPACITY;
  size_t k = (size_t)3 * n;
  int rc;
  if ((rc = upload(c, s.v0b, v0, k)) || (rc = upload(c, s.v1b, v1, k)) || (rc = upload(c, s.v2b, v2, k))) return rc;
  // missing normals: face normals are not implied; the caller passes them
  if ((rc = upload(c, s.n0b, n0 ? n0 : v0, k)) || (rc = upload(c, s.n1b, n1 ? n1 : v0, k)) ||
      (rc = upload(c, s.n2b, n2 ? n2 : v0, k)))
    return rc;
  std::vector<int> zeros;
  if (!mat_idx) zeros.assign(std::max(n, 1), 0);
  if ((rc = upload(c, s.tri_matb, mat_idx ? mat_idx : zeros.data(), (size_t)n))) return rc;
  s.d_v0 = s.v0b.p; s.d_v1 = s.v1b.p; s.d_v2 = s.v2b.p;
  s.d_n0 = s.n0b.p; s.d_n1 = s.n1b.p; s.d_n2 = s.n2b.p;
  s.d_tri_mat = s.tri_matb.p;
  s.n_tris = n;
  s.uvb.release();
  s.clear_bvh();
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return RX_OK;
}

int rx_scene_alloc_triangles(rx_scene* scene, int n) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  cudaSetDevice(c->device);
  if (n < 0) return set_error(c, "alloc_triangles: negative count"), RX_ERR_ARG;
  if (n >= (1 << 30)) return set_error(c, "alloc_triangles: %d triangles exceed the limit", n), RX_ERR_CAPACITY;
  return scene_alloc_triangles(c, &s, n);
}

int rx_scene_put_triangles(rx_scene* scene, int offset, int n, const float* v0, const float* v1, const float* v2,
                           const float* n0, const float* n1, const float* n2, const int* mat_idx) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  cudaSetDevice(c->device);
  if (n > 0 && (!v0 || !v1 || !v2)) return set_error(c, "put_triangles: bad arguments"), RX_ERR_ARG;
  const float* rows[6] = {v0, v1, v2, n0, n1, n2};
  return scene_put_triangles(c, &s, offset, n, rows, mat_idx);
}

int rx_scene_put_indexed(rx_scene* scene, int offset, int n_tris, int n_pos, const double* positions,
                         const int* tri_pos_idx, int n_nrm, const double* normals, const int* tri_nrm_idx,
                         const double* matrix, const double* normal_matrix, const int* tri_group_idx, int n_groups,
                         const int* group_mat) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  cudaSetDevice(c->device);
  return scene_put_indexed(c, &s, offset, n_tris, n_pos, positions, tri_pos_idx, n_nrm, normals, tri_nrm_idx, matrix,
                           normal_matrix, tri_group_idx, n_groups, group_mat);
}

int rx_scene_get_triangles(rx_scene* scene, int offset, int n, float* v0, float* v1, float* v2, float* n0, float* n1,
                           float* n2, int* mat_idx) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  cudaSetDevice(c->device);
  float* rows[6] = {v0, v1, v2, n0, n1, n2};
  return scene_get_triangles(c, &s, offset, n, rows, mat_idx);
}

int rx_scene_put_uvs(rx_scene* scene, int offset, int n, const float* uv0, const float* uv1, const float* uv2,
                     const int* has_uv) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  cudaSetDevice(c->device);
  return scene_put_uvs(c, &s, offset, n, uv0, uv1, uv2, has_uv);
}

int rx_scene_set_textures(rx_scene* scene, int n, const int* width, const int* height, const int* flip_v,
                          const unsigned char* texels) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  cudaSetDevice(c->device);
  return scene_set_textures(c, &s, n, width, height, flip_v, texels);
}

int rx_scene_set_material_textures(rx_scene* scene, int n, const int* texture_idx) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  cudaSetDevice(c->device);
  if (n != (int)s.user_mats.size() || (n > 0 && !texture_idx))
    return set_error(c, "set_material_textures: %d entries for a palette of %zu", n, s.user_mats.size()),
           RX_ERR_ARG;
  for (int i = 0; i < n; ++i) s.user_mats[i].texture = texture_idx[i] < 0 ? -1 : texture_idx[i];
  int rc = s.upload_palette(c);
  if (rc) return rc;
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  ++s.version;
  return RX_OK;
}

int rx_scene_set_materials(rx_scene* scene, int n, const int* type, const float* albedo, const float* roughness,
                           const float* ior, const float* emission) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  if (n < 0 || (n > 0 && (!type || !albedo || !roughness || !ior || !emission)))
    return set_error(c, "set_materials: bad arguments"), RX_ERR_ARG;
  s.user_mats.resize(n);
  for (int i = 0; i < n; ++i) {
    HostMat& m = s.user_mats[i];
    m.type = type[i];
    m.albedo[0] = albedo[3 * i]; m.albedo[1] = albedo[3 * i + 1]; m.albedo[2] = albedo[3 * i + 2];
    m.roughness = roughness[i];
    m.ior = ior[i];
    m.emission = emission[i];
    m.texture = -1;
  }
  // object materials follow the caller's palette: re-index the slots
  for (int i = 0; i < (int)s.objs.size(); ++i) s.objs[i].mat = n + i;
  ++s.version;
  cudaSetDevice(c->device);
  int rc = s.upload_palette(c);
  if (rc) return rc;
  return s.upload_linear_objects(c, s.method == RX_BVH_LBVH_SAH && s.n_bvh_spheres > 0);
}

int rx_scene_set_objects(rx_scene* scene, int n, const int* type, const float* center, const float* radius,
                         const float* normal, const float* offset, const float* extra, const float* v0,
                         const float* v1, const float* v2, const int* mat_type, const float* albedo,
                         const float* roughness, const float* ior, const float* emission) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  if (n < 0 || (n > 0 && (!type || !mat_type || !albedo || !roughness || !ior || !emission)))
    return set_error(c, "set_objects: bad arguments"), RX_ERR_ARG;
  s.objs.assign(n, ObjSlot());
  s.obj_mats.assign(n, HostMat());
  int base = (int)s.user_mats.size();
  auto g3 = [](const float* p, int i) { return p ? f3(p[3 * i], p[3 * i + 1], p[3 * i + 2]) : f3(0, 0, 0); };
  for (int i = 0; i < n; ++i) {
    ObjSlot& o = s.objs[i];
    o.type = type[i];
    if (o.type != 0 && o.type != 1 && o.type != 2 && o.type != 4)
      return set_error(c, "set_objects: slot %d has unsupported type %d", i, o.type), RX_ERR_ARG;
    o.mat = base + i;
    o.center = g3(center, i);
    o.radius = radius ? radius[i] : 0.0f;
    o.normal = g3(normal, i);
    o.offset = offset ? offset[i] : 0.0f;
    o.extra = g3(extra, i);
    o.v0 = g3(v0, i);
    o.v1 = g3(v1, i);
    o.v2 = g3(v2, i);
    HostMat& m = s.obj_mats[i];
    m.type = mat_type[i];
    m.albedo[0] = albedo[3 * i]; m.albedo[1] = albedo[3 * i + 1]; m.albedo[2] = albedo[3 * i + 2];
    m.roughness = roughness[i];
    m.ior = ior[i];
    m.emission = emission[i];
  }
  cudaSetDevice(c->device);
  s.clear_bvh();
  int rc = s.upload_palette(c);
  if (rc) return rc;
  return s.upload_linear_objects(c, false);
}

int rx_scene_set_lights(rx_scene* scene, int n, const int* kind, const float* p0, const float* p1, const float* p2,
                        const float* albedo, const float* emission, const float* area, const float* pick_pdf,
                        const float* alias_prob, const int* alias_idx) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  if (n < 0 || (n > 0 && (!kind || !p0 || !p1 || !albedo || !emission || !pick_pdf || !alias_prob || !alias_idx)))
    return set_error(c, "set_lights: bad arguments"), RX_ERR_ARG;
  std::vector<Light> L(std::max(n, 1));
  for (int i = 0; i < n; ++i) {
    Light& l = L[i];
    l.kind = kind[i];
    if (l.kind != 0 && l.kind != 1) return set_error(c, "set_lights: light %d has kind %d", i, l.kind), RX_ERR_ARG;
    l.p0 = f3(p0[3 * i], p0[3 * i + 1], p0[3 * i + 2]);
    l.p1 = f3(p1[3 * i], p1[3 * i + 1], p1[3 * i + 2]);
    l.p2 = p2 ? f3(p2[3 * i], p2[3 * i + 1], p2[3 * i + 2]) : f3(0, 0, 0);
    l.albedo = f3(albedo[3 * i], albedo[3 * i + 1], albedo[3 * i + 2]);
    l.emission = emission[i];
    l.area = area ? area[i] : 0.0f;
    l.pick_pdf = pick_pdf[i];
    if (alias_idx[i] < 0 || alias_idx[i] >= n)
      return set_error(c, "set_lights: alias index %d out of range", alias_idx[i]), RX_ERR_ARG;
  }
  cudaSetDevice(c->device);
  int rc;
  if ((rc = upload(c, s.d_lights, L.data(), L.size())) ||
      (rc = upload(c, s.d_alias_prob, alias_prob, (size_t)n)) || (rc = upload(c, s.d_alias_idx, alias_idx, (size_t)n)))
    return rc;
  s.n_lights = n;
  s.light_kind.assign(kind, kind + n);
  s.light_src.clear();  // sources refer to the previous list
  ++s.version;
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return RX_OK;
}

int rx_scene_set_light_sources(rx_scene* scene, int n, const int* source) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  if (n != s.n_lights || (n > 0 && !source))
    return set_error(c, "set_light_sources: %d sources for %d lights", n, s.n_lights), RX_ERR_ARG;
  s.light_src.assign(source, source + n);
  cudaSetDevice(c->device);
  return s.upload_light_maps(c);
}

int rx_bvh_build(rx_scene* scene, int method, int max_leaf, int spheres_in_bvh) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  cudaSetDevice(c->device);
  if (max_leaf < 1 || max_leaf > (1 << 20)) return set_error(c, "max_leaf must be >= 1"), RX_ERR_ARG;
  int rc;
  if ((long long)s.n_tris + (long long)s.objs.size() >= kMaxPrims)
    return set_error(c, "bvh_build: %d primitives exceed the %d-primitive limit", s.n_tris, kMaxPrims),
           RX_ERR_CAPACITY;
  if (method == RX_BVH_REFERENCE) {
    if (max_leaf > kMaxLeafPrims)
      return set_error(c, "bvh_build: leaves hold at most %d primitives", kMaxLeafPrims), RX_ERR_ARG;
    if ((rc = s.upload_linear_objects(c, false))) return rc;
    rc = build_reference(c, &s, max_leaf);
  } else if (method == RX_BVH_LBVH_SAH) {
    if (max_leaf > 15) return set_error(c, "LBVH leaves hold at most 15 primitives"), RX_ERR_ARG;
    rc = build_lbvh(c, &s, max_leaf, spheres_in_bvh, RX_SAH_CT, RX_SAH_CI);
  } else {
    return set_error(c, "Unknown BVH build method: %d", method), RX_ERR_ARG;
  }
  if (rc) return rc;
  if ((rc = s.upload_palette(c))) return rc;
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  CUDA_TRY(c, cudaGetLastError());
  return RX_OK;
}

int rx_bvh_set_reference(rx_scene* scene, int n_nodes, const float* node_min, const float* node_max, const int* left,
                         const int* right, const int* tri_start, const int* tri_count, const int* order) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  cudaSetDevice(c->device);
  if (n_nodes < 0 || (n_nodes > 0 && (!node_min || !node_max || !left || !right || !tri_start || !tri_count || !order)))
    return set_error(c, "bvh_set_reference: bad arguments"), RX_ERR_ARG;
  // validate the tree before it reaches a kernel
  for (int i = 0; i < n_nodes; ++i) {
    if (left[i] == -1) {
      if (tri_count[i] > kMaxLeafPrims)
        return set_error(c, "bvh_set_reference: leaf %d holds %d > %d triangles", i, tri_count[i], kMaxLeafPrims),
               RX_ERR_ARG;
      if (tri_start[i] < 0 || tri_count[i] < 0 || (long long)tri_start[i] + tri_count[i] > s.n_tris)
        return set_error(c, "bvh_set_reference: leaf %d range out of bounds", i), RX_ERR_ARG;
    } else if (left[i] <= 0 || left[i] >= n_nodes || right[i] <= 0 || right[i] >= n_nodes) {
      return set_error(c, "bvh_set_reference: node %d has child out of range", i), RX_ERR_ARG;
    }
  }
  for (int i = 0; i < s.n_tris; ++i)
    if (order[i] < 0 || order[i] >= s.n_tris) return set_error(c, "bvh_set_reference: bad order entry"), RX_ERR_ARG;
  int rc = s.upload_linear_objects(c, false);
  if (rc) return rc;
  rc = set_reference_nodes(c, &s, n_nodes, node_min, node_max, left, right, tri_start, tri_count, order);
  if (rc) return rc;
  return s.upload_palette(c);
}

int rx_bvh_info(rx_scene* scene, int* n_nodes, int* n_prims, int* method, int* leaf_size, int* depth) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  if (n_nodes) *n_nodes = s.n_nodes;
  if (n_prims) *n_prims = s.n_prims;
  if (method) *method = s.method;
  if (leaf_size) *leaf_size = s.leaf_size;
  if (depth) *depth = s.depth;
  return RX_OK;
}

int rx_bvh_export_reference(rx_scene* scene, float* node_min, float* node_max, int* left, int* right, int* tri_start,
                            int* tri_count, int* order) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  cudaSetDevice(c->device);
  if (s.method != RX_BVH_REFERENCE || !s.ref_left.p)
    return set_error(c, "export_reference needs a tree built with RX_BVH_REFERENCE"), RX_ERR_STATE;
  size_t nn = s.n_nodes;
  cudaStream_t st = c->stream;
  CUDA_TRY(c, cudaMemcpyAsync(node_min, s.ref_min.p, sizeof(float3) * nn, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(c, cudaMemcpyAsync(node_max, s.ref_max.p, sizeof(float3) * nn, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(c, cudaMemcpyAsync(left, s.ref_left.p, sizeof(int) * nn, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(c, cudaMemcpyAsync(right, s.ref_right.p, sizeof(int) * nn, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(c, cudaMemcpyAsync(tri_start, s.ref_start.p, sizeof(int) * nn, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(c, cudaMemcpyAsync(tri_count, s.ref_count.p, sizeof(int) * nn, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(c, cudaMemcpyAsync(order, s.order.p, sizeof(int) * s.n_tris, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(c, cudaStreamSynchronize(st));
  return RX_OK;
}

int rx_bvh_export_layout(rx_scene* scene, float* nodes, int* order) {
  if (!scene || !nodes || !order) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  cudaSetDevice(c->device);
  if (s.n_nodes <= 0) return set_error(c, "export_layout: no BVH"), RX_ERR_STATE;
  CUDA_TRY(c, cudaMemcpyAsync(nodes, s.d_nodes.p, sizeof(float4) * 4 * (size_t)s.n_nodes, cudaMemcpyDeviceToHost,
                              c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(order, s.order.p, sizeof(int) * (size_t)s.n_prims, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return RX_OK;
}

static int check_scene_ready(Scene& s) {
  if (s.n_tris > 0 && s.n_nodes == 0) return set_error(s.ctx, "scene has triangles but no BVH"), RX_ERR_STATE;
  return RX_OK;
}

static int finish_device(Ctx* c) {
  int e = 0;
  CUDA_TRY(c, cudaMemcpyAsync(&e, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (e) {
    cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
    set_error(c, "device error flags 0x%x", e);
    return RX_ERR_DEVICE;
  }
  return RX_OK;
}

int rx_trace_closest(rx_scene* scene, long n, const float* ro, const float* rd, float* t, int* id, float* u, float* v) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  cudaSetDevice(c->device);
  if (n < 0 || (n > 0 && (!ro || !rd || !t || !id || !u || !v))) return set_error(c, "trace_closest: bad arguments"), RX_ERR_ARG;
  int rc = check_scene_ready(s);
  if (rc) return rc;
  if (n == 0) return RX_OK;
  DevBuf<float> dro(c, 3 * n), drd(c, 3 * n), dt(c, n), du(c, n), dv(c, n);
  DevBuf<int> did(c, n);
  CUDA_TRY(c, cudaMemcpyAsync(dro.p, ro, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(drd.p, rd, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, c->stream));
  if ((rc = trace_closest(c, &s, n, dro.p, drd.p, dt.p, did.p, du.p, dv.p))) return rc;
  CUDA_TRY(c, cudaMemcpyAsync(t, dt.p, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(id, did.p, sizeof(int) * n, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(u, du.p, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(v, dv.p, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
  return finish_device(c);
}

int rx_trace_closest_device(rx_scene* scene, long n, const float* d_ro, const float* d_rd, float* d_t, int* d_id,
                            float* d_u, float* d_v) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  cudaSetDevice(c->device);
  int rc = check_scene_ready(s);
  if (rc) return rc;
  return trace_closest(c, &s, n, d_ro, d_rd, d_t, d_id, d_u, d_v);
}

int rx_trace_any(rx_scene* scene, long n, const float* ro, const float* rd, const float* tmax, int* occluded) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  cudaSetDevice(c->device);
  if (n < 0 || (n > 0 && (!ro || !rd || !tmax || !occluded))) return set_error(c, "trace_any: bad arguments"), RX_ERR_ARG;
  int rc = check_scene_ready(s);
  if (rc) return rc;
  if (n == 0) return RX_OK;
  DevBuf<float> dro(c, 3 * n), drd(c, 3 * n), dtm(c, n);
  DevBuf<int> docc(c, n);
  CUDA_TRY(c, cudaMemcpyAsync(dro.p, ro, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(drd.p, rd, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(dtm.p, tmax, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream));
  if ((rc = trace_any(c, &s, n, dro.p, drd.p, dtm.p, docc.p))) return rc;
  CUDA_TRY(c, cudaMemcpyAsync(occluded, docc.p, sizeof(int) * n, cudaMemcpyDeviceToHost, c->stream));
  return finish_device(c);
}

int rx_scene_intersect(rx_scene* scene, long n, const float* ro, const float* rd, float* t, int* kind, int* id,
                       float* u, float* v, float* normal) {
  if (!scene) return RX_ERR_ARG;
  Scene& s = scene->s;
  Ctx* c = s.ctx;
  LOCK(c);
  cudaSetDevice(c->device);
  if (n < 0 || (n > 0 && (!ro || !rd || !t || !kind || !id || !u || !v || !normal)))
    return set_error(c, "scene_intersect: bad arguments"), RX_ERR_ARG;
  int rc = check_scene_ready(s);
  if (rc) return rc;
  if (n == 0) return RX_OK;
  if ((rc = s.upload_palette(c))) return rc;
  DevBuf<float> dro(c, 3 * n), drd(c, 3 * n), dt(c, n), du(c, n), dv(c, n), dn(c, 3 * n);
  DevBuf<int> dk(c, n), did(c, n);
  CUDA_TRY(c, cudaMemcpyAsync(dro.p, ro, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(drd.p, rd, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, c->stream));
  if ((rc = scene_query(c, &s, n, dro.p, drd.p, dt.p, dk.p, did.p, du.p, dv.p, dn.p))) return rc;
  CUDA_TRY(c, cudaMemcpyAsync(t, dt.p, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(kind, dk.p, sizeof(int) * n, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(id, did.p, sizeof(int) * n, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(u, du.p, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(v, dv.p, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(normal, dn.p, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, c->stream));
  return finish_device(c);
}

int rx_accum_create(rx_ctx* ctx, int width, int height, rx_accum** out) {
  if (!ctx || !out) return set_error(nullptr, "rx_accum_create: NULL argument"), RX_ERR_ARG;
  LOCK(&ctx->c);
  cudaSetDevice(ctx->c.device);
  if (width <= 0 || height <= 0 || (long long)width * height > (1LL << 28))
    return set_error(&ctx->c, "accumulator size %dx%d is invalid", width, height), RX_ERR_ARG;
  Accum* a = accum_new(&ctx->c, width, height);
  if (!a) return set_error(&ctx->c, "out of device memory for a %dx%d accumulator", width, height), RX_ERR_CAPACITY;
  rx_accum* r = new rx_accum();
  r->a = a;
  r->ctx = &ctx->c;
  *out = r;
  return RX_OK;
}

int rx_accum_destroy(rx_accum* acc) {
  if (!acc) return RX_OK;
  Ctx* c = acc->ctx;
  LOCK(c);
  cudaSetDevice(c->device);
  accum_delete(acc->a);
  cudaStreamSynchronize(c->stream);
  delete acc;
  return RX_OK;
}

int rx_accum_reset(rx_accum* acc) {
  if (!acc) return RX_ERR_ARG;
  LOCK(acc->ctx);
  cudaSetDevice(acc->ctx->device);
  return accum_reset(acc->a);
}

int rx_render(rx_scene* scene, rx_accum* acc, const rx_render_params* params, int frames) {
  if (!scene || !acc || !params) return set_error(nullptr, "rx_render: NULL argument"), RX_ERR_ARG;
  if (scene->s.ctx != acc->ctx) return set_error(acc->ctx, "scene and accumulator belong to different contexts"), RX_ERR_ARG;
  LOCK(acc->ctx);
  cudaSetDevice(acc->ctx->device);
  return render(&scene->s, acc->a, params, frames);
}

int rx_accum_read(rx_accum* acc, int which, float* host_out) {
  if (!acc || !host_out) return RX_ERR_ARG;
  LOCK(acc->ctx);
  cudaSetDevice(acc->ctx->device);
  return accum_read(acc->a, which, host_out);
}

int rx_accum_info(rx_accum* acc, int* width, int* height, int* frames, long long* rays) {
  if (!acc) return RX_ERR_ARG;
  LOCK(acc->ctx);
  cudaSetDevice(acc->ctx->device);
  return accum_info(acc->a, width, height, frames, rays);
}

int rx_accum_denoise(rx_accum* acc, const rx_denoise_params* params, float* host_out) {
  if (!acc || !params) return RX_ERR_ARG;
  LOCK(acc->ctx);
  cudaSetDevice(acc->ctx->device);
  if (params->radius < 0 || params->passes < 1 || params->passes > 12)
    return set_error(acc->ctx, "denoise: radius must be >= 0 and passes in [1, 12]"), RX_ERR_ARG;
  return accum_denoise(acc->a, params, host_out);
}

int rx_accum_set_timing(rx_accum* acc, int on) {
  if (!acc) return RX_ERR_ARG;
  LOCK(acc->ctx);
  return accum_set_timing(acc->a, on);
}

int rx_accum_set_async(rx_accum* acc, int on) {
  if (!acc) return RX_ERR_ARG;
  LOCK(acc->ctx);
  return accum_set_async(acc->a, on);
}

int rx_accum_set_tail(rx_accum* acc, int max_paths) {
  if (!acc) return RX_ERR_ARG;
  LOCK(acc->ctx);
  return accum_set_tail(acc->a, max_paths);
}

int rx_accum_last_timing(rx_accum* acc, float* ms_total, float* ms_kernels, int n_kernels, int* launches) {
  if (!acc) return RX_ERR_ARG;
  LOCK(acc->ctx);
  return accum_last_timing(acc->a, ms_total, ms_kernels, n_kernels, launches);
}

int rx_batch_create(rx_ctx* ctx, rx_batch** out) {
  if (!ctx || !out) return set_error(nullptr, "rx_batch_create: NULL argument"), RX_ERR_ARG;
  LOCK(&ctx->c);
  rx_batch* r = new rx_batch();
  r->b = batch_new(&ctx->c);
  r->ctx = &ctx->c;
  *out = r;
  return RX_OK;
}

int rx_batch_destroy(rx_batch* b) {
  if (!b) return RX_OK;
  Ctx* c = b->ctx;
  LOCK(c);
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  batch_delete(b->b);
  delete b;
  return RX_OK;
}

int rx_batch_clear(rx_batch* b) {
  if (!b) return RX_ERR_ARG;
  LOCK(b->ctx);
  return batch_clear(b->b);
}

int rx_batch_add(rx_batch* b, rx_scene* scene, rx_accum* acc, const rx_render_params* params, int frames,
                 int* job) {
  if (!b || !scene || !acc || !params) return set_error(b ? b->ctx : nullptr, "rx_batch_add: NULL argument"), RX_ERR_ARG;
  LOCK(b->ctx);
  int idx = -1;
  int rc = batch_add(b->b, &scene->s, acc->a, params, frames, &idx);
  if (job) *job = idx;
  return rc;
}

int rx_batch_set_config(rx_batch* b, long long wave_paths, int extend_block) {
  if (!b) return RX_ERR_ARG;
  LOCK(b->ctx);
  return batch_set_config(b->b, wave_paths, extend_block);
}

int rx_batch_set_tail(rx_batch* b, int max_paths) {
  if (!b) return RX_ERR_ARG;
  LOCK(b->ctx);
  return batch_set_tail(b->b, max_paths);
}

int rx_batch_render(rx_batch* b) {
  if (!b) return RX_ERR_ARG;
  LOCK(b->ctx);
  cudaSetDevice(b->ctx->device);
  return batch_render(b->b);
}

int rx_batch_last_stats(rx_batch* b, float* ms, int* waves, int* launches) {
  if (!b) return RX_ERR_ARG;
  LOCK(b->ctx);
  return batch_last_stats(b->b, ms, waves, launches);
}

int rx_serve_create(rx_ctx* ctx, const rx_serve_config* cfg, rx_server** out) {
  if (!ctx || !cfg || !out) return set_error(nullptr, "rx_serve_create: NULL argument"), RX_ERR_ARG;
  if (cfg->hbm_budget <= 0 || cfg->max_active < 1 || cfg->step_paths < 1 || cfg->wave_paths < 1 ||
      cfg->wave_paths >= (1LL << 31) || cfg->preview_frames < 1 || cfg->pool_prewarm < 0 ||
      (cfg->extend_block != 64 && cfg->extend_block != 128 && cfg->extend_block != 256))
    return set_error(&ctx->c, "rx_serve_create: bad configuration"), RX_ERR_ARG;
  rx_server* s = new rx_server();
  s->s = serve_new(&ctx->c, cfg);
  s->ctx = &ctx->c;
  *out = s;
  return RX_OK;
}

int rx_serve_destroy(rx_server* s) {
  if (!s) return RX_OK;
  serve_delete(s->s);
  delete s;
  return RX_OK;
}

int rx_serve_submit(rx_server* s, rx_scene* scene, const rx_render_params* params, int frames, int* request) {
  if (!s || !scene || !params || !request) return set_error(s ? s->ctx : nullptr, "rx_serve_submit: NULL argument"),
                                                    RX_ERR_ARG;
  return serve_submit(s->s, &scene->s, params, frames, request);
}

int rx_serve_info(rx_server* s, int request, rx_request_info* out) {
  if (!s || !out) return RX_ERR_ARG;
  return serve_info(s->s, request, out);
}

int rx_serve_wait(rx_server* s, int request, int until_final, double timeout_s) {
  if (!s) return RX_ERR_ARG;
  return serve_wait(s->s, request, until_final, timeout_s);
}

int rx_serve_read(rx_server* s, int request, int which, float* host_out) {
  if (!s || !host_out) return RX_ERR_ARG;
  return serve_read(s->s, request, which, host_out);
}

int rx_serve_release(rx_server* s, int request) {
  if (!s) return RX_ERR_ARG;
  return serve_release(s->s, request);
}

int rx_serve_get_stats(rx_server* s, rx_serve_stats* out) {
  if (!s || !out) return RX_ERR_ARG;
  return serve_stats(s->s, out);
}

static cudaStream_t pick_stream(rx_ctx* ctx, void* stream) {
  return stream ? (cudaStream_t)stream : ctx->c.stream;
}

int rx_conv_bf16_fwd(rx_ctx* ctx, const rx_conv_desc* d, const void* x, const void* w, const float* bias, void* y,
                     float* y32, int relu, void* stream) {
  if (!ctx) return RX_ERR_ARG;
  cudaSetDevice(ctx->c.device);
  return conv_fwd(&ctx->c, d, x, w, bias, y, y32, relu, pick_stream(ctx, stream));
}

int rx_conv_bf16_bwd_data(rx_ctx* ctx, const rx_conv_desc* d, const void* dy, const void* w, void* w_rot, void* dx,
                          void* stream) {
  if (!ctx) return RX_ERR_ARG;
  cudaSetDevice(ctx->c.device);
  return conv_bwd_data(&ctx->c, d, dy, w, w_rot, dx, pick_stream(ctx, stream));
}

int rx_conv_bf16_bwd_weight(rx_ctx* ctx, const rx_conv_desc* d, const void* dy, const void* x, float* dw,
                            float* dbias, void* stream) {
  if (!ctx) return RX_ERR_ARG;
  cudaSetDevice(ctx->c.device);
  return conv_bwd_weight(&ctx->c, d, dy, x, dw, dbias, pick_stream(ctx, stream));
}

int rx_dn_layer(rx_ctx* ctx, const rx_dn_op* op, void* stream) {
  if (!ctx) return RX_ERR_ARG;
  cudaSetDevice(ctx->c.device);
  return dn_op(&ctx->c, op, pick_stream(ctx, stream));
}

int rx_dn_features(rx_ctx* ctx, long long P, const float* radiance, const float* albedo, const float* normal,
                   const float* depth, void* out, float* base, void* stream) {
  if (!ctx) return RX_ERR_ARG;
  cudaSetDevice(ctx->c.device);
  return dn_features(&ctx->c, P, radiance, albedo, normal, depth, out, base, pick_stream(ctx, stream));
}

int rx_dn_l1_loss(rx_ctx* ctx, long long P, const float* y32, int y_stride, const float* base, const float* target,
                  float scale, void* grad, int grad_stride, float* loss, void* stream) {
  if (!ctx) return RX_ERR_ARG;
  cudaSetDevice(ctx->c.device);
  return dn_l1_loss(&ctx->c, P, y32, y_stride, base, target, scale, grad, grad_stride, loss,
                    pick_stream(ctx, stream));
}

int rx_dn_output(rx_ctx* ctx, long long P, const float* y32, int y_stride, const float* base, float* out,
                 void* stream) {
  if (!ctx) return RX_ERR_ARG;
  cudaSetDevice(ctx->c.device);
  return dn_output(&ctx->c, P, y32, y_stride, base, out, pick_stream(ctx, stream));
}

int rx_dn_adam(rx_ctx* ctx, long long n, float* p, float* g, float* m, float* v, void* p16, float lr, float b1,
               float b2, float eps, int step, void* stream) {
  if (!ctx) return RX_ERR_ARG;
  cudaSetDevice(ctx->c.device);
  return dn_adam(&ctx->c, n, p, g, m, v, p16, lr, b1, b2, eps, step, pick_stream(ctx, stream));
}

int rx_obj_begin(rx_ctx* ctx, const void* text, long long n, rx_obj** out, int* lines, int* listed) {
  if (!ctx || !out || n < 0 || (n > 0 && !text)) return set_error(ctx ? &ctx->c : nullptr, "rx_obj_begin: bad arguments"), RX_ERR_ARG;
  if (n >= (1LL << 40)) return set_error(&ctx->c, "rx_obj_begin: %lld bytes exceed the limit", n), RX_ERR_CAPACITY;
  LOCK(&ctx->c);
  cudaSetDevice(ctx->c.device);
  *out = nullptr;
  ObjParse* o = nullptr;
  int rc = obj_begin(&ctx->c, text, n, &o);
  if (rc) return rc;
  rx_obj* h = new rx_obj();
  h->o = o;
  h->ctx = &ctx->c;
  int l = 0, s = 0;
  obj_info(o, &l, &s);
  if (lines) *lines = l;
  if (listed) *listed = s;
  *out = h;
  return RX_OK;
}

int rx_obj_listed(rx_obj* o, long long* offset, int* length, int* kind, int* flags, int* line) {
  if (!o || !offset || !length || !kind || !flags) return RX_ERR_ARG;
  LOCK(o->ctx);
  cudaSetDevice(o->ctx->device);
  return obj_listed(o->o, offset, length, kind, flags, line);
}

int rx_obj_correct(rx_obj* o, int n, const int* listed_pos, const int* kind, const int* ntri) {
  if (!o || n < 0 || (n > 0 && (!listed_pos || !kind || !ntri))) return RX_ERR_ARG;
  LOCK(o->ctx);
  cudaSetDevice(o->ctx->device);
  return obj_correct(o->o, n, listed_pos, kind, ntri);
}

int rx_obj_scan(rx_obj* o, int* totals, int* listed_prefix) {
  if (!o || !totals) return RX_ERR_ARG;
  LOCK(o->ctx);
  cudaSetDevice(o->ctx->device);
  return obj_scan(o->o, totals, listed_prefix);
}

int rx_obj_emit(rx_obj* o, const int* usemtl_gid, double* positions, double* normals, double* uvs, int* tri_pos_idx,
                int* tri_normal_idx, int* tri_uv_idx, int* tri_group_idx) {
  if (!o) return RX_ERR_ARG;
  LOCK(o->ctx);
  cudaSetDevice(o->ctx->device);
  return obj_emit(o->o, usemtl_gid, positions, normals, uvs, tri_pos_idx, tri_normal_idx, tri_uv_idx, tri_group_idx);
}

int rx_obj_device_ms(rx_obj* o, float* ms) {
  if (!o || !ms) return RX_ERR_ARG;
  LOCK(o->ctx);
  cudaSetDevice(o->ctx->device);
  return obj_device_ms(o->o, ms);
}

int rx_obj_end(rx_obj* o) {
  if (!o) return RX_OK;
  {
    LOCK(o->ctx);
    cudaSetDevice(o->ctx->device);
    obj_end(o->o);
  }
  delete o;
  return RX_OK;
}

int rx_scene_device_bytes(rx_scene* scene, long long* bytes) {
  if (!scene || !bytes) return RX_ERR_ARG;
  LOCK(scene->s.ctx);
  *bytes = (long long)scene_bytes(&scene->s);
  return RX_OK;
}

int rx_accum_set_f64(rx_accum* acc, int on) {
  if (!acc) return RX_ERR_ARG;
  LOCK(acc->ctx);
  cudaSetDevice(acc->ctx->device);
  return accum_set_f64(acc->a, on);
}

int rx_accum_read_f64(rx_accum* acc, double* host_out) {
  if (!acc || !host_out) return RX_ERR_ARG;
  LOCK(acc->ctx);
  cudaSetDevice(acc->ctx->device);
  return accum_read_f64(acc->a, host_out);
}

int rx_denoise(rx_ctx* ctx, int height, int width, const float* color, const float* normal, const float* albedo,
               const float* depth, const rx_denoise_params* params, float* out) {
  if (!ctx || !params) return set_error(nullptr, "rx_denoise: NULL argument"), RX_ERR_ARG;
  LOCK(&ctx->c);
  cudaSetDevice(ctx->c.device);
  if (height < 0 || width < 0 || (height * (long long)width > 0 && (!color || !out)))
    return set_error(&ctx->c, "rx_denoise: bad arguments"), RX_ERR_ARG;
  if (params->passes < 1 || params->passes > 12)
    return set_error(&ctx->c, "rx_denoise: passes must be in [1, 12]"), RX_ERR_ARG;
  return denoise_host(&ctx->c, height, width, color, normal, albedo, depth, params, out);
}

}  // extern "C"
