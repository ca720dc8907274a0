// Host-side runtime objects behind the C ABI: context (device, stream, error
// text), stream-ordered device buffers, scene and accumulation state.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "rx_internal.cuh"

namespace rx {

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 148;
  std::string err;
  std::recursive_mutex mu;
  std::atomic<int> hold_waiters{0};  // threads blocked in rx_ctx_hold (the serving loop lets them go first)
  int* d_err = nullptr;  // device error bits
  int conv_impl = 0;     // 0: warp-specialised tcgen05 where it fits, 1: mma.sync only, 2: tcgen05 streaming
  // pinned staging buffer of upload_staged / download_staged
  static constexpr int kPieceEvents = 32;
  void* stage = nullptr;
  size_t stage_bytes = 0;
  cudaEvent_t stage_done = nullptr;  // recorded after the last DMA that read `stage`
  cudaEvent_t piece_ev[kPieceEvents] = {};
};

void set_error(Ctx* ctx, const char* fmt, ...);

// One host array and its device destination (upload) or source (download).
struct HostPiece {
  void* dev;
  const void* host;
  size_t bytes;
};

// Copy `n` pageable host arrays to the device on the context's stream through
// the context's pinned buffer (threads fill it while the copy engine drains
// it).  The host arrays may be reused as soon as this returns; the device
// copies complete in stream order.
int upload_staged(Ctx* c, const HostPiece* arrays, int n);
// Copy `bytes` from the device to pageable host memory, in stream order, and
// wait for it: DMA into the pinned buffer piece by piece while threads copy
// the finished pieces out.
int download_staged(Ctx* c, void* host, const void* dev, size_t bytes);
bool host_stage_reserve(Ctx* c, size_t bytes);
void host_stage_free(Ctx* c);

#define CUDA_TRY(ctx, expr)                                                          \
  do {                                                                               \
    cudaError_t _e = (expr);                                                         \
    if (_e != cudaSuccess) {                                                         \
      ::rx::set_error((ctx), "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), \
                      __FILE__, __LINE__);                                           \
      return RX_ERR_CUDA;                                                            \
    }                                                                                \
  } while (0)

// Device buffer allocated and freed in stream order on the context's stream,
// so temporaries may be released right after the kernels that use them are
// enqueued.
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  Ctx* ctx = nullptr;
  bool failed = false;  // the last alloc() could not get its memory
  DevBuf() {}
  DevBuf(Ctx* c, size_t count) { alloc(c, count); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  bool alloc(Ctx* c, size_t count) {
    release();
    ctx = c;
    n = count;
    failed = false;
    if (count == 0) return true;
    if (cudaMallocAsync((void**)&p, sizeof(T) * count, c->stream) != cudaSuccess) {
      (void)cudaGetLastError();  // out of memory is not sticky: drop it here
      p = nullptr;
      n = 0;
      failed = true;
      return false;
    }
    return true;
  }
  bool ok() const { return !failed; }
  void release() {
    if (p && ctx) cudaFreeAsync(p, ctx->stream);
    p = nullptr;
    n = 0;
  }
  void swap(DevBuf& o) {
    std::swap(p, o.p);
    std::swap(n, o.n);
    std::swap(ctx, o.ctx);
    std::swap(failed, o.failed);
  }
  size_t bytes() const { return sizeof(T) * n; }
};

// True when every buffer got the memory its last alloc() asked for.
template <class... B>
inline bool all_ok(const B&... b) {
  return (b.ok() && ...);
}

struct HostMat {
  int type;
  float albedo[3];
  float roughness, ior, emission;
  int texture = -1;
};

struct Scene {
  Ctx* ctx = nullptr;
  // source triangles (caller order)
  int n_tris = 0;
  DevBuf<float> v0b, v1b, v2b, n0b, n1b, n2b;
  DevBuf<int> tri_matb;
  float *d_v0 = nullptr, *d_v1 = nullptr, *d_v2 = nullptr;
  float *d_n0 = nullptr, *d_n1 = nullptr, *d_n2 = nullptr;
  int* d_tri_mat = nullptr;
  // per source triangle uvs (2 float4), allocated by the first put_uvs
  DevBuf<float4> uvb;
  // albedo textures
  DevBuf<TexInfo> d_tex;
  DevBuf<unsigned char> d_texels;
  int n_tex = 0;
  // palette: caller materials followed by one entry per object slot
  std::vector<HostMat> user_mats;
  std::vector<HostMat> obj_mats;
  DevBuf<float4> mat_a, mat_b;
  int n_mats = 0;
  // object slots (reference _obj_* layout)
  std::vector<ObjSlot> objs;
  DevBuf<ObjSlot> d_objs;
  int n_lin = 0;
  std::vector<int> lin_slot;         // linear index -> object slot
  std::vector<int> bvh_sphere_slots;  // object slots of the BVH's spheres and cubes, in build order
  // lights
  DevBuf<Light> d_lights;
  DevBuf<float> d_alias_prob;
  DevBuf<int> d_alias_idx;
  int n_lights = 0;
  // traversal structure
  DevBuf<float4> d_nodes, d_prims, d_shade;
  int n_nodes = 0, n_prims = 0, n_bvh_spheres = 0;  // n_bvh_spheres: spheres and cubes in the BVH
  DevBuf<float4> d_nodes4;  // the LBVH 4-wide (8 float4 per node); traversal uses it when present
  int n_nodes4 = 0;
  float3 root_min = {0, 0, 0}, root_max = {0, 0, 0};
  int method = -1, exact_slab = 0, leaf_size = 0, depth = 0;
  // reference-format copy (reference builder / uploaded trees)
  DevBuf<int> ref_left, ref_right, ref_start, ref_count, order;
  DevBuf<float3> ref_min, ref_max;
  DevBuf<uint32_t> tmp_codes;
  uint64_t version = 0;  // bumped on every change; invalidates cached graphs

  void clear_bvh() {
    d_nodes.release();
    d_prims.release();
    d_shade.release();
    ref_left.release();
    ref_right.release();
    ref_start.release();
    ref_count.release();
    order.release();
    ref_min.release();
    ref_max.release();
    d_nodes4.release();
    n_nodes = n_prims = n_bvh_spheres = n_nodes4 = 0;
    depth = 0;
    method = -1;
    ++version;
  }
  int upload_palette(Ctx* c);
  int upload_linear_objects(Ctx* c, bool exclude_bvh_objects);
  DevScene view() const {
    DevScene s;
    s.nodes = d_nodes.p;
    s.n_nodes = n_nodes;
    s.nodes4 = n_nodes4 > 0 ? d_nodes4.p : nullptr;
    s.n_nodes4 = n_nodes4;
    s.root_min = root_min;
    s.root_max = root_max;
    s.prims = d_prims.p;
    s.shade = d_shade.p;
    s.n_prims = n_prims;
    s.mat_a = mat_a.p;
    s.mat_b = mat_b.p;
    s.n_mats = n_mats;
    s.objs = d_objs.p;
    s.n_objs = n_lin;
    s.lights = d_lights.p;
    s.alias_prob = d_alias_prob.p;
    s.alias_idx = d_alias_idx.p;
    s.n_lights = n_lights;
    s.exact_slab = exact_slab;
    s.uvs = uvb.p;
    s.tex = d_tex.p;
    s.texels = d_texels.p;
    s.n_tex = n_tex;
    const bool maps = !light_src.empty() && (int)light_src.size() == n_lights;
    s.light_of_tri = maps ? d_light_of_tri.p : nullptr;
    s.light_of_obj = maps ? d_light_of_obj.p : nullptr;
    s.light_of_lin = maps ? d_light_of_lin.p : nullptr;
    return s;
  }
  // per light: caller triangle index (triangle lights) or object slot
  // (sphere lights), as given to rx_scene_set_light_sources; the inverse
  // maps below are rebuilt whenever lights, triangles or linear objects change
  std::vector<int> light_src, light_kind;
  DevBuf<int> d_light_of_tri, d_light_of_obj, d_light_of_lin;
  int upload_light_maps(Ctx* c);
};

// BVH builders (rx_bvh.cu)
int build_reference(Ctx* ctx, Scene* sc, int leaf);
int build_lbvh(Ctx* ctx, Scene* sc, int max_leaf, int spheres_in_bvh, float c_t, float c_i);
int set_reference_nodes(Ctx* ctx, Scene* sc, int n_nodes, const float* node_min, const float* node_max,
                        const int* left, const int* right, const int* start, const int* count, const int* order);

// scene extraction on the device (rx_extract.cu); rows[] = v0, v1, v2, n0, n1, n2
int scene_alloc_triangles(Ctx* c, Scene* s, int n);
int scene_put_triangles(Ctx* c, Scene* s, int offset, int n, const float* const* rows, const int* mat_idx);
int scene_put_indexed(Ctx* c, Scene* s, int offset, int n_tris, int n_pos, const double* positions,
                      const int* tri_pos_idx, int n_nrm, const double* normals, const int* tri_nrm_idx,
                      const double* matrix, const double* normal_matrix, const int* tri_group_idx, int n_groups,
                      const int* group_mat);
int scene_get_triangles(Ctx* c, Scene* s, int offset, int n, float* const* rows, int* mat_idx);
int scene_put_uvs(Ctx* c, Scene* s, int offset, int n, const float* uv0, const float* uv1, const float* uv2,
                  const int* has_uv);
int scene_set_textures(Ctx* c, Scene* s, int n, const int* width, const int* height, const int* flip_v,
                       const unsigned char* texels);

// traversal entry points (rx_trace.cu)
int trace_closest(Ctx* ctx, Scene* sc, long n, const float* d_ro, const float* d_rd, float* d_t, int* d_id,
                  float* d_u, float* d_v);
int trace_any(Ctx* ctx, Scene* sc, long n, const float* d_ro, const float* d_rd, const float* d_tmax, int* d_occ);
int scene_query(Ctx* ctx, Scene* sc, long n, const float* d_ro, const float* d_rd, float* d_t, int* d_kind,
                int* d_id, float* d_u, float* d_v, float* d_n);

// Per-image accumulation and wavefront state (rx_render.cu)
struct Accum;
Accum* accum_new(Ctx* ctx, int w, int h);
void accum_delete(Accum* a);
int accum_reset(Accum* a);
int render(Scene* sc, Accum* a, const rx_render_params* p, int frames);
int accum_read(Accum* a, int which, float* host_out);
int accum_info(Accum* a, int* w, int* h, int* frames, long long* rays);
int accum_denoise(Accum* a, const rx_denoise_params* dp, float* host_out);
int accum_set_timing(Accum* a, int on);
int accum_set_async(Accum* a, int on);
int accum_set_tail(Accum* a, int max_paths);
int accum_last_timing(Accum* a, float* ms_total, float* ms_kernels, int n_kernels, int* launches);
int accum_set_f64(Accum* a, int on);
int accum_read_f64(Accum* a, double* host_out);

// Batches of jobs rendered as shared wavefronts (rx_render.cu)
struct Batch;
Batch* batch_new(Ctx* ctx);
void batch_delete(Batch* b);
int batch_clear(Batch* b);
int batch_add(Batch* b, Scene* sc, Accum* acc, const rx_render_params* p, int frames, int* job);
int batch_set_config(Batch* b, long long wave_paths, int ext_block);
int batch_set_tail(Batch* b, int max_paths);
int batch_render(Batch* b);
int batch_last_stats(Batch* b, float* ms, int* waves, int* launches);
void batch_use_graph(Batch* b, bool on);
int batch_reserve(Batch* b, long long cap);

// Serving loop (rx_serve.cu)
struct Server;
Server* serve_new(Ctx* ctx, const rx_serve_config* cfg);
void serve_delete(Server* s);
int serve_submit(Server* s, Scene* sc, const rx_render_params* p, int frames, int* id);
int serve_info(Server* s, int id, rx_request_info* out);
int serve_wait(Server* s, int id, int until_final, double timeout_s);
int serve_read(Server* s, int id, int which, float* host_out);
int serve_release(Server* s, int id);
int serve_stats(Server* s, rx_serve_stats* out);

// Learned denoiser kernels (rx_conv.cu)
int conv_fwd(Ctx* ctx, const rx_conv_desc* d, const void* x, const void* w, const float* bias, void* y, float* y32,
             int relu, cudaStream_t st);
int conv_bwd_data(Ctx* ctx, const rx_conv_desc* d, const void* dy, const void* w, void* w_rot, void* dx,
                  cudaStream_t st);
int conv_bwd_weight(Ctx* ctx, const rx_conv_desc* d, const void* dy, const void* x, float* dw, float* db,
                    cudaStream_t st);
int dn_op(Ctx* ctx, const rx_dn_op* o, cudaStream_t st);
int dn_features(Ctx* ctx, long long P, const float* rad, const float* alb, const float* nrm, const float* dep,
                void* out, float* base, cudaStream_t st);
int dn_l1_loss(Ctx* ctx, long long P, const float* y32, int y_stride, const float* base, const float* target,
               float scale, void* grad, int grad_stride, float* loss, cudaStream_t st);
int dn_output(Ctx* ctx, long long P, const float* y32, int y_stride, const float* base, float* out,
              cudaStream_t st);
int dn_adam(Ctx* ctx, long long n, float* p, float* g, float* m, float* v, void* p16, float lr, float b1, float b2,
            float eps, int step, cudaStream_t st);

// OBJ text parsing on the device (rx_obj.cu)
struct ObjParse;
int obj_begin(Ctx* ctx, const void* text, long long n, ObjParse** out);
int obj_info(ObjParse* o, int* lines, int* listed);
int obj_listed(ObjParse* o, long long* off, int* len, int* kind, int* flags, int* line);
int obj_correct(ObjParse* o, int n, const int* pos, const int* kind, const int* ntri);
int obj_scan(ObjParse* o, int* totals, int* listed_prefix);
int obj_emit(ObjParse* o, const int* usemtl_gid, double* pos, double* nrm, double* uv, int* tri_pos, int* tri_nrm,
             int* tri_uv, int* tri_grp);
void obj_end(ObjParse* o);
int obj_device_ms(ObjParse* o, float* ms);

// device bytes held by each object (serving admission)
size_t accum_bytes(const Accum* a);
size_t batch_bytes(const Batch* b);
size_t scene_bytes(const Scene* s);

// Denoise on caller buffers (rx_denoise.cu)
int denoise_host(Ctx* ctx, int h, int w, const float* color, const float* normal, const float* albedo,
                 const float* depth, const rx_denoise_params* dp, float* out);
int denoise_device(Ctx* ctx, int h, int w, const float4* d_color, const float4* d_guide_n, const float4* d_guide_a,
                   int has_normal, int has_albedo, int has_depth, const rx_denoise_params* dp, float4* d_out,
                   float4* d_scratch0, float4* d_scratch1, int to_display);

}  // namespace rx
