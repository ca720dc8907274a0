/*
 * roxy.h — C ABI of libroxy_cuda.so, the B200 (sm_100a) path-tracing hot path.
 *
 * Plain C: opaque handles, host pointers and sizes, int status codes.  Every
 * call returns RX_OK (0) or an RX_ERR_* code; rx_last_error() gives the text.
 * Host arrays passed in are copied before the call returns; the library never
 * keeps a host pointer.  Calls on one context are serialised by its mutex.
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to the roxy-dcc project root).
 */
#ifndef ROXY_H
#define ROXY_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  RX_OK = 0,
  RX_ERR_ARG = 1,       /* invalid argument (the reference raises ValueError) */
  RX_ERR_CAPACITY = 2,  /* size beyond a limit (the reference asserts)        */
  RX_ERR_CUDA = 3,      /* CUDA runtime error                                 */
  RX_ERR_STATE = 4,     /* call out of order (e.g. render before a BVH)       */
  RX_ERR_DEVICE = 5,    /* a kernel reported an internal error flag           */
  RX_ERR_TIMEOUT = 6    /* a wait ran out (serving)                           */
};

enum { RX_BVH_REFERENCE = 0, RX_BVH_LBVH_SAH = 1 };

enum {
  RX_ACC_RADIANCE = 0, /* running-mean linear radiance (H,W,3)  */
  RX_ACC_NORMAL = 1,   /* first-hit normal running mean (H,W,3) */
  RX_ACC_ALBEDO = 2,   /* first-hit albedo running mean (H,W,3) */
  RX_ACC_DEPTH = 3,    /* first-hit depth running mean (H,W)    */
  RX_ACC_DISPLAY = 4   /* sqrt(min(radiance, 1)) (H,W,3)        */
};

typedef struct rx_ctx rx_ctx;
typedef struct rx_scene rx_scene;
typedef struct rx_accum rx_accum;
typedef struct rx_batch rx_batch;

/* Arguments of one render call: the reference's render_kernel parameters
 * (rendering/taichi/trace.py:239-254) plus the sampling options. */
typedef struct {
  int width, height;
  float fov_tan, aspect;
  float cam_pos[3], cam_fwd[3], cam_right[3], cam_up[3];
  int max_depth;               /* bounce loop length (trace.py:149)            */
  int use_sky;                 /* sky gradient, else bg (trace.py:154-159)     */
  float bg[3];
  int direct_light_mode;       /* 0 one light, 1 all lights (trace.py:60-93)   */
  int direct_light_max_depth;  /* NEE at depth < this (trace.py:199,210)       */
  float sample_clamp;          /* clamp each sample to [0, c] if c > 0          */
  int reference_compat;        /* 1: sphere-light NEE only, emission counted
                                  again on BSDF hits, as trace.py does          */
  uint32_t seed;               /* counter-based RNG key                         */
  int wave_paths;              /* paths per wavefront (0 = automatic)           */
  int mis;                     /* default estimator only: weigh NEE and BSDF
                                  hits of listed lights by the power heuristic
                                  (needs rx_scene_set_light_sources)            */
} rx_render_params;

/* Edge-aware filter (rendering/denoise.py:23-104) and its a-trous extension:
 * pass i filters the previous pass with taps spaced 2^i apart; passes = 1 is
 * exactly edge_aware_denoise. */
typedef struct {
  int radius;
  int passes;
  float sigma_color, sigma_normal, sigma_albedo, sigma_depth;
  float amount;
  int use_normal, use_albedo, use_depth; /* guides used by rx_accum_denoise */
  int to_display;                        /* apply linear_to_display (denoise.py:107) */
} rx_denoise_params;

int rx_version(void);
int rx_device_count(int* out);

/* Context: device, stream, error text.  Replaces ti.init
 * (rendering/taichi/__init__.py:4-5). */
int rx_ctx_create(int device, rx_ctx** out);
int rx_ctx_destroy(rx_ctx* ctx);
const char* rx_last_error(const rx_ctx* ctx);
int rx_ctx_sync(rx_ctx* ctx);       /* waits for the device; reports kernel error flags */
void* rx_ctx_stream(rx_ctx* ctx); /* the cudaStream_t the library launches on */
/* Holds the context's lock across several calls made by this thread (no
 * reference counterpart: the reference is single-threaded).  Until
 * rx_ctx_release, calls from other threads on this context -- a serving
 * loop's render steps among them -- wait, while the holder's own calls
 * proceed; a scene built under the hold is built without interleaving with
 * other threads' work.  Holds nest; every hold needs its release, from the
 * same thread. */
int rx_ctx_hold(rx_ctx* ctx);
int rx_ctx_release(rx_ctx* ctx);

/* Scene state.  Replaces the module-global fields written by extract_scene
 * and GPUBVHBuilder.upload (rendering/taichi/fields.py:22-79,
 * rendering/taichi/extractor.py:19-50, rendering/taichi/bvh_builder.py:560-655). */
int rx_scene_create(rx_ctx* ctx, rx_scene** out);
int rx_scene_destroy(rx_scene* scene);
/* Triangles in caller order, float32 xyz triples, palette index per triangle
 * (TriangleBatch, bvh_builder.py:8-272). */
int rx_scene_set_triangles(rx_scene* scene, int n, const float* v0, const float* v1, const float* v2,
                           const float* n0, const float* n1, const float* n2, const int* mat_idx);
/* Scene extraction on the device: the triangle arrays are sized once, then
 * filled piecewise.  Replaces the host flattening of
 * rendering/taichi/extractor.py:60-96 (Mesh triangles and
 * IndexedMesh.indexed_triangle_arrays, scene/mesh.py:397-430) followed by the
 * field upload of bvh_builder.py:560-655.
 *   rx_scene_alloc_triangles  n rows, zero-filled; drops any BVH.
 *   rx_scene_put_triangles    rows [offset, offset+n) from host float32 rows
 *                             (n0..n2 NULL -> copies of v0; mat_idx NULL -> 0).
 *   rx_scene_put_indexed      rows [offset, offset+n_tris) from an indexed mesh:
 *                             positions (n_pos,3) float64, tri_pos_idx (n_tris,3),
 *                             normals (n_nrm,3) float64 + tri_nrm_idx (n_tris,3)
 *                             or NULL (a row with an index < 0 takes the face
 *                             normal), matrix: 16 float64 row-major world matrix
 *                             or NULL, normal_matrix: 16 float64 row-major
 *                             inverse transpose or NULL, tri_group_idx (n_tris,)
 *                             or NULL, group_mat (n_groups,) palette index of each
 *                             group.  Out-of-range indices -> RX_ERR_ARG.
 *   rx_scene_get_triangles    copies rows back (any output may be NULL). */
int rx_scene_alloc_triangles(rx_scene* scene, int n);
int rx_scene_put_triangles(rx_scene* scene, int offset, int n, const float* v0, const float* v1, const float* v2,
                           const float* n0, const float* n1, const float* n2, const int* mat_idx);
int rx_scene_put_indexed(rx_scene* scene, int offset, int n_tris, int n_pos, const double* positions,
                         const int* tri_pos_idx, int n_nrm, const double* normals, const int* tri_nrm_idx,
                         const double* matrix, const double* normal_matrix, const int* tri_group_idx,
                         int n_groups, const int* group_mat);
int rx_scene_get_triangles(rx_scene* scene, int offset, int n, float* v0, float* v1, float* v2, float* n0,
                           float* n1, float* n2, int* mat_idx);
/* Albedo textures (rendering/taichi/extractor.py:53-81 _upload_textures,
 * sampled as trace.py:96-136 _sample_texture / _bvh_albedo).
 *   rx_scene_put_uvs   per source triangle uv0..uv2 (n,2) float32 and has_uv
 *                      (n,) (NULL -> all 1) for rows [offset, offset+n); rows
 *                      never written have no uvs.  Triangle uploads drop them.
 *   rx_scene_set_textures  n RGB u8 images, width[i] x height[i], row-major,
 *                      concatenated in `texels`; flip_v[i] != 0 flips v.
 *   rx_scene_set_material_textures  texture index (-1 none) per entry of the
 *                      palette given to rx_scene_set_materials (call it after
 *                      that function, which resets them to -1).
 * A BVH triangle whose material has a texture and whose row has uvs shades
 * with albedo x bilinear texel / 255; a texture index >= n samples white. */
int rx_scene_put_uvs(rx_scene* scene, int offset, int n, const float* uv0, const float* uv1, const float* uv2,
                     const int* has_uv);
int rx_scene_set_textures(rx_scene* scene, int n, const int* width, const int* height, const int* flip_v,
                          const unsigned char* texels);
int rx_scene_set_material_textures(rx_scene* scene, int n, const int* texture_idx);
/* Material palette (fields.py:73-78). */
int rx_scene_set_materials(rx_scene* scene, int n, const int* type, const float* albedo,
                           const float* roughness, const float* ior, const float* emission);
/* Primitive slots (extractor.py:19-33 _write_slot): type 0 sphere, 1 plane,
 * 2 cube, 4 triangle, each with its own material. */
int rx_scene_set_objects(rx_scene* scene, int n, const int* type, const float* center, const float* radius,
                         const float* normal, const float* offset, const float* extra, const float* v0,
                         const float* v1, const float* v2, const int* mat_type, const float* albedo,
                         const float* roughness, const float* ior, const float* emission);
/* Explicit lights (extractor.py:36-50 plus emissive triangles): kind 0 sphere
 * (p0 centre, p1[0] radius), kind 1 triangle (p0, p1, p2); alias table over
 * pick_pdf for the one-light mode. */
int rx_scene_set_lights(rx_scene* scene, int n, const int* kind, const float* p0, const float* p1,
                        const float* p2, const float* albedo, const float* emission, const float* area,
                        const float* pick_pdf, const float* alias_prob, const int* alias_idx);
/* What each light of the last rx_scene_set_lights is: the caller's triangle
 * index (triangle lights) or the object slot (sphere lights).  Needed only
 * for multiple importance sampling (rx_render_params.mis): a BSDF ray that
 * hits a light then weighs its emission against the light-sampling pdf
 * (power heuristic, rendering/sampling.py:36-45 mis_power_weight). */
int rx_scene_set_light_sources(rx_scene* scene, int n, const int* source);

/* BVH build on the device.  RX_BVH_REFERENCE reproduces GPUBVHBuilder.build's
 * Morton method (bvh_builder.py:315-478) node for node; RX_BVH_LBVH_SAH builds
 * a Karras LBVH with SAH leaf collapse (core/bvh.py's role for the GPU path),
 * optionally with the sphere slots as BVH primitives. */
int rx_bvh_build(rx_scene* scene, int method, int max_leaf, int spheres_in_bvh);
/* Upload a tree already in the reference's node format (GPUBVHBuilder.upload,
 * bvh_builder.py:560-655); triangles must be set first, `order` maps leaf
 * order to caller order. */
int rx_bvh_set_reference(rx_scene* scene, int n_nodes, const float* node_min, const float* node_max,
                         const int* left, const int* right, const int* tri_start, const int* tri_count,
                         const int* order);
/* Node count, primitive count, method, leaf size, depth (levels). */
int rx_bvh_info(rx_scene* scene, int* n_nodes, int* n_prims, int* method, int* leaf_size, int* depth);
/* Reference-format export (GPUBVHBuilder.nodes / ordered_tris) of a tree built
 * with RX_BVH_REFERENCE or uploaded; arrays sized n_nodes (order: n_tris). */
int rx_bvh_export_reference(rx_scene* scene, float* node_min, float* node_max, int* left, int* right,
                            int* tri_start, int* tri_count, int* order);

/* Traversal-layout export for structural checks: n_nodes x 16 floats (the
 * 64-byte node records) and the leaf-order -> caller-order primitive map
 * (triangles < n_tris, spheres after them). */
int rx_bvh_export_layout(rx_scene* scene, float* nodes, int* order);

/* Closest hit over the BVH for n rays (bvh_intersect, intersect.py:81-152):
 * t (1e9 on miss), id = caller triangle index (-1 miss; spheres in the BVH
 * report -(slot + 2)), barycentrics u, v.  Host pointers. */
int rx_trace_closest(rx_scene* scene, long n, const float* ro, const float* rd, float* t, int* id, float* u,
                     float* v);
/* Any hit before tmax (bvh_occluded / scene_occluded, intersect.py:155-246). */
int rx_trace_any(rx_scene* scene, long n, const float* ro, const float* rd, const float* tmax, int* occluded);
/* Full scene query (scene_intersect, intersect.py:249-309): kind 0 miss,
 * 1 BVH triangle, 2 sphere in the BVH, 3 object slot; id = triangle index or
 * slot; normal is the un-flipped surface normal. */
int rx_scene_intersect(rx_scene* scene, long n, const float* ro, const float* rd, float* t, int* kind, int* id,
                       float* u, float* v, float* normal);
/* Device-pointer variants for callers that keep rays resident in HBM. */
int rx_trace_closest_device(rx_scene* scene, long n, const float* d_ro, const float* d_rd, float* d_t, int* d_id,
                            float* d_u, float* d_v);

/* Progressive accumulation buffers and the wavefront render.  Replaces
 * render_kernel and the TaichiRenderer frame loop (trace.py:239-283,
 * rendering/taichi_renderer.py:87-161). */
int rx_accum_create(rx_ctx* ctx, int width, int height, rx_accum** out);
int rx_accum_destroy(rx_accum* acc);
int rx_accum_reset(rx_accum* acc);
int rx_render(rx_scene* scene, rx_accum* acc, const rx_render_params* params, int frames);
int rx_accum_read(rx_accum* acc, int which, float* host_out);
/* frames accumulated and rays cast so far (rays counted as trace.py:150-151
 * and :78-79 count them: one per bounce including the primary, one per
 * shadow ray) */
int rx_accum_info(rx_accum* acc, int* width, int* height, int* frames, long long* rays);
/* Denoise the resident accumulators (taichi_renderer.py:67-79) into host_out (H,W,3). */
int rx_accum_denoise(rx_accum* acc, const rx_denoise_params* params, float* host_out);
/* Per-kernel CUDA-event timing of the next render calls (for profiling). */
int rx_accum_set_timing(rx_accum* acc, int on);
/* Asynchronous frames: with on != 0, rx_accum_reset and rx_render return once
 * their work is queued on the context's stream instead of waiting for it,
 * so back-to-back frames leave the GPU no idle gap.  Error bits the kernels
 * raise (an overflow, a bounded wait that ran out) then surface at the next
 * rx_ctx_sync; every call that copies to the host still waits.  Off by
 * default (each render returns with its frames done and checked, as the
 * reference's ti.sync() after render_kernel does, trace.py:282). */
int rx_accum_set_async(rx_accum* acc, int on);
/* Tail of a wave (no reference counterpart; the reference's megakernel
 * traces each path to the end in one thread, trace.py:139-236): from the
 * first bounce >= 1 whose queue holds at most max_paths paths, one launch
 * runs every remaining bounce of those paths, a thread per path, instead of
 * one extend and one shade launch per bounce.  Images and ray counts are
 * the same bit for bit either way.  0 turns it off; the default is 65536. */
int rx_accum_set_tail(rx_accum* acc, int max_paths);
/* ms of the last render, ms per kernel class (extend, shade, connect, other,
 * accumulate; n_kernels <= 5 of them) and the number of kernel launches it
 * made. */
int rx_accum_last_timing(rx_accum* acc, float* ms_total, float* ms_kernels, int n_kernels, int* launches);
/* Float64 sums of the clamped sample radiance next to the float32 running
 * means, for high-spp reference renders (no reference counterpart: the
 * reference accumulates in float32 only, trace.py:262-283).  Enable on a
 * reset accumulator; rx_accum_read_f64 writes the float64 mean (H,W,3). */
int rx_accum_set_f64(rx_accum* acc, int on);
int rx_accum_read_f64(rx_accum* acc, double* host_out);

/* Batched rendering: many (scene, accumulator, params, frames) jobs traced
 * as shared wavefronts, all waves of one call in one CUDA graph.  The
 * reference renders one scene per TaichiRenderer.render call
 * (taichi_renderer.py:87-191); a job's result here equals rendering it
 * alone with rx_render (same random numbers, same accumulation order).
 * Scenes and accumulators must outlive the batch's use of them; each job
 * needs its own accumulator.  rx_batch_add writes the job index to *job
 * (may be NULL).  rx_batch_set_config: paths per wave (>= 1) and the extend
 * kernel's block size (64, 128 or 256), normally chosen by the autotuner
 * (rendering/batch.py).  rx_batch_last_stats: device ms of the last render
 * call, its waves and kernel launches. */
int rx_batch_create(rx_ctx* ctx, rx_batch** out);
int rx_batch_destroy(rx_batch* batch);
int rx_batch_clear(rx_batch* batch);
int rx_batch_add(rx_batch* batch, rx_scene* scene, rx_accum* acc, const rx_render_params* params, int frames,
                 int* job);
int rx_batch_set_config(rx_batch* batch, long long wave_paths, int extend_block);
/* The batch counterpart of rx_accum_set_tail: from the first bounce >= 1
 * whose wave queue holds at most max_paths paths, of every scene of the
 * wave, one launch runs the remaining bounces a thread per path.  0 turns it
 * off; the default is 65536. */
int rx_batch_set_tail(rx_batch* batch, int max_paths);
int rx_batch_render(rx_batch* batch);
int rx_batch_last_stats(rx_batch* batch, float* ms, int* waves, int* launches);

/* Serving (no reference counterpart: the reference renders one
 * TaichiRenderer.render call at a time, taichi_renderer.py:87-191).  A host
 * thread owned by the server admits submitted requests while active slots
 * and the device-memory budget allow, gives each new request its preview
 * frames in the next step, then refines admitted requests within a
 * per-step path budget; every step is one batch of shared wavefronts.
 * Scenes stay owned by the caller and must outlive their requests; the
 * server creates and frees each request's accumulator (freed at
 * rx_serve_release).  Times are seconds since rx_serve_create. */
typedef struct rx_server rx_server;
typedef struct {
  long long hbm_budget;  /* bytes: wave state + accumulators + scenes in use */
  int max_active;        /* requests rendering at once                        */
  long long step_paths;  /* paths per serving step (bounds preview latency)   */
  long long wave_paths;  /* paths per wavefront within a step                 */
  int extend_block;      /* 64, 128 or 256                                    */
  int preview_frames;    /* frames of a request's first step                  */
  long long pool_prewarm; /* bytes mapped into the device allocation pool at
                             start, so admitting requests later maps none    */
} rx_serve_config;
enum { RX_REQ_QUEUED = 0, RX_REQ_ACTIVE = 1, RX_REQ_DONE = 2, RX_REQ_FAILED = 3 };
typedef struct {
  int state, frames_done, frames;
  double t_submit, t_admit, t_preview, t_final; /* -1 until reached */
  long long bytes;
} rx_request_info;
typedef struct {
  long long steps, admitted, completed, failed;
  int active, queued, max_active_seen;
  long long bytes_in_use, max_bytes_in_use;
  double busy_s, uptime_s;
} rx_serve_stats;
int rx_serve_create(rx_ctx* ctx, const rx_serve_config* config, rx_server** out);
int rx_serve_destroy(rx_server* server);
int rx_serve_submit(rx_server* server, rx_scene* scene, const rx_render_params* params, int frames, int* request);
int rx_serve_info(rx_server* server, int request, rx_request_info* out);
/* until_final 0: wait for the preview; RX_ERR_TIMEOUT after timeout_s */
int rx_serve_wait(rx_server* server, int request, int until_final, double timeout_s);
int rx_serve_read(rx_server* server, int request, int which, float* host_out);
int rx_serve_release(rx_server* server, int request);
int rx_serve_get_stats(rx_server* server, rx_serve_stats* out);
/* Device bytes a scene holds (what serving admission charges for it). */
int rx_scene_device_bytes(rx_scene* scene, long long* bytes);

/* Learned denoiser kernels (no reference counterpart; the reference's only
 * denoiser is edge_aware_denoise, denoise.py:23-104).  BF16 tensor-core 3x3
 * convolutions (stride 1, zero padding 1) with FP32 accumulation on NHWC
 * device tensors, and the element-wise layers of the network around them.
 * All pointers are device pointers; `stream` NULL means the context's
 * stream.  Activations are viewed through a channel stride and offset (a
 * concatenation is a wider tensor); channel counts are multiples of 16,
 * strides and offsets multiples of 8.  Weights: [Cout][3][3][Cin] bf16. */
typedef struct {
  int N, H, W;            /* images, height, width                    */
  int Cin, Cout;          /* input / output channels                  */
  int x_cstride, x_coff;  /* input view: channel stride and offset    */
  int y_cstride, y_coff;  /* output view                              */
} rx_conv_desc;
/* y = act(conv(x, w) + bias); relu != 0 applies max(., 0); y32 (optional)
 * receives the same values in float32 */
int rx_conv_bf16_fwd(rx_ctx* ctx, const rx_conv_desc* d, const void* x, const void* w, const float* bias, void* y,
                     float* y32, int relu, void* stream);
/* Forward convolution kernels.  impl = 0 (default): the warp-specialised
 * tcgen05 kernel (weights resident in shared memory, a ring of input rows,
 * accumulators in tensor memory) for every layer whose weights fit beside
 * four input rows in at most two output-channel groups, the mma.sync
 * kernel for the others.  impl = 1: mma.sync only.  impl = 2: the streaming
 * tcgen05 kernel (one 128-pixel row tile per CTA, weights staged per
 * 32-channel chunk) for 16, 32, 64 or 128 output channels, mma.sync for
 * other shapes.  A kernel whose internal wait runs out raises the device
 * error flag, reported by rx_ctx_sync. */
int rx_conv_set_impl(rx_ctx* ctx, int impl);
/* dx = gradient of the input for output gradient dy (in the y view);
 * w_rot: Cout*9*Cin bf16 of scratch the caller provides */
int rx_conv_bf16_bwd_data(rx_ctx* ctx, const rx_conv_desc* d, const void* dy, const void* w, void* w_rot, void* dx,
                          void* stream);
/* dw += gradient of the weights (float32 [Cout][3][3][Cin]); dbias (optional) += bias gradient */
int rx_conv_bf16_bwd_weight(rx_ctx* ctx, const rx_conv_desc* d, const void* dy, const void* x, float* dw,
                            float* dbias, void* stream);
enum { RX_DN_COPY = 0, RX_DN_RELU_MASK = 1, RX_DN_POOL = 2, RX_DN_POOL_BWD = 3, RX_DN_UP = 4, RX_DN_UP_BWD = 5 };
/* One element-wise layer from view a to view b (bf16, NHWC):
 *   COPY       b[..c] = a (flag: b += a), C channels, N x H x W pixels
 *   RELU_MASK  b = 0 where a <= 0 (a: a ReLU's output, b: its gradient)
 *   POOL       2x2 average, a is H x W, b is H/2 x W/2
 *   POOL_BWD   a is the H/2 x W/2 gradient, b (H x W) = a / 4 (flag: +=)
 *   UP         nearest 2x, a is H x W, b is 2H x 2W
 *   UP_BWD     a is the 2H x 2W gradient, b (H x W) = sum of 4 children */
typedef struct {
  int kind, N, H, W, C;
  const void* a;
  int a_stride, a_off;
  void* b;
  int b_stride, b_off;
  int flag;
} rx_dn_op;
int rx_dn_layer(rx_ctx* ctx, const rx_dn_op* op, void* stream);
/* 16-channel bf16 network input (log1p radiance, albedo, normal,
 * depth/(1+depth), zeros) from float32 planes of P pixels; base (optional,
 * float32 P x 3) receives log1p(radiance), the image the network corrects */
int rx_dn_features(rx_ctx* ctx, long long P, const float* radiance, const float* albedo, const float* normal,
                   const float* depth, void* out, float* base, void* stream);
/* L1 loss of y + base (first 3 channels of y32; base optional) against the
 * log1p target (P,3): *loss += sum |y + base - t|; grad (bf16, grad_stride
 * channels) = sign(y + base - t) * scale */
int rx_dn_l1_loss(rx_ctx* ctx, long long P, const float* y32, int y_stride, const float* base, const float* target,
                  float scale, void* grad, int grad_stride, float* loss, void* stream);
/* radiance (P,3) = max(expm1(y + base), 0) (base optional) */
int rx_dn_output(rx_ctx* ctx, long long P, const float* y32, int y_stride, const float* base, float* out,
                 void* stream);
/* Adam step `step` (1-based) on n float32 parameters; writes their bf16
 * copy p16 (optional) and clears g */
int rx_dn_adam(rx_ctx* ctx, long long n, float* p, float* g, float* m, float* v, void* p16, float lr, float b1,
               float b2, float eps, int step, void* stream);

/* edge_aware_denoise / a-trous on caller host buffers (denoise.py:23-104):
 * color (H,W,3); normal, albedo (H,W,3) and depth (H,W) may be NULL. */
int rx_denoise(rx_ctx* ctx, int height, int width, const float* color, const float* normal, const float* albedo,
               const float* depth, const rx_denoise_params* params, float* out);

/* ---- Wavefront OBJ text parsed on the device ----------------------------
 * Replaces the line loop of OBJReader._parse_indexed / load_as_indexed_mesh
 * (scene/io/obj_reader.py:345-441) with the same results: float64
 * positions (V,3), normals (N,3), uvs (T,2); int32 tri_pos_idx,
 * tri_normal_idx, tri_uv_idx (F,3) and tri_group_idx (F).  Sequence:
 *   rx_obj_begin   upload the text, split lines, classify them;
 *   rx_obj_listed  the lines the host must read itself: usemtl, mtllib, o,
 *                  g, unrecognised tokens, lines with non-ASCII bytes, and
 *                  lines whose numbers are outside the device's exact path
 *                  (RX_OBJ_HOST in flags);
 *   rx_obj_correct kind and triangle count of listed non-ASCII lines as
 *                  the host splits them (positions into the listed list);
 *   rx_obj_scan    totals {v, vn, vt, triangles, usemtl, faces, listed}
 *                  and, per listed line, the counts before it {v, vn, vt,
 *                  triangles, usemtl, faces};
 *   rx_obj_emit    the arrays (caller host buffers sized from the totals;
 *                  usemtl_gid = group id of each usemtl line in file order);
 *                  entries of RX_OBJ_HOST lines are left for the caller;
 *   rx_obj_end. */
typedef struct rx_obj rx_obj;
enum {
  RX_OBJ_SKIP = 0, RX_OBJ_V = 1, RX_OBJ_VN = 2, RX_OBJ_VT = 3, RX_OBJ_F = 4, RX_OBJ_USEMTL = 5,
  RX_OBJ_MTLLIB = 6, RX_OBJ_O = 7, RX_OBJ_G = 8, RX_OBJ_S = 9, RX_OBJ_OTHER = 10
};
enum { RX_OBJ_HOST = 1, RX_OBJ_NONASCII = 2 };
int rx_obj_begin(rx_ctx* ctx, const void* text, long long n, rx_obj** out, int* lines, int* listed);
int rx_obj_listed(rx_obj* o, long long* offset, int* length, int* kind, int* flags, int* line);
int rx_obj_correct(rx_obj* o, int n, const int* listed_pos, const int* kind, const int* ntri);
int rx_obj_scan(rx_obj* o, int* totals, int* listed_prefix);
int rx_obj_emit(rx_obj* o, const int* usemtl_gid, double* positions, double* normals, double* uvs, int* tri_pos_idx,
                int* tri_normal_idx, int* tri_uv_idx, int* tri_group_idx);
/* Device time (ms, CUDA events) of the parse so far: the kernels only, without
 * the text upload, the result copies and the host's reading of listed lines. */
int rx_obj_device_ms(rx_obj* o, float* ms);
int rx_obj_end(rx_obj* o);

/* Allocation-free a-trous denoise on caller device buffers.  No counterpart in
 * the reference: it exists for callers that cannot allocate device memory at
 * call time (a host that owns the whole device budget through its own
 * allocator, or a frame loop that must not pay the synchronisation an
 * allocation can imply).  It makes no cudaMalloc/cudaFree call: the two
 * intermediate pass buffers live in a fixed 32 MiB device array inside the
 * library, which limits height * width to 1,048,576 pixels (larger sizes
 * return RX_ERR_CAPACITY).  Buffers are float4 per pixel: colour (rgb, -),
 * normal guide (xyz, depth), albedo guide (rgb, -), output (rgb, 0); guides
 * are used as params->use_normal / use_albedo / use_depth say (a guide not in
 * use may be NULL).  d_out must not overlap the colour or a guide in use
 * (RX_ERR_ARG).  Runs on `stream` (a cudaStream_t, NULL = legacy default
 * stream) in the CUDA context current on the calling thread; the first call
 * in a context (per device, and again after cudaDeviceReset or in a caller's
 * own driver-API context) looks the array up and should come before any
 * stream capture.  Calls that can overlap on the GPU share the array and
 * race; the caller orders them.  Errors: rx_last_error(NULL). */
int rx_denoise_noalloc(int height, int width, const float* d_color, const float* d_guide_normal,
                       const float* d_guide_albedo, const rx_denoise_params* params, float* d_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ROXY_H */
