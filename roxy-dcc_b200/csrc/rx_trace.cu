// Ray-query entry points over a built scene: closest hit, any hit and the
// full scene query (linear object slots, then the BVH).  These are the
// parity hooks for the reference's bvh_intersect / bvh_occluded /
// scene_intersect (rendering/taichi/intersect.py:81-309) and a direct
// traversal benchmark.
#include "rx_internal.cuh"
#include "rx_runtime.h"

namespace rx {

__device__ __forceinline__ float3 ld3f(const float* p, long i) { return f3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }

template <bool EXACT>
__global__ void k_trace_closest(DevScene S, long n, const float* __restrict__ ro, const float* __restrict__ rd,
                                float* __restrict__ out_t, int* __restrict__ out_id, float* __restrict__ out_u,
                                float* __restrict__ out_v, int* err) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    float3 o = ld3f(ro, i), d = ld3f(rd, i);
    float t = 1e9f, u = 0.0f, v = 0.0f;
    int p = bvh_closest<EXACT>(S, o, d, t, u, v, err);
    int id = -1;
    if (p >= 0) {
      float4 a = __ldg(S.prims + 3 * (size_t)p);
      int src = __float_as_int(__ldg(S.shade + 3 * (size_t)p + 1).w);
      id = __float_as_int(a.w) == PRIM_TRI ? src : -(src + 2);
    }
    out_t[i] = t;
    out_id[i] = id;
    out_u[i] = p >= 0 ? u : 0.0f;
    out_v[i] = p >= 0 ? v : 0.0f;
  }
}

template <bool EXACT>
__global__ void k_trace_any(DevScene S, long n, const float* __restrict__ ro, const float* __restrict__ rd,
                            const float* __restrict__ tmax, int* __restrict__ out, int* err) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    out[i] = scene_any<EXACT>(S, ld3f(ro, i), ld3f(rd, i), tmax[i], err) ? 1 : 0;
  }
}

// Surface normal of a hit, un-flipped (intersect.py:265-304).
__device__ __forceinline__ float3 hit_normal(const DevScene& S, float3 o, float3 d, const SceneHit& h) {
  if (h.prim >= 0) {
    const float4* sp = S.shade + 3 * (size_t)h.prim;
    float4 a = __ldg(S.prims + 3 * (size_t)h.prim);
    if (__float_as_int(a.w) == PRIM_TRI) {
      float w = 1.0f - h.u - h.v;
      float3 n0 = xyz(__ldg(sp)), n1 = xyz(__ldg(sp + 1)), n2 = xyz(__ldg(sp + 2));
      return normalized((n0 * w + n1 * h.u) + n2 * h.v);
    }
    return analytic_normal(o + d * h.t, a, __ldg(S.prims + 3 * (size_t)h.prim + 1));
  }
  if (h.slot >= 0) {
    const ObjSlot& ob = S.objs[h.slot];
    if (ob.type == 0) return normalized((o + d * h.t) - ob.center);
    if (ob.type == 1) return ob.normal;
    if (ob.type == 2) return cube_normal(o + d * h.t, ob.center, ob.extra);
    return normalized(cross(ob.v1 - ob.v0, ob.v2 - ob.v0));
  }
  return f3(0.0f, 1.0f, 0.0f);
}

template <bool EXACT>
__global__ void k_scene_query(DevScene S, long n, const float* __restrict__ ro, const float* __restrict__ rd,
                              const int* __restrict__ lin_slot, float* __restrict__ out_t, int* __restrict__ out_kind,
                              int* __restrict__ out_id, float* __restrict__ out_u, float* __restrict__ out_v,
                              float* __restrict__ out_n, int* err) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    float3 o = ld3f(ro, i), d = ld3f(rd, i);
    SceneHit h = scene_closest<EXACT>(S, o, d, err);
    int kind = 0, id = -1;
    if (h.prim >= 0) {
      float4 a = __ldg(S.prims + 3 * (size_t)h.prim);
      id = __float_as_int(__ldg(S.shade + 3 * (size_t)h.prim + 1).w);
      kind = __float_as_int(a.w) == PRIM_TRI ? 1 : 2;
    } else if (h.slot >= 0) {
      kind = 3;
      id = lin_slot[h.slot];
    }
    float3 nn = kind ? hit_normal(S, o, d, h) : f3(0.0f, 1.0f, 0.0f);
    out_t[i] = h.t;
    out_kind[i] = kind;
    out_id[i] = id;
    out_u[i] = h.u;
    out_v[i] = h.v;
    out_n[3 * i] = nn.x;
    out_n[3 * i + 1] = nn.y;
    out_n[3 * i + 2] = nn.z;
  }
}

static int grid_for_rays(Ctx* ctx, long n) {
  long g = (n + 127) / 128;
  long cap = (long)ctx->num_sms * 16;
  if (g > cap) g = cap;
  return g < 1 ? 1 : (int)g;
}

int trace_closest(Ctx* ctx, Scene* sc, long n, const float* d_ro, const float* d_rd, float* d_t, int* d_id,
                  float* d_u, float* d_v) {
  DevScene S = sc->view();
  if (n <= 0) return RX_OK;
  if (S.exact_slab)
    k_trace_closest<true><<<grid_for_rays(ctx, n), 128, 0, ctx->stream>>>(S, n, d_ro, d_rd, d_t, d_id, d_u, d_v,
                                                                          ctx->d_err);
  else
    k_trace_closest<false><<<grid_for_rays(ctx, n), 128, 0, ctx->stream>>>(S, n, d_ro, d_rd, d_t, d_id, d_u, d_v,
                                                                           ctx->d_err);
  CUDA_TRY(ctx, cudaGetLastError());
  return RX_OK;
}

int trace_any(Ctx* ctx, Scene* sc, long n, const float* d_ro, const float* d_rd, const float* d_tmax, int* d_occ) {
  DevScene S = sc->view();
  if (n <= 0) return RX_OK;
  if (S.exact_slab)
    k_trace_any<true><<<grid_for_rays(ctx, n), 128, 0, ctx->stream>>>(S, n, d_ro, d_rd, d_tmax, d_occ, ctx->d_err);
  else
    k_trace_any<false><<<grid_for_rays(ctx, n), 128, 0, ctx->stream>>>(S, n, d_ro, d_rd, d_tmax, d_occ, ctx->d_err);
  CUDA_TRY(ctx, cudaGetLastError());
  return RX_OK;
}

int scene_query(Ctx* ctx, Scene* sc, long n, const float* d_ro, const float* d_rd, float* d_t, int* d_kind,
                int* d_id, float* d_u, float* d_v, float* d_n) {
  DevScene S = sc->view();
  if (n <= 0) return RX_OK;
  DevBuf<int> lin(ctx, std::max<size_t>(sc->lin_slot.size(), 1));
  if (!lin.ok()) return set_error(ctx, "scene query: out of device memory"), RX_ERR_CAPACITY;
  if (!sc->lin_slot.empty())
    cudaMemcpyAsync(lin.p, sc->lin_slot.data(), sizeof(int) * sc->lin_slot.size(), cudaMemcpyHostToDevice,
                    ctx->stream);
  if (S.exact_slab)
    k_scene_query<true><<<grid_for_rays(ctx, n), 128, 0, ctx->stream>>>(S, n, d_ro, d_rd, lin.p, d_t, d_kind, d_id,
                                                                        d_u, d_v, d_n, ctx->d_err);
  else
    k_scene_query<false><<<grid_for_rays(ctx, n), 128, 0, ctx->stream>>>(S, n, d_ro, d_rd, lin.p, d_t, d_kind, d_id,
                                                                         d_u, d_v, d_n, ctx->d_err);
  CUDA_TRY(ctx, cudaGetLastError());
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return RX_OK;
}

}  // namespace rx
