// GPU BVH construction.
//
// Two builders share the same front end (primitive bounds, centroid bounds,
// 30-bit Morton codes, a stable LSD radix sort written here):
//
//  * build_reference: the reference's Morton build
//    (rendering/taichi/bvh_builder.py:412-478).  Splitting the Morton order
//    at the count median makes the topology depend only on the primitive
//    count, so it is laid out level by level on the device and node bounds
//    are reduced bottom-up.  Node numbering is the reference's DFS pre-order
//    and the output equals GPUBVHBuilder's `nodes` / `ordered_tris` bit for
//    bit.
//  * build_lbvh: Karras' parallel LBVH ("Maximizing parallelism in the
//    construction of BVHs, octrees, and k-d trees", HPG 2012) over the same
//    codes, a bottom-up pass computing bounds and SAH costs, and an SAH
//    collapse of subtrees into leaves of up to `max_leaf` primitives, laid
//    out breadth-first so the top levels are contiguous.
//
// Both emit the traversal layout described in rx_internal.cuh.
#include <algorithm>
#include <cstdio>
#include <vector>

#include "rx_internal.cuh"
#include "rx_runtime.h"

namespace rx {

// L2-coherent load of a float3 written by another thread before a fence.
__device__ __forceinline__ float3 ldcg3(const float3* p) {
  const float* f = reinterpret_cast<const float*>(p);
  return f3(__ldcg(f), __ldcg(f + 1), __ldcg(f + 2));
}

// ----------------------------------------------------------------------------
// front end
// ----------------------------------------------------------------------------
// Primitive i < n_tris is a triangle, else analytic object i - n_tris
// (sphere or cube: obj_a = (centre, kind), obj_b = (radius, 0, 0, 0) or
// (half extents, 0)).  Triangle bounds are padded by 1e-4 and centroids are
// (v0 + v1 + v2) / 3 with the reference's float32 order
// (bvh_builder.py:363-368); an object's centroid is its centre.  box_centre
// != 0 (the LBVH): a triangle's key point is the centre of its bounding box
// instead, which on the benchmark scene's rays gives a tree with 2-4 % fewer
// node visits than the centroid.
__global__ void k_prim_bounds(int n_tris, const float* __restrict__ v0, const float* __restrict__ v1,
                              const float* __restrict__ v2, int n_obj, const float4* __restrict__ obj_a,
                              const float4* __restrict__ obj_b, int box_centre, float3* __restrict__ bmin,
                              float3* __restrict__ bmax, float3* __restrict__ cen) {
  int n = n_tris + n_obj;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (i < n_tris) {
      float3 a = f3(v0[3 * i], v0[3 * i + 1], v0[3 * i + 2]);
      float3 b = f3(v1[3 * i], v1[3 * i + 1], v1[3 * i + 2]);
      float3 c = f3(v2[3 * i], v2[3 * i + 1], v2[3 * i + 2]);
      const float3 lo = vmin(a, vmin(b, c)), hi = vmax(a, vmax(b, c));
      bmin[i] = lo - f3(1e-4f, 1e-4f, 1e-4f);
      bmax[i] = hi + f3(1e-4f, 1e-4f, 1e-4f);
      cen[i] = box_centre ? f3(0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z))
                          : f3(((a.x + b.x) + c.x) / 3.0f, ((a.y + b.y) + c.y) / 3.0f, ((a.z + b.z) + c.z) / 3.0f);
    } else {
      float4 a = obj_a[i - n_tris], b = obj_b[i - n_tris];
      float3 e = __float_as_int(a.w) == PRIM_SPHERE ? f3(b.x, b.x, b.x) : f3(b.x, b.y, b.z);
      bmin[i] = f3(a.x - e.x, a.y - e.y, a.z - e.z) - f3(1e-4f, 1e-4f, 1e-4f);
      bmax[i] = f3(a.x + e.x, a.y + e.y, a.z + e.z) + f3(1e-4f, 1e-4f, 1e-4f);
      cen[i] = f3(a.x, a.y, a.z);
    }
  }
}

// Two-stage exact min/max reduction of the centroids.
__global__ void k_reduce_bounds(int n, const float3* __restrict__ p, float3* __restrict__ part_min,
                                float3* __restrict__ part_max) {
  __shared__ float smin[3][256], smax[3][256];
  float3 lo = f3(INFINITY, INFINITY, INFINITY), hi = f3(-INFINITY, -INFINITY, -INFINITY);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    lo = vmin(lo, p[i]);
    hi = vmax(hi, p[i]);
  }
  int t = threadIdx.x;
  smin[0][t] = lo.x; smin[1][t] = lo.y; smin[2][t] = lo.z;
  smax[0][t] = hi.x; smax[1][t] = hi.y; smax[2][t] = hi.z;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (t < s) {
      for (int k = 0; k < 3; ++k) {
        smin[k][t] = fminf(smin[k][t], smin[k][t + s]);
        smax[k][t] = fmaxf(smax[k][t], smax[k][t + s]);
      }
    }
    __syncthreads();
  }
  if (t == 0) {
    part_min[blockIdx.x] = f3(smin[0][0], smin[1][0], smin[2][0]);
    part_max[blockIdx.x] = f3(smax[0][0], smax[1][0], smax[2][0]);
  }
}

// Second stage: one block of kBoundsThreads reduces the parts' boxes --
// the minimum over mins[] and the maximum over maxs[] -- into out[0],
// out[1].  Min and max are exact, so the result does not depend on the
// order.
constexpr int kBoundsThreads = 1024;
__global__ void __launch_bounds__(kBoundsThreads) k_bounds_final(int parts, const float3* __restrict__ mins,
                                                                 const float3* __restrict__ maxs,
                                                                 float3* __restrict__ out) {
  __shared__ float3 slo[kBoundsThreads], shi[kBoundsThreads];
  float3 lo = f3(INFINITY, INFINITY, INFINITY), hi = f3(-INFINITY, -INFINITY, -INFINITY);
  for (int k = threadIdx.x; k < parts; k += kBoundsThreads) {
    lo = vmin(lo, mins[k]);
    hi = vmax(hi, maxs[k]);
  }
  const int t = threadIdx.x;
  slo[t] = lo;
  shi[t] = hi;
  __syncthreads();
  for (int s = kBoundsThreads / 2; s > 0; s >>= 1) {
    if (t < s) {
      slo[t] = vmin(slo[t], slo[t + s]);
      shi[t] = vmax(shi[t], shi[t + s]);
    }
    __syncthreads();
  }
  if (t == 0) {
    out[0] = slo[0];
    out[1] = shi[0];
  }
}

__device__ __forceinline__ uint32_t expand10(uint32_t v) {
  v &= 0x000003ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

// 30-bit Morton code of each centroid, normalised over the centroid bounds
// exactly as bvh_builder.py:416-443 (extent <= 1e-12 replaced by 1).
// cubic != 0 (the LBVH): all three axes are normalised by the largest
// extent, so the grid's cells are cubes rather than the bounds' shape; on the
// benchmark scene's rays that tree visits 1.5-5 % fewer nodes.
// `bounds`: the centroid bounds (k_bounds_final).
__global__ void k_morton(int n, const float3* __restrict__ cen, const float3* __restrict__ bounds, int cubic,
                         uint32_t* __restrict__ codes, int* __restrict__ idx) {
  __shared__ float3 s_lo, s_ext;
  if (threadIdx.x == 0) {
    const float3 lo = bounds[0], hi = bounds[1];
    float3 e = hi - lo;
    if (e.x <= 1e-12f) e.x = 1.0f;
    if (e.y <= 1e-12f) e.y = 1.0f;
    if (e.z <= 1e-12f) e.z = 1.0f;
    if (cubic) {
      const float m = fmaxf(e.x, fmaxf(e.y, e.z));
      e = f3(m, m, m);
    }
    s_lo = lo;
    s_ext = e;
  }
  __syncthreads();
  float3 lo = s_lo, ext = s_ext;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float3 c = cen[i];
    float x = fminf(fmaxf((c.x - lo.x) / ext.x, 0.0f), 1.0f);
    float y = fminf(fmaxf((c.y - lo.y) / ext.y, 0.0f), 1.0f);
    float z = fminf(fmaxf((c.z - lo.z) / ext.z, 0.0f), 1.0f);
    uint32_t qx = (uint32_t)(x * 1023.0f), qy = (uint32_t)(y * 1023.0f), qz = (uint32_t)(z * 1023.0f);
    codes[i] = (expand10(qx) << 2) | (expand10(qy) << 1) | expand10(qz);
    idx[i] = i;
  }
}

// ----------------------------------------------------------------------------
// stable LSD radix sort, 8-bit digits, (key, value) pairs
// tile = 8 warps x 16 chunks x 32 keys = 4096 keys per block
// ----------------------------------------------------------------------------
constexpr int kSortWarps = 8;
constexpr int kSortChunks = 16;
constexpr int kSortTile = kSortWarps * kSortChunks * 32;

__global__ void k_sort_hist(int n, const uint32_t* __restrict__ keys, int shift, uint32_t* __restrict__ hist,
                            int nblocks) {
  __shared__ uint32_t h[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  int base = blockIdx.x * kSortTile;
  int end = min(base + kSortTile, n);
  for (int i = base + threadIdx.x; i < end; i += blockDim.x) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
  __syncthreads();
  for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[d * nblocks + blockIdx.x] = h[d];
}

// exclusive scan of hist[256 * nblocks] (digit-major), one block of 1024
__global__ void k_sort_scan(uint32_t* __restrict__ hist, int total) {
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int base = 0; base < total; base += blockDim.x) {
    int i = base + threadIdx.x;
    uint32_t v = i < total ? hist[i] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
      uint32_t w = warp_sums[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      warp_sums[lane] = w;
    }
    __syncthreads();
    uint32_t prefix = (wid > 0 ? warp_sums[wid - 1] : 0u) + carry;
    if (i < total) hist[i] = prefix + x - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = prefix + x;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kSortWarps * 32)
    k_sort_scatter(int n, const uint32_t* __restrict__ keys_in, const int* __restrict__ vals_in,
                   uint32_t* __restrict__ keys_out, int* __restrict__ vals_out, int shift,
                   const uint32_t* __restrict__ hist, int nblocks) {
  __shared__ uint32_t wcount[kSortWarps][256];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kSortWarps * 256; i += blockDim.x) (&wcount[0][0])[i] = 0;
  __syncthreads();
  int wbase = blockIdx.x * kSortTile + w * kSortChunks * 32;
  // pass 1: per-warp digit counts
  for (int c = 0; c < kSortChunks; ++c) {
    int i = wbase + c * 32 + lane;
    bool ok = i < n;
    uint32_t dgt = ok ? (keys_in[i] >> shift) & 255u : 256u;
    unsigned peers = __match_any_sync(0xffffffffu, dgt);
    int leader = __ffs(peers) - 1;
    if (ok && lane == leader) wcount[w][dgt] += __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // per-warp starting offsets (block offset from the scanned histogram)
  for (int d = threadIdx.x; d < 256; d += blockDim.x) {
    uint32_t run = hist[d * nblocks + blockIdx.x];
    for (int ww = 0; ww < kSortWarps; ++ww) {
      uint32_t c = wcount[ww][d];
      wcount[ww][d] = run;
      run += c;
    }
  }
  __syncthreads();
  // pass 2: stable scatter in key order
  unsigned lt = (1u << lane) - 1u;
  for (int c = 0; c < kSortChunks; ++c) {
    int i = wbase + c * 32 + lane;
    bool ok = i < n;
    uint32_t key = ok ? keys_in[i] : 0u;
    uint32_t dgt = ok ? (key >> shift) & 255u : 256u;
    unsigned peers = __match_any_sync(0xffffffffu, dgt);
    int leader = __ffs(peers) - 1;
    if (ok) {
      uint32_t pos = wcount[w][dgt] + __popc(peers & lt);
      keys_out[pos] = key;
      vals_out[pos] = vals_in[i];
    }
    __syncwarp();
    if (ok && lane == leader) wcount[w][dgt] += __popc(peers);
    __syncwarp();
  }
}

// Sorts (codes, idx) in place by the low `bits` bits of the key; stable.
static int radix_sort(Ctx* ctx, int n, uint32_t* keys, int* vals, int bits) {
  if (n <= 1) return RX_OK;
  cudaStream_t st = ctx->stream;
  int nblocks = (n + kSortTile - 1) / kSortTile;
  DevBuf<uint32_t> k2(ctx, n), hist(ctx, (size_t)256 * nblocks);
  DevBuf<int> v2(ctx, n);
  if (!all_ok(k2, hist, v2)) return set_error(ctx, "BVH sort: out of device memory"), RX_ERR_CAPACITY;
  uint32_t* ka = keys;
  uint32_t* kb = k2.p;
  int* va = vals;
  int* vb = v2.p;
  int passes = (bits + 7) / 8;
  for (int p = 0; p < passes; ++p) {
    int shift = 8 * p;
    k_sort_hist<<<nblocks, 256, 0, st>>>(n, ka, shift, hist.p, nblocks);
    k_sort_scan<<<1, 1024, 0, st>>>(hist.p, 256 * nblocks);
    k_sort_scatter<<<nblocks, kSortWarps * 32, 0, st>>>(n, ka, va, kb, vb, shift, hist.p, nblocks);
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (ka != keys) {
    cudaMemcpyAsync(keys, ka, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(vals, va, sizeof(int) * n, cudaMemcpyDeviceToDevice, st);
  }
  // k2, v2, hist are released after the stream drains (DevBuf defers frees)
  return RX_OK;
}

// ----------------------------------------------------------------------------
// reference topology: median-by-count split of the sorted order
// ----------------------------------------------------------------------------
// Number of leaves of the count-median tree over m primitives, leaf <= L.
// At every depth the subtree sizes are s or s + 1, so two counters suffice.
__host__ __device__ inline long long median_tree_leaves(long long m, int L) {
  if (m <= L) return 1;
  long long leaves = 0, s = m, cs = 1, cs1 = 0;
  while (cs + cs1 > 0) {
    if (s + 1 <= L) {
      leaves += cs + cs1;
      break;
    }
    if (s <= L) {
      leaves += cs;
      cs = 0;
    }
    long long h = s / 2, ncs = 0, ncs1 = 0;
    if ((s & 1) == 0) ncs += 2 * cs; else { ncs += cs; ncs1 += cs; }
    if (((s + 1) & 1) == 0) ncs1 += 2 * cs1; else { ncs += cs1; ncs1 += cs1; }
    s = h;
    cs = ncs;
    cs1 = ncs1;
  }
  return leaves;
}

struct RefNodeItem {
  int idx, start, count, parent;
};

__global__ void k_ref_level(const RefNodeItem* __restrict__ cur, int ncur, RefNodeItem* __restrict__ next,
                            int* __restrict__ next_count, int leaf, int* __restrict__ left, int* __restrict__ right,
                            int* __restrict__ tstart, int* __restrict__ tcount, int* __restrict__ parent) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncur; i += gridDim.x * blockDim.x) {
    RefNodeItem it = cur[i];
    parent[it.idx] = it.parent;
    if (it.count <= leaf) {
      left[it.idx] = -1;
      right[it.idx] = -1;
      tstart[it.idx] = it.start;
      tcount[it.idx] = it.count;
    } else {
      int nl = it.count / 2;
      int li = it.idx + 1;
      int ri = it.idx + 1 + (int)(2 * median_tree_leaves(nl, leaf) - 1);
      left[it.idx] = li;
      right[it.idx] = ri;
      tstart[it.idx] = -1;
      tcount[it.idx] = 0;
      int o = atomicAdd(next_count, 2);
      next[o] = RefNodeItem{li, it.start, nl, it.idx};
      next[o + 1] = RefNodeItem{ri, it.start + nl, it.count - nl, it.idx};
    }
  }
}

// Leaves reduce their primitives' bounds, then walk up: the second child to
// arrive at a parent combines both (min / max are exact, order-free).
__global__ void k_ref_bounds(int n_nodes, const int* __restrict__ left, const int* __restrict__ right,
                             const int* __restrict__ tstart, const int* __restrict__ tcount,
                             const int* __restrict__ parent, const int* __restrict__ order,
                             const float3* __restrict__ pmin, const float3* __restrict__ pmax,
                             float3* __restrict__ nmin, float3* __restrict__ nmax, int* __restrict__ flags) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes; i += gridDim.x * blockDim.x) {
    if (left[i] != -1) continue;
    float3 lo = f3(INFINITY, INFINITY, INFINITY), hi = f3(-INFINITY, -INFINITY, -INFINITY);
    for (int k = tstart[i]; k < tstart[i] + tcount[i]; ++k) {
      int t = order[k];
      lo = vmin(lo, pmin[t]);
      hi = vmax(hi, pmax[t]);
    }
    nmin[i] = lo;
    nmax[i] = hi;
    int node = parent[i];
    while (node >= 0) {
      __threadfence();
      if (atomicAdd(&flags[node], 1) == 0) break;  // first arrival: sibling finishes
      __threadfence();
      int l = left[node], r = right[node];
      float3 a0 = ldcg3(nmin + l), a1 = ldcg3(nmax + l);
      float3 b0 = ldcg3(nmin + r), b1 = ldcg3(nmax + r);
      nmin[node] = vmin(a0, b0);
      nmax[node] = vmax(a1, b1);
      node = parent[node];
    }
  }
}

// Reference-format nodes -> traversal layout (node index preserved, so the
// root stays 0).  A root leaf gets a wrapper node whose right child is an
// empty leaf.
__global__ void k_ref_to_layout(int n_nodes, const int* __restrict__ left, const int* __restrict__ right,
                                const int* __restrict__ tstart, const int* __restrict__ tcount,
                                const float3* __restrict__ nmin, const float3* __restrict__ nmax,
                                float4* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes; i += gridDim.x * blockDim.x) {
    int l, r;
    float3 l0, l1, r0, r1;
    int lw, rw, lc, rc;
    if (left[i] == -1) {
      if (i != 0) continue;  // leaves live inside their parent's record
      l0 = nmin[0]; l1 = nmax[0];
      lw = pack_leaf(tstart[0], tcount[0]); lc = tcount[0];
      r0 = f3(1e30f, 1e30f, 1e30f); r1 = r0;
      rw = pack_leaf(0, 0); rc = 0;
    } else {
      l = left[i];
      r = right[i];
      l0 = nmin[l]; l1 = nmax[l];
      r0 = nmin[r]; r1 = nmax[r];
      lw = left[l] == -1 ? pack_leaf(tstart[l], tcount[l]) : l;
      lc = left[l] == -1 ? tcount[l] : 0;
      rw = left[r] == -1 ? pack_leaf(tstart[r], tcount[r]) : r;
      rc = left[r] == -1 ? tcount[r] : 0;
    }
    float4* o = out + 4 * (size_t)i;
    o[0] = make_float4(l0.x, l1.x, l0.y, l1.y);
    o[1] = make_float4(l0.z, l1.z, r0.x, r1.x);
    o[2] = make_float4(r0.y, r1.y, r0.z, r1.z);
    o[3] = make_float4(__int_as_float(lw), __int_as_float(rw), __int_as_float(lc), __int_as_float(rc));
  }
}

// Primitives and shading records gathered into leaf order.
__global__ void k_gather_prims(int n, const int* __restrict__ order, int n_tris, const float* __restrict__ v0,
                               const float* __restrict__ v1, const float* __restrict__ v2,
                               const float* __restrict__ n0, const float* __restrict__ n1,
                               const float* __restrict__ n2, const int* __restrict__ tri_mat,
                               const float4* __restrict__ obj_a, const float4* __restrict__ obj_b,
                               const int* __restrict__ obj_mat, const int* __restrict__ obj_slot,
                               float4* __restrict__ prims, float4* __restrict__ shade) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    int i = order[k];
    float4* P = prims + 3 * (size_t)k;
    float4* S = shade + 3 * (size_t)k;
    if (i < n_tris) {
      float3 a = f3(v0[3 * i], v0[3 * i + 1], v0[3 * i + 2]);
      float3 b = f3(v1[3 * i], v1[3 * i + 1], v1[3 * i + 2]);
      float3 c = f3(v2[3 * i], v2[3 * i + 1], v2[3 * i + 2]);
      float3 e1 = b - a, e2 = c - a;
      P[0] = make_float4(a.x, a.y, a.z, __int_as_float(PRIM_TRI));
      P[1] = make_float4(e1.x, e1.y, e1.z, 0.0f);
      P[2] = make_float4(e2.x, e2.y, e2.z, 0.0f);
      S[0] = make_float4(n0[3 * i], n0[3 * i + 1], n0[3 * i + 2], __int_as_float(tri_mat ? tri_mat[i] : 0));
      S[1] = make_float4(n1[3 * i], n1[3 * i + 1], n1[3 * i + 2], __int_as_float(i));
      S[2] = make_float4(n2[3 * i], n2[3 * i + 1], n2[3 * i + 2], 0.0f);
    } else {
      int s = i - n_tris;
      P[0] = obj_a[s];
      P[1] = obj_b[s];
      P[2] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      S[0] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(obj_mat[s]));
      S[1] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(obj_slot[s]));
      S[2] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
  }
}

// ----------------------------------------------------------------------------
// Karras LBVH + SAH collapse
// ----------------------------------------------------------------------------
__device__ __forceinline__ int lcp(const uint32_t* codes, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  uint32_t a = codes[i], b = codes[j];
  if (a == b) return 32 + __clz((uint32_t)i ^ (uint32_t)j);
  return __clz(a ^ b);
}

// Internal node i of n - 1.  Children are encoded as c >= 0 internal, c < 0
// leaf ~prim (sorted position).
__global__ void k_karras(int n, const uint32_t* __restrict__ codes, int* __restrict__ kl, int* __restrict__ kr,
                         int* __restrict__ first, int* __restrict__ last, int* __restrict__ parent_int,
                         int* __restrict__ parent_leaf) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
    int d = (lcp(codes, n, i, i + 1) - lcp(codes, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = lcp(codes, n, i, i - d);
    int lmax = 2;
    while (lcp(codes, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
      if (lcp(codes, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = lcp(codes, n, i, j);
    int s = 0;
    int t = l;
    do {
      t = (t + 1) >> 1;
      if (lcp(codes, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    int gamma = i + s * d + min(d, 0);
    int lo = min(i, j), hi = max(i, j);
    int lc = (lo == gamma) ? ~gamma : gamma;
    int rc = (hi == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    kl[i] = lc;
    kr[i] = rc;
    first[i] = lo;
    last[i] = hi;
    if (lc >= 0) parent_int[lc] = i; else parent_leaf[~lc] = i;
    if (rc >= 0) parent_int[rc] = i; else parent_leaf[~rc] = i;
  }
}

__device__ __forceinline__ float half_area(float3 lo, float3 hi) {
  float3 e = hi - lo;
  return e.x * e.y + e.y * e.z + e.z * e.x;
}

// Bottom-up bounds and SAH cost.  cost(node) = min(C_i * count (if count <=
// max_leaf), C_t + (A_l cost_l + A_r cost_r) / A); collapse[] records which
// choice won.
__global__ void k_lbvh_bottom_up(int n, const int* __restrict__ order, const int* __restrict__ kl,
                                 const int* __restrict__ kr, const int* __restrict__ parent_int,
                                 const int* __restrict__ parent_leaf, const float3* __restrict__ pmin,
                                 const float3* __restrict__ pmax, float3* __restrict__ imin,
                                 float3* __restrict__ imax, float* __restrict__ icost, int* __restrict__ icount,
                                 int* __restrict__ collapse, int* __restrict__ flags, int max_leaf, float c_t,
                                 float c_i) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    int node = parent_leaf[k];
    while (node >= 0) {
      __threadfence();
      if (atomicAdd(&flags[node], 1) == 0) break;
      __threadfence();
      int l = kl[node], r = kr[node];
      float3 l0, l1, r0, r1;
      float lcost, rcost;
      int lcnt, rcnt;
      if (l < 0) {
        int p = order[~l];
        l0 = pmin[p]; l1 = pmax[p]; lcost = c_i; lcnt = 1;
      } else {
        l0 = ldcg3(imin + l); l1 = ldcg3(imax + l);
        lcost = __ldcg(icost + l); lcnt = __ldcg(icount + l);
      }
      if (r < 0) {
        int p = order[~r];
        r0 = pmin[p]; r1 = pmax[p]; rcost = c_i; rcnt = 1;
      } else {
        r0 = ldcg3(imin + r); r1 = ldcg3(imax + r);
        rcost = __ldcg(icost + r); rcnt = __ldcg(icount + r);
      }
      float3 lo = vmin(l0, r0), hi = vmax(l1, r1);
      float a = fmaxf(half_area(lo, hi), 1e-30f);
      float split = c_t + (half_area(l0, l1) * lcost + half_area(r0, r1) * rcost) / a;
      int cnt = lcnt + rcnt;
      float leafc = c_i * (float)cnt;
      int col = (cnt <= max_leaf && leafc <= split) ? 1 : 0;
      imin[node] = lo;
      imax[node] = hi;
      icost[node] = col ? leafc : split;
      icount[node] = cnt;
      collapse[node] = col;
      node = parent_int[node];
    }
  }
}

// Breadth-first level walks run without a host round trip per level: the
// walk's state lives on the device -- lv[0] nodes of the level being laid
// out, lv[1] output index of its first node, lv[2] nodes queued for the next
// level, lv[3] blocks of the current launch that have finished, lv[4] levels
// laid out, lv[5] set when a level would overflow the tree -- and the last
// block of each level launch advances it for the
// next launch.  Every block reads lv[0] and lv[1] before it counts itself
// finished, so the advance never races with a reader.  A launch that finds
// lv[0] == 0 (the walk is over) returns at once; the host enqueues levels in
// batches and reads lv back once per batch.
enum { LV_NCUR = 0, LV_BASE = 1, LV_NEXT = 2, LV_DONE = 3, LV_LEVELS = 4, LV_OVERFLOW = 5, LV_N = 8 };

__device__ __forceinline__ void level_advance(int* lv) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&lv[LV_DONE], 1) == (int)gridDim.x - 1) {
      const int ncur = lv[LV_NCUR];
      lv[LV_BASE] += ncur;
      lv[LV_NCUR] = atomicAdd(&lv[LV_NEXT], 0);
      lv[LV_NEXT] = 0;
      lv[LV_DONE] = 0;
      lv[LV_LEVELS] += 1;
      __threadfence();
    }
  }
}

// One breadth-first level of the collapsed tree.  `cur` holds Karras node
// ids; their output indices are base + position.  Kept internal children
// are appended to `next` and receive indices in the following level.
__global__ void k_lbvh_layout_level(const int* __restrict__ cur, int* __restrict__ next, int* __restrict__ lv,
                                    int n_total, const int* __restrict__ kl,
                                    const int* __restrict__ kr, const int* __restrict__ first,
                                    const int* __restrict__ last, const int* __restrict__ collapse,
                                    const int* __restrict__ order, const float3* __restrict__ pmin,
                                    const float3* __restrict__ pmax, const float3* __restrict__ imin,
                                    const float3* __restrict__ imax, float4* __restrict__ out) {
  const int ncur = lv[LV_NCUR], out_base = lv[LV_BASE];
  if (ncur <= 0) return;
  if (out_base + ncur > n_total) {  // cannot happen for a tree of n_total nodes
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      lv[LV_OVERFLOW] = 1;
      lv[LV_NCUR] = 0;
    }
    return;
  }
  const int next_base = out_base + ncur, next_cap = n_total - next_base;
  int* next_count = &lv[LV_NEXT];
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < ncur; q += gridDim.x * blockDim.x) {
    int node = cur[q];
    int words[2], counts[2];
    float3 b0[2], b1[2];
    int ch[2] = {kl[node], kr[node]};
    for (int s = 0; s < 2; ++s) {
      int c = ch[s];
      if (c < 0) {
        int p = order[~c];
        b0[s] = pmin[p]; b1[s] = pmax[p];
        words[s] = pack_leaf(~c, 1);  // one primitive at sorted position ~c
        counts[s] = 1;
      } else if (collapse[c]) {
        b0[s] = imin[c]; b1[s] = imax[c];
        words[s] = pack_leaf(first[c], last[c] - first[c] + 1);
        counts[s] = last[c] - first[c] + 1;
      } else {
        b0[s] = imin[c]; b1[s] = imax[c];
        int o = atomicAdd(next_count, 1);
        if (o < next_cap) next[o] = c;
        words[s] = next_base + o;
        counts[s] = 0;
      }
    }
    float4* o = out + 4 * (size_t)(out_base + q);
    o[0] = make_float4(b0[0].x, b1[0].x, b0[0].y, b1[0].y);
    o[1] = make_float4(b0[0].z, b1[0].z, b0[1].x, b1[1].x);
    o[2] = make_float4(b0[1].y, b1[1].y, b0[1].z, b1[1].z);
    o[3] = make_float4(__int_as_float(words[0]), __int_as_float(words[1]), __int_as_float(counts[0]),
                       __int_as_float(counts[1]));
  }
  level_advance(lv);
}

// 4-wide nodes from the laid-out binary tree, one level per launch.  The
// 4-wide node of binary node b starts from b's two children and, while it
// has fewer than four, opens the internal child of largest surface area
// (replacing it by its own two children): the children that the most rays
// enter are expanded first, which removes more node visits than always
// taking both grandchildren (6-8 % fewer visits per ray on the displaced
// icosphere).  Leaf children stay leaves; internal children that remain
// become 4-wide nodes of the next level.  Empty binary slots (count 0
// leaves) are dropped; unused slots get a box at 1e30 and count 0.
__global__ void k_bvh4_level(const int* __restrict__ cur, int* __restrict__ next, int* __restrict__ lv,
                             const float4* __restrict__ bin, int n_bin, float4* __restrict__ out4, int* err) {
  const int ncur = lv[LV_NCUR], out_base = lv[LV_BASE];
  if (ncur <= 0) return;
  if (out_base + ncur > n_bin) {  // a 4-wide tree has at most as many nodes as the binary one
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      lv[LV_OVERFLOW] = 1;
      lv[LV_NCUR] = 0;
    }
    return;
  }
  const int next_base = out_base + ncur, next_cap = n_bin - next_base;
  int* next_count = &lv[LV_NEXT];
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < ncur; q += gridDim.x * blockDim.x) {
    float mn[4][3], mx[4][3];
    int wd[4], ct[4];
    int k = 0;
    // appends child `side` of the binary record nb (nothing for an empty slot)
    auto add = [&](const float4* nb, int side) {
      const float4 n0 = nb[0], n1 = nb[1], n2 = nb[2], n3 = nb[3];
      const int w = __float_as_int(side ? n3.y : n3.x), c = __float_as_int(side ? n3.w : n3.z);
      if (w < 0 && c == 0) return;  // empty slot
      if (k >= 4) {                 // cannot happen: a node is opened only while k < 4
        atomicOr(err, ERR_BAD_NODE);
        return;
      }
      if (side == 0) {
        mn[k][0] = n0.x, mx[k][0] = n0.y, mn[k][1] = n0.z, mx[k][1] = n0.w, mn[k][2] = n1.x, mx[k][2] = n1.y;
      } else {
        mn[k][0] = n1.z, mx[k][0] = n1.w, mn[k][1] = n2.x, mx[k][1] = n2.y, mn[k][2] = n2.z, mx[k][2] = n2.w;
      }
      wd[k] = w;
      ct[k] = w >= 0 ? 0 : c;
      ++k;
    };
    const int b = cur[q];
    const float4* nb = bin + 4 * (size_t)b;
    add(nb, 0);
    add(nb, 1);
    while (k < 4) {
      int bi = -1;
      float ba = -1.0f;
      for (int i = 0; i < k; ++i) {
        if (wd[i] < 0) continue;
        if (wd[i] >= n_bin) {  // never entered: flagged and turned into an empty leaf
          atomicOr(err, ERR_BAD_NODE);
          wd[i] = pack_leaf(0, 0);
          ct[i] = 0;
          continue;
        }
        const float ex = mx[i][0] - mn[i][0], ey = mx[i][1] - mn[i][1], ez = mx[i][2] - mn[i][2];
        const float a = ex * ey + ey * ez + ez * ex;
        if (a > ba) {
          ba = a;
          bi = i;
        }
      }
      if (bi < 0) break;
      const float4* cb = bin + 4 * (size_t)wd[bi];
      // remove entry bi (the last entry moves into its place), then append
      // its two children
      --k;
      if (bi != k) {
        for (int a = 0; a < 3; ++a) mn[bi][a] = mn[k][a], mx[bi][a] = mx[k][a];
        wd[bi] = wd[k];
        ct[bi] = ct[k];
      }
      add(cb, 0);
      add(cb, 1);
    }
    for (int i = 0; i < k; ++i) {
      if (wd[i] < 0) continue;
      // an internal binary node becomes a 4-wide node of the next level
      const int o = atomicAdd(next_count, 1);
      if (o < next_cap) {
        next[o] = wd[i];
        wd[i] = next_base + o;
      } else {
        atomicOr(err, ERR_BAD_NODE);
        wd[i] = pack_leaf(0, 0);
      }
    }
    for (; k < 4; ++k) {
      mn[k][0] = mn[k][1] = mn[k][2] = 1e30f;
      mx[k][0] = mx[k][1] = mx[k][2] = 1e30f;
      wd[k] = pack_leaf(0, 0);
      ct[k] = 0;
    }
    float4* o = out4 + 8 * (size_t)(out_base + q);
    o[0] = make_float4(mn[0][0], mn[1][0], mn[2][0], mn[3][0]);
    o[1] = make_float4(mx[0][0], mx[1][0], mx[2][0], mx[3][0]);
    o[2] = make_float4(mn[0][1], mn[1][1], mn[2][1], mn[3][1]);
    o[3] = make_float4(mx[0][1], mx[1][1], mx[2][1], mx[3][1]);
    o[4] = make_float4(mn[0][2], mn[1][2], mn[2][2], mn[3][2]);
    o[5] = make_float4(mx[0][2], mx[1][2], mx[2][2], mx[3][2]);
    o[6] = make_float4(__int_as_float(wd[0]), __int_as_float(wd[1]), __int_as_float(wd[2]), __int_as_float(wd[3]));
    o[7] = make_float4(__int_as_float(ct[0]), __int_as_float(ct[1]), __int_as_float(ct[2]), __int_as_float(ct[3]));
  }
  level_advance(lv);
}

// Root record for a tree that is a single leaf of `cnt` primitives.
__global__ void k_single_leaf_root(const float3* __restrict__ bmin, const float3* __restrict__ bmax, int cnt,
                                   float4* __restrict__ out) {
  float3 l0 = bmin[0], l1 = bmax[0];
  float3 r0 = f3(1e30f, 1e30f, 1e30f);
  out[0] = make_float4(l0.x, l1.x, l0.y, l1.y);
  out[1] = make_float4(l0.z, l1.z, r0.x, r0.x);
  out[2] = make_float4(r0.y, r0.y, r0.z, r0.z);
  out[3] = make_float4(__int_as_float(pack_leaf(0, cnt)), __int_as_float(pack_leaf(0, 0)), __int_as_float(cnt), __int_as_float(0));
}

static int grid_for(Ctx* ctx, long long n, int block = 256) {
  long long g = (n + block - 1) / block;
  long long cap = (long long)ctx->num_sms * 32;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

// Shared front end: bounds, centroids, Morton codes, stable sort.
// lbvh_keys != 0: Morton keys of box centres on cubic cells (the LBVH); 0:
// the reference's centroids and per-axis normalisation.
static int front_end(Ctx* ctx, Scene* sc, int n_obj, const float4* d_obj_a, const float4* d_obj_b, int lbvh_keys,
                     DevBuf<float3>& pmin, DevBuf<float3>& pmax, DevBuf<int>& order) {
  int n = sc->n_tris + n_obj;
  cudaStream_t st = ctx->stream;
  DevBuf<float3> cen(ctx, n);
  const int parts = std::min(grid_for(ctx, n), 1024);
  DevBuf<float3> part_min(ctx, parts), part_max(ctx, parts);
  DevBuf<uint32_t> codes(ctx, n);
  DevBuf<float3> cbox(ctx, 2);
  if (!all_ok(pmin, pmax, order, cen, part_min, part_max, codes, cbox))
    return set_error(ctx, "BVH build: out of device memory"), RX_ERR_CAPACITY;
  k_prim_bounds<<<grid_for(ctx, n), 256, 0, st>>>(sc->n_tris, sc->d_v0, sc->d_v1, sc->d_v2, n_obj, d_obj_a, d_obj_b,
                                                   lbvh_keys, pmin.p, pmax.p, cen.p);
  k_reduce_bounds<<<parts, 256, 0, st>>>(n, cen.p, part_min.p, part_max.p);
  k_bounds_final<<<1, kBoundsThreads, 0, st>>>(parts, part_min.p, part_max.p, cbox.p);
  k_morton<<<grid_for(ctx, n), 256, 0, st>>>(n, cen.p, cbox.p, lbvh_keys, codes.p, order.p);
  if (int rc = radix_sort(ctx, n, codes.p, order.p, 30)) return rc;
  sc->tmp_codes.swap(codes);
  return RX_OK;
}

int build_reference(Ctx* ctx, Scene* sc, int leaf) {
  cudaStream_t st = ctx->stream;
  int n = sc->n_tris;
  sc->clear_bvh();
  if (n <= 0) return RX_OK;
  DevBuf<float3> pmin(ctx, n), pmax(ctx, n);
  DevBuf<int> order(ctx, n);
  if (int rc = front_end(ctx, sc, 0, nullptr, nullptr, 0, pmin, pmax, order)) return rc;
  long long n_nodes_ll = 2 * median_tree_leaves(n, leaf) - 1;
  int n_nodes = (int)n_nodes_ll;
  DevBuf<int> left(ctx, n_nodes), right(ctx, n_nodes), tstart(ctx, n_nodes), tcount(ctx, n_nodes);
  DevBuf<int> parent(ctx, n_nodes), flags(ctx, n_nodes);
  DevBuf<float3> nmin(ctx, n_nodes), nmax(ctx, n_nodes);
  DevBuf<RefNodeItem> la(ctx, n_nodes), lb(ctx, n_nodes);
  DevBuf<int> cnt(ctx, 1);
  if (!all_ok(left, right, tstart, tcount, parent, flags, nmin, nmax, la, lb, cnt))
    return set_error(ctx, "reference build: out of device memory"), RX_ERR_CAPACITY;
  RefNodeItem root{0, 0, n, -1};
  cudaMemcpyAsync(la.p, &root, sizeof(root), cudaMemcpyHostToDevice, st);
  int ncur = 1;
  RefNodeItem* cur = la.p;
  RefNodeItem* nxt = lb.p;
  int levels = 0;
  while (ncur > 0) {
    if (++levels > 256 || ncur > n_nodes)
      return set_error(ctx, "reference build: level walk did not terminate"), RX_ERR_DEVICE;
    cudaMemsetAsync(cnt.p, 0, sizeof(int), st);
    k_ref_level<<<grid_for(ctx, ncur), 256, 0, st>>>(cur, ncur, nxt, cnt.p, leaf, left.p, right.p, tstart.p,
                                                      tcount.p, parent.p);
    int h = 0;
    cudaMemcpyAsync(&h, cnt.p, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    ncur = h;
    std::swap(cur, nxt);
  }
  cudaMemsetAsync(flags.p, 0, sizeof(int) * n_nodes, st);
  k_ref_bounds<<<grid_for(ctx, n_nodes), 256, 0, st>>>(n_nodes, left.p, right.p, tstart.p, tcount.p, parent.p,
                                                        order.p, pmin.p, pmax.p, nmin.p, nmax.p, flags.p);
  sc->d_nodes.alloc(ctx, (size_t)4 * n_nodes);
  sc->d_prims.alloc(ctx, (size_t)3 * n);
  sc->d_shade.alloc(ctx, (size_t)3 * n);
  if (!all_ok(sc->d_nodes, sc->d_prims, sc->d_shade)) {
    sc->clear_bvh();
    return set_error(ctx, "reference build: out of device memory"), RX_ERR_CAPACITY;
  }
  k_ref_to_layout<<<grid_for(ctx, n_nodes), 256, 0, st>>>(n_nodes, left.p, right.p, tstart.p, tcount.p, nmin.p,
                                                           nmax.p, sc->d_nodes.p);
  k_gather_prims<<<grid_for(ctx, n), 256, 0, st>>>(n, order.p, sc->n_tris, sc->d_v0, sc->d_v1, sc->d_v2, sc->d_n0,
                                                    sc->d_n1, sc->d_n2, sc->d_tri_mat, nullptr, nullptr, nullptr, nullptr,
                                                    sc->d_prims.p, sc->d_shade.p);
  float3 rb[2];
  cudaMemcpyAsync(&rb[0], nmin.p, sizeof(float3), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&rb[1], nmax.p, sizeof(float3), cudaMemcpyDeviceToHost, st);
  // keep the reference-format arrays for export
  sc->ref_left.swap(left);
  sc->ref_right.swap(right);
  sc->ref_start.swap(tstart);
  sc->ref_count.swap(tcount);
  sc->ref_min.swap(nmin);
  sc->ref_max.swap(nmax);
  sc->order.swap(order);
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  sc->root_min = rb[0];
  sc->root_max = rb[1];
  sc->n_nodes = n_nodes;
  sc->n_prims = n;
  sc->n_bvh_spheres = 0;
  sc->method = RX_BVH_REFERENCE;
  sc->exact_slab = 1;
  sc->leaf_size = leaf;
  return RX_OK;
}

// Upload of an externally built tree in the reference's node format.
int set_reference_nodes(Ctx* ctx, Scene* sc, int n_nodes, const float* node_min, const float* node_max,
                        const int* left, const int* right, const int* start, const int* count, const int* order) {
  cudaStream_t st = ctx->stream;
  int n = sc->n_tris;
  sc->clear_bvh();
  if (n <= 0 || n_nodes <= 0) return RX_OK;
  DevBuf<int> l(ctx, n_nodes), r(ctx, n_nodes), s(ctx, n_nodes), c(ctx, n_nodes), ord(ctx, n);
  DevBuf<float3> nmin(ctx, n_nodes), nmax(ctx, n_nodes);
  sc->d_nodes.alloc(ctx, (size_t)4 * n_nodes);
  sc->d_prims.alloc(ctx, (size_t)3 * n);
  sc->d_shade.alloc(ctx, (size_t)3 * n);
  if (!all_ok(l, r, s, c, ord, nmin, nmax, sc->d_nodes, sc->d_prims, sc->d_shade)) {
    sc->clear_bvh();
    return set_error(ctx, "BVH upload: out of device memory"), RX_ERR_CAPACITY;
  }
  cudaMemcpyAsync(l.p, left, sizeof(int) * n_nodes, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(r.p, right, sizeof(int) * n_nodes, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s.p, start, sizeof(int) * n_nodes, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(c.p, count, sizeof(int) * n_nodes, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(nmin.p, node_min, sizeof(float3) * n_nodes, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(nmax.p, node_max, sizeof(float3) * n_nodes, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(ord.p, order, sizeof(int) * n, cudaMemcpyHostToDevice, st);
  k_ref_to_layout<<<grid_for(ctx, n_nodes), 256, 0, st>>>(n_nodes, l.p, r.p, s.p, c.p, nmin.p, nmax.p,
                                                           sc->d_nodes.p);
  k_gather_prims<<<grid_for(ctx, n), 256, 0, st>>>(n, ord.p, sc->n_tris, sc->d_v0, sc->d_v1, sc->d_v2, sc->d_n0,
                                                    sc->d_n1, sc->d_n2, sc->d_tri_mat, nullptr, nullptr, nullptr, nullptr,
                                                    sc->d_prims.p, sc->d_shade.p);
  sc->ref_left.swap(l);
  sc->ref_right.swap(r);
  sc->ref_start.swap(s);
  sc->ref_count.swap(c);
  sc->ref_min.swap(nmin);
  sc->ref_max.swap(nmax);
  sc->order.swap(ord);
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  sc->root_min = f3(node_min[0], node_min[1], node_min[2]);
  sc->root_max = f3(node_max[0], node_max[1], node_max[2]);
  sc->n_nodes = n_nodes;
  sc->n_prims = n;
  sc->n_bvh_spheres = 0;
  sc->method = RX_BVH_REFERENCE;
  sc->exact_slab = 1;
  sc->leaf_size = 0;
  return RX_OK;
}

// Runs a device-driven level walk: `launch(level, cur, next, lv)` enqueues
// one level (cur / next alternate between a and b); levels are enqueued in
// batches of kLevelBatch and the state is read back once per batch.  The
// root (node 0) is the only node of level 0.  Returns the total nodes laid
// out through *n_out and the number of levels through *levels.
constexpr int kLevelBatch = 16, kMaxLevels = 1024;
template <class F>
static int level_walk(Ctx* ctx, int* a, int* b, int* lv, int* n_out, int* levels, F launch) {
  cudaStream_t st = ctx->stream;
  const int init[LV_N] = {1, 0, 0, 0, 0, 0, 0, 0};
  CUDA_TRY(ctx, cudaMemsetAsync(a, 0, sizeof(int), st));
  CUDA_TRY(ctx, cudaMemcpyAsync(lv, init, sizeof(init), cudaMemcpyHostToDevice, st));
  int h[LV_N] = {0};
  for (int level = 0;;) {
    for (int k = 0; k < kLevelBatch; ++k, ++level) launch(level, (level & 1) ? b : a, (level & 1) ? a : b, lv);
    CUDA_TRY(ctx, cudaGetLastError());
    CUDA_TRY(ctx, cudaMemcpyAsync(h, lv, sizeof(h), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
    if (h[LV_OVERFLOW]) return set_error(ctx, "BVH level walk: a level overflowed the tree"), RX_ERR_DEVICE;
    if (h[LV_NCUR] == 0) break;
    if (level >= kMaxLevels) return set_error(ctx, "BVH level walk did not terminate"), RX_ERR_DEVICE;
  }
  *n_out = h[LV_BASE];
  *levels = h[LV_LEVELS];
  return RX_OK;
}

// Blocks for level `level` of a tree whose nodes have up to `fan` children:
// at most fan^level nodes, and never more than the whole tree's n.
static int level_grid(Ctx* ctx, int level, int fan_log2, long long n) {
  const long long bound = level * fan_log2 >= 40 ? n : std::min<long long>(n, 1LL << (level * fan_log2));
  long long g = (bound + 255) / 256;
  const long long cap = (long long)ctx->num_sms * 32;
  return (int)std::max<long long>(1, std::min(g, cap));
}

// The 4-wide copy of the laid-out binary tree (k_bvh4_level, level by
// level from the root, breadth first).
static int build_wide(Ctx* ctx, Scene* sc) {
  cudaStream_t st = ctx->stream;
  const int nb = sc->n_nodes;
  sc->n_nodes4 = 0;
  if (nb <= 0) return RX_OK;
  if (!sc->d_nodes4.alloc(ctx, (size_t)8 * nb)) return set_error(ctx, "out of device memory for the 4-wide BVH"), RX_ERR_CAPACITY;
  DevBuf<int> la(ctx, nb), lb(ctx, nb), lv(ctx, LV_N);
  if (!all_ok(la, lb, lv)) return set_error(ctx, "out of device memory"), RX_ERR_CAPACITY;
  int base = 0, levels = 0;
  int rc = level_walk(ctx, la.p, lb.p, lv.p, &base, &levels, [&](int level, int* cur, int* nxt, int* st_lv) {
    k_bvh4_level<<<level_grid(ctx, level, 2, nb), 256, 0, st>>>(cur, nxt, st_lv, sc->d_nodes.p, nb, sc->d_nodes4.p,
                                                              ctx->d_err);
  });
  if (rc) return rc;
  sc->n_nodes4 = base;
  return RX_OK;
}

int build_lbvh(Ctx* ctx, Scene* sc, int max_leaf, int spheres_in_bvh, float c_t, float c_i) {
  cudaStream_t st = ctx->stream;
  sc->clear_bvh();
  // bounded analytic objects (spheres, cubes) taken from the object slots
  // into the BVH; planes (unbounded) and slot triangles stay linear
  std::vector<float4> oa, ob;
  std::vector<int> obj_mat, obj_slot;
  sc->bvh_sphere_slots.clear();
  if (spheres_in_bvh) {
    for (int i = 0; i < (int)sc->objs.size(); ++i) {
      const ObjSlot& o = sc->objs[i];
      if (o.type == 0) {
        oa.push_back(make_float4(o.center.x, o.center.y, o.center.z, int_bits_as_float(PRIM_SPHERE)));
        ob.push_back(make_float4(o.radius, 0.0f, 0.0f, 0.0f));
      } else if (o.type == 2) {
        oa.push_back(make_float4(o.center.x, o.center.y, o.center.z, int_bits_as_float(PRIM_CUBE)));
        ob.push_back(make_float4(o.extra.x, o.extra.y, o.extra.z, 0.0f));
      } else {
        continue;
      }
      obj_mat.push_back(o.mat);
      obj_slot.push_back(i);
    }
  }
  sc->bvh_sphere_slots = obj_slot;
  sc->upload_linear_objects(ctx, spheres_in_bvh != 0);
  int n_obj = (int)oa.size();
  int n = sc->n_tris + n_obj;
  if (n <= 0) return RX_OK;
  DevBuf<float4> d_oa(ctx, std::max(n_obj, 1)), d_ob(ctx, std::max(n_obj, 1));
  DevBuf<int> d_obj_mat(ctx, std::max(n_obj, 1)), d_obj_slot(ctx, std::max(n_obj, 1));
  if (!all_ok(d_oa, d_ob, d_obj_mat, d_obj_slot)) return set_error(ctx, "LBVH: out of device memory"), RX_ERR_CAPACITY;
  if (n_obj) {
    cudaMemcpyAsync(d_oa.p, oa.data(), sizeof(float4) * n_obj, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_ob.p, ob.data(), sizeof(float4) * n_obj, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_obj_mat.p, obj_mat.data(), sizeof(int) * n_obj, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_obj_slot.p, obj_slot.data(), sizeof(int) * n_obj, cudaMemcpyHostToDevice, st);
  }
  DevBuf<float3> pmin(ctx, n), pmax(ctx, n);
  DevBuf<int> order(ctx, n);
  if (int rc = front_end(ctx, sc, n_obj, d_oa.p, d_ob.p, 1, pmin, pmax, order)) return rc;
  sc->d_prims.alloc(ctx, (size_t)3 * n);
  sc->d_shade.alloc(ctx, (size_t)3 * n);
  DevBuf<float3> rb(ctx, 2);
  if (!all_ok(sc->d_prims, sc->d_shade, rb)) {
    sc->clear_bvh();
    return set_error(ctx, "LBVH: out of device memory"), RX_ERR_CAPACITY;
  }
  k_gather_prims<<<grid_for(ctx, n), 256, 0, st>>>(n, order.p, sc->n_tris, sc->d_v0, sc->d_v1, sc->d_v2, sc->d_n0,
                                                    sc->d_n1, sc->d_n2, sc->d_tri_mat, d_oa.p, d_ob.p, d_obj_mat.p,
                                                    d_obj_slot.p, sc->d_prims.p, sc->d_shade.p);
  {
    // root box = union of all primitive boxes (two-stage parallel reduction)
    int parts = std::min(grid_for(ctx, n), 1024);
    DevBuf<float3> lo_min(ctx, parts), lo_max(ctx, parts), hi_min(ctx, parts), hi_max(ctx, parts);
    if (!all_ok(lo_min, lo_max, hi_min, hi_max)) {
      sc->clear_bvh();
      return set_error(ctx, "LBVH: out of device memory"), RX_ERR_CAPACITY;
    }
    k_reduce_bounds<<<parts, 256, 0, st>>>(n, pmin.p, lo_min.p, lo_max.p);
    k_reduce_bounds<<<parts, 256, 0, st>>>(n, pmax.p, hi_min.p, hi_max.p);
    k_bounds_final<<<1, kBoundsThreads, 0, st>>>(parts, lo_min.p, hi_max.p, rb.p);
  }
  float3 hb[2];
  cudaMemcpyAsync(hb, rb.p, sizeof(hb), cudaMemcpyDeviceToHost, st);
  int n_int = n - 1;
  if (n == 1) {
    if (!sc->d_nodes.alloc(ctx, 4)) {
      sc->clear_bvh();
      return set_error(ctx, "LBVH: out of device memory"), RX_ERR_CAPACITY;
    }
    k_single_leaf_root<<<1, 1, 0, st>>>(rb.p, rb.p + 1, 1, sc->d_nodes.p);
    sc->n_nodes = 1;
  } else {
    DevBuf<int> kl(ctx, n_int), kr(ctx, n_int), first(ctx, n_int), last(ctx, n_int);
    DevBuf<int> par_int(ctx, n_int), par_leaf(ctx, n), flags(ctx, n_int), icount(ctx, n_int), collapse(ctx, n_int);
    DevBuf<float3> imin(ctx, n_int), imax(ctx, n_int);
    DevBuf<float> icost(ctx, n_int);
    if (!all_ok(kl, kr, first, last, par_int, par_leaf, flags, icount, collapse, imin, imax, icost)) {
      sc->clear_bvh();
      return set_error(ctx, "LBVH: out of device memory"), RX_ERR_CAPACITY;
    }
    cudaMemsetAsync(par_int.p, 0xff, sizeof(int) * n_int, st);
    k_karras<<<grid_for(ctx, n_int), 256, 0, st>>>(n, sc->tmp_codes.p, kl.p, kr.p, first.p, last.p, par_int.p,
                                                    par_leaf.p);
    cudaMemsetAsync(flags.p, 0, sizeof(int) * n_int, st);
    k_lbvh_bottom_up<<<grid_for(ctx, n), 256, 0, st>>>(n, order.p, kl.p, kr.p, par_int.p, par_leaf.p, pmin.p,
                                                        pmax.p, imin.p, imax.p, icost.p, icount.p, collapse.p,
                                                        flags.p, max_leaf, c_t, c_i);
    int root_col = 0;
    cudaMemcpyAsync(&root_col, collapse.p, sizeof(int), cudaMemcpyDeviceToHost, st);
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
    if (root_col) {
      if (!sc->d_nodes.alloc(ctx, 4)) {
        sc->clear_bvh();
        return set_error(ctx, "LBVH: out of device memory"), RX_ERR_CAPACITY;
      }
      k_single_leaf_root<<<1, 1, 0, st>>>(rb.p, rb.p + 1, n, sc->d_nodes.p);
      sc->n_nodes = 1;
    } else {
      sc->d_nodes.alloc(ctx, (size_t)4 * n_int);
      DevBuf<int> la(ctx, n_int), lb(ctx, n_int), lv(ctx, LV_N);
      if (!all_ok(sc->d_nodes, la, lb, lv)) {
        sc->clear_bvh();
        return set_error(ctx, "LBVH: out of device memory"), RX_ERR_CAPACITY;
      }
      int base = 0, levels = 0;
      int rc = level_walk(ctx, la.p, lb.p, lv.p, &base, &levels, [&](int level, int* cur, int* nxt, int* st_lv) {
        k_lbvh_layout_level<<<level_grid(ctx, level, 1, n_int), 256, 0, st>>>(
            cur, nxt, st_lv, n_int, kl.p, kr.p, first.p, last.p, collapse.p, order.p, pmin.p, pmax.p,
            imin.p, imax.p, sc->d_nodes.p);
      });
      if (rc) {
        sc->clear_bvh();
        return rc;
      }
      sc->depth = levels;
      sc->n_nodes = base;
    }
  }
  sc->order.swap(order);
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  if (int rc = build_wide(ctx, sc)) {
    sc->clear_bvh();
    return rc;
  }
  sc->root_min = hb[0];
  sc->root_max = hb[1];
  sc->n_prims = n;
  sc->n_bvh_spheres = n_obj;
  sc->method = RX_BVH_LBVH_SAH;
  sc->exact_slab = 0;
  sc->leaf_size = max_leaf;
  return RX_OK;
}

}  // namespace rx
