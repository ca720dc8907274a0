// Scene extraction on the device.
//
// The reference flattens an IndexedMesh on the host before every render
// (scene/mesh.py:397-430 indexed_triangle_arrays, called from
// rendering/taichi/extractor.py:60-96): gather the three positions of each
// triangle, transform them by the object's world matrix in float64, take the
// vertex normals (or the normalised face normal of the untransformed
// triangle), transform them by the inverse-transpose matrix, normalise, and
// round everything to float32.  Here the caller uploads the mesh's own arrays
// (positions, index tables, per-group palette index) and one thread per
// triangle writes the float32 rows straight into the scene's triangle arrays.
//
// Arithmetic follows numpy's element-wise float64 order: a point row is
// ((x*m0 + y*m1) + z*m2) + m3, the length of a row is sqrt((x*x + y*y) + z*z)
// (np.linalg.norm along axis 1 sums left to right), numpy's cross product
// takes a1*b2 - a2*b1 etc., and the library is compiled without FMA
// contraction.  The reference multiplies by the matrix through BLAS, whose
// float64 results may differ from this order in the last bit; after the
// rounding to float32 the rows agree except when a float64 value lies within
// one float64 ulp of a float32 rounding boundary.
#include <vector>

#include "rx_internal.cuh"
#include "rx_runtime.h"

namespace rx {

struct IndexedArgs {
  int n_tris, n_pos, n_nrm, n_groups;
  const double* pos;      // (n_pos, 3)
  const int* tri_pos;     // (n_tris, 3)
  const double* nrm;      // (n_nrm, 3) or null
  const int* tri_nrm;     // (n_tris, 3) or null; a row with any index < 0 uses the face normal
  const int* tri_group;   // (n_tris,) or null (group 0)
  const int* group_mat;   // (n_groups,) palette index of each group
  double m[12];           // rows 0..2 of the world matrix
  double mw[4];           // row 3 (projective divide when |w| > 1e-12)
  double nm[9];           // rows 0..2, columns 0..2 of the normal matrix
  int has_m, has_nm;
  float *v0, *v1, *v2, *n0, *n1, *n2;  // destination rows, already offset
  int* mat;
  int* err;               // bit 1: position index, 2: normal index, 4: group index out of range
};

struct D3 {
  double x, y, z;
};

__device__ __forceinline__ D3 ldd3(const double* p, long i) { return D3{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }

__device__ __forceinline__ D3 xform_point(const IndexedArgs& A, D3 p) {
  if (!A.has_m) return p;
  const double* m = A.m;
  D3 r;
  r.x = ((p.x * m[0] + p.y * m[1]) + p.z * m[2]) + m[3];
  r.y = ((p.x * m[4] + p.y * m[5]) + p.z * m[6]) + m[7];
  r.z = ((p.x * m[8] + p.y * m[9]) + p.z * m[10]) + m[11];
  double w = ((p.x * A.mw[0] + p.y * A.mw[1]) + p.z * A.mw[2]) + A.mw[3];
  if (fabs(w) > 1e-12) {
    r.x = r.x / w;
    r.y = r.y / w;
    r.z = r.z / w;
  }
  return r;
}

__device__ __forceinline__ D3 xform_vector(const IndexedArgs& A, D3 v) {
  if (!A.has_nm) return v;
  const double* m = A.nm;
  return D3{(v.x * m[0] + v.y * m[1]) + v.z * m[2], (v.x * m[3] + v.y * m[4]) + v.z * m[5],
            (v.x * m[6] + v.y * m[7]) + v.z * m[8]};
}

__device__ __forceinline__ D3 normalize_row(D3 v) {
  double len = sqrt((v.x * v.x + v.y * v.y) + v.z * v.z);
  if (len > 1e-12) return D3{v.x / len, v.y / len, v.z / len};
  return v;
}

__device__ __forceinline__ void st3(float* p, long i, D3 v) {
  p[3 * i] = (float)v.x;
  p[3 * i + 1] = (float)v.y;
  p[3 * i + 2] = (float)v.z;
}

__global__ void __launch_bounds__(256) k_extract_indexed(IndexedArgs A) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < A.n_tris; t += (long)gridDim.x * blockDim.x) {
    int i0 = __ldg(A.tri_pos + 3 * t), i1 = __ldg(A.tri_pos + 3 * t + 1), i2 = __ldg(A.tri_pos + 3 * t + 2);
    int bad = 0;
    if ((unsigned)i0 >= (unsigned)A.n_pos || (unsigned)i1 >= (unsigned)A.n_pos || (unsigned)i2 >= (unsigned)A.n_pos) {
      bad |= 1;
      i0 = i1 = i2 = 0;
    }
    D3 p0 = ldd3(A.pos, i0), p1 = ldd3(A.pos, i1), p2 = ldd3(A.pos, i2);
    st3(A.v0, t, xform_point(A, p0));
    st3(A.v1, t, xform_point(A, p1));
    st3(A.v2, t, xform_point(A, p2));

    D3 q0, q1, q2;
    int j0 = -1, j1 = -1, j2 = -1;
    if (A.nrm && A.tri_nrm) {
      j0 = __ldg(A.tri_nrm + 3 * t);
      j1 = __ldg(A.tri_nrm + 3 * t + 1);
      j2 = __ldg(A.tri_nrm + 3 * t + 2);
    }
    if (j0 >= 0 && j1 >= 0 && j2 >= 0) {
      if (j0 >= A.n_nrm || j1 >= A.n_nrm || j2 >= A.n_nrm) {
        bad |= 2;
        j0 = j1 = j2 = 0;
      }
      q0 = ldd3(A.nrm, j0);
      q1 = ldd3(A.nrm, j1);
      q2 = ldd3(A.nrm, j2);
    } else {
      D3 a{p1.x - p0.x, p1.y - p0.y, p1.z - p0.z};
      D3 b{p2.x - p0.x, p2.y - p0.y, p2.z - p0.z};
      D3 c{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
      q0 = q1 = q2 = normalize_row(c);
    }
    st3(A.n0, t, normalize_row(xform_vector(A, q0)));
    st3(A.n1, t, normalize_row(xform_vector(A, q1)));
    st3(A.n2, t, normalize_row(xform_vector(A, q2)));

    int g = A.tri_group ? __ldg(A.tri_group + t) : 0;
    if ((unsigned)g >= (unsigned)A.n_groups) {
      bad |= 4;
      g = 0;
    }
    A.mat[t] = __ldg(A.group_mat + g);
    if (bad) atomicOr(A.err, bad);
  }
}

template <class T>
static int upload_tmp(Ctx* c, DevBuf<T>& b, const T* host, size_t n) {
  if (!b.alloc(c, n ? n : 1)) return set_error(c, "out of device memory (%zu elements)", n), RX_ERR_CAPACITY;
  if (n && host) CUDA_TRY(c, cudaMemcpyAsync(b.p, host, sizeof(T) * n, cudaMemcpyHostToDevice, c->stream));
  return RX_OK;
}

int scene_alloc_triangles(Ctx* c, Scene* s, int n) {
  size_t k = (size_t)3 * std::max(n, 1);
  if (!s->v0b.alloc(c, k) || !s->v1b.alloc(c, k) || !s->v2b.alloc(c, k) || !s->n0b.alloc(c, k) ||
      !s->n1b.alloc(c, k) || !s->n2b.alloc(c, k) || !s->tri_matb.alloc(c, std::max(n, 1)))
    return set_error(c, "alloc_triangles: out of device memory for %d triangles", n), RX_ERR_CAPACITY;
  // rows not written by a put call stay zero (degenerate, never hit)
  for (DevBuf<float>* b : {&s->v0b, &s->v1b, &s->v2b, &s->n0b, &s->n1b, &s->n2b})
    CUDA_TRY(c, cudaMemsetAsync(b->p, 0, b->bytes(), c->stream));
  CUDA_TRY(c, cudaMemsetAsync(s->tri_matb.p, 0, s->tri_matb.bytes(), c->stream));
  s->d_v0 = s->v0b.p; s->d_v1 = s->v1b.p; s->d_v2 = s->v2b.p;
  s->d_n0 = s->n0b.p; s->d_n1 = s->n1b.p; s->d_n2 = s->n2b.p;
  s->d_tri_mat = s->tri_matb.p;
  s->n_tris = n;
  s->uvb.release();
  s->clear_bvh();
  return RX_OK;
}

int scene_put_triangles(Ctx* c, Scene* s, int offset, int n, const float* const* rows, const int* mat_idx) {
  if (offset < 0 || n < 0 || (long long)offset + n > s->n_tris)
    return set_error(c, "put_triangles: rows [%d, %d) outside the %d allocated", offset, offset + n, s->n_tris),
           RX_ERR_ARG;
  if (n == 0) return RX_OK;
  float* dst[6] = {s->d_v0, s->d_v1, s->d_v2, s->d_n0, s->d_n1, s->d_n2};
  HostPiece up[7];
  for (int k = 0; k < 6; ++k)
    up[k] = {dst[k] + (size_t)3 * offset, rows[k] ? rows[k] : rows[0], sizeof(float) * 3 * (size_t)n};
  if (mat_idx) up[6] = {s->d_tri_mat + offset, mat_idx, sizeof(int) * (size_t)n};
  int rc = upload_staged(c, up, mat_idx ? 7 : 6);
  if (rc) return rc;
  if (!mat_idx) CUDA_TRY(c, cudaMemsetAsync(s->d_tri_mat + offset, 0, sizeof(int) * n, c->stream));
  ++s->version;
  return RX_OK;
}

int scene_put_indexed(Ctx* c, Scene* s, int offset, int n_tris, int n_pos, const double* positions,
                      const int* tri_pos_idx, int n_nrm, const double* normals, const int* tri_nrm_idx,
                      const double* matrix, const double* normal_matrix, const int* tri_group_idx, int n_groups,
                      const int* group_mat) {
  if (offset < 0 || n_tris < 0 || (long long)offset + n_tris > s->n_tris)
    return set_error(c, "put_indexed: rows [%d, %d) outside the %d allocated", offset, offset + n_tris, s->n_tris),
           RX_ERR_ARG;
  if (n_pos < 0 || n_nrm < 0 || n_groups < 1 || !group_mat || (n_tris > 0 && (!positions || !tri_pos_idx)))
    return set_error(c, "put_indexed: bad arguments"), RX_ERR_ARG;
  if (n_tris == 0) return RX_OK;
  IndexedArgs A;
  std::memset(&A, 0, sizeof(A));
  A.n_tris = n_tris;
  A.n_pos = n_pos;
  A.n_nrm = (normals && tri_nrm_idx) ? n_nrm : 0;
  A.n_groups = n_groups;
  if (matrix) {
    for (int i = 0; i < 12; ++i) A.m[i] = matrix[i];
    for (int i = 0; i < 4; ++i) A.mw[i] = matrix[12 + i];
    A.has_m = 1;
  }
  if (normal_matrix) {
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 3; ++k) A.nm[3 * r + k] = normal_matrix[4 * r + k];
    A.has_nm = 1;
  }
  DevBuf<double> d_pos, d_nrm;
  DevBuf<int> d_tri_pos, d_tri_nrm, d_group, d_group_mat, d_err;
  const bool has_n = A.n_nrm > 0;
  d_pos.alloc(c, (size_t)3 * std::max(n_pos, 1));
  d_tri_pos.alloc(c, (size_t)3 * n_tris);
  d_group_mat.alloc(c, (size_t)n_groups);
  d_err.alloc(c, 1);
  if (has_n) {
    d_nrm.alloc(c, (size_t)3 * n_nrm);
    d_tri_nrm.alloc(c, (size_t)3 * n_tris);
  }
  if (tri_group_idx) d_group.alloc(c, (size_t)n_tris);
  if (!all_ok(d_pos, d_tri_pos, d_group_mat, d_err, d_nrm, d_tri_nrm, d_group))
    return set_error(c, "put_indexed: out of device memory for %d triangles", n_tris), RX_ERR_CAPACITY;
  // one staged upload of every host array (about 52 B per triangle with
  // normals and groups, plus 24 B per position and normal)
  HostPiece up[6];
  int nu = 0;
  up[nu++] = {d_pos.p, positions, sizeof(double) * 3 * (size_t)n_pos};
  up[nu++] = {d_tri_pos.p, tri_pos_idx, sizeof(int) * 3 * (size_t)n_tris};
  up[nu++] = {d_group_mat.p, group_mat, sizeof(int) * (size_t)n_groups};
  if (has_n) {
    up[nu++] = {d_nrm.p, normals, sizeof(double) * 3 * (size_t)n_nrm};
    up[nu++] = {d_tri_nrm.p, tri_nrm_idx, sizeof(int) * 3 * (size_t)n_tris};
    A.nrm = d_nrm.p;
    A.tri_nrm = d_tri_nrm.p;
  }
  if (tri_group_idx) {
    up[nu++] = {d_group.p, tri_group_idx, sizeof(int) * (size_t)n_tris};
    A.tri_group = d_group.p;
  }
  int rc = upload_staged(c, up, nu);
  if (rc) return rc;
  A.pos = d_pos.p;
  A.tri_pos = d_tri_pos.p;
  A.group_mat = d_group_mat.p;
  A.v0 = s->d_v0 + (size_t)3 * offset;
  A.v1 = s->d_v1 + (size_t)3 * offset;
  A.v2 = s->d_v2 + (size_t)3 * offset;
  A.n0 = s->d_n0 + (size_t)3 * offset;
  A.n1 = s->d_n1 + (size_t)3 * offset;
  A.n2 = s->d_n2 + (size_t)3 * offset;
  A.mat = s->d_tri_mat + offset;
  A.err = d_err.p;
  CUDA_TRY(c, cudaMemsetAsync(d_err.p, 0, sizeof(int), c->stream));
  int blocks = (int)std::min<long long>((n_tris + 255) / 256, (long long)c->num_sms * 8);
  k_extract_indexed<<<blocks, 256, 0, c->stream>>>(A);
  CUDA_TRY(c, cudaGetLastError());
  int herr = 0;
  CUDA_TRY(c, cudaMemcpyAsync(&herr, d_err.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  ++s->version;
  if (herr & 1) return set_error(c, "put_indexed: a position index is outside [0, %d)", n_pos), RX_ERR_ARG;
  if (herr & 2) return set_error(c, "put_indexed: a normal index is outside [0, %d)", n_nrm), RX_ERR_ARG;
  if (herr & 4) return set_error(c, "put_indexed: a group index is outside [0, %d)", n_groups), RX_ERR_ARG;
  return RX_OK;
}

__global__ void k_pack_uvs(int n, const float* __restrict__ uv0, const float* __restrict__ uv1,
                           const float* __restrict__ uv2, const int* __restrict__ has_uv, float4* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    out[2 * (size_t)i] = make_float4(uv0[2 * i], uv0[2 * i + 1], uv1[2 * i], uv1[2 * i + 1]);
    out[2 * (size_t)i + 1] = make_float4(uv2[2 * i], uv2[2 * i + 1], __int_as_float(has_uv ? (has_uv[i] != 0) : 1),
                                         0.0f);
  }
}

int scene_put_uvs(Ctx* c, Scene* s, int offset, int n, const float* uv0, const float* uv1, const float* uv2,
                  const int* has_uv) {
  if (offset < 0 || n < 0 || (long long)offset + n > s->n_tris)
    return set_error(c, "put_uvs: rows [%d, %d) outside the %d present", offset, offset + n, s->n_tris), RX_ERR_ARG;
  if (n > 0 && (!uv0 || !uv1 || !uv2)) return set_error(c, "put_uvs: bad arguments"), RX_ERR_ARG;
  if (!s->uvb.p) {
    // rows without uvs read has_uv = 0
    if (!s->uvb.alloc(c, 2 * (size_t)std::max(s->n_tris, 1)))
      return set_error(c, "put_uvs: out of device memory"), RX_ERR_CAPACITY;
    CUDA_TRY(c, cudaMemsetAsync(s->uvb.p, 0, s->uvb.bytes(), c->stream));
  }
  if (n == 0) return RX_OK;
  DevBuf<float> d0(c, (size_t)2 * n), d1(c, (size_t)2 * n), d2(c, (size_t)2 * n);
  DevBuf<int> dh;
  if (has_uv) dh.alloc(c, (size_t)n);
  if (!all_ok(d0, d1, d2, dh)) return set_error(c, "put_uvs: out of device memory"), RX_ERR_CAPACITY;
  HostPiece up[4] = {{d0.p, uv0, sizeof(float) * 2 * (size_t)n},
                     {d1.p, uv1, sizeof(float) * 2 * (size_t)n},
                     {d2.p, uv2, sizeof(float) * 2 * (size_t)n},
                     {dh.p, has_uv, sizeof(int) * (size_t)n}};
  int rc = upload_staged(c, up, has_uv ? 4 : 3);
  if (rc) return rc;
  int blocks = (int)std::min<long long>((n + 255) / 256, (long long)c->num_sms * 8);
  k_pack_uvs<<<blocks, 256, 0, c->stream>>>(n, d0.p, d1.p, d2.p, has_uv ? dh.p : nullptr, s->uvb.p + 2 * (size_t)offset);
  CUDA_TRY(c, cudaGetLastError());
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  ++s->version;
  return RX_OK;
}

int scene_set_textures(Ctx* c, Scene* s, int n, const int* width, const int* height, const int* flip_v,
                       const unsigned char* texels) {
  if (n < 0 || (n > 0 && (!width || !height))) return set_error(c, "set_textures: bad arguments"), RX_ERR_ARG;
  std::vector<TexInfo> info(std::max(n, 1));
  long long total = 0;
  for (int i = 0; i < n; ++i) {
    if (width[i] < 0 || height[i] < 0 || width[i] > (1 << 16) || height[i] > (1 << 16))
      return set_error(c, "set_textures: texture %d has size %dx%d", i, width[i], height[i]), RX_ERR_ARG;
    info[i].offset = total;
    info[i].w = width[i];
    info[i].h = height[i];
    info[i].flip_v = flip_v ? (flip_v[i] != 0) : 0;
    info[i].pad = 0;
    total += 3LL * width[i] * height[i];
  }
  if (total > 0 && !texels) return set_error(c, "set_textures: texels is NULL"), RX_ERR_ARG;
  if (!s->d_tex.alloc(c, info.size()) || !s->d_texels.alloc(c, (size_t)std::max<long long>(total, 1)))
    return set_error(c, "set_textures: out of device memory for %lld texel bytes", total), RX_ERR_CAPACITY;
  CUDA_TRY(c, cudaMemcpyAsync(s->d_tex.p, info.data(), sizeof(TexInfo) * info.size(), cudaMemcpyHostToDevice,
                              c->stream));
  if (total > 0)
    CUDA_TRY(c, cudaMemcpyAsync(s->d_texels.p, texels, (size_t)total, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  s->n_tex = n;
  ++s->version;
  return RX_OK;
}

size_t scene_bytes(const Scene* s) {
  return s->v0b.bytes() + s->v1b.bytes() + s->v2b.bytes() + s->n0b.bytes() + s->n1b.bytes() + s->n2b.bytes() +
         s->tri_matb.bytes() + s->uvb.bytes() + s->d_tex.bytes() + s->d_texels.bytes() + s->mat_a.bytes() +
         s->mat_b.bytes() + s->d_objs.bytes() + s->d_lights.bytes() + s->d_alias_prob.bytes() +
         s->d_alias_idx.bytes() + s->d_nodes.bytes() + s->d_prims.bytes() + s->d_shade.bytes() +
         s->ref_left.bytes() + s->ref_right.bytes() + s->ref_start.bytes() + s->ref_count.bytes() +
         s->order.bytes() + s->ref_min.bytes() + s->ref_max.bytes() + s->tmp_codes.bytes();
}

int scene_get_triangles(Ctx* c, Scene* s, int offset, int n, float* const* rows, int* mat_idx) {
  if (offset < 0 || n < 0 || (long long)offset + n > s->n_tris)
    return set_error(c, "get_triangles: rows [%d, %d) outside the %d present", offset, offset + n, s->n_tris),
           RX_ERR_ARG;
  if (n == 0) return RX_OK;
  const float* src[6] = {s->d_v0, s->d_v1, s->d_v2, s->d_n0, s->d_n1, s->d_n2};
  int rc;
  for (int k = 0; k < 6; ++k)
    if (rows[k] && (rc = download_staged(c, rows[k], src[k] + (size_t)3 * offset, sizeof(float) * 3 * (size_t)n)))
      return rc;
  if (mat_idx && (rc = download_staged(c, mat_idx, s->d_tri_mat + offset, sizeof(int) * (size_t)n))) return rc;
  return RX_OK;
}

}  // namespace rx
