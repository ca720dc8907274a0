// Wavefront OBJ text -> indexed mesh arrays, parsed on the device.
//
// Semantics follow OBJReader._parse_indexed (scene/io/obj_reader.py:345-441):
// lines split as Python's universal-newline text iteration does ("\n",
// "\r\n", "\r"), tokens as str.split() does, `v`/`vn` keep their first three
// numbers and `vt` its first two (float64), faces are fan-triangulated
// ((v0, vi, vi+1)), an index i maps to i - 1 when positive and to
// count + i otherwise (count = records of that kind read so far), a missing
// or empty uv / normal field gives -1, and every triangle carries the group
// id of the `usemtl` in force ("default" = 0 before the first one).
//
// Pipeline (one handle per text):
//   1. line starts: bytes are counted in 16 KB blocks, scanned, scattered;
//   2. classify, one thread per line: the line's kind, its contribution to
//      the per-kind counts, and whether the host must read it.  Numbers
//      are converted on the device only when that is exact: a decimal with
//      at most 19 significant digits whose significand w <= 2^53 and whose
//      decimal exponent |q| <= 22 is w * 10^q or w / 10^-q in one IEEE
//      operation on exactly representable operands (Clinger's fast path),
//      so it equals Python's correctly rounded float(); indices are 1-9
//      digit integers.  Anything else (more digits, inf / nan, underscores,
//      malformed tokens, non-ASCII bytes) is listed for the host, as are
//      usemtl, mtllib, o, g and unrecognised lines;
//   3. exclusive scans of the per-line counts (positions, normals, uvs,
//      triangles, usemtl lines, face lines) give every line its output slots;
//   4. emit, one thread per line, writes the arrays; the host then fills in
//      the values of the lines it was given.
#include "rx_internal.cuh"
#include "rx_runtime.h"

namespace rx {

enum ObjKind { K_SKIP = 0, K_V, K_VN, K_VT, K_F, K_USEMTL, K_MTLLIB, K_O, K_G, K_S, K_OTHER };
enum { F_HOST = 1, F_NONASCII = 2 };
enum { C_V = 0, C_VN, C_VT, C_TRI, C_MTL, C_FACE, C_LIST, C_N };

constexpr int kLineBlock = 16384;  // bytes per block of the line-start pass
constexpr int kLineThreads = 256;  // 64 bytes per thread
constexpr int kScanItems = 4096;   // items per block of the scans (1024 threads x 4)

// ------------------------------------------------------------------ scans
__device__ __forceinline__ int warp_incl_scan(int v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// exclusive scan of one value per thread across the block; *total = sum
template <int NT>
__device__ __forceinline__ int block_excl_scan(int v, int* total) {
  __shared__ int warp_sum[NT / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int inc = warp_incl_scan(v);
  if (lane == 31) warp_sum[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    int s = lane < NT / 32 ? warp_sum[lane] : 0;
    s = warp_incl_scan(s);
    if (lane < NT / 32) warp_sum[lane] = s;
  }
  __syncthreads();
  const int base = warp ? warp_sum[warp - 1] : 0;
  *total = warp_sum[NT / 32 - 1];
  __syncthreads();  // warp_sum is reused by the next call
  return base + inc - v;
}

__global__ void __launch_bounds__(1024) k_scan_reduce(const int* __restrict__ a, long long m, int* __restrict__ sums) {
  const long long base = (long long)blockIdx.x * kScanItems + threadIdx.x * 4;
  int s = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (base + k < m) s += a[base + k];
  int tot;
  block_excl_scan<1024>(s, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// one block: exclusive scan of nb block sums in place, total in sums[nb]
__global__ void __launch_bounds__(1024) k_scan_top(int* __restrict__ sums, int nb) {
  const int per = (nb + 1023) / 1024;
  const int b0 = threadIdx.x * per;
  int s = 0;
  for (int k = 0; k < per; ++k)
    if (b0 + k < nb) s += sums[b0 + k];
  int tot;
  int run = block_excl_scan<1024>(s, &tot);
  for (int k = 0; k < per; ++k)
    if (b0 + k < nb) {
      int v = sums[b0 + k];
      sums[b0 + k] = run;
      run += v;
    }
  if (threadIdx.x == 0) sums[nb] = tot;
}

__global__ void __launch_bounds__(1024) k_scan_down(int* __restrict__ a, long long m, const int* __restrict__ sums) {
  const long long base = (long long)blockIdx.x * kScanItems + threadIdx.x * 4;
  int v[4], s = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = base + k < m ? a[base + k] : 0;
    s += v[k];
  }
  int tot;
  int run = block_excl_scan<1024>(s, &tot) + sums[blockIdx.x];
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (base + k < m) {
      a[base + k] = run;
      run += v[k];
    }
}

// exclusive scan of a[0..m) in place; the total lands in total_dev[0]
static int excl_scan(Ctx* ctx, int* a, long long m, int* total_dev) {
  cudaStream_t st = ctx->stream;
  const long long nb = (m + kScanItems - 1) / kScanItems;
  if (nb > (1LL << 24)) return set_error(ctx, "obj: too many lines"), RX_ERR_CAPACITY;
  DevBuf<int> sums(ctx, (size_t)std::max<long long>(nb, 1) + 1);
  if (!sums.p) return set_error(ctx, "obj: out of device memory"), RX_ERR_CAPACITY;
  if (nb > 0) {
    k_scan_reduce<<<(unsigned)nb, 1024, 0, st>>>(a, m, sums.p);
    k_scan_top<<<1, 1024, 0, st>>>(sums.p, (int)nb);
    k_scan_down<<<(unsigned)nb, 1024, 0, st>>>(a, m, sums.p);
    CUDA_TRY(ctx, cudaMemcpyAsync(total_dev, sums.p + nb, sizeof(int), cudaMemcpyDeviceToDevice, st));
  } else {
    CUDA_TRY(ctx, cudaMemsetAsync(total_dev, 0, sizeof(int), st));
  }
  CUDA_TRY(ctx, cudaGetLastError());
  return RX_OK;
}

// ------------------------------------------------------------ line starts
// A line starts at byte 0 and after "\n", or after an "\r" that is not
// followed by "\n".  Thread t of block b looks at bytes [b * 16384 + t * 64,
// +64); the text buffer is zero-padded to whole blocks, starts are only
// counted below n.
__device__ __forceinline__ int count_starts(const uint8_t* __restrict__ t, long long n, long long b0,
                                            uint64_t* mask) {
  uint4 q[4];
  const uint4* src = reinterpret_cast<const uint4*>(t + b0);
#pragma unroll
  for (int k = 0; k < 4; ++k) q[k] = src[k];
  const uint8_t* c = reinterpret_cast<const uint8_t*>(q);
  uint8_t prev = b0 > 0 ? t[b0 - 1] : '\n';
  uint64_t m = 0;
#pragma unroll
  for (int j = 0; j < 64; ++j) {
    const bool s = prev == '\n' || (prev == '\r' && c[j] != '\n');
    if (s && b0 + j < n) m |= 1ull << j;
    prev = c[j];
  }
  *mask = m;
  return __popcll(m);
}

__global__ void __launch_bounds__(kLineThreads) k_line_count(const uint8_t* __restrict__ t, long long n,
                                                             int* __restrict__ blk) {
  uint64_t m;
  const long long b0 = (long long)blockIdx.x * kLineBlock + threadIdx.x * 64;
  int c = count_starts(t, n, b0, &m);
  int tot;
  block_excl_scan<kLineThreads>(c, &tot);
  if (threadIdx.x == 0) blk[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kLineThreads) k_line_write(const uint8_t* __restrict__ t, long long n,
                                                             const int* __restrict__ blk_off,
                                                             long long* __restrict__ starts) {
  uint64_t m;
  const long long b0 = (long long)blockIdx.x * kLineBlock + threadIdx.x * 64;
  int c = count_starts(t, n, b0, &m);
  int tot;
  int o = block_excl_scan<kLineThreads>(c, &tot) + blk_off[blockIdx.x];
  while (m) {
    const int j = __ffsll((long long)m) - 1;
    starts[o++] = b0 + j;
    m &= m - 1;
  }
}

// ------------------------------------------------------------- tokenizer
// ASCII whitespace of str.split(): \t \n \v \f \r, \x1c-\x1f, space
__device__ __forceinline__ bool is_ws(uint8_t c) { return c == ' ' || (c >= 9 && c <= 13) || (c >= 28 && c <= 31); }

__device__ __forceinline__ bool next_token(const uint8_t*& p, const uint8_t* e, const uint8_t*& ts,
                                           const uint8_t*& te) {
  while (p < e && is_ws(*p)) ++p;
  if (p >= e) return false;
  ts = p;
  while (p < e && !is_ws(*p)) ++p;
  te = p;
  return true;
}

__device__ __forceinline__ bool tok_is(const uint8_t* ts, const uint8_t* te, const char* s) {
  const uint8_t* p = ts;
  for (; *s; ++s, ++p)
    if (p >= te || *p != (uint8_t)*s) return false;
  return p == te;
}

// powers of ten that doubles hold exactly
__constant__ double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11,
                                  1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};

// Python float() of a decimal token when it is exact in one IEEE operation
// (Clinger's fast path); false for every other token
__device__ bool parse_f64(const uint8_t* p, const uint8_t* e, double* out) {
  const double* p10 = kPow10;
  bool neg = false;
  if (p < e && (*p == '+' || *p == '-')) neg = *p++ == '-';
  uint64_t w = 0;
  int nd = 0, q = 0;
  bool any = false;
  while (p < e && *p >= '0' && *p <= '9') {
    any = true;
    if (w || *p != '0') {
      if (++nd > 19) return false;
      w = w * 10 + (*p - '0');
    }
    ++p;
  }
  if (p < e && *p == '.') {
    ++p;
    while (p < e && *p >= '0' && *p <= '9') {
      any = true;
      if (w || *p != '0') {
        if (++nd > 19) return false;
        w = w * 10 + (*p - '0');
      }
      --q;
      ++p;
    }
  }
  if (!any) return false;
  if (p < e && (*p == 'e' || *p == 'E')) {
    ++p;
    bool eneg = false;
    if (p < e && (*p == '+' || *p == '-')) eneg = *p++ == '-';
    if (p >= e || *p < '0' || *p > '9') return false;
    int x = 0;
    while (p < e && *p >= '0' && *p <= '9') {
      if (x < 100000) x = x * 10 + (*p - '0');
      ++p;
    }
    q += eneg ? -x : x;
  }
  if (p != e) return false;
  if (w == 0) {
    *out = neg ? -0.0 : 0.0;
    return true;
  }
  if (w > (1ull << 53) || q < -22 || q > 22) return false;
  const double v = q >= 0 ? (double)w * p10[q] : (double)w / p10[-q];
  *out = neg ? -v : v;
  return true;
}

// Python int() of a short decimal token ([+-]?[0-9]{1,9})
__device__ __forceinline__ bool parse_i32(const uint8_t* p, const uint8_t* e, int* out) {
  bool neg = false;
  if (p < e && (*p == '+' || *p == '-')) neg = *p++ == '-';
  if (p >= e || e - p > 9) return false;
  int v = 0;
  for (; p < e; ++p) {
    if (*p < '0' || *p > '9') return false;
    v = v * 10 + (*p - '0');
  }
  *out = neg ? -v : v;
  return true;
}

__device__ __forceinline__ int obj_index(int i, int count) { return i > 0 ? i - 1 : count + i; }

// one face vertex "v[/vt[/vn]]" (further fields ignored); false if a field
// the reference converts with int() is not a short decimal
__device__ __forceinline__ bool parse_face_vertex(const uint8_t* ts, const uint8_t* te, int lv, int lvt, int lvn,
                                                  int* vi, int* ti, int* ni) {
  const uint8_t* f[4];
  const uint8_t* fe[3];
  int nf = 0;
  f[0] = ts;
  for (const uint8_t* p = ts; p < te && nf < 3; ++p)
    if (*p == '/') {
      fe[nf] = p;
      f[++nf] = p + 1;
    }
  if (nf < 3) fe[nf] = te;
  const int nfields = nf + 1 > 3 ? 3 : nf + 1;
  int v;
  if (!parse_i32(f[0], fe[0], &v)) return false;
  *vi = obj_index(v, lv);
  *ti = -1;
  *ni = -1;
  if (nfields > 1 && fe[1] > f[1]) {
    if (!parse_i32(f[1], fe[1], &v)) return false;
    *ti = obj_index(v, lvt);
  }
  if (nfields > 2 && fe[2] > f[2]) {
    if (!parse_i32(f[2], fe[2], &v)) return false;
    *ni = obj_index(v, lvn);
  }
  return true;
}

// ------------------------------------------------------------- classify
__global__ void k_classify(const uint8_t* __restrict__ t, const long long* __restrict__ starts, int lines,
                           uint8_t* __restrict__ kind, uint8_t* __restrict__ flags, int* __restrict__ cnt) {
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < lines; l += gridDim.x * blockDim.x) {
    const uint8_t* s = t + starts[l];
    const uint8_t* e = t + starts[l + 1];
    int fl = 0;
    for (const uint8_t* p = s; p < e; ++p)
      if (*p >= 0x80) {
        fl = F_HOST | F_NONASCII;
        break;
      }
    int k = K_SKIP, ntri = 0;
    const uint8_t *p = s, *ts, *te;
    if (next_token(p, e, ts, te) && *ts != '#') {
      if (tok_is(ts, te, "v")) k = K_V;
      else if (tok_is(ts, te, "vn")) k = K_VN;
      else if (tok_is(ts, te, "vt")) k = K_VT;
      else if (tok_is(ts, te, "f")) k = K_F;
      else if (tok_is(ts, te, "usemtl")) k = K_USEMTL;
      else if (tok_is(ts, te, "mtllib")) k = K_MTLLIB;
      else if (tok_is(ts, te, "o")) k = K_O;
      else if (tok_is(ts, te, "g")) k = K_G;
      else if (tok_is(ts, te, "s")) k = K_S;
      else k = K_OTHER;
      if (k == K_V || k == K_VN || k == K_VT) {
        const int need = k == K_VT ? 2 : 3;
        for (int j = 0; j < need; ++j) {
          double v;
          if (!next_token(p, e, ts, te) || !parse_f64(ts, te, &v)) {
            fl |= F_HOST;
            break;
          }
        }
      } else if (k == K_F) {
        int nv = 0;
        while (next_token(p, e, ts, te)) {
          int a, b, c;
          if (!parse_face_vertex(ts, te, 0, 0, 0, &a, &b, &c)) fl |= F_HOST;
          ++nv;
        }
        ntri = nv > 2 ? nv - 2 : 0;
      }
    }
    kind[l] = (uint8_t)k;
    flags[l] = (uint8_t)fl;
    cnt[C_V * (long long)lines + l] = k == K_V;
    cnt[C_VN * (long long)lines + l] = k == K_VN;
    cnt[C_VT * (long long)lines + l] = k == K_VT;
    cnt[C_TRI * (long long)lines + l] = ntri;
    cnt[C_MTL * (long long)lines + l] = k == K_USEMTL;
    cnt[C_FACE * (long long)lines + l] = k == K_F;
    cnt[C_LIST * (long long)lines + l] =
        fl != 0 || k == K_USEMTL || k == K_MTLLIB || k == K_O || k == K_G || k == K_OTHER;
  }
}

// compact the listed lines (exclusive prefix of C_LIST already taken)
__global__ void k_list(const uint8_t* __restrict__ kind, const uint8_t* __restrict__ flags,
                       const int* __restrict__ cnt, int lines, int* __restrict__ listed) {
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < lines; l += gridDim.x * blockDim.x) {
    const int k = kind[l];
    if (flags[l] || k == K_USEMTL || k == K_MTLLIB || k == K_O || k == K_G || k == K_OTHER)
      listed[cnt[C_LIST * (long long)lines + l]] = l;
  }
}

// host corrections of listed lines (kind and triangle count as Python splits them)
__global__ void k_correct(int n, const int* __restrict__ line, const int* __restrict__ k_new,
                          const int* __restrict__ tri_new, uint8_t* __restrict__ kind, int* __restrict__ cnt,
                          int lines) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int l = line[i], k = k_new[i];
  kind[l] = (uint8_t)k;
  cnt[C_V * (long long)lines + l] = k == K_V;
  cnt[C_VN * (long long)lines + l] = k == K_VN;
  cnt[C_VT * (long long)lines + l] = k == K_VT;
  cnt[C_TRI * (long long)lines + l] = k == K_F ? tri_new[i] : 0;
  cnt[C_MTL * (long long)lines + l] = k == K_USEMTL;
  cnt[C_FACE * (long long)lines + l] = k == K_F;
}

__global__ void k_gather_prefix(int n, const int* __restrict__ listed, const int* __restrict__ cnt, int lines,
                                int* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int l = listed[i];
  for (int c = 0; c < C_LIST; ++c) out[(long long)i * C_LIST + c] = cnt[c * (long long)lines + l];
}

__global__ void k_gather_lines(int n, const int* __restrict__ listed, const long long* __restrict__ starts,
                               const uint8_t* __restrict__ kind, const uint8_t* __restrict__ flags,
                               long long* __restrict__ off, int* __restrict__ len, int* __restrict__ k_out,
                               int* __restrict__ f_out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int l = listed[i];
  off[i] = starts[l];
  len[i] = (int)(starts[l + 1] - starts[l]);
  k_out[i] = kind[l];
  f_out[i] = flags[l];
}

// ----------------------------------------------------------------- emit
__global__ void k_emit(const uint8_t* __restrict__ t, const long long* __restrict__ starts, int lines,
                       const uint8_t* __restrict__ kind, const uint8_t* __restrict__ flags,
                       const int* __restrict__ cnt, const int* __restrict__ mtl_gid, double* __restrict__ pos,
                       double* __restrict__ nrm, double* __restrict__ uv, int* __restrict__ tri_pos,
                       int* __restrict__ tri_nrm, int* __restrict__ tri_uv, int* __restrict__ tri_grp) {
  for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < lines; l += gridDim.x * blockDim.x) {
    const int k = kind[l];
    if (flags[l] || (k != K_V && k != K_VN && k != K_VT && k != K_F)) continue;
    const uint8_t *p = t + starts[l], *e = t + starts[l + 1], *ts, *te;
    next_token(p, e, ts, te);  // the keyword
    if (k == K_V || k == K_VN || k == K_VT) {
      const int need = k == K_VT ? 2 : 3;
      double* dst = k == K_V ? pos + 3LL * cnt[C_V * (long long)lines + l]
                  : k == K_VN ? nrm + 3LL * cnt[C_VN * (long long)lines + l]
                              : uv + 2LL * cnt[C_VT * (long long)lines + l];
      for (int j = 0; j < need; ++j) {
        next_token(p, e, ts, te);
        parse_f64(ts, te, dst + j);
      }
      continue;
    }
    const int lv = cnt[C_V * (long long)lines + l], lvn = cnt[C_VN * (long long)lines + l];
    const int lvt = cnt[C_VT * (long long)lines + l];
    long long tri = cnt[C_TRI * (long long)lines + l];
    const int m = cnt[C_MTL * (long long)lines + l];
    const int gid = m ? mtl_gid[m - 1] : 0;
    int v0 = 0, t0 = 0, n0 = 0, v1 = 0, t1 = 0, n1 = 0, nv = 0;
    while (next_token(p, e, ts, te)) {
      int v, tt, nn;
      parse_face_vertex(ts, te, lv, lvt, lvn, &v, &tt, &nn);
      if (nv == 0) {
        v0 = v, t0 = tt, n0 = nn;
      } else if (nv >= 2) {
        tri_pos[3 * tri] = v0, tri_pos[3 * tri + 1] = v1, tri_pos[3 * tri + 2] = v;
        tri_uv[3 * tri] = t0, tri_uv[3 * tri + 1] = t1, tri_uv[3 * tri + 2] = tt;
        tri_nrm[3 * tri] = n0, tri_nrm[3 * tri + 1] = n1, tri_nrm[3 * tri + 2] = nn;
        tri_grp[tri] = gid;
        ++tri;
      }
      v1 = v, t1 = tt, n1 = nn;
      ++nv;
    }
  }
}

// ------------------------------------------------------------- handle
struct ObjParse {
  Ctx* ctx = nullptr;
  long long n = 0;
  int lines = 0, n_listed = 0;
  int tot[C_N] = {0, 0, 0, 0, 0, 0, 0};
  bool scanned = false;
  DevBuf<uint8_t> text;
  DevBuf<long long> starts;  // lines + 1
  DevBuf<uint8_t> kind, flags;
  DevBuf<int> cnt;  // C_N x lines
  DevBuf<int> totals;
  DevBuf<int> listed;
  // CUDA-event pairs around each stretch of device work (no host waits or
  // copies of the text / results inside), summed by obj_device_ms
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> spans;
  void span_begin() {
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess) return;
    if (cudaEventCreate(&b) != cudaSuccess) {
      cudaEventDestroy(a);
      return;
    }
    cudaEventRecord(a, ctx->stream);
    spans.push_back({a, b});
  }
  void span_end() {
    if (!spans.empty()) cudaEventRecord(spans.back().second, ctx->stream);
  }
  ~ObjParse() {
    for (auto& s : spans) {
      cudaEventDestroy(s.first);
      cudaEventDestroy(s.second);
    }
  }
};

static int grid_for(Ctx* ctx, long long n, int per_block = 256) {
  return (int)std::max<long long>(1, std::min<long long>((n + per_block - 1) / per_block, (long long)ctx->num_sms * 16));
}

int obj_begin(Ctx* ctx, const void* text, long long n, ObjParse** out) {
  cudaStream_t st = ctx->stream;
  auto* o = new ObjParse();
  o->ctx = ctx;
  o->n = n;
  const long long nb = std::max<long long>(1, (n + kLineBlock - 1) / kLineBlock);
  const long long padded = nb * kLineBlock;
  auto fail = [&](int rc) {
    delete o;
    return rc;
  };
  if (!o->text.alloc(ctx, (size_t)padded) || !o->totals.alloc(ctx, C_N))
    return fail((set_error(ctx, "obj: out of device memory for %lld bytes", n), RX_ERR_CAPACITY));
  if (cudaMemsetAsync(o->text.p + n, 0, (size_t)(padded - n), st) != cudaSuccess ||
      (n > 0 && cudaMemcpyAsync(o->text.p, text, (size_t)n, cudaMemcpyHostToDevice, st) != cudaSuccess))
    return fail((set_error(ctx, "obj: text upload failed"), RX_ERR_CUDA));
  // line starts
  DevBuf<int> blk(ctx, (size_t)nb + 1);
  if (!blk.p) return fail((set_error(ctx, "obj: out of device memory"), RX_ERR_CAPACITY));
  o->span_begin();
  k_line_count<<<(unsigned)nb, kLineThreads, 0, st>>>(o->text.p, n, blk.p);
  int rc = excl_scan(ctx, blk.p, nb, blk.p + nb);
  o->span_end();
  if (rc) return fail(rc);
  int lines = 0;
  if (cudaMemcpyAsync(&lines, blk.p + nb, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return fail((set_error(ctx, "obj: %s", cudaGetErrorString(cudaGetLastError())), RX_ERR_CUDA));
  o->lines = lines;
  if (!o->starts.alloc(ctx, (size_t)lines + 1) || !o->kind.alloc(ctx, std::max(lines, 1)) ||
      !o->flags.alloc(ctx, std::max(lines, 1)) || !o->cnt.alloc(ctx, (size_t)C_N * std::max(lines, 1)))
    return fail((set_error(ctx, "obj: out of device memory for %d lines", lines), RX_ERR_CAPACITY));
  if (cudaMemcpyAsync(o->starts.p + lines, &o->n, sizeof(long long), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return fail((set_error(ctx, "obj: upload failed"), RX_ERR_CUDA));
  o->span_begin();
  k_line_write<<<(unsigned)nb, kLineThreads, 0, st>>>(o->text.p, n, blk.p, o->starts.p);
  if (lines > 0) {
    k_classify<<<grid_for(ctx, lines), 256, 0, st>>>(o->text.p, o->starts.p, lines, o->kind.p, o->flags.p, o->cnt.p);
    rc = excl_scan(ctx, o->cnt.p + (long long)C_LIST * lines, lines, o->totals.p + C_LIST);
    o->span_end();
    if (rc) return fail(rc);
    int nl = 0;
    if (cudaMemcpyAsync(&nl, o->totals.p + C_LIST, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return fail((set_error(ctx, "obj: %s", cudaGetErrorString(cudaGetLastError())), RX_ERR_CUDA));
    o->n_listed = nl;
    if (!o->listed.alloc(ctx, std::max(nl, 1))) return fail((set_error(ctx, "obj: out of device memory"), RX_ERR_CAPACITY));
    o->span_begin();
    k_list<<<grid_for(ctx, lines), 256, 0, st>>>(o->kind.p, o->flags.p, o->cnt.p, lines, o->listed.p);
    o->span_end();
  } else {
    o->span_end();
  }
  if (cudaGetLastError() != cudaSuccess) return fail((set_error(ctx, "obj: kernel launch failed"), RX_ERR_CUDA));
  *out = o;
  return RX_OK;
}

int obj_listed(ObjParse* o, long long* off, int* len, int* kind, int* flags, int* line) {
  Ctx* ctx = o->ctx;
  cudaStream_t st = ctx->stream;
  const int n = o->n_listed;
  if (n == 0) return RX_OK;
  DevBuf<long long> d_off(ctx, n);
  DevBuf<int> d_len(ctx, n), d_kind(ctx, n), d_flags(ctx, n);
  if (!d_off.p || !d_len.p || !d_kind.p || !d_flags.p) return set_error(ctx, "obj: out of device memory"), RX_ERR_CAPACITY;
  k_gather_lines<<<(n + 255) / 256, 256, 0, st>>>(n, o->listed.p, o->starts.p, o->kind.p, o->flags.p, d_off.p,
                                                  d_len.p, d_kind.p, d_flags.p);
  CUDA_TRY(ctx, cudaMemcpyAsync(off, d_off.p, sizeof(long long) * n, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaMemcpyAsync(len, d_len.p, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaMemcpyAsync(kind, d_kind.p, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaMemcpyAsync(flags, d_flags.p, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  if (line) CUDA_TRY(ctx, cudaMemcpyAsync(line, o->listed.p, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return RX_OK;
}

int obj_correct(ObjParse* o, int n, const int* pos, const int* kind, const int* ntri) {
  Ctx* ctx = o->ctx;
  cudaStream_t st = ctx->stream;
  if (o->scanned) return set_error(ctx, "obj_correct: the counts are already scanned"), RX_ERR_ARG;
  if (n <= 0) return RX_OK;
  std::vector<int> line(n);
  std::vector<int> all(o->n_listed);
  if (o->n_listed) {
    CUDA_TRY(ctx, cudaMemcpyAsync(all.data(), o->listed.p, sizeof(int) * o->n_listed, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
  }
  for (int i = 0; i < n; ++i) {
    if (pos[i] < 0 || pos[i] >= o->n_listed) return set_error(ctx, "obj_correct: listed position %d out of range", pos[i]), RX_ERR_ARG;
    if (kind[i] < K_SKIP || kind[i] > K_OTHER || ntri[i] < 0) return set_error(ctx, "obj_correct: bad kind or count"), RX_ERR_ARG;
    line[i] = all[pos[i]];
  }
  DevBuf<int> d_line(ctx, n), d_kind(ctx, n), d_tri(ctx, n);
  if (!d_line.p || !d_kind.p || !d_tri.p) return set_error(ctx, "obj: out of device memory"), RX_ERR_CAPACITY;
  CUDA_TRY(ctx, cudaMemcpyAsync(d_line.p, line.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  CUDA_TRY(ctx, cudaMemcpyAsync(d_kind.p, kind, sizeof(int) * n, cudaMemcpyHostToDevice, st));
  CUDA_TRY(ctx, cudaMemcpyAsync(d_tri.p, ntri, sizeof(int) * n, cudaMemcpyHostToDevice, st));
  k_correct<<<(n + 255) / 256, 256, 0, st>>>(n, d_line.p, d_kind.p, d_tri.p, o->kind.p, o->cnt.p, o->lines);
  CUDA_TRY(ctx, cudaGetLastError());
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return RX_OK;
}

int obj_scan(ObjParse* o, int* totals, int* listed_prefix) {
  Ctx* ctx = o->ctx;
  cudaStream_t st = ctx->stream;
  if (!o->scanned) {
    o->span_begin();
    for (int c = 0; c < C_LIST; ++c) {
      int rc = excl_scan(ctx, o->cnt.p + (long long)c * o->lines, o->lines, o->totals.p + c);
      if (rc) return rc;
    }
    o->span_end();
    CUDA_TRY(ctx, cudaMemcpyAsync(o->tot, o->totals.p, sizeof(int) * C_N, cudaMemcpyDeviceToHost, st));
    o->scanned = true;
  }
  if (listed_prefix && o->n_listed) {
    DevBuf<int> d(ctx, (size_t)o->n_listed * C_LIST);
    if (!d.p) return set_error(ctx, "obj: out of device memory"), RX_ERR_CAPACITY;
    k_gather_prefix<<<(o->n_listed + 255) / 256, 256, 0, st>>>(o->n_listed, o->listed.p, o->cnt.p, o->lines, d.p);
    CUDA_TRY(ctx, cudaMemcpyAsync(listed_prefix, d.p, sizeof(int) * C_LIST * o->n_listed, cudaMemcpyDeviceToHost, st));
  }
  CUDA_TRY(ctx, cudaGetLastError());
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  for (int c = 0; c < C_N; ++c) totals[c] = o->tot[c];
  return RX_OK;
}

int obj_emit(ObjParse* o, const int* usemtl_gid, double* pos, double* nrm, double* uv, int* tri_pos, int* tri_nrm,
             int* tri_uv, int* tri_grp) {
  Ctx* ctx = o->ctx;
  cudaStream_t st = ctx->stream;
  if (!o->scanned) return set_error(ctx, "obj_emit: scan first"), RX_ERR_ARG;
  const int nv = o->tot[C_V], nvn = o->tot[C_VN], nvt = o->tot[C_VT], nt = o->tot[C_TRI], nm = o->tot[C_MTL];
  DevBuf<double> d_pos(ctx, 3LL * nv), d_nrm(ctx, 3LL * nvn), d_uv(ctx, 2LL * nvt);
  DevBuf<int> d_tp(ctx, 3LL * nt), d_tn(ctx, 3LL * nt), d_tu(ctx, 3LL * nt), d_tg(ctx, nt), d_gid(ctx, std::max(nm, 1));
  if ((nv && !d_pos.p) || (nvn && !d_nrm.p) || (nvt && !d_uv.p) || (nt && (!d_tp.p || !d_tn.p || !d_tu.p || !d_tg.p)) ||
      !d_gid.p)
    return set_error(ctx, "obj: out of device memory for the mesh arrays"), RX_ERR_CAPACITY;
  if (nm) CUDA_TRY(ctx, cudaMemcpyAsync(d_gid.p, usemtl_gid, sizeof(int) * nm, cudaMemcpyHostToDevice, st));
  o->span_begin();
  if (o->lines > 0)
    k_emit<<<grid_for(ctx, o->lines), 256, 0, st>>>(o->text.p, o->starts.p, o->lines, o->kind.p, o->flags.p, o->cnt.p,
                                                   d_gid.p, d_pos.p, d_nrm.p, d_uv.p, d_tp.p, d_tn.p, d_tu.p, d_tg.p);
  o->span_end();
  CUDA_TRY(ctx, cudaGetLastError());
  auto d2h = [&](void* dst, const void* src, size_t bytes) {
    return bytes && dst ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st) : cudaSuccess;
  };
  CUDA_TRY(ctx, d2h(pos, d_pos.p, sizeof(double) * 3 * nv));
  CUDA_TRY(ctx, d2h(nrm, d_nrm.p, sizeof(double) * 3 * nvn));
  CUDA_TRY(ctx, d2h(uv, d_uv.p, sizeof(double) * 2 * nvt));
  CUDA_TRY(ctx, d2h(tri_pos, d_tp.p, sizeof(int) * 3 * nt));
  CUDA_TRY(ctx, d2h(tri_nrm, d_tn.p, sizeof(int) * 3 * nt));
  CUDA_TRY(ctx, d2h(tri_uv, d_tu.p, sizeof(int) * 3 * nt));
  CUDA_TRY(ctx, d2h(tri_grp, d_tg.p, sizeof(int) * nt));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return RX_OK;
}

void obj_end(ObjParse* o) {
  if (!o) return;
  Ctx* ctx = o->ctx;
  delete o;
  cudaStreamSynchronize(ctx->stream);
}

int obj_device_ms(ObjParse* o, float* ms) {
  float total = 0.0f;
  for (auto& s : o->spans) {
    float t = 0.0f;
    CUDA_TRY(o->ctx, cudaEventSynchronize(s.second));
    CUDA_TRY(o->ctx, cudaEventElapsedTime(&t, s.first, s.second));
    total += t;
  }
  *ms = total;
  return RX_OK;
}

int obj_info(ObjParse* o, int* lines, int* listed) {
  *lines = o->lines;
  *listed = o->n_listed;
  return RX_OK;
}

}  // namespace rx
