// Edge-aware a-trous denoise.
//
// Pass 0 is the reference's guided bilateral filter
// (rendering/denoise.py:23-104): taps over a (2r+1)^2 window with reflect
// padding, spatial weight 1 / (1 + dx^2 + dy^2), Gaussian range weights on
// colour and on the normal / albedo / depth guides, normalised, then blended
// with the source by `amount`.  The float32 operation order is the
// reference's (numpy evaluates the same expressions), so only expf's last
// bits can differ.  Pass i > 0 filters the previous pass with taps 2^i apart
// (a-trous); the blend with the source and linear_to_display are fused into
// the last pass.
//
// Layout: colour float4 (rgb, -), normal guide float4 (xyz, depth), albedo
// guide float4 (rgb, -) — the accumulators' own layout, so the renderer
// filters its resident buffers without a copy.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "rx_internal.cuh"
#include "rx_runtime.h"

namespace rx {

// numpy's "reflect" padding for any offset (period 2(n - 1)).
__device__ __forceinline__ int reflect_idx(int i, int n) {
  if ((unsigned)i < (unsigned)n) return i;  // inside the image: no reflection
  if (n == 1) return 0;
  int period = 2 * (n - 1);
  i %= period;
  if (i < 0) i += period;
  return i >= n ? period - i : i;
}

struct AtrousArgs {
  int H, W, r, step;
  int use_n, use_a, use_d;
  float s2c, s2n, s2a, s2d;  // 2 sigma^2 of each range term (float32 of the double value)
  float r2c, r2n, r2a, r2d;  // RN(1 / (2 sigma^2)) of the same float32 values
  int quot;                  // pass 0 forms its quotients with div_by (all 2 sigma^2 <= 2^30)
  int last;                  // fuse blend + display
  float keep, amount;        // f32(1 - amount), f32(amount)
  int to_display;
};

// One tap's weight.  EXACT (pass 0) is the reference's expression: each
// range term its own exp of (-d^2 / 2 sigma^2) in float32, multiplied in the
// reference's order.  The a-trous passes after it (no reference
// counterpart) sum the exponents and take one exp.
template <bool EXACT>
__device__ __forceinline__ float tap_weight(const AtrousArgs& A, float sw, float4 nb, float4 cc, float4 g, float4 cn,
                                            float4 al, float4 ca) {
  float ex = nb.x - cc.x, ey = nb.y - cc.y, ez = nb.z - cc.z;
  float d2 = (ex * ex + ey * ey) + ez * ez;
  if (EXACT) {
    // each quotient is the float the division gives (div_by)
    auto q = [&](float x, float s2, float r2) { return A.quot ? div_by(x, s2, r2) : x / s2; };
    float w = sw * expf(q(-d2, A.s2c, A.r2c));
    if (A.use_n) {
      float gx = g.x - cn.x, gy = g.y - cn.y, gz = g.z - cn.z;
      w = w * expf(q(-((gx * gx + gy * gy) + gz * gz), A.s2n, A.r2n));
    }
    if (A.use_a) {
      float hx = al.x - ca.x, hy = al.y - ca.y, hz = al.z - ca.z;
      w = w * expf(q(-((hx * hx + hy * hy) + hz * hz), A.s2a, A.r2a));
    }
    if (A.use_d) {
      float gd = g.w - cn.w;
      w = w * expf(q(-(gd * gd), A.s2d, A.r2d));
    }
    return w;
  }
  // fused multiply-adds throughout
  float e = __fmaf_rn(ez, ez, __fmaf_rn(ey, ey, ex * ex)) * A.r2c;
  if (A.use_n) {
    float gx = g.x - cn.x, gy = g.y - cn.y, gz = g.z - cn.z;
    e = __fmaf_rn(__fmaf_rn(gz, gz, __fmaf_rn(gy, gy, gx * gx)), A.r2n, e);
  }
  if (A.use_a) {
    float hx = al.x - ca.x, hy = al.y - ca.y, hz = al.z - ca.z;
    e = __fmaf_rn(__fmaf_rn(hz, hz, __fmaf_rn(hy, hy, hx * hx)), A.r2a, e);
  }
  if (A.use_d) {
    float gd = g.w - cn.w;
    e = __fmaf_rn(gd * gd, A.r2d, e);
  }
  return sw * __expf(-e);
}

// Normalised sum of one pixel; the last pass blends with the source and
// maps to display.  Pass 0 divides as the reference does; the later passes
// multiply by one correctly rounded reciprocal.
template <bool EXACT>
__device__ __forceinline__ float4 finish_pixel(const AtrousArgs& A, float ax, float ay, float az, float ws,
                                               const float4* __restrict__ src, long long c) {
  float den = fmaxf(ws, 1e-8f);
  float fx, fy, fz;
  const float r = __frcp_rn(den);
  if (EXACT) {
    fx = div_by(ax, den, r), fy = div_by(ay, den, r), fz = div_by(az, den, r);
  } else {
    fx = ax * r, fy = ay * r, fz = az * r;
  }
  if (A.last) {
    float4 s = __ldg(src + c);
    fx = s.x * A.keep + fx * A.amount;
    fy = s.y * A.keep + fy * A.amount;
    fz = s.z * A.keep + fz * A.amount;
    if (A.to_display) {
      fx = sqrtf(fminf(fmaxf(fx, 0.0f), 1.0f));
      fy = sqrtf(fminf(fmaxf(fy, 0.0f), 1.0f));
      fz = sqrtf(fminf(fmaxf(fz, 0.0f), 1.0f));
    }
  }
  return make_float4(fx, fy, fz, 0.0f);
}

// Shared-memory tiled pass.  Pixels whose coordinates agree modulo `step`
// form a sub-lattice on which the pass's taps (2^i apart) are direct
// neighbours, so a block filters a kAtTW x kAtTH tile of one sub-lattice
// from a shared-memory copy of the tile plus an r-wide halo: colour, the
// normal / depth guide and the albedo guide are read from HBM once per
// block (halo overhead (32 + 2r)(16 + 2r) / 512, 1.2x at r = 1) instead of
// (2r + 1)^2 times per pixel.  Halo pixels are loaded through the reflect
// padding, so every tap equals the one the reference indexes.  The grid is
// one-dimensional: block b = ((tile_y * tiles_x + tile_x) * step + ry) *
// step + rx, with the sub-lattice residue fastest so neighbouring blocks
// share cache lines.  256 threads: each filters two pixels of a column.
constexpr int kAtTW = 32, kAtTH = 16, kAtThreads = 256, kAtMaxTiledR = 8;

// Spatial weight 1 / (1 + dx^2 + dy^2), rounded to float32 from double as
// the reference's float64 kernel weights are.
__host__ __device__ constexpr float spatial_weight(int dx, int dy) {
  return (float)(1.0 / (1.0 + (double)(dx * dx + dy * dy)));
}

// R > 0: the radius as a compile-time constant (taps unrolled, weights
// folded); R == 0: A.r at run time, weights from a shared-memory table.
template <bool EXACT, int R>
__global__ void __launch_bounds__(kAtThreads) k_atrous_tiled(AtrousArgs A, int tiles_x, const float4* __restrict__ in,
                                                             const float4* __restrict__ src,
                                                             const float4* __restrict__ gn,
                                                             const float4* __restrict__ ga, float4* __restrict__ out) {
  extern __shared__ float4 sm[];
  const int r = R > 0 ? R : A.r, step = A.step;
  const int SW = kAtTW + 2 * r, SH = kAtTH + 2 * r, SN = SW * SH;
  const bool need_g = A.use_n || A.use_d;
  float4* s_c = sm;
  float4* s_g = sm + SN;
  float4* s_a = sm + (need_g ? 2 : 1) * SN;
  __shared__ float s_sw[(2 * kAtMaxTiledR + 1) * (2 * kAtMaxTiledR + 1)];
  if (R == 0) {
    const int d = 2 * r + 1;
    for (int i = threadIdx.x; i < d * d; i += kAtThreads) s_sw[i] = spatial_weight(i % d - r, i / d - r);
  }
  long long b = blockIdx.x;
  const int rx = (int)(b % step);
  b /= step;
  const int ry = (int)(b % step);
  b /= step;
  const int tx0 = (int)(b % tiles_x) * kAtTW;
  const int ty0 = (int)(b / tiles_x) * kAtTH;
  for (int i = threadIdx.x; i < SN; i += kAtThreads) {
    const int sy = i / SW, sx = i - sy * SW;
    const int gy = reflect_idx(ry + step * (ty0 + sy - r), A.H);
    const int gx = reflect_idx(rx + step * (tx0 + sx - r), A.W);
    const long long q = (long long)gy * A.W + gx;
    s_c[i] = __ldg(in + q);
    if (need_g) s_g[i] = __ldg(gn + q);
    if (A.use_a) s_a[i] = __ldg(ga + q);
  }
  __syncthreads();
  const int tx = threadIdx.x & (kAtTW - 1);
  const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll 1
  for (int ty = threadIdx.x / kAtTW; ty < kAtTH; ty += kAtThreads / kAtTW) {
    const int x = rx + step * (tx0 + tx), y = ry + step * (ty0 + ty);
    if (x >= A.W || y >= A.H) continue;
    const int ci = (ty + r) * SW + tx + r;
    const float4 cc = s_c[ci];
    const float4 cn = need_g ? s_g[ci] : zero;
    const float4 ca = A.use_a ? s_a[ci] : zero;
    float ax = 0.0f, ay = 0.0f, az = 0.0f, ws = 0.0f;
#pragma unroll
    for (int dy = -r; dy <= r; ++dy) {
      const int row = ci + dy * SW;
#pragma unroll
      for (int dx = -r; dx <= r; ++dx) {
        const int q = row + dx;
        const float4 nb = s_c[q];
        const float4 g = need_g ? s_g[q] : zero;
        const float4 al = A.use_a ? s_a[q] : zero;
        const float sw = R > 0 ? spatial_weight(dx, dy) : s_sw[(dy + r) * (2 * r + 1) + dx + r];
        const float w = tap_weight<EXACT>(A, sw, nb, cc, g, cn, al, ca);
        ax = ax + nb.x * w;
        ay = ay + nb.y * w;
        az = az + nb.z * w;
        ws = ws + w;
      }
    }
    const long long c = (long long)y * A.W + x;
    out[c] = finish_pixel<EXACT>(A, ax, ay, az, ws, src, c);
  }
}

// Radius 1 (the renderer's default): a tap's weight is symmetric in its two
// pixels, bit for bit even in pass 0 ((a - b)^2 equals (b - a)^2 exactly
// and the spatial weight depends on |dx|, |dy|), so each pair of
// neighbours is weighed once.  A block loads a 32-column x 16-row grid of
// the sub-lattice (tiles of outputs plus their one-pixel halo), every grid
// pixel of rows 0-14 weighs its four forward neighbours (right, down-left,
// down, down-right) into shared memory, and each output then gathers its
// nine weights -- the centre's is 1 -- and sums its taps in the reference's
// order: 4.6 weight evaluations per output instead of 9.
// P = 1 (pass 0, step 1): one 30 x 14 output tile, lane = grid column.
// P = 2 (step >= 2): two adjacent x residues side by side, grid column c
// of residue plane k stored at c * 2 + k, so two neighbouring lanes read
// and write two adjacent pixels and every 32-byte sector a warp touches is
// used whole (one residue per block would use half of each); 2 x 14 x 14
// outputs.
constexpr int kA1H = 14, kA1GW = 32, kA1GH = 16, kA1Src = (kA1H + 1) * kA1GW;

template <bool EXACT, int P>
__global__ void __launch_bounds__(kAtThreads) k_atrous_r1(AtrousArgs A, int tiles_x, const float4* __restrict__ in,
                                                          const float4* __restrict__ src,
                                                          const float4* __restrict__ gn,
                                                          const float4* __restrict__ ga, float4* __restrict__ out) {
  constexpr int PW = kA1GW / P, OW = PW - 2, NOUT = P * OW * kA1H;
  __shared__ float4 s_c[kA1GW * kA1GH], s_g[kA1GW * kA1GH], s_a[kA1GW * kA1GH];
  __shared__ float s_w[4][kA1Src];  // forward weights: right, down-left, down, down-right
  const int step = A.step;
  const bool need_g = A.use_n || A.use_d;
  const int xres = step / P;  // x residue groups
  long long b = blockIdx.x;
  const int rx0 = (int)(b % xres) * P;
  b /= xres;
  const int ry = (int)(b % step);
  b /= step;
  const int tx0 = (int)(b % tiles_x) * OW;
  const int ty0 = (int)(b / tiles_x) * kA1H;
  const int lane = threadIdx.x & 31;
  {
    const int col = lane / P, plane = lane % P;
    const int gx = reflect_idx(rx0 + plane + step * (tx0 + col - 1), A.W);
    for (int sy = threadIdx.x >> 5; sy < kA1GH; sy += kAtThreads / 32) {
      const int gy = reflect_idx(ry + step * (ty0 + sy - 1), A.H);
      const long long q = (long long)gy * A.W + gx;
      const int i = sy * kA1GW + lane;
      s_c[i] = __ldg(in + q);
      if (need_g) s_g[i] = __ldg(gn + q);
      if (A.use_a) s_a[i] = __ldg(ga + q);
    }
  }
  __syncthreads();
  const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  for (int i = threadIdx.x; i < kA1Src; i += kAtThreads) {
    const int c = (i & 31) / P;
    const float4 oc = s_c[i], og = need_g ? s_g[i] : zero, oa = A.use_a ? s_a[i] : zero;
    // right (dx 1), down-left (dx -1, dy 1), down (dy 1), down-right (1, 1)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int dx = k == 0 ? 1 : k - 2, dy = k == 0 ? 0 : 1;
      const int tc = c + dx;
      float w = 0.0f;
      if (tc >= 0 && tc < PW) {
        const int t = i + dy * kA1GW + dx * P;
        w = tap_weight<EXACT>(A, spatial_weight(dx, dy), s_c[t], oc, need_g ? s_g[t] : zero, og,
                              A.use_a ? s_a[t] : zero, oa);
      }
      s_w[k][i] = w;
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < NOUT; j += kAtThreads) {
    const int oy = j / (P * OW), rem = j - oy * (P * OW);
    const int plane = rem % P, ox = rem / P;
    const int x = rx0 + plane + step * (tx0 + ox), y = ry + step * (ty0 + oy);
    if (x >= A.W || y >= A.H) continue;
    const int p = (oy + 1) * kA1GW + (ox + 1) * P + plane;
    constexpr int U = kA1GW, L = P;  // one grid row up, one grid column left
    // taps in the reference's order: dy -1..1 outer, dx -1..1 inner
    const int tq[9] = {p - U - L, p - U, p - U + L, p - L, p, p + L, p + U - L, p + U, p + U + L};
    const float tw[9] = {s_w[3][p - U - L], s_w[2][p - U], s_w[1][p - U + L], s_w[0][p - L], 1.0f,
                         s_w[0][p], s_w[1][p], s_w[2][p], s_w[3][p]};
    float ax = 0.0f, ay = 0.0f, az = 0.0f, ws = 0.0f;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const float4 nb = s_c[tq[k]];
      const float w = tw[k];
      if (EXACT) {
        ax = ax + nb.x * w;
        ay = ay + nb.y * w;
        az = az + nb.z * w;
      } else {
        ax = __fmaf_rn(nb.x, w, ax);
        ay = __fmaf_rn(nb.y, w, ay);
        az = __fmaf_rn(nb.z, w, az);
      }
      ws = ws + w;
    }
    const long long c = (long long)y * A.W + x;
    out[c] = finish_pixel<EXACT>(A, ax, ay, az, ws, src, c);
  }
}

// Radii beyond kAtMaxTiledR: every tap gathered from global memory.
template <bool EXACT>
__global__ void __launch_bounds__(256) k_atrous_gather(AtrousArgs A, const float4* __restrict__ in,
                                                       const float4* __restrict__ src, const float4* __restrict__ gn,
                                                       const float4* __restrict__ ga, float4* __restrict__ out) {
  const long long c = blockIdx.x * 256LL + threadIdx.x;
  if (c >= (long long)A.H * A.W) return;
  const int y = (int)(c / A.W), x = (int)(c - (long long)y * A.W);
  const bool need_g = A.use_n || A.use_d;
  const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const float4 cc = __ldg(in + c);
  const float4 cn = need_g ? __ldg(gn + c) : zero;
  const float4 ca = A.use_a ? __ldg(ga + c) : zero;
  float ax = 0.0f, ay = 0.0f, az = 0.0f, ws = 0.0f;
  for (int dy = -A.r; dy <= A.r; ++dy) {
    const int yy = reflect_idx(y + dy * A.step, A.H);
    for (int dx = -A.r; dx <= A.r; ++dx) {
      const int xx = reflect_idx(x + dx * A.step, A.W);
      const long long q = (long long)yy * A.W + xx;
      const float4 nb = __ldg(in + q);
      const float4 g = need_g ? __ldg(gn + q) : zero;
      const float4 al = A.use_a ? __ldg(ga + q) : zero;
      const float sw = (float)(1.0 / (1.0 + (double)(dx * dx + dy * dy)));
      const float w = tap_weight<EXACT>(A, sw, nb, cc, g, cn, al, ca);
      ax = ax + nb.x * w;
      ay = ay + nb.y * w;
      az = az + nb.z * w;
      ws = ws + w;
    }
  }
  out[c] = finish_pixel<EXACT>(A, ax, ay, az, ws, src, c);
}

__global__ void k_copy_display(long long n, const float4* __restrict__ in, float4* __restrict__ out, int to_display) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float4 v = in[i];
    if (to_display)
      v = make_float4(sqrtf(fminf(fmaxf(v.x, 0.0f), 1.0f)), sqrtf(fminf(fmaxf(v.y, 0.0f), 1.0f)),
                      sqrtf(fminf(fmaxf(v.z, 0.0f), 1.0f)), 0.0f);
    out[i] = v;
  }
}

static float two_sigma2(float s) {
  double v = (double)s * (double)s;
  if (v < 1e-8) v = 1e-8;
  return (float)(2.0 * v);
}

// Dynamic shared memory of one tiled block: colour, plus each guide in use.
static size_t atrous_smem(const AtrousArgs& A) {
  const size_t px = (size_t)(kAtTW + 2 * A.r) * (kAtTH + 2 * A.r);
  return px * sizeof(float4) * (1 + ((A.use_n || A.use_d) ? 1 : 0) + (A.use_a ? 1 : 0));
}

// Enqueues `passes` a-trous passes on `st`: pass i reads `in` (the colour for
// i = 0) and writes scratch half (i & 1), the last pass writes `out` (and
// reads `color` again for the blend).  A is filled except step / last.
static cudaError_t atrous_passes(cudaStream_t st, AtrousArgs A, int passes, const float4* color, const float4* gn,
                                 const float4* ga, float4* out, float4* s0, float4* s1) {
  const long long P = (long long)A.H * A.W;
  A.r2c = 1.0f / A.s2c, A.r2n = 1.0f / A.s2n, A.r2a = 1.0f / A.s2a, A.r2d = 1.0f / A.s2d;
  A.quot = std::max(std::max(A.s2c, A.s2n), std::max(A.s2a, A.s2d)) <= 0x1p+30f;
  const float4* in = color;
  for (int i = 0; i < passes; ++i) {
    A.step = 1 << i;
    A.last = i == passes - 1;
    const bool exact = i == 0;
    float4* o = A.last ? out : ((i & 1) ? s1 : s0);
    if (A.r == 1) {
      const int P = A.step >= 2 ? 2 : 1, ow = kA1GW / P - 2;
      const long long sub_w = (A.W + A.step - 1) / A.step, sub_h = (A.H + A.step - 1) / A.step;
      const long long tiles_x = (sub_w + ow - 1) / ow, tiles_y = (sub_h + kA1H - 1) / kA1H;
      const long long blocks = tiles_x * tiles_y * (A.step / P) * A.step;
      if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
      auto kern = P == 1 ? (exact ? k_atrous_r1<true, 1> : k_atrous_r1<false, 1>)
                         : (exact ? k_atrous_r1<true, 2> : k_atrous_r1<false, 2>);
      kern<<<(unsigned)blocks, kAtThreads, 0, st>>>(A, (int)tiles_x, in, color, gn, ga, o);
    } else if (A.r <= kAtMaxTiledR) {
      const long long sub_w = (A.W + A.step - 1) / A.step, sub_h = (A.H + A.step - 1) / A.step;
      const long long tiles_x = (sub_w + kAtTW - 1) / kAtTW, tiles_y = (sub_h + kAtTH - 1) / kAtTH;
      const long long blocks = tiles_x * tiles_y * A.step * A.step;
      const size_t smem = atrous_smem(A);
      if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
      auto kern = A.r == 1   ? (exact ? k_atrous_tiled<true, 1> : k_atrous_tiled<false, 1>)
                  : A.r == 2 ? (exact ? k_atrous_tiled<true, 2> : k_atrous_tiled<false, 2>)
                             : (exact ? k_atrous_tiled<true, 0> : k_atrous_tiled<false, 0>);
      if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
      }
      kern<<<(unsigned)blocks, kAtThreads, smem, st>>>(A, (int)tiles_x, in, color, gn, ga, o);
    } else {
      const long long blocks = (P + 255) / 256;
      if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
      if (exact)
        k_atrous_gather<true><<<(unsigned)blocks, 256, 0, st>>>(A, in, color, gn, ga, o);
      else
        k_atrous_gather<false><<<(unsigned)blocks, 256, 0, st>>>(A, in, color, gn, ga, o);
    }
    in = o;
  }
  return cudaGetLastError();
}

int denoise_device(Ctx* ctx, int h, int w, const float4* d_color, const float4* d_gn, const float4* d_ga,
                   int has_normal, int has_albedo, int has_depth, const rx_denoise_params* dp, float4* d_out,
                   float4* d_s0, float4* d_s1, int to_display) {
  cudaStream_t st = ctx->stream;
  long long P = (long long)h * w;
  int passes = std::max(dp->passes, 1);
  double amount = std::min(std::max((double)dp->amount, 0.0), 1.0);
  if (dp->radius <= 0 || dp->amount <= 0.0f) {
    int blocks = (int)std::min<long long>((P + 255) / 256, (long long)ctx->num_sms * 16);
    k_copy_display<<<std::max(blocks, 1), 256, 0, st>>>(P, d_color, d_out, to_display);
    CUDA_TRY(ctx, cudaGetLastError());
    return RX_OK;
  }
  AtrousArgs A;
  A.H = h;
  A.W = w;
  A.r = dp->radius;
  A.use_n = has_normal;
  A.use_a = has_albedo;
  A.use_d = has_depth;
  A.s2c = two_sigma2(dp->sigma_color);
  A.s2n = two_sigma2(dp->sigma_normal);
  A.s2a = two_sigma2(dp->sigma_albedo);
  A.s2d = two_sigma2(dp->sigma_depth);
  A.keep = (float)(1.0 - amount);
  A.amount = (float)amount;
  A.to_display = to_display;
  CUDA_TRY(ctx, atrous_passes(st, A, passes, d_color, d_gn, d_ga, d_out, d_s0, d_s1));
  return RX_OK;
}

__global__ void k_pack_in(long long n, const float* __restrict__ a, int ca, const float* __restrict__ d,
                          float4* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float4 v = make_float4(0, 0, 0, 0);
    if (a) {
      if (ca == 3) v = make_float4(a[3 * i], a[3 * i + 1], a[3 * i + 2], 0.0f);
    }
    if (d) v.w = d[i];
    out[i] = v;
  }
}

__global__ void k_unpack3(long long n, const float4* __restrict__ in, float* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float4 v = in[i];
    out[3 * i] = v.x;
    out[3 * i + 1] = v.y;
    out[3 * i + 2] = v.z;
  }
}

int denoise_host(Ctx* ctx, int h, int w, const float* color, const float* normal, const float* albedo,
                 const float* depth, const rx_denoise_params* dp, float* out) {
  cudaStream_t st = ctx->stream;
  long long P = (long long)h * w;
  if (P <= 0) return RX_OK;
  DevBuf<float> hc(ctx, 3 * P), hn(ctx, normal ? 3 * P : 0), ha(ctx, albedo ? 3 * P : 0), hd(ctx, depth ? P : 0);
  DevBuf<float4> c4(ctx, P), n4(ctx, P), a4(ctx, P), o4(ctx, P), s0(ctx, P), s1(ctx, P);
  DevBuf<float> ho(ctx, 3 * P);
  if (!c4.p || !o4.p || !s0.p || !s1.p || !hc.p || !ho.p || !n4.p || !a4.p)
    return set_error(ctx, "out of device memory for a %dx%d denoise", h, w), RX_ERR_CAPACITY;
  CUDA_TRY(ctx, cudaMemcpyAsync(hc.p, color, sizeof(float) * 3 * P, cudaMemcpyHostToDevice, st));
  if (normal) CUDA_TRY(ctx, cudaMemcpyAsync(hn.p, normal, sizeof(float) * 3 * P, cudaMemcpyHostToDevice, st));
  if (albedo) CUDA_TRY(ctx, cudaMemcpyAsync(ha.p, albedo, sizeof(float) * 3 * P, cudaMemcpyHostToDevice, st));
  if (depth) CUDA_TRY(ctx, cudaMemcpyAsync(hd.p, depth, sizeof(float) * P, cudaMemcpyHostToDevice, st));
  int blocks = (int)std::min<long long>((P + 255) / 256, (long long)ctx->num_sms * 16);
  blocks = std::max(blocks, 1);
  k_pack_in<<<blocks, 256, 0, st>>>(P, hc.p, 3, nullptr, c4.p);
  k_pack_in<<<blocks, 256, 0, st>>>(P, normal ? hn.p : nullptr, 3, depth ? hd.p : nullptr, n4.p);
  k_pack_in<<<blocks, 256, 0, st>>>(P, albedo ? ha.p : nullptr, 3, nullptr, a4.p);
  int rc = denoise_device(ctx, h, w, c4.p, n4.p, a4.p, normal != nullptr, albedo != nullptr, depth != nullptr, dp,
                          o4.p, s0.p, s1.p, dp->to_display);
  if (rc) return rc;
  k_unpack3<<<blocks, 256, 0, st>>>(P, o4.p, ho.p);
  CUDA_TRY(ctx, cudaMemcpyAsync(out, ho.p, sizeof(float) * 3 * P, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return RX_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant (rx_denoise_noalloc).
//
// Some callers cannot allocate device memory when they denoise: a host
// application that owns the whole device-memory budget through its own
// allocator (a compositor or plugin host, a serving process with a fixed
// HBM budget), or a frame loop that must not pay the device-wide
// synchronisation a cudaMalloc / cudaFree can imply.  For them the two
// intermediate a-trous buffers live in this file-scope device array instead
// of per-call allocations.  It is sized for kNoAllocMaxPixels pixels
// (2 x 16 B x 2^20 = 32 MiB) and every GPU that loads the library keeps it
// until the process exits.
//
// The host never dereferences `g_noalloc_scratch`: in host code the name is
// only a stand-in, so its device address is looked up once per device with
// cudaGetSymbolAddress (with that device current) the first time the entry
// point runs there.  Make that first call on a device before any stream
// capture.  Every pass writes every pixel of its output before the next pass
// reads it, so nothing in the array has to start at zero; it keeps the last
// call's contents.  All calls share the one array: calls whose kernels can
// overlap on the GPU (different streams, or host threads on one device
// without ordering) race on it and must be serialised by the caller.
// ---------------------------------------------------------------------------
constexpr long long kNoAllocMaxPixels = 1LL << 20;
static __device__ __align__(256) float4 g_noalloc_scratch[2 * kNoAllocMaxPixels];

// The array's device address differs per CUDA context (the module is loaded
// into each context), so the looked-up address is cached per context,
// identified by cuCtxGetId: an id the driver never hands out twice in a
// process, so a context created after cudaDeviceReset, or a caller's own
// driver-API context, gets a fresh lookup instead of a stale address.  The
// driver calls are reached through the runtime's entry-point table (the
// library does not link libcuda).  Without them the address is looked up on
// every call, which also allocates nothing.
typedef int (*PfnCtxGetCurrent)(void**);
typedef int (*PfnCtxGetId)(void*, unsigned long long*);
static std::mutex g_noalloc_mu;
static bool g_noalloc_fn_init = false;
static PfnCtxGetCurrent g_ctx_get_current = nullptr;
static PfnCtxGetId g_ctx_get_id = nullptr;
constexpr int kNoAllocCache = 16;
static unsigned long long g_noalloc_ctx[kNoAllocCache] = {};
static float4* g_noalloc_ptr[kNoAllocCache] = {};
static int g_noalloc_next = 0;

// Device address of the scratch array in the context current on this thread.
static int noalloc_scratch(float4** out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_fn_init) {
    g_noalloc_fn_init = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_current = reinterpret_cast<PfnCtxGetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_id = reinterpret_cast<PfnCtxGetId>(f);
    (void)cudaGetLastError();
  }
  // make the runtime's context current (a no-op when one already is)
  cudaError_t e = cudaFree(nullptr);
  if (e != cudaSuccess)
    return set_error(nullptr, "rx_denoise_noalloc: no usable CUDA context: %s", cudaGetErrorString(e)), RX_ERR_CUDA;
  unsigned long long id = 0;
  void* cu = nullptr;
  const bool have_id = g_ctx_get_current && g_ctx_get_id && g_ctx_get_current(&cu) == 0 && cu &&
                       g_ctx_get_id(cu, &id) == 0;
  if (have_id) {
    for (int i = 0; i < kNoAllocCache; ++i)
      if (g_noalloc_ptr[i] && g_noalloc_ctx[i] == id) {
        *out = g_noalloc_ptr[i];
        return RX_OK;
      }
  }
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    return set_error(nullptr, "rx_denoise_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e)), RX_ERR_CUDA;
  if (have_id) {
    g_noalloc_ctx[g_noalloc_next] = id;
    g_noalloc_ptr[g_noalloc_next] = static_cast<float4*>(p);
    g_noalloc_next = (g_noalloc_next + 1) % kNoAllocCache;
  }
  *out = static_cast<float4*>(p);
  return RX_OK;
}

// True when [a, a + an) and [b, b + bn) share a byte.
static bool overlaps(const void* a, size_t an, const void* b, size_t bn) {
  if (!a || !b) return false;
  const char* pa = static_cast<const char*>(a);
  const char* pb = static_cast<const char*>(b);
  return pa < pb + bn && pb < pa + an;
}

}  // namespace rx

extern "C" int rx_denoise_noalloc(int height, int width, const float* d_color, const float* d_guide_normal,
                                  const float* d_guide_albedo, const rx_denoise_params* params, float* d_out,
                                  void* stream) {
  using namespace rx;
  if (!params || height < 0 || width < 0) return set_error(nullptr, "rx_denoise_noalloc: bad arguments"), RX_ERR_ARG;
  long long P = (long long)height * width;
  if (P > kNoAllocMaxPixels)
    return set_error(nullptr, "rx_denoise_noalloc: %d x %d = %lld pixels exceeds the %lld-pixel scratch limit",
                     height, width, P, kNoAllocMaxPixels),
           RX_ERR_CAPACITY;
  if (P == 0) return RX_OK;
  if (!d_color || !d_out) return set_error(nullptr, "rx_denoise_noalloc: NULL colour or output"), RX_ERR_ARG;
  const bool need_n = params->use_normal || params->use_depth;
  if (need_n && !d_guide_normal)
    return set_error(nullptr, "rx_denoise_noalloc: normal/depth guide requested but NULL"), RX_ERR_ARG;
  if (params->use_albedo && !d_guide_albedo)
    return set_error(nullptr, "rx_denoise_noalloc: albedo guide requested but NULL"), RX_ERR_ARG;
  if (params->radius < 0 || params->passes < 1 || params->passes > 12)
    return set_error(nullptr, "rx_denoise_noalloc: radius must be >= 0 and passes in [1, 12]"), RX_ERR_ARG;
  const size_t bytes = (size_t)P * sizeof(float4);
  if (overlaps(d_out, bytes, d_color, bytes) || (need_n && overlaps(d_out, bytes, d_guide_normal, bytes)) ||
      (params->use_albedo && overlaps(d_out, bytes, d_guide_albedo, bytes)))
    return set_error(nullptr, "rx_denoise_noalloc: the output must not overlap the colour or a guide in use"),
           RX_ERR_ARG;
  // an error left pending by earlier, unrelated work is not this call's
  (void)cudaGetLastError();
  float4* scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const float4* color = reinterpret_cast<const float4*>(d_color);
  const float4* gn = need_n ? reinterpret_cast<const float4*>(d_guide_normal) : nullptr;
  const float4* ga = params->use_albedo ? reinterpret_cast<const float4*>(d_guide_albedo) : nullptr;
  float4* out = reinterpret_cast<float4*>(d_out);
  cudaError_t e = cudaSuccess;
  if (params->radius <= 0 || params->amount <= 0.0f) {
    int blocks = (int)std::min<long long>((P + 255) / 256, 4096);
    k_copy_display<<<blocks, 256, 0, st>>>(P, color, out, params->to_display);
    e = cudaGetLastError();
  } else {
    double amount = std::min(std::max((double)params->amount, 0.0), 1.0);
    AtrousArgs A;
    A.H = height;
    A.W = width;
    A.r = params->radius;
    A.use_n = params->use_normal;
    A.use_a = params->use_albedo;
    A.use_d = params->use_depth;
    A.s2c = two_sigma2(params->sigma_color);
    A.s2n = two_sigma2(params->sigma_normal);
    A.s2a = two_sigma2(params->sigma_albedo);
    A.s2d = two_sigma2(params->sigma_depth);
    A.keep = (float)(1.0 - amount);
    A.amount = (float)amount;
    A.to_display = params->to_display;
    e = atrous_passes(st, A, params->passes, color, gn, ga, out, scratch, scratch + kNoAllocMaxPixels);
  }
  if (e != cudaSuccess)
    return set_error(nullptr, "rx_denoise_noalloc: launch failed: %s", cudaGetErrorString(e)), RX_ERR_CUDA;
  return RX_OK;
}
