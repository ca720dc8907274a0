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
  int last;                  // fuse blend + display
  float keep, amount;        // f32(1 - amount), f32(amount)
  int to_display;
};

__global__ void __launch_bounds__(256) k_atrous(AtrousArgs A, const float4* __restrict__ in,
                                                const float4* __restrict__ src, const float4* __restrict__ gn,
                                                const float4* __restrict__ ga, float4* __restrict__ out) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= A.W || y >= A.H) return;
  long long c = (long long)y * A.W + x;
  float4 cc = __ldg(in + c);
  float4 cn = A.use_n || A.use_d ? __ldg(gn + c) : make_float4(0, 0, 0, 0);
  float4 ca = A.use_a ? __ldg(ga + c) : make_float4(0, 0, 0, 0);
  float ax = 0.0f, ay = 0.0f, az = 0.0f, ws = 0.0f;
  for (int dy = -A.r; dy <= A.r; ++dy) {
    int yy = reflect_idx(y + dy * A.step, A.H);
    for (int dx = -A.r; dx <= A.r; ++dx) {
      int xx = reflect_idx(x + dx * A.step, A.W);
      long long q = (long long)yy * A.W + xx;
      float4 nb = __ldg(in + q);
      float ex = nb.x - cc.x, ey = nb.y - cc.y, ez = nb.z - cc.z;
      float d2 = (ex * ex + ey * ey) + ez * ez;
      float sw = (float)(1.0 / (1.0 + (double)(dx * dx + dy * dy)));
      float w = sw * expf(-d2 / A.s2c);
      if (A.use_n || A.use_d) {
        float4 g = __ldg(gn + q);
        if (A.use_n) {
          float gx = g.x - cn.x, gy = g.y - cn.y, gz = g.z - cn.z;
          w = w * expf(-((gx * gx + gy * gy) + gz * gz) / A.s2n);
        }
        if (A.use_a) {
          float4 al = __ldg(ga + q);
          float hx = al.x - ca.x, hy = al.y - ca.y, hz = al.z - ca.z;
          w = w * expf(-((hx * hx + hy * hy) + hz * hz) / A.s2a);
        }
        if (A.use_d) {
          float gd = g.w - cn.w;
          w = w * expf(-(gd * gd) / A.s2d);
        }
      } else if (A.use_a) {
        float4 al = __ldg(ga + q);
        float hx = al.x - ca.x, hy = al.y - ca.y, hz = al.z - ca.z;
        w = w * expf(-((hx * hx + hy * hy) + hz * hz) / A.s2a);
      }
      ax = ax + nb.x * w;
      ay = ay + nb.y * w;
      az = az + nb.z * w;
      ws = ws + w;
    }
  }
  float den = fmaxf(ws, 1e-8f);
  float fx = ax / den, fy = ay / den, fz = az / den;
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
  out[c] = make_float4(fx, fy, fz, 0.0f);
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
  dim3 blk(32, 8);
  dim3 grd((w + 31) / 32, (h + 7) / 8);
  const float4* in = d_color;
  for (int i = 0; i < passes; ++i) {
    A.step = 1 << i;
    A.last = i == passes - 1;
    float4* o = A.last ? d_out : ((i & 1) ? d_s1 : d_s0);
    k_atrous<<<grd, blk, 0, st>>>(A, in, d_color, d_gn, d_ga, o);
    in = o;
  }
  CUDA_TRY(ctx, cudaGetLastError());
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

static std::mutex g_noalloc_mu;
static float4* g_noalloc_ptr[64] = {};

// Device address of the scratch array on the current device.
static int noalloc_scratch(float4** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_error(nullptr, "rx_denoise_noalloc: cudaGetDevice: %s", cudaGetErrorString(e)),
                               RX_ERR_CUDA;
  if (dev < 0 || dev >= 64) return set_error(nullptr, "rx_denoise_noalloc: device %d out of range", dev), RX_ERR_ARG;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return set_error(nullptr, "rx_denoise_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e)), RX_ERR_CUDA;
    g_noalloc_ptr[dev] = static_cast<float4*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return RX_OK;
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
  if ((params->use_normal || params->use_depth) && !d_guide_normal)
    return set_error(nullptr, "rx_denoise_noalloc: normal/depth guide requested but NULL"), RX_ERR_ARG;
  if (params->use_albedo && !d_guide_albedo)
    return set_error(nullptr, "rx_denoise_noalloc: albedo guide requested but NULL"), RX_ERR_ARG;
  if (params->radius < 0 || params->passes < 1 || params->passes > 12)
    return set_error(nullptr, "rx_denoise_noalloc: radius must be >= 0 and passes in [1, 12]"), RX_ERR_ARG;
  float4* scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const float4* color = reinterpret_cast<const float4*>(d_color);
  const float4* gn = reinterpret_cast<const float4*>(d_guide_normal);
  const float4* ga = reinterpret_cast<const float4*>(d_guide_albedo);
  float4* out = reinterpret_cast<float4*>(d_out);
  if (params->radius <= 0 || params->amount <= 0.0f) {
    int blocks = (int)std::min<long long>((P + 255) / 256, 4096);
    k_copy_display<<<blocks, 256, 0, st>>>(P, color, out, params->to_display);
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
    dim3 blk(32, 8);
    dim3 grd((width + 31) / 32, (height + 7) / 8);
    const float4* in = color;
    for (int i = 0; i < params->passes; ++i) {
      A.step = 1 << i;
      A.last = i == params->passes - 1;
      float4* o = A.last ? out : scratch + (size_t)(i & 1) * kNoAllocMaxPixels;
      k_atrous<<<grd, blk, 0, st>>>(A, in, color, gn, ga, o);
      in = o;
    }
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_error(nullptr, "rx_denoise_noalloc: launch failed: %s", cudaGetErrorString(e)), RX_ERR_CUDA;
  return RX_OK;
}
