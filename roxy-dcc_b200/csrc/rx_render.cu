// Wavefront path tracer.
//
// The reference runs one megakernel thread per pixel per frame
// (rendering/taichi/trace.py:239-283) that loops over bounces with five
// material branches.  Here one wavefront holds `spf` frames x W x H paths
// whose state lives in structure-of-arrays buffers in HBM; each bounce is
//
//   extend  (closest hit for the active queue, plus any-hit for the shadow
//            rays the previous bounce emitted, adding unoccluded
//            contributions)                            rx_internal.cuh traversal
//   shade   (materials, emission, NEE sample, scatter, Russian roulette;
//            warp-aggregated pushes into the next queue and the shadow queue)
//
// followed by one accumulate pass that applies the sample clamp and folds
// the frames into the running means exactly as the reference does.  The
// per-wave launch sequence is captured once as a CUDA graph and replayed.
//
// Random numbers come from Philox4x32-10 keyed by (pixel, sample, bounce,
// slot), so a path's numbers do not depend on scheduling.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "rx_internal.cuh"
#include "rx_runtime.h"

namespace rx {

constexpr int kMaxBounce = 64;
// Default queue length at or below which k_tail runs a wave's remaining
// bounces path by path (tuned on the 1080p benchmark frame).
constexpr int kTailPaths = 1 << 16;
// counters, 64 per kind (one per bounce): queue lengths, extend fetch,
// shade fetch, shadow record counts; then the bounce + 1 at which k_tail
// took the wave over (0: not taken) and k_tail's fetch counter
enum { C_Q = 0, C_FE = 64, C_FS = 128, C_S = 192, C_TAIL = 256, C_FT = 257, C_N = 260 };
constexpr float kPi = 3.14159265358979323846f;
constexpr float kTwoPi = 6.283185307179586f;

struct RenderK {
  int W, H;
  long long P;
  int spf;
  float fov_tan, aspect;
  float3 cam_pos, cam_fwd, cam_right, cam_up;
  int max_depth, use_sky;
  float3 bg;
  int mode, dlmd;
  float clamp;
  int compat;
  int mis;  // power-heuristic MIS between NEE and BSDF hits of listed lights
  int camera0;  // bounce 0 makes its camera rays in place (no k_generate)
  uint32_t seed;
  long long shadow_cap;
  long long queue_cap;
};

__device__ __forceinline__ float fractf_(float x) { return x - floorf(x); }

// camera.py:23-30 with a counter-based per-pixel phase in place of the
// sin-hash: jitter = fract(phase + (frame + 1) * R2).
__device__ __forceinline__ float3 camera_dir(const RenderK& K, int px, int py, int frame) {
  uint32_t ph[4];
  philox((uint32_t)((long long)py * K.W + px), 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, K.seed, kKeyHi, ph);
  float i = (float)(frame + 1);
  float jx = fractf_(u01(ph[0]) + i * 0.7548776662466927f);
  float jy = fractf_(u01(ph[1]) + i * 0.5698402909980532f);
  float u = ((float)px + jx) / (float)K.W * 2.0f - 1.0f;
  float v = 1.0f - ((float)py + jy) / (float)K.H * 2.0f;
  float ndx = u * K.aspect * K.fov_tan;
  float ndy = v * K.fov_tan;
  return normalized((K.cam_fwd + K.cam_right * ndx) + K.cam_up * ndy);
}

struct PathRng {
  uint32_t pix, smp, bounce, seed;
  uint32_t blk[3][4];
  unsigned have;
  __device__ void init(uint32_t p, uint32_t s, uint32_t b, uint32_t k) {
    pix = p; smp = s; bounce = b; seed = k; have = 0;
  }
  __device__ float get(int slot) {
    int bi = slot >> 2;
    if (bi < 3) {
      if (!(have & (1u << bi))) {
        philox(pix, smp, bounce, (uint32_t)bi, seed, kKeyHi, blk[bi]);
        have |= 1u << bi;
      }
      return u01(blk[bi][slot & 3]);
    }
    uint32_t o[4];
    philox(pix, smp, bounce, (uint32_t)bi, seed, kKeyHi, o);
    return u01(o[slot & 3]);
  }
};

// ---------------------------------------------------------------- scattering
// scatter.py:14-38
__device__ __forceinline__ float3 diffuse_scatter(float3 n, float r1, float r2) {
  float phi = kTwoPi * r1;
  float r = sqrtf(r2);
  float sp, cp;
  sincosf(phi, &sp, &cp);
  float lx = cp * r, ly = sp * r;
  float lz = sqrtf(fmaxf(0.0f, 1.0f - r2));
  float3 helper = fabsf(n.x) > 0.9f ? f3(0.0f, 1.0f, 0.0f) : f3(1.0f, 0.0f, 0.0f);
  float3 bt = normalized(cross(n, helper));
  float3 tg = cross(bt, n);
  float3 s = normalized((tg * lx + bt * ly) + n * lz);
  if (dot(s, s) < 1e-8f) s = n;
  return normalized(s);
}

// scatter.py:6-11
__device__ __forceinline__ float3 random_unit_vector(float r1, float r2) {
  float theta = acosf(1.0f - 2.0f * r1);
  float phi = kTwoPi * r2;
  float st = sinf(theta);
  float sp, cp;
  sincosf(phi, &sp, &cp);
  return f3(st * cp, st * sp, cosf(theta));
}

__device__ __forceinline__ float3 reflect(float3 d, float3 n) { return d - (2.0f * dot(d, n)) * n; }

__device__ __forceinline__ float3 refract(float3 d, float3 n, float eta) {
  float c = fminf(-dot(d, n), 1.0f);
  float3 perp = eta * (d + c * n);
  float3 par = -sqrtf(fabsf(1.0f - dot(perp, perp))) * n;
  return perp + par;
}

__device__ __forceinline__ float schlick(float c, float eta) {
  float r0 = powf((1.0f - eta) / (1.0f + eta), 2.0f);
  return r0 + (1.0f - r0) * powf(1.0f - c, 5.0f);
}

// trace.py:23-57 cone sampling of a sphere light.
__device__ __forceinline__ void sphere_light_sample(float3 hit_p, float3 center, float radius, float ru1, float ru2,
                                                    float3& ldir, float& t_light, float& sop) {
  float3 to_c = center - hit_p;
  float dist2 = fmaxf(dot(to_c, to_c), 1e-6f);
  float dist = sqrtf(dist2);
  float3 axis = to_c / dist;
  float sin2 = fminf(radius * radius / dist2, 1.0f);
  float cos_max = sqrtf(fmaxf(0.0f, 1.0f - sin2));
  float cos_t = 1.0f - ru1 * (1.0f - cos_max);
  float sin_t = sqrtf(fmaxf(0.0f, 1.0f - cos_t * cos_t));
  float phi = kTwoPi * ru2;
  float3 helper = fabsf(axis.x) > 0.9f ? f3(0.0f, 1.0f, 0.0f) : f3(1.0f, 0.0f, 0.0f);
  float3 bt = normalized(cross(axis, helper));
  float3 tg = cross(bt, axis);
  float sp, cp;
  sincosf(phi, &sp, &cp);
  ldir = normalized((tg * (cp * sin_t) + bt * (sp * sin_t)) + axis * cos_t);
  float3 oc = hit_p - center;
  float hb = dot(oc, ldir);
  float c = dot(oc, oc) - radius * radius;
  float disc = fmaxf(hb * hb - c, 0.0f);
  t_light = -hb - sqrtf(disc);
  sop = 2.0f * (1.0f - cos_max);
}

// One light sample without visibility: direction, shadow distance and the
// contribution it adds if unoccluded (albedo * L * geometry * weight);
// pdf = the density of the sampled direction in solid angle (the light's
// own sampling, without the pick probability).  The cone sample's `sop` is
// its solid angle over pi.
__device__ __forceinline__ bool light_sample(const Light& L, float ru1, float ru2, float3 hit_p, float3 n, float3 alb,
                                             float weight, float3& dir, float& max_t, float3& val, float& pdf) {
  float3 base = (alb * L.albedo) * L.emission;
  if (L.kind == 0) {
    float3 ldir;
    float tl, sop;
    sphere_light_sample(hit_p, L.p0, L.p1.x, ru1, ru2, ldir, tl, sop);
    float ndotl = dot(n, ldir);
    if (!(ndotl > 0.0f)) return false;
    max_t = tl * 0.999f;
    if (!(max_t > 0.001f)) return false;
    dir = ldir;
    val = ((base * ndotl) * sop) * weight;
    pdf = sop > 0.0f ? 1.0f / (kPi * sop) : 0.0f;
    return true;
  }
  float su = sqrtf(ru1);
  float b1 = su * (1.0f - ru2);
  float b2 = su * ru2;
  float3 e1 = L.p1 - L.p0, e2 = L.p2 - L.p0;
  float3 y = (L.p0 + e1 * b1) + e2 * b2;
  float3 to = y - hit_p;
  float d2 = dot(to, to);
  float d = sqrtf(d2);
  float3 wi = to * (1.0f / d);
  float ndotl = dot(n, wi);
  if (!(ndotl > 0.0f)) return false;
  float3 ln = normalized(cross(e1, e2));
  float cos_l = fabsf(dot(ln, wi));
  max_t = d * 0.999f;
  if (!(max_t > 0.001f)) return false;
  float g = (((ndotl * cos_l) * L.area) / (kPi * d2)) * weight;
  dir = wi;
  val = base * g;
  pdf = cos_l * L.area > 0.0f ? d2 / (cos_l * L.area) : 3.0e38f;
  return true;
}

// Solid-angle density with which light L's own sampling picks direction d
// from point o, given that d reaches L at distance t (the BSDF-hit side of
// the MIS weight; same formulas as light_sample).
__device__ __forceinline__ float light_dir_pdf(const Light& L, float3 o, float3 d, float t) {
  if (L.kind == 0) {
    float3 to_c = L.p0 - o;
    float dist2 = fmaxf(dot(to_c, to_c), 1e-6f);
    float sin2 = fminf(L.p1.x * L.p1.x / dist2, 1.0f);
    float sop = 2.0f * (1.0f - sqrtf(fmaxf(0.0f, 1.0f - sin2)));
    return sop > 0.0f ? 1.0f / (kPi * sop) : 0.0f;
  }
  float3 ln = normalized(cross(L.p1 - L.p0, L.p2 - L.p0));
  float cos_l = fabsf(dot(ln, d));
  return cos_l * L.area > 0.0f ? (t * t) / (cos_l * L.area) : 3.0e38f;
}

// power heuristic (beta = 2) weight of the strategy with density a against
// one with density b (rendering/sampling.py:36-45)
__device__ __forceinline__ float mis_power(float a, float b) {
  a = fmaxf(a, 0.0f);
  b = fmaxf(b, 0.0f);
  if (a >= 1.0e18f) return 1.0f;
  if (b >= 1.0e18f) return 0.0f;
  const float aa = a * a, bb = b * b;
  return aa + bb > 0.0f ? aa / (aa + bb) : 0.0f;
}

// ------------------------------------------------------------- path sources
// Where a path's scene, render parameters, pixel and sample index come from.
// SingleSrc: one scene and one parameter block for the whole wave (kernel
// parameters).  BatchSrc: a wave made of segments of several jobs (scene +
// accumulator + parameters); a per-path segment index selects them.

// Paths [path0, path0 + frames * P) of a wave belong to job `job`: its next
// `frames` frames, counted from the job's frame base at the start of the wave.
struct WaveSeg {
  long long path0;
  long long acc0;  // first accumulate thread of the segment (prefix sum of P)
  long long P;
  int frames;
  int job;
};

// Accumulation targets of one job (an Accum's buffers).
struct JobAcc {
  float4 *acc_r, *acc_n, *acc_a, *pixels;
  double* acc64;
  int* frame_base;
  unsigned long long* rays;
};

// Strip index s of a frame -> pixel: kStripRows-row strips walked column by
// column (32-bit: a frame holds fewer than 2^31 pixels).
constexpr int kStripRows = 2;  // a power of two (2: 6,316 against 6,262 Mrays/s with 4 on the 1080p benchmark)
__device__ __forceinline__ void strip_pixel(const RenderK& K, long long s, int& px, int& py) {
  const int si = (int)s, ws = kStripRows * K.W;
  const int strip = si / ws, r = si - strip * ws;
  const int hs = min(kStripRows, K.H - kStripRows * strip);
  if (hs == kStripRows) {  // every strip but a short last one
    px = r / kStripRows;
    py = kStripRows * strip + (r & (kStripRows - 1));
    return;
  }
  const int c = r / hs;
  px = c;
  py = kStripRows * strip + (r - c * hs);
}

// Single renders store path state at index f * P + s: frame f of the wave,
// s the pixel's strip index.  Camera item t of a wave: frames go in groups
// of kCamFrames (fewer when the wave's frame count is not a multiple);
// within a group consecutive items are one pixel's samples and pixels
// follow the strips, so a warp traces a 2 x 2 pixel block x 8 samples,
// rays that differ only by their sub-pixel jitter, and stores their state
// as eight runs of 4 consecutive paths.  Any order gives the same image: a
// path's random numbers depend on its pixel, sample and bounce.
constexpr int kCamFrames = 8;
// the largest power of two up to kCamFrames that divides `frames`
__device__ __forceinline__ int group_of(int frames) {
  int g = kCamFrames;
  while (frames % g) g >>= 1;
  return g;
}
__device__ __forceinline__ int camera_group(const RenderK& K) { return group_of(K.spf); }
__device__ __forceinline__ long long camera_path(const RenderK& K, long long t, int& px, int& py, int& f) {
  const int g = camera_group(K);
  const long long span = (long long)g * K.P;
  const long long c = t / span;
  const int r = (int)(t - c * span);
  const int s = r / g;
  f = (int)(c * g) + (r - s * g);
  strip_pixel(K, s, px, py);
  return (long long)f * K.P + s;
}

struct SingleSrc {
  static constexpr bool kBatch = false;
  static constexpr bool kWide = false;  // the traversal picks the 4-wide tree when the scene has one
  DevScene S;
  RenderK K;
  __device__ __forceinline__ int seg(long long) const { return 0; }
  __device__ __forceinline__ DevScene scene(int) const { return S; }
  __device__ __forceinline__ RenderK params(int) const { return K; }
  // sample index of path p = f * P + strip index (fb: the accumulator's
  // frame base); the path's pixel travels in its throughput's w
  __device__ __forceinline__ uint32_t sample(int, long long p, int fb) const {
    return (uint32_t)(fb + (int)(p / K.P));
  }
  // With K.camera0, bounce 0 has no queue: its items are the wave's camera
  // paths in k_generate's order, and k_extend / k_shade make each camera ray
  // where they need it instead of reading the state k_generate would write.
  const int* fbase = nullptr;  // the accumulator's frame base
  __device__ __forceinline__ long long camera_items(int b) const {
    return b == 0 && K.camera0 ? (long long)K.spf * K.P : 0;
  }
  __device__ __forceinline__ int frame0() const { return *fbase; }
  // camera ray of item t; pix / smp: its pixel (row major) and sample
  __device__ __forceinline__ int camera_ray(long long t, int fb, float3& o, float3& d, uint32_t& pix,
                                            uint32_t& smp) const {
    int px, py, f;
    const long long p = camera_path(K, t, px, py, f);
    o = K.cam_pos;
    d = camera_dir(K, px, py, fb + f);
    pix = (uint32_t)(py * K.W + px);
    smp = (uint32_t)(fb + f);
    return (int)p;
  }
};

struct BatchSrc {
  static constexpr bool kBatch = true;
  static constexpr bool kWide = false;
  const int* pseg;  // segment of each path
  const WaveSeg* segs;
  const DevScene* scenes;
  const RenderK* ks;
  const JobAcc* accs;
  unsigned long long* job_rays;  // rays traced per job in this wave
  __device__ __forceinline__ int seg(long long p) const { return __ldg(pseg + p); }
  // This source traverses the binary tree (BatchSrc4: the 4-wide one); a
  // kernel with both traversals inlined spills at 64 registers.
  __device__ __forceinline__ DevScene scene(int si) const {
    DevScene s = scenes[segs[si].job];
    s.nodes4 = nullptr;
    return s;
  }
  __device__ __forceinline__ RenderK params(int si) const { return ks[segs[si].job]; }
  // sample index of path p (the path's pixel travels in its throughput's w)
  __device__ __forceinline__ uint32_t sample(int si, long long p, int) const {
    const WaveSeg g = segs[si];
    return (uint32_t)(*accs[g.job].frame_base + (int)((p - g.path0) / g.P));
  }
  // batches keep k_generate_batch's queue and path state at bounce 0
  __device__ __forceinline__ long long camera_items(int) const { return 0; }
  __device__ __forceinline__ int frame0() const { return 0; }
  __device__ __forceinline__ int camera_ray(long long, int, float3&, float3&, uint32_t&, uint32_t&) const {
    return 0;
  }
};

// A batch whose scenes all have a 4-wide tree (LBVH builds): extend traverses
// that tree only.
struct BatchSrc4 : BatchSrc {
  static constexpr bool kWide = true;
  __device__ __forceinline__ DevScene scene(int si) const { return scenes[segs[si].job]; }
};

// -------------------------------------------------------------------- kernels
// Camera ray and empty path state of path p (pixel px, py; sample `frame`).
__device__ __forceinline__ void init_path(const RenderK& K, int px, int py, int frame, long long p,
                                          float4* __restrict__ ray_o, float4* __restrict__ ray_d,
                                          float4* __restrict__ thr, float4* __restrict__ rad,
                                          float4* __restrict__ gn, float4* __restrict__ ga) {
  float3 d = camera_dir(K, px, py, frame);
  ray_o[p] = make_float4(K.cam_pos.x, K.cam_pos.y, K.cam_pos.z, 1.0f);
  ray_d[p] = make_float4(d.x, d.y, d.z, 0.0f);
  thr[p] = make_float4(1.0f, 1.0f, 1.0f, __uint_as_float((uint32_t)(py * K.W + px)));  // w: the pixel
  rad[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  gn[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  ga[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

__global__ void k_generate(RenderK K, const int* __restrict__ frame_base, float4* __restrict__ ray_o,
                           float4* __restrict__ ray_d, float4* __restrict__ thr, float4* __restrict__ rad,
                           float4* __restrict__ gn, float4* __restrict__ ga, int* __restrict__ q0,
                           int* __restrict__ counters) {
  long long total = (long long)K.spf * K.P;
  int fb = *frame_base;
  long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += stride) {
    int px, py, f;
    const long long p = camera_path(K, t, px, py, f);
    init_path(K, px, py, fb + f, p, ray_o, ray_d, thr, rad, gn, ga);
    q0[t] = (int)p;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) counters[C_Q + 0] = (int)total;
}

// Segment holding position x of a sorted prefix array (path0 or acc0).
template <bool ACC>
__device__ __forceinline__ int find_seg(const WaveSeg* __restrict__ segs, int n_segs, long long x) {
  int lo = 0, hi = n_segs - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    long long v = ACC ? segs[mid].acc0 : segs[mid].path0;
    if (v <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void k_generate_batch(BatchSrc src, int n_segs, long long total, float4* __restrict__ ray_o,
                                 float4* __restrict__ ray_d, float4* __restrict__ thr, float4* __restrict__ rad,
                                 float4* __restrict__ gn, float4* __restrict__ ga, int* __restrict__ q0,
                                 int* __restrict__ pseg, int* __restrict__ counters) {
  long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += stride) {
    int si = find_seg<false>(src.segs, n_segs, t);
    WaveSeg g = src.segs[si];
    RenderK K = src.ks[g.job];
    int fb = *src.accs[g.job].frame_base;
    // the single-render order and layout per segment: samples of a pixel
    // on consecutive items, path state at path0 + f * P + strip index
    const long long l = t - g.path0;
    const int gs = group_of(g.frames);
    const long long span = (long long)gs * g.P;
    const long long c = l / span;
    const int r = (int)(l - c * span);
    const int si2 = r / gs;
    const int f = (int)(c * gs) + (r - si2 * gs);
    int px, py;
    strip_pixel(K, si2, px, py);
    long long p = g.path0 + (long long)f * g.P + si2;
    init_path(K, px, py, fb + f, p, ray_o, ray_d, thr, rad, gn, ga);
    pseg[p] = si;
    q0[t] = (int)p;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) counters[C_Q + 0] = (int)total;
}

// One extend item of shadow records: a path's shadow rays of one bounce sit
// in consecutive records; the first carries their count (the others 0) and
// this item traces them all, adding the visible contributions in light
// order.  Only this item writes the path's radiance in this launch: no
// atomics, and the sum does not depend on scheduling.  Returns the rays
// traced; job = the path's job (batches).
template <bool EXACT, class Src>
__device__ __forceinline__ int shadow_item(const Src& src, const float4* __restrict__ shadow, long long j,
                                           long long ns, float4* __restrict__ rad, int* err, int& job) {
  const float4* sp = shadow + 3 * (size_t)j;
  const int cnt = min(__float_as_int(sp[2].w), (int)(ns - j));
  if (cnt <= 0) return 0;
  const int p = __float_as_int(sp[1].w);
  const int si = src.seg(p);
  const DevScene S = src.scene(si);
  if constexpr (Src::kBatch) job = src.segs[si].job;
  float3 sum = f3(0.0f, 0.0f, 0.0f);
  bool any = false;
  for (int k = 0; k < cnt; ++k) {
    float4 s0 = sp[3 * k], s1 = sp[3 * k + 1];
    if (!scene_any<EXACT, Src::kWide>(S, xyz(s0), xyz(s1), s0.w, err)) {
      sum = any ? sum + xyz(sp[3 * k + 2]) : xyz(sp[3 * k + 2]);
      any = true;
    }
  }
  if (any) {
    float4 r = rad[p];
    rad[p] = make_float4(r.x + sum.x, r.y + sum.y, r.z + sum.z, r.w);
  }
  return cnt;
}

// 1024 resident threads per SM (64 registers): traversal is latency bound,
// and the extra warps hide more of it than the registers they cost.
// CAM: the bounce-0 launch of a single render (camera items, no shadow
// rays); the other launches are compiled without that code.
template <bool EXACT, class Src, int BS, bool CAM = false>
__global__ void __launch_bounds__(BS, 1024 / BS)
    k_extend(Src src, int b, const int* __restrict__ qin, int* counters, const float4* __restrict__ ray_o,
             const float4* __restrict__ ray_d, float4* __restrict__ hits, int sb, const float4* __restrict__ shadow,
             float4* __restrict__ rad, long long shadow_cap, int* err) {
  // Items [0, n): closest hit of bounce b's queue.  Items [n, n + ns): the
  // shadow rays bounce sb (the previous one) emitted, traced any-hit here so
  // they share this launch instead of paying for a small one of their own.
  // Camera items (bounce 0 without k_generate): item i is camera path i of
  // the wave, its ray made here; this launch also sets the bounce-0 count.
  // Nothing to do once k_tail has taken the wave over.
  if (*(volatile int*)&counters[C_TAIL]) return;
  const long long cam_n = CAM ? src.camera_items(b) : 0;
  const int fb = cam_n ? src.frame0() : 0;
  if (cam_n && blockIdx.x == 0 && threadIdx.x == 0) counters[C_Q + 0] = (int)cam_n;
  const int n = cam_n ? (int)cam_n : (b >= 0 ? *(volatile int*)&counters[C_Q + b] : 0);
  long long ns = sb >= 0 ? *(volatile int*)&counters[C_S + sb] : 0;
  if (ns > shadow_cap) ns = shadow_cap;
  const int total = n + (int)ns;
  int* fetch = &counters[C_FE + (b >= 0 ? b : kMaxBounce - 1)];
  const int lane = threadIdx.x & 31;
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(fetch, 32);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= total) break;
    int i = base + lane;
    int job = -1, rays_here = 0;
    if (i < n) {
      float3 o, d;
      int p;
      if (cam_n) {
        uint32_t pix_unused, smp_unused;
        p = src.camera_ray(i, fb, o, d, pix_unused, smp_unused);
      } else {
        p = qin[i];
        o = xyz(ray_o[p]);
        d = xyz(ray_d[p]);
      }
      const int si = src.seg(p);
      const DevScene S = src.scene(si);
      if constexpr (Src::kBatch) {
        job = src.segs[si].job;
        rays_here = 1;
      }
      SceneHit h = scene_closest<EXACT, Src::kWide>(S, o, d, err);
      int code = h.prim >= 0 ? h.prim : (h.slot >= 0 ? -(h.slot + 2) : -1);
      hits[i] = make_float4(h.t, __int_as_float(code), h.u, h.v);
    } else if (i < total) {
      // (no shadow rays precede bounce 0)
      if constexpr (!CAM) rays_here = shadow_item<EXACT>(src, shadow, i - n, ns, rad, err, job);
    }
    if constexpr (Src::kBatch) {
      // rays traced, counted per job (lanes of a warp mostly share one)
      unsigned m = __match_any_sync(0xffffffffu, job);
      int tot = __reduce_add_sync(m, rays_here);
      if (job >= 0 && lane == __ffs(m) - 1) atomicAdd(src.job_rays + job, (unsigned long long)tot);
    }
  }
}

// warp-aggregated append: one atomic per warp, ranks by ballot / popc
__device__ __forceinline__ int warp_append(bool want, int* counter) {
  unsigned m = __ballot_sync(0xffffffffu, want);
  if (!m) return -1;
  int lane = threadIdx.x & 31;
  int leader = __ffs(m) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(counter, __popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  return want ? base + __popc(m & ((1u << lane) - 1u)) : -1;
}

// warp-aggregated append of cnt >= 0 consecutive entries per lane
__device__ __forceinline__ int warp_append_n(int cnt, int* counter) {
  const int lane = threadIdx.x & 31;
  int x = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  int total = __shfl_sync(0xffffffffu, x, 31);
  int base = 0;
  if (lane == 0 && total > 0) base = atomicAdd(counter, total);
  base = __shfl_sync(0xffffffffu, base, 0);
  return base + x - cnt;
}

// Next-event estimation at a vertex (trace.py:23-93), shared by k_shade
// (which writes shadow records) and k_tail (which traces them at once).
// direct_light_mode "one": one light, picked uniformly in compat mode, by
// the alias table otherwise.  nee_p: the point lights are sampled from.
__device__ __forceinline__ bool nee_one(const DevScene& S, const RenderK& K, bool mis, PathRng& rng, float3 nee_p,
                                        float3 nrm, float3 alb, float nee_scale, float3& dir, float& max_t,
                                        float3& val) {
  int li;
  float w;
  if (K.compat) {
    int cnt = S.n_lights;
    li = min((int)(rng.get(SLOT_LIGHT_PICK) * (float)cnt), cnt - 1);
    w = (float)cnt;
  } else {
    int nl = S.n_lights;
    int col = min((int)(rng.get(SLOT_LIGHT_PICK) * (float)nl), nl - 1);
    li = rng.get(SLOT_LIGHT_ACCEPT) < __ldg(S.alias_prob + col) ? col : __ldg(S.alias_idx + col);
    w = 1.0f / S.lights[li].pick_pdf;
  }
  float pdf;
  bool ok = light_sample(S.lights[li], rng.get(SLOT_LIGHT_U1), rng.get(SLOT_LIGHT_U2), nee_p, nrm, alb, w, dir, max_t,
                         val, pdf);
  // MIS: this light sample against the BSDF lobe that NEE stands in for
  // (density nee_scale * cos / pi)
  if (ok && mis) val = val * mis_power(pdf * S.lights[li].pick_pdf, nee_scale * dot(nrm, dir) / kPi);
  return ok;
}

// direct_light_mode "all": light li with its own random slots
__device__ __forceinline__ bool nee_light(const DevScene& S, bool mis, PathRng& rng, int li, float3 nee_p, float3 nrm,
                                          float3 alb, float nee_scale, float3& dir, float& max_t, float3& val) {
  int s1 = SLOT_ALL_LIGHTS + 4 * li;
  float pdf;
  bool ok = light_sample(S.lights[li], rng.get(s1), rng.get(s1 + 1), nee_p, nrm, alb, 1.0f, dir, max_t, val, pdf);
  if (ok && mis) val = val * mis_power(pdf, nee_scale * dot(nrm, dir) / kPi);
  return ok;
}

// Radiance a visible shadow ray adds: the throughput before this vertex's
// albedo times the light sample's value (times the glossy lobe's weight).
__device__ __forceinline__ float3 nee_contribution(float3 thr_nee, float3 val, float nee_scale) {
  float3 c = thr_nee * val;
  if (nee_scale != 1.0f) c = c * nee_scale;
  return c;
}

// One path vertex (trace.py:139-236): the ray (o, d) with throughput thr
// and current index of refraction cur_ior met the hit record h = (t, code,
// u, v); prev_w is the previous vertex's NEE weight (0: no NEE there, else
// its BSDF density for MIS).  Returns the radiance to add, the next ray when
// the path goes on, and what next-event estimation at this vertex needs.
// k_shade runs it once per launch over a queue of paths, k_tail bounce after
// bounce for one path; the arithmetic is the same for both.
// `out` receives the first-hit guides (out.guides(normal + depth, albedo),
// on a surface hit) and the next ray (out.next(origin, ior, direction, NEE
// weight, throughput), when the path goes on) where they are formed, so
// k_shade stores them at once instead of keeping them in registers.
struct Vertex {
  float3 add = {0.0f, 0.0f, 0.0f};
  bool has_add = false;
  bool hit = false;  // a surface was hit
  bool alive = false;
  bool do_nee = false;
  float nee_scale = 1.0f;
  float3 hit_p = {0.0f, 0.0f, 0.0f}, nrm = {0.0f, 0.0f, 1.0f}, alb = {0.0f, 0.0f, 0.0f}, thr_nee = {0.0f, 0.0f, 0.0f};
};

template <class Out>
__device__ __forceinline__ void shade_vertex(const DevScene& S, const RenderK& K, bool mis, int b, bool last_bounce,
                                             float3 o, float3 d, float3 thr, float cur_ior, float prev_w, float4 h,
                                             PathRng& rng, Vertex& v, Out& out) {
  const bool prev_nee = prev_w != 0.0f;
  const int code = __float_as_int(h.y);
  if (code == -1) {
    // trace.py:154-159
    float3 sky;
    if (K.use_sky) {
      float t = 0.5f * (d.y + 1.0f);
      sky = f3(1.0f, 1.0f, 1.0f) * (1.0f - t) + f3(0.5f, 0.7f, 1.0f) * t;
    } else {
      sky = K.bg;
    }
    v.add = thr * sky;
    v.has_add = true;
    return;
  }
  float t = h.x;
  float3 nn;
  int m;
  int src_tri = -1;
  bool listed;
  if (code >= 0) {
    const float4* sp = S.shade + 3 * (size_t)code;
    float4 pa = __ldg(S.prims + 3 * (size_t)code);
    float4 s0 = __ldg(sp);
    m = __float_as_int(s0.w);
    if (__float_as_int(pa.w) == PRIM_TRI) {
      float w = 1.0f - h.z - h.w;
      float4 s1 = __ldg(sp + 1);
      src_tri = __float_as_int(s1.w);
      nn = normalized((xyz(s0) * w + xyz(s1) * h.z) + xyz(__ldg(sp + 2)) * h.w);
    } else {
      nn = analytic_normal(o + d * t, pa, __ldg(S.prims + 3 * (size_t)code + 1));
    }
    // triangles and spheres can be lights; cubes are not in the light list
    listed = __float_as_int(pa.w) != PRIM_CUBE;
  } else {
    const ObjSlot& ob = S.objs[-code - 2];
    m = ob.mat;
    if (ob.type == 0) nn = normalized((o + d * t) - ob.center);
    else if (ob.type == 1) nn = ob.normal;
    else if (ob.type == 2) nn = cube_normal(o + d * t, ob.center, ob.extra);
    else nn = normalized(cross(ob.v1 - ob.v0, ob.v2 - ob.v0));
    listed = ob.type == 0;
  }
  bool front = dot(nn, d) < 0.0f;
  if (!front) nn = -nn;
  const float3 hit_p = o + d * t;
  v.hit_p = hit_p;
  float4 ma = __ldg(S.mat_a + m), mb = __ldg(S.mat_b + m);
  int mt = __float_as_int(ma.w);
  float3 albedo = xyz(ma);
  float rough = mb.x, ior = mb.y, em = mb.z;
  int tex = __float_as_int(mb.w);
  if (src_tri >= 0 && tex >= 0) albedo = textured_albedo(S, src_tri, tex, h.z, h.w, albedo);
  // textured emitters are left out of the light list (their radiance
  // varies over the surface), so BSDF hits always count them
  listed = listed && mt == 3 && em > 0.0f && !(src_tri >= 0 && tex >= 0);
  v.hit = true;
  out.guides(make_float4(nn.x, nn.y, nn.z, t), make_float4(albedo.x, albedo.y, albedo.z, 0.0f));
  if (mt == 3) {
    // trace.py:194-196; with NEE on the previous diffuse vertex the
    // default estimator already counted this emitter, unless MIS
    // shares it between the two samples
    if (!(!K.compat && prev_nee && listed)) {
      v.add = (thr * albedo) * em;
      v.has_add = true;
    } else if (mis) {
      int li = -1;
      if (code >= 0)
        li = src_tri >= 0 ? __ldg(S.light_of_tri + src_tri)
                          : __ldg(S.light_of_obj + __float_as_int(__ldg(S.shade + 3 * (size_t)code + 1).w));
      else
        li = __ldg(S.light_of_lin + (-code - 2));
      if (li >= 0) {
        // prev_w: density of this direction under the previous vertex's BSDF
        const Light& L = S.lights[li];
        float pl = light_dir_pdf(L, o, d, t) * (K.mode == 0 ? L.pick_pdf : 1.0f);
        v.add = ((thr * albedo) * em) * mis_power(prev_w, pl);
        v.has_add = true;
      }
    }
    return;
  }
  bool nee_here = false;
  bool can_nee = b < K.dlmd && S.n_lights > 0;
  float3 nd = d;
  if (mt == 0) {
    if (can_nee) {
      v.do_nee = true;
      nee_here = true;
    }
    nd = diffuse_scatter(nn, rng.get(SLOT_BSDF_U1), rng.get(SLOT_BSDF_U2));
  } else if (mt == 1) {
    float3 ru = random_unit_vector(rng.get(SLOT_FUZZ_U1), rng.get(SLOT_FUZZ_U2));
    nd = normalized(reflect(d, nn) + ru * rough);
  } else if (mt == 4) {
    if (can_nee) {
      v.do_nee = true;
      v.nee_scale = rough;
    }
    if (rng.get(SLOT_LOBE) < rough) {
      nd = diffuse_scatter(nn, rng.get(SLOT_BSDF_U1), rng.get(SLOT_BSDF_U2));
      nee_here = v.do_nee;
    } else {
      float3 ru = random_unit_vector(rng.get(SLOT_FUZZ_U1), rng.get(SLOT_FUZZ_U2));
      nd = normalized(reflect(d, nn) + ru * rough);
    }
  } else if (mt == 2) {
    float eta;
    if (front) {
      eta = cur_ior / ior;
      cur_ior = ior;
    } else {
      eta = cur_ior / 1.0f;
      cur_ior = 1.0f;
    }
    float c = fminf(-dot(d, nn), 1.0f);
    float s = sqrtf(1.0f - c * c);
    bool refl = eta * s > 1.0f;
    if (!refl) refl = schlick(c, eta) > rng.get(SLOT_LOBE);
    nd = refl ? reflect(d, nn) : refract(d, nn, eta);
  }
  v.thr_nee = thr;
  thr = thr * albedo;
  v.alb = albedo;
  v.nrm = nn;
  bool alive = true;
  if (b > 2) {
    float rr = fmaxf(thr.x, fmaxf(thr.y, thr.z));
    if (rng.get(SLOT_RR) > rr) alive = false;
    else thr = thr / rr;
  }
  if (last_bounce) alive = false;
  v.alive = alive;
  if (alive) {
    // w: 0 = no NEE here; with MIS the BSDF density of nd through the lobe
    // NEE stands in for (nee_scale * cos / pi), else 1
    float nee_w = 0.0f;
    if (nee_here) nee_w = mis ? fmaxf(v.nee_scale * dot(nn, nd) / kPi, 1e-30f) : 1.0f;
    out.next(hit_p + nn * 1e-4f, cur_ior, nd, nee_w, thr);
  }
}

// k_shade's vertex output: guides of bounce 0 and the next ray go to the
// path's state at once
struct PathStateOut {
  float4* gn;
  float4* ga;
  float4* ray_o;
  float4* ray_d;
  float4* thr;
  int p, b;
  uint32_t pix;  // the path's pixel, kept in thr.w for the later bounces
  __device__ __forceinline__ void guides(float4 n, float4 a) {
    if (b == 0) {
      gn[p] = n;
      ga[p] = a;
    }
  }
  __device__ __forceinline__ void next(float3 o, float ior, float3 d, float w, float3 t) {
    ray_o[p] = make_float4(o.x, o.y, o.z, ior);
    ray_d[p] = make_float4(d.x, d.y, d.z, w);
    thr[p] = make_float4(t.x, t.y, t.z, __uint_as_float(pix));
  }
};

template <class Src>
__global__ void __launch_bounds__(128, Src::kBatch ? 5 : 1) k_shade(Src src, int b, const int* __restrict__ qin,
                                               int* __restrict__ qout, int* counters,
                                               const int* __restrict__ frame_base, float4* __restrict__ ray_o,
                                               float4* __restrict__ ray_d, float4* __restrict__ thr_b,
                                               float4* __restrict__ rad_b, float4* __restrict__ gn,
                                               float4* __restrict__ ga, const float4* __restrict__ hits,
                                               float4* __restrict__ shadow, int* err) {
  // camera items: bounce 0 without k_generate (see k_extend); the path's
  // state is the camera ray, unit throughput and no radiance yet.  Nothing
  // to do once k_tail has taken the wave over.
  if (*(volatile int*)&counters[C_TAIL]) return;
  const long long cam_n = src.camera_items(b);
  const int n = cam_n ? (int)cam_n : *(volatile int*)&counters[C_Q + b];
  const int fb = frame_base ? *frame_base : 0;
  const int lane = threadIdx.x & 31;
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(&counters[C_FS + b], 32);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n) break;
    int i = base + lane;
    bool valid = i < n;
    // lanes past the end take the first item's job (they write nothing)
    const int si = src.seg(cam_n ? 0 : qin[valid ? i : base]);
    const DevScene S = src.scene(si);
    const RenderK K = src.params(si);
    // MIS needs the emitter -> light maps (rx_scene_set_light_sources)
    const bool mis = K.mis && S.light_of_lin != nullptr;
    const bool last_bounce = (b + 1) >= K.max_depth;
    bool alive = false;
    bool do_nee = false;
    float nee_scale = 1.0f;
    int p = 0;
    float3 hit_p = f3(0, 0, 0), nrm = f3(0, 0, 1), alb = f3(0, 0, 0), thr_nee = f3(0, 0, 0);
    PathRng rng;
    if (valid) {
      float4 o4, d4, t4;
      uint32_t pix_id, smp;
      if (cam_n) {
        float3 co, cd;
        p = src.camera_ray(i, fb, co, cd, pix_id, smp);
        o4 = make_float4(co.x, co.y, co.z, 1.0f);
        d4 = make_float4(cd.x, cd.y, cd.z, 0.0f);
        t4 = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
      } else {
        p = qin[i];
        o4 = ray_o[p];
        d4 = ray_d[p];
        t4 = thr_b[p];
        pix_id = __float_as_uint(t4.w);
        smp = src.sample(si, p, fb);
      }
      const float4 h = hits[i];
      rng.init(pix_id, smp, (uint32_t)b, K.seed);
      Vertex v;
      PathStateOut out{gn, ga, ray_o, ray_d, thr_b, p, b, pix_id};
      shade_vertex(S, K, mis, b, last_bounce, xyz(o4), xyz(d4), xyz(t4), o4.w, d4.w, h, rng, v, out);
      if (!v.hit && cam_n) {  // no first hit: empty guides
        gn[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        ga[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      }
      alive = v.alive;
      do_nee = v.do_nee;
      nee_scale = v.nee_scale;
      hit_p = v.hit_p;
      nrm = v.nrm;
      alb = v.alb;
      thr_nee = v.thr_nee;
      if (cam_n) {
        rad_b[p] = make_float4(v.add.x, v.add.y, v.add.z, 0.0f);  // the path's first radiance
      } else if (v.has_add) {
        float4 r = rad_b[p];
        rad_b[p] = make_float4(r.x + v.add.x, r.y + v.add.y, r.z + v.add.z, 0.0f);
      }
    }
    // next-event estimation: shadow records for connect.  The default
    // estimator samples lights from the normal-offset point the shadow ray
    // starts at (a grazing shadow ray then cannot clip the sampled emitter's
    // own plane); reference_compat samples from the hit point as trace.py
    // does.
    const float3 nee_p = K.compat ? hit_p : hit_p + nrm * 1e-4f;
    // shadow record: (origin, t_max), (dir, path), (contribution, count),
    // count = number of this path's records starting here (0 on followers)
    auto write_rec = [&](long long slot, float3 dir, float max_t, float3 val, int count) {
      float3 so = hit_p + nrm * 1e-4f;
      float3 c = nee_contribution(thr_nee, val, nee_scale);
      float4* sp = shadow + 3 * (size_t)slot;
      sp[0] = make_float4(so.x, so.y, so.z, max_t);
      sp[1] = make_float4(dir.x, dir.y, dir.z, __int_as_float(p));
      sp[2] = make_float4(c.x, c.y, c.z, __int_as_float(count));
    };
    // direct_light_mode "one": one light picked (uniformly in compat mode,
    // by the alias table otherwise)
    auto sample_one = [&](float3& dir, float& max_t, float3& val) {
      return nee_one(S, K, mis, rng, nee_p, nrm, alb, nee_scale, dir, max_t, val);
    };
    // direct_light_mode "all": light li with its own random slots
    auto sample_li = [&](int li, float3& dir, float& max_t, float3& val) {
      return nee_light(S, mis, rng, li, nee_p, nrm, alb, nee_scale, dir, max_t, val);
    };
    bool one_light = false;  // warp-uniform: one scene, mode "one"
    if constexpr (!Src::kBatch) one_light = K.mode == 0;
    if (one_light) {
      bool emit = false;
      float3 dir = f3(0, 0, 0), val = f3(0, 0, 0);
      float max_t = 0.0f;
      if (do_nee) emit = sample_one(dir, max_t, val);
      int slot = warp_append(emit, &counters[C_S + b]);
      if (emit) {
        if (slot < K.shadow_cap) write_rec(slot, dir, max_t, val, 1);
        else atomicOr(err, ERR_SHADOW_OVERFLOW);
      }
    } else {
      // mode "all" (and batches, whose lanes may differ in mode and light
      // count): count this path's shadow rays, reserve that many consecutive
      // records, then sample again (same random numbers) to write them
      int cnt = 0;
      float3 dir0 = f3(0, 0, 0), val0 = f3(0, 0, 0);
      float mt0 = 0.0f;
      if (do_nee) {
        if (K.mode == 0) {
          cnt = sample_one(dir0, mt0, val0) ? 1 : 0;
        } else {
          for (int li = 0; li < S.n_lights; ++li) {
            float3 d, v;
            float mt;
            if (sample_li(li, d, mt, v)) ++cnt;
          }
        }
      }
      long long base = warp_append_n(cnt, &counters[C_S + b]);
      if (cnt > 0) {
        if (base + cnt <= K.shadow_cap) {
          if (K.mode == 0) {
            write_rec(base, dir0, mt0, val0, 1);
          } else {
            int k = 0;
            for (int li = 0; li < S.n_lights && k < cnt; ++li) {
              float3 d, v;
              float mt;
              if (sample_li(li, d, mt, v)) {
                write_rec(base + k, d, mt, v, k == 0 ? cnt : 0);
                ++k;
              }
            }
          }
        } else {
          atomicOr(err, ERR_SHADOW_OVERFLOW);
        }
      }
    }
    int q = warp_append(alive, &counters[C_Q + b + 1]);
    if (alive) {
      if (q < K.queue_cap) qout[q] = p;
      else atomicOr(err, ERR_QUEUE_OVERFLOW);
    }
  }
}

// k_tail's vertex output: the next ray stays in registers (no guides: the
// tail starts at bounce 1 or later)
struct RegisterOut {
  float3 o, d, t;
  float ior, w;
  __device__ __forceinline__ void guides(float4, float4) {}
  __device__ __forceinline__ void next(float3 o_, float ior_, float3 d_, float w_, float3 t_) {
    o = o_;
    ior = ior_;
    d = d_;
    w = w_;
    t = t_;
  }
};

// The tail of a wave.  Launched after bounce b's k_extend (b >= 1): when that
// bounce's queue holds at most `max_paths` paths, one thread per path shades
// bounce b from the hit record k_extend wrote, then traces, shades and runs
// next-event estimation for each of the path's remaining bounces itself,
// tracing its shadow rays at once.  Late bounces hold few, incoherent rays,
// and a one-bounce launch lasts as long as its slowest ray; this launch lasts
// as long as its slowest path.  Radiance is added in the order of the
// one-bounce launches (a bounce's emission, then its shadow rays, then the
// next bounce's), with the same random numbers and arithmetic
// (shade_vertex, nee_one / nee_light), so images and ray counts are the same
// bit for bit.  The launch that takes over sets counters[C_TAIL] = b + 1;
// the wave's later k_extend, k_shade and k_tail launches then return at once.
template <bool EXACT, class Src>
__global__ void __launch_bounds__(128) k_tail(Src src, int b, const int* __restrict__ qin, int* counters,
                                              int max_paths, const int* __restrict__ frame_base,
                                              const float4* __restrict__ ray_o, const float4* __restrict__ ray_d,
                                              const float4* __restrict__ thr_b, float4* __restrict__ rad_b,
                                              const float4* __restrict__ hits, int* err) {
  const int taken = *(volatile int*)&counters[C_TAIL];
  if (taken != 0 && taken != b + 1) return;  // an earlier bounce's launch took over
  const int n = *(volatile int*)&counters[C_Q + b];
  if (n > max_paths) return;  // the one-bounce launches go on
  // every block of this launch reads the same queue length and flag (0 or
  // b + 1), so all of them take over
  if (threadIdx.x == 0) counters[C_TAIL] = b + 1;
  const int fb = frame_base ? *frame_base : 0;
  const int lane = threadIdx.x & 31;
  int n_closest = 0, n_shadow = 0;  // rays traced here, counted as the one-bounce launches count them
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(&counters[C_FT], 32);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n) break;
    const int i = base + lane;
    int job = -1, rays_here = 0;  // batches: the rays this lane traced, counted for its job
    if (i < n) {
      const int p = qin[i];
      const int si = src.seg(p);
      const DevScene S = src.scene(si);
      const RenderK K = src.params(si);
      if constexpr (Src::kBatch) job = src.segs[si].job;
      const int closest0 = n_closest, shadow0 = n_shadow;
      const bool mis = K.mis && S.light_of_lin != nullptr;
      const float4 o4 = ray_o[p], d4 = ray_d[p], t4 = thr_b[p];
      float3 o = xyz(o4), d = xyz(d4), thr = xyz(t4);
      float ior = o4.w, w = d4.w;
      float4 h = hits[i];
      float4 r = rad_b[p];
      const uint32_t pix_id = __float_as_uint(t4.w), smp = src.sample(si, p, fb);
      for (int bb = b;; ++bb) {
        PathRng rng;
        rng.init(pix_id, smp, (uint32_t)bb, K.seed);
        Vertex v;
        RegisterOut out;
        shade_vertex(S, K, mis, bb, (bb + 1) >= K.max_depth, o, d, thr, ior, w, h, rng, v, out);
        if (v.has_add) r = make_float4(r.x + v.add.x, r.y + v.add.y, r.z + v.add.z, 0.0f);
        if (v.do_nee) {
          // the shadow rays this vertex would have written as records, traced
          // in record order and summed as the next extend launch sums them
          const float3 nee_p = K.compat ? v.hit_p : v.hit_p + v.nrm * 1e-4f;
          const float3 so = v.hit_p + v.nrm * 1e-4f;
          float3 sum = f3(0.0f, 0.0f, 0.0f);
          bool any = false;
          auto shadow_ray = [&](float3 dir, float max_t, float3 val) {
            ++n_shadow;
            if (!scene_any<EXACT, Src::kWide>(S, so, dir, max_t, err)) {
              const float3 c = nee_contribution(v.thr_nee, val, v.nee_scale);
              sum = any ? sum + c : c;
              any = true;
            }
          };
          float3 dir, val;
          float max_t;
          if (K.mode == 0) {
            if (nee_one(S, K, mis, rng, nee_p, v.nrm, v.alb, v.nee_scale, dir, max_t, val)) shadow_ray(dir, max_t, val);
          } else {
            for (int li = 0; li < S.n_lights; ++li)
              if (nee_light(S, mis, rng, li, nee_p, v.nrm, v.alb, v.nee_scale, dir, max_t, val))
                shadow_ray(dir, max_t, val);
          }
          if (any) r = make_float4(r.x + sum.x, r.y + sum.y, r.z + sum.z, r.w);
        }
        if (!v.alive) break;
        ++n_closest;
        o = out.o;
        d = out.d;
        thr = out.t;
        ior = out.ior;
        w = out.w;
        const SceneHit hh = scene_closest<EXACT, Src::kWide>(S, o, d, err);
        const int code = hh.prim >= 0 ? hh.prim : (hh.slot >= 0 ? -(hh.slot + 2) : -1);
        h = make_float4(hh.t, __int_as_float(code), hh.u, hh.v);
      }
      rad_b[p] = r;
      rays_here = (n_closest - closest0) + (n_shadow - shadow0);
    }
    if constexpr (Src::kBatch) {
      // rays traced, counted per job as k_extend counts them
      unsigned m = __match_any_sync(0xffffffffu, job);
      int tot = __reduce_add_sync(m, rays_here);
      if (job >= 0 && tot && lane == __ffs(m) - 1) atomicAdd(src.job_rays + job, (unsigned long long)tot);
    }
  }
  if constexpr (!Src::kBatch) {
    // every lane leaves the fetch loop together
    n_closest = __reduce_add_sync(0xffffffffu, n_closest);
    n_shadow = __reduce_add_sync(0xffffffffu, n_shadow);
    if (lane == 0) {
      if (n_closest) atomicAdd(&counters[C_Q + b + 1], n_closest);
      if (n_shadow) atomicAdd(&counters[C_S + b], n_shadow);
    }
  }
}

// trace.py:262-283: clamp, running mean of radiance and first-hit guides,
// display = sqrt(min(acc, 1)).  Frames of the wave are folded in order.
// One pixel: fold `spf` frames (paths path0 + f * P + src) into the running
// means, starting at frame index fb.
// src: the pixel's path index within a frame (path path0 + f * P + src);
// pix: its accumulator index.
__device__ __forceinline__ void accumulate_pixel(float clamp, int spf, int fb, long long P, long long path0,
                                                 long long src, long long pix, const float4* __restrict__ rad,
                                                 const float4* __restrict__ gn, const float4* __restrict__ ga,
                                                 const JobAcc& A) {
  float4 a = A.acc_r[pix], an = A.acc_n[pix], aa = A.acc_a[pix];
  double sx = 0.0, sy = 0.0, sz = 0.0;
  const bool f64 = A.acc64 != nullptr;
  auto fold = [&](float4 s, float4 g, float4 al, int frame) {
    if (clamp > 0.0f) {
      s.x = fminf(fmaxf(s.x, 0.0f), clamp);
      s.y = fminf(fmaxf(s.y, 0.0f), clamp);
      s.z = fminf(fmaxf(s.z, 0.0f), clamp);
    }
    if (f64) {
      sx += (double)s.x;
      sy += (double)s.y;
      sz += (double)s.z;
    }
    if (frame == 0) {
      a = make_float4(s.x, s.y, s.z, 0.0f);
      an = g;
      aa = make_float4(al.x, al.y, al.z, 0.0f);
    } else {
      const float F = (float)frame, F1 = (float)(frame + 1), r = __frcp_rn(F1);
      auto mean = [&](float acc, float smp) { return div_by(acc * F + smp, F1, r); };
      a = make_float4(mean(a.x, s.x), mean(a.y, s.y), mean(a.z, s.z), 0.0f);
      an = make_float4(mean(an.x, g.x), mean(an.y, g.y), mean(an.z, g.z), mean(an.w, g.w));
      aa = make_float4(mean(aa.x, al.x), mean(aa.y, al.y), mean(aa.z, al.z), 0.0f);
    }
  };
  // the wave's samples are read once: streaming loads, kU frames in flight
  // per thread ahead of the (sequential) running-mean updates
  constexpr int kU = 4;
  int f = 0;
  for (; f + kU <= spf; f += kU) {
    float4 s[kU], g[kU], al[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const long long p = path0 + (long long)(f + u) * P + src;
      s[u] = __ldcs(rad + p);
      g[u] = __ldcs(gn + p);
      al[u] = __ldcs(ga + p);
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) fold(s[u], g[u], al[u], fb + f + u);
  }
  for (; f < spf; ++f) {
    const long long p = path0 + (long long)f * P + src;
    fold(__ldcs(rad + p), __ldcs(gn + p), __ldcs(ga + p), fb + f);
  }
  A.acc_r[pix] = a;
  A.acc_n[pix] = an;
  A.acc_a[pix] = aa;
  if (A.acc64) {
    // float64 sums of the clamped samples (reference renders for relMSE)
    A.acc64[3 * pix] += sx;
    A.acc64[3 * pix + 1] += sy;
    A.acc64[3 * pix + 2] += sz;
  }
  A.pixels[pix] = make_float4(sqrtf(fminf(a.x, 1.0f)), sqrtf(fminf(a.y, 1.0f)), sqrtf(fminf(a.z, 1.0f)), 0.0f);
}

__global__ void k_accumulate(RenderK K, JobAcc A, const float4* __restrict__ rad, const float4* __restrict__ gn,
                             const float4* __restrict__ ga) {
  int fb = *A.frame_base;
  // pixels in strip order: a frame's samples are read contiguously
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < K.P;
       s += (long long)gridDim.x * blockDim.x) {
    int px, py;
    strip_pixel(K, s, px, py);
    accumulate_pixel(K.clamp, K.spf, fb, K.P, 0, s, (long long)py * K.W + px, rad, gn, ga, A);
  }
}

__global__ void k_accumulate_batch(BatchSrc src, int n_segs, long long total, const float4* __restrict__ rad,
                                   const float4* __restrict__ gn, const float4* __restrict__ ga) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    int si = find_seg<true>(src.segs, n_segs, t);
    WaveSeg g = src.segs[si];
    JobAcc A = src.accs[g.job];
    // pixels in strip order, as the segment's path state is laid out
    const RenderK& K = src.ks[g.job];
    int px, py;
    strip_pixel(K, t - g.acc0, px, py);
    accumulate_pixel(K.clamp, g.frames, *A.frame_base, g.P, g.path0, t - g.acc0, (long long)py * K.W + px, rad, gn,
                     ga, A);
  }
}

// After a batch wave: each job's frame base and ray count advance.
__global__ void k_finish_batch(BatchSrc src, int n_segs) {
  for (int si = blockIdx.x * blockDim.x + threadIdx.x; si < n_segs; si += gridDim.x * blockDim.x) {
    WaveSeg g = src.segs[si];
    const JobAcc& A = src.accs[g.job];
    *A.frame_base += g.frames;
    *A.rays += src.job_rays[g.job];
    src.job_rays[g.job] = 0;
  }
}

__global__ void k_finish(const int* __restrict__ counters, int max_depth, int* __restrict__ frame_base,
                         unsigned long long* __restrict__ rays, int spf) {
  unsigned long long r = 0;
  for (int b = 0; b < max_depth; ++b) r += (unsigned long long)counters[C_Q + b] + (unsigned long long)counters[C_S + b];
  *rays += r;
  *frame_base += spf;
}

__global__ void k_pack(long long P, const float4* __restrict__ src, int comp, float* __restrict__ dst) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P; i += (long long)gridDim.x * blockDim.x) {
    float4 v = src[i];
    if (comp == 1) {
      dst[i] = v.w;
    } else {
      dst[3 * i] = v.x;
      dst[3 * i + 1] = v.y;
      dst[3 * i + 2] = v.z;
    }
  }
}

// -------------------------------------------------------------------- host
enum { K_EXTEND = 0, K_SHADE = 1, K_CONNECT = 2, K_OTHER = 3, K_ACCUM = 4, K_CLASSES = 5 };

struct Accum {
  Ctx* ctx = nullptr;
  int W = 0, H = 0;
  long long P = 0;
  DevBuf<float4> acc_r, acc_n, acc_a, pixels;
  DevBuf<double> acc64;  // optional float64 radiance sums (3 per pixel)
  DevBuf<int> frame_base;
  DevBuf<unsigned long long> rays;
  int frames = 0;
  // wavefront state
  long long cap = 0, shadow_cap = 0;
  DevBuf<float4> ray_o, ray_d, thr, rad, gn, ga, hits, shadow;
  DevBuf<int> q0, q1, counters;
  // graph cache
  cudaGraphExec_t gexec = nullptr;
  bool g_timed = false;
  Scene* g_scene = nullptr;
  uint64_t g_ver = 0;
  rx_render_params g_params;
  int g_spf = 0;
  int g_launches = 0;
  int g_events = 0;  // timing events the captured wave records
  // reset / render return once queued (errors surface at rx_ctx_sync)
  bool async = false;
  // timing
  int timing = 0;
  std::vector<cudaEvent_t> ev;
  std::vector<int> ev_class;
  float last_ms = 0.0f;
  float last_k[K_CLASSES] = {0, 0, 0, 0, 0};
  int last_launches = 0;
  // denoise scratch
  DevBuf<float4> dn0, dn1, dn_out;
  int occ_ext = 0, occ_shade = 0, occ_tail = 0;
  // k_tail takes a wave over at the first bounce (>= 1) whose queue holds at
  // most this many paths; 0: never
  int tail_paths = kTailPaths;

  void drop_graph() {
    if (gexec) cudaGraphExecDestroy(gexec);
    gexec = nullptr;
  }
  ~Accum() {
    drop_graph();
    for (auto e : ev) cudaEventDestroy(e);
  }
};

// Device buffer -> caller's host memory through the context's pinned buffer,
// the DMA of later pieces overlapping the threaded copy-out of earlier ones.
static int read_to_host(Accum* a, void* host_out, const void* dev, size_t bytes) {
  return download_staged(a->ctx, host_out, dev, bytes);
}

Accum* accum_new(Ctx* ctx, int w, int h) {
  Accum* a = new Accum();
  a->ctx = ctx;
  a->W = w;
  a->H = h;
  a->P = (long long)w * h;
  bool ok = a->acc_r.alloc(ctx, a->P) && a->acc_n.alloc(ctx, a->P) && a->acc_a.alloc(ctx, a->P) &&
            a->pixels.alloc(ctx, a->P) && a->frame_base.alloc(ctx, 1) && a->rays.alloc(ctx, 1) &&
            a->counters.alloc(ctx, C_N);
  if (!ok) {
    delete a;
    return nullptr;
  }
  accum_reset(a);
  return a;
}

void accum_delete(Accum* a) { delete a; }

int accum_reset(Accum* a) {
  Ctx* ctx = a->ctx;
  cudaStream_t st = ctx->stream;
  cudaMemsetAsync(a->acc_r.p, 0, a->acc_r.bytes(), st);
  cudaMemsetAsync(a->acc_n.p, 0, a->acc_n.bytes(), st);
  cudaMemsetAsync(a->acc_a.p, 0, a->acc_a.bytes(), st);
  cudaMemsetAsync(a->pixels.p, 0, a->pixels.bytes(), st);
  if (a->acc64.p) cudaMemsetAsync(a->acc64.p, 0, a->acc64.bytes(), st);
  cudaMemsetAsync(a->frame_base.p, 0, sizeof(int), st);
  cudaMemsetAsync(a->rays.p, 0, sizeof(unsigned long long), st);
  a->frames = 0;
  if (a->async) return RX_OK;
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return RX_OK;
}

static RenderK make_k(const rx_render_params* p, const Accum* a, int spf, long long shadow_cap) {
  RenderK K;
  K.W = p->width;
  K.H = p->height;
  K.P = (long long)p->width * p->height;
  K.spf = spf;
  K.fov_tan = p->fov_tan;
  K.aspect = p->aspect;
  K.cam_pos = f3(p->cam_pos[0], p->cam_pos[1], p->cam_pos[2]);
  K.cam_fwd = f3(p->cam_fwd[0], p->cam_fwd[1], p->cam_fwd[2]);
  K.cam_right = f3(p->cam_right[0], p->cam_right[1], p->cam_right[2]);
  K.cam_up = f3(p->cam_up[0], p->cam_up[1], p->cam_up[2]);
  K.max_depth = p->max_depth;
  K.use_sky = p->use_sky;
  K.bg = f3(p->bg[0], p->bg[1], p->bg[2]);
  K.mode = p->direct_light_mode;
  K.dlmd = p->direct_light_max_depth;
  K.clamp = p->sample_clamp;
  K.compat = p->reference_compat;
  K.mis = p->reference_compat ? 0 : p->mis;
  // single renders make bounce 0's camera rays in place (batches and
  // zero-bounce renders run k_generate)
  K.camera0 = p->max_depth > 0 ? 1 : 0;
  K.seed = p->seed;
  K.shadow_cap = shadow_cap;
  K.queue_cap = a->cap;
  return K;
}

static int blocks_for(Ctx* ctx, const void* fn, int block) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, 0);
  if (per_sm < 1) per_sm = 1;
  return per_sm * ctx->num_sms;
}

static void launch_extend(Accum* a, const DevScene& S, const RenderK& K, int b, const int* qin, int sb) {
  Ctx* ctx = a->ctx;
  SingleSrc src{S, K, a->frame_base.p};
  auto go = [&](auto kernel) {
    kernel<<<a->occ_ext, 128, 0, ctx->stream>>>(src, b, qin, a->counters.p, a->ray_o.p, a->ray_d.p, a->hits.p, sb,
                                                 a->shadow.p, a->rad.p, K.shadow_cap, ctx->d_err);
  };
  const bool cam = b == 0 && K.camera0;
  if (S.exact_slab) {
    if (cam) go(k_extend<true, SingleSrc, 128, true>);
    else go(k_extend<true, SingleSrc, 128>);
  } else {
    if (cam) go(k_extend<false, SingleSrc, 128, true>);
    else go(k_extend<false, SingleSrc, 128>);
  }
}

static void launch_tail(Accum* a, const DevScene& S, const RenderK& K, int b, const int* qin) {
  Ctx* ctx = a->ctx;
  SingleSrc src{S, K, a->frame_base.p};
  auto go = [&](auto kernel) {
    kernel<<<a->occ_tail, 128, 0, ctx->stream>>>(src, b, qin, a->counters.p, a->tail_paths, a->frame_base.p,
                                                  a->ray_o.p, a->ray_d.p, a->thr.p, a->rad.p, a->hits.p, ctx->d_err);
  };
  if (S.exact_slab) go(k_tail<true, SingleSrc>);
  else go(k_tail<false, SingleSrc>);
}

// Records the launch sequence of one wave on the context stream.  With
// `timed`, an event is recorded after every kernel (class in ev_class).
static void enqueue_wave(Accum* a, Scene* sc, const RenderK& K, bool timed, int* n_launch, int* n_events) {
  Ctx* ctx = a->ctx;
  cudaStream_t st = ctx->stream;
  DevScene S = sc->view();
  int launches = 0;
  int ev_i = 0;
  auto mark = [&](int cls) {
    if (timed) {
      // External: inside stream capture this becomes an event-record node
      cudaEventRecordWithFlags(a->ev[ev_i], st, cudaEventRecordExternal);
      a->ev_class[ev_i] = cls;
      ++ev_i;
    }
  };
  mark(K_OTHER);
  cudaMemsetAsync(a->counters.p, 0, sizeof(int) * C_N, st);
  if (!K.camera0) {
    long long total = (long long)K.spf * K.P;
    int gblocks = (int)std::min<long long>((total + 255) / 256, (long long)ctx->num_sms * 16);
    k_generate<<<std::max(gblocks, 1), 256, 0, st>>>(K, a->frame_base.p, a->ray_o.p, a->ray_d.p, a->thr.p,
                                                      a->rad.p, a->gn.p, a->ga.p, a->q0.p, a->counters.p);
    ++launches;
  }
  mark(K_OTHER);
  for (int b = 0; b < K.max_depth; ++b) {
    const int* qin = (b & 1) ? a->q1.p : a->q0.p;
    int* qout = (b & 1) ? a->q0.p : a->q1.p;
    // the previous bounce's shadow rays ride along in this extend launch
    int sb = (b >= 1 && b - 1 < K.dlmd && S.n_lights > 0) ? b - 1 : -1;
    launch_extend(a, S, K, b, qin, sb);
    ++launches;
    mark(K_EXTEND);
    if (b >= 1 && a->tail_paths > 0) {
      // takes the wave over once the queue is short (then the launches
      // below return at once); its time counts as extend time
      launch_tail(a, S, K, b, qin);
      ++launches;
      mark(K_EXTEND);
    }
    k_shade<SingleSrc><<<a->occ_shade, 128, 0, st>>>(SingleSrc{S, K, a->frame_base.p}, b, qin, qout, a->counters.p,
                                                      a->frame_base.p, a->ray_o.p, a->ray_d.p, a->thr.p, a->rad.p,
                                                      a->gn.p, a->ga.p, a->hits.p, a->shadow.p, ctx->d_err);
    ++launches;
    mark(K_SHADE);
  }
  if (K.max_depth > 0 && K.max_depth - 1 < K.dlmd && S.n_lights > 0) {
    // shadow rays of the last bounce: an extend launch with no bounce rays
    launch_extend(a, S, K, -1, nullptr, K.max_depth - 1);
    ++launches;
    mark(K_CONNECT);
  }
  int ablocks = (int)std::min<long long>((K.P + 255) / 256, (long long)ctx->num_sms * 16);
  JobAcc A{a->acc_r.p, a->acc_n.p, a->acc_a.p, a->pixels.p, a->acc64.p, a->frame_base.p, a->rays.p};
  k_accumulate<<<std::max(ablocks, 1), 256, 0, st>>>(K, A, a->rad.p, a->gn.p, a->ga.p);
  mark(K_ACCUM);
  k_finish<<<1, 1, 0, st>>>(a->counters.p, K.max_depth, a->frame_base.p, a->rays.p, K.spf);
  launches += 2;
  mark(K_OTHER);
  *n_launch = launches;
  *n_events = ev_i;
}

static int ensure_wave_buffers(Accum* a, long long cap, long long shadow_cap) {
  Ctx* ctx = a->ctx;
  if (cap > a->cap) {
    a->drop_graph();
    bool ok = a->ray_o.alloc(ctx, cap) && a->ray_d.alloc(ctx, cap) && a->thr.alloc(ctx, cap) &&
              a->rad.alloc(ctx, cap) && a->gn.alloc(ctx, cap) && a->ga.alloc(ctx, cap) &&
              a->hits.alloc(ctx, cap) && a->q0.alloc(ctx, cap) && a->q1.alloc(ctx, cap);
    if (!ok) {
      a->cap = 0;
      set_error(ctx, "out of device memory for %lld wavefront paths", cap);
      return RX_ERR_CAPACITY;
    }
    a->cap = cap;
  }
  if (shadow_cap > a->shadow_cap) {
    a->drop_graph();
    if (!a->shadow.alloc(ctx, (size_t)3 * shadow_cap)) {
      a->shadow_cap = 0;
      set_error(ctx, "out of device memory for %lld shadow rays", shadow_cap);
      return RX_ERR_CAPACITY;
    }
    a->shadow_cap = shadow_cap;
  }
  if (!a->occ_ext) {
    a->occ_ext = blocks_for(ctx, (const void*)k_extend<false, SingleSrc, 128>, 128);
    a->occ_shade = blocks_for(ctx, (const void*)k_shade<SingleSrc>, 128);
    a->occ_tail = blocks_for(ctx, (const void*)k_tail<false, SingleSrc>, 128);
  }
  return RX_OK;
}

static int check_device_error(Ctx* ctx) {
  int e = 0;
  CUDA_TRY(ctx, cudaMemcpyAsync(&e, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (e) {
    cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream);
    set_error(ctx, "device error flags 0x%x (stack/queue/shadow overflow)", e);
    return RX_ERR_DEVICE;
  }
  return RX_OK;
}

int render(Scene* sc, Accum* a, const rx_render_params* p, int frames) {
  Ctx* ctx = a->ctx;
  if (!p || frames < 0) return set_error(ctx, "render: bad arguments"), RX_ERR_ARG;
  if (p->width != a->W || p->height != a->H)
    return set_error(ctx, "render: %dx%d does not match the accumulator %dx%d", p->width, p->height, a->W, a->H),
           RX_ERR_ARG;
  if (p->max_depth < 0 || p->max_depth > kMaxBounce - 1)
    return set_error(ctx, "render: max_depth must be in [0, %d]", kMaxBounce - 1), RX_ERR_ARG;
  if (p->direct_light_mode != 0 && p->direct_light_mode != 1)
    return set_error(ctx, "direct_light_mode must be 'one' or 'all'"), RX_ERR_ARG;
  if (sc->n_tris > 0 && sc->n_nodes == 0) return set_error(ctx, "render: scene has triangles but no BVH"), RX_ERR_STATE;
  if (frames == 0) return RX_OK;
  int rc = sc->upload_palette(ctx);
  if (rc) return rc;
  // Paths per wavefront.  Each extend launch ends in a tail where the last,
  // longest rays run on an emptying GPU; larger waves amortise it (measured on
  // the 1080p 64-spp icosphere scene, extend / frame time: 16 M paths 43.7 /
  // 58.2 ms, 32 M 35.1 / 47.6 ms, 64 M 30.7 / 42.7 ms, 128 M (the whole
  // frame in one wave) 28.0 / 39.9 ms).  By default the wave is the largest
  // power of two from 32 M to 128 M paths whose state (path SoA, queues,
  // hit and shadow records: ~120 B + 48 B per shadow record slot) fits in a
  // quarter of the free device memory; 128 M paths hold ~22 GB.
  long long target = p->wave_paths;
  if (target <= 0) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
      cudaGetLastError();
      free_b = 0;
    }
    const long long per_path = 120 + 48LL * (p->direct_light_mode == 1 ? std::max(sc->n_lights, 1) : 1);
    target = 1LL << 27;
    while (target > (1LL << 25) && (long long)(free_b / 4) < target * per_path) target >>= 1;
  }
  int spf = (int)std::max<long long>(1, std::min<long long>(frames, target / std::max<long long>(a->P, 1)));
  long long cap = (long long)spf * a->P;
  if (cap >= (1LL << 31)) return set_error(ctx, "render: wavefront of %lld paths is too large", cap), RX_ERR_CAPACITY;
  int nl = sc->n_lights;
  long long shadow_cap = cap * (p->direct_light_mode == 1 ? std::max(nl, 1) : 1);
  rc = ensure_wave_buffers(a, cap, shadow_cap);
  if (rc) return rc;
  if (p->max_depth == 0) {
    // no bounce: every sample is black (the reference's loop never runs)
  }
  bool timed = a->timing != 0;
  int max_events = 4 + 3 * std::max(p->max_depth, 1) + 4;
  if (timed && (int)a->ev.size() < max_events) {
    for (int i = (int)a->ev.size(); i < max_events; ++i) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      a->ev.push_back(e);
    }
    a->ev_class.resize(a->ev.size());
    a->drop_graph();
  }
  cudaStream_t st = ctx->stream;
  float k_ms[K_CLASSES] = {0, 0, 0, 0, 0};
  float total_ms = 0.0f;
  int launches_total = 0;
  int remaining = frames;
  while (remaining > 0) {
    int k = std::min(spf, remaining);
    RenderK K = make_k(p, a, k, shadow_cap);
    int nlaunch = 0, nevent = 0;
    if (k == spf) {
      bool cached = a->gexec && a->g_scene == sc && a->g_ver == sc->version && a->g_spf == spf &&
                    a->g_timed == timed && std::memcmp(&a->g_params, p, sizeof(*p)) == 0;
      if (!cached) {
        cudaGraph_t g;
        CUDA_TRY(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        enqueue_wave(a, sc, K, timed, &nlaunch, &nevent);
        CUDA_TRY(ctx, cudaStreamEndCapture(st, &g));
        // same launch sequence with new arguments (another scene, other
        // parameters): update the executable graph in place, else rebuild it
        bool updated = false;
        if (a->gexec) {
          cudaGraphExecUpdateResultInfo info;
          updated = cudaGraphExecUpdate(a->gexec, g, &info) == cudaSuccess;
          if (!updated) {
            cudaGetLastError();
            a->drop_graph();
          }
        }
        if (!updated) {
          cudaError_t e = cudaGraphInstantiate(&a->gexec, g, 0);
          if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            a->gexec = nullptr;
            CUDA_TRY(ctx, e);
          }
        }
        cudaGraphDestroy(g);
        a->g_scene = sc;
        a->g_ver = sc->version;
        a->g_spf = spf;
        a->g_timed = timed;
        a->g_params = *p;
        a->g_launches = nlaunch;
        a->g_events = nevent;
      }
      nlaunch = a->g_launches;
      nevent = a->g_events;
      CUDA_TRY(ctx, cudaGraphLaunch(a->gexec, st));
    } else {
      enqueue_wave(a, sc, K, timed, &nlaunch, &nevent);
    }
    launches_total += nlaunch;
    if (timed) {
      CUDA_TRY(ctx, cudaStreamSynchronize(st));
      // events: start, after generate, after each bounce kernel (extend,
      // tail, shade), after the last shadow rays, accumulate and finish;
      // interval i - 1 -> i counts for the class of the kernel ending at i
      for (int i = 1; i < nevent; ++i) {
        float ms = 0.0f;
        CUDA_TRY(ctx, cudaEventElapsedTime(&ms, a->ev[i - 1], a->ev[i]));
        k_ms[a->ev_class[i]] += ms;
        total_ms += ms;
      }
    }
    remaining -= k;
  }
  a->frames += frames;
  a->last_launches = launches_total;
  if (timed) {
    a->last_ms = total_ms;
    for (int i = 0; i < K_CLASSES; ++i) a->last_k[i] = k_ms[i];
  }
  if (a->async && !timed) {
    CUDA_TRY(ctx, cudaGetLastError());
    return RX_OK;
  }
  return check_device_error(ctx);
}

int accum_read(Accum* a, int which, float* host_out) {
  Ctx* ctx = a->ctx;
  const float4* src = nullptr;
  int comp = 3;
  switch (which) {
    case RX_ACC_RADIANCE: src = a->acc_r.p; break;
    case RX_ACC_NORMAL: src = a->acc_n.p; break;
    case RX_ACC_ALBEDO: src = a->acc_a.p; break;
    case RX_ACC_DEPTH: src = a->acc_n.p; comp = 1; break;
    case RX_ACC_DISPLAY: src = a->pixels.p; break;
    default: return set_error(ctx, "accum_read: unknown buffer %d", which), RX_ERR_ARG;
  }
  DevBuf<float> tmp(ctx, (size_t)a->P * comp);
  if (!tmp.ok()) return set_error(ctx, "accum_read: out of device memory"), RX_ERR_CAPACITY;
  int blocks = (int)std::min<long long>((a->P + 255) / 256, (long long)ctx->num_sms * 16);
  k_pack<<<std::max(blocks, 1), 256, 0, ctx->stream>>>(a->P, src, comp, tmp.p);
  return read_to_host(a, host_out, tmp.p, tmp.bytes());
}

int accum_set_f64(Accum* a, int on) {
  Ctx* ctx = a->ctx;
  if (on && !a->acc64.p) {
    if (a->frames != 0)
      return set_error(ctx, "accum_set_f64: enable float64 sums before the first frame (reset first)"),
             RX_ERR_ARG;
    if (!a->acc64.alloc(ctx, 3 * (size_t)a->P))
      return set_error(ctx, "accum_set_f64: out of device memory"), RX_ERR_CAPACITY;
    CUDA_TRY(ctx, cudaMemsetAsync(a->acc64.p, 0, a->acc64.bytes(), ctx->stream));
  } else if (!on) {
    a->acc64.release();
  }
  a->drop_graph();  // k_accumulate's arguments changed
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return RX_OK;
}

int accum_read_f64(Accum* a, double* host_out) {
  Ctx* ctx = a->ctx;
  if (!a->acc64.p) return set_error(ctx, "accum_read_f64: float64 sums are not enabled"), RX_ERR_ARG;
  int fb = 0;
  CUDA_TRY(ctx, cudaMemcpyAsync(&fb, a->frame_base.p, sizeof(fb), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(ctx, cudaMemcpyAsync(host_out, a->acc64.p, a->acc64.bytes(), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (fb > 0) {
    double inv = 1.0 / (double)fb;
    for (size_t i = 0; i < a->acc64.n; ++i) host_out[i] *= inv;
  }
  return RX_OK;
}

int accum_info(Accum* a, int* w, int* h, int* frames, long long* rays) {
  Ctx* ctx = a->ctx;
  unsigned long long r = 0;
  int fb = 0;
  CUDA_TRY(ctx, cudaMemcpyAsync(&r, a->rays.p, sizeof(r), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(ctx, cudaMemcpyAsync(&fb, a->frame_base.p, sizeof(fb), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (w) *w = a->W;
  if (h) *h = a->H;
  if (frames) *frames = fb;
  if (rays) *rays = (long long)r;
  return RX_OK;
}

int accum_set_timing(Accum* a, int on) {
  a->timing = on;
  return RX_OK;
}

int accum_set_async(Accum* a, int on) {
  a->async = on != 0;
  return RX_OK;
}

int accum_set_tail(Accum* a, int max_paths) {
  if (max_paths < 0) return set_error(a->ctx, "accum_set_tail: max_paths must be >= 0"), RX_ERR_ARG;
  if (max_paths != a->tail_paths) a->drop_graph();  // the graph holds the launches
  a->tail_paths = max_paths;
  return RX_OK;
}

int accum_last_timing(Accum* a, float* ms_total, float* ms_kernels, int n_kernels, int* launches) {
  if (ms_total) *ms_total = a->last_ms;
  for (int i = 0; i < n_kernels && i < K_CLASSES; ++i) ms_kernels[i] = a->last_k[i];
  if (launches) *launches = a->last_launches;
  return RX_OK;
}

int accum_denoise(Accum* a, const rx_denoise_params* dp, float* host_out) {
  Ctx* ctx = a->ctx;
  if (!a->dn0.p) {
    if (!a->dn0.alloc(ctx, a->P) || !a->dn1.alloc(ctx, a->P) || !a->dn_out.alloc(ctx, a->P))
      return set_error(ctx, "out of device memory for denoise buffers"), RX_ERR_CAPACITY;
  }
  int rc = denoise_device(ctx, a->H, a->W, a->acc_r.p, a->acc_n.p, a->acc_a.p, dp->use_normal, dp->use_albedo,
                          dp->use_depth, dp, a->dn_out.p, a->dn0.p, a->dn1.p, dp->to_display);
  if (rc) return rc;
  if (host_out) {
    DevBuf<float> tmp(ctx, (size_t)a->P * 3);
    if (!tmp.ok()) return set_error(ctx, "accum_denoise: out of device memory"), RX_ERR_CAPACITY;
    int blocks = (int)std::min<long long>((a->P + 255) / 256, (long long)ctx->num_sms * 16);
    k_pack<<<std::max(blocks, 1), 256, 0, ctx->stream>>>(a->P, a->dn_out.p, 3, tmp.p);
    CUDA_TRY(ctx, cudaMemcpyAsync(host_out, tmp.p, tmp.bytes(), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return RX_OK;
}

// ------------------------------------------------------------------ batches
// Many (scene, accumulator, parameters, frames) jobs rendered as shared
// wavefronts: each wave packs frames of several jobs into one path space, so
// one extend and one shade launch per bounce serve every scene, short jobs
// leave the queues early and small images no longer pay a launch sequence
// each.  All waves of a render call are captured into one CUDA graph.  A
// job's random numbers are keyed exactly as in a render of its own, so its
// result does not depend on what it is batched with.
struct BatchJob {
  Scene* sc;
  Accum* acc;
  rx_render_params p;
  int frames;
};

struct PlannedWave {
  int seg0, nseg;
  long long paths, acc_threads, shadow;
  int max_depth;
};

struct Batch {
  Ctx* ctx = nullptr;
  std::vector<BatchJob> jobs;
  long long wave_paths = 1LL << 25;
  int ext_block = 128;
  int tail_paths = kTailPaths;  // k_tail's threshold (0: never)
  bool use_graph = true;
  long long cap = 0, shadow_cap = 0;
  DevBuf<float4> ray_o, ray_d, thr, rad, gn, ga, hits, shadow;
  DevBuf<int> q0, q1, counters, pseg;
  DevBuf<DevScene> d_scenes;
  DevBuf<RenderK> d_ks;
  DevBuf<JobAcc> d_accs;
  DevBuf<unsigned long long> d_job_rays;
  DevBuf<WaveSeg> d_segs;
  cudaGraphExec_t gexec = nullptr;
  std::vector<unsigned char> g_key;
  int g_launches = 0, g_waves = 0;
  float last_ms = 0.0f;
  int last_waves = 0, last_launches = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  void drop_graph() {
    if (gexec) cudaGraphExecDestroy(gexec);
    gexec = nullptr;
    g_key.clear();
  }
  ~Batch() {
    drop_graph();
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
};

Batch* batch_new(Ctx* ctx) {
  Batch* b = new Batch();
  b->ctx = ctx;
  return b;
}

void batch_delete(Batch* b) { delete b; }

int batch_clear(Batch* b) {
  b->jobs.clear();
  return RX_OK;
}

int batch_add(Batch* b, Scene* sc, Accum* acc, const rx_render_params* p, int frames, int* job) {
  Ctx* ctx = b->ctx;
  if (!sc || !acc || !p || frames < 0) return set_error(ctx, "batch_add: bad arguments"), RX_ERR_ARG;
  // scenes may come from another context of the same device (built on its
  // stream, which its builders synchronise); accumulators are this context's
  if (sc->ctx->device != ctx->device || acc->ctx != ctx)
    return set_error(ctx, "batch_add: job on another device or context"), RX_ERR_ARG;
  if (p->width != acc->W || p->height != acc->H)
    return set_error(ctx, "batch_add: %dx%d does not match the accumulator %dx%d", p->width, p->height, acc->W,
                     acc->H),
           RX_ERR_ARG;
  if (p->max_depth < 0 || p->max_depth > kMaxBounce - 1)
    return set_error(ctx, "batch_add: max_depth must be in [0, %d]", kMaxBounce - 1), RX_ERR_ARG;
  if (p->direct_light_mode != 0 && p->direct_light_mode != 1)
    return set_error(ctx, "direct_light_mode must be 'one' or 'all'"), RX_ERR_ARG;
  for (const BatchJob& j : b->jobs)
    if (j.acc == acc) return set_error(ctx, "batch_add: two jobs share one accumulator"), RX_ERR_ARG;
  b->jobs.push_back(BatchJob{sc, acc, *p, frames});
  *job = (int)b->jobs.size() - 1;
  return RX_OK;
}

int batch_set_config(Batch* b, long long wave_paths, int ext_block) {
  if (wave_paths < 1 || wave_paths >= (1LL << 31))
    return set_error(b->ctx, "batch_set_config: wave_paths out of range"), RX_ERR_ARG;
  if (ext_block != 64 && ext_block != 128 && ext_block != 256)
    return set_error(b->ctx, "batch_set_config: extend block must be 64, 128 or 256"), RX_ERR_ARG;
  if (wave_paths != b->wave_paths || ext_block != b->ext_block) b->drop_graph();
  b->wave_paths = wave_paths;
  b->ext_block = ext_block;
  return RX_OK;
}

int batch_set_tail(Batch* b, int max_paths) {
  if (max_paths < 0) return set_error(b->ctx, "batch_set_tail: max_paths must be >= 0"), RX_ERR_ARG;
  if (max_paths != b->tail_paths) b->drop_graph();
  b->tail_paths = max_paths;
  return RX_OK;
}

static std::vector<PlannedWave> plan_waves(const Batch* b, std::vector<WaveSeg>& segs) {
  std::vector<PlannedWave> waves;
  std::vector<int> rem(b->jobs.size());
  for (size_t j = 0; j < b->jobs.size(); ++j) rem[j] = b->jobs[j].frames;
  for (;;) {
    PlannedWave w{(int)segs.size(), 0, 0, 0, 0, 0};
    long long left = b->wave_paths;
    for (size_t j = 0; j < b->jobs.size() && left > 0; ++j) {
      if (rem[j] == 0) continue;
      const BatchJob& J = b->jobs[j];
      long long P = (long long)J.p.width * J.p.height;
      if (P == 0) {
        rem[j] = 0;
        continue;
      }
      if (w.nseg > 0 && P > left) continue;
      int k = (int)std::max<long long>(1, std::min<long long>(rem[j], left / P));
      segs.push_back(WaveSeg{w.paths, w.acc_threads, P, k, (int)j});
      ++w.nseg;
      w.paths += k * P;
      w.acc_threads += P;
      left -= k * P;
      rem[j] -= k;
      int nl = J.sc->n_lights;
      w.shadow += k * P * (J.p.direct_light_mode == 1 ? std::max(nl, 1) : 1);
      w.max_depth = std::max(w.max_depth, J.p.max_depth);
    }
    if (w.nseg == 0) break;
    waves.push_back(w);
  }
  return waves;
}

template <int BS>
static void launch_extend_batch(Batch* B, const BatchSrc& src, bool wide, int occ, int b, const int* qin, int sb) {
  auto go = [&](auto kernel, const auto& s) {
    kernel<<<occ, BS, 0, B->ctx->stream>>>(s, b, qin, B->counters.p, B->ray_o.p, B->ray_d.p, B->hits.p, sb,
                                           B->shadow.p, B->rad.p, B->shadow_cap, B->ctx->d_err);
  };
  if (wide) go(k_extend<false, BatchSrc4, BS>, BatchSrc4{src});
  else go(k_extend<false, BatchSrc, BS>, src);
}

template <class S>
static int batch_ext_blocks_t(Ctx* ctx, int bs) {
  if (bs == 64) return blocks_for(ctx, (const void*)k_extend<false, S, 64>, 64);
  if (bs == 256) return blocks_for(ctx, (const void*)k_extend<false, S, 256>, 256);
  return blocks_for(ctx, (const void*)k_extend<false, S, 128>, 128);
}

static int batch_ext_blocks(Ctx* ctx, int bs, bool wide) {
  return wide ? batch_ext_blocks_t<BatchSrc4>(ctx, bs) : batch_ext_blocks_t<BatchSrc>(ctx, bs);
}

static void enqueue_batch(Batch* B, const std::vector<PlannedWave>& waves, int* n_launch) {
  Ctx* ctx = B->ctx;
  cudaStream_t st = ctx->stream;
  // the 4-wide traversal when every scene of the batch has that tree
  bool wide = true;
  for (const BatchJob& j : B->jobs) wide = wide && j.sc->n_nodes4 > 0 && !j.sc->exact_slab;
  int occ_ext = batch_ext_blocks(ctx, B->ext_block, wide);
  int occ_shade = blocks_for(ctx, (const void*)k_shade<BatchSrc>, 128);
  int occ_tail = wide ? blocks_for(ctx, (const void*)k_tail<false, BatchSrc4>, 128)
                      : blocks_for(ctx, (const void*)k_tail<false, BatchSrc>, 128);
  int launches = 0;
  for (const PlannedWave& w : waves) {
    BatchSrc src{B->pseg.p, B->d_segs.p + w.seg0, B->d_scenes.p, B->d_ks.p, B->d_accs.p, B->d_job_rays.p};
    cudaMemsetAsync(B->counters.p, 0, sizeof(int) * C_N, st);
    int gblocks = (int)std::min<long long>((w.paths + 255) / 256, (long long)ctx->num_sms * 16);
    k_generate_batch<<<std::max(gblocks, 1), 256, 0, st>>>(src, w.nseg, w.paths, B->ray_o.p, B->ray_d.p, B->thr.p,
                                                            B->rad.p, B->gn.p, B->ga.p, B->q0.p, B->pseg.p,
                                                            B->counters.p);
    ++launches;
    auto ext = [&](int b, const int* qin, int sb) {
      if (B->ext_block == 64) launch_extend_batch<64>(B, src, wide, occ_ext, b, qin, sb);
      else if (B->ext_block == 256) launch_extend_batch<256>(B, src, wide, occ_ext, b, qin, sb);
      else launch_extend_batch<128>(B, src, wide, occ_ext, b, qin, sb);
      ++launches;
    };
    for (int b = 0; b < w.max_depth; ++b) {
      const int* qin = (b & 1) ? B->q1.p : B->q0.p;
      int* qout = (b & 1) ? B->q0.p : B->q1.p;
      ext(b, qin, b >= 1 ? b - 1 : -1);
      if (b >= 1 && B->tail_paths > 0) {
        auto tail = [&](auto kernel, const auto& s) {
          kernel<<<occ_tail, 128, 0, st>>>(s, b, qin, B->counters.p, B->tail_paths, nullptr, B->ray_o.p, B->ray_d.p,
                                           B->thr.p, B->rad.p, B->hits.p, ctx->d_err);
        };
        if (wide) tail(k_tail<false, BatchSrc4>, BatchSrc4{src});
        else tail(k_tail<false, BatchSrc>, src);
        ++launches;
      }
      k_shade<BatchSrc><<<occ_shade, 128, 0, st>>>(src, b, qin, qout, B->counters.p, nullptr, B->ray_o.p,
                                                    B->ray_d.p, B->thr.p, B->rad.p, B->gn.p, B->ga.p, B->hits.p,
                                                    B->shadow.p, ctx->d_err);
      ++launches;
    }
    if (w.max_depth > 0) ext(-1, nullptr, w.max_depth - 1);
    int ablocks = (int)std::min<long long>((w.acc_threads + 255) / 256, (long long)ctx->num_sms * 16);
    k_accumulate_batch<<<std::max(ablocks, 1), 256, 0, st>>>(src, w.nseg, w.acc_threads, B->rad.p, B->gn.p,
                                                              B->ga.p);
    k_finish_batch<<<(w.nseg + 127) / 128, 128, 0, st>>>(src, w.nseg);
    launches += 2;
  }
  *n_launch = launches;
}

template <class T>
static void key_put(std::vector<unsigned char>& k, const T& v) {
  const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
  k.insert(k.end(), p, p + sizeof(T));
}

int batch_render(Batch* B) {
  Ctx* ctx = B->ctx;
  if (B->jobs.empty()) return RX_OK;
  for (const BatchJob& j : B->jobs) {
    if (j.sc->n_tris > 0 && j.sc->n_nodes == 0)
      return set_error(ctx, "batch_render: a scene has triangles but no BVH"), RX_ERR_STATE;
    int rc = j.sc->upload_palette(ctx);
    if (rc) return rc;
  }
  std::vector<WaveSeg> segs;
  std::vector<PlannedWave> waves = plan_waves(B, segs);
  if (waves.empty()) return RX_OK;
  long long cap = 0, shadow_cap = 0;
  for (const PlannedWave& w : waves) {
    cap = std::max(cap, w.paths);
    shadow_cap = std::max(shadow_cap, w.shadow);
  }
  if (cap >= (1LL << 31)) return set_error(ctx, "batch_render: a wave of %lld paths is too large", cap), RX_ERR_CAPACITY;
  // wave buffers
  if (cap > B->cap) {
    B->drop_graph();
    bool ok = B->ray_o.alloc(ctx, cap) && B->ray_d.alloc(ctx, cap) && B->thr.alloc(ctx, cap) &&
              B->rad.alloc(ctx, cap) && B->gn.alloc(ctx, cap) && B->ga.alloc(ctx, cap) && B->hits.alloc(ctx, cap) &&
              B->q0.alloc(ctx, cap) && B->q1.alloc(ctx, cap) && B->pseg.alloc(ctx, cap);
    if (!ok) {
      B->cap = 0;
      return set_error(ctx, "batch_render: out of device memory for %lld wavefront paths", cap), RX_ERR_CAPACITY;
    }
    B->cap = cap;
  }
  if (shadow_cap > B->shadow_cap) {
    B->drop_graph();
    if (!B->shadow.alloc(ctx, (size_t)3 * shadow_cap)) {
      B->shadow_cap = 0;
      return set_error(ctx, "batch_render: out of device memory for %lld shadow rays", shadow_cap), RX_ERR_CAPACITY;
    }
    B->shadow_cap = shadow_cap;
  }
  if (!B->counters.p && !B->counters.alloc(ctx, C_N))
    return set_error(ctx, "batch_render: out of device memory"), RX_ERR_CAPACITY;
  // job tables and segments; the captured graph is reused while they match
  size_t nj = B->jobs.size();
  std::vector<DevScene> scenes(nj);
  std::vector<RenderK> ks(nj);
  std::vector<JobAcc> accs(nj);
  std::vector<unsigned char> key;
  for (size_t j = 0; j < nj; ++j) {
    const BatchJob& J = B->jobs[j];
    scenes[j] = J.sc->view();
    ks[j] = make_k(&J.p, J.acc, 0, B->shadow_cap);
    ks[j].camera0 = 0;
    ks[j].queue_cap = B->cap;
    Accum* a = J.acc;
    accs[j] = JobAcc{a->acc_r.p, a->acc_n.p, a->acc_a.p, a->pixels.p, a->acc64.p, a->frame_base.p, a->rays.p};
    key_put(key, J.sc);
    key_put(key, J.sc->version);
    key_put(key, J.acc);
    key_put(key, a->acc64.p);
    key_put(key, J.p);
    key_put(key, J.frames);
  }
  key_put(key, B->wave_paths);
  key_put(key, B->ext_block);
  key_put(key, B->cap);
  key_put(key, B->shadow_cap);
  cudaStream_t st = ctx->stream;
  bool cached = B->use_graph && B->gexec && key == B->g_key;
  if (!cached) {
    B->drop_graph();
    if (!B->d_scenes.alloc(ctx, nj) || !B->d_ks.alloc(ctx, nj) || !B->d_accs.alloc(ctx, nj) ||
        !B->d_job_rays.alloc(ctx, nj) || !B->d_segs.alloc(ctx, segs.size()))
      return set_error(ctx, "batch_render: out of device memory for job tables"), RX_ERR_CAPACITY;
    CUDA_TRY(ctx, cudaMemcpyAsync(B->d_scenes.p, scenes.data(), sizeof(DevScene) * nj, cudaMemcpyHostToDevice, st));
    CUDA_TRY(ctx, cudaMemcpyAsync(B->d_ks.p, ks.data(), sizeof(RenderK) * nj, cudaMemcpyHostToDevice, st));
    CUDA_TRY(ctx, cudaMemcpyAsync(B->d_accs.p, accs.data(), sizeof(JobAcc) * nj, cudaMemcpyHostToDevice, st));
    CUDA_TRY(ctx, cudaMemsetAsync(B->d_job_rays.p, 0, sizeof(unsigned long long) * nj, st));
    CUDA_TRY(ctx, cudaMemcpyAsync(B->d_segs.p, segs.data(), sizeof(WaveSeg) * segs.size(), cudaMemcpyHostToDevice,
                                  st));
    if (B->use_graph) {
      cudaGraph_t g;
      CUDA_TRY(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      int nl = 0;
      enqueue_batch(B, waves, &nl);
      CUDA_TRY(ctx, cudaStreamEndCapture(st, &g));
      CUDA_TRY(ctx, cudaGraphInstantiate(&B->gexec, g, 0));
      cudaGraphDestroy(g);
      B->g_key = key;
      B->g_launches = nl;
      B->g_waves = (int)waves.size();
    }
  }
  if (!B->e0) {
    CUDA_TRY(ctx, cudaEventCreate(&B->e0));
    CUDA_TRY(ctx, cudaEventCreate(&B->e1));
  }
  CUDA_TRY(ctx, cudaEventRecord(B->e0, st));
  if (B->use_graph) {
    CUDA_TRY(ctx, cudaGraphLaunch(B->gexec, st));
  } else {
    // job sets that change every call (serving): launch directly
    int nl = 0;
    enqueue_batch(B, waves, &nl);
    CUDA_TRY(ctx, cudaGetLastError());
    B->g_launches = nl;
    B->g_waves = (int)waves.size();
  }
  CUDA_TRY(ctx, cudaEventRecord(B->e1, st));
  CUDA_TRY(ctx, cudaEventSynchronize(B->e1));
  CUDA_TRY(ctx, cudaEventElapsedTime(&B->last_ms, B->e0, B->e1));
  B->last_waves = B->g_waves;
  B->last_launches = B->g_launches;
  for (const BatchJob& j : B->jobs) j.acc->frames += j.frames;
  return check_device_error(ctx);
}

int batch_reserve(Batch* B, long long cap) {
  Ctx* ctx = B->ctx;
  if (cap > B->cap) {
    B->drop_graph();
    bool ok = B->ray_o.alloc(ctx, cap) && B->ray_d.alloc(ctx, cap) && B->thr.alloc(ctx, cap) &&
              B->rad.alloc(ctx, cap) && B->gn.alloc(ctx, cap) && B->ga.alloc(ctx, cap) && B->hits.alloc(ctx, cap) &&
              B->q0.alloc(ctx, cap) && B->q1.alloc(ctx, cap) && B->pseg.alloc(ctx, cap);
    if (!ok) {
      B->cap = 0;
      return set_error(ctx, "batch_reserve: out of device memory for %lld wavefront paths", cap), RX_ERR_CAPACITY;
    }
    B->cap = cap;
  }
  if (cap > B->shadow_cap) {
    B->drop_graph();
    if (!B->shadow.alloc(ctx, (size_t)3 * cap)) {
      B->shadow_cap = 0;
      return set_error(ctx, "batch_reserve: out of device memory for %lld shadow rays", cap), RX_ERR_CAPACITY;
    }
    B->shadow_cap = cap;
  }
  if (!B->counters.p && !B->counters.alloc(ctx, C_N))
    return set_error(ctx, "batch_reserve: out of device memory"), RX_ERR_CAPACITY;
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return RX_OK;
}

void batch_use_graph(Batch* B, bool on) {
  if (!on) B->drop_graph();
  B->use_graph = on;
}

size_t accum_bytes(const Accum* a) {
  return a->acc_r.bytes() + a->acc_n.bytes() + a->acc_a.bytes() + a->pixels.bytes() + a->acc64.bytes() +
         a->ray_o.bytes() + a->ray_d.bytes() + a->thr.bytes() + a->rad.bytes() + a->gn.bytes() + a->ga.bytes() +
         a->hits.bytes() + a->shadow.bytes() + a->q0.bytes() + a->q1.bytes() + a->dn0.bytes() + a->dn1.bytes() +
         a->dn_out.bytes() + 64;
}

size_t batch_bytes(const Batch* B) {
  return B->ray_o.bytes() + B->ray_d.bytes() + B->thr.bytes() + B->rad.bytes() + B->gn.bytes() + B->ga.bytes() +
         B->hits.bytes() + B->shadow.bytes() + B->q0.bytes() + B->q1.bytes() + B->pseg.bytes();
}

int batch_last_stats(Batch* B, float* ms, int* waves, int* launches) {
  if (ms) *ms = B->last_ms;
  if (waves) *waves = B->last_waves;
  if (launches) *launches = B->last_launches;
  return RX_OK;
}

}  // namespace rx
