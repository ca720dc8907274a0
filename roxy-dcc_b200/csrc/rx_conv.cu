// BF16 tensor-core kernels of the learned denoiser: 3x3 convolutions
// (forward, gradient of the input, gradient of the weights) as implicit
// GEMMs with FP32 accumulation, and the small element-wise layers around
// them (2x2 average pool, nearest 2x upsample, channel copies for the skip
// concatenations, ReLU masks, loss, Adam).
//
// Layout: activations NHWC bf16, read and written through a channel stride
// and offset so that a concatenated buffer is just a wider tensor;
// weights [Cout][3][3][Cin] bf16 (K = tap * Cin + ci), biases fp32.
// Channel counts are multiples of 16.
//
// Tensor-core path: tiles staged in shared memory by cp.async (16-byte
// copies, zero-filled outside the image), fragments loaded with ldmatrix
// and multiplied with mma.sync m16n8k16 bf16 -> f32.
#include <cuda_bf16.h>

#include <algorithm>

#include "rx_internal.cuh"
#include "rx_runtime.h"

namespace rx {

using bf16 = __nv_bfloat16;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// 16-byte global -> shared copy; `valid` false writes zeros (no bytes read)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(smem)), "l"(gmem),
               "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// ------------------------------------------------------------- forward conv
// y[p][co] = act(bias[co] + sum_{tap, ci} x[p + off(tap)][ci] * w[co][tap][ci])
// GEMM: M = pixels (64 per block), N = output channels (BN per block),
// K = 9 taps x Cin, BK channels per stage.  4 warps as 2 (M) x 2 (N).
template <int BN, int BK>
__global__ void __launch_bounds__(128) k_conv_fwd(rx_conv_desc d, const bf16* __restrict__ x,
                                                  const bf16* __restrict__ w, const float* __restrict__ bias,
                                                  bf16* __restrict__ y, float* __restrict__ y32, int relu) {
  constexpr int BM = 64, LDS = BK + 8;
  constexpr int KC = BK / 8;              // 16-byte chunks per row
  constexpr int A_PER = BM * KC / 128;    // A chunks per thread
  constexpr int B_CH = BN * KC;           // B chunks per stage
  constexpr int NT = BN / 16;             // n8 tiles per warp
  __shared__ __align__(16) bf16 sA[2][BM][LDS];
  __shared__ __align__(16) bf16 sB[2][BN][LDS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 1, wn = warp >> 1;
  const long long HW = (long long)d.H * d.W;
  const long long P = (long long)d.N * HW;
  const long long m0 = (long long)blockIdx.x * BM;
  const int n0 = blockIdx.y * BN;
  const int CB = d.Cin / BK;
  const int KT = 9 * CB;

  int a_row[A_PER], a_kc[A_PER], a_y[A_PER], a_x[A_PER];
  long long a_img[A_PER];
  bool a_ok[A_PER];
#pragma unroll
  for (int i = 0; i < A_PER; ++i) {
    int c = tid + i * 128;
    a_row[i] = c / KC;
    a_kc[i] = c % KC;
    long long pix = m0 + a_row[i];
    a_ok[i] = pix < P;
    long long n = a_ok[i] ? pix / HW : 0;
    long long r = a_ok[i] ? pix - n * HW : 0;
    a_img[i] = n * HW;
    a_y[i] = (int)(r / d.W);
    a_x[i] = (int)(r % d.W);
  }

  auto load = [&](int kt, int buf) {
    int tap = kt / CB, c0 = (kt % CB) * BK;
    int dy = tap / 3 - 1, dx = tap % 3 - 1;
#pragma unroll
    for (int i = 0; i < A_PER; ++i) {
      int yy = a_y[i] + dy, xx = a_x[i] + dx;
      bool ok = a_ok[i] && yy >= 0 && yy < d.H && xx >= 0 && xx < d.W;
      const bf16* src =
          ok ? x + (a_img[i] + (long long)yy * d.W + xx) * d.x_cstride + d.x_coff + c0 + a_kc[i] * 8 : x;
      cp_async16(&sA[buf][a_row[i]][a_kc[i] * 8], src, ok);
    }
    for (int c = tid; c < B_CH; c += 128) {
      int row = c / KC, kc = c % KC;
      int co = n0 + row;
      bool ok = co < d.Cout;
      const bf16* src = ok ? w + ((long long)co * 9 + tap) * d.Cin + c0 + kc * 8 : w;
      cp_async16(&sB[buf][row][kc * 8], src, ok);
    }
  };

  float acc[2][NT][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[i][j][k] = 0.0f;

  load(0, 0);
  cp_async_commit();
  for (int kt = 0; kt < KT; ++kt) {
    int buf = kt & 1;
    if (kt + 1 < KT) load(kt + 1, buf ^ 1);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < BK / 16; ++ks) {
      uint32_t af[2][4];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
        ldsm_x4(af[mi], &sA[buf][wm * 32 + mi * 16 + (lane & 15)][ks * 16 + (lane >> 4) * 8]);
#pragma unroll
      for (int nj = 0; nj < NT / 2; ++nj) {
        uint32_t bfr[4];
        ldsm_x4(bfr, &sB[buf][wn * (BN / 2) + nj * 16 + (lane & 7) + (lane >> 4) * 8][ks * 16 + ((lane >> 3) & 1) * 8]);
#pragma unroll
        for (int mi = 0; mi < 2; ++mi) {
          mma_bf16(acc[mi][2 * nj], af[mi], bfr[0], bfr[1]);
          mma_bf16(acc[mi][2 * nj + 1], af[mi], bfr[2], bfr[3]);
        }
      }
    }
    __syncthreads();
  }
  cp_async_wait<0>();

  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < NT; ++ni)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        long long m = m0 + wm * 32 + mi * 16 + g + h * 8;
        int co = n0 + wn * (BN / 2) + ni * 8 + 2 * t;
        if (m >= P || co >= d.Cout) continue;
        float v0 = acc[mi][ni][2 * h], v1 = acc[mi][ni][2 * h + 1];
        if (bias) {
          v0 += bias[co];
          v1 += bias[co + 1];
        }
        if (relu) {
          v0 = fmaxf(v0, 0.0f);
          v1 = fmaxf(v1, 0.0f);
        }
        *reinterpret_cast<__nv_bfloat162*>(y + m * d.y_cstride + d.y_coff + co) = __floats2bfloat162_rn(v0, v1);
        if (y32) {
          y32[m * d.y_cstride + d.y_coff + co] = v0;
          y32[m * d.y_cstride + d.y_coff + co + 1] = v1;
        }
      }
}

// ------------------------------------------- forward conv on tcgen05 (UMMA)
// One CTA computes 128 consecutive pixels of one image row (the MMA's M)
// for all COUT output channels (its N), accumulating in tensor memory.
// Per chunk of 32 input channels it stages, with cp.async, a halo of 3 rows
// x 130 pixels and the 9 taps' weights in shared memory in the canonical
// K-major, no-swizzle layout (core matrices of 8 rows x 16 bytes): channel
// chunk planes [kc][row][pixel][8 channels] and [tap][kc][co][8].  A tap's
// A operand is then the same descriptor with its start moved by whole
// pixels, so the halo is loaded once for all 9 taps.  One thread issues
// 9 taps x 2 K-steps of tcgen05.mma (kind::f16, BF16 in, FP32 accumulate)
// per chunk and commits them to the chunk buffer's mbarrier; two buffers
// overlap the next chunk's copies with the current MMAs.
namespace tc {
constexpr int TILE = 128, HALO_W = TILE + 2, KCH = 4;  // 4 chunks of 8 channels = 32
constexpr int HALO_BYTES = KCH * 3 * HALO_W * 16;      // 24960
constexpr unsigned long long kSpinCycles = 4000000000ull;  // ~2 s at 1.9 GHz

__host__ __device__ constexpr int stage_bytes(int cout) { return HALO_BYTES + 9 * KCH * cout * 16; }

// K-major, no-swizzle shared-memory matrix descriptor (Blackwell version 1)
__device__ __forceinline__ uint64_t desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// instruction descriptor: FP32 accumulate, BF16 A and B, both K-major, M=128
__host__ __device__ constexpr uint32_t idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  unsigned long long t0 = clock64();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > kSpinCycles) return false;
  }
}
}  // namespace tc

template <int COUT>
__global__ void __launch_bounds__(128, 1) k_conv_fwd_tc(rx_conv_desc d, const bf16* __restrict__ x,
                                                        const bf16* __restrict__ w, const float* __restrict__ bias,
                                                        bf16* __restrict__ y, float* __restrict__ y32, int relu,
                                                        int* err) {
  constexpr int SB = tc::stage_bytes(COUT);
  constexpr int TCOLS = COUT < 32 ? 32 : COUT;  // tensor-memory columns (power of two >= 32)
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) unsigned long long bars[2];
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int x0 = blockIdx.x * tc::TILE, yrow = blockIdx.y, n = blockIdx.z;
  const int nch = (d.Cin + 31) / 32;

  if (tid == 0) {
    abort_flag = 0;
    for (int b = 0; b < 2; ++b)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&bars[b])));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base)),
                 "r"(TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_base;

  auto load = [&](int ch, int buf) {
    unsigned char* base = smem + buf * SB;
    const int c0 = ch * 32;
    // halo: chunk index ((r * HALO_W + px) * KCH + kc); 16 bytes each
    for (int c = tid; c < 3 * tc::HALO_W * tc::KCH; c += 128) {
      int kc = c % tc::KCH, rp = c / tc::KCH;
      int px = rp % tc::HALO_W, r = rp / tc::HALO_W;
      int yy = yrow + r - 1, xx = x0 + px - 1, ci = c0 + kc * 8;
      bool ok = yy >= 0 && yy < d.H && xx >= 0 && xx < d.W && ci < d.Cin;
      const bf16* src = ok ? x + (((long long)n * d.H + yy) * d.W + xx) * d.x_cstride + d.x_coff + ci : x;
      cp_async16(base + ((kc * 3 + r) * tc::HALO_W + px) * 16, src, ok);
    }
    // weights: chunk index ((co * 9 + tap) * KCH + kc)
    unsigned char* wb = base + tc::HALO_BYTES;
    for (int c = tid; c < COUT * 9 * tc::KCH; c += 128) {
      int kc = c % tc::KCH, ct = c / tc::KCH;
      int tap = ct % 9, co = ct / 9;
      int ci = c0 + kc * 8;
      bool ok = co < d.Cout && ci < d.Cin;
      const bf16* src = ok ? w + ((long long)co * 9 + tap) * d.Cin + ci : w;
      cp_async16(wb + ((tap * tc::KCH + kc) * COUT + co) * 16, src, ok);
    }
  };

  load(0, 0);
  cp_async_commit();
  bool ok_all = true;
  for (int ch = 0; ch < nch; ++ch) {
    const int buf = ch & 1;
    if (ch + 1 < nch) {
      const int nb = (ch + 1) & 1;
      if (ch + 1 >= 2) {
        // the MMAs of chunk ch - 1 read buffer nb: wait for their commit
        if (!tc::mbar_wait(smem_u32(&bars[nb]), (uint32_t)(((ch - 1) >> 1) & 1))) abort_flag = 1;
      }
      __syncthreads();
      if (abort_flag) {
        ok_all = false;
        break;
      }
      load(ch + 1, nb);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    // copies visible to the tensor cores (async proxy) before the MMAs
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t hb = smem_u32(smem + buf * SB);
      const uint32_t wb = hb + tc::HALO_BYTES;
      constexpr uint32_t ID = tc::idesc(COUT);
#pragma unroll 1
      for (int tap = 0; tap < 9; ++tap) {
        const int dy = tap / 3, dx = tap % 3;
#pragma unroll
        for (int k2 = 0; k2 < 2; ++k2) {
          uint64_t ad = tc::desc(hb + (((2 * k2) * 3 + dy) * tc::HALO_W + dx) * 16, 3 * tc::HALO_W * 16, 128);
          uint64_t bd = tc::desc(wb + ((tap * tc::KCH + 2 * k2) * COUT) * 16, COUT * 16, 128);
          uint32_t acc = (ch > 0 || tap > 0 || k2 > 0) ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
              "l"(ad), "l"(bd), "r"(ID), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                       smem_u32(&bars[buf]))
                   : "memory");
    }
  }
  if (ok_all) {
    const int last = nch - 1;
    if (!tc::mbar_wait(smem_u32(&bars[last & 1]), (uint32_t)((last >> 1) & 1))) ok_all = false;
  }
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (ok_all) {
    // accumulator row = pixel (warp's 32 lanes), columns = output channels
    const int xx = x0 + warp * 32 + lane;
    const long long m = ((long long)n * d.H + yrow) * d.W + xx;
#pragma unroll 1
    for (int c0 = 0; c0 < COUT; c0 += 16) {
      uint32_t r[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      if (xx < d.W && c0 < d.Cout) {
        float v[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          v[k] = __uint_as_float(r[k]) + (bias ? bias[c0 + k] : 0.0f);
          if (relu) v[k] = fmaxf(v[k], 0.0f);
        }
        uint4 pk[2];
        uint32_t* pw = reinterpret_cast<uint32_t*>(pk);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
          pw[k] = *reinterpret_cast<uint32_t*>(&h);
        }
        uint4* dst = reinterpret_cast<uint4*>(y + m * d.y_cstride + d.y_coff + c0);
        dst[0] = pk[0];
        dst[1] = pk[1];
        if (y32) {
#pragma unroll
          for (int k = 0; k < 16; ++k) y32[m * d.y_cstride + d.y_coff + c0 + k] = v[k];
        }
      }
    }
  } else if (tid == 0) {
    atomicOr(err, ERR_BAD_NODE);
  }
  cp_async_wait<0>();
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS));
}

// cp.async.wait_group with a run-time count (0..3; larger waits for 3)
__device__ __forceinline__ void cp_async_wait_n(int n) {
  switch (n) {
    case 0: cp_async_wait<0>(); break;
    case 1: cp_async_wait<1>(); break;
    case 2: cp_async_wait<2>(); break;
    default: cp_async_wait<3>(); break;
  }
}

// --------------------------------------- forward conv, warp-specialised
// Persistent row-strip kernel for layers whose weights fit in shared memory
// beside a ring of input rows.  The weights are loaded once per CTA.  Each
// CTA owns a contiguous range of 128-pixel row tiles ordered with the row
// fastest, so consecutive tiles are vertically adjacent and share two of
// their three input rows: the input is a ring of S row slots [slot][kc]
// [pixel][8] (130 pixels, all input channels), and every input row is read
// once per strip instead of three times.  Three jobs run in separate warps
// that hand work to one another through mbarriers, so that copies, MMAs
// and epilogues of different rows overlap:
//   warps 5-6: producers.  Each input row of the strip (130 pixels, zero
//     outside the image) is copied with coalesced 16-byte cp.async into a
//     ring slot [kc][130 px x 16 B]; once a row's copies have landed the 64
//     producers make them visible to the tensor cores (proxy fence) and
//     arrive on `full[slot]`; a slot is refilled after `empty[slot]`.
//   warp 4 (one thread): MMA issuer.  Output row y reads the slots of rows
//     y-1, y, y+1; it accumulates into one of two tensor-memory buffers,
//     commits to `acc_full[buf]`, and releases row y-1's slot (its last
//     reader) with a commit to `empty`.
//   warps 0-3: epilogue.  Warp w reads tensor-memory lanes 32 w .. 32 w + 31
//     (its 32 pixels), adds the bias, applies ReLU, stores bf16 (and fp32),
//     then arrives on `acc_empty[buf]`.
// Output channels may be split into G groups of NG (blockIdx.x % G) when
// all the weights do not fit in shared memory beside the ring; the G CTAs
// of a strip run side by side and share its input rows through L2.
// Every wait is bounded: a wait that runs out (or sees another role give
// up) raises the shared abort flag, the roles stop, outstanding copies and
// MMAs are waited for (bounded), the device error flag is set.
namespace tc {
constexpr int PLANE = HALO_W * 16;  // one 8-channel chunk of one row
__host__ __device__ constexpr int slot_bytes(int cin) { return (cin / 8) * PLANE; }
__host__ __device__ constexpr int weights_bytes(int cin, int cout) { return 9 * cin * cout * 2; }
constexpr int kMaxSlots = 8;
}  // namespace tc

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// single-thread bounded wait; gives up when the abort flag is raised
__device__ __forceinline__ bool mbar_wait_abortable(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
  const unsigned long long t0 = clock64();
  for (;;) {
    if (mbar_try(bar, parity)) return true;
    if (*abort_flag) return false;
    if (clock64() - t0 > tc::kSpinCycles) {
      *abort_flag = 1;
      return false;
    }
  }
}

// whole-warp bounded wait with a warp-uniform outcome
__device__ __forceinline__ bool mbar_wait_warp(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
  const unsigned long long t0 = clock64();
  for (;;) {
    const bool ok = mbar_try(bar, parity);
    if (__all_sync(0xffffffffu, ok)) return true;
    const bool stop = *abort_flag || clock64() - t0 > tc::kSpinCycles;
    if (__any_sync(0xffffffffu, stop)) {
      *abort_flag = 1;
      return false;
    }
  }
}

// acc_in (may be null): fp32 partial sums [pixel][Cout] of the other input
// channels, added before the bias (a layer split over its input channels,
// conv_fwd); y (may be null): bf16 output.
template <int NG>
__global__ void __launch_bounds__(224, 1) k_conv_fwd_ws(rx_conv_desc d, const bf16* __restrict__ x,
                                                        const bf16* __restrict__ w, const float* __restrict__ bias,
                                                        bf16* __restrict__ y, float* __restrict__ y32,
                                                        const float* __restrict__ acc_in, int relu, int S, int G,
                                                        long long per_cta, int* err) {
  constexpr int TCOLS = 2 * NG < 32 ? 32 : 2 * NG;  // two accumulators
  constexpr int kProducers = 64;                     // warps 5 and 6
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long full[tc::kMaxSlots], empty[tc::kMaxSlots];
  __shared__ __align__(8) unsigned long long acc_full[2], acc_empty[2], mma_done;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;
  __shared__ float sbias[NG];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int KC = d.Cin / 8;
  const int SB = tc::slot_bytes(d.Cin);
  unsigned char* smem = smem_raw + ((128 - (smem_u32(smem_raw) & 127)) & 127);
  unsigned char* wsm = smem;                                 // [tap][kc][co][8]
  unsigned char* rsm = smem + tc::weights_bytes(d.Cin, NG);  // S x [kc][PLANE]
  const int grp = blockIdx.x % G;
  const int xt = (d.W + tc::TILE - 1) / tc::TILE;
  const long long total = (long long)d.N * xt * d.H;  // row tiles, row fastest
  const long long u0 = (long long)(blockIdx.x / G) * per_cta;
  const long long uend = u0 + per_cta < total ? u0 + per_cta : total;

  if (tid == 0) {
    abort_flag = 0;
    for (int s = 0; s < S; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&full[s])), "r"(kProducers));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&empty[s])));
    }
    for (int b = 0; b < 2; ++b) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&acc_full[b])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;\n" ::"r"(smem_u32(&acc_empty[b])));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&mma_done)));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  for (int c = tid; c < NG; c += blockDim.x) sbias[c] = bias ? bias[grp * NG + c] : 0.0f;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base)),
                 "r"(TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  // this group's weights, once: chunk ((co * 9 + tap) * KC + kc) -> [tap][kc][co][8]
  for (int c = tid; c < NG * 9 * KC; c += blockDim.x) {
    int kc = c % KC, ct = c / KC;
    int tap = ct % 9, co = ct / 9;
    const bf16* src = w + ((long long)(grp * NG + co) * 9 + tap) * d.Cin + kc * 8;
    cp_async16(wsm + ((tap * KC + kc) * NG + co) * 16, src, true);
  }
  cp_async_commit();
  cp_async_wait<0>();
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_base;

  if (warp >= 5) {
    // ------------------------------------------------ producers (cp.async)
    // consecutive threads copy consecutive 16-byte chunks of a pixel row,
    // so each warp request is coalesced; a row is signalled `lag` rows
    // after it was issued, once its copies have landed
    const int ptid = tid - 5 * 32;
    const int lag = S - 3 < 2 ? S - 3 : 2;
    auto signal = [&](int q) {
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(&full[q % S])) : "memory");
    };
    int k = 0;  // rows issued
    bool ok = true;
    for (long long u = u0; u < uend && ok;) {
      const long long col = u / d.H;
      const int ylo = (int)(u - col * d.H);
      const int yhi = (int)((long long)ylo + (uend - u) < d.H ? (long long)ylo + (uend - u) : d.H);
      const int n = (int)(col / xt), x0 = (int)(col % xt) * tc::TILE;
      for (int r = ylo - 1; r <= yhi; ++r, ++k) {
        const int s = (int)(k % S);
        if (!mbar_wait_warp(smem_u32(&empty[s]), (uint32_t)(((k / S) & 1) ^ 1), &abort_flag)) {
          ok = false;
          break;
        }
        unsigned char* base = rsm + s * SB;
        const bool row_ok = r >= 0 && r < d.H;
        const long long rbase = ((long long)n * d.H + r) * d.W;
        for (int c = ptid; c < tc::HALO_W * KC; c += kProducers) {
          const int kc = c % KC, px = c / KC;
          const int xx = x0 + px - 1;
          const bool in = row_ok && xx >= 0 && xx < d.W;
          const bf16* src = in ? x + (rbase + xx) * d.x_cstride + d.x_coff + kc * 8 : x;
          cp_async16(base + kc * tc::PLANE + px * 16, src, in);
        }
        cp_async_commit();
        if (k >= lag) {
          cp_async_wait_n(lag);
          signal(k - lag);
        }
      }
      u += yhi - ylo;
    }
    cp_async_wait<0>();
    if (ok)
      for (int q = k > lag ? k - lag : 0; q < k; ++q) signal(q);
  } else if (warp == 4) {
    // ------------------------------------------------ MMA issuer
    if (lane == 0) {
      const uint32_t rb = smem_u32(rsm), wb = smem_u32(wsm);
      constexpr uint32_t ID = tc::idesc(NG);
      // descriptor words (K-major, no swizzle): SBO 128 B and version 1 in
      // the high word; LBO = one plane (A) or NG x 16 B (B) in the low word
      constexpr uint32_t desc_hi = (128u >> 4) | (1u << 14);
      const uint32_t a_lbo = (uint32_t)(tc::PLANE >> 4) << 16;
      const uint32_t b_lo0 = (wb >> 4) | ((uint32_t)NG << 16);
      int kb = 0;  // ring index of the segment's first row (ylo - 1)
      int i = 0;         // output rows issued
      bool ok = true;
      for (long long u = u0; u < uend && ok;) {
        const long long col = u / d.H;
        const int ylo = (int)(u - col * d.H);
        const int yhi = (int)((long long)ylo + (uend - u) < d.H ? (long long)ylo + (uend - u) : d.H);
        const int nrows = yhi - ylo;
        for (int yy = ylo; yy < yhi; ++yy, ++i) {
          const int kr = kb + (yy - ylo);  // ring index of row yy - 1
          int slot[3];
          for (int q = 0; q < 3; ++q) {
            slot[q] = (kr + q) % S;
            if (ok) ok = mbar_wait_abortable(smem_u32(&full[slot[q]]), (uint32_t)(((kr + q) / S) & 1), &abort_flag);
          }
          const int b = i & 1;
          if (ok) ok = mbar_wait_abortable(smem_u32(&acc_empty[b]), (uint32_t)(((i >> 1) & 1) ^ 1), &abort_flag);
          if (!ok) break;
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          const uint32_t acc_t = tmem + (uint32_t)(b * NG);
          // The issue loop runs on one thread, so its integer work sets
          // the MMA rate: descriptors are stepped, not rebuilt.  Low words
          // hold (address >> 4) | (LBO >> 4) << 16; a byte offset of 16 k
          // adds k.  A: next chunk pair +2 planes, next tap column +1
          // pixel; B walks [tap][kc][co] in order, 2 NG x 16 B per step.
          uint32_t b_lo = b_lo0;
          uint32_t acc = 0u;
#pragma unroll 1
          for (int tap = 0; tap < 9; ++tap) {
            const int dy = tap / 3, dx = tap % 3;
            uint32_t a_lo = ((rb + (uint32_t)(slot[dy] * SB)) >> 4) + (uint32_t)dx + a_lbo;
#pragma unroll 2
            for (int kc0 = 0; kc0 < KC; kc0 += 2) {
              const uint64_t ad = ((uint64_t)desc_hi << 32) | a_lo;
              const uint64_t bd = ((uint64_t)desc_hi << 32) | b_lo;
              asm volatile(
                  "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                  "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(acc_t),
                  "l"(ad), "l"(bd), "r"(ID), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
              acc = 1u;
              a_lo += 2 * (tc::PLANE >> 4);
              b_lo += 2 * NG;
            }
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                           smem_u32(&acc_full[b]))
                       : "memory");
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                           smem_u32(&empty[slot[0]]))
                       : "memory");
        }
        if (!ok) break;
        // rows yhi - 1 and yhi have no later reader in this segment
        for (int q = 0; q < 2; ++q)
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                           smem_u32(&empty[(kb + nrows + q) % S]))
                       : "memory");
        kb += nrows + 2;
        u += nrows;
      }
      // every MMA issued has finished before the tensor memory is released
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                       smem_u32(&mma_done))
                   : "memory");
      const unsigned long long t0 = clock64();
      while (!mbar_try(smem_u32(&mma_done), 0u) && clock64() - t0 < tc::kSpinCycles) {
      }
    }
  } else {
    // ------------------------------------------------ epilogue (warps 0-3)
    const int qtr = warp;  // tensor-memory lanes 32 qtr .. 32 qtr + 31
    int i = 0;
    bool ok = true;
    for (long long u = u0; u < uend && ok;) {
      const long long col = u / d.H;
      const int ylo = (int)(u - col * d.H);
      const int yhi = (int)((long long)ylo + (uend - u) < d.H ? (long long)ylo + (uend - u) : d.H);
      const int n = (int)(col / xt), x0 = (int)(col % xt) * tc::TILE;
      for (int yy = ylo; yy < yhi; ++yy, ++i) {
        const int b = i & 1;
        if (!mbar_wait_warp(smem_u32(&acc_full[b]), (uint32_t)((i >> 1) & 1), &abort_flag)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const int xx = x0 + qtr * 32 + lane;
        const long long m = ((long long)n * d.H + yy) * d.W + xx;
#pragma unroll 1
        for (int c0 = 0; c0 < NG; c0 += 16) {
          uint32_t r[16];
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
              "[%16];\n"
              : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
              : "r"(tmem + ((uint32_t)(qtr * 32) << 16) + (uint32_t)(b * NG + c0)));
          asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
          if (xx < d.W) {
            float v[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
            if (acc_in) {
              const float4* a4 = reinterpret_cast<const float4*>(acc_in + m * d.Cout + grp * NG + c0);
#pragma unroll
              for (int k = 0; k < 4; ++k) {
                const float4 a = a4[k];
                v[4 * k] += a.x;
                v[4 * k + 1] += a.y;
                v[4 * k + 2] += a.z;
                v[4 * k + 3] += a.w;
              }
            }
#pragma unroll
            for (int k = 0; k < 16; ++k) {
              v[k] = v[k] + sbias[c0 + k];
              if (relu) v[k] = fmaxf(v[k], 0.0f);
            }
            const long long o = m * d.y_cstride + d.y_coff + grp * NG + c0;
            if (y) {
              uint4 pk[2];
              uint32_t* pw = reinterpret_cast<uint32_t*>(pk);
#pragma unroll
              for (int k = 0; k < 8; ++k) {
                __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
                pw[k] = *reinterpret_cast<uint32_t*>(&h);
              }
              uint4* dst = reinterpret_cast<uint4*>(y + o);
              dst[0] = pk[0];
              dst[1] = pk[1];
            }
            if (y32) {
              float4* d32 = reinterpret_cast<float4*>(y32 + o);
#pragma unroll
              for (int k = 0; k < 4; ++k) d32[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
            }
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncwarp();
        if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(&acc_empty[b])) : "memory");
      }
      u += yhi - ylo;
    }
  }

  __syncwarp();
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (tid == 0 && abort_flag) atomicOr(err, ERR_BAD_NODE);
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS));
}

// ------------------------------------------------------- weight gradient
// dw[co][tap][ci] += sum_p dy[p][co] * x[p + off(tap)][ci]
// GEMM: M = output channels (64), N = input channels (64), K = pixels
// (32 per stage, `pix_per_block` per block, split-K with atomics).
__global__ void __launch_bounds__(128) k_conv_wgrad(rx_conv_desc d, const bf16* __restrict__ dy,
                                                    const bf16* __restrict__ x, float* __restrict__ dw,
                                                    int pix_per_block) {
  constexpr int BM = 64, BN = 64, BK = 32, LDA = BM + 8, LDB = BN + 8;
  __shared__ __align__(16) bf16 sA[2][BK][LDA];
  __shared__ __align__(16) bf16 sB[2][BK][LDB];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 1, wn = warp >> 1;
  const long long HW = (long long)d.H * d.W;
  const long long P = (long long)d.N * HW;
  const int tap = blockIdx.z;
  const int dyo = tap / 3 - 1, dxo = tap % 3 - 1;
  const int co_blocks = (d.Cout + BM - 1) / BM;
  const int co0 = (blockIdx.y % co_blocks) * BM;
  const int ci0 = (blockIdx.y / co_blocks) * BN;
  const long long p_begin = (long long)blockIdx.x * pix_per_block;
  const long long p_end = P < p_begin + pix_per_block ? P : p_begin + pix_per_block;
  const int KT = (int)((p_end - p_begin + BK - 1) / BK);

  auto load = [&](int kt, int buf) {
    long long pb = p_begin + (long long)kt * BK;
    // 32 pixels x 8 chunks of dy and of x: 256 chunks each, 2 per thread
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      int c = tid + i * 128;
      int r = c >> 3, kc = c & 7;
      long long p = pb + r;
      bool pok = p < p_end;
      int co = co0 + kc * 8;
      bool ok = pok && co < d.Cout;
      const bf16* src = ok ? dy + p * d.y_cstride + d.y_coff + co : dy;
      cp_async16(&sA[buf][r][kc * 8], src, ok);
      long long n = pok ? p / HW : 0;
      long long rem = pok ? p - n * HW : 0;
      int yy = (int)(rem / d.W) + dyo, xx = (int)(rem % d.W) + dxo;
      int ci = ci0 + kc * 8;
      bool okx = pok && ci < d.Cin && yy >= 0 && yy < d.H && xx >= 0 && xx < d.W;
      const bf16* srcx = okx ? x + (n * HW + (long long)yy * d.W + xx) * d.x_cstride + d.x_coff + ci : x;
      cp_async16(&sB[buf][r][kc * 8], srcx, okx);
    }
  };

  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[i][j][k] = 0.0f;

  if (KT > 0) {
    load(0, 0);
    cp_async_commit();
  }
  for (int kt = 0; kt < KT; ++kt) {
    int buf = kt & 1;
    if (kt + 1 < KT) load(kt + 1, buf ^ 1);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < BK / 16; ++ks) {
      const int j = lane >> 3, r = lane & 7;
      uint32_t af[2][4];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
        ldsm_x4_t(af[mi], &sA[buf][ks * 16 + r + (j >> 1) * 8][wm * 32 + mi * 16 + (j & 1) * 8]);
#pragma unroll
      for (int nj = 0; nj < 2; ++nj) {
        uint32_t bfr[4];
        ldsm_x4_t(bfr, &sB[buf][ks * 16 + r + (j & 1) * 8][wn * 32 + nj * 16 + (j >> 1) * 8]);
#pragma unroll
        for (int mi = 0; mi < 2; ++mi) {
          mma_bf16(acc[mi][2 * nj], af[mi], bfr[0], bfr[1]);
          mma_bf16(acc[mi][2 * nj + 1], af[mi], bfr[2], bfr[3]);
        }
      }
    }
    __syncthreads();
  }
  cp_async_wait<0>();
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        int co = co0 + wm * 32 + mi * 16 + g + h * 8;
        int ci = ci0 + wn * 32 + ni * 8 + 2 * t;
        if (co >= d.Cout || ci >= d.Cin) continue;
        float* dst = dw + ((long long)co * 9 + tap) * d.Cin + ci;
        atomicAdd(dst, acc[mi][ni][2 * h]);
        atomicAdd(dst + 1, acc[mi][ni][2 * h + 1]);
      }
}

// dbias[co] += sum_p dy[p][co]
__global__ void k_bias_grad(rx_conv_desc d, const bf16* __restrict__ dy, float* __restrict__ db, int pix_per_block) {
  const long long P = (long long)d.N * d.H * d.W;
  long long p0 = (long long)blockIdx.x * pix_per_block;
  long long p1 = P < p0 + pix_per_block ? P : p0 + pix_per_block;
  for (int co = threadIdx.x; co < d.Cout; co += blockDim.x) {
    float s = 0.0f;
    for (long long p = p0; p < p1; ++p) s += __bfloat162float(dy[p * d.y_cstride + d.y_coff + co]);
    atomicAdd(db + co, s);
  }
}

// w_rot[ci][tap][co] = w[co][8 - tap][ci]: the weights of the input-gradient
// convolution (a 3x3 convolution of dy with the flipped, transposed kernel)
__global__ void k_rot_weights(int Cout, int Cin, const bf16* __restrict__ w, bf16* __restrict__ wr) {
  long long n = (long long)Cout * 9 * Cin;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    int ci = (int)(i % Cin);
    int tap = (int)((i / Cin) % 9);
    int co = (int)(i / ((long long)Cin * 9));
    wr[((long long)ci * 9 + (8 - tap)) * Cout + co] = w[i];
  }
}

// ------------------------------------------------------------ element-wise
// Every element-wise kernel walks (pixel, channel) of an NHWC view
// (stride, offset) with a grid-stride loop.
#define RX_EW_LOOP(count) \
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (count); i += (long long)gridDim.x * blockDim.x)

// dst = src (channels [0, C) of each view); accumulate: dst += src
__global__ void k_copy_ch(long long P, int C, const bf16* __restrict__ src, int s_stride, int s_off,
                          bf16* __restrict__ dst, int d_stride, int d_off, int accumulate) {
  RX_EW_LOOP(P * C) {
    long long p = i / C;
    int c = (int)(i % C);
    float v = __bfloat162float(src[p * s_stride + s_off + c]);
    bf16* o = dst + p * d_stride + d_off + c;
    if (accumulate) v += __bfloat162float(*o);
    *o = __float2bfloat16_rn(v);
  }
}

// g = y > 0 ? g : 0  (gradient through a ReLU whose output is y)
__global__ void k_relu_mask(long long P, int C, const bf16* __restrict__ yv, int y_stride, int y_off,
                            bf16* __restrict__ g, int g_stride, int g_off) {
  RX_EW_LOOP(P * C) {
    long long p = i / C;
    int c = (int)(i % C);
    if (!(__bfloat162float(yv[p * y_stride + y_off + c]) > 0.0f)) g[p * g_stride + g_off + c] = __float2bfloat16_rn(0.0f);
  }
}

// 2x2 average pool (H, W even): out (N, H/2, W/2, C)
__global__ void k_pool2(int N, int H, int W, int C, const bf16* __restrict__ x, int x_stride, int x_off,
                        bf16* __restrict__ y, int y_stride, int y_off) {
  int h2 = H / 2, w2 = W / 2;
  RX_EW_LOOP((long long)N * h2 * w2 * C) {
    int c = (int)(i % C);
    long long q = i / C;
    int xo = (int)(q % w2), yo = (int)((q / w2) % h2);
    long long n = q / ((long long)w2 * h2);
    long long b = (n * H + 2 * yo) * W + 2 * xo;
    float s = __bfloat162float(x[b * x_stride + x_off + c]) + __bfloat162float(x[(b + 1) * x_stride + x_off + c]) +
              __bfloat162float(x[(b + W) * x_stride + x_off + c]) +
              __bfloat162float(x[(b + W + 1) * x_stride + x_off + c]);
    y[q * y_stride + y_off + c] = __float2bfloat16_rn(0.25f * s);
  }
}

// The same two layers on 8-channel (16-byte) chunks, for views whose
// channel count, stride and offset are multiples of 8: one item per chunk
// of an input pixel (upsample: one load, four stores) or of an output pixel
// (pool: four loads, one store); same float32 sum order as above.
__device__ __forceinline__ void chunk_index(long long i, int CK, int W, int H, int& ck, int& x, int& y, long long& n) {
  ck = (int)(i % CK);
  long long q = i / CK;
  x = (int)(q % W);
  q /= W;
  y = (int)(q % H);
  n = q / H;
}

__global__ void k_up2_v8(int N, int H, int W, int C, const bf16* __restrict__ x, int x_stride, int x_off,
                         bf16* __restrict__ y, int y_stride, int y_off) {
  const int CK = C >> 3;
  RX_EW_LOOP((long long)N * H * W * CK) {
    int ck, xx, yy;
    long long n;
    chunk_index(i, CK, W, H, ck, xx, yy, n);
    const uint4 v = *reinterpret_cast<const uint4*>(x + ((n * H + yy) * W + xx) * x_stride + x_off + ck * 8);
    const long long o = (n * 2 * H + 2 * yy) * 2LL * W + 2 * xx;
    bf16* d = y + y_off + ck * 8;
    *reinterpret_cast<uint4*>(d + o * y_stride) = v;
    *reinterpret_cast<uint4*>(d + (o + 1) * y_stride) = v;
    *reinterpret_cast<uint4*>(d + (o + 2LL * W) * y_stride) = v;
    *reinterpret_cast<uint4*>(d + (o + 2LL * W + 1) * y_stride) = v;
  }
}

__global__ void k_pool2_v8(int N, int H, int W, int C, const bf16* __restrict__ x, int x_stride, int x_off,
                           bf16* __restrict__ y, int y_stride, int y_off) {
  const int CK = C >> 3, h2 = H / 2, w2 = W / 2;
  RX_EW_LOOP((long long)N * h2 * w2 * CK) {
    int ck, xo, yo;
    long long n;
    chunk_index(i, CK, w2, h2, ck, xo, yo, n);
    const long long b = (n * H + 2 * yo) * W + 2 * xo;
    const bf16* s = x + x_off + ck * 8;
    uint4 q[4] = {*reinterpret_cast<const uint4*>(s + b * x_stride),
                  *reinterpret_cast<const uint4*>(s + (b + 1) * x_stride),
                  *reinterpret_cast<const uint4*>(s + (b + W) * x_stride),
                  *reinterpret_cast<const uint4*>(s + (b + W + 1) * x_stride)};
    const bf16* e[4] = {reinterpret_cast<const bf16*>(&q[0]), reinterpret_cast<const bf16*>(&q[1]),
                        reinterpret_cast<const bf16*>(&q[2]), reinterpret_cast<const bf16*>(&q[3])};
    uint4 out;
    bf16* o = reinterpret_cast<bf16*>(&out);
#pragma unroll
    for (int k = 0; k < 8; ++k)
      o[k] = __float2bfloat16_rn(0.25f * (__bfloat162float(e[0][k]) + __bfloat162float(e[1][k]) +
                                          __bfloat162float(e[2][k]) + __bfloat162float(e[3][k])));
    *reinterpret_cast<uint4*>(y + ((n * h2 + yo) * w2 + xo) * y_stride + y_off + ck * 8) = out;
  }
}

// gradient of the pool: each input pixel gets a quarter of its output's
// gradient; accumulate adds to dx
__global__ void k_pool2_bwd(int N, int H, int W, int C, const bf16* __restrict__ dy, int dy_stride, int dy_off,
                            bf16* __restrict__ dx, int dx_stride, int dx_off, int accumulate) {
  RX_EW_LOOP((long long)N * H * W * C) {
    int c = (int)(i % C);
    long long p = i / C;
    int xx = (int)(p % W), yy = (int)((p / W) % H);
    long long n = p / ((long long)W * H);
    long long q = (n * (H / 2) + yy / 2) * (W / 2) + xx / 2;
    float v = 0.25f * __bfloat162float(dy[q * dy_stride + dy_off + c]);
    bf16* o = dx + p * dx_stride + dx_off + c;
    if (accumulate) v += __bfloat162float(*o);
    *o = __float2bfloat16_rn(v);
  }
}

// nearest 2x upsample: out (N, 2H, 2W, C) from x (N, H, W, C)
__global__ void k_up2(int N, int H, int W, int C, const bf16* __restrict__ x, int x_stride, int x_off,
                      bf16* __restrict__ y, int y_stride, int y_off) {
  RX_EW_LOOP((long long)N * 4 * H * W * C) {
    int c = (int)(i % C);
    long long p = i / C;
    int xx = (int)(p % (2 * W)), yy = (int)((p / (2 * W)) % (2 * H));
    long long n = p / (4LL * W * H);
    long long q = (n * H + yy / 2) * W + xx / 2;
    y[p * y_stride + y_off + c] = x[q * x_stride + x_off + c];
  }
}

// gradient of the upsample: sum of the four children
__global__ void k_up2_bwd(int N, int H, int W, int C, const bf16* __restrict__ dy, int dy_stride, int dy_off,
                          bf16* __restrict__ dx, int dx_stride, int dx_off) {
  RX_EW_LOOP((long long)N * H * W * C) {
    int c = (int)(i % C);
    long long q = i / C;
    int xx = (int)(q % W), yy = (int)((q / W) % H);
    long long n = q / ((long long)W * H);
    long long b = (n * 2 * H + 2 * yy) * 2 * W + 2 * xx;
    long long w2 = 2LL * W;
    float s = __bfloat162float(dy[b * dy_stride + dy_off + c]) + __bfloat162float(dy[(b + 1) * dy_stride + dy_off + c]) +
              __bfloat162float(dy[(b + w2) * dy_stride + dy_off + c]) +
              __bfloat162float(dy[(b + w2 + 1) * dy_stride + dy_off + c]);
    dx[q * dx_stride + dx_off + c] = __float2bfloat16_rn(s);
  }
}

// Network input: 16 channels (log1p radiance, albedo, normal, depth/(1+depth),
// six zeros) from float32 (P, 3) planes; base (optional) receives the
// float32 log1p radiance the network's output is added to.
__global__ void k_features(long long P, const float* __restrict__ rad, const float* __restrict__ alb,
                           const float* __restrict__ nrm, const float* __restrict__ dep, bf16* __restrict__ out,
                           float* __restrict__ base) {
  RX_EW_LOOP(P) {
    float f[16];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      f[k] = log1pf(fmaxf(rad[3 * i + k], 0.0f));
      f[3 + k] = alb[3 * i + k];
      f[6 + k] = nrm[3 * i + k];
      if (base) base[3 * i + k] = f[k];
    }
    float dd = fmaxf(dep[i], 0.0f);
    f[9] = dd / (1.0f + dd);
#pragma unroll
    for (int k = 10; k < 16; ++k) f[k] = 0.0f;
    __nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(out + 16 * i);
#pragma unroll
    for (int k = 0; k < 8; ++k) o[k] = __floats2bfloat162_rn(f[2 * k], f[2 * k + 1]);
  }
}

// L1 loss in log1p space of y + base (base optional) against target t
// (P, 3): sum |y + base - t| into *loss, gradient sign(.) * scale into g
// (bf16, channel stride gs; pad channels 3..gs-1 zero)
__global__ void k_l1_loss(long long P, const float* __restrict__ y32, int y_stride, const float* __restrict__ base,
                          const float* __restrict__ t, float scale, bf16* __restrict__ g, int gs,
                          float* __restrict__ loss) {
  float s = 0.0f;
  RX_EW_LOOP(P) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      float dlt = (y32[i * y_stride + k] + (base ? base[3 * i + k] : 0.0f)) - t[3 * i + k];
      s += fabsf(dlt);
      g[i * gs + k] = __float2bfloat16_rn(dlt > 0.0f ? scale : (dlt < 0.0f ? -scale : 0.0f));
    }
    for (int k = 3; k < gs; ++k) g[i * gs + k] = __float2bfloat16_rn(0.0f);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, s);
}

// radiance = max(expm1(y + base), 0) from the head's first three channels
__global__ void k_output(long long P, const float* __restrict__ y32, int y_stride, const float* __restrict__ base,
                         float* __restrict__ out) {
  RX_EW_LOOP(P) {
#pragma unroll
    for (int k = 0; k < 3; ++k)
      out[3 * i + k] = fmaxf(expm1f(y32[i * y_stride + k] + (base ? base[3 * i + k] : 0.0f)), 0.0f);
  }
}

// Adam (Kingma and Ba, 2015) on float32 master weights; writes the bf16
// copy the convolutions read and clears the gradient
__global__ void k_adam(long long n, float* __restrict__ p, float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, bf16* __restrict__ p16, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  RX_EW_LOOP(n) {
    float gi = g[i];
    float mi = b1 * m[i] + (1.0f - b1) * gi;
    float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    if (p16) p16[i] = __float2bfloat16_rn(pi);
    g[i] = 0.0f;
  }
}

static int ew_blocks(Ctx* ctx, long long n) {
  return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, (long long)ctx->num_sms * 32));
}

static bool conv_ok(const rx_conv_desc* d) {
  return d && d->N > 0 && d->H > 0 && d->W > 0 && d->Cin > 0 && d->Cout > 0 && d->Cin % 16 == 0 &&
         d->Cout % 16 == 0 && d->x_cstride % 8 == 0 && d->x_coff % 8 == 0 && d->y_cstride % 8 == 0 &&
         d->y_coff % 8 == 0 && d->x_coff + d->Cin <= d->x_cstride && d->y_coff + d->Cout <= d->y_cstride;
}

template <int COUT>
static int launch_tc(Ctx* ctx, const rx_conv_desc* d, const bf16* x, const bf16* w, const float* bias, bf16* y,
                     float* y32, int relu, cudaStream_t st) {
  constexpr int smem = 2 * tc::stage_bytes(COUT);
  static int attr_dev = -1;
  if (attr_dev != ctx->device) {
    CUDA_TRY(ctx, cudaFuncSetAttribute(k_conv_fwd_tc<COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr_dev = ctx->device;
  }
  dim3 grid((unsigned)((d->W + tc::TILE - 1) / tc::TILE), (unsigned)d->H, (unsigned)d->N);
  k_conv_fwd_tc<COUT><<<grid, 128, smem, st>>>(*d, x, w, bias, y, y32, relu, ctx->d_err);
  CUDA_TRY(ctx, cudaGetLastError());
  return RX_OK;
}

template <int NG>
static int launch_ws_ng(Ctx* ctx, const rx_conv_desc* d, const bf16* x, const bf16* w, const float* bias, bf16* y,
                        float* y32, const float* acc_in, int relu, int S, int smem, cudaStream_t st, int* rc) {
  const int limit = 232448 - 1024;  // opt-in shared memory per block, less the static part
  static int attr_dev = -1;
  if (attr_dev != ctx->device) {
    if (cudaFuncSetAttribute(k_conv_fwd_ws<NG>, cudaFuncAttributeMaxDynamicSharedMemorySize, limit) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    attr_dev = ctx->device;
  }
  // resident CTAs per SM from shared memory (dynamic + static + the
  // per-block reservation), capped so that every resident CTA gets its
  // tensor memory
  cudaFuncAttributes fa{};
  int smem_sm = 0, reserved = 0;
  cudaFuncGetAttributes(&fa, k_conv_fwd_ws<NG>);
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->device);
  cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, ctx->device);
  constexpr int tcols = 2 * NG < 32 ? 32 : 2 * NG;
  int per_sm = smem_sm / (smem + (int)fa.sharedSizeBytes + reserved);
  per_sm = std::max(1, std::min(std::min(per_sm, 512 / tcols), 9));  // 9 x 224 threads
  const int G = d->Cout / NG;
  const long long total = (long long)d->N * d->H * ((d->W + tc::TILE - 1) / tc::TILE);
  const long long strips_want = std::max<long long>(1, (long long)ctx->num_sms * per_sm / G);
  const long long per_cta = (total + std::min(total, strips_want) - 1) / std::min(total, strips_want);
  const long long strips = (total + per_cta - 1) / per_cta;
  k_conv_fwd_ws<NG><<<(unsigned)(strips * G), 224, smem, st>>>(*d, x, w, bias, y, y32, acc_in, relu, S, G,
                                                                 per_cta, ctx->d_err);
  cudaError_t e = cudaGetLastError();
  *rc = e == cudaSuccess ? RX_OK : (set_error(ctx, "conv_bf16_fwd: %s", cudaGetErrorString(e)), RX_ERR_CUDA);
  return 1;
}

// Warp-specialised tcgen05 kernel: the widest output-channel group (128,
// 64, 32 or 16, dividing Cout) whose weights fit in shared memory beside a
// ring of at least 4 input rows (6 where they fit).  Returns 1 if it
// launched, 0 if the shape or the pointers do not suit it.
// Output-channel group for the warp-specialised kernel at this Cin / Cout,
// and the ring's row slots; 0 when the weights do not fit.
static int ws_group(int Cin, int Cout, int* S_out, int* smem_out) {
  const int limit = 232448 - 1024;
  const int SB = tc::slot_bytes(Cin);
  int NG = 0;
  // at most two groups: every group re-reads the input rows, and a UMMA's
  // cost is mostly its A (pixel) operand read, so narrow groups do not pay
  for (int ng = 128; ng >= 16; ng >>= 1)
    if (Cout % ng == 0 && Cout / ng <= 2 && tc::weights_bytes(Cin, ng) + 4 * SB + 128 <= limit) {
      NG = ng;
      break;
    }
  if (!NG) return 0;
  *S_out = std::min(6, (limit - 128 - tc::weights_bytes(Cin, NG)) / SB);
  *smem_out = tc::weights_bytes(Cin, NG) + *S_out * SB + 128;
  return NG;
}

static int launch_ws(Ctx* ctx, const rx_conv_desc* d, const bf16* x, const bf16* w, const float* bias, bf16* y,
                     float* y32, const float* acc_in, int relu, cudaStream_t st, int* rc) {
  if (((uintptr_t)x & 15) || ((uintptr_t)w & 15) || ((uintptr_t)y & 15) || ((uintptr_t)y32 & 15) ||
      ((uintptr_t)acc_in & 15))
    return 0;
  int S = 0, smem = 0;
  const int NG = ws_group(d->Cin, d->Cout, &S, &smem);
  switch (NG) {
    case 128: return launch_ws_ng<128>(ctx, d, x, w, bias, y, y32, acc_in, relu, S, smem, st, rc);
    case 64: return launch_ws_ng<64>(ctx, d, x, w, bias, y, y32, acc_in, relu, S, smem, st, rc);
    case 32: return launch_ws_ng<32>(ctx, d, x, w, bias, y, y32, acc_in, relu, S, smem, st, rc);
    case 16: return launch_ws_ng<16>(ctx, d, x, w, bias, y, y32, acc_in, relu, S, smem, st, rc);
    default: return 0;
  }
}

// Input channels [p * cp, (p + 1) * cp) of weights [Cout][9][Cin] as
// contiguous [Cout][9][cp], for p = 0, 1 (16-byte chunks).
__global__ void k_weight_halves(int Cout, int Cin, const uint4* __restrict__ w, uint4* __restrict__ out) {
  const int cp8 = Cin / 16, c8 = Cin / 8;  // chunks per half row, per row
  const long long n = (long long)Cout * 9 * c8;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long row = i / c8;
    const int k = (int)(i - row * c8), half = k / cp8;
    out[(long long)half * Cout * 9 * cp8 + row * cp8 + (k - half * cp8)] = w[i];
  }
}

// A layer whose weights do not fit beside the row ring in one launch, run
// as two launches over the halves of its input channels: the first writes
// fp32 partial sums, the second adds them before the bias and activation
// (sum over channels [0, Cin/2), then [Cin/2, Cin), then + bias).  Returns
// 1 if it launched.
static int launch_ws_split(Ctx* ctx, const rx_conv_desc* d, const bf16* x, const bf16* w, const float* bias, bf16* y,
                           float* y32, int relu, cudaStream_t st, int* rc) {
  const int cp = d->Cin / 2;
  int S = 0, smem = 0;
  if (d->Cin % 32 || !ws_group(cp, d->Cout, &S, &smem)) return 0;
  if (((uintptr_t)x & 15) || ((uintptr_t)w & 15) || ((uintptr_t)y & 15) || ((uintptr_t)y32 & 15)) return 0;
  const long long P = (long long)d->N * d->H * d->W;
  const size_t wbytes = sizeof(bf16) * (size_t)d->Cout * 9 * d->Cin;
  void* halves = nullptr;
  float* part = nullptr;
  // stream-ordered on the caller's stream, which runs the launches
  if (cudaMallocAsync(&halves, wbytes, st) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (cudaMallocAsync((void**)&part, sizeof(float) * (size_t)P * d->Cout, st) != cudaSuccess) {
    cudaGetLastError();
    cudaFreeAsync(halves, st);
    return 0;
  }
  const long long chunks = (long long)d->Cout * 9 * (d->Cin / 8);
  k_weight_halves<<<(int)std::min<long long>((chunks + 255) / 256, (long long)ctx->num_sms * 8), 256, 0, st>>>(
      d->Cout, d->Cin, reinterpret_cast<const uint4*>(w), static_cast<uint4*>(halves));
  const bf16* w0 = static_cast<const bf16*>(halves);
  const bf16* w1 = w0 + (size_t)d->Cout * 9 * cp;
  rx_conv_desc d0 = *d, d1 = *d;
  d0.Cin = d1.Cin = cp;
  d1.x_coff = d->x_coff + cp;
  d0.y_cstride = d->Cout;  // the partial sums: [pixel][Cout]
  d0.y_coff = 0;
  const int first = launch_ws(ctx, &d0, x, w0, nullptr, nullptr, part, nullptr, 0, st, rc);
  int second = 0;
  if (first && *rc == RX_OK) second = launch_ws(ctx, &d1, x, w1, bias, y, y32, part, relu, st, rc);
  cudaFreeAsync(part, st);
  cudaFreeAsync(halves, st);
  if (!first) return 0;  // the kernel is not available: the caller falls back
  if (*rc == RX_OK && !second) {
    // same kernel and shape as the first launch, so this does not happen
    set_error(ctx, "conv_bf16_fwd: second half of a split layer did not launch");
    *rc = RX_ERR_CUDA;
  }
  return 1;
}

int conv_fwd(Ctx* ctx, const rx_conv_desc* d, const void* x, const void* w, const float* bias, void* y, float* y32,
             int relu, cudaStream_t st) {
  if (!conv_ok(d) || !x || !w || !y)
    return set_error(ctx, "conv_bf16_fwd: bad descriptor (channels multiples of 16, strides of 8)"), RX_ERR_ARG;
  if (ctx->conv_impl == 0) {
    int rc = RX_OK;
    if (launch_ws(ctx, d, static_cast<const bf16*>(x), static_cast<const bf16*>(w), bias, static_cast<bf16*>(y), y32,
                  nullptr, relu, st, &rc) ||
        launch_ws_split(ctx, d, static_cast<const bf16*>(x), static_cast<const bf16*>(w), bias,
                        static_cast<bf16*>(y), y32, relu, st, &rc))
      return rc;
  } else if (ctx->conv_impl == 2 && d->H <= 65535 && d->N <= 65535) {
    const bf16* xb = static_cast<const bf16*>(x);
    const bf16* wb = static_cast<const bf16*>(w);
    bf16* yb = static_cast<bf16*>(y);
    switch (d->Cout) {
      case 16: return launch_tc<16>(ctx, d, xb, wb, bias, yb, y32, relu, st);
      case 32: return launch_tc<32>(ctx, d, xb, wb, bias, yb, y32, relu, st);
      case 64: return launch_tc<64>(ctx, d, xb, wb, bias, yb, y32, relu, st);
      case 128: return launch_tc<128>(ctx, d, xb, wb, bias, yb, y32, relu, st);
      default: break;
    }
  }
  long long P = (long long)d->N * d->H * d->W;
  dim3 grid((unsigned)((P + 63) / 64), 1);
  const bf16* xb = static_cast<const bf16*>(x);
  const bf16* wb = static_cast<const bf16*>(w);
  bf16* yb = static_cast<bf16*>(y);
  bool bk32 = d->Cin % 32 == 0;
  if (d->Cout >= 128) {
    grid.y = (unsigned)((d->Cout + 127) / 128);
    if (bk32) k_conv_fwd<128, 32><<<grid, 128, 0, st>>>(*d, xb, wb, bias, yb, y32, relu);
    else k_conv_fwd<128, 16><<<grid, 128, 0, st>>>(*d, xb, wb, bias, yb, y32, relu);
  } else if (d->Cout > 32) {
    grid.y = (unsigned)((d->Cout + 63) / 64);
    if (bk32) k_conv_fwd<64, 32><<<grid, 128, 0, st>>>(*d, xb, wb, bias, yb, y32, relu);
    else k_conv_fwd<64, 16><<<grid, 128, 0, st>>>(*d, xb, wb, bias, yb, y32, relu);
  } else {
    grid.y = (unsigned)((d->Cout + 31) / 32);
    if (bk32) k_conv_fwd<32, 32><<<grid, 128, 0, st>>>(*d, xb, wb, bias, yb, y32, relu);
    else k_conv_fwd<32, 16><<<grid, 128, 0, st>>>(*d, xb, wb, bias, yb, y32, relu);
  }
  CUDA_TRY(ctx, cudaGetLastError());
  return RX_OK;
}

int conv_bwd_data(Ctx* ctx, const rx_conv_desc* d, const void* dy, const void* w, void* w_rot, void* dx,
                  cudaStream_t st) {
  if (!conv_ok(d) || !dy || !w || !w_rot || !dx) return set_error(ctx, "conv_bf16_bwd_data: bad arguments"), RX_ERR_ARG;
  long long nw = (long long)d->Cout * 9 * d->Cin;
  k_rot_weights<<<ew_blocks(ctx, nw), 256, 0, st>>>(d->Cout, d->Cin, static_cast<const bf16*>(w),
                                                   static_cast<bf16*>(w_rot));
  CUDA_TRY(ctx, cudaGetLastError());
  // dx = conv(dy, w_rot): input channels Cout (read from the y view), output Cin (the x view)
  rx_conv_desc t = *d;
  t.Cin = d->Cout;
  t.Cout = d->Cin;
  t.x_cstride = d->y_cstride;
  t.x_coff = d->y_coff;
  t.y_cstride = d->x_cstride;
  t.y_coff = d->x_coff;
  return conv_fwd(ctx, &t, dy, w_rot, nullptr, dx, nullptr, 0, st);
}

int conv_bwd_weight(Ctx* ctx, const rx_conv_desc* d, const void* dy, const void* x, float* dw, float* db,
                    cudaStream_t st) {
  if (!conv_ok(d) || !dy || !x || !dw) return set_error(ctx, "conv_bf16_bwd_weight: bad arguments"), RX_ERR_ARG;
  long long P = (long long)d->N * d->H * d->W;
  // enough pixel chunks to fill the GPU with every (tap, channel block)
  int cb = ((d->Cout + 63) / 64) * ((d->Cin + 63) / 64);
  long long want = (long long)ctx->num_sms * 4 / std::max(1, 9 * cb) + 1;
  int ppb = (int)std::max<long long>(256, ((P + want - 1) / want + 31) / 32 * 32);
  dim3 grid((unsigned)((P + ppb - 1) / ppb), (unsigned)cb, 9);
  k_conv_wgrad<<<grid, 128, 0, st>>>(*d, static_cast<const bf16*>(dy), static_cast<const bf16*>(x), dw, ppb);
  CUDA_TRY(ctx, cudaGetLastError());
  if (db) {
    int bppb = 4096;
    k_bias_grad<<<(unsigned)((P + bppb - 1) / bppb), 128, 0, st>>>(*d, static_cast<const bf16*>(dy), db, bppb);
    CUDA_TRY(ctx, cudaGetLastError());
  }
  return RX_OK;
}

int dn_op(Ctx* ctx, const rx_dn_op* o, cudaStream_t st) {
  if (!o) return set_error(ctx, "dn_op: NULL"), RX_ERR_ARG;
  const bf16* a = static_cast<const bf16*>(o->a);
  bf16* b = static_cast<bf16*>(o->b);
  long long P = (long long)o->N * o->H * o->W;
  // 16-byte chunks when channel count, strides, offsets and bases allow
  const bool v8 = o->C % 8 == 0 && o->a_stride % 8 == 0 && o->a_off % 8 == 0 && o->b_stride % 8 == 0 &&
                  o->b_off % 8 == 0 && ((uintptr_t)a & 15) == 0 && ((uintptr_t)b & 15) == 0;
  switch (o->kind) {
    case RX_DN_COPY:
      k_copy_ch<<<ew_blocks(ctx, P * o->C), 256, 0, st>>>(P, o->C, a, o->a_stride, o->a_off, b, o->b_stride, o->b_off,
                                                         o->flag);
      break;
    case RX_DN_RELU_MASK:
      k_relu_mask<<<ew_blocks(ctx, P * o->C), 256, 0, st>>>(P, o->C, a, o->a_stride, o->a_off, b, o->b_stride,
                                                           o->b_off);
      break;
    case RX_DN_POOL:
      if (o->H % 2 || o->W % 2) return set_error(ctx, "dn_op: pool needs even H and W"), RX_ERR_ARG;
      if (v8)
        k_pool2_v8<<<ew_blocks(ctx, P / 4 * (o->C / 8)), 256, 0, st>>>(o->N, o->H, o->W, o->C, a, o->a_stride,
                                                                      o->a_off, b, o->b_stride, o->b_off);
      else
        k_pool2<<<ew_blocks(ctx, P / 4 * o->C), 256, 0, st>>>(o->N, o->H, o->W, o->C, a, o->a_stride, o->a_off, b,
                                                             o->b_stride, o->b_off);
      break;
    case RX_DN_POOL_BWD:
      if (o->H % 2 || o->W % 2) return set_error(ctx, "dn_op: pool needs even H and W"), RX_ERR_ARG;
      k_pool2_bwd<<<ew_blocks(ctx, P * o->C), 256, 0, st>>>(o->N, o->H, o->W, o->C, a, o->a_stride, o->a_off, b,
                                                           o->b_stride, o->b_off, o->flag);
      break;
    case RX_DN_UP:
      if (v8)
        k_up2_v8<<<ew_blocks(ctx, P * (o->C / 8)), 256, 0, st>>>(o->N, o->H, o->W, o->C, a, o->a_stride, o->a_off, b,
                                                                o->b_stride, o->b_off);
      else
        k_up2<<<ew_blocks(ctx, 4 * P * o->C), 256, 0, st>>>(o->N, o->H, o->W, o->C, a, o->a_stride, o->a_off, b,
                                                           o->b_stride, o->b_off);
      break;
    case RX_DN_UP_BWD:
      k_up2_bwd<<<ew_blocks(ctx, P * o->C), 256, 0, st>>>(o->N, o->H, o->W, o->C, a, o->a_stride, o->a_off, b,
                                                         o->b_stride, o->b_off);
      break;
    default:
      return set_error(ctx, "dn_op: unknown kind %d", o->kind), RX_ERR_ARG;
  }
  CUDA_TRY(ctx, cudaGetLastError());
  return RX_OK;
}

int dn_features(Ctx* ctx, long long P, const float* rad, const float* alb, const float* nrm, const float* dep,
                void* out, float* base, cudaStream_t st) {
  if (P <= 0 || !rad || !alb || !nrm || !dep || !out) return set_error(ctx, "dn_features: bad arguments"), RX_ERR_ARG;
  k_features<<<ew_blocks(ctx, P), 256, 0, st>>>(P, rad, alb, nrm, dep, static_cast<bf16*>(out), base);
  CUDA_TRY(ctx, cudaGetLastError());
  return RX_OK;
}

int dn_l1_loss(Ctx* ctx, long long P, const float* y32, int y_stride, const float* base, const float* target,
               float scale, void* grad, int grad_stride, float* loss, cudaStream_t st) {
  if (P <= 0 || !y32 || !target || !grad || !loss || y_stride < 3 || grad_stride < 3)
    return set_error(ctx, "dn_l1_loss: bad arguments"), RX_ERR_ARG;
  k_l1_loss<<<ew_blocks(ctx, P), 256, 0, st>>>(P, y32, y_stride, base, target, scale, static_cast<bf16*>(grad),
                                               grad_stride, loss);
  CUDA_TRY(ctx, cudaGetLastError());
  return RX_OK;
}

int dn_output(Ctx* ctx, long long P, const float* y32, int y_stride, const float* base, float* out,
              cudaStream_t st) {
  if (P <= 0 || !y32 || !out || y_stride < 3) return set_error(ctx, "dn_output: bad arguments"), RX_ERR_ARG;
  k_output<<<ew_blocks(ctx, P), 256, 0, st>>>(P, y32, y_stride, base, out);
  CUDA_TRY(ctx, cudaGetLastError());
  return RX_OK;
}

int dn_adam(Ctx* ctx, long long n, float* p, float* g, float* m, float* v, void* p16, float lr, float b1, float b2,
            float eps, int step, cudaStream_t st) {
  if (n <= 0 || !p || !g || !m || !v || step < 1) return set_error(ctx, "dn_adam: bad arguments"), RX_ERR_ARG;
  float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  k_adam<<<ew_blocks(ctx, n), 256, 0, st>>>(n, p, g, m, v, static_cast<bf16*>(p16), lr, b1, b2, eps, c1, c2);
  CUDA_TRY(ctx, cudaGetLastError());
  return RX_OK;
}

}  // namespace rx
