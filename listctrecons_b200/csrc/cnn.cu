// Learned 2.5D residual correction after backprojection (no reference counterpart; the
// reference stops at the FDK volume, Src/Reconstructor.cpp).
//
// Network: 5 neighbouring slices of the (calibrated) FDK volume as channels -> 8 zero-padded
// 3x3 convolutions (5->32, 6 x 32->32, 32->1), ReLU between them -> a residual r added to the
// centre slice.  BF16 weights and activations, FP32 accumulation.
//
// HBM layout: every activation / delta is channels-last bf16 [B][H][W+2][32] (64 bytes per
// pixel; one zero pad column on each side, pixel x at column x+1; channels beyond a layer's
// width are zero).  Weights are packed per layer as bf16 [N][9 taps x 32 channels].
//
// Convolution = implicit GEMM on tcgen05 in a persistent, warp-specialised kernel: a tile is
// 8 px x 16 rows (M 128) x N output channels (N = 32, or 16 for the 1-channel last layer) over
// K = 9 taps x 32 channels.  Per tile, three 4-D TMA boxes {32 ch, 8 px, 18 rows, 1 slice} with
// 64-byte swizzle (one per column offset; rows outside the image come back as TMA's zero fill)
// serve all nine taps, each row offset being a whole swizzle atom; the packed weights
// (9 x N x 64 bytes) are loaded once per CTA; two M128 x N x K16 MMAs per tap accumulate in one
// of two TMEM buffers.  Fused epilogues: bias + ReLU -> bf16 (forward), ReLU mask of the
// previous activation -> bf16 delta (backward data), FP32 residual (training), and the
// acceptance gate writing the corrected volume (inference).
// Weight gradients: the same tcgen05 machinery with K = pixels (both operands MN-major).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <new>
#include <vector>

#include "lct_internal.h"
#include "tc_ptx.cuh"

namespace lct {

constexpr int kCnnLayers = 8, kCnnC = 32, kCnnTaps = 9, kCnnK = kCnnTaps * kCnnC;  // K = 288
constexpr int kCnnParams = 57249;     // sum over layers of cin*cout*9 + cout
constexpr int kWSlot = kCnnC * kCnnK;  // packed weights of one layer, elements
// output tile 8 px x 16 rows = the M 128 of one MMA; M row m = row * 8 + px
constexpr int kConvTW = 8, kConvTH = 16, kConvM = kConvTW * kConvTH;
constexpr int kConvStages = 6;    // A boxes in flight (3 per tile)
constexpr int kConvThreads = 192; // warp 0 TMA, warp 1 MMA + TMEM, warps 2-5 epilogue

LCT_HD constexpr int cnn_cin(int l) { return l == 0 ? 5 : 32; }
LCT_HD constexpr int cnn_cout(int l) { return l == kCnnLayers - 1 ? 1 : 32; }
LCT_HD constexpr int cnn_off(int l) { return l == 0 ? 0 : 1472 + (l - 1) * 9248; }

enum ConvEpi : int { kEpiRelu = 0, kEpiMask = 1, kEpiResid = 2, kEpiGate = 3 };

struct ConvArgs {
  int H, W, wp, tiles_x, tiles_y;
  long long n_tiles;
  const float* bias;               // [N] (forward epilogues)
  __nv_bfloat16* out_act;          // Relu / Mask: [B][H][wp][32]
  const __nv_bfloat16* mask_act;   // Mask: activation whose sign gates the delta
  float* out_f;                    // Resid: r [B][H][W]; Gate: corrected slices [B][H][W]
  const float* xc;                 // Gate: plain slices [B][H][W]
  float calib, inv_scale, bound;   // Gate
  unsigned long long* n_reject;    // Gate
  int* status;
};

template <int N>
struct ConvCfg {
  // one A box: 32 channels x 8 px x 18 rows (the tile's rows and one halo row on each side)
  static constexpr uint32_t BoxA = kConvTW * (kConvTH + 2) * kCnnC * 2;  // 9216 B
  static constexpr uint32_t RowA = kConvTW * kCnnC * 2;                  // 512 B = one atom
  static constexpr uint32_t TapB = N * kCnnC * 2;        // 2 KB (N=32) or 1 KB (N=16)
  static constexpr uint32_t BBytes = kCnnTaps * TapB;
  static constexpr uint32_t Smem = 1024 + kConvStages * BoxA + BBytes + 256;
  static constexpr uint32_t TmemCols = 64;  // two 32-column accumulators
  static constexpr uint32_t Idesc = (1u << 4) | (1u << 7) | (1u << 10) |
                                    ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kConvM >> 4) << 24);
};

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

__device__ __forceinline__ void conv_tile(const ConvArgs& a, long long t, int& x0, int& y0,
                                          int& b) {
  const long long per = (long long)a.tiles_x * a.tiles_y;
  b = (int)(t / per);
  const int r = (int)(t % per);
  y0 = (r / a.tiles_x) * kConvTH;
  x0 = (r % a.tiles_x) * kConvTW;
}

__device__ __forceinline__ bool conv_aborted(int* flag) {
  return *reinterpret_cast<volatile int*>(flag) != 0;
}

// Persistent implicit-GEMM 3x3 convolution: CTA c takes tiles c, c + grid, ...  Per tile, three
// A boxes (one per column offset dx) feed nine taps: tap (dy, dx) reads box dx from row dy,
// i.e. at +dy * 512 bytes -- a whole 64-byte-swizzle atom, so every operand start stays on the
// swizzle pattern.  Two TMEM accumulators let the epilogue of one tile overlap the MMAs of the
// next.  Every wait is bounded; on a timeout the CTA drains its copies and MMAs, raises the
// device status word and leaves its remaining tiles unwritten.
template <int N, int EPI>
__global__ void __launch_bounds__(kConvThreads, 3)
    conv_tc_kernel(const __grid_constant__ CUtensorMap mx, const __grid_constant__ CUtensorMap mw,
                   const ConvArgs a) {
  using Cfg = ConvCfg<N>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint8_t* sa = smem;
  uint8_t* sb = smem + kConvStages * Cfg::BoxA;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sb + Cfg::BBytes);
  // full[S] empty[S] wbar acc_full[2] acc_empty[2] mma_done
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kConvStages + 6);
  __shared__ int s_abort;
  __shared__ float s_bias[32];  // the layer's biases, read by every tile's epilogue

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t full0 = smem_u32(&bars[0]);
  const uint32_t empty0 = smem_u32(&bars[kConvStages]);
  const uint32_t wbar = smem_u32(&bars[2 * kConvStages]);
  const uint32_t accf0 = smem_u32(&bars[2 * kConvStages + 1]);
  const uint32_t acce0 = smem_u32(&bars[2 * kConvStages + 3]);
  const uint32_t mdone = smem_u32(&bars[2 * kConvStages + 5]);

  if (threadIdx.x < 32)
    s_bias[threadIdx.x] = (EPI != kEpiMask && threadIdx.x < N) ? a.bias[threadIdx.x] : 0.f;
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int s = 0; s < kConvStages; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    mbar_init(wbar, 1);
    for (int i = 0; i < 2; ++i) {
      mbar_init(accf0 + 8 * i, 1);
      mbar_init(acce0 + 8 * i, 4);  // one arrival per epilogue warp
    }
    mbar_init(mdone, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(Cfg::TmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      // producer: the layer's packed weights once, then three A boxes per tile
      mbar_expect_tx(wbar, Cfg::BBytes);
      for (int k = 0; k < kCnnTaps; ++k)
        tma_load_2d(smem_u32(sb + k * Cfg::TapB), &mw, k * kCnnC, 0, wbar);
      long long kg = 0;
      bool stop = false;
      for (long long t = blockIdx.x; t < a.n_tiles && !stop; t += gridDim.x) {
        int x0, y0, b;
        conv_tile(a, t, x0, y0, b);
        for (int l = 0; l < 3; ++l, ++kg) {
          const int s = (int)(kg % kConvStages);
          if (kg >= kConvStages &&
              !mbar_wait(empty0 + 8 * s, (uint32_t)(((kg / kConvStages) - 1) & 1))) {
            atomicExch(&s_abort, 1);
            stop = true;
            break;
          }
          if (conv_aborted(&s_abort)) {
            stop = true;
            break;
          }
          mbar_expect_tx(full0 + 8 * s, Cfg::BoxA);
          // pixel x of the tile, column offset dx = l - 1, sits at padded column x + l
          tma_load_4d(smem_u32(sa + s * Cfg::BoxA), &mx, 0, x0 + l, y0 - 1, b, full0 + 8 * s);
        }
      }
      if (conv_aborted(&s_abort)) {  // let copies in flight land before the CTA exits
        mbar_wait(wbar, 0);
        for (long long k = (kg > kConvStages ? kg - kConvStages : 0); k < kg; ++k)
          mbar_wait(full0 + 8 * (int)(k % kConvStages), (uint32_t)((k / kConvStages) & 1));
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issuer
      bool ok = mbar_wait(wbar, 0);
      if (!ok) atomicExch(&s_abort, 1);
      long long kg = 0;
      int it = 0;
      for (long long t = blockIdx.x; t < a.n_tiles && ok; t += gridDim.x, ++it) {
        const int buf = it & 1;
        if (it >= 2 && !mbar_wait(acce0 + 8 * buf, (uint32_t)(((it >> 1) - 1) & 1))) {
          atomicExch(&s_abort, 1);
          break;
        }
        if (conv_aborted(&s_abort)) break;
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(buf * 32);
        for (int l = 0; l < 3 && ok; ++l, ++kg) {
          const int s = (int)(kg % kConvStages);
          if (!mbar_wait(full0 + 8 * s, (uint32_t)((kg / kConvStages) & 1))) {
            atomicExch(&s_abort, 1);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t base = smem_u32(sa + s * Cfg::BoxA);
#pragma unroll
          for (int dy = 0; dy < 3; ++dy) {
            const uint64_t da = desc_sw64(base + dy * Cfg::RowA);
            const uint64_t db = desc_sw64(smem_u32(sb + (dy * 3 + l) * Cfg::TapB));
            umma_bf16(d, da, db, Cfg::Idesc, (l | dy) ? 1u : 0u);
            umma_bf16(d, da + 2, db + 2, Cfg::Idesc, 1u);  // +32 bytes: channels 16..31
          }
          umma_commit(empty0 + 8 * s);
        }
        if (!ok) break;
        umma_commit(accf0 + 8 * buf);
      }
      umma_commit(mdone);  // every MMA issued above has finished once this arrives
      if (!mbar_wait(mdone, 0)) atomicExch(&s_abort, 1);
    }
  } else {
    // epilogue: warp w reads TMEM lanes 32 * (w % 4) ... + 31
    const int qd = warp & 3;
    const int m = qd * 32 + lane;
    const int yy = m / kConvTW, px = m % kConvTW;
    const float* bias = s_bias;
    int it = 0;
    for (long long t = blockIdx.x; t < a.n_tiles; t += gridDim.x, ++it) {
      const int buf = it & 1;
      // warp-uniform decision: the TMEM load below is .sync.aligned
      const bool got = __all_sync(0xFFFFFFFFu, mbar_wait(accf0 + 8 * buf, (uint32_t)((it >> 1) & 1)));
      if (!got) {
        if (lane == 0) atomicExch(&s_abort, 1);
        break;
      }
      if (__any_sync(0xFFFFFFFFu, conv_aborted(&s_abort))) break;
      tc_fence_after();
      int x0, y0, b;
      conv_tile(a, t, x0, y0, b);
      const int x = x0 + px, y = y0 + yy;
      const bool in = x < a.W && y < a.H;
      const uint32_t ta = tmem + (uint32_t)(buf * 32) + ((uint32_t)(qd * 32) << 16);
      if constexpr (N == 32) {
        uint32_t r[32];
        tmem_ld32(ta, r);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(acce0 + 8 * buf);
        if (in) {
          const long long pix = ((long long)b * a.H + y) * a.wp + x + 1;
          uint4* dst = reinterpret_cast<uint4*>(a.out_act + pix * kCnnC);
          if constexpr (EPI == kEpiRelu) {
#pragma unroll
            for (int g = 0; g < 4; ++g) {
              float v[8];
#pragma unroll
              for (int j = 0; j < 8; ++j)
                v[j] = fmaxf(__uint_as_float(r[8 * g + j]) + bias[8 * g + j], 0.f);
              dst[g] = make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]),
                                  pack_bf16x2(v[4], v[5]), pack_bf16x2(v[6], v[7]));
            }
          } else {
            const uint4* msk = reinterpret_cast<const uint4*>(a.mask_act + pix * kCnnC);
#pragma unroll
            for (int g = 0; g < 4; ++g) {
              const uint4 mv = msk[g];
              const uint32_t mwd[4] = {mv.x, mv.y, mv.z, mv.w};
              float v[8];
#pragma unroll
              for (int j = 0; j < 8; ++j) {
                const int16_t bits = (int16_t)((mwd[j >> 1] >> (16 * (j & 1))) & 0xFFFFu);
                v[j] = bits > 0 ? __uint_as_float(r[8 * g + j]) : 0.f;
              }
              dst[g] = make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]),
                                  pack_bf16x2(v[4], v[5]), pack_bf16x2(v[6], v[7]));
            }
          }
        }
      } else {
        uint32_t r[16];
        tmem_ld16(ta, r);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(acce0 + 8 * buf);
        const long long o = ((long long)b * a.H + y) * a.W + x;
        const float rr = __uint_as_float(r[0]) + bias[0];
        if constexpr (EPI == kEpiResid) {
          if (in) a.out_f[o] = rr;
        } else {
          bool rej = false;
          if (in) {
            const float plain = a.calib * a.xc[o];
            const float dlt = rr * a.inv_scale;
            const bool keep = fabsf(dlt) <= a.bound;  // NaN fails the test: plain is kept
            a.out_f[o] = keep ? plain + dlt : plain;
            rej = !keep;
          }
          const unsigned msk = __ballot_sync(0xFFFFFFFFu, rej);
          if (lane == 0 && msk && a.n_reject)
            atomicAdd(a.n_reject, (unsigned long long)__popc(msk));
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0 && conv_aborted(&s_abort) && a.status) atomicExch(a.status, kDevWaitTimeout);
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(Cfg::TmemCols)
                 : "memory");
}

// Network input: channel k of slice b = k_in * plane(b, k), k < 5; pads and channels >= 5 zero.
// plane(b, k) = b*5 + k for stacked training inputs [B][5][H][W], or the volume slice
// clamp(z0 + b + k - 2, 0, nz - 1) for inference over a volume [nz][H][W].
__global__ void cnn_prep_kernel(const float* __restrict__ src, int vol_mode, int z0, int nz,
                                int B, int H, int W, int wp, float k_in,
                                __nv_bfloat16* __restrict__ a0) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)B * H * wp) return;
  const int col = (int)(i % wp);
  const long long q = i / wp;
  const int y = (int)(q % H), b = (int)(q / H), x = col - 1;
  float v[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  if (x >= 0 && x < W) {
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      long long plane;
      if (vol_mode) {
        int z = z0 + b + k - 2;
        z = z < 0 ? 0 : (z > nz - 1 ? nz - 1 : z);
        plane = z;
      } else {
        plane = (long long)b * 5 + k;
      }
      v[k] = __fmul_rn(k_in, src[(plane * H + y) * W + x]);
    }
  }
  uint4* dst = reinterpret_cast<uint4*>(a0 + i * kCnnC);
  dst[0] = make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]), pack_bf16x2(v[4], 0.f), 0u);
  dst[1] = make_uint4(0u, 0u, 0u, 0u);
  dst[2] = make_uint4(0u, 0u, 0u, 0u);
  dst[3] = make_uint4(0u, 0u, 0u, 0u);
}

// MSE loss of (k_in x_c + r) against s t and its gradient 2 d / n -> channel 0 of the last
// layer's delta (bf16, padded layout); sum of d^2 accumulated in FP64.
__global__ void __launch_bounds__(256) cnn_loss_kernel(const float* __restrict__ in5,
                                                       const float* __restrict__ r,
                                                       const float* __restrict__ tgt, int B,
                                                       int H, int W, int wp, float k_in, float s,
                                                       float two_over_n, __nv_bfloat16* dz,
                                                       double* loss) {
  __shared__ float red[8];
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long hw = (long long)H * W;
  float d2 = 0.f;
  if (p < B * hw) {
    const long long b = p / hw, pix = p % hw;
    const int y = (int)(pix / W), x = (int)(pix % W);
    const float xc = in5[(b * 5 + 2) * hw + pix];
    const float yv = __fadd_rn(__fmul_rn(k_in, xc), r[p]);
    const float d = __fsub_rn(yv, __fmul_rn(s, tgt[p]));
    d2 = d * d;
    dz[((b * H + y) * wp + x + 1) * kCnnC] = __float2bfloat16_rn(__fmul_rn(d, two_over_n));
  }
  for (int o = 16; o; o >>= 1) d2 += __shfl_xor_sync(0xFFFFFFFFu, d2, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = d2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double sum = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) sum += red[w];
    atomicAdd(loss, sum);
  }
}

// Weight gradients of one layer on tcgen05, no transposes: with K = pixels, both channels-last
// operands are MN-major (32 channels = one 64-byte swizzle row per pixel, 8 pixels = one atom).
//   D_dx[dy * 32 + ci][co] += sum_p act[p + (dy - 1, dx - 1)][ci] * dz[p][co]
// Per 8 px x 16 rows tile: one activation box {32 ch, 8 px, 19 rows} per dx whose rows r and
// r + 1 .. are the dy blocks (M = 128: the three dy blocks at +512 B and one discarded block),
// and one delta box {32 ch, 8 px, 16 rows} (N = 32); K = 128 pixels = 8 MMAs of K16 per dx.
// A CTA accumulates over all its tiles in three TMEM accumulators and adds them to the gradient
// once.  Pads and rows outside the image are zero in the deltas, so they add nothing.
constexpr int kDwStages = 3, kDwThreads = 128, kDwRows = kConvTH + 3;
struct DwCfg {
  static constexpr uint32_t BoxA = kConvTW * kDwRows * kCnnC * 2;  // 9728 B
  static constexpr uint32_t BoxD = kConvTW * kConvTH * kCnnC * 2;  // 8192 B
  static constexpr uint32_t Stage = 3 * BoxA + BoxD;               // 37376 B, 512-aligned
  static constexpr uint32_t Smem = 1024 + kDwStages * Stage + 128;
  static constexpr uint32_t TmemCols = 128;                         // 3 x 32 used
  static constexpr uint32_t Idesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                                    ((uint32_t)(32 >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
};

__global__ void __launch_bounds__(kDwThreads)
    cnn_dw_tc_kernel(const __grid_constant__ CUtensorMap ma, const __grid_constant__ CUtensorMap mz,
                     const ConvArgs a, int cin, int cout, float* __restrict__ gw) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kDwStages * DwCfg::Stage);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kDwStages + 1);
  __shared__ int s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t full0 = smem_u32(&bars[0]);
  const uint32_t empty0 = smem_u32(&bars[kDwStages]);
  const uint32_t mdone = smem_u32(&bars[2 * kDwStages]);
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int s = 0; s < kDwStages; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    mbar_init(mdone, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(DwCfg::TmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    long long it = 0;
    for (long long t = blockIdx.x; t < a.n_tiles; t += gridDim.x, ++it) {
      const int s = (int)(it % kDwStages);
      if (it >= kDwStages &&
          !mbar_wait(empty0 + 8 * s, (uint32_t)(((it / kDwStages) - 1) & 1))) {
        atomicExch(&s_abort, 1);
        break;
      }
      if (conv_aborted(&s_abort)) break;
      int x0, y0, b;
      conv_tile(a, t, x0, y0, b);
      uint8_t* st = smem + s * DwCfg::Stage;
      const uint32_t fb = full0 + 8 * s;
      mbar_expect_tx(fb, DwCfg::Stage);
      for (int dx = 0; dx < 3; ++dx)  // pixel x, column offset dx - 1: padded column x + dx
        tma_load_4d(smem_u32(st + dx * DwCfg::BoxA), &ma, 0, x0 + dx, y0 - 1, b, fb);
      tma_load_4d(smem_u32(st + 3 * DwCfg::BoxA), &mz, 0, x0 + 1, y0, b, fb);
    }
    if (conv_aborted(&s_abort))  // let copies in flight land before the CTA exits
      for (long long k = (it > kDwStages ? it - kDwStages : 0); k < it; ++k)
        mbar_wait(full0 + 8 * (int)(k % kDwStages), (uint32_t)((k / kDwStages) & 1));
  } else if (warp == 1 && lane == 0) {
    long long it = 0;
    bool first = true;
    for (long long t = blockIdx.x; t < a.n_tiles; t += gridDim.x, ++it) {
      const int s = (int)(it % kDwStages);
      if (!mbar_wait(full0 + 8 * s, (uint32_t)((it / kDwStages) & 1))) {
        atomicExch(&s_abort, 1);
        break;
      }
      tc_fence_after();
      const uint32_t st = smem_u32(smem + s * DwCfg::Stage);
#pragma unroll
      for (int dx = 0; dx < 3; ++dx) {
#pragma unroll
        for (int k = 0; k < kConvTH / 2; ++k) {  // K16 = two 8-pixel atoms = 1024 B
          const uint64_t da = desc_mn_sw64(st + dx * DwCfg::BoxA + k * 1024, 512, 512);
          const uint64_t dz = desc_mn_sw64(st + 3 * DwCfg::BoxA + k * 1024, 512, 512);
          umma_bf16(tmem + dx * 32, da, dz, DwCfg::Idesc, (first && k == 0) ? 0u : 1u);
        }
      }
      first = false;
      umma_commit(empty0 + 8 * s);
    }
    umma_commit(mdone);
  }
  __syncwarp();
  const bool done = __all_sync(0xFFFFFFFFu, mbar_wait(mdone, 0));
  __syncthreads();
  tc_fence_after();
  if (!done || conv_aborted(&s_abort)) {
    if (threadIdx.x == 0 && a.status) atomicExch(a.status, kDevWaitTimeout);
  } else if (blockIdx.x < a.n_tiles) {
    // warp w holds rows 32 w ..: dy = w (w = 3 is the discarded block), ci = lane
    const int dy = warp, ci = lane;
#pragma unroll
    for (int dx = 0; dx < 3; ++dx) {
      uint32_t r[32];
      tmem_ld32(tmem + dx * 32 + ((uint32_t)(warp * 32) << 16), r);
      if (dy < 3 && ci < cin) {
#pragma unroll
        for (int co = 0; co < 32; ++co)
          if (co < cout) atomicAdd(&gw[((co * cin + ci) * 3 + dy) * 3 + dx], __uint_as_float(r[co]));
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(DwCfg::TmemCols)
                 : "memory");
}

// Bias gradients: sum of the deltas over the slices' padded pixels (pads are zero).
__global__ void __launch_bounds__(256) cnn_db_kernel(const __nv_bfloat16* __restrict__ dz,
                                                     long long n_pix, int cout,
                                                     float* __restrict__ gb) {
  __shared__ float red[8][kCnnC];
  const int c = threadIdx.x & 31, g = threadIdx.x >> 5;
  float acc = 0.f;
  for (long long p = (long long)blockIdx.x * 8 + g; p < n_pix; p += (long long)gridDim.x * 8)
    acc += __bfloat162float(dz[p * kCnnC + c]);
  red[g][c] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    float v = 0.f;
    for (int k = 0; k < 8; ++k) v += red[k][threadIdx.x];
    if (threadIdx.x < cout) atomicAdd(&gb[threadIdx.x], v);
  }
}

__global__ void cnn_adam_kernel(float* __restrict__ p, const float* __restrict__ g,
                                float* __restrict__ m, float* __restrict__ v, int n, float lr,
                                float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

// FP32 master weights -> bf16 GEMM operands.  Forward slot l: [co][tap*32 + ci].  Backward
// (data) slot l: [ci][tap*32 + co] holding W[co][ci][8 - tap] (the flipped, transposed kernel).
__global__ void cnn_pack_kernel(const float* __restrict__ p, __nv_bfloat16* __restrict__ wf,
                                __nv_bfloat16* __restrict__ wb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kCnnLayers * kWSlot) return;
  const int l = i / kWSlot, rem = i % kWSlot, row = rem / kCnnK, k = rem % kCnnK;
  const int tap = k / kCnnC, c = k % kCnnC;
  const int cin = cnn_cin(l), cout = cnn_cout(l);
  const float* w = p + cnn_off(l);
  float f = 0.f, bwd = 0.f;
  if (row < cout && c < cin) f = w[(row * cin + c) * 9 + tap];
  if (l > 0 && row < cin && c < cout) bwd = w[(c * cin + row) * 9 + (8 - tap)];
  wf[i] = __float2bfloat16_rn(f);
  wb[i] = __float2bfloat16_rn(bwd);
}

}  // namespace lct

using namespace lct;

struct lct_cnn {
  int device = 0, cap = 0, H = 0, W = 0, wp = 0, sms = 148;
  bool train = false;
  int n_act = 0;
  long long act_elems = 0;
  float* d_p = nullptr;  // params, grads, Adam m, Adam v: 4 x kCnnParams
  float* d_g = nullptr;
  float* d_m = nullptr;
  float* d_v = nullptr;
  __nv_bfloat16* d_wf = nullptr;  // 8 forward slots
  __nv_bfloat16* d_wb = nullptr;  // 8 backward slots (slot 0 unused)
  __nv_bfloat16* d_act = nullptr; // n_act activation buffers
  __nv_bfloat16* d_dz = nullptr;  // training: 3 delta buffers
  float* d_r = nullptr;           // training: residual [cap][H][W]
  double* d_loss = nullptr;
  unsigned long long* d_rej = nullptr;
  CUtensorMap m_act[kCnnLayers], m_dz[3], m_wf[kCnnLayers], m_wb[kCnnLayers];
  CUtensorMap m_dwa[kCnnLayers], m_dwz[3];  // weight-gradient boxes
  float calib = 1.f, in_scale = 1.f;
  int adam_t = 0;
  long long last_n = 0;
};

namespace lct {

static __nv_bfloat16* act_buf(lct_cnn* c, int i) { return c->d_act + (size_t)i * c->act_elems; }
static __nv_bfloat16* dz_buf(lct_cnn* c, int i) { return c->d_dz + (size_t)i * c->act_elems; }
// input buffer of layer l (training keeps every activation; inference ping-pongs two)
static int act_in(const lct_cnn* c, int l) { return c->train ? l : (l & 1); }

// channels-last bf16 [cap][H][wp][32], box {32 ch, 8 px, rows, 1 slice}, 64-byte swizzle
static int act_map(CUtensorMap* m, const void* base, int cap, int H, int wp, int rows) {
  auto fn = tensor_map_encoder();
  if (!fn) return LCT_ERR_UNSUPPORTED;
  cuuint64_t dims[4] = {(cuuint64_t)kCnnC, (cuuint64_t)wp, (cuuint64_t)H, (cuuint64_t)cap};
  cuuint64_t strides[3] = {(cuuint64_t)kCnnC * 2, (cuuint64_t)wp * kCnnC * 2,
                           (cuuint64_t)H * wp * kCnnC * 2};
  cuuint32_t box[4] = {(cuuint32_t)kCnnC, (cuuint32_t)kConvTW, (cuuint32_t)rows, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? LCT_OK : LCT_ERR_UNSUPPORTED;
}

static int weight_map(CUtensorMap* m, const void* base, int rows) {
  auto fn = tensor_map_encoder();
  if (!fn) return LCT_ERR_UNSUPPORTED;
  cuuint64_t dims[2] = {(cuuint64_t)kCnnK, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)kCnnK * 2};
  cuuint32_t box[2] = {(cuuint32_t)kCnnC, (cuuint32_t)rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? LCT_OK : LCT_ERR_UNSUPPORTED;
}

// per device: dynamic shared memory set, and resident CTAs per SM of each variant
static bool conv_attr_done[64];
static int conv_occ[64][2];
static int dw_occ[64];

template <typename K>
static int tc_attr(K kernel, int smem_bytes, int threads, int* occ) {
  int st = cuda_status(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            smem_bytes));
  // all of the unified L1 as shared memory, so that several CTAs fit on an SM
  if (!st)
    st = cuda_status(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                          cudaSharedmemCarveoutMaxShared));
  // resident CTAs per SM from the kernel's own resources (shared memory, registers, threads);
  // the runtime's occupancy query answers 1 for this kernel although three fit.  CTAs never
  // wait on one another, so a grid larger than what is resident only queues.
  cudaFuncAttributes fa;
  int dev = 0;
  cudaDeviceProp pr;
  if (!st) st = cuda_status(cudaFuncGetAttributes(&fa, kernel));
  if (!st) st = cuda_status(cudaGetDevice(&dev));
  if (!st) st = cuda_status(cudaGetDeviceProperties(&pr, dev));
  if (st) return st;
  const size_t smem = smem_bytes + fa.sharedSizeBytes + pr.reservedSharedMemPerBlock;
  const int by_smem = (int)(pr.sharedMemPerMultiprocessor / smem);
  const int regs_warp = ((fa.numRegs * 32 + 255) / 256) * 256;
  const int by_regs = pr.regsPerMultiprocessor / (regs_warp * (threads / 32));
  const int by_threads = pr.maxThreadsPerMultiProcessor / threads;
  int o = by_smem < by_regs ? by_smem : by_regs;
  o = o < by_threads ? o : by_threads;
  *occ = o;
  return o < 1 ? LCT_ERR_UNSUPPORTED : LCT_OK;
}

static int conv_prepare(int dev) {
  if (dev < 0 || dev >= 64) return LCT_ERR_UNSUPPORTED;
  static std::mutex mu;  // host threads may create workspaces on one device together
  std::lock_guard<std::mutex> lock(mu);
  if (conv_attr_done[dev]) return LCT_OK;
  int st, o[4];
  if ((st = tc_attr(conv_tc_kernel<32, kEpiRelu>, ConvCfg<32>::Smem, kConvThreads, &o[0]))) return st;
  if ((st = tc_attr(conv_tc_kernel<32, kEpiMask>, ConvCfg<32>::Smem, kConvThreads, &o[1]))) return st;
  if ((st = tc_attr(conv_tc_kernel<16, kEpiResid>, ConvCfg<16>::Smem, kConvThreads, &o[2]))) return st;
  if ((st = tc_attr(conv_tc_kernel<16, kEpiGate>, ConvCfg<16>::Smem, kConvThreads, &o[3]))) return st;
  if ((st = tc_attr(cnn_dw_tc_kernel, DwCfg::Smem, kDwThreads, &dw_occ[dev]))) return st;
  conv_occ[dev][0] = o[0] < o[1] ? o[0] : o[1];
  conv_occ[dev][1] = o[2] < o[3] ? o[2] : o[3];
  conv_attr_done[dev] = true;
  return LCT_OK;
}

template <int N, int EPI>
static int launch_conv(const CUtensorMap& mx, const CUtensorMap& mw, ConvArgs a, int B, int dev,
                       int sms, cudaStream_t s) {
  a.n_tiles = (long long)B * a.tiles_x * a.tiles_y;
  if (a.n_tiles <= 0) return LCT_OK;
  const long long resident = (long long)sms * conv_occ[dev][N == 32 ? 0 : 1];
  const unsigned grid = (unsigned)(a.n_tiles < resident ? a.n_tiles : resident);
  conv_tc_kernel<N, EPI><<<grid, kConvThreads, ConvCfg<N>::Smem, s>>>(mx, mw, a);
  return launch_status();
}

static ConvArgs conv_args(const lct_cnn* c) {
  ConvArgs a = {};
  a.H = c->H;
  a.W = c->W;
  a.wp = c->wp;
  a.tiles_x = (c->W + kConvTW - 1) / kConvTW;
  a.tiles_y = (c->H + kConvTH - 1) / kConvTH;
  a.status = device_status_ptr();
  return a;
}

static int run_pack(lct_cnn* c, cudaStream_t s) {
  cnn_pack_kernel<<<(kCnnLayers * kWSlot + 255) / 256, 256, 0, s>>>(c->d_p, c->d_wf, c->d_wb);
  return launch_status();
}

static int run_prep(lct_cnn* c, const float* src, int vol_mode, int z0, int nz, int B,
                    cudaStream_t s) {
  const long long n = (long long)B * c->H * c->wp;
  const float k_in = c->calib * c->in_scale;
  cnn_prep_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, vol_mode, z0, nz, B, c->H,
                                                             c->W, c->wp, k_in, act_buf(c, 0));
  return launch_status();
}

// hidden layers 0..6 of the forward pass on B slices already in act_buf(0)
static int run_hidden(lct_cnn* c, int B, cudaStream_t s) {
  ConvArgs a = conv_args(c);
  int st;
  for (int l = 0; l < kCnnLayers - 1; ++l) {
    a.bias = c->d_p + cnn_off(l) + cnn_cin(l) * cnn_cout(l) * 9;
    a.out_act = act_buf(c, c->train ? l + 1 : ((l + 1) & 1));
    if ((st = launch_conv<32, kEpiRelu>(c->m_act[act_in(c, l)], c->m_wf[l], a, B, c->device,
                                        c->sms, s)))
      return st;
  }
  return LCT_OK;
}

static int last_bias_and_args(lct_cnn* c, ConvArgs& a) {
  a = conv_args(c);
  const int l = kCnnLayers - 1;
  a.bias = c->d_p + cnn_off(l) + cnn_cin(l) * cnn_cout(l) * 9;
  return LCT_OK;
}

static int cnn_forward_impl(lct_cnn* c, const float* d_in5, int B, cudaStream_t s) {
  int st;
  if ((st = run_prep(c, d_in5, 0, 0, 0, B, s))) return st;
  if ((st = run_hidden(c, B, s))) return st;
  ConvArgs a;
  last_bias_and_args(c, a);
  a.out_f = c->d_r;
  return launch_conv<16, kEpiResid>(c->m_act[act_in(c, kCnnLayers - 1)], c->m_wf[kCnnLayers - 1],
                                    a, B, c->device, c->sms, s);
}

static int cnn_backward_impl(lct_cnn* c, const float* d_in5, const float* d_target, int B,
                             cudaStream_t s) {
  int st;
  const long long n = (long long)B * c->H * c->W;
  if ((st = cuda_status(cudaMemsetAsync(c->d_g, 0, sizeof(float) * kCnnParams, s)))) return st;
  if ((st = cuda_status(cudaMemsetAsync(c->d_loss, 0, sizeof(double), s)))) return st;
  cnn_loss_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
      d_in5, c->d_r, d_target, B, c->H, c->W, c->wp, c->calib * c->in_scale, c->in_scale,
      (float)(2.0 / (double)n), dz_buf(c, 2), c->d_loss);
  if ((st = launch_status())) return st;
  c->last_n = n;
  ConvArgs a = conv_args(c);
  ConvArgs da = conv_args(c);
  da.n_tiles = (long long)B * da.tiles_x * da.tiles_y;
  const long long dw_res = (long long)c->sms * dw_occ[c->device];
  const unsigned dw_grid = (unsigned)(da.n_tiles < dw_res ? da.n_tiles : dw_res);
  const long long n_pix = (long long)B * c->H * c->wp;
  const unsigned db_grid = (unsigned)std::min<long long>((n_pix + 7) / 8, (long long)c->sms * 8);
  int cur = 2;
  for (int l = kCnnLayers - 1; l >= 0; --l) {
    float* gw = c->d_g + cnn_off(l);
    float* gb = gw + cnn_cin(l) * cnn_cout(l) * 9;
    cnn_dw_tc_kernel<<<dw_grid, kDwThreads, DwCfg::Smem, s>>>(c->m_dwa[l], c->m_dwz[cur], da,
                                                                cnn_cin(l), cnn_cout(l), gw);
    if ((st = launch_status())) return st;
    cnn_db_kernel<<<db_grid, 256, 0, s>>>(dz_buf(c, cur), n_pix, cnn_cout(l), gb);
    if ((st = launch_status())) return st;
    if (l == 0) break;
    const int nxt = cur == 2 ? 0 : (cur ^ 1);
    a.out_act = dz_buf(c, nxt);
    a.mask_act = act_buf(c, l);
    if ((st = launch_conv<32, kEpiMask>(c->m_dz[cur], c->m_wb[l], a, B, c->device, c->sms, s)))
      return st;
    cur = nxt;
  }
  return LCT_OK;
}

static int cnn_adam_impl(lct_cnn* c, float lr, float b1, float b2, float eps, cudaStream_t s) {
  ++c->adam_t;
  const float c1 = (float)(1.0 / (1.0 - std::pow((double)b1, c->adam_t)));
  const float c2 = (float)(1.0 / (1.0 - std::pow((double)b2, c->adam_t)));
  cnn_adam_kernel<<<(kCnnParams + 255) / 256, 256, 0, s>>>(c->d_p, c->d_g, c->d_m, c->d_v,
                                                          kCnnParams, lr, b1, b2, eps, c1, c2);
  int st = launch_status();
  return st ? st : run_pack(c, s);
}

// He-normal weights (std sqrt(2 / (9 cin)), the last layer x0.1 so training starts near the
// identity), zero biases; splitmix64 + Box-Muller, so a seed gives the same network everywhere.
static void init_params(std::vector<float>& p, uint64_t seed) {
  uint64_t st = seed ^ 0x6c6374636e6eULL;
  auto next = [&st]() {
    uint64_t z = (st += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  };
  auto unif = [&]() { return ((double)(next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); };
  p.assign(kCnnParams, 0.f);
  for (int l = 0; l < kCnnLayers; ++l) {
    const int nw = cnn_cin(l) * cnn_cout(l) * 9;
    const double sd = std::sqrt(2.0 / (9.0 * cnn_cin(l))) * (l == kCnnLayers - 1 ? 0.1 : 1.0);
    for (int i = 0; i < nw; ++i) {
      const double u1 = unif(), u2 = unif();
      p[cnn_off(l) + i] = (float)(sd * std::sqrt(-2.0 * std::log(u1)) *
                                  std::cos(2.0 * 3.141592653589793 * u2));
    }
  }
}

static void free_cnn(lct_cnn* c) {
  if (!c) return;
  cudaFree(c->d_p);
  cudaFree(c->d_wf);
  cudaFree(c->d_act);
  cudaFree(c->d_dz);
  cudaFree(c->d_r);
  cudaFree(c->d_loss);
  cudaFree(c->d_rej);
  delete c;
}

}  // namespace lct

LCT_API int lct_cnn_param_count(int64_t* n) {
  if (!n) return LCT_ERR_ARG;
  *n = kCnnParams;
  return LCT_OK;
}

LCT_API int lct_cnn_create(int max_slices, int ny, int nx, int flags, uint64_t seed,
                           lct_cnn** out) {
  if (!out || max_slices <= 0 || ny <= 0 || nx <= 0) return LCT_ERR_ARG;
  *out = nullptr;
  if ((flags & ~LCT_CNN_TRAIN) != 0) return LCT_ERR_ARG;
  const long long wp = (long long)nx + 2;
  if (wp > (1LL << 30) || ny > (1 << 30)) return LCT_ERR_ARG;
  lct_cnn* c = new (std::nothrow) lct_cnn;
  if (!c) return LCT_ERR_ALLOC;
  c->cap = max_slices;
  c->H = ny;
  c->W = nx;
  c->wp = (int)wp;
  c->train = (flags & LCT_CNN_TRAIN) != 0;
  c->n_act = c->train ? kCnnLayers : 2;
  c->act_elems = (long long)max_slices * ny * wp * kCnnC;
  int st = cuda_status(cudaGetDevice(&c->device));
  if (!st) st = cuda_status(cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device));
  if (!st) st = conv_prepare(c->device);
  if (!st) st = cuda_status(cudaMalloc(&c->d_p, sizeof(float) * 4 * kCnnParams));
  if (!st) {
    c->d_g = c->d_p + kCnnParams;
    c->d_m = c->d_g + kCnnParams;
    c->d_v = c->d_m + kCnnParams;
    st = cuda_status(cudaMemset(c->d_p, 0, sizeof(float) * 4 * kCnnParams));
  }
  if (!st) st = cuda_status(cudaMalloc(&c->d_wf, sizeof(__nv_bfloat16) * 2 * kCnnLayers * kWSlot));
  if (!st) c->d_wb = c->d_wf + kCnnLayers * kWSlot;
  const size_t act_bytes = sizeof(__nv_bfloat16) * (size_t)c->act_elems;
  if (!st) st = cuda_status(cudaMalloc(&c->d_act, act_bytes * c->n_act));
  if (!st) st = cuda_status(cudaMemset(c->d_act, 0, act_bytes * c->n_act));
  if (!st && c->train) {
    st = cuda_status(cudaMalloc(&c->d_dz, act_bytes * 3));
    if (!st) st = cuda_status(cudaMemset(c->d_dz, 0, act_bytes * 3));
    if (!st) st = cuda_status(cudaMalloc(&c->d_r, sizeof(float) * (size_t)max_slices * ny * nx));
  }
  if (!st) st = cuda_status(cudaMalloc(&c->d_loss, sizeof(double)));
  if (!st) st = cuda_status(cudaMalloc(&c->d_rej, sizeof(unsigned long long)));
  for (int i = 0; i < c->n_act && !st; ++i)
    st = act_map(&c->m_act[i], act_buf(c, i), c->cap, c->H, c->wp, kConvTH + 2);
  for (int i = 0; i < 3 && !st && c->train; ++i)
    st = act_map(&c->m_dz[i], dz_buf(c, i), c->cap, c->H, c->wp, kConvTH + 2);
  for (int i = 0; i < c->n_act && !st && c->train; ++i)  // weight gradients: 19-row boxes
    st = act_map(&c->m_dwa[i], act_buf(c, i), c->cap, c->H, c->wp, kDwRows);
  for (int i = 0; i < 3 && !st && c->train; ++i)
    st = act_map(&c->m_dwz[i], dz_buf(c, i), c->cap, c->H, c->wp, kConvTH);
  for (int l = 0; l < kCnnLayers && !st; ++l) {
    st = weight_map(&c->m_wf[l], c->d_wf + (size_t)l * kWSlot, l == kCnnLayers - 1 ? 16 : 32);
    if (!st) st = weight_map(&c->m_wb[l], c->d_wb + (size_t)l * kWSlot, 32);
  }
  if (!st) {
    std::vector<float> p;
    init_params(p, seed);
    st = cuda_status(cudaMemcpy(c->d_p, p.data(), sizeof(float) * kCnnParams, cudaMemcpyHostToDevice));
  }
  if (!st) st = run_pack(c, nullptr);
  if (!st) st = cuda_status(cudaDeviceSynchronize());
  if (st) {
    free_cnn(c);
    return st;
  }
  *out = c;
  return LCT_OK;
}

// Parameter, gradient, loss and counter copies wait for every stream first: the caller's training
// or inference may be queued on a non-blocking stream that the default stream does not order.
LCT_API int lct_cnn_set_params(lct_cnn* c, const float* params, int on_device) {
  if (!c || !params) return LCT_ERR_ARG;
  int st = cuda_status(cudaDeviceSynchronize());
  if (st) return st;
  st = cuda_status(cudaMemcpy(c->d_p, params, sizeof(float) * kCnnParams,
                                  on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice));
  if (!st) st = cuda_status(cudaMemset(c->d_m, 0, sizeof(float) * 2 * kCnnParams));
  c->adam_t = 0;
  if (!st) st = run_pack(c, nullptr);
  if (!st) st = cuda_status(cudaDeviceSynchronize());
  return st;
}

LCT_API int lct_cnn_get_params(const lct_cnn* c, float* params, int on_device) {
  if (!c || !params) return LCT_ERR_ARG;
  const int st = cuda_status(cudaDeviceSynchronize());
  if (st) return st;
  return cuda_status(cudaMemcpy(params, c->d_p, sizeof(float) * kCnnParams,
                                on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost));
}

LCT_API int lct_cnn_get_grads(const lct_cnn* c, float* grads, int on_device) {
  if (!c || !grads || !c->train) return LCT_ERR_ARG;
  const int st = cuda_status(cudaDeviceSynchronize());
  if (st) return st;
  return cuda_status(cudaMemcpy(grads, c->d_g, sizeof(float) * kCnnParams,
                                on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost));
}

LCT_API int lct_cnn_set_scales(lct_cnn* c, float calib, float in_scale) {
  if (!c || !(calib > 0.f) || !(in_scale > 0.f) || !std::isfinite(calib) || !std::isfinite(in_scale))
    return LCT_ERR_ARG;
  c->calib = calib;
  c->in_scale = in_scale;
  return LCT_OK;
}

LCT_API int lct_cnn_get_scales(const lct_cnn* c, float* calib, float* in_scale) {
  if (!c || !calib || !in_scale) return LCT_ERR_ARG;
  *calib = c->calib;
  *in_scale = c->in_scale;
  return LCT_OK;
}

LCT_API int lct_cnn_forward(lct_cnn* c, const float* d_in5, int n_slices, float* d_resid,
                            lct_stream stream) {
  if (!c || !d_in5 || n_slices <= 0 || n_slices > c->cap) return LCT_ERR_ARG;
  if (!c->train) return LCT_ERR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  int st = cnn_forward_impl(c, d_in5, n_slices, s);
  if (!st && d_resid)
    st = cuda_status(cudaMemcpyAsync(d_resid, c->d_r, sizeof(float) * (size_t)n_slices * c->H * c->W,
                                     cudaMemcpyDeviceToDevice, s));
  return st;
}

LCT_API int lct_cnn_backward(lct_cnn* c, const float* d_in5, const float* d_target, int n_slices,
                             lct_stream stream) {
  if (!c || !d_in5 || !d_target || n_slices <= 0 || n_slices > c->cap) return LCT_ERR_ARG;
  if (!c->train) return LCT_ERR_UNSUPPORTED;
  return cnn_backward_impl(c, d_in5, d_target, n_slices, (cudaStream_t)stream);
}

LCT_API int lct_cnn_adam_step(lct_cnn* c, float lr, float beta1, float beta2, float eps,
                              lct_stream stream) {
  if (!c || !c->train || !(lr >= 0.f) || !(beta1 >= 0.f && beta1 < 1.f) ||
      !(beta2 >= 0.f && beta2 < 1.f) || !(eps > 0.f))
    return LCT_ERR_ARG;
  return cnn_adam_impl(c, lr, beta1, beta2, eps, (cudaStream_t)stream);
}

LCT_API int lct_cnn_train_step(lct_cnn* c, const float* d_in5, const float* d_target,
                               int n_slices, float lr, lct_stream stream) {
  if (!c || !d_in5 || !d_target || n_slices <= 0 || n_slices > c->cap || !(lr >= 0.f))
    return LCT_ERR_ARG;
  if (!c->train) return LCT_ERR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  int st = cnn_forward_impl(c, d_in5, n_slices, s);
  if (!st) st = cnn_backward_impl(c, d_in5, d_target, n_slices, s);
  if (!st) st = cnn_adam_impl(c, lr, 0.9f, 0.999f, 1e-8f, s);
  return st;
}

LCT_API int lct_cnn_last_loss(const lct_cnn* c, double* loss) {
  if (!c || !loss || !c->train) return LCT_ERR_ARG;
  if (c->last_n <= 0) return LCT_ERR_ARG;  // no backward pass yet
  double sum = 0.0;
  int st = cuda_status(cudaDeviceSynchronize());
  if (!st) st = cuda_status(cudaMemcpy(&sum, c->d_loss, sizeof(double), cudaMemcpyDeviceToHost));
  if (!st) *loss = sum / (double)c->last_n;
  return st;
}

namespace lct {

// Gated inference of the slices [z0, z1) of a volume of nz slices (passes of at most max_slices;
// the 5-slice inputs read the neighbours, edge slices replicated).  Rejections add to the
// counter that cnn_reset_rejects clears.
int cnn_infer_range(lct_cnn* c, const float* d_vol, float* d_out, int nz, int z0, int z1,
                    float bound, cudaStream_t s) {
  if (!c || !d_vol || !d_out || nz <= 0 || d_vol == d_out || !(bound >= 0.f)) return LCT_ERR_ARG;
  if (z0 < 0 || z1 > nz || z0 > z1) return LCT_ERR_ARG;
  const long long plane = (long long)c->H * c->W;
  int st = LCT_OK;
  for (int zb = z0; zb < z1 && !st; zb += c->cap) {
    const int B = z1 - zb < c->cap ? z1 - zb : c->cap;
    if ((st = run_prep(c, d_vol, 1, zb, nz, B, s))) break;
    if ((st = run_hidden(c, B, s))) break;
    ConvArgs a;
    last_bias_and_args(c, a);
    a.out_f = d_out + (size_t)zb * plane;
    a.xc = d_vol + (size_t)zb * plane;
    a.calib = c->calib;
    a.inv_scale = 1.f / c->in_scale;
    a.bound = bound;
    a.n_reject = c->d_rej;
    st = launch_conv<16, kEpiGate>(c->m_act[act_in(c, kCnnLayers - 1)], c->m_wf[kCnnLayers - 1],
                                   a, B, c->device, c->sms, s);
  }
  return st;
}

int cnn_reset_rejects(lct_cnn* c, cudaStream_t s) {
  return cuda_status(cudaMemsetAsync(c->d_rej, 0, sizeof(unsigned long long), s));
}

int cnn_passes(const lct_cnn* c, int nslices) { return (nslices + c->cap - 1) / c->cap; }

}  // namespace lct

LCT_API int lct_cnn_infer_volume(lct_cnn* c, const float* d_vol, float* d_out, int nz,
                                 float bound, int64_t* n_rejected, lct_stream stream) {
  if (!c || !d_vol || !d_out || nz <= 0 || d_vol == d_out || !(bound >= 0.f)) return LCT_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  int st = cnn_reset_rejects(c, s);
  if (!st) st = cnn_infer_range(c, d_vol, d_out, nz, 0, nz, bound, s);
  if (!st && n_rejected) {
    unsigned long long v = 0;
    st = cuda_status(cudaMemcpyAsync(&v, c->d_rej, sizeof(v), cudaMemcpyDeviceToHost, s));
    if (!st) st = cuda_status(cudaStreamSynchronize(s));
    if (!st) *n_rejected = (int64_t)v;
  }
  return st;
}

LCT_API int lct_cnn_get_shape(const lct_cnn* c, int* max_slices, int* ny, int* nx) {
  if (!c || !max_slices || !ny || !nx) return LCT_ERR_ARG;
  *max_slices = c->cap;
  *ny = c->H;
  *nx = c->W;
  return LCT_OK;
}

LCT_API int lct_cnn_last_rejected(const lct_cnn* c, int64_t* n) {
  if (!c || !n) return LCT_ERR_ARG;
  unsigned long long v = 0;
  int st = cuda_status(cudaDeviceSynchronize());
  if (!st) st = cuda_status(cudaMemcpy(&v, c->d_rej, sizeof(v), cudaMemcpyDeviceToHost));
  if (!st) *n = (int64_t)v;
  return st;
}

LCT_API void lct_cnn_destroy(lct_cnn* c) { free_cnn(c); }
