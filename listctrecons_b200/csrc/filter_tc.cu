// Stage 3 on the tensor cores: the row convolution as a Toeplitz GEMM, BF16x3 on tcgen05.
//
// out[r][n] = sum_k rows[r][k] * h[n - k + ns]  (CUDA/Filter.cu:42-46) is out = R * T with
// T[k][n] = h[n - k + ns].  Both operands are split into bf16 high and low parts
// (x = hi + lo + O(2^-18 x)), and the product is accumulated in FP32 as
//   R*T ~= Rhi*Thi + Rhi*Tlo + Rlo*Thi
// (the dropped Rlo*Tlo term and the split residue are ~2^-16 relative per product).
//
// GEMM D[M x N] = A[M x K] B[K x N] with A = rows (K-major, as stored) and B given K-major as
// B^T[n][k] = h[n - k + ns] (itself Toeplitz, materialised once per taps, zero padded to
// Npad = Kpad = ns rounded up to 256).  One CTA computes a 128 x 256 tile of D:
//   * 4 warps; warp 0 / lane 0 issues TMA loads (tiled, 128-byte swizzle, no multicast) of the
//     four 64-deep K slices (A hi/lo 128 x 64, B hi/lo 256 x 64) into a 2-stage ring;
//   * warp 1 / lane 0 issues tcgen05.mma.kind::f16 (M128 N256 K16, BF16 in, FP32 accumulate
//     in TMEM, 3 products per K16 step) and frees each stage with tcgen05.commit;
//   * all 4 warps drain the 128 x 256 FP32 accumulator from TMEM (tcgen05.ld 32x32b) and store
//     the columns n < ns.
// Every mbarrier wait is bounded; a wait that runs out raises the device status word, the CTA
// stops issuing work, waits (bounded) for the copies it started, frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <mutex>

#include "lct_internal.h"
#include "tc_ptx.cuh"

namespace lct {

constexpr int kTcM = 128, kTcK = 64, kTcStages = 2, kTcThreads = 128, kTcPad = 256;

// P = bf16 planes per operand: P = 2 -> 3 products (BF16x3), P = 3 -> 6 products (BF16x6).
// Both keep a 96 KB stage: 128 x 256 tiles for P = 2, 128 x 128 for P = 3.
template <int P>
struct TcCfg {
  static constexpr int N = P == 2 ? 256 : 128;
  static constexpr uint32_t TileA = kTcM * kTcK * 2;
  static constexpr uint32_t TileB = N * kTcK * 2;
  static constexpr uint32_t Stage = P * TileA + P * TileB;
  static constexpr uint32_t Smem = kTcStages * Stage + 128 + 1024;  // + barriers + alignment
  static constexpr uint32_t TmemCols = N;
  // kind::f16 instruction descriptor: FP32 D, BF16 A and B, both K-major, M x N
  static constexpr uint32_t Idesc = (1u << 4) | (1u << 7) | (1u << 10) |
                                    ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);
};

__host__ __device__ inline int tc_pad(int ns) { return (ns + kTcPad - 1) / kTcPad * kTcPad; }

// ---------------------------------------------------------------------------------------
// operand preparation
// ---------------------------------------------------------------------------------------
// x = p[0] + p[1] (+ p[2]) + residue: each plane the bf16 rounding of what the previous left
template <int P>
__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16 (&p)[P]) {
#pragma unroll
  for (int i = 0; i < P; ++i) {
    p[i] = __float2bfloat16_rn(x);
    x -= __bfloat162float(p[i]);
  }
}

// rows fp32 [M][ns] -> P planes [M][kpad] (zero columns k >= ns); plane stride m * kpad
template <int P>
__global__ void __launch_bounds__(256) split_rows_kernel(const float* __restrict__ rows, long long m,
                                                         int ns, int kpad,
                                                         __nv_bfloat16* __restrict__ planes) {
  const long long r = blockIdx.x;
  if (r >= m) return;
  const long long pstride = m * kpad;
  for (int k = threadIdx.x; k < kpad; k += blockDim.x) {
    __nv_bfloat16 v[P];
    split_bf16<P>(k < ns ? rows[r * ns + k] : 0.0f, v);
#pragma unroll
    for (int i = 0; i < P; ++i) planes[i * pstride + r * kpad + k] = v[i];
  }
}

// The same split, 4 columns per thread and kSplitRows rows per block: 16-byte loads and 8-byte
// stores (4 bf16) per plane instead of scalar ones.  Needs ns and kpad multiples of 4 and a
// 16-byte aligned row base; every element is split exactly as above.
constexpr int kSplitRows = 4;

template <int P>
__global__ void __launch_bounds__(256) split_rows4_kernel(const float4* __restrict__ rows,
                                                          long long m, int ns4, int kpad4,
                                                          uint2* __restrict__ planes) {
  const long long r0 = (long long)blockIdx.x * kSplitRows;
  const long long pstride4 = m * kpad4;  // plane stride in groups of 4
  for (int j = 0; j < kSplitRows; ++j) {
    const long long r = r0 + j;
    if (r >= m) return;
    for (int k4 = threadIdx.x; k4 < kpad4; k4 += blockDim.x) {
      const float4 x = k4 < ns4 ? __ldg(rows + r * ns4 + k4) : make_float4(0.f, 0.f, 0.f, 0.f);
      __nv_bfloat16 v0[P], v1[P], v2[P], v3[P];
      split_bf16<P>(x.x, v0);
      split_bf16<P>(x.y, v1);
      split_bf16<P>(x.z, v2);
      split_bf16<P>(x.w, v3);
#pragma unroll
      for (int i = 0; i < P; ++i) {
        uint2 q;
        q.x = (unsigned)__bfloat16_as_ushort(v0[i]) | ((unsigned)__bfloat16_as_ushort(v1[i]) << 16);
        q.y = (unsigned)__bfloat16_as_ushort(v2[i]) | ((unsigned)__bfloat16_as_ushort(v3[i]) << 16);
        planes[i * pstride4 + r * kpad4 + k4] = q;
      }
    }
  }
}

// B^T[n][k] = h[n - k + ns] for n, k < ns, else 0; P planes [kpad][kpad]
template <int P>
__global__ void __launch_bounds__(256) toeplitz_kernel(const float* __restrict__ h, int ns, int kpad,
                                                       __nv_bfloat16* __restrict__ planes) {
  const int n = blockIdx.x;
  const long long pstride = (long long)kpad * kpad;
  for (int k = threadIdx.x; k < kpad; k += blockDim.x) {
    __nv_bfloat16 v[P];
    split_bf16<P>((n < ns && k < ns) ? h[n - k + ns] : 0.0f, v);
#pragma unroll
    for (int i = 0; i < P; ++i) planes[i * pstride + (long long)n * kpad + k] = v[i];
  }
}

// ---------------------------------------------------------------------------------------
// the GEMM: grid (kpad / N, ceil(M / 128)), 128 threads, TcCfg<P>::Smem dynamic shared memory.
// Products per K16 step: P = 2: (0,0) (0,1) (1,0);  P = 3: those and (0,2) (1,1) (2,0).
// ---------------------------------------------------------------------------------------
template <int P>
struct TcMaps {
  CUtensorMap a[P];
  CUtensorMap b[P];
};

template <int P>
__global__ void __launch_bounds__(kTcThreads, 1)
    filter_tc_kernel(const __grid_constant__ TcMaps<P> maps, float* __restrict__ out, long long m,
                     int ns, int ktiles, int* status) {
  using Cfg = TcCfg<P>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kTcStages * Cfg::Stage);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kTcStages + 1);
  __shared__ int s_abort;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n0 = blockIdx.x * Cfg::N;
  const long long m0 = (long long)blockIdx.y * kTcM;
  const uint32_t full0 = smem_u32(&bars[0]);
  const uint32_t empty0 = smem_u32(&bars[kTcStages]);
  const uint32_t accum = smem_u32(&bars[2 * kTcStages]);

  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int s = 0; s < kTcStages; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    mbar_init(accum, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
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

  if (warp == 0 && lane == 0) {
    // producer: TMA ring, stage = P A-planes then P B-planes
    int issued = 0;
    for (int kt = 0; kt < ktiles; ++kt) {
      const int s = kt % kTcStages;
      if (kt >= kTcStages && !mbar_wait(empty0 + 8 * s, ((kt / kTcStages) - 1) & 1)) {
        atomicExch(&s_abort, 1);
        break;
      }
      if (atomicAdd(&s_abort, 0)) break;
      uint8_t* st = smem + s * Cfg::Stage;
      const uint32_t fb = full0 + 8 * s;
      mbar_expect_tx(fb, Cfg::Stage);
      const int k0 = kt * kTcK;
#pragma unroll
      for (int i = 0; i < P; ++i) tma_load_2d(smem_u32(st + i * Cfg::TileA), &maps.a[i], k0, (int)m0, fb);
#pragma unroll
      for (int i = 0; i < P; ++i)
        tma_load_2d(smem_u32(st + P * Cfg::TileA + i * Cfg::TileB), &maps.b[i], k0, n0, fb);
      issued = kt + 1;
    }
    // copies still in flight land on their full barriers before the CTA may exit
    for (int kt = (issued > kTcStages ? issued - kTcStages : 0); kt < issued; ++kt)
      if (atomicAdd(&s_abort, 0)) mbar_wait(full0 + 8 * (kt % kTcStages), (kt / kTcStages) & 1);
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    for (int kt = 0; kt < ktiles; ++kt) {
      const int s = kt % kTcStages;
      if (!mbar_wait(full0 + 8 * s, (kt / kTcStages) & 1)) {
        atomicExch(&s_abort, 1);
        break;
      }
      tc_fence_after();
      uint8_t* st = smem + s * Cfg::Stage;
      uint64_t a[P], b[P];
#pragma unroll
      for (int i = 0; i < P; ++i) {
        a[i] = desc_sw128(smem_u32(st + i * Cfg::TileA));
        b[i] = desc_sw128(smem_u32(st + P * Cfg::TileA + i * Cfg::TileB));
      }
#pragma unroll
      for (int j = 0; j < kTcK / 16; ++j) {
        const uint64_t dk = (uint64_t)((j * 32) >> 4);  // 16 bf16 = 32 bytes along K
        umma_bf16(tmem, a[0] + dk, b[0] + dk, Cfg::Idesc, (kt | j) ? 1u : 0u);
        umma_bf16(tmem, a[0] + dk, b[1] + dk, Cfg::Idesc, 1u);
        umma_bf16(tmem, a[1] + dk, b[0] + dk, Cfg::Idesc, 1u);
        if (P == 3) {
          umma_bf16(tmem, a[0] + dk, b[P - 1] + dk, Cfg::Idesc, 1u);
          umma_bf16(tmem, a[1] + dk, b[1] + dk, Cfg::Idesc, 1u);
          umma_bf16(tmem, a[P - 1] + dk, b[0] + dk, Cfg::Idesc, 1u);
        }
      }
      umma_commit(empty0 + 8 * s);
    }
    umma_commit(accum);
  }
  __syncwarp();

  // epilogue: warp w owns TMEM lanes (rows) 32w .. 32w + 31
  const bool done = mbar_wait(accum, 0);
  tc_fence_after();
  if (!done || atomicAdd(&s_abort, 0)) {
    if (threadIdx.x == 0 && status) atomicExch(status, kDevWaitTimeout);
  } else {
    const long long row = m0 + warp * 32 + lane;
    float* orow = out + row * ns;
    // 16-byte stores only where every row start is 16-byte aligned
    const bool vec = ((ns & 3) == 0) && ((reinterpret_cast<uintptr_t>(out) & 15) == 0);
#pragma unroll 1
    for (int c = 0; c < Cfg::N / 32; ++c) {
      uint32_t r[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * 32), r);
      const int col0 = n0 + c * 32;
      if (row < m) {
        if (vec && col0 + 32 <= ns) {
#pragma unroll
          for (int i = 0; i < 32; i += 4)
            *reinterpret_cast<float4*>(orow + col0 + i) =
                make_float4(__uint_as_float(r[i]), __uint_as_float(r[i + 1]),
                            __uint_as_float(r[i + 2]), __uint_as_float(r[i + 3]));
        } else {
#pragma unroll
          for (int i = 0; i < 32; ++i)
            if (col0 + i < ns) orow[col0 + i] = __uint_as_float(r[i]);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(Cfg::TmemCols)
                 : "memory");
}

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// 2-D bf16 tensor [rows][cols] (cols contiguous), box {64, box_rows}, 128-byte swizzle
static int make_map(CUtensorMap* map, const void* base, long long rows, int cols, int box_rows) {
  auto fn = tensor_map_encoder();
  if (!fn) return LCT_ERR_UNSUPPORTED;
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
  cuuint32_t box[2] = {(cuuint32_t)kTcK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? LCT_OK : LCT_ERR_ARG;
}

static int planes_of(int mode) { return mode == LCT_FILTER_BF16X6 ? 3 : 2; }

// scratch: P Toeplitz planes [kpad][kpad], then P row planes [rows_cap][kpad]
size_t tc_scratch_bytes(int ns, long long rows_cap, int mode) {
  const long long kp = tc_pad(ns);
  const int P = planes_of(mode);
  return sizeof(__nv_bfloat16) * (size_t)P * ((size_t)rows_cap * kp + (size_t)kp * kp);
}

int tc_build_toeplitz(int ns, const float* d_h, void* scratch, int mode, cudaStream_t s) {
  const int kp = tc_pad(ns);
  __nv_bfloat16* b = static_cast<__nv_bfloat16*>(scratch);
  if (planes_of(mode) == 3)
    toeplitz_kernel<3><<<kp, 256, 0, s>>>(d_h, ns, kp, b);
  else
    toeplitz_kernel<2><<<kp, 256, 0, s>>>(d_h, ns, kp, b);
  return launch_status();
}

static bool tc_attr_done[2][64];

template <int P>
static int tc_filter_p(int ns, float* d_rows, long long nrows, void* scratch, cudaStream_t s) {
  using Cfg = TcCfg<P>;
  const int kp = tc_pad(ns);
  const long long mt = (nrows + kTcM - 1) / kTcM;
  if (mt > 65535) return LCT_ERR_ARG;
  __nv_bfloat16* b = static_cast<__nv_bfloat16*>(scratch);
  __nv_bfloat16* a = b + (size_t)P * kp * kp;
  if (ns % 4 == 0 && kp % 4 == 0 && reinterpret_cast<uintptr_t>(d_rows) % 16 == 0 &&
      reinterpret_cast<uintptr_t>(a) % 8 == 0)
    split_rows4_kernel<P><<<(unsigned)((nrows + kSplitRows - 1) / kSplitRows), 256, 0, s>>>(
        reinterpret_cast<const float4*>(d_rows), nrows, ns / 4, kp / 4, reinterpret_cast<uint2*>(a));
  else
    split_rows_kernel<P><<<(unsigned)nrows, 256, 0, s>>>(d_rows, nrows, ns, kp, a);
  int st = launch_status();
  if (st) return st;
  TcMaps<P> maps;
  for (int i = 0; i < P; ++i) {
    if ((st = make_map(&maps.a[i], a + (size_t)i * nrows * kp, nrows, kp, kTcM))) return st;
    if ((st = make_map(&maps.b[i], b + (size_t)i * kp * kp, kp, kp, Cfg::N))) return st;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  {
    static std::mutex mu;  // host threads may share a device
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 64 || !tc_attr_done[P - 2][dev]) {
      if ((st = cuda_status(cudaFuncSetAttribute(filter_tc_kernel<P>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 Cfg::Smem))))
        return st;
      if (dev < 64) tc_attr_done[P - 2][dev] = true;
    }
  }
  dim3 grid(kp / Cfg::N, (unsigned)mt);
  filter_tc_kernel<P><<<grid, kTcThreads, Cfg::Smem, s>>>(maps, d_rows, nrows, ns, kp / kTcK,
                                                          device_status_ptr());
  return launch_status();
}

// split + GEMM over nrows rows (nrows <= rows_cap the scratch was sized for), in place
int tc_filter(int ns, float* d_rows, long long nrows, void* scratch, long long rows_cap, int mode,
              cudaStream_t s) {
  if (nrows <= 0) return LCT_OK;
  if (nrows > rows_cap || nrows > 0x7fffffffLL) return LCT_ERR_ARG;
  return planes_of(mode) == 3 ? tc_filter_p<3>(ns, d_rows, nrows, scratch, s)
                              : tc_filter_p<2>(ns, d_rows, nrows, scratch, s);
}

// stage-level entry: stream-ordered scratch for this call
int launch_filter_tc(int ns, const float* d_h, float* d_rows, long long nrows, int mode,
                     cudaStream_t s) {
  if (nrows <= 0) return LCT_OK;
  void* scratch = nullptr;
  if (cuda_status(cudaMallocAsync(&scratch, tc_scratch_bytes(ns, nrows, mode), s)))
    return LCT_ERR_ALLOC;
  int st = tc_build_toeplitz(ns, d_h, scratch, mode, s);
  if (!st) st = tc_filter(ns, d_rows, nrows, scratch, nrows, mode, s);
  int st2 = cuda_status(cudaFreeAsync(scratch, s));
  return st ? st : st2;
}

}  // namespace lct
