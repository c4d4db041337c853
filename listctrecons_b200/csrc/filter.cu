// Stage 3: ramp-filter taps (host) and row convolution kernels.
//
// The reference convolves each detector row with 2*ns taps, out[is] = sum_{k<ns}
// h[is-k+ns] * row[k] (CUDA/Filter.cu:42-46), i.e. out = row * T with the Toeplitz matrix
// T[k][is] = h[is-k+ns].  LCT_FILTER_FP32 keeps that sum's order (FP32 FMA, k increasing) so
// results are bit-exact with the reference kernel; it tiles R rows per CTA so each tap read
// from shared memory feeds R FMAs.  LCT_FILTER_BF16X3 runs the same product as a GEMM on the
// tensor cores (filter_tc.cu).
#include <cmath>
#include <vector>

#include "lct_internal.h"

namespace lct {

// ---------------------------------------------------------------------------------------
// Taps.  With W(f) a frequency window, every kernel here is
//   h(n) = (1/ds) * 2 * integral_0^{1/2} f W(f) cos(2 pi n f) df,
// which for W = 1 is exactly the reference's Ram-Lak expression (Src/Filter.cpp:13-19) and
// for W = sinc(f) the Shepp-Logan kernel -2 / (pi^2 ds (4n^2 - 1)) (Shepp & Logan 1974;
// Kak & Slaney, "Principles of Computerized Tomographic Imaging", ch. 3), both with the
// reference's scaling (the discrete sum's ds factor folded into the taps).
// ---------------------------------------------------------------------------------------

// continuous-argument kernels (x in samples), FP64
static double ramlak_x(double x, double ds) {
  if (x == 0.0) return 0.25 / ds;
  const double px = kRefPi * x;
  return (std::sin(px) / px + (std::cos(px) - 1.0) / (px * px)) / (2.0 * ds);
}

static double shepp_logan_x(double x, double ds) {
  // (1/pi) [ (1 - cos(pi u1 / 2)) / (pi u1) + (1 - cos(pi u2 / 2)) / (pi u2) ], u = 1 +- 2x
  auto term = [](double u) {
    if (std::fabs(u) < 1e-12) return 0.0;
    return (1.0 - std::cos(kRefPi * u / 2.0)) / (kRefPi * u);
  };
  return (term(1.0 + 2.0 * x) + term(1.0 - 2.0 * x)) / kRefPi / ds;
}

static double base_kernel(int kind, double x, double ds) {
  return kind == LCT_FILTER_SHEPP_LOGAN ? shepp_logan_x(x, ds) : ramlak_x(x, ds);
}

static double windowed(int kind, int window, int n, double ds) {
  switch (window) {
    case LCT_WINDOW_HANN:  // 0.5 + 0.5 cos(2 pi f): a [1/4, 1/2, 1/4] smoothing of the taps
      return 0.5 * base_kernel(kind, n, ds) +
             0.25 * (base_kernel(kind, n - 1, ds) + base_kernel(kind, n + 1, ds));
    case LCT_WINDOW_HAMMING:  // 0.54 + 0.46 cos(2 pi f)
      return 0.54 * base_kernel(kind, n, ds) +
             0.23 * (base_kernel(kind, n - 1, ds) + base_kernel(kind, n + 1, ds));
    case LCT_WINDOW_COSINE:  // cos(pi f): mean of the kernel half a sample either side
      return 0.5 * (base_kernel(kind, n - 0.5, ds) + base_kernel(kind, n + 0.5, ds));
    default:
      return base_kernel(kind, n, ds);
  }
}

}  // namespace lct

using namespace lct;

LCT_API int lct_filter_taps(int kind, int window, int ns, float ds, float* h) {
  if (!h || ns <= 0 || !(ds > 0.f)) return LCT_ERR_ARG;
  if (kind != LCT_FILTER_RAMLAK && kind != LCT_FILTER_SHEPP_LOGAN) return LCT_ERR_ARG;
  if (window < LCT_WINDOW_NONE || window > LCT_WINDOW_COSINE) return LCT_ERR_ARG;
  for (int i = 0; i < 2 * ns; ++i) {
    int n = i - ns;
    if (kind == LCT_FILTER_RAMLAK && window == LCT_WINDOW_NONE) {
      // Src/Filter.cpp:13-19, the same expression (double, stored as float)
      if (n == 0)
        h[i] = 0.25 / ds;
      else
        h[i] = (std::sin(n * kRefPi) / (n * kRefPi) +
                (std::cos(n * kRefPi) - 1) / (n * n * kRefPi * kRefPi)) /
               (2 * ds);
    } else {
      h[i] = (float)windowed(kind, window, n, (double)ds);
    }
  }
  return LCT_OK;
}

namespace lct {

// ---------------------------------------------------------------------------------------
// FP32 convolution in the reference's order.  CTA = R rows x all ns outputs; thread `is`
// keeps R accumulators; taps and rows staged in shared memory (rows read as float4
// broadcasts).
// ---------------------------------------------------------------------------------------
constexpr int kFiltRows = 16;
constexpr int kFiltThreads = 256;

__host__ __device__ __forceinline__ int filt_rows_offset(int ns) { return (2 * ns + 8 + 3) / 4 * 4; }

__global__ void __launch_bounds__(kFiltThreads) filter_fp32_kernel(const float* __restrict__ h,
                                                                   float* __restrict__ rows,
                                                                   long long nrows, int ns,
                                                                   int nsp) {
  extern __shared__ __align__(16) float sm[];
  float* s_h = sm;  // 2*ns taps with 4 zero pads either side (indices down to -3)
  // rows start on a 16-byte boundary (float4 reads): offset rounded up to 4 floats
  float* s_r = sm + filt_rows_offset(ns);  // kFiltRows x nsp, zero padded to nsp (multiple of 4)
  const long long r0 = (long long)blockIdx.x * kFiltRows;
  for (int i = threadIdx.x; i < 2 * ns + 8; i += blockDim.x) {
    int k = i - 4;
    s_h[i] = (k >= 0 && k < 2 * ns) ? h[k] : 0.0f;
  }
  for (int r = 0; r < kFiltRows; ++r) {
    const bool ok = r0 + r < nrows;
    for (int k = threadIdx.x; k < nsp; k += blockDim.x)
      s_r[r * nsp + k] = (ok && k < ns) ? rows[(r0 + r) * ns + k] : 0.0f;
  }
  __syncthreads();
  const float* hs = s_h + 4;
  for (int is = threadIdx.x; is < ns; is += blockDim.x) {
    float acc[kFiltRows];
#pragma unroll
    for (int r = 0; r < kFiltRows; ++r) acc[r] = 0.0f;
    for (int k = 0; k < nsp; k += 4) {
      // padded columns k >= ns carry row value 0 and leave acc unchanged
      const float h0 = hs[is - k + ns], h1 = hs[is - k - 1 + ns];
      const float h2 = hs[is - k - 2 + ns], h3 = hs[is - k - 3 + ns];
#pragma unroll
      for (int r = 0; r < kFiltRows; ++r) {
        const float4 v = *reinterpret_cast<const float4*>(s_r + r * nsp + k);
        acc[r] = fmaf(h0, v.x, acc[r]);
        acc[r] = fmaf(h1, v.y, acc[r]);
        acc[r] = fmaf(h2, v.z, acc[r]);
        acc[r] = fmaf(h3, v.w, acc[r]);
      }
    }
#pragma unroll
    for (int r = 0; r < kFiltRows; ++r)
      if (r0 + r < nrows) rows[(r0 + r) * ns + is] = acc[r];
  }
}


int launch_filter_rows(int ns, const float* d_h, float* d_rows, long long nrows, int mode,
                       cudaStream_t s) {
  if (nrows <= 0) return LCT_OK;
  if (mode == LCT_FILTER_BF16X3 || mode == LCT_FILTER_BF16X6)
    return launch_filter_tc(ns, d_h, d_rows, nrows, mode, s);
  const int nsp = (ns + 3) / 4 * 4;
  const size_t smem = sizeof(float) * (filt_rows_offset(ns) + (size_t)kFiltRows * nsp);
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (smem > 48 * 1024 && dev < 64 && !attr_set[dev]) {
    int st = cuda_status(cudaFuncSetAttribute(filter_fp32_kernel,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              227 * 1024));
    if (st) return st;
    attr_set[dev] = true;
  }
  const long long nblk = (nrows + kFiltRows - 1) / kFiltRows;
  if (nblk > 0x7fffffffLL) return LCT_ERR_ARG;
  filter_fp32_kernel<<<(unsigned)nblk, kFiltThreads, smem, s>>>(d_h, d_rows, nrows, ns, nsp);
  return launch_status();
}

}  // namespace lct

LCT_API int lct_filter_rows(int ns, const float* d_h, float* d_rows, int64_t nrows, int mode,
                            lct_stream stream) {
  if (ns <= 0 || ns > 3072 || !d_h || !d_rows || nrows < 0) return LCT_ERR_ARG;
  if (mode != LCT_FILTER_FP32 && mode != LCT_FILTER_BF16X3 && mode != LCT_FILTER_BF16X6)
    return LCT_ERR_ARG;
  return launch_filter_rows(ns, d_h, d_rows, nrows, mode, (cudaStream_t)stream);
}
