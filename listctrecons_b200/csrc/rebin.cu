// Stage 1 (rebinning) and stage 2 (pre-weighting) kernels.
//
// Data layout: fan and parallel views are [view][row][col] float32, the reference's layout
// (CUDA/Rebiner.cu:45,90).  The fan-to-parallel rebin only interpolates along the view axis
// (columns and rows sit at texel centres in the reference's tex3D call, CUDA/Rebiner.cu:100),
// so each output is a two-tap lerp between fan views i0 and i0+1 of the same (row, col).
// Threads run along columns: every warp load and store is a contiguous row segment.
#include <cmath>

#include "lct_internal.h"
#include "tex_emul.cuh"

namespace lct {

struct RebinArgs {
  int ns, nt, n_angle, n_angle_add;
  float ws, wt, ds, dt, dso, orbit, pitch;
  int add;
};

static RebinArgs rebin_args(const lct_geom& g) {
  RebinArgs a;
  a.ns = g.ns; a.nt = g.nt; a.n_angle = g.n_angle; a.n_angle_add = g.n_angle_add;
  a.ws = g.ws; a.wt = g.wt; a.ds = g.ds; a.dt = g.dt; a.dso = g.dso; a.orbit = g.orbit;
  a.pitch = g.pitch; a.add = g.add_projections;
  return a;
}

// Fan view index and weight of rebinned (ia, is).
//   TEX8:  CUDA/Rebiner.cu:92-100 in FP32, operation for operation (round-to-nearest
//          intrinsics so nothing is contracted), then the texture unit's floor/frac with an
//          8-bit weight.  Indices are bit-exact with the reference's.
//   EXACT: the same formula in FP64.
template <int INTERP>
__device__ __forceinline__ void fan2par_index(const RebinArgs& a, int ia, int is, int& i0,
                                              float& w) {
  if (INTERP == LCT_INTERP_TEX8) {
    float ss = __fmul_rn(__fsub_rn((float)is, a.ws), a.ds);
    float alpha = __fdiv_rn(ss, a.dso);
    float beta_idx = __fadd_rn((float)ia, __fdiv_rn(alpha, a.orbit));
    float cz = __fadd_rn(__fadd_rn(beta_idx, (float)a.add), 0.5f);
    lin_axis<LCT_INTERP_TEX8>(cz, i0, w);
  } else {
    double ss = ((double)is - (double)a.ws) * (double)a.ds;
    double bidx = (double)ia + (ss / (double)a.dso) / (double)a.orbit + (double)a.add;
    double f = floor(bidx);
    i0 = (int)f;
    w = (float)(bidx - f);
  }
}

// grid (n_angle, ceil(nt/RT)), block 256: thread -> column, loops over RT rows.
constexpr int kRebinRows = 8;

template <int INTERP, int ADDR>
__global__ void __launch_bounds__(256) rebin_fan2par_kernel(const float* __restrict__ fan,
                                                            float* __restrict__ par, RebinArgs a) {
  const int ia = blockIdx.x;
  const int it0 = blockIdx.y * kRebinRows;
  const int it1 = min(a.nt, it0 + kRebinRows);
  const long long plane = (long long)a.nt * a.ns;
  for (int is = threadIdx.x; is < a.ns; is += blockDim.x) {
    int i0;
    float w;
    fan2par_index<INTERP>(a, ia, is, i0, w);
    long long v0 = i0, v1 = (long long)i0 + 1;
    bool ok0 = true, ok1 = true;
    if (ADDR == LCT_ADDR_CLAMP) {
      v0 = v0 < 0 ? 0 : (v0 >= a.n_angle_add ? a.n_angle_add - 1 : v0);
      v1 = v1 < 0 ? 0 : (v1 >= a.n_angle_add ? a.n_angle_add - 1 : v1);
    } else {
      ok0 = v0 >= 0 && v0 < a.n_angle_add;
      ok1 = v1 >= 0 && v1 < a.n_angle_add;
    }
    const float* p0 = fan + v0 * plane + is;
    const float* p1 = fan + v1 * plane + is;
    float* o = par + (long long)ia * plane + is;
    for (int it = it0; it < it1; ++it) {
      long long r = (long long)it * a.ns;
      float t0 = ok0 ? __ldg(p0 + r) : 0.0f;
      float t1 = ok1 ? __ldg(p1 + r) : 0.0f;
      o[r] = fmaf(w, t1, (1.0f - w) * t0);
    }
  }
}

template <int INTERP>
__global__ void rebin_fan2par_index_kernel(int* __restrict__ idx, float* __restrict__ wout,
                                           RebinArgs a) {
  const int ia = blockIdx.x;
  for (int is = threadIdx.x; is < a.ns; is += blockDim.x) {
    int i0;
    float w;
    fan2par_index<INTERP>(a, ia, is, i0, w);
    idx[(long long)ia * a.ns + is] = i0;
    wout[(long long)ia * a.ns + is] = w;
  }
}

// Scan mode: global parallel view g reads fan coordinate g + s(is), s = alpha(is)/orbit in
// FP64 (the same shift for every view, so every view of the scan is rebinned identically).
// A thread makes kRebinViews consecutive views of its column: view g + k reads fan views
// v0 + k and v0 + k + 1, so kRebinViews outputs take kRebinViews + 1 loads (each view index
// clamped or zero-filled on its own, exactly as two independent taps would be).
// fan_ring > 0: the fan buffer is a ring of fan_ring views, fan view v (relative to fan_first)
// at slot v mod fan_ring (bounded-memory runs); 0: linear.
constexpr int kRebinViews = 4;

template <int INTERP, int ADDR>
__global__ void __launch_bounds__(256) rebin_fan2par_scan_kernel(
    const float* __restrict__ fan, long long fan_first, long long fan_count, long long fan_ring,
    float* __restrict__ par, long long g0, long long nviews, RebinArgs a) {
  const long long lv = (long long)blockIdx.x * kRebinViews;  // first local view of the block
  const int nk = (int)min((long long)kRebinViews, nviews - lv);
  const long long g = g0 + lv;
  const int it0 = blockIdx.y * kRebinRows;
  const int it1 = min(a.nt, it0 + kRebinRows);
  const long long plane = (long long)a.nt * a.ns;
  for (int is = threadIdx.x; is < a.ns; is += blockDim.x) {
    double s = (((double)is - (double)a.ws) * (double)a.ds / (double)a.dso) / (double)a.orbit;
    double fs = floor(s);
    float w = (float)(s - fs);
    if (INTERP == LCT_INTERP_TEX8) w = q8(w);
    const long long v0 = g + (long long)fs - fan_first;
    const float* p[kRebinViews + 1];
    bool ok[kRebinViews + 1];
#pragma unroll
    for (int k = 0; k <= kRebinViews; ++k) {
      long long v = v0 + k;
      ok[k] = true;
      if (ADDR == LCT_ADDR_CLAMP)
        v = v < 0 ? 0 : (v >= fan_count ? fan_count - 1 : v);
      else
        ok[k] = v >= 0 && v < fan_count;
      if (!ok[k]) v = 0;
      if (fan_ring > 0) v %= fan_ring;
      p[k] = fan + v * plane + is;
    }
    float* o = par + lv * plane + is;
    for (int it = it0; it < it1; ++it) {
      const long long r = (long long)it * a.ns;
      float t[kRebinViews + 1];
#pragma unroll
      for (int k = 0; k <= kRebinViews; ++k) t[k] = (ok[k] && k <= nk) ? __ldg(p[k] + r) : 0.0f;
#pragma unroll
      for (int k = 0; k < kRebinViews; ++k)
        if (k < nk) o[k * plane + r] = fmaf(w, t[k + 1], (1.0f - w) * t[k]);
    }
  }
}

// Scan mode, four consecutive columns per thread (ns a multiple of 4, so every row of four is
// one aligned float4): a thread makes kRebinViews views x 4 columns.  The four columns' view
// shifts floor(s) differ by at most one when 3 |ds / (dso orbit)| < 1 (the host checks), so fan
// views f0 .. f0 + kRebinViews + 1 (f0 = the group's smallest floor) hold every tap: six float4
// loads per row for sixteen outputs, each warp load one contiguous 512-byte row segment of one
// fan view.  Each output is fmaf(w, t1, (1 - w) t0) with the same w, t0, t1 as the one-column
// kernel above, so the results are bit-identical to it.
template <int INTERP, int ADDR>
__global__ void __launch_bounds__(256) rebin_fan2par_scan4_kernel(
    const float* __restrict__ fan, long long fan_first, long long fan_count, long long fan_ring,
    float* __restrict__ par, long long g0, long long nviews, RebinArgs a) {
  constexpr int kTaps = kRebinViews + 2;
  const long long lv = (long long)blockIdx.x * kRebinViews;
  const int nk = (int)min((long long)kRebinViews, nviews - lv);
  const long long g = g0 + lv;
  const int it0 = blockIdx.y * kRebinRows;
  const int it1 = min(a.nt, it0 + kRebinRows);
  const long long plane = (long long)a.nt * a.ns;
  const int groups = a.ns >> 2;
  for (int q = threadIdx.x; q < groups; q += blockDim.x) {
    const int is0 = q << 2;
    float w[4];
    long long fl[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const double sc = (((double)(is0 + c) - (double)a.ws) * (double)a.ds / (double)a.dso) / (double)a.orbit;
      const double fs = floor(sc);
      w[c] = (float)(sc - fs);
      if (INTERP == LCT_INTERP_TEX8) w[c] = q8(w[c]);
      fl[c] = (long long)fs;
    }
    const long long f0 = min(min(fl[0], fl[1]), min(fl[2], fl[3]));
    bool hi[4];  // the column's taps start one fan view after f0
#pragma unroll
    for (int c = 0; c < 4; ++c) hi[c] = fl[c] != f0;
    const long long v0 = g + f0 - fan_first;
    float* o = par + lv * plane + is0;
    // the common case: all kTaps fan views present, none clamped or zero-filled, and consecutive
    // in the buffer (no ring wrap among them) -- one base pointer and the plane stride address
    // every tap and no load is predicated (0.44 ms instead of 0.47 ms on config 2's scan)
    const long long slot0 = fan_ring > 0 ? (v0 >= 0 ? v0 % fan_ring : -1) : v0;
    if (nk == kRebinViews && v0 >= 0 && v0 + kTaps <= fan_count &&
        (fan_ring == 0 || slot0 + kTaps <= fan_ring)) {
      const float4* b = reinterpret_cast<const float4*>(fan + slot0 * plane + is0);
      const long long p4 = plane >> 2;  // ns is a multiple of 4
      for (int it = it0; it < it1; ++it) {
        const long long r4 = ((long long)it * a.ns) >> 2;
        float4 t[kTaps];
#pragma unroll
        for (int m = 0; m < kTaps; ++m) t[m] = __ldg(b + m * p4 + r4);
#pragma unroll
        for (int k = 0; k < kRebinViews; ++k) {
          const float4 lo = t[k], mid = t[k + 1], up = t[k + 2];
          float4 out;
          out.x = fmaf(w[0], hi[0] ? up.x : mid.x, (1.0f - w[0]) * (hi[0] ? mid.x : lo.x));
          out.y = fmaf(w[1], hi[1] ? up.y : mid.y, (1.0f - w[1]) * (hi[1] ? mid.y : lo.y));
          out.z = fmaf(w[2], hi[2] ? up.z : mid.z, (1.0f - w[2]) * (hi[2] ? mid.z : lo.z));
          out.w = fmaf(w[3], hi[3] ? up.w : mid.w, (1.0f - w[3]) * (hi[3] ? mid.w : lo.w));
          *reinterpret_cast<float4*>(o + k * plane + (long long)it * a.ns) = out;
        }
      }
      continue;
    }
    const float4* p[kTaps];
    bool ok[kTaps];
#pragma unroll
    for (int m = 0; m < kTaps; ++m) {
      long long v = v0 + m;
      ok[m] = m <= nk + 1;
      if (ADDR == LCT_ADDR_CLAMP)
        v = v < 0 ? 0 : (v >= fan_count ? fan_count - 1 : v);
      else
        ok[m] = ok[m] && v >= 0 && v < fan_count;
      if (!ok[m]) v = 0;
      if (fan_ring > 0) v %= fan_ring;
      p[m] = reinterpret_cast<const float4*>(fan + v * plane + is0);
    }
    for (int it = it0; it < it1; ++it) {
      const long long r4 = ((long long)it * a.ns) >> 2;  // float4 offset of the row segment
      float4 t[kTaps];
#pragma unroll
      for (int m = 0; m < kTaps; ++m) t[m] = ok[m] ? __ldg(p[m] + r4) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int k = 0; k < kRebinViews; ++k) {
        if (k < nk) {
          const float4 lo = t[k], mid = t[k + 1], up = t[k + 2];
          float4 out;
          out.x = fmaf(w[0], hi[0] ? up.x : mid.x, (1.0f - w[0]) * (hi[0] ? mid.x : lo.x));
          out.y = fmaf(w[1], hi[1] ? up.y : mid.y, (1.0f - w[1]) * (hi[1] ? mid.y : lo.y));
          out.z = fmaf(w[2], hi[2] ? up.z : mid.z, (1.0f - w[2]) * (hi[2] ? mid.z : lo.z));
          out.w = fmaf(w[3], hi[3] ? up.w : mid.w, (1.0f - w[3]) * (hi[3] ? mid.w : lo.w));
          *reinterpret_cast<float4*>(o + k * plane + (long long)it * a.ns) = out;
        }
      }
    }
  }
}

// CUDA/Rebiner.cu:13-29: an offset copy (texel-centre fetch of fan view ia + add).
template <int ADDR>
__global__ void __launch_bounds__(256) rebin_null_kernel(const float* __restrict__ fan,
                                                         float* __restrict__ par, RebinArgs a) {
  const int ia = blockIdx.x;
  const long long plane = (long long)a.nt * a.ns;
  long long v = (long long)ia + a.add;
  bool ok = true;
  if (ADDR == LCT_ADDR_CLAMP)
    v = v < 0 ? 0 : (v >= a.n_angle_add ? a.n_angle_add - 1 : v);
  else
    ok = v >= 0 && v < a.n_angle_add;
  for (long long e = threadIdx.x; e < plane; e += blockDim.x)
    par[(long long)ia * plane + e] = ok ? __ldg(fan + v * plane + e) : 0.0f;
}

// Trilinear sample of a [nz][ny][nx] float volume at texture coordinates (x, y, z).
template <int INTERP, int ADDR, class T>
__device__ __forceinline__ float tex3d_lin(const float* __restrict__ v, int nx, int ny, int nz,
                                           T x, T y, T z) {
  int i, j, k;
  float a, b, c;
  lin_axis<INTERP>(x, i, a);
  lin_axis<INTERP>(y, j, b);
  lin_axis<INTERP>(z, k, c);
  // (x, y) corner weights: the texture unit's rule for TEX8 (exact products otherwise); the
  // slices are then combined with the z weight
  float wxy[2][2];
  if (INTERP == LCT_INTERP_TEX8) {
    tex_bilinear_weights(a, b, wxy[0][0], wxy[0][1], wxy[1][0], wxy[1][1]);
  } else {
    wxy[0][0] = (1.0f - a) * (1.0f - b);
    wxy[0][1] = a * (1.0f - b);
    wxy[1][0] = (1.0f - a) * b;
    wxy[1][1] = a * b;
  }
  float s = 0.0f;
#pragma unroll
  for (int dk = 0; dk < 2; ++dk)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj)
#pragma unroll
      for (int di = 0; di < 2; ++di) {
        int ii = i + di, jj = j + dj, kk = k + dk;
        float wgt = wxy[dj][di] * (dk ? c : 1.0f - c);
        if (ADDR == LCT_ADDR_CLAMP) {
          ii = min(max(ii, 0), nx - 1);
          jj = min(max(jj, 0), ny - 1);
          kk = min(max(kk, 0), nz - 1);
        } else if (ii < 0 || ii >= nx || jj < 0 || jj >= ny || kk < 0 || kk >= nz) {
          continue;
        }
        if (wgt != 0.0f) s = fmaf(wgt, __ldg(v + ((long long)kk * ny + jj) * nx + ii), s);
      }
  return s;
}

// CUDA/Rebiner.cu:156-179.  TEX8 keeps the reference's FP32 expression (its double
// sub-expression through PI included) with an accurate cosine; EXACT evaluates it in FP64.
template <int INTERP, int ADDR>
__global__ void __launch_bounds__(256) rebin_pi_ori_kernel(const float* __restrict__ fan,
                                                           float* __restrict__ par, RebinArgs a) {
  const int ia = blockIdx.x, it = blockIdx.y;
  for (int is = threadIdx.x; is < a.ns; is += blockDim.x) {
    float* out = par + ((long long)ia * a.nt + it) * a.ns + is;
    if (INTERP == LCT_INTERP_TEX8) {
      float s = (is - a.ws) * a.ds;
      float gamma = asinf(s / a.dso);
      float pidx = gamma * a.dso / a.ds + a.ws;
      double num = (double)((it - a.wt) * a.pitch / (float)(2 * (a.nt - 1))) -
                   (double)(gamma * a.pitch) / (2 * kRefPi);
      float q = (float)(num / (double)cosf(gamma));
      float qidx = q / a.dt + a.wt;
      float bidx = ia + gamma / a.orbit + (float)a.add;
      *out = tex3d_lin<INTERP, ADDR>(fan, a.ns, a.nt, a.n_angle_add, pidx + 0.5f, qidx + 0.5f,
                                     bidx + 0.5f);
    } else {
      double s = ((double)is - a.ws) * (double)a.ds;
      double gamma = asin(s / a.dso);
      double pidx = gamma * a.dso / a.ds + a.ws;
      double q = (((double)it - a.wt) * a.pitch / (2.0 * (a.nt - 1)) - gamma * a.pitch / (2 * kRefPi)) /
                 cos(gamma);
      double qidx = q / a.dt + a.wt;
      double bidx = (double)ia + gamma / a.orbit + a.add;
      *out = tex3d_lin<INTERP, ADDR>(fan, a.ns, a.nt, a.n_angle_add, pidx + 0.5, qidx + 0.5,
                                     bidx + 0.5);
    }
  }
}

// CUDA/PreWeighting.cu:8-29, in place.  temp2 is evaluated in double as in the reference
// (PI is a double literal there).
__global__ void __launch_bounds__(256) weight_pi_ori_kernel(float* __restrict__ par, RebinArgs a) {
  const int ia = blockIdx.x, it = blockIdx.y;
  for (int is = threadIdx.x; is < a.ns; is += blockDim.x) {
    float s = (is - a.ws) * a.ds;
    float t = (it - a.wt) * a.pitch / (float)(2 * a.nt);
    float gamma = asinf(s / a.dso);
    float temp = a.dso * a.dso - s * s;
    float temp2 = (float)((double)t - (double)(gamma * a.pitch) / (2 * kRefPi));
    float weight = sqrtf(temp) / sqrtf(temp + temp2 * temp2);
    par[((long long)ia * a.nt + it) * a.ns + is] *= weight;
  }
}

int launch_rebin_fan2par_scan(const lct_geom& g, const float* d_fan, long long fan_first,
                              long long fan_count, float* d_par, long long g0,
                              long long nviews, int interp, int addr, cudaStream_t s,
                              long long fan_ring, int width) {
  if (nviews <= 0) return LCT_OK;
  if (nviews > 0x7fffffffLL || fan_ring < 0) return LCT_ERR_ARG;
  RebinArgs a = rebin_args(g);
  dim3 grid((unsigned)((nviews + kRebinViews - 1) / kRebinViews), (g.nt + kRebinRows - 1) / kRebinRows);
  bool tex = interp == LCT_INTERP_TEX8, clamp = addr == LCT_ADDR_CLAMP;
  // four columns per thread when rows are float4-aligned and a group's shifts span at most one
  // view (3 |ds / (dso orbit)| < 1); `width` 1 forces the one-column kernel
  const double rate = std::fabs((double)g.ds / (double)g.dso / (double)g.orbit);
  const bool aligned = g.ns % 4 == 0 && reinterpret_cast<uintptr_t>(d_fan) % 16 == 0 &&
                       reinterpret_cast<uintptr_t>(d_par) % 16 == 0;
  if (width != 1 && aligned && 3.0 * rate < 1.0) {
    const int threads = std::min(256, std::max(32, ((g.ns / 4 + 31) / 32) * 32));
    if (tex && clamp)
      rebin_fan2par_scan4_kernel<LCT_INTERP_TEX8, LCT_ADDR_CLAMP><<<grid, threads, 0, s>>>(d_fan, fan_first, fan_count, fan_ring, d_par, g0, nviews, a);
    else if (tex)
      rebin_fan2par_scan4_kernel<LCT_INTERP_TEX8, LCT_ADDR_BORDER><<<grid, threads, 0, s>>>(d_fan, fan_first, fan_count, fan_ring, d_par, g0, nviews, a);
    else if (clamp)
      rebin_fan2par_scan4_kernel<LCT_INTERP_EXACT, LCT_ADDR_CLAMP><<<grid, threads, 0, s>>>(d_fan, fan_first, fan_count, fan_ring, d_par, g0, nviews, a);
    else
      rebin_fan2par_scan4_kernel<LCT_INTERP_EXACT, LCT_ADDR_BORDER><<<grid, threads, 0, s>>>(d_fan, fan_first, fan_count, fan_ring, d_par, g0, nviews, a);
    return launch_status();
  }
  if (width == 4) return LCT_ERR_UNSUPPORTED;
  if (tex && clamp)
    rebin_fan2par_scan_kernel<LCT_INTERP_TEX8, LCT_ADDR_CLAMP><<<grid, 256, 0, s>>>(d_fan, fan_first, fan_count, fan_ring, d_par, g0, nviews, a);
  else if (tex)
    rebin_fan2par_scan_kernel<LCT_INTERP_TEX8, LCT_ADDR_BORDER><<<grid, 256, 0, s>>>(d_fan, fan_first, fan_count, fan_ring, d_par, g0, nviews, a);
  else if (clamp)
    rebin_fan2par_scan_kernel<LCT_INTERP_EXACT, LCT_ADDR_CLAMP><<<grid, 256, 0, s>>>(d_fan, fan_first, fan_count, fan_ring, d_par, g0, nviews, a);
  else
    rebin_fan2par_scan_kernel<LCT_INTERP_EXACT, LCT_ADDR_BORDER><<<grid, 256, 0, s>>>(d_fan, fan_first, fan_count, fan_ring, d_par, g0, nviews, a);
  return launch_status();
}

}  // namespace lct

using namespace lct;

static int check_modes(int interp, int addr) {
  if (interp != LCT_INTERP_TEX8 && interp != LCT_INTERP_EXACT) return LCT_ERR_ARG;
  if (addr != LCT_ADDR_BORDER && addr != LCT_ADDR_CLAMP) return LCT_ERR_ARG;
  return LCT_OK;
}

LCT_API int lct_rebin_fan2par_scan(const lct_geom* g, const float* d_fan, int64_t fan_first,
                                   int64_t fan_count, float* d_par, int64_t g0, int64_t nviews,
                                   int interp, int addr, int width, lct_stream stream) {
  int st = check_geom(g);
  if (st) return st;
  if ((st = check_modes(interp, addr))) return st;
  if (!d_fan || !d_par || fan_count <= 0 || nviews < 0) return LCT_ERR_ARG;
  if (width != 0 && width != 1 && width != 4) return LCT_ERR_ARG;
  return launch_rebin_fan2par_scan(*g, d_fan, fan_first, fan_count, d_par, g0, nviews, interp,
                                   addr, (cudaStream_t)stream, 0, width);
}

LCT_API int lct_rebin_fan2par(const lct_geom* g, const float* d_fan, float* d_par, int interp,
                              int addr, lct_stream stream) {
  int st = check_geom(g);
  if (st) return st;
  if ((st = check_modes(interp, addr))) return st;
  if (!d_fan || !d_par) return LCT_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  RebinArgs a = rebin_args(*g);
  dim3 grid(g->n_angle, (g->nt + kRebinRows - 1) / kRebinRows);
  bool tex = interp == LCT_INTERP_TEX8, clamp = addr == LCT_ADDR_CLAMP;
  if (tex && clamp)
    rebin_fan2par_kernel<LCT_INTERP_TEX8, LCT_ADDR_CLAMP><<<grid, 256, 0, s>>>(d_fan, d_par, a);
  else if (tex)
    rebin_fan2par_kernel<LCT_INTERP_TEX8, LCT_ADDR_BORDER><<<grid, 256, 0, s>>>(d_fan, d_par, a);
  else if (clamp)
    rebin_fan2par_kernel<LCT_INTERP_EXACT, LCT_ADDR_CLAMP><<<grid, 256, 0, s>>>(d_fan, d_par, a);
  else
    rebin_fan2par_kernel<LCT_INTERP_EXACT, LCT_ADDR_BORDER><<<grid, 256, 0, s>>>(d_fan, d_par, a);
  return launch_status();
}

LCT_API int lct_rebin_fan2par_index(const lct_geom* g, int interp, int32_t* d_idx, float* d_w,
                                    lct_stream stream) {
  int st = check_geom(g);
  if (st) return st;
  if ((st = check_modes(interp, LCT_ADDR_BORDER))) return st;
  if (!d_idx || !d_w) return LCT_ERR_ARG;
  RebinArgs a = rebin_args(*g);
  cudaStream_t s = (cudaStream_t)stream;
  if (interp == LCT_INTERP_TEX8)
    rebin_fan2par_index_kernel<LCT_INTERP_TEX8><<<g->n_angle, 256, 0, s>>>(d_idx, d_w, a);
  else
    rebin_fan2par_index_kernel<LCT_INTERP_EXACT><<<g->n_angle, 256, 0, s>>>(d_idx, d_w, a);
  return launch_status();
}

LCT_API int lct_rebin_null(const lct_geom* g, const float* d_fan, float* d_par, int addr,
                           lct_stream stream) {
  int st = check_geom(g);
  if (st) return st;
  if ((st = check_modes(LCT_INTERP_TEX8, addr))) return st;
  if (!d_fan || !d_par) return LCT_ERR_ARG;
  RebinArgs a = rebin_args(*g);
  cudaStream_t s = (cudaStream_t)stream;
  if (addr == LCT_ADDR_CLAMP)
    rebin_null_kernel<LCT_ADDR_CLAMP><<<g->n_angle, 256, 0, s>>>(d_fan, d_par, a);
  else
    rebin_null_kernel<LCT_ADDR_BORDER><<<g->n_angle, 256, 0, s>>>(d_fan, d_par, a);
  return launch_status();
}

// TEX8 PI-original rebin through the texture unit, as the reference samples it
// (CUDA/Rebiner.cu:156-179): all three coordinates off texel centres, so the unit's trilinear
// filter -- which register emulation matches only to within two 8-bit weight steps -- is used
// itself.  Coordinates as in rebin_pi_ori_kernel's TEX8 branch.
__global__ void __launch_bounds__(256) rebin_pi_ori_tex_kernel(cudaTextureObject_t tex,
                                                               float* __restrict__ par, RebinArgs a) {
  const int ia = blockIdx.x, it = blockIdx.y;
  for (int is = threadIdx.x; is < a.ns; is += blockDim.x) {
    float s = (is - a.ws) * a.ds;
    float gamma = asinf(s / a.dso);
    float pidx = gamma * a.dso / a.ds + a.ws;
    double num = (double)((it - a.wt) * a.pitch / (float)(2 * (a.nt - 1))) -
                 (double)(gamma * a.pitch) / (2 * kRefPi);
    float q = (float)(num / (double)cosf(gamma));
    float qidx = q / a.dt + a.wt;
    float bidx = ia + gamma / a.orbit + (float)a.add;
    par[((long long)ia * a.nt + it) * a.ns + is] = tex3D<float>(tex, pidx + 0.5f, qidx + 0.5f, bidx + 0.5f);
  }
}

int lct::launch_rebin_pi_ori_tex(const lct_geom& g, const ViewTexture& t, int addr,
                                 const float* d_fan, float* d_par, cudaStream_t s) {
  const cudaTextureObject_t tex = view_texture_for(t, addr);
  if (!tex || t.ns != g.ns || t.nt != g.nt || t.depth < g.n_angle_add) return LCT_ERR_ARG;
  int st = view_texture_fill(t, d_fan, g.n_angle_add, 0, s);
  if (st) return st;
  rebin_pi_ori_tex_kernel<<<dim3(g.n_angle, g.nt), 256, 0, s>>>(tex, d_par, rebin_args(g));
  return launch_status();
}

LCT_API int lct_rebin_pi_ori(const lct_geom* g, const float* d_fan, float* d_par, int interp,
                             int addr, lct_stream stream) {
  int st = check_geom(g);
  if (st) return st;
  if ((st = check_modes(interp, addr))) return st;
  if (!d_fan || !d_par || g->nt < 2) return LCT_ERR_ARG;
  RebinArgs a = rebin_args(*g);
  dim3 grid(g->n_angle, g->nt);
  cudaStream_t s = (cudaStream_t)stream;
  bool tex = interp == LCT_INTERP_TEX8, clamp = addr == LCT_ADDR_CLAMP;
  if (tex) {
    // the fan block as a 3-D texture for the call (the reference binds it per block too,
    // CUDA/Rebiner.cu:181-230); released after the kernel, so this mode synchronises the stream
    ViewTexture t;
    if ((st = view_texture_create(t, g->ns, g->nt, g->n_angle_add, addr))) return st;
    st = launch_rebin_pi_ori_tex(*g, t, addr, d_fan, d_par, s);
    const int st2 = cuda_status(cudaStreamSynchronize(s));
    view_texture_destroy(t);
    return st ? st : st2;
  }
  if (clamp)
    rebin_pi_ori_kernel<LCT_INTERP_EXACT, LCT_ADDR_CLAMP><<<grid, 256, 0, s>>>(d_fan, d_par, a);
  else
    rebin_pi_ori_kernel<LCT_INTERP_EXACT, LCT_ADDR_BORDER><<<grid, 256, 0, s>>>(d_fan, d_par, a);
  return launch_status();
}

LCT_API int lct_weight_pi_ori(const lct_geom* g, float* d_par, lct_stream stream) {
  int st = check_geom(g);
  if (st) return st;
  if (!d_par) return LCT_ERR_ARG;
  RebinArgs a = rebin_args(*g);
  weight_pi_ori_kernel<<<dim3(g->n_angle, g->nt), 256, 0, (cudaStream_t)stream>>>(d_par, a);
  return launch_status();
}
