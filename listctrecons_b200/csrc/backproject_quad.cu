// Stage 4, fast path: backprojection from filtered views packed in quad layout.
//
// Same algorithm and window logic as bp_par_pairs_kernel (backproject.cu): one thread per
// (x, y) voxel column of NZ slices, z-invariant terms once per view, each conjugate pair
// {ia, ia + half} of a full window evaluated once and doubled (both samples outside the rows:
// each added once).  What changes is the per-sample cost:
//   * a bilinear sample is ONE 16-byte load of the 2 x 2 texel block at the clamped sample
//     origin (quad layout, lct_internal.h); border/clamp addressing lives in the packed data,
//     so there are no per-texel bounds tests;
//   * the row coordinate of slice j is one FMA, qhat = zc[j] * k + m (EXACT: h + j * k dz with
//     the slice index a constant), with k and m per view;
//   * the pair weights are branch-free selects around one reciprocal;
//   * views whose window covers every slice of the thread's chunk run an unpredicated loop.
// EXACT keeps FP64 view trigonometry and full FP32 weights; TEX8 keeps the reference's order
// for the sample column (phat/dso, theta*dso/ds) and the texture unit's 8-bit weight rules.
// EXACT also: floor, fraction and index of a sample from one round-down add (no conversions)
// and one wide multiply-add for its address; per-view terms staged in shared memory 128 views
// at a time; a warp-uniform path without out tests, selects or row clamps when a chunk's first
// and last slices project inside the detector rows, where the view and its conjugate run as
// packed FP32 pairs (FFMA2 / FADD2: half the instructions for the row, floor, fraction and first
// two bilinear FMAs of the two samples, each lane rounded as in the scalar form); an L1 prefetch
// of the next view's tile footprint; a polynomial asin on tiles within dso / 2 of the axis.
#include <climits>
#include <cmath>
#include <mutex>
#include <type_traits>

#include "lct_internal.h"
#include "tc_ptx.cuh"
#include "tex_emul.cuh"

namespace lct {

// tile 16 x 16 voxel columns (warps of 16 x 2): its footprint on the detector, |16 cos| + |16 sin|
// voxels wide, averages 20% narrower over the views than a 32 x 8 tile's; kQVB views staged per batch
constexpr int kQTX = 16, kQTY = 16, kQVB = 128;

// cos/sin of a view angle in FP64 rounded to float (sincospi: no large-argument reduction)
__device__ __forceinline__ void view_trig_pi(const float* __restrict__ betas, int v, float& c,
                                             float& s) {
  double sd, cd;
  sincospi((double)__ldg(betas + v) * 0.31830988618379067154, &sd, &cd);
  c = (float)cd;
  s = (float)sd;
}

// TEX8 (the reference's sampling) takes the reference's own __cosf / __sinf of the FP32 view
// angle (CUDA/Backprojector.cu:53, 61-62); EXACT the FP64 view_trig_pi
template <int INTERP>
__device__ __forceinline__ void view_trig_mode(const float* __restrict__ betas, int v, float& c,
                                               float& s) {
  if (INTERP == LCT_INTERP_TEX8) {
    const float b = __ldg(betas + v);
    c = __cosf(b);
    s = __sinf(b);
  } else {
    view_trig_pi(betas, v, c, s);
  }
}

struct BpQuadArgs {
  const float4* quads;  // slab s's local view ia is view slab_view[s] + ia of quads (mod qring)
  long long qring;      // > 0: quads is a ring of qring views; 0: linear
  const float* betas;
  float* img;
  long long qstride;    // float4 per view
  int qcols;            // ns + 3
  int ns, nt, n_angle, nx, ny, nz;
  float ws, wt, ds, dso, dso2, inv_dso, dso_over_ds, orbit, inv_orbit, z0, dzv, kq;
  float wx, wy, wz, dx, dy, dz;
  int half;
  int zchunks;
  int gx, gy, gz;  // tile grid (work-list decoding)
  int view_lo, view_hi, part;  // BpLaunch::view_lo / view_hi / part
  float kqdz;           // kq * dz (EXACT: row step per slice = kqdz / l)
  unsigned qrow_bytes;  // bytes per quad row, 16 * qcols
  int rows_inside_ok;   // 2 wt + 2.5 < nt + 3: |qhat| <= wt puts floor(qhat + wt + 2) in [1, nt + 2]
  int slab_view[kBpMaxSlabs];
  int slab_z0[kBpMaxSlabs];
  int a_min[kBpMaxZ], a_mid[kBpMaxZ], a_max[kBpMaxZ];
};

// quad pack: grid (views, nt + 3), block 256 over the ns + 3 quad columns; view v goes to slot
// (vbase + v) mod ring of a ring of quads (ring > 0), else to view v
template <int ADDR>
__global__ void __launch_bounds__(256) quad_pack_kernel(const float* __restrict__ rows, int ns,
                                                        int nt, float4* __restrict__ quads,
                                                        long long vbase, long long ring) {
  const long long v = blockIdx.x;
  const int j = (int)blockIdx.y - 2;
  const float* view = rows + v * (long long)nt * ns;
  const long long slot = ring > 0 ? (vbase + v) % ring : v;
  float4* out = quads + slot * quad_view_elems(ns, nt) + (long long)blockIdx.y * quad_cols(ns);
  auto texel = [&](int r, int c) -> float {
    if (ADDR == LCT_ADDR_CLAMP) {
      r = min(max(r, 0), nt - 1);
      c = min(max(c, 0), ns - 1);
    } else if (r < 0 || r >= nt || c < 0 || c >= ns) {
      return 0.0f;
    }
    return __ldg(view + (long long)r * ns + c);
  };
  for (int q = threadIdx.x; q < ns + 3; q += blockDim.x) {
    const int i = q - 2;
    const float t00 = texel(j, i), t01 = texel(j, i + 1), t10 = texel(j + 1, i),
                t11 = texel(j + 1, i + 1);
    // differences {T00, dy, dx, dxy}: a bilinear sample is then T00 + a dx + b (dy + a dxy), the
    // pair (T00, dy) + a (dx, dxy) one packed FMA
    out[q] = make_float4(t00, t10 - t00, t01 - t00, (t11 - t10) - (t01 - t00));
  }
}

int launch_quad_pack(const float* rows, long long views, int ns, int nt, int addr, float4* quads,
                     cudaStream_t s, long long vbase, long long ring) {
  if (views <= 0) return LCT_OK;
  if (views > 0x7fffffffLL || nt + 3 > 65535 || vbase < 0 || ring < 0) return LCT_ERR_ARG;
  if (ring > 0 && views > ring) return LCT_ERR_ARG;  // a piece would overwrite itself
  dim3 grid((unsigned)views, nt + 3);
  if (addr == LCT_ADDR_CLAMP)
    quad_pack_kernel<LCT_ADDR_CLAMP><<<grid, 256, 0, s>>>(rows, ns, nt, quads, vbase, ring);
  else
    quad_pack_kernel<LCT_ADDR_BORDER><<<grid, 256, 0, s>>>(rows, ns, nt, quads, vbase, ring);
  return launch_status();
}

// Base of local view ia of a slab whose local view 0 is view sv of the quads (ring-aware).
__device__ __forceinline__ const float4* quad_view_ptr(const BpQuadArgs& A, int sv, int ia) {
  long long v = (long long)sv + ia;
  if (A.qring > 0) v %= A.qring;
  return A.quads + v * A.qstride;
}

// Bilinear sample at origin column already applied to qb (qb = view base + clamped column);
// q_idx is the row coordinate in texel units (texel centres at integers).
template <int INTERP>
__device__ __forceinline__ float quad_sample(const float4* __restrict__ qb, int qcols, int nt,
                                             float a, float q_idx) {
  float yb;
  if (INTERP == LCT_INTERP_TEX8)
    yb = __fsub_rn(__fadd_rn(q_idx, 0.5f), 0.5f);  // the reference's texture coordinate
  else
    yb = q_idx;
  const float fy = floorf(yb);
  float b = yb - fy;
  int j = (int)fy;
  j = min(max(j, -2), nt);
  const float4 v = __ldg(qb + (j + 2) * qcols);  // T00, dy, dx, dxy
  if (INTERP == LCT_INTERP_TEX8) {
    // texture unit: w01 = a - w11, w10 = b - w11, w00 = 1 - a - b + w11, so the sample is
    // T00 + a dx + b dy + w11 dxy with w11 = round-half-up(a b) on the 1/256 grid
    b = q8(b);
    const float w11 = floorf(a * b * 256.0f + 0.5f) * (1.0f / 256.0f);
    return fmaf(w11, v.w, fmaf(b, v.y, fmaf(a, v.z, v.x)));
  }
  return fmaf(b, fmaf(a, v.w, v.y), fmaf(a, v.z, v.x));
}

// EXACT floor without conversions: for |x| < 2^22, x + 1.5 * 2^23 rounded toward -inf is
// 1.5 * 2^23 + floor(x) exactly, so its bit pattern is kMagicBits + floor(x) and subtracting the
// constant back (exact: both operands lie within a factor of two) gives floor(x).  Outside that
// range the bit pattern still orders like x, so a clamp on it clamps floor(x).
constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23
constexpr int kMagicBits = 0x4B400000;

// view base biased so that a column bit pattern (clamped to kMagicBits + [-2, ns]) times 16 and a
// row bit pattern (clamped to kMagicBits + [0, nt + 2]) times the row pitch add up to the quad's
// address: one wide multiply-add per sample
__device__ __forceinline__ unsigned long long quad_view_bias(const float4* view, unsigned qrow_bytes) {
  return reinterpret_cast<unsigned long long>(view) - (unsigned long long)(kMagicBits - 2) * 16ull -
         (unsigned long long)kMagicBits * qrow_bytes;
}

// EXACT sample: u = row coordinate + 2 (texel centres at integers), so floor(u) is the quad row;
// col = quad_view_bias(view) + 16 * (column bit pattern).  CLAMP false: the caller has shown
// that 1 <= u < nt + 3 (rows inside the detector), so the row needs no clamp.
template <bool CLAMP>
__device__ __forceinline__ float quad_sample_exact(unsigned long long col, unsigned qrow_bytes,
                                                   int nt, float a, float u) {
  const float t = __fadd_rd(u, kMagic);
  const float b = u - (t - kMagic);
  int rb = __float_as_int(t);
  if (CLAMP) rb = min(max(rb, kMagicBits), kMagicBits + nt + 2);
  const float4 v = __ldg(reinterpret_cast<const float4*>(
      col + (unsigned long long)(unsigned)rb * qrow_bytes));  // T00, dy, dx, dxy
  return fmaf(b, fmaf(a, v.w, v.y), fmaf(a, v.z, v.x));
}

// Blackwell's packed FP32 pairs (FFMA2, FADD2, FMUL2): one instruction for two lanes, each lane
// rounded exactly as the scalar operation; x - y is written fma(y, -1, x), one rounding like the
// subtraction.
__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 f2sub(float2 x, float2 y) {
  return __ffma2_rn(y, make_float2(-1.0f, -1.0f), x);
}

// EXACT column: weight a and 16 * (clamped column bit pattern) added to the biased view base
__device__ __forceinline__ unsigned long long quad_col_exact(unsigned long long vbias, float p,
                                                             int ns, float& a) {
  const float t = __fadd_rd(p, kMagic);
  a = p - (t - kMagic);
  const int cb = min(max(__float_as_int(t), kMagicBits - 2), kMagicBits + ns);
  return vbias + (unsigned long long)(unsigned)cb * 16ull;
}

// Prefetch boxes of one tile in view ia (b1) and its conjugate (b2): {row_lo, row_hi, col_lo,
// col_hi} in quad rows/columns, from the tile's four corners at its first and last slice, widened
// by one row and column (the interior can bulge slightly past the corners) and clamped to the
// view's quads.  Only the L1 prefetch reads them.
__device__ __forceinline__ void prefetch_boxes(const BpQuadArgs& A, float c1, float s1, float c2,
                                               float s2, int ia, float x0, float x1, float y0,
                                               float y1, float zc0, float zcl, int4& b1, int4& b2) {
  b1 = make_int4(INT_MAX, INT_MIN, INT_MAX, INT_MIN);
  b2 = b1;
  const float zb1 = fmaf((float)ia, A.dzv, A.z0), zb2 = fmaf((float)(ia + A.half), A.dzv, A.z0);
  const float wt2 = A.wt + 2.0f;
#pragma unroll 1
  for (int c = 0; c < 4; ++c) {
    const float x = (c & 1) ? x1 : x0, y = (c >> 1) ? y1 : y0;
    const float phat = fmaf(-x, c1, -__fmul_rn(y, s1));
    const float theta = asinf(__fmul_rn(phat, A.inv_dso));
    const float tho = __fmul_rn(theta, A.inv_orbit);
    const float t = fmaf(-phat, phat, A.dso2);
    const float sq = __fmul_rn(t, rsqrtf(t));
    const float k1 = __fdividef(A.kq, fmaf(x, s1, fmaf(-y, c1, sq)));
    const float k2 = __fdividef(A.kq, fmaf(x, s2, fmaf(-y, c2, sq)));
    const float zr1 = fmaf(tho, A.dzv, zb1), zr2 = fmaf(-tho, A.dzv, zb2);
    for (int e = 0; e < 2; ++e) {
      const float zc = e ? zcl : zc0;
      const int r1 = __float2int_rd(fmaf(zc - zr1, k1, wt2));
      const int r2 = __float2int_rd(fmaf(zc - zr2, k2, wt2));
      b1.x = min(b1.x, r1); b1.y = max(b1.y, r1);
      b2.x = min(b2.x, r2); b2.y = max(b2.y, r2);
    }
    const int q1 = __float2int_rd(fmaf(theta, A.dso_over_ds, A.ws)) + 2;
    const int q2 = __float2int_rd(fmaf(-theta, A.dso_over_ds, A.ws)) + 2;
    b1.z = min(b1.z, q1); b1.w = max(b1.w, q1);
    b2.z = min(b2.z, q2); b2.w = max(b2.w, q2);
  }
  auto fit = [&](int4& b) {
    b.x = min(max(b.x - 1, 0), A.nt + 2);
    b.y = min(max(b.y + 1, b.x), A.nt + 2);
    b.z = min(max(b.z - 1, 0), A.ns + 2);
    b.w = min(max(b.w + 1, b.z), A.ns + 2);
  };
  fit(b1);
  fit(b2);
}

// asin on |x| <= 0.5 as x + x^3 P(x^2), P of degree 4 fitted by least squares (weighted for the
// relative error of asin) at 400 Chebyshev nodes of x^2 in [0, 0.25]; largest error 0.65 ulp
// against the FP64 arcsin over [-0.5, 0.5] in float32 Horner evaluation
__device__ __forceinline__ float asin_half(float x) {
  const float t = __fmul_rn(x, x);
  const float p = fmaf(fmaf(fmaf(fmaf(0.042095039039850235f, t, 0.024220509454607964f), t,
                                 0.04546250030398369f), t, 0.07495353370904922f), t,
                       0.16666752099990845f);
  return fmaf(__fmul_rn(x, t), p, x);
}

// Column of a sample: clamped origin offset and weight
template <int INTERP>
__device__ __forceinline__ void quad_col(float p_idx, int ns, int& off, float& a) {
  float xb;
  if (INTERP == LCT_INTERP_TEX8)
    xb = __fsub_rn(__fadd_rn(p_idx, 0.5f), 0.5f);
  else
    xb = p_idx;
  const float fx = floorf(xb);
  a = xb - fx;
  if (INTERP == LCT_INTERP_TEX8) a = q8(a);
  int i = (int)fx;
  off = min(max(i, -2), ns) + 2;
}

// One tile: voxel columns [bx*kQTX, +kQTX) x [by*kQTY, +kQTY), slab/slice chunk bz.  Called with
// CTA-uniform arguments by every thread of a 256-thread CTA.
template <int NZ, int INTERP, bool PART, bool RING>
__device__ __forceinline__ void bp_quad_tile(const BpQuadArgs& A, int bx, int by, int bz) {
  __shared__ float4 s_cs[kQVB];      // cos, sin of view ia and of its conjugate ia + half
  __shared__ int2 s_jr[kQVB];        // slices [jlo, jhi) of the chunk whose window holds ia
  __shared__ float2 s_zb[kQVB];      // EXACT: source z of both views without the fan-angle term
  __shared__ ulonglong2 s_qv[kQVB];  // bases of both views (EXACT: biased, quad_view_bias)
  __shared__ ulonglong2 s_pfb[kQVB]; // EXACT: prefetch box origins of both views
  __shared__ int4 s_pfs[kQVB];       // EXACT: prefetch box rows and column spans

  const int tid = threadIdx.y * kQTX + threadIdx.x;
  const int ix = bx * kQTX + threadIdx.x;
  const int iy = by * kQTY + threadIdx.y;
  const int slab = bz / A.zchunks;
  const int z0 = (bz % A.zchunks) * NZ;
  const int nzc = min(NZ, A.nz - z0);

  // explicit roundings (_rn, fmaf) wherever a product meets a sum: plain mul/add pairs may be
  // contracted differently in each instantiation, and the work-list kernel must reproduce a
  // scan's own launch bit for bit
  const float xc = __fmul_rn((float)ix - A.wx, A.dx);
  const float yc = __fmul_rn((float)iy - A.wy, A.dy);
  const float zc0 = __fmul_rn((float)z0 - A.wz, A.dz);
  const float wt2 = A.wt + 2.0f;
  // EXACT prefetch: the tile's corner coordinates and last slice
  const float xr0 = __fmul_rn((float)(bx * kQTX) - A.wx, A.dx);
  const float xr1 = __fmul_rn((float)(min(bx * kQTX + kQTX, A.nx) - 1) - A.wx, A.dx);
  const float yr0 = __fmul_rn((float)(by * kQTY) - A.wy, A.dy);
  const float yr1 = __fmul_rn((float)(min(by * kQTY + kQTY, A.ny) - 1) - A.wy, A.dy);
  const float zcl = __fmul_rn((float)(z0 + nzc - 1) - A.wz, A.dz);
  // |phat| <= the largest corner radius of the tile (the norm's maximum over a rectangle), so
  // when that is below dso / 2 every view of the tile takes the polynomial asin
  const float rx = fmaxf(fabsf(xr0), fabsf(xr1)), ry = fmaxf(fabsf(yr0), fabsf(yr1));
  const bool asin_poly = sqrtf(fmaf(rx, rx, ry * ry)) * A.inv_dso < 0.49f;
  float zc[NZ];
#pragma unroll
  for (int j = 0; j < NZ; ++j) zc[j] = ((float)(z0 + j) - A.wz) * A.dz;

  int vlo = INT_MAX, vhi = INT_MIN;
  for (int j = 0; j < nzc; ++j) {
    vlo = min(vlo, A.a_min[z0 + j]);
    vhi = max(vhi, A.a_mid[z0 + j]);
  }
  if (PART) {
    vlo = max(vlo, A.view_lo);
    vhi = min(vhi, A.view_hi);
  }
  const int sv = A.slab_view[slab];
  const float4* quads = A.quads + (long long)sv * A.qstride;  // linear buffers: slab's view 0
  const float* betas = A.betas + sv;
  const float wt = A.wt;

  float acc[NZ];
#pragma unroll
  for (int j = 0; j < NZ; ++j) acc[j] = 0.0f;
  if (PART && A.part >= kBpMiddle && ix < A.nx && iy < A.ny) {  // continue earlier parts' sums
    const float* in = A.img + ((long long)(A.slab_z0[slab] + z0) * A.ny + iy) * A.nx + ix;
#pragma unroll
    for (int j = 0; j < NZ; ++j)
      if (j < nzc) acc[j] = in[j * (long long)A.nx * A.ny];
  }

  for (int vb = vlo; vb < vhi; vb += kQVB) {
    __syncthreads();
    if (tid < kQVB && vb + tid < vhi) {
      const int ia = vb + tid;
      float c1, s1, c2, s2;
      view_trig_mode<INTERP>(betas, ia, c1, s1);
      view_trig_mode<INTERP>(betas, ia + A.half, c2, s2);
      s_cs[tid] = make_float4(c1, s1, c2, s2);
      const float4* v1 = RING ? quad_view_ptr(A, sv, ia) : quads + (long long)ia * A.qstride;
      const float4* v2 = RING ? quad_view_ptr(A, sv, ia + A.half)
                              : quads + (long long)(ia + A.half) * A.qstride;
      if (INTERP != LCT_INTERP_EXACT)
        s_qv[tid] = make_ulonglong2(reinterpret_cast<unsigned long long>(v1),
                                    reinterpret_cast<unsigned long long>(v2));
      if (INTERP == LCT_INTERP_EXACT) {
        s_zb[tid] = make_float2(fmaf((float)ia, A.dzv, A.z0), fmaf((float)(ia + A.half), A.dzv, A.z0));
        s_qv[tid] = make_ulonglong2(quad_view_bias(v1, A.qrow_bytes), quad_view_bias(v2, A.qrow_bytes));
        int4 b1, b2;
        prefetch_boxes(A, c1, s1, c2, s2, ia, xr0, xr1, yr0, yr1, zc0, zcl, b1, b2);
        s_pfb[tid] = make_ulonglong2(
            reinterpret_cast<unsigned long long>(v1) + (unsigned long long)b1.x * A.qrow_bytes + 16ull * b1.z,
            reinterpret_cast<unsigned long long>(v2) + (unsigned long long)b2.x * A.qrow_bytes + 16ull * b2.z);
        s_pfs[tid] = make_int4(b1.y - b1.x + 1, b1.w - b1.z, b2.y - b2.x + 1, b2.w - b2.z);
      }
      int jlo = nzc, jhi = 0;
      for (int j = 0; j < nzc; ++j)
        if (ia >= A.a_min[z0 + j] && ia < A.a_mid[z0 + j]) {
          jlo = min(jlo, j);
          jhi = max(jhi, j + 1);
        }
      s_jr[tid] = make_int2(jlo, jhi);
    }
    __syncthreads();
    const int nv = min(kQVB, vhi - vb);
    for (int k = 0; k < nv; ++k) {
      const int ia = vb + k;
      if (INTERP == LCT_INTERP_EXACT && k + 1 < nv) {
        // the next view's footprint into L1 while this one is sampled (a hint: no result depends
        // on it, and every address lies inside that view's quads)
        const int pf_conj = tid >> 7, pf_row = (tid >> 3) & 15, pf_line = tid & 7;
        const int4 sz = s_pfs[k + 1];
        const int rows = pf_conj ? sz.z : sz.x, cspan = pf_conj ? sz.w : sz.y;
        if (pf_row < rows && 8 * pf_line <= cspan + 7) {
          const ulonglong2 bs = s_pfb[k + 1];
          const unsigned long long a = (pf_conj ? bs.y : bs.x) +
                                       (unsigned long long)pf_row * A.qrow_bytes +
                                       16ull * (unsigned)min(8 * pf_line, cspan);
          asm volatile("prefetch.global.L1 [%0];" ::"l"(a));
        }
      }
      const int2 jr = s_jr[k];
      const int jlo = jr.x, jhi = jr.y;
      const float4 cs = s_cs[k];
      const float cb = cs.x, sb = cs.y, cb2 = cs.z, sb2 = cs.w;
      // CUDA/Backprojector.cu:53-64, z-invariant part
      const float phat = fmaf(-xc, cb, -__fmul_rn(yc, sb));
      float theta, delta_p, tho, sq;
      if (INTERP == LCT_INTERP_TEX8) {
        theta = asinf(__fdiv_rn(phat, A.dso));
        delta_p = __fdiv_rn(__fmul_rn(theta, A.dso), A.ds);
        tho = __fdiv_rn(theta, A.orbit);
        sq = sqrtf(fmaf(-phat, phat, A.dso2));
      } else {
        const float sx = __fmul_rn(phat, A.inv_dso);
        if (asin_poly)
          theta = asin_half(sx);
        else
          theta = asinf(sx);
        delta_p = 0.0f;  // EXACT: the columns are fmaf(+-theta, dso/ds, ws)
        tho = __fmul_rn(theta, A.inv_orbit);
        const float t = fmaf(-phat, phat, A.dso2);
        sq = __fmul_rn(t, rsqrtf(t));
      }
      const float l1 = fmaf(xc, sb, fmaf(-yc, cb, sq));
      const float l2 = fmaf(xc, sb2, fmaf(-yc, cb2, sq));
      if constexpr (INTERP == LCT_INTERP_EXACT) {
        // source z from the staged per-view term: zr = (ia + tho) dzv + z0
        const float2 zb = s_zb[k];
        const ulonglong2 qv = s_qv[k];
        const float zr1 = fmaf(tho, A.dzv, zb.x), zr2 = fmaf(-tho, A.dzv, zb.y);
        // slice j: qhat = h + j kd with k = kq / l, kd = k dz (one FMA with a constant j, no
        // per-slice z register); weights halved around one reciprocal -- the factor 2 is
        // restored, exactly, at the output
        const float r1 = __fdividef(1.0f, l1), r2 = __fdividef(1.0f, l2);
        const float kd1 = __fmul_rn(A.kqdz, r1), kd2 = __fmul_rn(A.kqdz, r2);
        const float h1 = __fmul_rn(__fsub_rn(zc0, zr1), __fmul_rn(A.kq, r1));
        const float h2 = __fmul_rn(__fsub_rn(zc0, zr2), __fmul_rn(A.kq, r2));
        const float u1 = __fadd_rn(h1, wt2), u2 = __fadd_rn(h2, wt2);
        float a1, a2;
        const unsigned long long q1 = quad_col_exact(qv.x, fmaf(theta, A.dso_over_ds, A.ws), A.ns, a1);
        const unsigned long long q2 = quad_col_exact(qv.y, fmaf(-theta, A.dso_over_ds, A.ws), A.ns, a2);
        // INSIDE: both samples of every slice lie within the detector rows (no tests, no selects)
        auto slice_x = [&](int j, auto inside) {
          const float fj = (float)j;
          const float qh1 = fmaf(fj, kd1, h1), qh2 = fmaf(fj, kd2, h2);
          // the pair weights sum to one in every case -- (-qh2, qh1) / (qh1 - qh2), (0, 1),
          // (1, 0), (1/2, 1/2) -- so w1 s1 + w2 s2 = s2 + w1 (s1 - s2)
          const float in1 = -qh2 * __fdividef(1.0f, qh1 - qh2);
          float w1 = in1;
          if constexpr (!decltype(inside)::value) {
            const bool out1 = fabsf(qh1) > wt, out2 = fabsf(qh2) > wt;
            w1 = out1 ? (out2 ? 0.5f : 0.0f) : (out2 ? 1.0f : in1);
          }
          constexpr bool kClamp = !decltype(inside)::value;
          const float s1 = quad_sample_exact<kClamp>(q1, A.qrow_bytes, A.nt, a1, fmaf(fj, kd1, u1));
          const float s2 = quad_sample_exact<kClamp>(q2, A.qrow_bytes, A.nt, a2, fmaf(fj, kd2, u2));
          acc[j] = fmaf(w1, s1 - s2, acc[j] + s2);
        };
        // qhat(j) = fmaf(j, kd, h) is monotone in j (monotone rounding of a linear function),
        // so the chunk's first and last slices bound every |qhat|: when both are inside for both
        // views in every lane of the warp, every out test of the chunk is false and the selects
        // are skipped with no change to any result.  The row coordinate u = qhat + wt + 2 (equal
        // to within a few ulps, far below half a row) then lies in (1.5, 2 wt + 2.5), inside the
        // quad rows when rows_inside_ok.  Plain comparisons: a NaN fails them.
        bool inside = false;
        if (jlo == 0 && jhi == NZ) {
          const float e1 = fmaf((float)(NZ - 1), kd1, h1), e2 = fmaf((float)(NZ - 1), kd2, h2);
          inside = A.rows_inside_ok && fabsf(h1) <= wt && fabsf(e1) <= wt &&
                   fabsf(h2) <= wt && fabsf(e2) <= wt;
        }
        if (__all_sync(0xffffffffu, inside)) {
          // the two views of the pair as one packed FP32 pair per slice: each lane is
          // slice_x(j, inside) rounded the same way
          const float2 KD = make_float2(kd1, kd2), H = make_float2(h1, h2), U = make_float2(u1, u2);
          const float2 A1 = f2(a1), A2 = f2(a2);
#pragma unroll
          for (int j = 0; j < NZ; ++j) {
            const float2 J = f2((float)j);
            const float2 qh = __ffma2_rn(J, KD, H);
            const float w1 = -qh.y * __fdividef(1.0f, qh.x - qh.y);
            const float2 u = __ffma2_rn(J, KD, U);
            const float2 t = __fadd2_rd(u, f2(kMagic));
            const float2 b = f2sub(u, __fadd2_rn(t, f2(-kMagic)));
            const float4 v0 = __ldg(reinterpret_cast<const float4*>(
                q1 + (unsigned long long)(unsigned)__float_as_int(t.x) * A.qrow_bytes));
            const float4 v1 = __ldg(reinterpret_cast<const float4*>(
                q2 + (unsigned long long)(unsigned)__float_as_int(t.y) * A.qrow_bytes));
            const float2 p0 = __ffma2_rn(A1, make_float2(v0.z, v0.w), make_float2(v0.x, v0.y));
            const float2 p1 = __ffma2_rn(A2, make_float2(v1.z, v1.w), make_float2(v1.x, v1.y));
            const float s1 = fmaf(b.x, p0.y, p0.x), s2 = fmaf(b.y, p1.y, p1.x);
            acc[j] = fmaf(w1, s1 - s2, acc[j] + s2);
          }
        } else {
#pragma unroll
          for (int j = 0; j < NZ; ++j)
            if (j >= jlo && j < jhi) slice_x(j, std::false_type{});
        }
        continue;
      }
      const float zr1 = fmaf((float)ia + tho, A.dzv, A.z0);
      const float zr2 = fmaf((float)(ia + A.half) - tho, A.dzv, A.z0);
      const float k1 = __fdividef(A.kq, l1), k2 = __fdividef(A.kq, l2);
      const float m1 = -zr1 * k1, m2 = -zr2 * k2;
      int o1, o2;
      float a1, a2;
      quad_col<INTERP>(delta_p + A.ws, A.ns, o1, a1);
      quad_col<INTERP>(-delta_p + A.ws, A.ns, o2, a2);
      const ulonglong2 qb = s_qv[k];
      const float4* q1 = reinterpret_cast<const float4*>(qb.x) + o1;
      const float4* q2 = reinterpret_cast<const float4*>(qb.y) + o2;
      auto slice = [&](int j) {
        const float qh1 = fmaf(zc[j], k1, m1), qh2 = fmaf(zc[j], k2, m2);
        const bool out1 = fabsf(qh1) > wt, out2 = fabsf(qh2) > wt;
        const float r = __fdividef(2.0f, qh1 - qh2);
        float w1 = -qh2 * r, w2 = qh1 * r;
        w1 = out1 ? (out2 ? 1.0f : 0.0f) : (out2 ? 2.0f : w1);
        w2 = out1 ? (out2 ? 1.0f : 2.0f) : (out2 ? 0.0f : w2);
        const float s1 = quad_sample<INTERP>(q1, A.qcols, A.nt, a1, qh1 + wt);
        const float s2 = quad_sample<INTERP>(q2, A.qcols, A.nt, a2, qh2 + wt);
        acc[j] = fmaf(w1, s1, fmaf(w2, s2, acc[j]));
      };
      if (jlo == 0 && jhi == NZ) {
#pragma unroll
        for (int j = 0; j < NZ; ++j) slice(j);
      } else {
#pragma unroll
        for (int j = 0; j < NZ; ++j)
          if (j >= jlo && j < jhi) slice(j);
      }
    }
  }

  if (ix < A.nx && iy < A.ny) {
    float* out = A.img + ((long long)(A.slab_z0[slab] + z0) * A.ny + iy) * A.nx + ix;
    const long long plane = (long long)A.nx * A.ny;
    const bool raw = PART && (A.part == kBpFirst || A.part == kBpMiddle);  // more parts follow
#pragma unroll
    for (int j = 0; j < NZ; ++j) {
      if (j < nzc && raw) {
        out[j * plane] = acc[j];
      } else if (j < nzc) {
        const int span = A.a_max[z0 + j] - A.a_min[z0 + j];
        // CUDA/Backprojector.cu:96, evaluated in double (PI is a double literal there)
        // EXACT accumulates halved weights: x4 restores both the halving and the pair doubling
        const float sc = INTERP == LCT_INTERP_EXACT ? 4.0f : 2.0f;
        out[j * plane] = span > 0 ? (float)((double)(acc[j] * sc) * kRefPi / (double)(float)span) : 0.0f;
      }
    }
  }
}

// PART: a view range of the slabs with raw sums carried in img (BpLaunch::part); the whole-
// launch instantiation has none of that code.  RING: the quads are a ring (bounded recons); the
// linear instantiation has no modulo in its view bases.
template <int NZ, int INTERP, int MINB, bool PART, bool RING>
__global__ void __launch_bounds__(kQTX* kQTY, MINB) bp_quad_kernel(const __grid_constant__ BpQuadArgs A) {
  bp_quad_tile<NZ, INTERP, PART, RING>(A, blockIdx.x, blockIdx.y, blockIdx.z);
}

// EXACT with every view's tile footprint staged in shared memory by TMA.  Per view pair the
// footprint boxes of the view and of its conjugate -- kTmaBH quad rows x kTmaBW quad columns each,
// from the tile's corners at its first and last slice (the prefetch boxes above) -- are loaded
// with one cp.async.bulk.tensor each (no multicast) into a kTmaStages-deep ring, one mbarrier per
// stage for "landed" (transaction bytes) and one for "consumed" (one arrive per warp).  Thread 0
// issues the loads kTmaStages views ahead.  The samples then read shared memory: the same
// floor / fraction / bit-pattern arithmetic as the global path, the address one 32-bit multiply-add
// into the box.  Every warp checks, per view, that its lanes' quad rows (first and last slice:
// rows are monotone in the slice) and columns lie inside the boxes; a warp that is not inside,
// or a view whose footprint exceeds a box, reads global memory as the quad kernel does, so the
// result never depends on the box estimate.  Bit-identical to bp_quad_kernel (same arithmetic
// on the same quad values).  Every mbarrier wait is bounded.
constexpr int kTmaBW = 36;   // quad columns per box
constexpr int kTmaBH = 16;   // quad rows per box
constexpr int kTmaStages = 2;
constexpr unsigned kTmaRowBytes = kTmaBW * 16;
constexpr unsigned kTmaBoxBytes = kTmaBW * kTmaBH * 16;
constexpr unsigned kTmaStageBytes = 2 * kTmaBoxBytes;
constexpr int kTmaSmem = kTmaStages * kTmaStageBytes + 128;  // + alignment slack

template <int NZ>
__device__ __forceinline__ void bp_tma_tile(const BpQuadArgs& A, const CUtensorMap* map, int bx,
                                            int by, int bz, uint32_t stage0, uint32_t full0,
                                            uint32_t empty0, int* status) {
  __shared__ float4 s_cs[kQVB];       // cos, sin of view ia and of its conjugate ia + half
  __shared__ int2 s_jr[kQVB];         // slices [jlo, jhi) of the chunk whose window holds ia
  __shared__ float2 s_zb[kQVB];       // source z of both views without the fan-angle term
  __shared__ ulonglong2 s_qv[kQVB];   // biased global bases of both views (the fallback)
  __shared__ int4 s_box[kQVB];        // box origins: row0, col0 of the view and of the conjugate
  __shared__ int2 s_slot[kQVB];       // quad-buffer view slots (TMA z) of both views; x < 0: no box
  __shared__ int s_abort;

  const int tid = threadIdx.y * kQTX + threadIdx.x;
  const int lane = tid & 31;
  const int ix = bx * kQTX + threadIdx.x;
  const int iy = by * kQTY + threadIdx.y;
  const int slab = bz / A.zchunks;
  const int z0 = (bz % A.zchunks) * NZ;
  const int nzc = min(NZ, A.nz - z0);

  const float xc = __fmul_rn((float)ix - A.wx, A.dx);
  const float yc = __fmul_rn((float)iy - A.wy, A.dy);
  const float zc0 = __fmul_rn((float)z0 - A.wz, A.dz);
  const float wt2 = A.wt + 2.0f;
  const float xr0 = __fmul_rn((float)(bx * kQTX) - A.wx, A.dx);
  const float xr1 = __fmul_rn((float)(min(bx * kQTX + kQTX, A.nx) - 1) - A.wx, A.dx);
  const float yr0 = __fmul_rn((float)(by * kQTY) - A.wy, A.dy);
  const float yr1 = __fmul_rn((float)(min(by * kQTY + kQTY, A.ny) - 1) - A.wy, A.dy);
  const float zcl = __fmul_rn((float)(z0 + nzc - 1) - A.wz, A.dz);
  const float rx = fmaxf(fabsf(xr0), fabsf(xr1)), ry = fmaxf(fabsf(yr0), fabsf(yr1));
  const bool asin_poly = sqrtf(fmaf(rx, rx, ry * ry)) * A.inv_dso < 0.49f;

  int vlo = INT_MAX, vhi = INT_MIN;
  for (int j = 0; j < nzc; ++j) {
    vlo = min(vlo, A.a_min[z0 + j]);
    vhi = max(vhi, A.a_mid[z0 + j]);
  }
  const int sv = A.slab_view[slab];
  const float* betas = A.betas + sv;
  const float wt = A.wt;
  float acc[NZ];
#pragma unroll
  for (int j = 0; j < NZ; ++j) acc[j] = 0.0f;
  if (tid == 0) s_abort = 0;
  long long kk = 0;  // ring uses so far (stage = kk mod kTmaStages, phase = kk / kTmaStages)

  // thread 0: the loads of batch view q (ring use kq) into its stage; a plain arrive when the
  // view has no box, so the stage's "landed" phase completes either way
  auto issue = [&](int q, long long kq) {
    const int st = (int)(kq % kTmaStages);
    const uint32_t fb = full0 + 8 * st;
    const int2 sl = s_slot[q];
    if (sl.x < 0 || s_abort) {
      mbar_arrive(fb);
      return;
    }
    const int4 b = s_box[q];
    mbar_expect_tx(fb, kTmaStageBytes);
    const uint32_t dst = stage0 + st * kTmaStageBytes;
    tma_load_3d(dst, map, 4 * b.y, b.x, sl.x, fb);
    tma_load_3d(dst + kTmaBoxBytes, map, 4 * b.w, b.z, sl.y, fb);
  };

  for (int vb = vlo; vb < vhi; vb += kQVB) {
    __syncthreads();
    if (tid < kQVB && vb + tid < vhi) {
      const int ia = vb + tid;
      float c1, s1, c2, s2;
      view_trig_pi(betas, ia, c1, s1);
      view_trig_pi(betas, ia + A.half, c2, s2);
      s_cs[tid] = make_float4(c1, s1, c2, s2);
      const float4* v1 = quad_view_ptr(A, sv, ia);
      const float4* v2 = quad_view_ptr(A, sv, ia + A.half);
      s_zb[tid] = make_float2(fmaf((float)ia, A.dzv, A.z0), fmaf((float)(ia + A.half), A.dzv, A.z0));
      s_qv[tid] = make_ulonglong2(quad_view_bias(v1, A.qrow_bytes), quad_view_bias(v2, A.qrow_bytes));
      int4 b1, b2;
      prefetch_boxes(A, c1, s1, c2, s2, ia, xr0, xr1, yr0, yr1, zc0, zcl, b1, b2);
      const bool fits = b1.y - b1.x + 1 <= kTmaBH && b1.w - b1.z + 1 <= kTmaBW &&
                        b2.y - b2.x + 1 <= kTmaBH && b2.w - b2.z + 1 <= kTmaBW;
      s_box[tid] = make_int4(b1.x, b1.z, b2.x, b2.z);
      const long long q1 = (long long)(v1 - A.quads) / A.qstride;
      const long long q2 = (long long)(v2 - A.quads) / A.qstride;
      s_slot[tid] = fits ? make_int2((int)q1, (int)q2) : make_int2(-1, -1);
      int jlo = nzc, jhi = 0;
      for (int j = 0; j < nzc; ++j)
        if (ia >= A.a_min[z0 + j] && ia < A.a_mid[z0 + j]) {
          jlo = min(jlo, j);
          jhi = max(jhi, j + 1);
        }
      s_jr[tid] = make_int2(jlo, jhi);
    }
    __syncthreads();
    const int nv = min(kQVB, vhi - vb);
    const long long kbase = kk;
    if (tid == 0)
      for (int q = 0; q < kTmaStages && q < nv; ++q) issue(q, kbase + q);
    for (int k = 0; k < nv; ++k) {
      const long long kq = kbase + k;
      const int st = (int)(kq % kTmaStages);
      const uint32_t parity = (uint32_t)((kq / kTmaStages) & 1);
      const int2 sl = s_slot[k];
      bool smem_ok = sl.x >= 0;
      if (!mbar_wait(full0 + 8 * st, parity)) {  // bounded: a load that never lands
        if (status) atomicExch(status, kDevWaitTimeout);
        s_abort = 1;
        smem_ok = false;
      }
      const int2 jr = s_jr[k];
      const int jlo = jr.x, jhi = jr.y;
      const float4 cs = s_cs[k];
      const float cb = cs.x, sb = cs.y, cb2 = cs.z, sb2 = cs.w;
      const float phat = fmaf(-xc, cb, -__fmul_rn(yc, sb));
      const float sx = __fmul_rn(phat, A.inv_dso);
      const float theta = asin_poly ? asin_half(sx) : asinf(sx);
      const float tho = __fmul_rn(theta, A.inv_orbit);
      const float tq = fmaf(-phat, phat, A.dso2);
      const float sq = __fmul_rn(tq, rsqrtf(tq));
      const float l1 = fmaf(xc, sb, fmaf(-yc, cb, sq));
      const float l2 = fmaf(xc, sb2, fmaf(-yc, cb2, sq));
      const float2 zb = s_zb[k];
      const ulonglong2 qv = s_qv[k];
      const float zr1 = fmaf(tho, A.dzv, zb.x), zr2 = fmaf(-tho, A.dzv, zb.y);
      const float r1 = __fdividef(1.0f, l1), r2 = __fdividef(1.0f, l2);
      const float kd1 = __fmul_rn(A.kqdz, r1), kd2 = __fmul_rn(A.kqdz, r2);
      const float h1 = __fmul_rn(__fsub_rn(zc0, zr1), __fmul_rn(A.kq, r1));
      const float h2 = __fmul_rn(__fsub_rn(zc0, zr2), __fmul_rn(A.kq, r2));
      const float u1 = __fadd_rn(h1, wt2), u2 = __fadd_rn(h2, wt2);
      float a1, a2;
      const unsigned long long q1 = quad_col_exact(qv.x, fmaf(theta, A.dso_over_ds, A.ws), A.ns, a1);
      const unsigned long long q2 = quad_col_exact(qv.y, fmaf(-theta, A.dso_over_ds, A.ws), A.ns, a2);
      // the thread's quad columns (0 .. ns + 2) and its first / last slice's quad rows
      const int qc1 = (int)((q1 - qv.x) >> 4) - (kMagicBits - 2);
      const int qc2 = (int)((q2 - qv.y) >> 4) - (kMagicBits - 2);
      auto qrow = [&](float u) {
        const int rb = __float_as_int(__fadd_rd(u, kMagic));
        return min(max(rb, kMagicBits), kMagicBits + A.nt + 2) - kMagicBits;
      };
      const int4 bo = s_box[k];
      bool in_box = false;
      if (smem_ok && jlo < jhi) {
        const float fa = (float)jlo, fb = (float)(jhi - 1);
        const int ra1 = qrow(fmaf(fa, kd1, u1)), rb1 = qrow(fmaf(fb, kd1, u1));
        const int ra2 = qrow(fmaf(fa, kd2, u2)), rb2 = qrow(fmaf(fb, kd2, u2));
        in_box = min(ra1, rb1) >= bo.x && max(ra1, rb1) < bo.x + kTmaBH && qc1 >= bo.y &&
                 qc1 < bo.y + kTmaBW && min(ra2, rb2) >= bo.z && max(ra2, rb2) < bo.z + kTmaBH &&
                 qc2 >= bo.w && qc2 < bo.w + kTmaBW;
      } else if (smem_ok) {
        in_box = true;  // no slice of this thread uses the view
      }
      const bool use_smem = __all_sync(0xffffffffu, in_box);
      // shared-memory bases biased like the global ones: + row bit pattern * row bytes
      const uint32_t sbase = stage0 + st * kTmaStageBytes;
      const uint32_t sbv = sbase + 16u * (uint32_t)(qc1 - bo.y) -
                           (uint32_t)(kMagicBits + bo.x) * kTmaRowBytes;
      const uint32_t sbc = sbase + kTmaBoxBytes + 16u * (uint32_t)(qc2 - bo.w) -
                           (uint32_t)(kMagicBits + bo.z) * kTmaRowBytes;
      auto sample = [&](bool smem, bool clamp, unsigned long long gq, uint32_t sq0, float a,
                        float u) -> float {
        const float t = __fadd_rd(u, kMagic);
        const float b = u - (t - kMagic);
        int rb = __float_as_int(t);
        if (clamp) rb = min(max(rb, kMagicBits), kMagicBits + A.nt + 2);
        const float4 v = smem ? lds128(sq0 + (uint32_t)rb * kTmaRowBytes)
                              : __ldg(reinterpret_cast<const float4*>(
                                    gq + (unsigned long long)(unsigned)rb * A.qrow_bytes));
        return fmaf(b, fmaf(a, v.w, v.y), fmaf(a, v.z, v.x));  // T00, dy, dx, dxy
      };
      auto slice_x = [&](int j, auto inside, auto smem) {
        const float fj = (float)j;
        const float qh1 = fmaf(fj, kd1, h1), qh2 = fmaf(fj, kd2, h2);
        const float in1 = -qh2 * __fdividef(1.0f, qh1 - qh2);
        float w1 = in1;
        if constexpr (!decltype(inside)::value) {
          const bool out1 = fabsf(qh1) > wt, out2 = fabsf(qh2) > wt;
          w1 = out1 ? (out2 ? 0.5f : 0.0f) : (out2 ? 1.0f : in1);
        }
        constexpr bool kClamp = !decltype(inside)::value;
        constexpr bool kSmem = decltype(smem)::value;
        const float s1 = sample(kSmem, kClamp, q1, sbv, a1, fmaf(fj, kd1, u1));
        const float s2 = sample(kSmem, kClamp, q2, sbc, a2, fmaf(fj, kd2, u2));
        acc[j] = fmaf(w1, s1 - s2, acc[j] + s2);
      };
      bool inside = false;
      if (jlo == 0 && jhi == NZ) {
        const float e1 = fmaf((float)(NZ - 1), kd1, h1), e2 = fmaf((float)(NZ - 1), kd2, h2);
        inside = A.rows_inside_ok && fabsf(h1) <= wt && fabsf(e1) <= wt && fabsf(h2) <= wt &&
                 fabsf(e2) <= wt;
      }
      const bool all_inside = __all_sync(0xffffffffu, inside);
      if (use_smem) {
        if (all_inside) {
#pragma unroll
          for (int j = 0; j < NZ; ++j) slice_x(j, std::true_type{}, std::true_type{});
        } else {
#pragma unroll
          for (int j = 0; j < NZ; ++j)
            if (j >= jlo && j < jhi) slice_x(j, std::false_type{}, std::true_type{});
        }
      } else {
        if (all_inside) {
#pragma unroll
          for (int j = 0; j < NZ; ++j) slice_x(j, std::true_type{}, std::false_type{});
        } else {
#pragma unroll
          for (int j = 0; j < NZ; ++j)
            if (j >= jlo && j < jhi) slice_x(j, std::false_type{}, std::false_type{});
        }
      }
      // this warp is done with the stage; thread 0 refills it kTmaStages views ahead
      __syncwarp();
      if (lane == 0) mbar_arrive(empty0 + 8 * st);
      if (tid == 0 && k + kTmaStages < nv) {
        if (!mbar_wait(empty0 + 8 * st, parity)) {
          if (status) atomicExch(status, kDevWaitTimeout);
          s_abort = 1;
        }
        issue(k + kTmaStages, kq + kTmaStages);
      }
    }
    kk = kbase + nv;
  }
  // after a wait that ran out, the copies still in flight land before the CTA exits (bounded)
  if (tid == 0 && s_abort)
    for (long long kq = (kk > kTmaStages ? kk - kTmaStages : 0); kq < kk; ++kq)
      mbar_wait(full0 + 8 * (int)(kq % kTmaStages), (uint32_t)((kq / kTmaStages) & 1));
  __syncthreads();

  if (ix < A.nx && iy < A.ny) {
    float* out = A.img + ((long long)(A.slab_z0[slab] + z0) * A.ny + iy) * A.nx + ix;
    const long long plane = (long long)A.nx * A.ny;
#pragma unroll
    for (int j = 0; j < NZ; ++j) {
      if (j < nzc) {
        const int span = A.a_max[z0 + j] - A.a_min[z0 + j];
        // CUDA/Backprojector.cu:96 in double; x4 restores the halved weights and the pair doubling
        out[j * plane] = span > 0 ? (float)((double)(acc[j] * 4.0f) * kRefPi / (double)(float)span) : 0.0f;
      }
    }
  }
}

template <int NZ, int MINB>
__global__ void __launch_bounds__(kQTX* kQTY, MINB)
    bp_tma_kernel(const __grid_constant__ BpQuadArgs A, const __grid_constant__ CUtensorMap map,
                  int* status) {
  extern __shared__ uint8_t tma_smem_raw[];
  __shared__ __align__(8) uint64_t bars[2 * kTmaStages];
  const uint32_t stage0 = (smem_u32(tma_smem_raw) + 127u) & ~127u;
  const uint32_t full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[kTmaStages]);
  const int tid = threadIdx.y * kQTX + threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < kTmaStages; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, kQTX * kQTY / 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  bp_tma_tile<NZ>(A, &map, blockIdx.x, blockIdx.y, blockIdx.z, stage0, full0, empty0, status);
}

// TEX8 sampled by the texture unit itself: the filtered views in a 3-D cudaArray (x = column,
// y = row, z = view slot; cudaFilterModeLinear, unnormalised, the recon's addressing) and every
// sample one tex3D at (p_idx + 0.5, q_idx + 0.5, slot + 0.5) -- the reference's own fetch
// (CUDA/Backprojector.cu:85-86), with z on a texel centre.  The per-view and per-slice arithmetic
// is the quad kernel's TEX8 path (the reference's order); only the sample differs: the unit's
// 8-bit weights replace their register emulation.  Slab s's local view ia sits at slot
// (slab_view[s] + ia) mod qring (qring 0: no wrap).
template <int NZ, bool PART>
__device__ __forceinline__ void bp_tex_tile(const BpQuadArgs& A, cudaTextureObject_t tex, int bx,
                                            int by, int bz) {
  __shared__ float4 s_cs[kQVB];  // cos, sin of view ia and of its conjugate ia + half
  __shared__ int2 s_jr[kQVB];    // slices [jlo, jhi) of the chunk whose window holds ia
  __shared__ float2 s_zs[kQVB];  // texture z of both views (slot + 0.5)

  const int tid = threadIdx.y * kQTX + threadIdx.x;
  const int ix = bx * kQTX + threadIdx.x;
  const int iy = by * kQTY + threadIdx.y;
  const int slab = bz / A.zchunks;
  const int z0 = (bz % A.zchunks) * NZ;
  const int nzc = min(NZ, A.nz - z0);
  const float xc = __fmul_rn((float)ix - A.wx, A.dx);
  const float yc = __fmul_rn((float)iy - A.wy, A.dy);
  float zc[NZ];
#pragma unroll
  for (int j = 0; j < NZ; ++j) zc[j] = ((float)(z0 + j) - A.wz) * A.dz;

  int vlo = INT_MAX, vhi = INT_MIN;
  for (int j = 0; j < nzc; ++j) {
    vlo = min(vlo, A.a_min[z0 + j]);
    vhi = max(vhi, A.a_mid[z0 + j]);
  }
  if (PART) {
    vlo = max(vlo, A.view_lo);
    vhi = min(vhi, A.view_hi);
  }
  const int sv = A.slab_view[slab];
  const float* betas = A.betas + sv;
  const float wt = A.wt;

  float acc[NZ];
#pragma unroll
  for (int j = 0; j < NZ; ++j) acc[j] = 0.0f;
  if (PART && A.part >= kBpMiddle && ix < A.nx && iy < A.ny) {  // continue earlier parts' sums
    const float* in = A.img + ((long long)(A.slab_z0[slab] + z0) * A.ny + iy) * A.nx + ix;
#pragma unroll
    for (int j = 0; j < NZ; ++j)
      if (j < nzc) acc[j] = in[j * (long long)A.nx * A.ny];
  }

  for (int vb = vlo; vb < vhi; vb += kQVB) {
    __syncthreads();
    if (tid < kQVB && vb + tid < vhi) {
      const int ia = vb + tid;
      float c1, s1, c2, s2;
      view_trig_mode<LCT_INTERP_TEX8>(betas, ia, c1, s1);
      view_trig_mode<LCT_INTERP_TEX8>(betas, ia + A.half, c2, s2);
      s_cs[tid] = make_float4(c1, s1, c2, s2);
      long long v1 = (long long)sv + ia, v2 = v1 + A.half;
      if (A.qring > 0) {
        v1 %= A.qring;
        v2 %= A.qring;
      }
      s_zs[tid] = make_float2((float)v1 + 0.5f, (float)v2 + 0.5f);
      int jlo = nzc, jhi = 0;
      for (int j = 0; j < nzc; ++j)
        if (ia >= A.a_min[z0 + j] && ia < A.a_mid[z0 + j]) {
          jlo = min(jlo, j);
          jhi = max(jhi, j + 1);
        }
      s_jr[tid] = make_int2(jlo, jhi);
    }
    __syncthreads();
    const int nv = min(kQVB, vhi - vb);
    for (int k = 0; k < nv; ++k) {
      const int ia = vb + k;
      const int2 jr = s_jr[k];
      const int jlo = jr.x, jhi = jr.y;
      const float4 cs = s_cs[k];
      const float2 zs = s_zs[k];
      const float cb = cs.x, sb = cs.y, cb2 = cs.z, sb2 = cs.w;
      // CUDA/Backprojector.cu:53-64, z-invariant part, in the reference's order
      const float phat = fmaf(-xc, cb, -__fmul_rn(yc, sb));
      const float theta = asinf(__fdiv_rn(phat, A.dso));
      const float delta_p = __fdiv_rn(__fmul_rn(theta, A.dso), A.ds);
      const float tho = __fdiv_rn(theta, A.orbit);
      const float sq = sqrtf(fmaf(-phat, phat, A.dso2));
      const float l1 = fmaf(xc, sb, fmaf(-yc, cb, sq));
      const float l2 = fmaf(xc, sb2, fmaf(-yc, cb2, sq));
      const float zr1 = fmaf((float)ia + tho, A.dzv, A.z0);
      const float zr2 = fmaf((float)(ia + A.half) - tho, A.dzv, A.z0);
      const float k1 = __fdividef(A.kq, l1), k2 = __fdividef(A.kq, l2);
      const float m1 = -zr1 * k1, m2 = -zr2 * k2;
      const float x1 = __fadd_rn(delta_p + A.ws, 0.5f), x2 = __fadd_rn(-delta_p + A.ws, 0.5f);
      auto slice = [&](int j) {
        const float qh1 = fmaf(zc[j], k1, m1), qh2 = fmaf(zc[j], k2, m2);
        const bool out1 = fabsf(qh1) > wt, out2 = fabsf(qh2) > wt;
        const float r = __fdividef(2.0f, qh1 - qh2);
        float w1 = -qh2 * r, w2 = qh1 * r;
        w1 = out1 ? (out2 ? 1.0f : 0.0f) : (out2 ? 2.0f : w1);
        w2 = out1 ? (out2 ? 1.0f : 2.0f) : (out2 ? 0.0f : w2);
        const float s1 = tex3D<float>(tex, x1, __fadd_rn(qh1 + wt, 0.5f), zs.x);
        const float s2 = tex3D<float>(tex, x2, __fadd_rn(qh2 + wt, 0.5f), zs.y);
        acc[j] = fmaf(w1, s1, fmaf(w2, s2, acc[j]));
      };
      if (jlo == 0 && jhi == NZ) {
#pragma unroll
        for (int j = 0; j < NZ; ++j) slice(j);
      } else {
#pragma unroll
        for (int j = 0; j < NZ; ++j)
          if (j >= jlo && j < jhi) slice(j);
      }
    }
  }

  if (ix < A.nx && iy < A.ny) {
    float* out = A.img + ((long long)(A.slab_z0[slab] + z0) * A.ny + iy) * A.nx + ix;
    const long long plane = (long long)A.nx * A.ny;
    const bool raw = PART && (A.part == kBpFirst || A.part == kBpMiddle);  // more parts follow
#pragma unroll
    for (int j = 0; j < NZ; ++j) {
      if (j < nzc && raw) {
        out[j * plane] = acc[j];
      } else if (j < nzc) {
        const int span = A.a_max[z0 + j] - A.a_min[z0 + j];
        // CUDA/Backprojector.cu:96 in double; x2 restores the pair doubling
        out[j * plane] = span > 0 ? (float)((double)(acc[j] * 2.0f) * kRefPi / (double)(float)span) : 0.0f;
      }
    }
  }
}

template <int NZ, int MINB, bool PART>
__global__ void __launch_bounds__(kQTX* kQTY, MINB)
    bp_tex_kernel(const __grid_constant__ BpQuadArgs A, cudaTextureObject_t tex) {
  bp_tex_tile<NZ, PART>(A, tex, blockIdx.x, blockIdx.y, blockIdx.z);
}

// Persistent work list over several scans: item i belongs to the scan s with
// prefix[s] <= i < prefix[s + 1] and is tile i - prefix[s] of that scan's grid.  Each CTA takes
// items from *counter (zero before the launch) until the list is exhausted; a scan's tiles run
// exactly the arithmetic of its own launch.
template <int NZ, int INTERP, int MINB>
__global__ void __launch_bounds__(kQTX* kQTY, MINB)
    bp_quad_worklist_kernel(const BpQuadArgs* __restrict__ args, const int* __restrict__ prefix,
                            int n_scans, int* __restrict__ counter) {
  __shared__ BpQuadArgs sA;
  __shared__ int s_item, s_scan;
  const int tid = threadIdx.y * kQTX + threadIdx.x;
  const int total = prefix[n_scans];
  for (;;) {
    __syncthreads();  // the previous tile is done with sA
    if (tid == 0) {
      const int item = atomicAdd(counter, 1);
      int sc = 0;
      while (sc + 1 < n_scans && prefix[sc + 1] <= item) ++sc;
      s_item = item;
      s_scan = sc;
    }
    __syncthreads();
    const int item = s_item;
    if (item >= total) return;
    const int* src = reinterpret_cast<const int*>(args + s_scan);
    int* dst = reinterpret_cast<int*>(&sA);
    for (int i = tid; i < (int)(sizeof(BpQuadArgs) / sizeof(int)); i += kQTX * kQTY) dst[i] = src[i];
    __syncthreads();
    const int local = item - prefix[s_scan];
    const int bx = local % sA.gx;
    const int by = (local / sA.gx) % sA.gy;
    const int bz = local / (sA.gx * sA.gy);
    bp_quad_tile<NZ, INTERP, false, false>(sA, bx, by, bz);
  }
}

bool bp_windows_full(const lct_geom& g, const lct_img& ig, int nz) {
  const float dzv = g.pitch / (float)g.n_proj_turn;
  const int half = g.n_proj_turn / 2;
  for (int z = 0; z < nz; ++z) {
    BpWindow w = bp_window(g, ig, z, dzv, half);
    if (!(w.a_min == w.a_mid - half && w.a_max == w.a_mid + half)) return false;
  }
  return true;
}

static int build_bp_quad_args(const lct_geom& g, const lct_img& ig, const BpLaunch& L,
                              const float4* quads, BpQuadArgs& a, int& nzt) {
  if (L.nz <= 0 || L.nz > kBpMaxZ || L.n_slabs <= 0 || L.n_slabs > kBpMaxSlabs) return LCT_ERR_ARG;
  if (!bp_windows_full(g, ig, L.nz)) return LCT_ERR_UNSUPPORTED;
  a.quads = quads;
  a.qring = L.quad_ring;
  if (a.qring < 0) return LCT_ERR_ARG;
  a.betas = L.betas;
  a.img = L.img;
  a.qstride = quad_view_elems(g.ns, g.nt);
  a.qcols = (int)quad_cols(g.ns);
  a.ns = g.ns;
  a.nt = g.nt;
  a.n_angle = L.n_angle;
  a.nx = ig.nx;
  a.ny = ig.ny;
  a.nz = L.nz;
  a.ws = g.ws;
  a.wt = g.wt;
  a.ds = g.ds;
  a.dso = g.dso;
  a.dso2 = g.dso * g.dso;
  a.inv_dso = 1.0f / g.dso;
  a.dso_over_ds = g.dso / g.ds;
  a.orbit = g.orbit;
  a.inv_orbit = 1.0f / g.orbit;
  a.z0 = g.source_z0;
  a.dzv = g.pitch / (float)g.n_proj_turn;  // CUDA/Backprojector.cu:149
  a.kq = g.dso * (float)g.z_dir / g.dt;
  a.kqdz = a.kq * ig.dz;
  a.qrow_bytes = (unsigned)(quad_cols(g.ns) * 16);
  a.rows_inside_ok = (2.0 * (double)g.wt + 2.5 < (double)g.nt + 3.0) ? 1 : 0;
  a.wx = ig.wx;
  a.wy = ig.wy;
  a.wz = ig.wz;
  a.dx = ig.dx;
  a.dy = ig.dy;
  a.dz = ig.dz;
  a.half = g.n_proj_turn / 2;  // CUDA/Backprojector.cu:148
  for (int z = 0; z < L.nz; ++z) {
    BpWindow w = bp_window(g, ig, z, a.dzv, a.half);
    a.a_min[z] = w.a_min;
    a.a_mid[z] = w.a_mid;
    a.a_max[z] = w.a_max;
  }
  for (int i = 0; i < L.n_slabs; ++i) {
    a.slab_view[i] = L.slab_view[i];
    a.slab_z0[i] = L.slab_z0[i];
  }
  nzt = L.nz_thread;
  if (nzt != 4 && nzt != 8 && nzt != 16) nzt = 8;
  a.zchunks = (L.nz + nzt - 1) / nzt;
  a.gx = (ig.nx + kQTX - 1) / kQTX;
  a.gy = (ig.ny + kQTY - 1) / kQTY;
  a.gz = L.n_slabs * a.zchunks;
  if (L.part < kBpWhole || L.part > kBpLast || L.view_lo > L.view_hi) return LCT_ERR_ARG;
  a.view_lo = L.view_lo;
  a.view_hi = L.view_hi;
  a.part = L.part;
  if (a.gz > 65535) return LCT_ERR_ARG;
  return LCT_OK;
}

int launch_bp_par_quads(const lct_geom& g, const lct_img& ig, const BpLaunch& L,
                        const float4* quads, cudaStream_t s) {
  static thread_local BpQuadArgs a;
  int nzt = 8;
  int st = build_bp_quad_args(g, ig, L, quads, a, nzt);
  if (st) return st;
  dim3 grid(a.gx, a.gy, a.gz);
  dim3 block(kQTX, kQTY);
  const bool tex = L.interp == LCT_INTERP_TEX8;
  int minb = L.minb;
  if (minb < 1 || minb > 4) minb = 4;  // measured best on B200 (4 CTAs x 256 threads per SM)
  const bool part = L.part != kBpWhole || L.view_lo > 0 || L.view_hi < (1 << 30);
#define LCT_BPQ(NZV, MB)                                                                          \
  do {                                                                                            \
    if (part && tex) bp_quad_kernel<NZV, LCT_INTERP_TEX8, MB, true, false><<<grid, block, 0, s>>>(a); \
    else if (part) bp_quad_kernel<NZV, LCT_INTERP_EXACT, MB, true, false><<<grid, block, 0, s>>>(a);  \
    else if (tex) bp_quad_kernel<NZV, LCT_INTERP_TEX8, MB, false, false><<<grid, block, 0, s>>>(a);   \
    else bp_quad_kernel<NZV, LCT_INTERP_EXACT, MB, false, false><<<grid, block, 0, s>>>(a);           \
  } while (0)
  // quad rings (bounded recons): 4 CTAs per SM
#define LCT_BPQR(NZV)                                                                            \
  do {                                                                                           \
    if (part && tex) bp_quad_kernel<NZV, LCT_INTERP_TEX8, 4, true, true><<<grid, block, 0, s>>>(a); \
    else if (part) bp_quad_kernel<NZV, LCT_INTERP_EXACT, 4, true, true><<<grid, block, 0, s>>>(a);  \
    else if (tex) bp_quad_kernel<NZV, LCT_INTERP_TEX8, 4, false, true><<<grid, block, 0, s>>>(a);   \
    else bp_quad_kernel<NZV, LCT_INTERP_EXACT, 4, false, true><<<grid, block, 0, s>>>(a);           \
  } while (0)
  if (a.qring > 0) {
    switch (nzt) {
      case 4: LCT_BPQR(4); break;
      case 16: LCT_BPQR(16); break;
      default: LCT_BPQR(8);
    }
#undef LCT_BPQR
    return launch_status();
  }
#define LCT_BPQ_NZ(NZV)            \
  do {                             \
    switch (minb) {                \
      case 1: LCT_BPQ(NZV, 1); break; \
      case 3: LCT_BPQ(NZV, 3); break; \
      case 4: LCT_BPQ(NZV, 4); break; \
      default: LCT_BPQ(NZV, 2);    \
    }                              \
  } while (0)
  switch (nzt) {
    case 4: LCT_BPQ_NZ(4); break;
    case 16: LCT_BPQ_NZ(16); break;
    default: LCT_BPQ_NZ(8);
  }
#undef LCT_BPQ_NZ
#undef LCT_BPQ
  return launch_status();
}

// Tensor map of a quad buffer for the TMA-staged kernel: 3-D float tensor {4 (ns + 3) floats,
// nt + 3 rows, views}, box {4 kTmaBW, kTmaBH, 1}, no swizzle, out-of-range reads as zero.
int bp_tma_map(CUtensorMap* map, const float4* quads, int ns, int nt, long long views) {
  auto fn = tensor_map_encoder();
  if (!fn) return LCT_ERR_UNSUPPORTED;
  if (reinterpret_cast<uintptr_t>(quads) % 16 != 0 || views <= 0 || views > 0x7fffffffLL)
    return LCT_ERR_ARG;
  const cuuint64_t dims[3] = {(cuuint64_t)(4 * quad_cols(ns)), (cuuint64_t)(nt + 3),
                              (cuuint64_t)views};
  const cuuint64_t strides[2] = {(cuuint64_t)(16 * quad_cols(ns)),
                                 (cuuint64_t)(16 * quad_view_elems(ns, nt))};
  const cuuint32_t box[3] = {(cuuint32_t)(4 * kTmaBW), (cuuint32_t)kTmaBH, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float4*>(quads), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? LCT_OK : LCT_ERR_UNSUPPORTED;
}

int launch_bp_par_quads_tma(const lct_geom& g, const lct_img& ig, const BpLaunch& L,
                            const float4* quads, const CUtensorMap& map, cudaStream_t s) {
  if (L.interp != LCT_INTERP_EXACT) return LCT_ERR_UNSUPPORTED;
  const bool part = L.part != kBpWhole || L.view_lo > 0 || L.view_hi < (1 << 30);
  if (part) return launch_bp_par_quads(g, ig, L, quads, s);  // parts stay on the L1 kernel
  static thread_local BpQuadArgs a;
  int nzt = 8;
  int st = build_bp_quad_args(g, ig, L, quads, a, nzt);
  if (st) return st;
  if (nzt != 8) return launch_bp_par_quads(g, ig, L, quads, s);  // the staged kernel is NZ 8
  dim3 grid(a.gx, a.gy, a.gz);
  dim3 block(kQTX, kQTY);
  int minb = L.minb;
  if (minb < 2 || minb > 4) minb = 4;
  int* status = device_status_ptr();
  switch (minb) {
    case 2: bp_tma_kernel<8, 2><<<grid, block, kTmaSmem, s>>>(a, map, status); break;
    case 3: bp_tma_kernel<8, 3><<<grid, block, kTmaSmem, s>>>(a, map, status); break;
    default: bp_tma_kernel<8, 4><<<grid, block, kTmaSmem, s>>>(a, map, status);
  }
  return launch_status();
}

int launch_bp_par_texture(const lct_geom& g, const lct_img& ig, const BpLaunch& L,
                          cudaTextureObject_t tex, cudaStream_t s) {
  if (L.interp != LCT_INTERP_TEX8) return LCT_ERR_UNSUPPORTED;
  static thread_local BpQuadArgs a;
  int nzt = 8;
  int st = build_bp_quad_args(g, ig, L, nullptr, a, nzt);
  if (st) return st;
  dim3 grid(a.gx, a.gy, a.gz);
  dim3 block(kQTX, kQTY);
  int minb = L.minb;
  if (minb < 1 || minb > 4) minb = 4;
  const bool part = L.part != kBpWhole || L.view_lo > 0 || L.view_hi < (1 << 30);
#define LCT_BPT(NZV, MB)                                                         \
  do {                                                                           \
    if (part) bp_tex_kernel<NZV, MB, true><<<grid, block, 0, s>>>(a, tex);       \
    else bp_tex_kernel<NZV, MB, false><<<grid, block, 0, s>>>(a, tex);           \
  } while (0)
#define LCT_BPT_NZ(NZV)                  \
  do {                                   \
    switch (minb) {                      \
      case 2: LCT_BPT(NZV, 2); break;    \
      case 3: LCT_BPT(NZV, 3); break;    \
      default: LCT_BPT(NZV, 4);          \
    }                                    \
  } while (0)
  switch (nzt) {
    case 4: LCT_BPT_NZ(4); break;
    case 16: LCT_BPT_NZ(16); break;
    default: LCT_BPT_NZ(8);
  }
#undef LCT_BPT_NZ
#undef LCT_BPT
  return launch_status();
}

int bp_quad_args_size() { return (int)sizeof(BpQuadArgs); }

int bp_quad_args_build(const lct_geom& g, const lct_img& ig, const BpLaunch& L,
                       const float4* quads, void* out, int* tiles) {
  BpQuadArgs* a = static_cast<BpQuadArgs*>(out);
  int nzt = 8;
  int st = build_bp_quad_args(g, ig, L, quads, *a, nzt);
  if (st) return st;
  *tiles = a->gx * a->gy * a->gz;
  return LCT_OK;
}

int launch_bp_quad_worklist(const void* d_args, const int* d_prefix, int n_scans, int* d_counter,
                            int nz_thread, int interp, int minb, cudaStream_t s) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (minb < 1 || minb > 4) minb = 4;
  const BpQuadArgs* args = static_cast<const BpQuadArgs*>(d_args);
  dim3 grid(sms * minb), block(kQTX, kQTY);
  const bool tex = interp == LCT_INTERP_TEX8;
#define LCT_BPW(NZV, MB)                                                                        \
  do {                                                                                          \
    if (tex)                                                                                    \
      bp_quad_worklist_kernel<NZV, LCT_INTERP_TEX8, MB><<<grid, block, 0, s>>>(args, d_prefix, n_scans, d_counter); \
    else                                                                                        \
      bp_quad_worklist_kernel<NZV, LCT_INTERP_EXACT, MB><<<grid, block, 0, s>>>(args, d_prefix, n_scans, d_counter); \
  } while (0)
#define LCT_BPW_NZ(NZV)                  \
  do {                                   \
    switch (minb) {                      \
      case 2: LCT_BPW(NZV, 2); break;    \
      case 3: LCT_BPW(NZV, 3); break;    \
      default: LCT_BPW(NZV, 4);          \
    }                                    \
  } while (0)
  switch (nz_thread) {
    case 4: LCT_BPW_NZ(4); break;
    case 16: LCT_BPW_NZ(16); break;
    default: LCT_BPW_NZ(8);
  }
#undef LCT_BPW_NZ
#undef LCT_BPW
  return launch_status();
}

}  // namespace lct
