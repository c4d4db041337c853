// Scan simulator (no reference counterpart): analytic line integrals of an ellipsoid phantom
// along the helical fan-beam rays of the reference geometry, plus Poisson noise.
//
// Geometry, recovered from the reference kernels (the rebin takes fan view ia + alpha/orbit
// for parallel view ia, CUDA/Rebiner.cu:92-100; the backprojector inverts it with
// theta = asin(phat/dso) and lhat = sqrt(dso^2 - phat^2) + x sin b - y cos b,
// CUDA/Backprojector.cu:53-61):
//   source at angle b, couch z:  S = (-R sin b, R cos b, z)
//   column is:   fan angle a = (is - ws) ds / R (equiangular)
//   in-plane ray direction:      (sin(b - a), -cos(b - a))
//   row it:      iso-scaled height t = (it - wt) dt; the ray rises t / R per unit in-plane length
// Noise: counts ~ Poisson(I0 exp(-p)) drawn from a counter-based Philox4x32-10 stream
// (Salmon et al., SC'11) -- Knuth's product method below 30 expected counts, a rounded
// normal N(l, l) above -- clamped to >= 1, then p = -ln(counts / I0).  The CPU oracle
// evaluates the identical formulas, so GPU and CPU scans agree to rounding.
#include <cmath>

#include "lct_internal.h"

namespace lct {

constexpr int kSimMaxEllipsoids = 128;

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
    const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

__device__ double noisy_integral(double p, double i0, uint64_t seed, uint64_t idx) {
  if (i0 <= 0.0) return p;
  uint32_t c[4] = {(uint32_t)idx, (uint32_t)(idx >> 32), 0x4c435430u, 0u};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double u1 = ((double)c[0] + 0.5) * (1.0 / 4294967296.0);
  const double u2 = ((double)c[1] + 0.5) * (1.0 / 4294967296.0);
  const double lam = i0 * exp(-p);
  double n;
  if (lam < 30.0) {
    const double L = exp(-lam);
    double prod = u1;
    int k = 0, j = 0;
    uint32_t cc[4] = {c[2], c[3], 0x4b4e5554u, 0u};
    while (prod > L && k < 1000) {
      ++k;
      if (j == 4) {
        philox4x32_10(cc, (uint32_t)seed, (uint32_t)(seed >> 32));
        j = 0;
      }
      prod *= ((double)cc[j++] + 0.5) * (1.0 / 4294967296.0);
    }
    n = k;
  } else {
    const double z = sqrt(-2.0 * log(u1)) * cos(2.0 * kRefPi * u2);
    n = floor(lam + sqrt(lam) * z + 0.5);
  }
  if (n < 1.0) n = 1.0;
  return -log(n / i0);
}

// grid (ceil(ns/128), nt, views), block 128; ellipsoids staged in shared memory
__global__ void __launch_bounds__(128) sim_project_kernel(const double* __restrict__ ell, int ne,
                                                          int ns, int nt, float ds, float dt,
                                                          float ws, float wt, float dso,
                                                          const double* __restrict__ angles,
                                                          const double* __restrict__ zpos,
                                                          long long v0, double i0, uint64_t seed,
                                                          float* __restrict__ fan) {
  __shared__ double s_e[kSimMaxEllipsoids * 16];
  for (int i = threadIdx.x; i < ne * 16; i += blockDim.x) s_e[i] = ell[i];
  __syncthreads();
  const int is = blockIdx.x * blockDim.x + threadIdx.x;
  const int it = blockIdx.y;
  const long long v = v0 + blockIdx.z;
  if (is >= ns) return;
  const double R = dso;
  const double b = angles[v], z = zpos[v];
  const double S[3] = {-R * sin(b), R * cos(b), z};
  const double t = ((double)it - wt) * dt;
  const double a = ((double)is - ws) * ds / R;
  const double D[3] = {sin(b - a), -cos(b - a), t / R};
  const double dn = sqrt(D[0] * D[0] + D[1] * D[1] + D[2] * D[2]);
  double p = 0.0;
  for (int m = 0; m < ne; ++m) {
    const double* e = s_e + 16 * m;  // cx cy cz ax ay az rot[9] mu
    const double* Rm = e + 6;
    const double q[3] = {S[0] - e[0], S[1] - e[1], S[2] - e[2]};
    double sv[3], dv[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      sv[r] = Rm[0 * 3 + r] * q[0] + Rm[1 * 3 + r] * q[1] + Rm[2 * 3 + r] * q[2];
      dv[r] = Rm[0 * 3 + r] * D[0] + Rm[1 * 3 + r] * D[1] + Rm[2 * 3 + r] * D[2];
    }
    sv[0] /= e[3]; sv[1] /= e[4]; sv[2] /= e[5];
    dv[0] /= e[3]; dv[1] /= e[4]; dv[2] /= e[5];
    const double A = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2];
    const double B = sv[0] * dv[0] + sv[1] * dv[1] + sv[2] * dv[2];
    const double C = sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2] - 1.0;
    const double disc = B * B - A * C;
    if (disc > 0.0) p += e[15] * 2.0 * sqrt(disc) / A * dn;
  }
  const uint64_t idx = ((uint64_t)v * nt + it) * ns + is;
  fan[((long long)blockIdx.z * nt + it) * ns + is] = (float)noisy_integral(p, i0, seed, idx);
}

// voxelised phantom: one thread per voxel, ss^3 sub-samples, ellipsoids in shared memory
__global__ void __launch_bounds__(128) voxelise_kernel(const double* __restrict__ ell, int ne,
                                                       int nx, int ny, double x0, double y0,
                                                       double z0, double dx, double dy,
                                                       double dz, int ss, float* __restrict__ out) {
  __shared__ double s_e[kSimMaxEllipsoids * 16];
  for (int i = threadIdx.x; i < ne * 16; i += blockDim.x) s_e[i] = ell[i];
  __syncthreads();
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y, iz = blockIdx.z;
  if (ix >= nx) return;
  double acc = 0.0;
  for (int sz = 0; sz < ss; ++sz)
    for (int sy = 0; sy < ss; ++sy)
      for (int sx = 0; sx < ss; ++sx) {
        const double P[3] = {x0 + (ix + (sx + 0.5) / ss - 0.5) * dx,
                             y0 + (iy + (sy + 0.5) / ss - 0.5) * dy,
                             z0 + (iz + (sz + 0.5) / ss - 0.5) * dz};
        for (int m = 0; m < ne; ++m) {
          const double* e = s_e + 16 * m;
          const double* R = e + 6;
          const double p[3] = {P[0] - e[0], P[1] - e[1], P[2] - e[2]};
          const double u0 = (R[0] * p[0] + R[3] * p[1] + R[6] * p[2]) / e[3];
          const double u1 = (R[1] * p[0] + R[4] * p[1] + R[7] * p[2]) / e[4];
          const double u2 = (R[2] * p[0] + R[5] * p[1] + R[8] * p[2]) / e[5];
          if (u0 * u0 + u1 * u1 + u2 * u2 <= 1.0) acc += e[15];
        }
      }
  out[((long long)iz * ny + iy) * nx + ix] = (float)(acc / ((double)ss * ss * ss));
}

}  // namespace lct

using namespace lct;

LCT_API int lct_voxelise(const double* d_ellipsoids, int n_ellipsoids, int nx, int ny, int nz,
                         double x0, double y0, double z0, double dx, double dy, double dz, int ss,
                         float* d_out, lct_stream stream) {
  if (!d_ellipsoids || n_ellipsoids < 0 || n_ellipsoids > kSimMaxEllipsoids || !d_out) return LCT_ERR_ARG;
  if (nx <= 0 || ny <= 0 || nz <= 0 || ny > 65535 || nz > 65535 || ss <= 0 || ss > 16) return LCT_ERR_ARG;
  dim3 grid((nx + 127) / 128, ny, nz);
  voxelise_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(d_ellipsoids, n_ellipsoids, nx, ny, x0,
                                                          y0, z0, dx, dy, dz, ss, d_out);
  return launch_status();
}

LCT_API int lct_sim_project(const double* d_ellipsoids, int n_ellipsoids, int ns, int nt,
                            float ds, float dt, float ws, float wt, float dso,
                            const double* d_angles, const double* d_zpos, int64_t v0, int64_t v1,
                            double i0, uint64_t seed, float* d_fan, lct_stream stream) {
  if (!d_ellipsoids || n_ellipsoids < 0 || n_ellipsoids > kSimMaxEllipsoids) return LCT_ERR_ARG;
  if (ns <= 0 || nt <= 0 || !d_angles || !d_zpos || !d_fan || v1 < v0 || v0 < 0) return LCT_ERR_ARG;
  if (!(ds > 0.f) || !(dt > 0.f) || !(dso > 0.f)) return LCT_ERR_ARG;
  const long long nv = v1 - v0;
  cudaStream_t s = (cudaStream_t)stream;
  for (long long c = 0; c < nv; c += 65535) {
    const long long cnt = nv - c < 65535 ? nv - c : 65535;
    dim3 grid((ns + 127) / 128, nt, (unsigned)cnt);
    sim_project_kernel<<<grid, 128, 0, s>>>(d_ellipsoids, n_ellipsoids, ns, nt, ds, dt, ws, wt,
                                            dso, d_angles, d_zpos, v0 + c, i0, seed,
                                            d_fan + c * (long long)nt * ns);
    int st = launch_status();
    if (st) return st;
  }
  return LCT_OK;
}
