/*
 * fdk_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's helical cone-beam FDK hot path, used as the checker for
 * the CUDA path (tests/, __graft_entry__.smoke) and as the timed CPU baseline (bench.py).
 * Nothing on the product path links, loads or calls this file.
 *
 * Every function restates one reference kernel formula for formula, and cites it.  Two
 * interpolation modes:
 *
 *   ORC_EXACT   -- the same formulas evaluated in FP64 (coordinates, weights, sums): the
 *                  "FP64 re-execution" every result is reported against.
 *   ORC_TEXEMU  -- the reference's FP32 coordinate arithmetic, in its order, followed by an
 *                  emulation of the hardware linear texture filter: x_B = x - 0.5,
 *                  i = floor(x_B), weight = frac(x_B) held with 8 fractional bits (the
 *                  linear-filtering rule of the CUDA C++ Programming Guide, "Texture
 *                  Fetching").  The weight rounding rule is a setting (orc_set_tex_quant) that
 *                  the GPU tests pin against the texture hardware.  Sums are FP64.
 *
 * Addressing: ORC_BORDER (texels outside the array read 0) or ORC_CLAMP (edge texel).
 *
 * The f32 entry points (suffix _f32) run the same loops in single precision with exact
 * weights; they exist only to time a CPU execution of the reference formulas.
 *
 * Parity of this file is pinned by tests against (a) the reference's own host code built
 * from its sources (planner, taps) and (b) golden outputs of the reference's own CUDA path
 * built from its sources and run on a B200 (tests/golden/).
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
/* Include/Common.h:3 -- a double literal */
#define REF_PI 3.141592653589793238462643383

typedef struct orc_geom { /* CTGeom, Include/DataStructs.h:15-28 */
  float orbit, orbit_start;
  int ns, nt;
  float ws, wt;
  int n_angle, n_angle_add;
  float ds, dt;
  float pitch;
  float source_z0;
  float dso;
  int n_proj_turn;
  int z_dir;
  int add_projections;
} orc_geom;

typedef struct orc_img { /* ImgGeom, Include/DataStructs.h:109-115 */
  int nx, ny, nz;
  float wx, wy, wz;
  float dx, dy, dz;
} orc_img;

enum { ORC_EXACT = 0, ORC_TEXEMU = 1 };
enum { ORC_BORDER = 0, ORC_CLAMP = 1 };
enum { ORC_Q_NEAREST = 0, ORC_Q_TRUNC = 1 };

static int g_tex_quant = ORC_Q_NEAREST;
void orc_set_tex_quant(int q) { g_tex_quant = q; }
int orc_get_tex_quant(void) { return g_tex_quant; }

int orc_num_threads(void) { return omp_get_max_threads(); }
void orc_set_num_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
}

/* ----------------------------------------------------------------------------------------
 * texture-fetch emulation
 * -------------------------------------------------------------------------------------- */
static inline double q8(double a) {
  if (g_tex_quant == ORC_Q_TRUNC) return floor(a * 256.0) / 256.0;
  return floor(a * 256.0 + 0.5) / 256.0;
}

/* one axis of linear filtering at texture coordinate c (texel centres at i + 0.5) */
static inline void lin_axis(double c, int interp, long* i0, double* w) {
  double xb = c - 0.5;
  double f = floor(xb);
  *i0 = (long)f;
  double a = xb - f;
  *w = (interp == ORC_TEXEMU) ? q8(a) : a;
}

static inline double texel3(const float* v, long nx, long ny, long nz, long i, long j, long k,
                            int addr) {
  if (addr == ORC_CLAMP) {
    i = i < 0 ? 0 : (i >= nx ? nx - 1 : i);
    j = j < 0 ? 0 : (j >= ny ? ny - 1 : j);
    k = k < 0 ? 0 : (k >= nz ? nz - 1 : k);
  } else if (i < 0 || i >= nx || j < 0 || j >= ny || k < 0 || k >= nz) {
    return 0.0;
  }
  return (double)v[(k * ny + j) * nx + i];
}

/* tex3D with cudaFilterModeLinear, unnormalised coordinates.
   TEXEMU corner weights in the (x, y) plane follow the rule measured on the B200 texture unit
   (tests/golden/tex_hw.npz): a = q8(frac x), b = q8(frac y), w11 = round-half-up(a*b) on the
   1/256 grid, w01 = a - w11, w10 = b - w11, w00 = 1 - a - b + w11.  It is exact for every
   sample the reference takes (one axis off-centre in the rebin, x and y off-centre with z at a
   texel centre in the backprojection); with all three axes off-centre the two z slices are
   combined with the q8 z weight, which the hardware matches to within 1/256. */
static double tex3d_lin(const float* v, long nx, long ny, long nz, double x, double y, double z,
                        int interp, int addr) {
  long i, j, k;
  double a, b, c;
  lin_axis(x, interp, &i, &a);
  lin_axis(y, interp, &j, &b);
  lin_axis(z, interp, &k, &c);
  double wxy[2][2];
  if (interp == ORC_TEXEMU) {
    wxy[1][1] = floor(a * b * 256.0 + 0.5) / 256.0;
    wxy[0][1] = a - wxy[1][1];
    wxy[1][0] = b - wxy[1][1];
    wxy[0][0] = 1.0 - a - b + wxy[1][1];
  } else {
    wxy[0][0] = (1.0 - a) * (1.0 - b);
    wxy[0][1] = a * (1.0 - b);
    wxy[1][0] = (1.0 - a) * b;
    wxy[1][1] = a * b;
  }
  double s = 0.0;
  for (int dk = 0; dk < 2; ++dk) {
    double wk = dk ? c : 1.0 - c;
    if (wk == 0.0) continue;
    for (int dj = 0; dj < 2; ++dj)
      for (int di = 0; di < 2; ++di) {
        double w = wk * wxy[dj][di];
        if (w == 0.0) continue;
        s += w * texel3(v, nx, ny, nz, i + di, j + dj, k + dk, addr);
      }
  }
  return s;
}

/* raw sampler, exposed so tests can compare it with the texture hardware */
void orc_tex3d_sample(const float* v, int nx, int ny, int nz, const float* coords, long n,
                      int interp, int addr, double* out) {
#pragma omp parallel for schedule(static)
  for (long q = 0; q < n; ++q)
    out[q] = tex3d_lin(v, nx, ny, nz, coords[3 * q], coords[3 * q + 1], coords[3 * q + 2],
                       interp, addr);
}

/* ----------------------------------------------------------------------------------------
 * Rebin: fan -> parallel (CUDA/Rebiner.cu:82-103), null (:13-29), PI-original (:156-179)
 * -------------------------------------------------------------------------------------- */

/* view-axis texture coordinate of rebinned (ia, is); CUDA/Rebiner.cu:92-100 */
static inline double fan2par_coord(const orc_geom* g, int ia, int is, int interp) {
  if (interp == ORC_TEXEMU) {
    float ss = ((float)is - g->ws) * g->ds;
    float alpha = ss / g->dso;
    float beta_idx = (float)ia + alpha / g->orbit;
    float cz = (beta_idx + (float)g->add_projections) + 0.5f;
    return (double)cz;
  }
  double ss = ((double)is - (double)g->ws) * (double)g->ds;
  double alpha = ss / (double)g->dso;
  double beta_idx = (double)ia + alpha / (double)g->orbit;
  return beta_idx + (double)g->add_projections + 0.5;
}

/* Integer view index and weight the rebin uses for (ia, is); tests compare them bit for bit
   with the CUDA kernel's. */
void orc_rebin_fan2par_index(const orc_geom* g, int interp, int32_t* idx, float* w) {
#pragma omp parallel for schedule(static)
  for (int ia = 0; ia < g->n_angle; ++ia)
    for (int is = 0; is < g->ns; ++is) {
      long i0;
      double a;
      lin_axis(fan2par_coord(g, ia, is, interp), interp, &i0, &a);
      idx[(long)ia * g->ns + is] = (int32_t)i0;
      w[(long)ia * g->ns + is] = (float)a;
    }
}

/* fan [n_angle_add][nt][ns] -> out [n_angle][nt][ns] */
void orc_rebin_fan2par(const orc_geom* g, const float* fan, double* out, int interp, int addr) {
  const long ns = g->ns, nt = g->nt, na = g->n_angle_add;
#pragma omp parallel for schedule(static)
  for (int ia = 0; ia < g->n_angle; ++ia)
    for (int is = 0; is < g->ns; ++is) {
      long i0;
      double a;
      lin_axis(fan2par_coord(g, ia, is, interp), interp, &i0, &a);
      for (int it = 0; it < g->nt; ++it) {
        double v0 = texel3(fan, ns, nt, na, is, it, i0, addr);
        double v1 = texel3(fan, ns, nt, na, is, it, i0 + 1, addr);
        out[((long)ia * nt + it) * ns + is] = (1.0 - a) * v0 + a * v1;
      }
    }
}

/* CUDA/Rebiner.cu:13-29: par[ia][it][is] = fan[ia + add][it][is] */
void orc_rebin_null(const orc_geom* g, const float* fan, double* out, int addr) {
  const long ns = g->ns, nt = g->nt, na = g->n_angle_add;
#pragma omp parallel for schedule(static)
  for (int ia = 0; ia < g->n_angle; ++ia)
    for (int it = 0; it < g->nt; ++it)
      for (int is = 0; is < g->ns; ++is)
        out[((long)ia * nt + it) * ns + is] =
            texel3(fan, ns, nt, na, is, it, (long)ia + g->add_projections, addr);
}

/* CUDA/Rebiner.cu:156-179, trilinear resample to the PI-original row geometry */
void orc_rebin_pi_ori(const orc_geom* g, const float* fan, double* out, int interp, int addr) {
  const long ns = g->ns, nt = g->nt, na = g->n_angle_add;
#pragma omp parallel for schedule(static)
  for (int ia = 0; ia < g->n_angle; ++ia)
    for (int it = 0; it < g->nt; ++it)
      for (int is = 0; is < g->ns; ++is) {
        double x, y, z;
        if (interp == ORC_TEXEMU) {
          float s = ((float)is - g->ws) * g->ds;
          float gamma = asinf(s / g->dso);
          float pidx = gamma * g->dso / g->ds + g->ws;
          double num = (double)(((float)it - g->wt) * g->pitch / (float)(2 * (g->nt - 1))) -
                       (double)(gamma * g->pitch) / (2 * REF_PI);
          float q = (float)(num / (double)cosf(gamma));
          float qidx = q / g->dt + g->wt;
          float bidx = (float)ia + gamma / g->orbit + (float)g->add_projections;
          x = (double)(pidx + 0.5f);
          y = (double)(qidx + 0.5f);
          z = (double)(bidx + 0.5f);
        } else {
          double s = ((double)is - g->ws) * (double)g->ds;
          double gamma = asin(s / g->dso);
          double pidx = gamma * g->dso / g->ds + g->ws;
          double q = (((double)it - g->wt) * g->pitch / (2.0 * (g->nt - 1)) -
                      gamma * g->pitch / (2 * M_PI)) /
                     cos(gamma);
          double qidx = q / g->dt + g->wt;
          double bidx = (double)ia + gamma / g->orbit + g->add_projections;
          x = pidx + 0.5;
          y = qidx + 0.5;
          z = bidx + 0.5;
        }
        out[((long)ia * nt + it) * ns + is] = tex3d_lin(fan, ns, nt, na, x, y, z, interp, addr);
      }
}

/* The texture coordinates CUDA/Rebiner.cu:156-179 samples at (its FP32 expressions, as the TEXEMU
   branch above), [n_angle][nt][ns][3] = (x, y, z): the texture unit sampled at these is the
   hardware reference for the TEX8 PI-original rebin. */
void orc_rebin_pi_ori_coords(const orc_geom* g, float* xyz) {
  const long ns = g->ns, nt = g->nt;
#pragma omp parallel for schedule(static)
  for (int ia = 0; ia < g->n_angle; ++ia)
    for (int it = 0; it < g->nt; ++it)
      for (int is = 0; is < g->ns; ++is) {
        float s = ((float)is - g->ws) * g->ds;
        float gamma = asinf(s / g->dso);
        float pidx = gamma * g->dso / g->ds + g->ws;
        double num = (double)(((float)it - g->wt) * g->pitch / (float)(2 * (g->nt - 1))) -
                     (double)(gamma * g->pitch) / (2 * REF_PI);
        float q = (float)(num / (double)cosf(gamma));
        float qidx = q / g->dt + g->wt;
        float bidx = (float)ia + gamma / g->orbit + (float)g->add_projections;
        float* o = xyz + 3 * (((long)ia * nt + it) * ns + is);
        o[0] = pidx + 0.5f;
        o[1] = qidx + 0.5f;
        o[2] = bidx + 0.5f;
      }
}

/* CUDA/PreWeighting.cu:8-29, in place, [n_angle][nt][ns] */
void orc_weight_pi_ori(const orc_geom* g, double* proj) {
  const long ns = g->ns, nt = g->nt;
#pragma omp parallel for schedule(static)
  for (int ia = 0; ia < g->n_angle; ++ia)
    for (int it = 0; it < g->nt; ++it)
      for (int is = 0; is < g->ns; ++is) {
        double s = ((double)is - g->ws) * (double)g->ds;
        double t = ((double)it - g->wt) * g->pitch / (2.0 * g->nt);
        double gamma = asin(s / g->dso);
        double temp = (double)g->dso * g->dso - s * s;
        double temp2 = t - gamma * g->pitch / (2 * M_PI);
        double w = sqrt(temp) / sqrt(temp + temp2 * temp2);
        proj[((long)ia * nt + it) * ns + is] *= w;
      }
}

/* ----------------------------------------------------------------------------------------
 * Filter: taps (Src/Filter.cpp:8-20) and row convolution (CUDA/Filter.cu:10-50)
 * -------------------------------------------------------------------------------------- */
void orc_ramp_taps(int ns, float ds, float* h) {
  for (int i = 0; i < 2 * ns; ++i) {
    int n = i - ns;
    if (n == 0)
      h[i] = (float)(0.25 / ds);
    else
      h[i] = (float)((sin(n * REF_PI) / (n * REF_PI) + (cos(n * REF_PI) - 1) / (n * n * REF_PI * REF_PI)) /
                     (2 * ds));
  }
}

/* Shepp-Logan kernel with the reference's scaling (its Ram-Lak taps carry the ds factor of the
   discrete sum): h(n) = -2 / (pi^2 ds (4 n^2 - 1)), Shepp & Logan (1974); Kak & Slaney,
   "Principles of Computerized Tomographic Imaging", ch. 3. */
void orc_shepp_logan_taps(int ns, float ds, float* h) {
  for (int i = 0; i < 2 * ns; ++i) {
    double n = (double)(i - ns);
    h[i] = (float)(-2.0 / (M_PI * M_PI * (double)ds * (4.0 * n * n - 1.0)));
  }
}

/* out[r][is] = sum_{k<ns} h[is - k + ns] * in[r][k]
   mode 0: FP64 accumulation; mode 1: FP32 fused multiply-add in increasing k, the order of
   CUDA/Filter.cu:42-46 (bit-exact with that kernel). */
void orc_filter_rows(const float* h, int ns, const float* in, double* out, long nrows, int mode) {
#pragma omp parallel for schedule(static)
  for (long r = 0; r < nrows; ++r) {
    const float* row = in + r * ns;
    for (int is = 0; is < ns; ++is) {
      if (mode == 1) {
        float acc = 0.0f;
        for (int k = 0; k < ns; ++k) acc = fmaf(h[is - k + ns], row[k], acc);
        out[r * ns + is] = acc;
      } else {
        double acc = 0.0;
        for (int k = 0; k < ns; ++k) acc += (double)h[is - k + ns] * (double)row[k];
        out[r * ns + is] = acc;
      }
    }
  }
}

/* ----------------------------------------------------------------------------------------
 * Backprojection, rebinned parallel helical (CUDA/Backprojector.cu:12-99)
 * -------------------------------------------------------------------------------------- */

/* view window of slice iz: CUDA/Backprojector.cu:37-42 (always FP32, as in the reference) */
void orc_bp_window(const orc_geom* g, const orc_img* ig, int iz, float dz_per_view, int na1_half,
                   int* a_min, int* a_max) {
  float zc = ((float)iz - ig->wz) * ig->dz;
  int a_middle = (int)roundf((zc - g->source_z0) / dz_per_view);
  a_middle = a_middle < 0 ? 0 : a_middle;
  a_middle = a_middle > g->n_angle - 1 ? g->n_angle - 1 : a_middle;
  int lo = (a_middle - na1_half >= 0) ? (a_middle - na1_half) : 0;
  int hi = (a_middle + na1_half < g->n_angle) ? (a_middle + na1_half) : g->n_angle - 1;
  *a_min = lo;
  *a_max = hi;
}

/* proj [n_angle][nt][ns] (filtered), betas[n_angle]; img [nz][ny][nx].
   A conjugate view past the last one (possible only for clamped windows) samples outside the
   array; its angle is taken from the last view so no read leaves betas[n_angle] (the
   reference reads past the copied angles there).
   Voxel rows [y0, y1) only (the CPU baseline times a bounded sample). */
void orc_bp_par_rows(const orc_geom* g, const orc_img* ig, const float* betas, const float* proj,
                     double* img, int interp, int addr, int y0, int y1) {
  const long ns = g->ns, nt = g->nt, na = g->n_angle;
  const int na1_half = g->n_proj_turn / 2;                       /* Backprojector.cu:148 */
  const float dzv = g->pitch / (float)g->n_proj_turn;            /* Backprojector.cu:149 */
  const int nyz = (y1 - y0) * ig->nz;
#pragma omp parallel for schedule(dynamic, 1)
  for (int q = 0; q < nyz; ++q) {
    int iz = q / (y1 - y0), iy = y0 + q % (y1 - y0);
    int a_min, a_max;
    orc_bp_window(g, ig, iz, dzv, na1_half, &a_min, &a_max);
    for (int ix = 0; ix < ig->nx; ++ix) {
      double sum = 0.0;
      if (interp == ORC_TEXEMU) {
        float xc = ((float)ix - ig->wx) * ig->dx;
        float yc = ((float)iy - ig->wy) * ig->dy;
        float zc = ((float)iz - ig->wz) * ig->dz;
        for (int ia = a_min; ia < a_max; ++ia) {
          float beta = betas[ia];
          int ia2 = ia + na1_half < a_max ? ia + na1_half : ia - na1_half;
          ia2 = ia2 < 0 ? ia + na1_half : ia2;
          float beta2 = betas[ia2 < g->n_angle ? ia2 : g->n_angle - 1];
          float cb = (float)cos((double)beta), sb = (float)sin((double)beta);
          float cb2 = (float)cos((double)beta2), sb2 = (float)sin((double)beta2);
          float phat = -xc * cb - yc * sb;
          float theta = asinf(phat / g->dso);
          float delta_p = theta * g->dso / g->ds;
          float p_idx = delta_p + g->ws;
          float p_idx2 = -delta_p + g->ws;
          float z_ray = g->source_z0 + ((float)ia + theta / g->orbit) * dzv;
          float z_ray2 = g->source_z0 + ((float)ia2 - theta / g->orbit) * dzv;
          float sq = sqrtf(g->dso * g->dso - phat * phat);
          float lhat = sq + xc * sb - yc * cb;
          float lhat2 = sq + xc * sb2 - yc * cb2;
          float qhat = (zc - z_ray) * g->dso * (float)g->z_dir / (lhat * g->dt);
          float qhat2 = (zc - z_ray2) * g->dso * (float)g->z_dir / (lhat2 * g->dt);
          float q_idx = qhat + g->wt, q_idx2 = qhat2 + g->wt;
          float ww, ww2;
          if (fabsf(qhat) > g->wt) {
            ww = 0.0f;
            ww2 = 1.0f;
          } else if (fabsf(qhat2) > g->wt) {
            ww = 1.0f;
            ww2 = 0.0f;
          } else {
            ww = -qhat2 / (qhat - qhat2);
            ww2 = qhat / (qhat - qhat2);
          }
          double s1 = tex3d_lin(proj, ns, nt, na, (double)(p_idx + 0.5f), (double)(q_idx + 0.5f),
                                (double)((float)ia + 0.5f), interp, addr);
          double s2 = tex3d_lin(proj, ns, nt, na, (double)(p_idx2 + 0.5f),
                                (double)(q_idx2 + 0.5f), (double)((float)ia2 + 0.5f), interp,
                                addr);
          sum += s1 * ww + s2 * ww2;
        }
      } else {
        double xc = ((double)ix - ig->wx) * ig->dx;
        double yc = ((double)iy - ig->wy) * ig->dy;
        double zc = ((double)iz - ig->wz) * ig->dz;
        double dso = g->dso, ds = g->ds, dt = g->dt, wt = g->wt, orbit = g->orbit;
        double dzvd = (double)g->pitch / (double)g->n_proj_turn;
        for (int ia = a_min; ia < a_max; ++ia) {
          double beta = betas[ia];
          int ia2 = ia + na1_half < a_max ? ia + na1_half : ia - na1_half;
          ia2 = ia2 < 0 ? ia + na1_half : ia2;
          double beta2 = betas[ia2 < g->n_angle ? ia2 : g->n_angle - 1];
          double phat = -xc * cos(beta) - yc * sin(beta);
          double theta = asin(phat / dso);
          double delta_p = theta * dso / ds;
          double p_idx = delta_p + g->ws, p_idx2 = -delta_p + g->ws;
          double z_ray = g->source_z0 + (ia + theta / orbit) * dzvd;
          double z_ray2 = g->source_z0 + (ia2 - theta / orbit) * dzvd;
          double sq = sqrt(dso * dso - phat * phat);
          double lhat = sq + xc * sin(beta) - yc * cos(beta);
          double lhat2 = sq + xc * sin(beta2) - yc * cos(beta2);
          double qhat = (zc - z_ray) * dso * g->z_dir / (lhat * dt);
          double qhat2 = (zc - z_ray2) * dso * g->z_dir / (lhat2 * dt);
          double ww, ww2;
          if (fabs(qhat) > wt) {
            ww = 0.0;
            ww2 = 1.0;
          } else if (fabs(qhat2) > wt) {
            ww = 1.0;
            ww2 = 0.0;
          } else {
            ww = -qhat2 / (qhat - qhat2);
            ww2 = qhat / (qhat - qhat2);
          }
          double s1 = tex3d_lin(proj, ns, nt, na, p_idx + 0.5, qhat + wt + 0.5, ia + 0.5,
                                ORC_EXACT, addr);
          double s2 = tex3d_lin(proj, ns, nt, na, p_idx2 + 0.5, qhat2 + wt + 0.5, ia2 + 0.5,
                                ORC_EXACT, addr);
          sum += s1 * ww + s2 * ww2;
        }
      }
      /* Backprojector.cu:96 -- evaluated in double because PI is a double literal */
      img[((long)iz * ig->ny + iy) * ig->nx + ix] =
          (a_max > a_min) ? sum * 2.0 * REF_PI / (double)(float)(a_max - a_min) : 0.0;
    }
  }
}

void orc_bp_par(const orc_geom* g, const orc_img* ig, const float* betas, const float* proj,
                double* img, int interp, int addr) {
  orc_bp_par_rows(g, ig, betas, proj, img, interp, addr, 0, ig->ny);
}

/* tex3d_lin at a view-axis coordinate on a texel centre (z = ia + 0.5, so the z weight is 0
   and only layer k contributes): the same operations in the same order as tex3d_lin, without
   its loop over the second layer. */
static inline double tex_layer(const float* v, long nx, long ny, long nz, double x, double y,
                               long k, int interp, int addr) {
  long i, j;
  double a, b;
  lin_axis(x, interp, &i, &a);
  lin_axis(y, interp, &j, &b);
  double w[4];
  if (interp == ORC_TEXEMU) {
    w[3] = floor(a * b * 256.0 + 0.5) / 256.0;
    w[1] = a - w[3];
    w[2] = b - w[3];
    w[0] = 1.0 - a - b + w[3];
  } else {
    w[0] = (1.0 - a) * (1.0 - b);
    w[1] = a * (1.0 - b);
    w[2] = (1.0 - a) * b;
    w[3] = a * b;
  }
  double s = 0.0;
  for (int c = 0; c < 4; ++c) {
    double wc = 1.0 * w[c];
    if (wc == 0.0) continue;
    s += wc * texel3(v, nx, ny, nz, i + (c & 1), j + (c >> 1), k, addr);
  }
  return s;
}

/* orc_bp_par_rows with the loops interchanged: per voxel row iy, views ia outermost, then the
   row's voxel columns, then every slice whose window holds ia.  The z-invariant terms are
   evaluated once per (column, view) instead of once per (voxel, view) and a view's samples stay
   in cache across the row; each voxel still sums its views in increasing ia with the same
   expressions, so the result is bit-identical to orc_bp_par_rows (pinned by
   tests/test_oracle_kat.py) and several times faster, which makes whole-slab FP64 checks of
   full-size volumes practical.  cos/sin of every view angle come from tables evaluated with the
   same libm calls.  Rows y0, y0 + ystep, ... below y1 are computed; the others are left as they
   are in img. */
void orc_bp_par_cols(const orc_geom* g, const orc_img* ig, const float* betas, const float* proj,
                     double* img, int interp, int addr, int y0, int y1, int ystep) {
  const long ns = g->ns, nt = g->nt, na = g->n_angle;
  const int na1_half = g->n_proj_turn / 2;                       /* Backprojector.cu:148 */
  const float dzv = g->pitch / (float)g->n_proj_turn;            /* Backprojector.cu:149 */
  const int nz = ig->nz, nx = ig->nx;
  int* amin = (int*)malloc(sizeof(int) * (size_t)(nz > 0 ? nz : 1));
  int* amax = (int*)malloc(sizeof(int) * (size_t)(nz > 0 ? nz : 1));
  double* cosd = (double*)malloc(sizeof(double) * (size_t)(na > 0 ? na : 1));
  double* sind = (double*)malloc(sizeof(double) * (size_t)(na > 0 ? na : 1));
  int lo = (int)na, hi = 0;
  for (int iz = 0; iz < nz; ++iz) {
    orc_bp_window(g, ig, iz, dzv, na1_half, &amin[iz], &amax[iz]);
    if (amax[iz] > amin[iz]) {
      lo = amin[iz] < lo ? amin[iz] : lo;
      hi = amax[iz] > hi ? amax[iz] : hi;
    }
  }
  for (long a = 0; a < na; ++a) {
    cosd[a] = cos((double)betas[a]);
    sind[a] = sin((double)betas[a]);
  }
#pragma omp parallel
  {
    double* sum = (double*)malloc(sizeof(double) * (size_t)(nz > 0 ? nz : 1) * (size_t)nx);
    const int step = ystep > 0 ? ystep : 1;
    const int nrow = y1 > y0 ? (y1 - y0 + step - 1) / step : 0;
#pragma omp for schedule(dynamic, 1)
    for (int r = 0; r < nrow; ++r) {
      const int iy = y0 + r * step;
      for (long q = 0; q < (long)nz * nx; ++q) sum[q] = 0.0;
      for (int ia = lo; ia < hi; ++ia) {
        /* conjugate candidates: ia + half [0] and ia - half [1] (ia + half when negative) */
        const int c2[2] = {ia + na1_half, ia - na1_half < 0 ? ia + na1_half : ia - na1_half};
        const int b2[2] = {c2[0] < g->n_angle ? c2[0] : g->n_angle - 1,
                           c2[1] < g->n_angle ? c2[1] : g->n_angle - 1};
        for (int ix = 0; ix < nx; ++ix) {
          double* acc = sum + (long)ix * nz;
          if (interp == ORC_TEXEMU) {
            float xc = ((float)ix - ig->wx) * ig->dx;
            float yc = ((float)iy - ig->wy) * ig->dy;
            float cb = (float)cosd[ia], sb = (float)sind[ia];
            float phat = -xc * cb - yc * sb;
            float theta = asinf(phat / g->dso);
            float delta_p = theta * g->dso / g->ds;
            float p_idx = delta_p + g->ws;
            float p_idx2 = -delta_p + g->ws;
            float z_ray = g->source_z0 + ((float)ia + theta / g->orbit) * dzv;
            float sq = sqrtf(g->dso * g->dso - phat * phat);
            float lhat = sq + xc * sb - yc * cb;
            float z_ray2c[2], lhat2c[2];
            for (int c = 0; c < 2; ++c) {
              float cb2 = (float)cosd[b2[c]], sb2 = (float)sind[b2[c]];
              z_ray2c[c] = g->source_z0 + ((float)c2[c] - theta / g->orbit) * dzv;
              lhat2c[c] = sq + xc * sb2 - yc * cb2;
            }
            for (int iz = 0; iz < nz; ++iz) {
              if (ia < amin[iz] || ia >= amax[iz]) continue;
              float zc = ((float)iz - ig->wz) * ig->dz;
              int ia2 = ia + na1_half < amax[iz] ? ia + na1_half : ia - na1_half;
              const int c = (ia2 < 0 || ia2 == ia + na1_half) ? 0 : 1;
              ia2 = ia2 < 0 ? ia + na1_half : ia2;
              float qhat = (zc - z_ray) * g->dso * (float)g->z_dir / (lhat * g->dt);
              float qhat2 = (zc - z_ray2c[c]) * g->dso * (float)g->z_dir / (lhat2c[c] * g->dt);
              float q_idx = qhat + g->wt, q_idx2 = qhat2 + g->wt;
              float ww, ww2;
              if (fabsf(qhat) > g->wt) {
                ww = 0.0f;
                ww2 = 1.0f;
              } else if (fabsf(qhat2) > g->wt) {
                ww = 1.0f;
                ww2 = 0.0f;
              } else {
                ww = -qhat2 / (qhat - qhat2);
                ww2 = qhat / (qhat - qhat2);
              }
              double s1 = tex_layer(proj, ns, nt, na, (double)(p_idx + 0.5f),
                                    (double)(q_idx + 0.5f), ia, interp, addr);
              double s2 = tex_layer(proj, ns, nt, na, (double)(p_idx2 + 0.5f),
                                    (double)(q_idx2 + 0.5f), ia2, interp, addr);
              acc[iz] += s1 * ww + s2 * ww2;
            }
          } else {
            double xc = ((double)ix - ig->wx) * ig->dx;
            double yc = ((double)iy - ig->wy) * ig->dy;
            double dso = g->dso, ds = g->ds, dt = g->dt, wt = g->wt, orbit = g->orbit;
            double dzvd = (double)g->pitch / (double)g->n_proj_turn;
            double phat = -xc * cosd[ia] - yc * sind[ia];
            double theta = asin(phat / dso);
            double delta_p = theta * dso / ds;
            double p_idx = delta_p + g->ws, p_idx2 = -delta_p + g->ws;
            double z_ray = g->source_z0 + (ia + theta / orbit) * dzvd;
            double sq = sqrt(dso * dso - phat * phat);
            double lhat = sq + xc * sind[ia] - yc * cosd[ia];
            double z_ray2c[2], lhat2c[2];
            for (int c = 0; c < 2; ++c) {
              z_ray2c[c] = g->source_z0 + (c2[c] - theta / orbit) * dzvd;
              lhat2c[c] = sq + xc * sind[b2[c]] - yc * cosd[b2[c]];
            }
            for (int iz = 0; iz < nz; ++iz) {
              if (ia < amin[iz] || ia >= amax[iz]) continue;
              double zc = ((double)iz - ig->wz) * ig->dz;
              int ia2 = ia + na1_half < amax[iz] ? ia + na1_half : ia - na1_half;
              const int c = (ia2 < 0 || ia2 == ia + na1_half) ? 0 : 1;
              ia2 = ia2 < 0 ? ia + na1_half : ia2;
              double qhat = (zc - z_ray) * dso * g->z_dir / (lhat * dt);
              double qhat2 = (zc - z_ray2c[c]) * dso * g->z_dir / (lhat2c[c] * dt);
              double ww, ww2;
              if (fabs(qhat) > wt) {
                ww = 0.0;
                ww2 = 1.0;
              } else if (fabs(qhat2) > wt) {
                ww = 1.0;
                ww2 = 0.0;
              } else {
                ww = -qhat2 / (qhat - qhat2);
                ww2 = qhat / (qhat - qhat2);
              }
              double s1 = tex_layer(proj, ns, nt, na, p_idx + 0.5, qhat + wt + 0.5, ia,
                                    ORC_EXACT, addr);
              double s2 = tex_layer(proj, ns, nt, na, p_idx2 + 0.5, qhat2 + wt + 0.5, ia2,
                                    ORC_EXACT, addr);
              acc[iz] += s1 * ww + s2 * ww2;
            }
          }
        }
      }
      for (int iz = 0; iz < nz; ++iz)
        for (int ix = 0; ix < nx; ++ix)
          img[((long)iz * ig->ny + iy) * nx + ix] =
              (amax[iz] > amin[iz])
                  ? sum[(long)ix * nz + iz] * 2.0 * REF_PI / (double)(float)(amax[iz] - amin[iz])
                  : 0.0;
    }
    free(sum);
  }
  free(amin);
  free(amax);
  free(cosd);
  free(sind);
}

/* CUDA/Backprojector.cu:171-250, PI-window backprojection */
void orc_bp_pi_ori(const orc_geom* g, const orc_img* ig, const float* betas, const float* proj,
                   double* img, int interp, int addr) {
  const long ns = g->ns, nt = g->nt, na = g->n_angle;
  const int na1_half = g->n_proj_turn / 2;
  const float dzv = g->pitch / (float)g->n_proj_turn;
  const int nyz = ig->ny * ig->nz;
#pragma omp parallel for schedule(dynamic, 1)
  for (int q = 0; q < nyz; ++q) {
    int iz = q / ig->ny, iy = q % ig->ny;
    for (int ix = 0; ix < ig->nx; ++ix) {
      double xc = ((double)ix - ig->wx) * ig->dx;
      double yc = ((double)iy - ig->wy) * ig->dy;
      double zc = ((double)iz - ig->wz) * ig->dz;
      float zcf = ((float)iz - ig->wz) * ig->dz;
      int a_middle = (int)roundf((zcf - g->source_z0) / dzv);
      a_middle = a_middle < 0 ? 0 : a_middle;
      a_middle = a_middle > g->n_angle - 1 ? g->n_angle - 1 : a_middle;
      double sum = 0.0;
      double temp2 = (double)g->pitch / (2 * M_PI);
      int ia;
      /* walk back while |t| <= pitch/4 (Backprojector.cu:200-222) */
      for (ia = a_middle; ia >= 0; --ia) {
        double beta = betas[ia], cb = cos(beta), sb = sin(beta);
        double s = -xc * cb - yc * sb;
        double gamma = asin(s / g->dso);
        double temp1 = sqrt((double)g->dso * g->dso - s * s);
        double zoff = zc - (g->source_z0 + (double)dzv * ia);
        double t = temp1 * (zoff - gamma * temp2) / (temp1 + xc * sb - yc * cb) + gamma * temp2;
        t *= g->z_dir;
        if (t > g->pitch / 4.0 || t < -g->pitch / 4.0) break;
        double is = s / g->ds + g->ws;
        double it = t * 2 * (g->nt - 1) / g->pitch + g->wt;
        sum += tex3d_lin(proj, ns, nt, na, is + 0.5, it + 0.5, ia + 0.5, interp, addr);
      }
      int a_min = ia;
      /* forward na1_half views (Backprojector.cu:224-245); the reference has no bound
         against n_angle here, views past the end read the border (0). */
      for (ia = a_middle + 1; ia <= a_min + na1_half; ++ia) {
        if (ia >= g->n_angle) break;
        double beta = betas[ia], cb = cos(beta), sb = sin(beta);
        double s = -xc * cb - yc * sb;
        double gamma = asin(s / g->dso);
        double temp1 = sqrt((double)g->dso * g->dso - s * s);
        double zoff = zc - (g->source_z0 + (double)dzv * ia);
        double t = temp1 * (zoff - gamma * temp2) / (temp1 + xc * sb - yc * cb) + gamma * temp2;
        t *= g->z_dir;
        double is = s / g->ds + g->ws;
        double it = t * 2 * (g->nt - 1) / g->pitch + g->wt;
        sum += tex3d_lin(proj, ns, nt, na, is + 0.5, it + 0.5, ia + 0.5, interp, addr);
      }
      img[((long)iz * ig->ny + iy) * ig->nx + ix] = sum * REF_PI / na1_half;
    }
  }
}

/* ----------------------------------------------------------------------------------------
 * FP32 restatements, timed as the CPU baseline (exact weights, border addressing).
 * -------------------------------------------------------------------------------------- */
static inline float texel3f(const float* v, long nx, long ny, long nz, long i, long j, long k) {
  if (i < 0 || i >= nx || j < 0 || j >= ny || k < 0 || k >= nz) return 0.0f;
  return v[(k * ny + j) * nx + i];
}

static inline float bilin_f32(const float* v, long nx, long ny, long nz, float x, float y,
                              long k) {
  float xb = x - 0.5f, yb = y - 0.5f;
  float fx = floorf(xb), fy = floorf(yb);
  long i = (long)fx, j = (long)fy;
  float a = xb - fx, b = yb - fy;
  return (1.0f - b) * ((1.0f - a) * texel3f(v, nx, ny, nz, i, j, k) +
                       a * texel3f(v, nx, ny, nz, i + 1, j, k)) +
         b * ((1.0f - a) * texel3f(v, nx, ny, nz, i, j + 1, k) +
              a * texel3f(v, nx, ny, nz, i + 1, j + 1, k));
}

/* CUDA/Backprojector.cu:12-99 in FP32 over voxel rows [y0, y1) of all nz slices */
void orc_bp_par_rows_f32(const orc_geom* g, const orc_img* ig, const float* betas,
                         const float* proj, float* img, int y0, int y1) {
  const long ns = g->ns, nt = g->nt, na = g->n_angle;
  const int na1_half = g->n_proj_turn / 2;
  const float dzv = g->pitch / (float)g->n_proj_turn;
  const int nyz = (y1 - y0) * ig->nz;
#pragma omp parallel for schedule(dynamic, 1)
  for (int q = 0; q < nyz; ++q) {
    int iz = q / (y1 - y0), iy = y0 + q % (y1 - y0);
    int a_min, a_max;
    orc_bp_window(g, ig, iz, dzv, na1_half, &a_min, &a_max);
    float yc = ((float)iy - ig->wy) * ig->dy;
    float zc = ((float)iz - ig->wz) * ig->dz;
    for (int ix = 0; ix < ig->nx; ++ix) {
      float xc = ((float)ix - ig->wx) * ig->dx;
      float sum = 0.0f;
      for (int ia = a_min; ia < a_max; ++ia) {
        float beta = betas[ia];
        int ia2 = ia + na1_half < a_max ? ia + na1_half : ia - na1_half;
        ia2 = ia2 < 0 ? ia + na1_half : ia2;
        float beta2 = betas[ia2 < g->n_angle ? ia2 : g->n_angle - 1];
        float cb = cosf(beta), sb = sinf(beta), cb2 = cosf(beta2), sb2 = sinf(beta2);
        float phat = -xc * cb - yc * sb;
        float theta = asinf(phat / g->dso);
        float delta_p = theta * g->dso / g->ds;
        float z_ray = g->source_z0 + ((float)ia + theta / g->orbit) * dzv;
        float z_ray2 = g->source_z0 + ((float)ia2 - theta / g->orbit) * dzv;
        float sq = sqrtf(g->dso * g->dso - phat * phat);
        float lhat = sq + xc * sb - yc * cb, lhat2 = sq + xc * sb2 - yc * cb2;
        float qhat = (zc - z_ray) * g->dso * (float)g->z_dir / (lhat * g->dt);
        float qhat2 = (zc - z_ray2) * g->dso * (float)g->z_dir / (lhat2 * g->dt);
        float ww, ww2;
        if (fabsf(qhat) > g->wt) {
          ww = 0.0f;
          ww2 = 1.0f;
        } else if (fabsf(qhat2) > g->wt) {
          ww = 1.0f;
          ww2 = 0.0f;
        } else {
          ww = -qhat2 / (qhat - qhat2);
          ww2 = qhat / (qhat - qhat2);
        }
        sum += bilin_f32(proj, ns, nt, na, delta_p + g->ws + 0.5f, qhat + g->wt + 0.5f, ia) * ww +
               bilin_f32(proj, ns, nt, na, -delta_p + g->ws + 0.5f, qhat2 + g->wt + 0.5f, ia2) *
                   ww2;
      }
      img[((long)iz * ig->ny + iy) * ig->nx + ix] =
          (float)(sum * 2.0f * REF_PI / (float)(a_max - a_min));
    }
  }
}

/* CUDA/Rebiner.cu:82-103 + CUDA/Filter.cu:10-50 in FP32, views [v0, v1) of a block */
void orc_rebin_filter_f32(const orc_geom* g, const float* fan, const float* h, float* out, int v0,
                          int v1) {
  const long ns = g->ns, nt = g->nt, na = g->n_angle_add;
#pragma omp parallel for schedule(static)
  for (int ia = v0; ia < v1; ++ia) {
    float* row = (float*)malloc(sizeof(float) * ns);
    for (int it = 0; it < g->nt; ++it) {
      for (int is = 0; is < g->ns; ++is) {
        float ss = ((float)is - g->ws) * g->ds;
        float cz = ((float)ia + (ss / g->dso) / g->orbit + (float)g->add_projections) + 0.5f;
        float zb = cz - 0.5f, fz = floorf(zb);
        float a = zb - fz;
        long k = (long)fz;
        row[is] = (1.0f - a) * texel3f(fan, ns, nt, na, is, it, k) +
                  a * texel3f(fan, ns, nt, na, is, it, k + 1);
      }
      float* o = out + ((long)(ia - v0) * nt + it) * ns;
      for (int is = 0; is < g->ns; ++is) {
        float acc = 0.0f;
        for (int k = 0; k < g->ns; ++k) acc = fmaf(h[is - k + ns], row[k], acc);
        o[is] = acc;
      }
    }
    free(row);
  }
}

/* ----------------------------------------------------------------------------------------
 * Scan simulator: seeded ellipsoid phantom, analytic helical fan-beam line integrals,
 * Poisson noise.  Geometry (recovered from the reference kernels): source at angle b and
 * couch z sits at (-R sin b, R cos b, z); detector column is has fan angle
 * a = (is - ws) ds / R; the in-plane ray direction is (sin(b - a), -cos(b - a)); detector row
 * it has iso-scaled height t = (it - wt) dt, i.e. the ray rises t / R per unit in-plane length.
 * -------------------------------------------------------------------------------------- */
typedef struct orc_ellipsoid {
  double cx, cy, cz;    /* centre, mm */
  double ax, ay, az;    /* semi-axes, mm */
  double rot[9];        /* row-major rotation, ellipsoid frame -> world */
  double mu;            /* attenuation, 1/mm */
} orc_ellipsoid;

static double ray_ellipsoids(const orc_ellipsoid* e, int ne, const double S[3], const double D[3]) {
  double dn = sqrt(D[0] * D[0] + D[1] * D[1] + D[2] * D[2]);
  double sum = 0.0;
  for (int m = 0; m < ne; ++m) {
    const double* R = e[m].rot;
    double p[3] = {S[0] - e[m].cx, S[1] - e[m].cy, S[2] - e[m].cz};
    double s[3], d[3];
    for (int r = 0; r < 3; ++r) {
      s[r] = R[0 * 3 + r] * p[0] + R[1 * 3 + r] * p[1] + R[2 * 3 + r] * p[2];
      d[r] = R[0 * 3 + r] * D[0] + R[1 * 3 + r] * D[1] + R[2 * 3 + r] * D[2];
    }
    s[0] /= e[m].ax; s[1] /= e[m].ay; s[2] /= e[m].az;
    d[0] /= e[m].ax; d[1] /= e[m].ay; d[2] /= e[m].az;
    double A = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    double B = s[0] * d[0] + s[1] * d[1] + s[2] * d[2];
    double C = s[0] * s[0] + s[1] * s[1] + s[2] * s[2] - 1.0;
    double disc = B * B - A * C;
    if (disc > 0.0) sum += e[m].mu * 2.0 * sqrt(disc) / A * dn;
  }
  return sum;
}

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
   SC'11): 10 rounds of the published round function and key schedule. */
static void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

static double noisy_integral(double p, double i0, uint64_t seed, uint64_t idx) {
  if (i0 <= 0.0) return p;
  uint32_t c[4] = {(uint32_t)idx, (uint32_t)(idx >> 32), 0x4c435430u, 0u};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  double u1 = ((double)c[0] + 0.5) * (1.0 / 4294967296.0);
  double u2 = ((double)c[1] + 0.5) * (1.0 / 4294967296.0);
  double lam = i0 * exp(-p);
  double n;
  if (lam < 30.0) { /* Knuth multiplication method, counter-based uniforms */
    double L = exp(-lam), prod = u1;
    int k = 0;
    uint32_t cc[4] = {c[2], c[3], 0x4b4e5554u, 0u};
    int j = 0;
    while (prod > L && k < 1000) {
      ++k;
      if (j == 4) {
        philox4x32_10(cc, (uint32_t)seed, (uint32_t)(seed >> 32));
        j = 0;
      }
      prod *= ((double)cc[j++] + 0.5) * (1.0 / 4294967296.0);
    }
    n = k;
  } else { /* rounded normal approximation N(lam, lam) */
    double z = sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
    n = floor(lam + sqrt(lam) * z + 0.5);
  }
  if (n < 1.0) n = 1.0;
  return -log(n / i0);
}

/* fan [nviews][nt][ns] for views [v0, v1) of a scan with angles[] (rad) and zpos[] (mm) */
void orc_sim_project(const orc_ellipsoid* e, int ne, int ns, int nt, float ds, float dt, float ws,
                     float wt, float dso, const double* angles, const double* zpos, long v0,
                     long v1, double i0, uint64_t seed, float* fan) {
#pragma omp parallel for schedule(dynamic, 1)
  for (long v = v0; v < v1; ++v) {
    double b = angles[v], z = zpos[v];
    double S[3] = {-dso * sin(b), dso * cos(b), z};
    for (int it = 0; it < nt; ++it) {
      double t = ((double)it - wt) * dt;
      for (int is = 0; is < ns; ++is) {
        double a = ((double)is - ws) * ds / dso;
        double D[3] = {sin(b - a), -cos(b - a), t / dso};
        double p = ray_ellipsoids(e, ne, S, D);
        uint64_t idx = ((uint64_t)v * nt + it) * ns + is;
        fan[((v - v0) * nt + it) * (long)ns + is] = (float)noisy_integral(p, i0, seed, idx);
      }
    }
  }
}

/* voxelised phantom: mean attenuation over ss^3 sub-samples per voxel, [nz][ny][nx] with
   voxel (ix, iy, iz) centred at (x0 + ix dx, y0 + iy dy, z0 + iz dz) */
void orc_voxelise(const orc_ellipsoid* e, int ne, int nx, int ny, int nz, double x0, double y0,
                  double z0, double dx, double dy, double dz, int ss, float* out) {
#pragma omp parallel for schedule(dynamic, 1)
  for (long q = 0; q < (long)ny * nz; ++q) {
    int iz = (int)(q / ny), iy = (int)(q % ny);
    for (int ix = 0; ix < nx; ++ix) {
      double acc = 0.0;
      for (int sz = 0; sz < ss; ++sz)
        for (int sy = 0; sy < ss; ++sy)
          for (int sx = 0; sx < ss; ++sx) {
            double P[3] = {x0 + (ix + (sx + 0.5) / ss - 0.5) * dx,
                           y0 + (iy + (sy + 0.5) / ss - 0.5) * dy,
                           z0 + (iz + (sz + 0.5) / ss - 0.5) * dz};
            for (int m = 0; m < ne; ++m) {
              const double* R = e[m].rot;
              double p[3] = {P[0] - e[m].cx, P[1] - e[m].cy, P[2] - e[m].cz};
              double u0 = (R[0] * p[0] + R[3] * p[1] + R[6] * p[2]) / e[m].ax;
              double u1 = (R[1] * p[0] + R[4] * p[1] + R[7] * p[2]) / e[m].ay;
              double u2 = (R[2] * p[0] + R[5] * p[1] + R[8] * p[2]) / e[m].az;
              if (u0 * u0 + u1 * u1 + u2 * u2 <= 1.0) acc += e[m].mu;
            }
          }
      out[((long)iz * ny + iy) * nx + ix] = (float)(acc / ((double)ss * ss * ss));
    }
  }
}
