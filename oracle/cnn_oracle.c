/* TEST INFRASTRUCTURE ONLY: FP64 CPU restatement of the learned 2.5D residual correction
 * (forward, MSE loss, backward) used to check the GPU kernels' outputs and gradients.
 *
 * The reference has no learned part; the network is defined here and in the product's
 * cnn.cu identically:
 *   input  : 5 neighbouring slices x_k (k = 0..4 <-> z-2..z+2) of the plain FDK volume, scaled by
 *            k_in (= calibration x input scale, one float) -> a_0[k] = q(k_in * x_k) in FP32,
 *            channels 5..31 zero
 *   layers : l = 0..7, 3x3 convolution (zero outside the image), cin = 5,32,...,32,
 *            cout = 32,...,32,1;  a_{l+1} = q(relu(b_l + W_l * a_l)) for l < 7;
 *            r = b_7 + W_7 * a_7 (one channel)
 *   output : y = k_in * x_2 + r (the residual correction, in network units)
 *   loss   : L = mean_p (y - s t)^2 for a target slice t (phantom units), s = input scale
 * q() is round-to-nearest-even to bfloat16 when bf16 != 0 (the storage points of the GPU
 * path: input activations, weights, hidden activations, backward deltas) and the identity when
 * bf16 == 0 (pure FP64, used for finite-difference checks of the backward formulas).
 *
 * Parameter layout: for l = 0..7: W_l[cout][cin][3][3], then b_l[cout].
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define CNN_L 8
#define CNN_C 32

static const int kCin[CNN_L] = {5, 32, 32, 32, 32, 32, 32, 32};
static const int kCout[CNN_L] = {32, 32, 32, 32, 32, 32, 32, 1};

int orc_cnn_param_count(void) {
  int n = 0;
  for (int l = 0; l < CNN_L; ++l) n += kCin[l] * kCout[l] * 9 + kCout[l];
  return n;
}

static int param_off(int l) {
  int n = 0;
  for (int j = 0; j < l; ++j) n += kCin[j] * kCout[j] * 9 + kCout[j];
  return n;
}

/* round-to-nearest-even to bfloat16 (finite inputs), returned as a double */
static double bf16q(double v) {
  float f = (float)v;
  uint32_t u;
  memcpy(&u, &f, 4);
  u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
  memcpy(&f, &u, 4);
  return (double)f;
}

#define Q(v) (bf16 ? bf16q(v) : (v))

/* act [B][H][W][32] */
static void conv_fwd(const double* w, const double* bias, int cin, int cout, const double* in,
                     int B, int H, int W, double* out) {
#pragma omp parallel for schedule(static)
  for (long p = 0; p < (long)B * H * W; ++p) {
    int b = (int)(p / ((long)H * W)), y = (int)(p / W % H), x = (int)(p % W);
    for (int co = 0; co < cout; ++co) {
      double acc = bias[co];
      for (int ky = 0; ky < 3; ++ky) {
        int yy = y + ky - 1;
        if (yy < 0 || yy >= H) continue;
        for (int kx = 0; kx < 3; ++kx) {
          int xx = x + kx - 1;
          if (xx < 0 || xx >= W) continue;
          const double* a = in + (((long)b * H + yy) * W + xx) * CNN_C;
          const double* wk = w + (long)co * cin * 9 + ky * 3 + kx;
          for (int ci = 0; ci < cin; ++ci) acc += wk[ci * 9] * a[ci];
        }
      }
      out[p * CNN_C + co] = acc;
    }
  }
}

/* forward; acts (optional) receives a_0..a_7 [8][B][H][W][32]; r_out [B][H][W] */
static void forward(const double* params, const float* in5, int B, int H, int W, float k_in,
                    int bf16, double* acts, double* r_out) {
  const long n = (long)B * H * W;
  double* wq = (double*)malloc(sizeof(double) * orc_cnn_param_count());
  for (int i = 0; i < orc_cnn_param_count(); ++i) wq[i] = params[i];
  for (int l = 0; l < CNN_L; ++l) {
    double* w = wq + param_off(l);
    for (int i = 0; i < kCin[l] * kCout[l] * 9; ++i) w[i] = Q(w[i]);
  }
  double* a = acts;
  for (long p = 0; p < n; ++p) {
    int b = (int)(p / ((long)H * W));
    long pix = p % ((long)H * W);
    for (int c = 0; c < CNN_C; ++c) {
      double v = 0.0;
      if (c < 5) {
        float f = k_in * in5[((long)b * 5 + c) * H * W + pix]; /* FP32 product, as on the GPU */
        v = Q((double)f);
      }
      a[p * CNN_C + c] = v;
    }
  }
  double* z = (double*)malloc(sizeof(double) * n * CNN_C);
  for (int l = 0; l < CNN_L; ++l) {
    const double* w = wq + param_off(l);
    const double* bias = w + kCin[l] * kCout[l] * 9;
    conv_fwd(w, bias, kCin[l], kCout[l], acts + (long)l * n * CNN_C, B, H, W, z);
    if (l < CNN_L - 1) {
      double* nxt = acts + (long)(l + 1) * n * CNN_C;
      for (long i = 0; i < n * CNN_C; ++i) nxt[i] = Q(z[i] > 0.0 ? z[i] : 0.0);
    } else {
      for (long p = 0; p < n; ++p) r_out[p] = z[p * CNN_C];
    }
  }
  free(z);
  free(wq);
}

void orc_cnn_forward(const double* params, const float* in5, int B, int H, int W, float k_in,
                     int bf16, double* r_out) {
  const long n = (long)B * H * W;
  double* acts = (double*)malloc(sizeof(double) * CNN_L * n * CNN_C);
  forward(params, in5, B, H, W, k_in, bf16, acts, r_out);
  free(acts);
}

/* loss and its gradient with respect to the parameters (straight through the weight rounding) */
double orc_cnn_loss_grad(const double* params, const float* in5, const float* target, int B,
                         int H, int W, float k_in, float s, int bf16, double* grad) {
  const long n = (long)B * H * W;
  const int np = orc_cnn_param_count();
  double* acts = (double*)malloc(sizeof(double) * CNN_L * n * CNN_C);
  double* r = (double*)malloc(sizeof(double) * n);
  forward(params, in5, B, H, W, k_in, bf16, acts, r);
  double* wq = (double*)malloc(sizeof(double) * np);
  for (int i = 0; i < np; ++i) wq[i] = params[i];
  for (int l = 0; l < CNN_L; ++l) {
    double* w = wq + param_off(l);
    for (int i = 0; i < kCin[l] * kCout[l] * 9; ++i) w[i] = Q(w[i]);
  }
  double loss = 0.0;
  double* dz = (double*)calloc((size_t)n * CNN_C, sizeof(double));
  double* da = (double*)malloc(sizeof(double) * n * CNN_C);
  for (long p = 0; p < n; ++p) {
    int b = (int)(p / ((long)H * W));
    long pix = p % ((long)H * W);
    double xc = (double)(float)(k_in * in5[((long)b * 5 + 2) * H * W + pix]);
    double d = xc + r[p] - (double)s * (double)target[p];
    loss += d * d;
    dz[p * CNN_C] = Q(2.0 * d / (double)n);
  }
  loss /= (double)n;
  memset(grad, 0, sizeof(double) * np);
  for (int l = CNN_L - 1; l >= 0; --l) {
    const int cin = kCin[l], cout = kCout[l];
    const double* a = acts + (long)l * n * CNN_C;
    const double* w = wq + param_off(l);
    double* gw = grad + param_off(l);
    double* gb = gw + cin * cout * 9;
    /* weight and bias gradients */
#pragma omp parallel for schedule(dynamic, 1)
    for (int co = 0; co < cout; ++co) {
      double sb = 0.0;
      for (long p = 0; p < n; ++p) sb += dz[p * CNN_C + co];
      gb[co] = sb;
      for (int ci = 0; ci < cin; ++ci)
        for (int ky = 0; ky < 3; ++ky)
          for (int kx = 0; kx < 3; ++kx) {
            double acc = 0.0;
            for (long p = 0; p < n; ++p) {
              int b = (int)(p / ((long)H * W)), y = (int)(p / W % H), x = (int)(p % W);
              int yy = y + ky - 1, xx = x + kx - 1;
              if (yy < 0 || yy >= H || xx < 0 || xx >= W) continue;
              acc += dz[p * CNN_C + co] * a[(((long)b * H + yy) * W + xx) * CNN_C + ci];
            }
            gw[((long)co * cin + ci) * 9 + ky * 3 + kx] = acc;
          }
    }
    if (l == 0) break;
    /* delta of the previous layer: transposed convolution, then the ReLU mask */
#pragma omp parallel for schedule(static)
    for (long p = 0; p < n; ++p) {
      int b = (int)(p / ((long)H * W)), y = (int)(p / W % H), x = (int)(p % W);
      for (int ci = 0; ci < CNN_C; ++ci) {
        double acc = 0.0;
        if (ci < cin)
          for (int ky = 0; ky < 3; ++ky) {
            int yy = y - (ky - 1);
            if (yy < 0 || yy >= H) continue;
            for (int kx = 0; kx < 3; ++kx) {
              int xx = x - (kx - 1);
              if (xx < 0 || xx >= W) continue;
              const double* d = dz + (((long)b * H + yy) * W + xx) * CNN_C;
              for (int co = 0; co < cout; ++co)
                acc += w[((long)co * cin + ci) * 9 + ky * 3 + kx] * d[co];
            }
          }
        da[p * CNN_C + ci] = acc;
      }
    }
    for (long i = 0; i < n * CNN_C; ++i) dz[i] = a[i] > 0.0 ? Q(da[i]) : 0.0;
  }
  free(da);
  free(dz);
  free(wq);
  free(r);
  free(acts);
  return loss;
}
