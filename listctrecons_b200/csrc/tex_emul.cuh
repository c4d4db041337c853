// Linear-filter arithmetic of the texture hardware, done in registers.
//
// For cudaFilterModeLinear with unnormalised coordinates, a fetch at coordinate x reads texels
// i = floor(x - 0.5) and i + 1 with weight a = frac(x - 0.5) on the second, and a is held with
// 8 fractional bits (CUDA C++ Programming Guide, "Texture Fetching", linear filtering).  The
// product's TEX8 interpolation reproduces that weight; EXACT keeps the full FP32 fraction.
#pragma once

#include <cuda_runtime.h>

namespace lct {

// 8-fractional-bit weight (round to nearest, ties up), as measured on the texture unit.
__host__ __device__ __forceinline__ float q8(float a) {
  return floorf(a * 256.0f + 0.5f) * (1.0f / 256.0f);
}

// Bilinear corner weights of the texture unit, measured on B200 (tests/test_gpu_texture.py,
// fixture tests/golden/tex_hw.npz): with a = q8(frac x) and b = q8(frac y), the far corner
// gets w11 = round-half-up(a*b) on the 1/256 grid and the others follow by subtraction, so each
// axis keeps its weight exactly: w01 = a - w11, w10 = b - w11, w00 = 1 - a - b + w11.
// Every product and difference here is exact in FP32 (multiples of 2^-16).
__host__ __device__ __forceinline__ void tex_bilinear_weights(float a, float b, float& w00,
                                                              float& w01, float& w10,
                                                              float& w11) {
  w11 = floorf(a * b * 256.0f + 0.5f) * (1.0f / 256.0f);
  w01 = a - w11;
  w10 = b - w11;
  w00 = (1.0f - a - b) + w11;
}

template <int INTERP>
__device__ __forceinline__ void lin_axis(float coord, int& i, float& w) {
  // coord is a texture coordinate (texel centres at i + 0.5); coord - 0.5f is exact for
  // coord in [0.5, 2^23], the range every caller produces for in-range samples.
  float xb = __fsub_rn(coord, 0.5f);
  float f = floorf(xb);
  i = (int)f;
  float a = __fsub_rn(xb, f);
  w = (INTERP == LCT_INTERP_TEX8) ? q8(a) : a;
}

// FP64 coordinate (EXACT paths that keep their geometry in double).
template <int INTERP>
__device__ __forceinline__ void lin_axis(double coord, int& i, float& w) {
  double xb = coord - 0.5;
  double f = floor(xb);
  i = (int)f;
  float a = (float)(xb - f);
  w = (INTERP == LCT_INTERP_TEX8) ? q8(a) : a;
}

}  // namespace lct
