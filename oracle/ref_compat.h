/*
 * ref_compat.h -- TEST INFRASTRUCTURE ONLY (the oracle side; never shipped, never on the
 * product path).
 *
 * Forced-include header (`nvcc -include ref_compat.h`) that lets the reference's own CUDA
 * sources (CUDA/Rebiner.cu, CUDA/Backprojector.cu) compile unmodified on CUDA 12, where the
 * legacy texture-reference API they use was removed.  It supplies:
 *
 *   - a `texture<T, dim, mode>` stand-in (the macro below turns each file-scope
 *     `texture<...> name;` into a `__device__` object holding a cudaTextureObject_t);
 *   - cudaBindTextureToArray / cudaUnbindTexture overloads for it;
 *   - a device tex3D() overload that forwards to the texture-object tex3D.
 *
 * Binding semantics follow the legacy runtime: the attributes held in the host-side object
 * (filterMode, normalized, addressMode[]) are captured when the texture is bound.  The
 * reference assigns addressMode = Border *after* binding (CUDA/Rebiner.cu:137-139,
 * CUDA/Backprojector.cu:134-136), so the first bind of each texture runs with the legacy
 * default (Clamp, from the texture<> constructor defaults: point filter, clamp addressing,
 * unnormalised) and every later bind runs with Border.  The product exposes the same choice
 * as an explicit addressing mode (LCT_ADDR_LEGACY).
 *
 * This header only adapts an API; the reference's kernel bodies and host flow compile as they
 * lie under the reference tree.
 */
#pragma once
#include <cuda_runtime.h>
#include <cuda.h>
#include <cstdio>
#include <iostream>

template <class T, int Dim, enum cudaTextureReadMode Mode>
struct lct_compat_texture {
  cudaTextureObject_t obj = 0;
  enum cudaTextureFilterMode filterMode = cudaFilterModePoint;
  int normalized = 0;
  enum cudaTextureAddressMode addressMode[3] = {cudaAddressModeClamp, cudaAddressModeClamp,
                                                cudaAddressModeClamp};
  cudaChannelFormatDesc channelDesc = {};
};

template <class T, int Dim, enum cudaTextureReadMode Mode>
static cudaError_t cudaBindTextureToArray(const lct_compat_texture<T, Dim, Mode>* tex,
                                          cudaArray_const_t arr,
                                          const cudaChannelFormatDesc* /*desc*/) {
  auto* t = const_cast<lct_compat_texture<T, Dim, Mode>*>(tex);
  if (t->obj) {
    cudaDestroyTextureObject(t->obj);
    t->obj = 0;
  }
  cudaResourceDesc rd = {};
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = const_cast<cudaArray_t>(arr);
  cudaTextureDesc td = {};
  for (int i = 0; i < 3; ++i) td.addressMode[i] = t->addressMode[i];
  td.filterMode = t->filterMode;
  td.readMode = Mode;
  td.normalizedCoords = t->normalized;
  cudaError_t e = cudaCreateTextureObject(&t->obj, &rd, &td, nullptr);
  if (e != cudaSuccess) return e;
  /* publish the handle to the device copy of the object */
  return cudaMemcpyToSymbol(*tex, t, sizeof(*t));
}

template <class T, int Dim, enum cudaTextureReadMode Mode>
static cudaError_t cudaUnbindTexture(const lct_compat_texture<T, Dim, Mode>& tex) {
  auto* t = const_cast<lct_compat_texture<T, Dim, Mode>*>(&tex);
  cudaError_t e = cudaSuccess;
  if (t->obj) e = cudaDestroyTextureObject(t->obj);
  t->obj = 0;
  return e;
}

__device__ inline float tex3D(
    const lct_compat_texture<float, cudaTextureType3D, cudaReadModeElementType>& t, float x,
    float y, float z) {
  return tex3D<float>(t.obj, x, y, z);
}

#define texture __device__ lct_compat_texture
