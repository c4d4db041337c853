// Filtered views as a 3-D texture for the texture-unit backprojector (TEX8): the reference binds
// its filtered block to a 3-D array the same way (CUDA/Backprojector.cu:111-136), here once per
// recon with a texture object instead of a legacy texture reference, and filled by stream-ordered
// copies from the linear filtered views.
#include "lct_internal.h"

namespace lct {

static int make_tex_object(cudaArray_t arr, int addr, cudaTextureObject_t* out) {
  cudaResourceDesc rd = {};
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = arr;
  cudaTextureDesc td = {};
  const cudaTextureAddressMode m = addr == LCT_ADDR_CLAMP ? cudaAddressModeClamp : cudaAddressModeBorder;
  td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = m;
  td.filterMode = cudaFilterModeLinear;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 0;
  return cuda_status(cudaCreateTextureObject(out, &rd, &td, nullptr));
}

int view_texture_create(ViewTexture& t, int ns, int nt, long long depth, int addr) {
  if (ns <= 0 || nt <= 0 || depth <= 0) return LCT_ERR_ARG;
  int dev = 0, maxw = 0, maxh = 0, maxd = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxTexture3DWidth, dev);
  cudaDeviceGetAttribute(&maxh, cudaDevAttrMaxTexture3DHeight, dev);
  cudaDeviceGetAttribute(&maxd, cudaDevAttrMaxTexture3DDepth, dev);
  if (ns > maxw || nt > maxh || depth > maxd) return LCT_ERR_UNSUPPORTED;
  cudaChannelFormatDesc desc = cudaCreateChannelDesc<float>();
  int st = cuda_status(cudaMalloc3DArray(&t.arr, &desc, make_cudaExtent(ns, nt, (size_t)depth)));
  if (st) return st;
  t.addr = addr == LCT_ADDR_CLAMP ? LCT_ADDR_CLAMP : LCT_ADDR_BORDER;
  if ((st = make_tex_object(t.arr, t.addr, &t.tex))) {
    cudaFreeArray(t.arr);
    t.arr = nullptr;
    return st;
  }
  t.ns = ns;
  t.nt = nt;
  t.depth = depth;
  return LCT_OK;
}

int view_texture_add_other_mode(ViewTexture& t) {
  if (!t.arr) return LCT_ERR_ARG;
  if (t.tex_other) return LCT_OK;
  return make_tex_object(t.arr, t.addr == LCT_ADDR_CLAMP ? LCT_ADDR_BORDER : LCT_ADDR_CLAMP,
                         &t.tex_other);
}

cudaTextureObject_t view_texture_for(const ViewTexture& t, int addr) {
  const int a = addr == LCT_ADDR_CLAMP ? LCT_ADDR_CLAMP : LCT_ADDR_BORDER;
  return a == t.addr ? t.tex : t.tex_other;
}

void view_texture_destroy(ViewTexture& t) {
  if (t.tex) cudaDestroyTextureObject(t.tex);
  if (t.tex_other) cudaDestroyTextureObject(t.tex_other);
  if (t.arr) cudaFreeArray(t.arr);
  t = ViewTexture();
}

int view_texture_fill(const ViewTexture& t, const float* rows, long long views, long long slot0,
                      cudaStream_t s) {
  if (views <= 0) return LCT_OK;
  if (!t.arr || slot0 < 0 || views > t.depth) return LCT_ERR_ARG;
  long long v = 0, slot = slot0 % t.depth;
  while (v < views) {
    const long long n = std::min(views - v, t.depth - slot);
    cudaMemcpy3DParms p = {};
    p.srcPtr = make_cudaPitchedPtr((void*)(rows + v * (long long)t.nt * t.ns), t.ns * sizeof(float),
                                   t.ns, t.nt);
    p.dstArray = t.arr;
    p.dstPos = make_cudaPos(0, 0, (size_t)slot);
    p.extent = make_cudaExtent(t.ns, t.nt, (size_t)n);
    p.kind = cudaMemcpyDeviceToDevice;
    int st = cuda_status(cudaMemcpy3DAsync(&p, s));
    if (st) return st;
    v += n;
    slot = (slot + n) % t.depth;
  }
  return LCT_OK;
}

}  // namespace lct
