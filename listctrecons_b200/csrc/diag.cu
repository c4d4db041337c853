// Diagnostics: sample the texture hardware directly, so tests can pin the register-side
// emulation of linear filtering (tex_emul.cuh, and the CPU oracle) against it.
#include <vector>

#include "lct_internal.h"

namespace lct {

__global__ void tex3d_sample_kernel(cudaTextureObject_t tex, const float* __restrict__ coords,
                                    long long n, float* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = tex3D<float>(tex, coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]);
}

}  // namespace lct

using namespace lct;

LCT_API int lct_diag_tex3d_sample(const float* vol, int nx, int ny, int nz, const float* coords,
                                  int64_t n, int addr, float* out) {
  if (!vol || !coords || !out || nx <= 0 || ny <= 0 || nz <= 0 || n < 0) return LCT_ERR_ARG;
  if (addr != LCT_ADDR_BORDER && addr != LCT_ADDR_CLAMP) return LCT_ERR_ARG;
  if (n == 0) return LCT_OK;
  cudaArray_t arr = nullptr;
  cudaTextureObject_t tex = 0;
  float *d_coords = nullptr, *d_out = nullptr;
  int st = LCT_OK;
  cudaChannelFormatDesc desc = cudaCreateChannelDesc<float>();
  cudaExtent ext = make_cudaExtent(nx, ny, nz);
  do {
    if ((st = cuda_status(cudaMalloc3DArray(&arr, &desc, ext)))) break;
    cudaMemcpy3DParms p = {};
    p.srcPtr = make_cudaPitchedPtr((void*)vol, nx * sizeof(float), nx, ny);
    p.dstArray = arr;
    p.extent = ext;
    p.kind = cudaMemcpyHostToDevice;
    if ((st = cuda_status(cudaMemcpy3D(&p)))) break;
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td = {};
    cudaTextureAddressMode m = addr == LCT_ADDR_CLAMP ? cudaAddressModeClamp : cudaAddressModeBorder;
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = m;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    if ((st = cuda_status(cudaCreateTextureObject(&tex, &rd, &td, nullptr)))) break;
    if ((st = cuda_status(cudaMalloc(&d_coords, sizeof(float) * 3 * n)))) break;
    if ((st = cuda_status(cudaMalloc(&d_out, sizeof(float) * n)))) break;
    if ((st = cuda_status(cudaMemcpy(d_coords, coords, sizeof(float) * 3 * n, cudaMemcpyHostToDevice)))) break;
    tex3d_sample_kernel<<<(unsigned)((n + 255) / 256), 256>>>(tex, d_coords, n, d_out);
    if ((st = launch_status())) break;
    st = cuda_status(cudaMemcpy(out, d_out, sizeof(float) * n, cudaMemcpyDeviceToHost));
  } while (0);
  if (tex) cudaDestroyTextureObject(tex);
  if (arr) cudaFreeArray(arr);
  if (d_coords) cudaFree(d_coords);
  if (d_out) cudaFree(d_out);
  return st;
}
