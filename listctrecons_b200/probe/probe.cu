// liblctprobe.so -- measurement probes, kept out of the product library liblct.so.
//
//   lctp_tex3d_sample    samples a 3-D float texture through the texture hardware, so tests can
//                        pin the register-side emulation of linear filtering (the product's TEX8
//                        kernels and the CPU oracle) against the unit itself;
//   lctp_l1_load_gbs     the L1 hit bandwidth of 16-byte global loads (LDG.128 through the
//                        non-coherent path, the load the backprojector samples with), timed with
//                        CUDA events: the measured peak the backprojector's on-chip roofline is
//                        quoted against.
//
// Plain C types; every function returns 0 on success, else a cudaError_t value.
#include <cuda_runtime.h>

#include <cstdint>

#define LCTP_API extern "C" __attribute__((visibility("default")))

namespace {

__global__ void tex3d_sample_kernel(cudaTextureObject_t tex, const float* __restrict__ coords,
                                    long long n, float* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = tex3D<float>(tex, coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]);
}

// Every CTA re-reads one 16 KiB buffer (resident in each SM's L1 after the first pass): each warp
// instruction is one LDG.128 of 512 contiguous, aligned bytes, eight independent loads per
// unrolled step, the step's window moving by one warp row each iteration.  The loads are volatile
// asm (ld.global.nc.v4.f32, the non-coherent path __ldg takes), so none is hoisted or merged.
constexpr int kL1Vec = 1024;  // float4 in the buffer (16 KiB)
__device__ __forceinline__ float4 ldg128_volatile(const float4* p) {
  float4 v;
  asm volatile("ld.global.nc.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "l"(p));
  return v;
}
__global__ void __launch_bounds__(256) l1_load_kernel(const float4* __restrict__ buf, int iters,
                                                      float* __restrict__ sink) {
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int it = 0; it < iters; it += 8) {
    const int base = (int)threadIdx.x + 32 * (it >> 3);
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const float4 v = ldg128_volatile(buf + ((base + u * 256) & (kL1Vec - 1)));
      acc.x += v.x;
      acc.y += v.y;
      acc.z += v.z;
      acc.w += v.w;
    }
  }
  // the buffer is zero, so nothing is written; the compiler cannot know that
  if (acc.x + acc.y + acc.z + acc.w != 0.f) sink[blockIdx.x * blockDim.x + threadIdx.x] = acc.x;
}

}  // namespace

LCTP_API int lctp_tex3d_sample(const float* vol, int nx, int ny, int nz, const float* coords,
                               int64_t n, int clamp, float* out) {
  if (!vol || !coords || !out || nx <= 0 || ny <= 0 || nz <= 0 || n < 0)
    return (int)cudaErrorInvalidValue;
  if (n == 0) return 0;
  cudaArray_t arr = nullptr;
  cudaTextureObject_t tex = 0;
  float *d_coords = nullptr, *d_out = nullptr;
  cudaError_t e = cudaSuccess;
  cudaChannelFormatDesc desc = cudaCreateChannelDesc<float>();
  cudaExtent ext = make_cudaExtent(nx, ny, nz);
  do {
    if ((e = cudaMalloc3DArray(&arr, &desc, ext)) != cudaSuccess) break;
    cudaMemcpy3DParms p = {};
    p.srcPtr = make_cudaPitchedPtr((void*)vol, nx * sizeof(float), nx, ny);
    p.dstArray = arr;
    p.extent = ext;
    p.kind = cudaMemcpyHostToDevice;
    if ((e = cudaMemcpy3D(&p)) != cudaSuccess) break;
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td = {};
    cudaTextureAddressMode m = clamp ? cudaAddressModeClamp : cudaAddressModeBorder;
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = m;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    if ((e = cudaCreateTextureObject(&tex, &rd, &td, nullptr)) != cudaSuccess) break;
    if ((e = cudaMalloc(&d_coords, sizeof(float) * 3 * n)) != cudaSuccess) break;
    if ((e = cudaMalloc(&d_out, sizeof(float) * n)) != cudaSuccess) break;
    if ((e = cudaMemcpy(d_coords, coords, sizeof(float) * 3 * n, cudaMemcpyHostToDevice)) != cudaSuccess)
      break;
    tex3d_sample_kernel<<<(unsigned)((n + 255) / 256), 256>>>(tex, d_coords, n, d_out);
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    e = cudaMemcpy(out, d_out, sizeof(float) * n, cudaMemcpyDeviceToHost);
  } while (0);
  if (tex) cudaDestroyTextureObject(tex);
  if (arr) cudaFreeArray(arr);
  if (d_coords) cudaFree(d_coords);
  if (d_out) cudaFree(d_out);
  return (int)e;
}

// L1 hit bandwidth of LDG.128 on the current device, GB/s (bytes the threads load / CUDA-event
// time of `reps` launches after `warm` untimed ones).  Full occupancy: 8 CTAs of 256 threads per
// SM; `iters` loads per thread (a multiple of 8).  Synchronous.
LCTP_API int lctp_l1_load_gbs(int iters, int warm, int reps, double* gbs, double* ms_per_launch) {
  if (!gbs || iters <= 0 || iters % 8 || reps <= 0 || warm < 0) return (int)cudaErrorInvalidValue;
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
    return (int)e;
  const int grid = sms * 8;
  float4* buf = nullptr;
  float* sink = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  do {
    if ((e = cudaMalloc(&buf, sizeof(float4) * kL1Vec)) != cudaSuccess) break;
    if ((e = cudaMemset(buf, 0, sizeof(float4) * kL1Vec)) != cudaSuccess) break;
    if ((e = cudaMalloc(&sink, sizeof(float) * grid * 256)) != cudaSuccess) break;
    if ((e = cudaEventCreate(&e0)) != cudaSuccess) break;
    if ((e = cudaEventCreate(&e1)) != cudaSuccess) break;
    for (int r = 0; r < warm; ++r) l1_load_kernel<<<grid, 256>>>(buf, iters, sink);
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    cudaEventRecord(e0);
    for (int r = 0; r < reps; ++r) l1_load_kernel<<<grid, 256>>>(buf, iters, sink);
    cudaEventRecord(e1);
    if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
    float ms = 0.f;
    if ((e = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess) break;
    const double bytes = (double)grid * 256.0 * (double)iters * 16.0 * reps;
    *gbs = bytes / (ms * 1e-3) / 1e9;
    if (ms_per_launch) *ms_per_launch = ms / reps;
  } while (0);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (buf) cudaFree(buf);
  if (sink) cudaFree(sink);
  return (int)e;
}
