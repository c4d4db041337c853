// Status codes, CUDA error bookkeeping, the device status word and geometry checks.
#include <cmath>
#include <mutex>

#include "lct_internal.h"

namespace lct {

static thread_local int t_last_cuda_error = 0;

void set_cuda_error(cudaError_t e) { t_last_cuda_error = (int)e; }

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return LCT_OK;
  set_cuda_error(e);
  return LCT_ERR_CUDA;
}

int launch_status() { return cuda_status(cudaGetLastError()); }

// One word per device, kept in the module's own global memory (no allocation).
static __device__ int g_device_status = 0;

int* device_status_ptr() {
  static std::mutex mu;
  static int* ptrs[64] = {nullptr};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!ptrs[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_device_status) != cudaSuccess) return nullptr;
    ptrs[dev] = static_cast<int*>(p);
  }
  return ptrs[dev];
}

int check_geom(const lct_geom* g) {
  if (!g) return LCT_ERR_ARG;
  if (g->ns <= 0 || g->nt <= 0 || g->n_angle <= 0 || g->n_angle_add < g->n_angle) return LCT_ERR_ARG;
  if (!(g->ds > 0.f) || !(g->dt > 0.f) || !(g->dso > 0.f) || g->n_proj_turn < 2) return LCT_ERR_ARG;
  if (!std::isfinite(g->orbit) || g->orbit == 0.f || !std::isfinite(g->pitch)) return LCT_ERR_ARG;
  if (g->z_dir != 1 && g->z_dir != -1) return LCT_ERR_ARG;
  if ((long long)g->ns * g->nt * (long long)g->n_angle_add > (1LL << 40)) return LCT_ERR_ARG;
  return LCT_OK;
}

int check_img(const lct_img* ig) {
  if (!ig) return LCT_ERR_ARG;
  if (ig->nx <= 0 || ig->ny <= 0 || ig->nz <= 0) return LCT_ERR_ARG;
  if (!(ig->dx > 0.f) || !(ig->dy > 0.f) || !std::isfinite(ig->dz)) return LCT_ERR_ARG;
  return LCT_OK;
}

// CUDA/Backprojector.cu:33-42 with ia_step = 1 (:151).  FP32, same operation order.
BpWindow bp_window(const lct_geom& g, const lct_img& ig, int iz, float dz_per_view,
                   int na1_half) {
  float zc = ((float)iz - ig.wz) * ig.dz;
  int a_middle = (int)roundf((zc - g.source_z0) / dz_per_view);
  a_middle = a_middle < 0 ? 0 : a_middle;
  a_middle = a_middle > g.n_angle - 1 ? g.n_angle - 1 : a_middle;
  BpWindow w;
  w.a_min = (a_middle - na1_half >= 0) ? (a_middle - na1_half) : 0;
  w.a_max = (a_middle + na1_half < g.n_angle) ? (a_middle + na1_half) : g.n_angle - 1;
  w.a_mid = a_middle;
  return w;
}

}  // namespace lct

using namespace lct;

LCT_API const char* lct_status_string(int status) {
  switch (status) {
    case LCT_OK: return "ok";
    case LCT_ERR_ARG: return "invalid argument";
    case LCT_ERR_CUDA: return "CUDA error";
    case LCT_ERR_ALLOC: return "allocation failed";
    case LCT_ERR_RANGE: return "requested reconstruction is outside of allowed data range";
    case LCT_ERR_DEVICE: return "device status word raised";
    case LCT_ERR_UNSUPPORTED: return "unsupported option";
    case LCT_ERR_IO: return "file missing or short";
    case LCT_ERR_SCRATCH: return "problem larger than the fixed scratch of the allocation-free entry point";
    default: return "unknown status";
  }
}

LCT_API int lct_last_cuda_error(void) { return t_last_cuda_error; }

LCT_API int lct_version(void) { return 100; }

LCT_API int lct_device_status(int* code_out) {
  int* p = device_status_ptr();
  if (!p) return LCT_ERR_CUDA;
  int v = 0;
  int st = cuda_status(cudaMemcpy(&v, p, sizeof(int), cudaMemcpyDeviceToHost));
  if (st) return st;
  int zero = 0;
  st = cuda_status(cudaMemcpy(p, &zero, sizeof(int), cudaMemcpyHostToDevice));
  if (code_out) *code_out = v;
  if (st) return st;
  return v ? LCT_ERR_DEVICE : LCT_OK;
}
