// lct_backproject_par_noalloc: the backprojection entry point for callers that cannot let
// this library allocate device memory.
//
// lct_backproject_par repacks the filtered views into quad layout in scratch it allocates on
// the stream (cudaMallocAsync/cudaFreeAsync).  Some callers cannot allow that: an application
// that owns and budgets every byte of device memory itself, a scanner loop that must never stall
// or fail on an allocation in the middle of an acquisition, or a plugin host whose memory comes
// from its own allocator rather than the CUDA runtime's.  This variant takes its scratch from a
// fixed array compiled into the library instead, and calls no cudaMalloc, cudaFree or other
// allocating routine.
//
// Costs and limits, stated for the caller:
//   * the array is kNoAllocScratchBytes = 64 MiB; every GPU on which this part of the library is
//     loaded holds it until the process exits;
//   * a block whose quad views need more (n_angle * (nt + 3) * (ns + 3) * 16 bytes) is refused
//     with LCT_ERR_SCRATCH before anything is launched;
//   * all calls on a device share the one array and it keeps the last call's contents.  Each call
//     overwrites every element it reads before reading it, so nothing needs clearing, but two
//     calls whose kernels overlap on the GPU (different streams, no ordering between them) race
//     on the array: order them, or use lct_backproject_par;
//   * every call looks up the array's device address for the current device
//     (cudaGetSymbolAddress, a host-side lookup, so the address stays right after a device
//     reset); the first call on a device may also load this library's device code there, so make
//     it before any stream capture.
// Windows that are not a full rotation need no scratch: those blocks run the same general
// kernel lct_backproject_par uses for them.
#include "lct_internal.h"

namespace lct {

constexpr size_t kNoAllocScratchBytes = 64ull << 20;

static __device__ __align__(256) float4 g_noalloc_quads[kNoAllocScratchBytes / sizeof(float4)];

// Device address of the scratch array for the current device.  In host code the name
// g_noalloc_quads is only a stand-in for the symbol, never a device address.  Looked up on every
// call: the lookup is host-side, and a cached address would go stale after a device reset.
static int noalloc_scratch(float4** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_quads);
  if (e != cudaSuccess) return cuda_status(e);
  *out = static_cast<float4*>(p);
  return LCT_OK;
}

}  // namespace lct

using namespace lct;

LCT_API int lct_backproject_par_noalloc(const lct_geom* g, const lct_img* ig,
                                        const float* d_betas, const float* d_proj, float* d_img,
                                        int interp, int addr, lct_stream stream) {
  int st = check_geom(g);
  if (st) return st;
  if ((st = check_img(ig))) return st;
  if (!d_betas || !d_proj || !d_img) return LCT_ERR_ARG;
  if (interp != LCT_INTERP_TEX8 && interp != LCT_INTERP_EXACT) return LCT_ERR_ARG;
  if (addr != LCT_ADDR_BORDER && addr != LCT_ADDR_CLAMP) return LCT_ERR_ARG;
  // blocks the quad kernel does not take need no scratch: the allocation-free general path
  if (!(ig->nz <= kBpMaxZ && bp_windows_full(*g, *ig, ig->nz)))
    return lct_backproject_par(g, ig, d_betas, d_proj, d_img, interp, addr, stream);
  const unsigned long long need =
      (unsigned long long)sizeof(float4) * (unsigned long long)g->n_angle *
      (unsigned long long)quad_view_elems(g->ns, g->nt);
  if (need > kNoAllocScratchBytes) return LCT_ERR_SCRATCH;
  float4* q = nullptr;
  if ((st = noalloc_scratch(&q))) return st;
  cudaStream_t s = (cudaStream_t)stream;
  if ((st = launch_quad_pack(d_proj, g->n_angle, g->ns, g->nt, addr, q, s))) return st;
  BpLaunch L;
  L.proj = d_proj;
  L.betas = d_betas;
  L.img = d_img;
  L.view_stride = (long long)g->nt * g->ns;
  L.n_angle = g->n_angle;
  L.nz = ig->nz;
  L.n_slabs = 1;
  L.slab_view[0] = 0;
  L.slab_z0[0] = 0;
  L.interp = interp;
  L.addr = addr;
  L.nz_thread = 8;
  return launch_bp_par_quads(*g, *ig, L, q, s);
}
