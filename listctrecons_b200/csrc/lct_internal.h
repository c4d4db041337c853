// Internal helpers shared by the liblct translation units (not installed, not part of the ABI).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "lct.h"

#define LCT_API extern "C" __attribute__((visibility("default")))
#ifdef __CUDACC__
#define LCT_HD __host__ __device__
#else
#define LCT_HD
#endif

namespace lct {

// Include/Common.h:3-4.  PI is a double literal there; where the reference evaluates an
// expression in double because of it, the product does the same.
constexpr double kRefPi = 3.141592653589793238462643383;
constexpr int kBlockSlices = 32;

// Thread-local record of the last CUDA error turned into LCT_ERR_CUDA.
void set_cuda_error(cudaError_t e);
int cuda_status(cudaError_t e);  // LCT_OK or LCT_ERR_CUDA (records e)
int launch_status();             // cudaGetLastError() -> status

// Device status word (file-scope __device__ int in common.cu).  Kernels raise it on a work
// item they refuse (an index outside its buffer) instead of trapping.
int* device_status_ptr();  // per current device, resolved with cudaGetSymbolAddress
enum DeviceStatus : int {
  kDevOk = 0,
  kDevIndexRange = 1,  // an index computed from the geometry fell outside its buffer
  kDevWaitTimeout = 2, // a bounded wait in a pipelined kernel ran out
};

// Validation of the mirrored reference structs.
int check_geom(const lct_geom* g);
int check_img(const lct_img* ig);

// Per-slice view windows of the parallel-beam backprojection (CUDA/Backprojector.cu:37-42),
// always evaluated in FP32 exactly as the reference does.
struct BpWindow {
  int a_min, a_mid, a_max;
};
BpWindow bp_window(const lct_geom& g, const lct_img& ig, int iz, float dz_per_view,
                   int na1_half);

// Launch description for the parallel-beam backprojection kernels (backproject.cu).
constexpr int kBpMaxZ = 32;      // slices sharing one window table
constexpr int kBpMaxSlabs = 256; // slabs in one launch (scan mode)
struct BpLaunch {
  const float* proj;   // filtered views; slab s's local view 0 is proj + slab_view[s]*view_stride
  const float* betas;  // view angles; slab s's local view 0 is betas + slab_view[s]
  float* img;          // slab s, local slice z -> img + (slab_z0[s] + z) * nx * ny
  long long view_stride;
  int n_angle;         // local views per slab
  int nz;              // slices per slab (<= kBpMaxZ)
  int n_slabs;
  int slab_view[kBpMaxSlabs];
  int slab_z0[kBpMaxSlabs];
  int interp, addr;
  int nz_thread;       // slices per thread (8, 16, 32; 0 = choose)
  int minb = 0;        // quad kernel: resident CTAs per SM the register budget targets (0 = 4)
  // quad kernel only: a part of the slabs' views, [view_lo, view_hi) in slab-local indices,
  // carried between parts as raw FP32 sums in img (part kBpWhole / First / Middle / Last); the
  // parts of one slab run in order on one stream and sum every view in the same sequence as a
  // whole launch
  int view_lo = 0, view_hi = 1 << 30;
  int part = 0;
  // quad kernel only: > 0 when the quads are a ring of that many views (slab s's local view ia
  // at slot (slab_view[s] + ia) mod quad_ring; bounded-memory runs); 0: linear
  long long quad_ring = 0;
};
enum BpPart : int { kBpWhole = 0, kBpFirst = 1, kBpMiddle = 2, kBpLast = 3 };
int launch_bp_par(const lct_geom& g, const lct_img& ig, const BpLaunch& L, cudaStream_t s);

// Filtered views in quad layout for the backprojector.  Per view, entry (j, i) for
// j in [-2, nt], i in [-2, ns] (stored at (j + 2) * (ns + 3) + (i + 2)) holds the 2 x 2 texel
// block with top-left (j, i) as {T00, T10 - T00, T01 - T00, T11 - T10 - T01 + T00} (row
// difference before column difference), texels outside the detector read as 0 (LCT_ADDR_BORDER)
// or clamped to the edge (LCT_ADDR_CLAMP).  A bilinear sample is then one 16-byte load at its
// clamped origin and three FMAs -- the first two, (T00, dy) + a (dx, dxy), as one packed FP32
// pair; the padding ring makes every clamped origin valid.
LCT_HD inline long long quad_cols(int ns) { return (long long)ns + 3; }
LCT_HD inline long long quad_view_elems(int ns, int nt) { return (long long)(nt + 3) * (ns + 3); }
// ring > 0: quads is a ring of `ring` views and rows view v is packed into slot
// (vbase + v) mod ring; 0: into view v.
int launch_quad_pack(const float* rows, long long views, int ns, int nt, int addr, float4* quads,
                     cudaStream_t s, long long vbase = 0, long long ring = 0);
// Backprojection from quad-layout views (full windows only; L.proj is ignored, L.quads used).
int launch_bp_par_quads(const lct_geom& g, const lct_img& ig, const BpLaunch& L,
                        const float4* quads, cudaStream_t s);
// EXACT backprojection with each view's tile footprint staged in shared memory by TMA (the
// quads' tensor map from bp_tma_map, over the same quad buffer); whole launches with 8 slices per
// thread (other launches go to launch_bp_par_quads).
int bp_tma_map(CUtensorMap* map, const float4* quads, int ns, int nt, long long views);
int launch_bp_par_quads_tma(const lct_geom& g, const lct_img& ig, const BpLaunch& L,
                            const float4* quads, const CUtensorMap& map, cudaStream_t s);
// Backprojection sampled by the texture unit (TEX8 only): tex holds the filtered views as a
// 3-D array, slab s's local view ia at z slot (slab_view[s] + ia) mod L.quad_ring (0: no wrap).
int launch_bp_par_texture(const lct_geom& g, const lct_img& ig, const BpLaunch& L,
                          cudaTextureObject_t tex, cudaStream_t s);
// A 3-D float texture of `depth` filtered views (x = column, y = row, z = view slot) with linear
// filtering and BORDER or CLAMP addressing; filled from linear views by view_texture_fill
// (slot0 onward, wrapping at depth).  view_texture_add_other_mode adds a second texture object
// over the same array with the other addressing; view_texture_for picks the one for `addr`
// (0 when that mode has none).
struct ViewTexture {
  cudaArray_t arr = nullptr;
  cudaTextureObject_t tex = 0;
  cudaTextureObject_t tex_other = 0;
  int addr = 0;
  int ns = 0, nt = 0;
  long long depth = 0;
};
int view_texture_create(ViewTexture& t, int ns, int nt, long long depth, int addr);
int view_texture_add_other_mode(ViewTexture& t);
cudaTextureObject_t view_texture_for(const ViewTexture& t, int addr);
void view_texture_destroy(ViewTexture& t);
// PI-original rebin sampled by the texture unit from a caller-owned texture of the fan block
// (depth >= n_angle_add): fills it and launches on s, stream-ordered, no allocation
int launch_rebin_pi_ori_tex(const lct_geom& g, const ViewTexture& t, int addr, const float* d_fan,
                            float* d_par, cudaStream_t s);
int view_texture_fill(const ViewTexture& t, const float* rows, long long views, long long slot0,
                      cudaStream_t s);
// True when every slice window of the block is a full rotation (the pairs kernels apply).
bool bp_windows_full(const lct_geom& g, const lct_img& ig, int nz);
// Work-list backprojection over several scans (batch): per-scan kernel arguments are built on
// the host into an opaque record of bp_quad_args_size() bytes, copied to the device, and one
// persistent launch runs every scan's tiles.
int bp_quad_args_size();
int bp_quad_args_build(const lct_geom& g, const lct_img& ig, const BpLaunch& L,
                       const float4* quads, void* out, int* tiles);
int launch_bp_quad_worklist(const void* d_args, const int* d_prefix, int n_scans, int* d_counter,
                            int nz_thread, int interp, int minb, cudaStream_t s);

// Rebinning, scan mode: each global parallel view g in [g0, g0 + nviews) is interpolated
// from the fan buffer whose view 0 is global fan view `fan_first`, with the view shift of
// column is taken from an FP64 table (alpha(is)/orbit), identical for every view.
// fan_ring > 0: d_fan is a ring of fan_ring views (fan view v - fan_first at slot v mod ring).
// width: 0 = four columns per thread where the geometry allows (float4 rows), 1 = one column,
// 4 = four or LCT_ERR_UNSUPPORTED.
int launch_rebin_fan2par_scan(const lct_geom& g, const float* d_fan, long long fan_first,
                              long long fan_count, float* d_par, long long g0,
                              long long nviews, int interp, int addr, cudaStream_t s,
                              long long fan_ring = 0, int width = 0);

// BF16x3 tensor-core filter with caller-owned scratch (filter_tc.cu): tc_scratch_bytes() for
// rows_cap rows; tc_build_toeplitz once per taps, then tc_filter per batch of rows (in place).
size_t tc_scratch_bytes(int ns, long long rows_cap, int mode);
int tc_build_toeplitz(int ns, const float* d_h, void* scratch, int mode, cudaStream_t s);
int tc_filter(int ns, float* d_rows, long long nrows, void* scratch, long long rows_cap, int mode,
              cudaStream_t s);
int launch_filter_tc(int ns, const float* d_h, float* d_rows, long long nrows, int mode,
                     cudaStream_t s);

// Filter over nrows rows of ns samples (filter.cu).
int launch_filter_rows(int ns, const float* d_h, float* d_rows, long long nrows, int mode,
                       cudaStream_t s);

}  // namespace lct
