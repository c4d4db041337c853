// lct_recon internals shared by recon.cu and batch.cu (not part of the ABI).
#pragma once

#include <algorithm>
#include <vector>

#include "lct_internal.h"

namespace lct {
// The copy and compute streams of a streamed run: owned by a recon, or shared by a batch.
// prep carries the per-piece rebin / filter / pack of streamed runs, apart from the caller's
// stream (measured on config 2 host to host: 85.5 -> 84.3 ms per volume with the first slab's
// growing pieces; the device's highest stream priority for it measured 0.4-0.7% slower on the
// same box, on config 2 and on the bounded config 5).
struct StreamSet {
  cudaStream_t up = nullptr, down = nullptr, bp[2] = {}, cnn = nullptr, prep = nullptr;
};
int streams_create(StreamSet& ss);  // creates the missing streams (non-blocking)
void streams_destroy(StreamSet& ss);
// fork: every stream of the set waits for the work queued on s so far (ev records it);
// join: s waits for every stream of the set (ev5: five events, recorded on the set's streams)
constexpr int kForkJoinEvents = 6;  // events a run keeps for its fork (1) and join (5)
int streams_fork(const StreamSet& ss, cudaStream_t s, cudaEvent_t ev);
int streams_join(const StreamSet& ss, cudaStream_t s, const cudaEvent_t* ev5);

// The first slab of a streamed run is backprojected in parts as its views arrive; a part needs
// the conjugates (half a turn on) of its pairs.  The piece that crosses half a turn ends
// kFirstPairs pairs past it, so the first part starts then and not up to a piece later, and the
// pieces after it grow with the pairs already available (at least 2 kFirstPairs views) up to the
// full piece: each part's views are uploaded and packed while the part before it runs, instead
// of the backprojector waiting for a whole piece after a short first part.
constexpr long long kFirstPairs = 64;
inline long long first_part_target(long long done, long long target, long long gfirst,
                                   long long half) {
  const long long pivot = gfirst + half + kFirstPairs;
  if (done < pivot) return target > pivot ? pivot : target;
  const long long grow = std::max<long long>(2 * kFirstPairs, done - (gfirst + half));
  return std::min(target, done + grow);
}

// Pinned host staging: a 2 MiB-aligned anonymous mapping with transparent huge pages requested,
// faulted in one touch per 2 MiB and registered with the driver -- about twice as fast to set up
// as cudaHostAlloc, which pins 4 KiB pages (measured on B200 hosts: 128 MB in 30 ms against
// 65 ms).  Falls back to cudaHostAlloc where the mapping or the registration is refused.
struct PinnedBuf {
  float* p = nullptr;
  void* map = nullptr;  // the mapping (null: cudaHostAlloc memory)
  size_t map_bytes = 0;
};
int pinned_alloc(size_t bytes, PinnedBuf& b);  // LCT_OK or LCT_ERR_ALLOC
void pinned_free(PinnedBuf& b);
}  // namespace lct

struct lct_recon {
  lct_plan_info info;
  std::vector<lct_block_info> blocks;
  lct_recon_opts o;
  long long plane = 0;           // nt * ns
  long long fan_first = 0, fan_count = 0;
  long long g_first = 0, g_count = 0;  // scan mode
  float* d_fan = nullptr;
  float* d_par = nullptr;
  float* d_betas = nullptr;
  float* d_h = nullptr;
  float* d_img = nullptr;
  float4* d_quad = nullptr;  // filtered views in quad layout (backprojection input)
  void* d_tc = nullptr;      // BF16x3 filter operands (row and Toeplitz planes)
  long long tc_rows = 0;
  bool quads = false;        // full windows: the pairs kernels (quads or texture) apply
  bool tex_bp = false;       // the pairs backprojection samples a 3-D texture (TEX8) instead
  lct::ViewTexture vtex;     // filtered views as that texture (scan: global views; block: one block)
  lct::ViewTexture pi_tex;   // PI-original rebin in TEX8: the fan block as a texture, reused per block
  bool tma_bp = false;       // EXACT pairs backprojection with TMA-staged footprints (same quads)
  CUtensorMap tma_map;       // d_quad as the staged kernel's tensor
  cudaEvent_t ev[6] = {};
  float times[5] = {};
  float io_times[3] = {};  // lct_recon_io_times
  lct_cnn* cnn = nullptr;    // learned correction after backprojection (not owned)
  float cnn_bound = 0.f;
  float* d_plain = nullptr;  // plain FDK volume when the learned correction runs
  cudaEvent_t ev_cnn[2] = {};
  float cnn_ms = 0.f;
  // streaming runs from host fan buffers: streams and per-slab events (created on first use)
  lct::StreamSet ss;
  std::vector<cudaEvent_t> sev;
  bool streamed = false;  // the last run overlapped its copies with the compute
  int device = 0;
  long long voxel_updates = 0;
  int launches = 0;
  // bounded device memory (lct_recon_create_bounded): d_fan, d_quad and d_img are rings and
  // d_par / d_tc hold one piece; 0 rings mean whole buffers
  bool bounded = false;
  long long piece = 0;       // views rebinned, filtered and packed per step
  long long fan_ring = 0;    // fan views in d_fan (0: fan_count, linear)
  long long quad_ring = 0;   // views in d_quad (0: g_count, linear)
  int img_ring = 0;          // slabs in d_img for host / file output (0: the whole volume)
  long long device_bytes = 0;
  // pinned host staging of lct_recon_run_file and of pageable host volumes, one buffer per slot:
  // each is pinned on first use by the reader or writer thread that fills or drains it (so the
  // pipeline starts after one slot, not after all of them) and kept until destroy
  std::vector<lct::PinnedBuf> h_fan_slots;  // fan chunks of fan_chunk_views views
  long long fan_chunk_views = 0;
  std::vector<lct::PinnedBuf> h_img_slots;  // slabs
};

namespace lct {
// backprojection slices per thread: the requested 4 / 8 / 16, else the measured default (8,
// or 4 when a view stays active for fewer than 6 slices: (feed / 2) / dz)
inline int pick_bp_nz(const lct_geom& g, const lct_img& ig, int requested) {
  if (requested == 4 || requested == 8 || requested == 16) return requested;
  const double act = 0.5 * (double)g.pitch / (double)ig.dz;
  return act < 6.0 ? 4 : 8;
}
// kernels one filter call launches
inline int filter_launches(int mode) { return mode == LCT_FILTER_FP32 ? 1 : 2; }
// addressing of block b (LEGACY: clamped first block, border afterwards)
inline int block_addr(const lct_recon* r, int b) {
  if (r->o.addr == LCT_ADDR_LEGACY) return b == 0 ? LCT_ADDR_CLAMP : LCT_ADDR_BORDER;
  return r->o.addr;
}

// creation steps shared by lct_recon_create and lct_recon_create_bounded (recon.cu)
int recon_setup(const lct_plan* plan, const lct_recon_opts* opts, lct_recon** out);
int recon_alloc_common(lct_recon* r, const lct_plan* plan);
int recon_alloc_status(int st);

// the texture sampler when asked for (TEX8, full windows, one addressing mode for every slab);
// AUTO is quads, which measured faster on B200 for TEX8 too
inline bool want_texture(const lct_recon_opts& o, bool full_windows) {
  return full_windows && o.backprojector == LCT_BP_PAR && o.interp == LCT_INTERP_TEX8 &&
         o.addr != LCT_ADDR_LEGACY && o.bp_sampler == LCT_BP_SAMPLER_TEXTURE;
}
// the filtered views [v0, v0 + nv) (at par) into the backprojector's input: texture slots or
// quads, ring-aware (bounded recons)
int recon_pack(lct_recon* r, const float* par, long long nv, long long v0, int addr, cudaStream_t s);
// one pairs backprojection launch (quads or texture)
int recon_bp_pairs(lct_recon* r, BpLaunch& L, cudaStream_t s);

// scan-mode stages of one recon, on any stream (used by lct_recon_run and the batch graphs)
int recon_stage_rebin(lct_recon* r, const float* d_fan, cudaStream_t s);
int recon_stage_filter(lct_recon* r, cudaStream_t s);
int recon_stage_bp(lct_recon* r, float* d_img, cudaStream_t s);
void recon_bp_launch(const lct_recon* r, int b0, int b1, float* d_img, BpLaunch& L);
bool recon_bp_quads_all(const lct_recon* r);
// Streamed scan-mode run from a host fan buffer (lct_recon_run's path) on compute stream s and
// the streams of ss, which the caller has forked from s and joins afterwards.
bool recon_streamable(const lct_recon* r);
int recon_run_streamed(lct_recon* r, const float* fan_host, long long skip, float* d_img,
                       float* d_out, float* image_host, cudaStream_t s, const StreamSet& ss);
// Runs of a bounded recon (recon_bounded.cu): fan from a host or device pointer (fan points at
// the run's first view), volume to a device or host pointer.
int recon_run_bounded_ptr(lct_recon* r, const float* fan, bool fan_on_device, float* image,
                          bool image_on_device, cudaStream_t s);
void recon_free_bounded(lct_recon* r);  // pinned staging of lct_recon_run_file
// True for host memory the driver has pinned (cudaHostAlloc, cudaHostRegister): copies to it are
// asynchronous.  A copy to pageable memory returns only once it is done, holding the thread that
// queues the pipeline.
bool host_pinned(const void* p);
// learned correction of slices [z0, z1) of an nz-slice volume (cnn.cu)
int cnn_infer_range(lct_cnn* c, const float* d_vol, float* d_out, int nz, int z0, int z1,
                    float bound, cudaStream_t s);
int cnn_reset_rejects(lct_cnn* c, cudaStream_t s);
int cnn_passes(const lct_cnn* c, int nslices);  // kernel passes of prep + 8 convolutions
}  // namespace lct
