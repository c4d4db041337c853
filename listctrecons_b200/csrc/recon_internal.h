// lct_recon internals shared by recon.cu and batch.cu (not part of the ABI).
#pragma once

#include <vector>

#include "lct_internal.h"

namespace lct {
// The copy and compute streams of a streamed run: owned by a recon, or shared by a batch.
struct StreamSet {
  cudaStream_t up = nullptr, down = nullptr, bp[2] = {}, cnn = nullptr;
};
int streams_create(StreamSet& ss);  // creates the missing streams (non-blocking)
void streams_destroy(StreamSet& ss);
// fork: every stream of the set waits for the work queued on s so far (ev records it);
// join: s waits for every stream of the set (ev4: four events, recorded on the set's streams)
int streams_fork(const StreamSet& ss, cudaStream_t s, cudaEvent_t ev);
int streams_join(const StreamSet& ss, cudaStream_t s, const cudaEvent_t* ev4);
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
  bool quads = false;        // full windows: the quad-layout pairs kernel applies
  cudaEvent_t ev[6] = {};
  float times[5] = {};
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
};

namespace lct {
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
// learned correction of slices [z0, z1) of an nz-slice volume (cnn.cu)
int cnn_infer_range(lct_cnn* c, const float* d_vol, float* d_out, int nz, int z0, int z1,
                    float bound, cudaStream_t s);
int cnn_reset_rejects(lct_cnn* c, cudaStream_t s);
int cnn_passes(const lct_cnn* c, int nslices);  // kernel passes of prep + 8 convolutions
}  // namespace lct
