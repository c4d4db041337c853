// Batched reconstruction of many independent helical scans (uneven length, pitch, rows, columns,
// volume): every buffer is owned per scan (one lct_recon each, allocated once), and a run is
//   upload fans -> [graph] rebin all scans -> [graph] filter + quad pack all scans
//               -> [graph] persistent work-list backprojection over every scan's tiles (one
//                  launch per thread shape: each scan keeps the shape its own run would use)
//               -> download volumes.
// The three stage graphs are captured once at create (after one eager warm-up run, which also
// sets kernel attributes and loads modules).  The work-list kernel balances the uneven scans
// across the SMs; each tile runs the arithmetic of its scan's own launch, so a scan's volume is
// bit-identical to lct_recon_run with the same options.
#include <map>
#include <new>
#include <utility>
#include <vector>

#include "recon_internal.h"

// One work list per backprojection thread shape: the scans that share a shape (slices per
// thread, CTAs per SM) run in one persistent launch.
struct BpGroup {
  int nz = 8, minb = 4, n = 0;
  void* d_args = nullptr;    // per-scan backprojection arguments
  int* d_prefix = nullptr;   // tile prefix sums, n + 1
  int* d_counter = nullptr;  // work-list cursor, zeroed by the graph before each launch
};

struct lct_batch {
  std::vector<lct_recon*> recs;
  cudaGraphExec_t exec[3] = {};
  std::vector<BpGroup> groups;
  bool worklist = false;
  int interp = LCT_INTERP_TEX8;
  cudaEvent_t ev[6] = {};
  float times[5] = {};
  int launches = 0;
  lct::StreamSet ss;              // streamed runs from host fans (created on first use)
  std::vector<cudaEvent_t> sev;   // their fork / join events
};

namespace lct {

static void free_batch(lct_batch* b) {
  if (!b) return;
  for (auto& e : b->exec)
    if (e) cudaGraphExecDestroy(e);
  for (auto* r : b->recs) lct_recon_destroy(r);
  for (auto& gr : b->groups) {
    cudaFree(gr.d_args);
    cudaFree(gr.d_prefix);
    cudaFree(gr.d_counter);
  }
  for (auto& e : b->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : b->sev)
    if (e) cudaEventDestroy(e);
  streams_destroy(b->ss);
  delete b;
}

static int batch_stage(lct_batch* b, int stage, cudaStream_t s) {
  int st = LCT_OK;
  if (stage == 2 && b->worklist) {
    for (auto& gr : b->groups) {
      if ((st = cuda_status(cudaMemsetAsync(gr.d_counter, 0, sizeof(int), s)))) return st;
      if ((st = launch_bp_quad_worklist(gr.d_args, gr.d_prefix, gr.n, gr.d_counter, gr.nz,
                                        b->interp, gr.minb, s)))
        return st;
    }
    return LCT_OK;
  }
  for (auto* r : b->recs) {
    if (stage == 0)
      st = recon_stage_rebin(r, r->d_fan, s);
    else if (stage == 1)
      st = recon_stage_filter(r, s);
    else
      st = recon_stage_bp(r, r->d_img, s);
    if (st) return st;
  }
  return LCT_OK;
}

}  // namespace lct

using namespace lct;

LCT_API int lct_batch_create(const lct_plan* const* plans, int n, const lct_recon_opts* opts,
                             lct_batch** out) {
  if (!plans || n <= 0 || !out) return LCT_ERR_ARG;
  *out = nullptr;
  lct_recon_opts o;
  if (opts)
    o = *opts;
  else
    lct_recon_opts_default(&o);
  if (o.mode != LCT_MODE_SCAN) return LCT_ERR_UNSUPPORTED;
  lct_batch* b = new (std::nothrow) lct_batch;
  if (!b) return LCT_ERR_ALLOC;
  int st = LCT_OK;
  // one autotune for the batch: on the scan with the most backprojection work
  const bool tune = o.bp_nz == -1;
  if (tune) o.bp_nz = 0;
  for (int i = 0; i < n && !st; ++i) {
    lct_recon* r = nullptr;
    st = lct_recon_create(plans[i], &o, &r);
    if (!st) b->recs.push_back(r);
  }
  cudaStream_t s = nullptr;
  if (!st) st = cuda_status(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  if (!st && tune) {
    lct_recon* big = b->recs[0];
    for (auto* r : b->recs)
      if (r->voxel_updates > big->voxel_updates) big = r;
    int nz = 8, mb = 4;
    st = lct_recon_autotune(big, &nz, &mb);
    for (auto* r : b->recs) {
      r->o.bp_nz = nz;
      r->o.bp_minb = mb;
    }
  }
  // work list: every scan on the quad kernel with one interpolation and thread shape (texture-
  // sampled scans keep their own launches, as in their single-scan runs)
  if (!st) {
    b->worklist = true;
    b->interp = b->recs[0]->o.interp;
    for (auto* r : b->recs)
      if (!recon_bp_quads_all(r) || r->o.interp != b->interp) b->worklist = false;
  }
  if (!st && b->worklist) {
    // each scan keeps the thread shape its own run would use (the slices-per-thread heuristic,
    // or the requested / autotuned shape); scans sharing a shape share a work list
    const int asz = bp_quad_args_size();
    std::map<std::pair<int, int>, std::vector<int>> by_shape;
    for (int i = 0; i < n; ++i) {
      lct_recon* r = b->recs[i];
      BpLaunch L;
      recon_bp_launch(r, 0, r->info.n_blocks_run, r->d_img, L);
      r->o.bp_nz = L.nz_thread;  // the scan's own launches use the same shape
      r->o.bp_minb = L.minb > 0 ? L.minb : 4;
      by_shape[{r->o.bp_nz, r->o.bp_minb}].push_back(i);
    }
    for (auto& kv : by_shape) {
      if (st) break;
      BpGroup gr;
      gr.nz = kv.first.first;
      gr.minb = kv.first.second;
      gr.n = (int)kv.second.size();
      std::vector<char> args((size_t)asz * gr.n);
      std::vector<int> prefix(gr.n + 1, 0);
      for (int k = 0; k < gr.n && !st; ++k) {
        lct_recon* r = b->recs[kv.second[k]];
        BpLaunch L;
        recon_bp_launch(r, 0, r->info.n_blocks_run, r->d_img, L);
        int tiles = 0;
        st = bp_quad_args_build(r->info.ctg, r->info.ig, L, r->d_quad,
                                args.data() + (size_t)asz * k, &tiles);
        prefix[k + 1] = prefix[k] + tiles;
      }
      b->groups.push_back(gr);
      BpGroup& g = b->groups.back();
      if (!st) st = cuda_status(cudaMalloc(&g.d_args, args.size()));
      if (!st) st = cuda_status(cudaMalloc(&g.d_prefix, sizeof(int) * (gr.n + 1)));
      if (!st) st = cuda_status(cudaMalloc(&g.d_counter, sizeof(int)));
      if (!st)
        st = cuda_status(cudaMemcpy(g.d_args, args.data(), args.size(), cudaMemcpyHostToDevice));
      if (!st)
        st = cuda_status(cudaMemcpy(g.d_prefix, prefix.data(), sizeof(int) * (gr.n + 1),
                                    cudaMemcpyHostToDevice));
    }
  }
  // eager warm-up on zeroed fans, then capture one graph per stage
  for (auto* r : b->recs)
    if (!st) st = cuda_status(cudaMemsetAsync(r->d_fan, 0, sizeof(float) * r->fan_count * r->plane, s));
  for (int k = 0; k < 3 && !st; ++k) st = batch_stage(b, k, s);
  if (!st) st = cuda_status(cudaStreamSynchronize(s));
  for (int k = 0; k < 3 && !st; ++k) {
    cudaGraph_t g = nullptr;
    if ((st = cuda_status(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal)))) break;
    int st_stage = batch_stage(b, k, s);
    int st_end = cuda_status(cudaStreamEndCapture(s, &g));
    st = st_stage ? st_stage : st_end;
    if (!st) st = cuda_status(cudaGraphInstantiate(&b->exec[k], g, 0));
    if (g) cudaGraphDestroy(g);
  }
  for (auto& e : b->ev)
    if (!st) st = cuda_status(cudaEventCreate(&e));
  if (s) cudaStreamDestroy(s);
  if (st) {
    free_batch(b);
    return st;
  }
  *out = b;
  return LCT_OK;
}

// Host fans: every scan's streamed run (recon_run_streamed) back to back on shared streams --
// one upload stream (the scans arrive in order), one download stream, two backprojection
// streams -- forked once and joined once, so a scan's uploads, rebin and filter overlap the
// previous scans' backprojections.  Same kernels per scan as the graphs: bit-identical volumes.
static int batch_run_streamed(lct_batch* b, const float* const* fans, const int64_t* fan_view0,
                              float* const* images, int image_on_device, cudaStream_t s) {
  int st = streams_create(b->ss);
  while (!st && b->sev.size() < (size_t)kForkJoinEvents) {
    cudaEvent_t e;
    st = cuda_status(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    if (!st) b->sev.push_back(e);
  }
  for (int i = 1; i < 4 && !st; ++i) st = cuda_status(cudaEventRecord(b->ev[i], s));
  if (!st) st = streams_fork(b->ss, s, b->sev[0]);
  for (size_t i = 0; i < b->recs.size() && !st; ++i) {
    lct_recon* r = b->recs[i];
    if (!fans[i] || !images[i]) return LCT_ERR_ARG;
    const long long skip = r->fan_first + r->info.data_offset - fan_view0[i];
    if (skip < 0) return LCT_ERR_ARG;
    float* d_out = image_on_device ? images[i] : r->d_img;
    r->launches = 0;
    st = recon_run_streamed(r, fans[i], skip, d_out, d_out, image_on_device ? nullptr : images[i],
                            s, b->ss);
    b->launches += r->launches;
  }
  if (!st) st = streams_join(b->ss, s, b->sev.data() + 1);
  if (!st) st = cuda_status(cudaEventRecord(b->ev[4], s));
  if (!st) st = cuda_status(cudaEventRecord(b->ev[5], s));
  if (!st) st = cuda_status(cudaEventSynchronize(b->ev[5]));
  for (int i = 0; i < 5 && !st; ++i) cudaEventElapsedTime(&b->times[i], b->ev[i], b->ev[i + 1]);
  return st;
}

LCT_API int lct_batch_run(lct_batch* b, const float* const* fans, const int64_t* fan_view0,
                          int fan_on_device, float* const* images, int image_on_device,
                          lct_stream stream) {
  if (!b || !fans || !fan_view0 || !images) return LCT_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  int st;
  b->launches = 0;
  if ((st = cuda_status(cudaEventRecord(b->ev[0], s)))) return st;
  bool streamed = !fan_on_device;
  for (auto* r : b->recs) streamed = streamed && recon_streamable(r) && !r->cnn;
  if (streamed) return batch_run_streamed(b, fans, fan_view0, images, image_on_device, s);
  const cudaMemcpyKind up = fan_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  for (size_t i = 0; i < b->recs.size(); ++i) {
    lct_recon* r = b->recs[i];
    if (!fans[i] || !images[i]) return LCT_ERR_ARG;
    const long long skip = r->fan_first + r->info.data_offset - fan_view0[i];
    if (skip < 0) return LCT_ERR_ARG;
    if ((st = cuda_status(cudaMemcpyAsync(r->d_fan, fans[i] + skip * r->plane,
                                          sizeof(float) * r->fan_count * r->plane, up, s))))
      return st;
    ++b->launches;
  }
  for (int k = 0; k < 3; ++k) {
    if ((st = cuda_status(cudaEventRecord(b->ev[k + 1], s)))) return st;
    if ((st = cuda_status(cudaGraphLaunch(b->exec[k], s)))) return st;
    ++b->launches;
  }
  if ((st = cuda_status(cudaEventRecord(b->ev[4], s)))) return st;
  const cudaMemcpyKind down = image_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  for (size_t i = 0; i < b->recs.size(); ++i) {
    lct_recon* r = b->recs[i];
    const size_t bytes = sizeof(float) * (size_t)r->info.n_blocks_run * kBlockSlices *
                         r->info.ig.nx * r->info.ig.ny;
    if ((st = cuda_status(cudaMemcpyAsync(images[i], r->d_img, bytes, down, s)))) return st;
    ++b->launches;
  }
  if ((st = cuda_status(cudaEventRecord(b->ev[5], s)))) return st;
  if ((st = cuda_status(cudaEventSynchronize(b->ev[5])))) return st;
  for (int i = 0; i < 5; ++i) cudaEventElapsedTime(&b->times[i], b->ev[i], b->ev[i + 1]);
  return LCT_OK;
}

LCT_API int lct_batch_fan_range(const lct_batch* b, int scan, int64_t* first, int64_t* count) {
  if (!b || scan < 0 || scan >= (int)b->recs.size()) return LCT_ERR_ARG;
  return lct_recon_fan_range(b->recs[scan], first, count);
}

LCT_API int lct_batch_stats_get(const lct_batch* b, lct_recon_stats* total) {
  if (!b || !total) return LCT_ERR_ARG;
  lct_recon_stats t = {};
  for (auto* r : b->recs) {
    lct_recon_stats x;
    lct_recon_stats_get(r, &x);
    t.voxel_updates += x.voxel_updates;
    t.h2d_bytes += x.h2d_bytes;
    t.d2h_bytes += x.d2h_bytes;
    t.rebinned_views += x.rebinned_views;
  }
  t.launches = b->launches;
  *total = t;
  return LCT_OK;
}

LCT_API int lct_batch_last_times(const lct_batch* b, float* ms5) {
  if (!b || !ms5) return LCT_ERR_ARG;
  for (int i = 0; i < 5; ++i) ms5[i] = b->times[i];
  return LCT_OK;
}

LCT_API void lct_batch_destroy(lct_batch* b) { free_batch(b); }
