// Whole reconstruction: FDKReconstructor::reconstruct (Src/Reconstructor.cpp:30-49) with the
// stages ReconstrctorAbstractFactory builds (Src/ReconstructorAbstractFactory.cpp:11-33).
//
// Ownership follows the reference's GPUMemoryCtrl model (Include/GPUMemoryCtrl.h:6-62): one
// owner allocates each device buffer once, at lct_recon_create, sized from the plan; run()
// never allocates.  Buffers:
//   fan   fan views [fan_first, fan_first + fan_count) -- the union of every block's window
//   par   rebinned views, filtered in place:
//           block mode: n_angle views, reused by every block (the reference's projGpu)
//           scan mode:  global parallel views [g_first, g_first + g_count), each once
//   betas the ViewAngleFile contents (all readings); block b reads from
//         block_proj_start + add_projections (CUDA/Backprojector.cu:145)
//   img   n_blocks_run * 32 slices, block b at slice 32 b (CUDA/Backprojector.cu:158)
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <vector>

#include "lct_internal.h"

namespace lct {
const float* plan_angles(const lct_plan* p);
const lct_scan_params& plan_params(const lct_plan* p);
}  // namespace lct

#include "recon_internal.h"

namespace lct {

static void free_recon(lct_recon* r) {
  if (!r) return;
  cudaFree(r->d_fan);
  cudaFree(r->d_par);
  cudaFree(r->d_betas);
  cudaFree(r->d_h);
  cudaFree(r->d_img);
  cudaFree(r->d_quad);
  view_texture_destroy(r->vtex);
  view_texture_destroy(r->pi_tex);
  cudaFree(r->d_tc);
  cudaFree(r->d_plain);
  for (auto& e : r->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : r->ev_cnn)
    if (e) cudaEventDestroy(e);
  for (auto& e : r->sev)
    if (e) cudaEventDestroy(e);
  streams_destroy(r->ss);
  recon_free_bounded(r);
  delete r;
}

}  // namespace lct

using namespace lct;

LCT_API void lct_recon_opts_default(lct_recon_opts* o) {
  if (!o) return;
  o->mode = LCT_MODE_SCAN;
  o->rebinner = LCT_REBIN_FAN2PAR;
  o->preweight = LCT_PW_NONE;
  o->filter_kind = LCT_FILTER_RAMLAK;
  o->window = LCT_WINDOW_NONE;
  o->filter_mode = LCT_FILTER_FP32;
  o->backprojector = LCT_BP_PAR;
  o->interp = LCT_INTERP_TEX8;
  o->addr = LCT_ADDR_BORDER;
  o->bp_nz = 0;
  o->bp_minb = 0;
  o->bp_sampler = LCT_BP_SAMPLER_AUTO;
}

namespace lct {

// Options check and the plan-derived fields of a recon (no allocation).
int recon_setup(const lct_plan* plan, const lct_recon_opts* opts, lct_recon** out) {
  if (!plan || !out) return LCT_ERR_ARG;
  *out = nullptr;
  lct_recon_opts o;
  if (opts)
    o = *opts;
  else
    lct_recon_opts_default(&o);
  if (o.mode != LCT_MODE_BLOCK && o.mode != LCT_MODE_SCAN) return LCT_ERR_ARG;
  if (o.rebinner < LCT_REBIN_FAN2PAR || o.rebinner > LCT_REBIN_PI_ORI) return LCT_ERR_ARG;
  if (o.preweight != LCT_PW_NONE && o.preweight != LCT_PW_PI_ORI) return LCT_ERR_ARG;
  if (o.backprojector != LCT_BP_PAR && o.backprojector != LCT_BP_PI_ORI) return LCT_ERR_ARG;
  if (o.interp != LCT_INTERP_TEX8 && o.interp != LCT_INTERP_EXACT) return LCT_ERR_ARG;
  if (o.addr < LCT_ADDR_BORDER || o.addr > LCT_ADDR_LEGACY) return LCT_ERR_ARG;
  if (o.filter_mode < LCT_FILTER_FP32 || o.filter_mode > LCT_FILTER_BF16X6) return LCT_ERR_ARG;
  if (o.mode == LCT_MODE_SCAN && o.rebinner == LCT_REBIN_PI_ORI) return LCT_ERR_UNSUPPORTED;

  lct_recon* r = new (std::nothrow) lct_recon;
  if (!r) return LCT_ERR_ALLOC;
  r->o = o;
  lct_plan_info_get(plan, &r->info);
  const lct_geom& g = r->info.ctg;
  const int nb = r->info.n_blocks_run;
  if (nb <= 0 || nb > kBpMaxSlabs) {
    delete r;
    return nb <= 0 ? LCT_ERR_RANGE : LCT_ERR_UNSUPPORTED;
  }
  for (int b = 0; b < nb; ++b) {
    lct_block_info bi;
    lct_plan_block(plan, r->info.first_block + b, &bi);
    r->blocks.push_back(bi);
  }
  r->plane = (long long)g.nt * g.ns;
  long long lo = r->blocks[0].block_proj_start, hi = lo + g.n_angle_add;
  for (auto& bi : r->blocks) {
    lo = std::min<long long>(lo, bi.block_proj_start);
    hi = std::max<long long>(hi, (long long)bi.block_proj_start + g.n_angle_add);
  }
  const long long readings = r->info.n_readings;
  const long long off = r->info.data_offset;
  if (lo + off < 0 || hi + off > readings) {
    // the reference would read outside the raw file here (Src/DataReader.cpp:14)
    delete r;
    return LCT_ERR_RANGE;
  }
  r->fan_first = lo;
  r->fan_count = hi - lo;
  r->g_first = lo + g.add_projections;
  r->g_count = r->fan_count - 2LL * g.add_projections;
  cudaGetDevice(&r->device);
  {
    // sum of the reference's per-voxel view counts (same windows in every block)
    const float dzv = g.pitch / (float)g.n_proj_turn;
    long long per_block = 0;
    for (int z = 0; z < kBlockSlices; ++z) {
      BpWindow w = bp_window(g, r->info.ig, z, dzv, g.n_proj_turn / 2);
      per_block += (long long)(w.a_max - w.a_min) * r->info.ig.nx * r->info.ig.ny;
    }
    r->voxel_updates = per_block * nb;
  }
  r->quads = o.backprojector == LCT_BP_PAR && bp_windows_full(g, r->info.ig, kBlockSlices);
  r->tex_bp = want_texture(o, r->quads);
  r->tma_bp = r->quads && !r->tex_bp && o.interp == LCT_INTERP_EXACT &&
              o.bp_sampler == LCT_BP_SAMPLER_QUADS_TMA;
  *out = r;
  return LCT_OK;
}

// Allocations every recon has: view angles, taps, the tensor-core filter's operands for
// tc_rows rows (BF16 modes), timing events.
int recon_alloc_common(lct_recon* r, const lct_plan* plan) {
  const lct_geom& g = r->info.ctg;
  const long long readings = r->info.n_readings;
  int st;
  auto track = [&](size_t bytes) { r->device_bytes += (long long)bytes; };
  if ((st = cuda_status(cudaMalloc(&r->d_betas, sizeof(float) * readings)))) return st;
  track(sizeof(float) * readings);
  if ((st = cuda_status(cudaMalloc(&r->d_h, sizeof(float) * 2 * g.ns)))) return st;
  track(sizeof(float) * 2 * g.ns);
  if ((st = cuda_status(cudaMemcpy(r->d_betas, plan_angles(plan), sizeof(float) * readings,
                                   cudaMemcpyHostToDevice))))
    return st;
  std::vector<float> h(2 * (size_t)g.ns);
  if ((st = lct_filter_taps(r->o.filter_kind, r->o.window, g.ns, g.ds, h.data()))) return st;
  if ((st = cuda_status(cudaMemcpy(r->d_h, h.data(), sizeof(float) * h.size(),
                                   cudaMemcpyHostToDevice))))
    return st;
  if (r->o.filter_mode != LCT_FILTER_FP32) {
    const size_t b = tc_scratch_bytes(g.ns, r->tc_rows, r->o.filter_mode);
    if ((st = cuda_status(cudaMalloc(&r->d_tc, b)))) return st;
    track(b);
    if ((st = tc_build_toeplitz(g.ns, r->d_h, r->d_tc, r->o.filter_mode, 0))) return st;
    if ((st = cuda_status(cudaDeviceSynchronize()))) return st;
  }
  for (auto& e : r->ev)
    if ((st = cuda_status(cudaEventCreate(&e)))) return st;
  return LCT_OK;
}

int recon_alloc_status(int st) {
  return st == LCT_ERR_CUDA && lct_last_cuda_error() == cudaErrorMemoryAllocation ? LCT_ERR_ALLOC : st;
}

}  // namespace lct

LCT_API int lct_recon_create(const lct_plan* plan, const lct_recon_opts* opts, lct_recon** out) {
  lct_recon* r = nullptr;
  int st = recon_setup(plan, opts, &r);
  if (st) return st;
  const lct_recon_opts& o = r->o;
  const lct_geom& g = r->info.ctg;
  const int nb = r->info.n_blocks_run;
  const long long par_views = o.mode == LCT_MODE_SCAN ? r->g_count : g.n_angle;
  const size_t img_elems = (size_t)nb * kBlockSlices * r->info.ig.nx * r->info.ig.ny;
  auto alloc = [&](void** p, size_t bytes) {
    int e = cuda_status(cudaMalloc(p, bytes));
    if (!e) r->device_bytes += (long long)bytes;
    return e;
  };
  do {
    if ((st = alloc((void**)&r->d_fan, sizeof(float) * r->fan_count * r->plane))) break;
    if ((st = alloc((void**)&r->d_par, sizeof(float) * par_views * r->plane))) break;
    if ((st = alloc((void**)&r->d_img, sizeof(float) * img_elems))) break;
    if (r->tex_bp) {
      // a 3-D texture holds at most the device's depth limit of views: beyond it, quads
      if ((st = view_texture_create(r->vtex, g.ns, g.nt, par_views,
                                    o.addr == LCT_ADDR_CLAMP ? LCT_ADDR_CLAMP : LCT_ADDR_BORDER))) {
        if (st != LCT_ERR_UNSUPPORTED) break;
        r->tex_bp = false;
        st = LCT_OK;
      } else {
        r->device_bytes += (long long)sizeof(float) * par_views * r->plane;
      }
    }
    if (r->quads && !r->tex_bp &&
        (st = alloc((void**)&r->d_quad, sizeof(float4) * par_views * quad_view_elems(g.ns, g.nt))))
      break;
    if (o.rebinner == LCT_REBIN_PI_ORI && o.interp == LCT_INTERP_TEX8) {
      // the fan block as a 3-D texture once per recon, with both addressings (legacy addressing
      // clamps the first block), instead of an array allocated and freed per block
      if ((st = view_texture_create(r->pi_tex, g.ns, g.nt, g.n_angle_add, LCT_ADDR_BORDER)) ||
          (st = view_texture_add_other_mode(r->pi_tex))) {
        if (st != LCT_ERR_UNSUPPORTED) break;
        view_texture_destroy(r->pi_tex);  // beyond the texture limits: the per-call path
        st = LCT_OK;
      } else {
        r->device_bytes += (long long)sizeof(float) * g.n_angle_add * r->plane;
      }
    }
    if (r->tma_bp && bp_tma_map(&r->tma_map, r->d_quad, g.ns, g.nt, par_views) != LCT_OK)
      r->tma_bp = false;  // no tensor-map encoder in this driver: the L1 quad kernel
    if (o.filter_mode != LCT_FILTER_FP32) r->tc_rows = par_views * g.nt;
    st = recon_alloc_common(r, plan);
  } while (0);
  if (st) {
    free_recon(r);
    return recon_alloc_status(st);
  }
  if (o.bp_nz == -1 && (st = lct_recon_autotune(r, nullptr, nullptr))) {
    free_recon(r);
    return st;
  }
  *out = r;
  return LCT_OK;
}

namespace lct {
int recon_stage_bp(lct_recon* r, float* d_img, cudaStream_t s);
}

// Backprojection autotuner: times the quad kernel over slices per thread x CTAs per SM on this
// recon's own buffers and keeps the fastest; results are cached per geometry class (detector,
// volume, window, interpolation and views-per-slice), so a class is tuned once per process.
LCT_API int lct_recon_autotune(lct_recon* r, int* nz_out, int* minb_out) {
  if (r && r->bounded) return LCT_ERR_UNSUPPORTED;  // no whole-scan buffers to time on
  if (!r) return LCT_ERR_ARG;
  const lct_geom& g = r->info.ctg;
  const lct_img& ig = r->info.ig;
  if (r->o.mode != LCT_MODE_SCAN || !r->quads || r->o.addr == LCT_ADDR_LEGACY) {
    if (nz_out) *nz_out = pick_bp_nz(g, ig, r->o.bp_nz);
    if (minb_out) *minb_out = r->o.bp_minb > 0 ? r->o.bp_minb : 4;
    return LCT_OK;
  }
  static std::mutex mu;
  static std::map<std::vector<long long>, std::pair<int, int>> cache;
  const std::vector<long long> key = {g.ns, g.nt, ig.nx, ig.ny, g.n_angle, g.n_proj_turn,
                                      r->o.interp, (long long)(1000.0 * g.pitch / ig.dz),
                                      (long long)r->info.n_blocks_run, (long long)r->tex_bp,
                                      (long long)r->tma_bp};
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) {
      r->o.bp_nz = it->second.first;
      r->o.bp_minb = it->second.second;
      if (nz_out) *nz_out = r->o.bp_nz;
      if (minb_out) *minb_out = r->o.bp_minb;
      return LCT_OK;
    }
  }
  cudaStream_t s;
  int st = cuda_status(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  if (st) return st;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const size_t qbytes = sizeof(float4) * (size_t)r->g_count * quad_view_elems(g.ns, g.nt);
  if (!r->tex_bp) st = cuda_status(cudaMemsetAsync(r->d_quad, 0, qbytes, s));
  float best = 1e30f;
  int bnz = 8, bmb = 4;
  const int nzs[3] = {4, 8, 16}, mbs[3] = {2, 3, 4};
  for (int i = 0; i < 3 && !st; ++i)
    for (int j = 0; j < 3 && !st; ++j) {
      r->o.bp_nz = nzs[i];
      r->o.bp_minb = mbs[j];
      if ((st = recon_stage_bp(r, r->d_img, s))) break;  // warm
      cudaEventRecord(e0, s);
      if ((st = recon_stage_bp(r, r->d_img, s))) break;
      cudaEventRecord(e1, s);
      if ((st = cuda_status(cudaEventSynchronize(e1)))) break;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best) {
        best = ms;
        bnz = nzs[i];
        bmb = mbs[j];
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(s);
  r->o.bp_nz = bnz;
  r->o.bp_minb = bmb;
  if (st) return st;
  {
    std::lock_guard<std::mutex> lock(mu);
    cache[key] = {bnz, bmb};
  }
  if (nz_out) *nz_out = bnz;
  if (minb_out) *minb_out = bmb;
  return LCT_OK;
}

LCT_API int lct_recon_fan_range(const lct_recon* r, int64_t* first, int64_t* count) {
  if (!r) return LCT_ERR_ARG;
  if (first) *first = r->fan_first + r->info.data_offset;
  if (count) *count = r->fan_count;
  return LCT_OK;
}

LCT_API int lct_recon_stats_get(const lct_recon* r, lct_recon_stats* out) {
  if (!r || !out) return LCT_ERR_ARG;
  out->voxel_updates = r->voxel_updates;
  out->h2d_bytes = r->fan_count * r->plane * (long long)sizeof(float);
  out->d2h_bytes = (long long)r->info.n_blocks_run * kBlockSlices * r->info.ig.nx * r->info.ig.ny *
                   (long long)sizeof(float);
  out->rebinned_views = r->o.mode == LCT_MODE_SCAN ? r->g_count
                                                   : (long long)r->info.n_blocks_run * r->info.ctg.n_angle;
  out->launches = r->launches;
  return LCT_OK;
}

LCT_API int lct_recon_last_times(const lct_recon* r, float* ms5) {
  if (!r || !ms5) return LCT_ERR_ARG;
  std::memcpy(ms5, r->times, sizeof(r->times));
  return LCT_OK;
}

static int run_rebin(lct_recon* r, const lct_geom& g, const float* fan_block, float* par, int addr,
                     cudaStream_t s) {
  const int interp = r->o.interp;
  switch (r->o.rebinner) {
    case LCT_REBIN_NULL: return lct_rebin_null(&g, fan_block, par, addr, s);
    case LCT_REBIN_PI_ORI:
      if (interp == LCT_INTERP_TEX8 && r->pi_tex.arr)  // the recon's own texture of the fan block
        return launch_rebin_pi_ori_tex(g, r->pi_tex, addr, fan_block, par, s);
      return lct_rebin_pi_ori(&g, fan_block, par, interp, addr, s);
    default: return lct_rebin_fan2par(&g, fan_block, par, interp, addr, s);
  }
}

static int run_filter(lct_recon* r, const lct_geom& g, long long nrows, cudaStream_t s) {
  if (r->o.filter_mode != LCT_FILTER_FP32)
    return tc_filter(g.ns, r->d_par, nrows, r->d_tc, r->tc_rows, r->o.filter_mode, s);
  return launch_filter_rows(g.ns, r->d_h, r->d_par, nrows, LCT_FILTER_FP32, s);
}

// Block mode: the reference's per-block flow, every stage per block.
static int run_blocks(lct_recon* r, const float* d_fan, float* d_img, cudaStream_t s) {
  const lct_geom& g = r->info.ctg;
  const lct_img& ig = r->info.ig;
  const long long slab = (long long)kBlockSlices * ig.nx * ig.ny;
  const int bp_nz = pick_bp_nz(g, ig, r->o.bp_nz);
  int st;
  for (int b = 0; b < r->info.n_blocks_run; ++b) {
    const lct_block_info& bi = r->blocks[b];
    const int addr = block_addr(r, b);
    const float* fan_block = d_fan + (bi.block_proj_start - r->fan_first) * r->plane;
    if ((st = run_rebin(r, g, fan_block, r->d_par, addr, s))) return st;
    r->launches++;
    if (r->o.preweight == LCT_PW_PI_ORI) {
      if ((st = lct_weight_pi_ori(&g, r->d_par, s))) return st;
      r->launches++;
    }
    if ((st = run_filter(r, g, (long long)g.n_angle * g.nt, s))) return st;
    r->launches += filter_launches(r->o.filter_mode);
    const float* betas = r->d_betas + bi.block_proj_start + g.add_projections;
    float* img_b = d_img + (long long)b * slab;
    if (r->o.backprojector == LCT_BP_PI_ORI) {
      st = lct_backproject_pi_ori(&g, &ig, betas, r->d_par, img_b, r->o.interp, addr, s);
    } else {
      BpLaunch L;
      L.proj = r->d_par;
      L.betas = betas;
      L.img = img_b;
      L.view_stride = r->plane;
      L.n_angle = g.n_angle;
      L.nz = kBlockSlices;
      L.n_slabs = 1;
      L.slab_view[0] = 0;
      L.slab_z0[0] = 0;
      L.interp = r->o.interp;
      L.addr = addr;
      L.nz_thread = bp_nz;
      L.minb = r->o.bp_minb;
      if (r->quads) {
        if ((st = recon_pack(r, r->d_par, g.n_angle, 0, addr, s))) return st;
        r->launches++;
        st = recon_bp_pairs(r, L, s);
      } else {
        st = launch_bp_par(g, ig, L, s);
      }
    }
    if (st) return st;
    r->launches++;
  }
  return LCT_OK;
}

namespace lct {

// Scan mode, stage 1: rebin every global view once (FP64 per-column shifts), pre-weight.
int recon_stage_rebin(lct_recon* r, const float* d_fan, cudaStream_t s) {
  const lct_geom& g = r->info.ctg;
  const int addr0 = r->o.addr == LCT_ADDR_CLAMP ? LCT_ADDR_CLAMP : LCT_ADDR_BORDER;
  int st;
  if (r->o.rebinner == LCT_REBIN_NULL) {
    lct_geom gg = g;
    gg.n_angle = (int)r->g_count;
    gg.n_angle_add = (int)r->fan_count;
    if ((st = lct_rebin_null(&gg, d_fan, r->d_par, addr0, s))) return st;
  } else {
    if ((st = launch_rebin_fan2par_scan(g, d_fan, r->fan_first, r->fan_count, r->d_par,
                                        r->g_first, r->g_count, r->o.interp, addr0, s)))
      return st;
  }
  r->launches++;
  if (r->o.preweight == LCT_PW_PI_ORI) {
    lct_geom gg = g;
    gg.n_angle = (int)r->g_count;
    gg.n_angle_add = (int)r->g_count;
    if ((st = lct_weight_pi_ori(&gg, r->d_par, s))) return st;
    r->launches++;
  }
  return LCT_OK;
}

// Scan mode, stage 2: filter every rebinned view once, pack the backprojector's quads.
int recon_stage_filter(lct_recon* r, cudaStream_t s) {
  const lct_geom& g = r->info.ctg;
  int st;
  if ((st = run_filter(r, g, r->g_count * g.nt, s))) return st;
  r->launches += filter_launches(r->o.filter_mode);
  if (r->quads && r->o.backprojector == LCT_BP_PAR) {
    // border-addressed quads; a clamped (legacy first) slab reads the FP32 views directly
    const int packed = r->o.addr == LCT_ADDR_CLAMP ? LCT_ADDR_CLAMP : LCT_ADDR_BORDER;
    if ((st = recon_pack(r, r->d_par, r->g_count, 0, packed, s))) return st;
    r->launches++;
  }
  return LCT_OK;
}

// Scan mode, stage 3: the launch description of the slabs [b0, b1) (one addressing mode).
void recon_bp_launch(const lct_recon* r, int b0, int b1, float* d_img, BpLaunch& L) {
  const lct_geom& g = r->info.ctg;
  L.proj = r->d_par;
  L.img = d_img;
  L.view_stride = r->plane;
  L.n_angle = g.n_angle;
  L.nz = kBlockSlices;
  L.n_slabs = b1 - b0;
  for (int b = b0; b < b1; ++b) {
    const long long gv = r->blocks[b].block_proj_start + g.add_projections;
    L.slab_view[b - b0] = (int)(gv - r->g_first);
    L.slab_z0[b - b0] = b * kBlockSlices;
  }
  L.interp = r->o.interp;
  L.addr = block_addr(r, b0);
  L.nz_thread = pick_bp_nz(g, r->info.ig, r->o.bp_nz);
  L.minb = r->o.bp_minb;
  // betas are indexed by the same slab offset: shift the base by g_first
  L.betas = r->d_betas + r->g_first;
}

int recon_pack(lct_recon* r, const float* par, long long nv, long long v0, int addr, cudaStream_t s) {
  const lct_geom& g = r->info.ctg;
  if (r->tex_bp) return view_texture_fill(r->vtex, par, nv, v0, s);
  if (r->quad_ring > 0)
    return launch_quad_pack(par, nv, g.ns, g.nt, addr, r->d_quad, s, v0, r->quad_ring);
  return launch_quad_pack(par, nv, g.ns, g.nt, addr, r->d_quad + v0 * quad_view_elems(g.ns, g.nt), s);
}

int recon_bp_pairs(lct_recon* r, BpLaunch& L, cudaStream_t s) {
  L.quad_ring = r->quad_ring;
  if (r->tex_bp) return launch_bp_par_texture(r->info.ctg, r->info.ig, L, r->vtex.tex, s);
  if (r->tma_bp) return launch_bp_par_quads_tma(r->info.ctg, r->info.ig, L, r->d_quad, r->tma_map, s);
  return launch_bp_par_quads(r->info.ctg, r->info.ig, L, r->d_quad, s);
}

bool recon_bp_quads_all(const lct_recon* r) {
  return r->quads && !r->tex_bp && r->o.backprojector == LCT_BP_PAR &&
         r->o.addr != LCT_ADDR_LEGACY;
}

int recon_stage_bp(lct_recon* r, float* d_img, cudaStream_t s) {
  const lct_geom& g = r->info.ctg;
  const lct_img& ig = r->info.ig;
  const int nb = r->info.n_blocks_run;
  const long long slab = (long long)kBlockSlices * ig.nx * ig.ny;
  int st;
  if (r->o.backprojector == LCT_BP_PI_ORI) {
    for (int b = 0; b < nb; ++b) {
      const long long gv = r->blocks[b].block_proj_start + g.add_projections;
      st = lct_backproject_pi_ori(&g, &ig, r->d_betas + gv, r->d_par + (gv - r->g_first) * r->plane,
                                  d_img + (long long)b * slab, r->o.interp, block_addr(r, b), s);
      if (st) return st;
      r->launches++;
    }
    return LCT_OK;
  }
  // one launch over every slab; with LEGACY addressing slab 0 runs apart (clamped)
  int b0 = 0;
  while (b0 < nb) {
    const int addr = block_addr(r, b0);
    int b1 = b0 + 1;
    while (b1 < nb && block_addr(r, b1) == addr) ++b1;
    BpLaunch L;
    recon_bp_launch(r, b0, b1, d_img, L);
    const int packed = r->o.addr == LCT_ADDR_CLAMP ? LCT_ADDR_CLAMP : LCT_ADDR_BORDER;
    if (r->quads && addr == packed)
      st = recon_bp_pairs(r, L, s);
    else
      st = launch_bp_par(g, ig, L, s);
    if (st) return st;
    r->launches++;
    b0 = b1;
  }
  return LCT_OK;
}

}  // namespace lct

// Scan mode from a HOST fan buffer with the copies overlapped: slabs are taken in the order their
// view windows end; for each, the fan views up to that end are uploaded on a copy stream, the
// new global views are rebinned, filtered and packed on the compute stream, and the slab is
// backprojected on one of two alternating streams, the first slab in parts as its views land
// (the new views come in pieces of at most 512, each uploaded, then rebinned, filtered and
// packed); its volume -- or, with a network attached, the corrected slab once the slabs
// on either side are backprojected -- is downloaded on a second copy stream.  Every view is
// uploaded, rebinned and filtered once by the same kernels as the unstreamed run, so the volume
// is bit-identical to it.
namespace lct {

int streams_create(StreamSet& ss) {
  cudaStream_t* all[5] = {&ss.up, &ss.down, &ss.bp[0], &ss.bp[1], &ss.cnn};
  for (auto* a : all) {
    if (*a) continue;
    const int st = cuda_status(cudaStreamCreateWithFlags(a, cudaStreamNonBlocking));
    if (st) return st;
  }
  if (!ss.prep) {
    const int st = cuda_status(cudaStreamCreateWithFlags(&ss.prep, cudaStreamNonBlocking));
    if (st) return st;
  }
  return LCT_OK;
}

void streams_destroy(StreamSet& ss) {
  for (cudaStream_t* a : {&ss.up, &ss.down, &ss.bp[0], &ss.bp[1], &ss.cnn, &ss.prep})
    if (*a) {
      cudaStreamDestroy(*a);
      *a = nullptr;
    }
}

int streams_fork(const StreamSet& ss, cudaStream_t s, cudaEvent_t ev) {
  int st = cuda_status(cudaEventRecord(ev, s));
  for (cudaStream_t x : {ss.up, ss.down, ss.bp[0], ss.bp[1], ss.cnn, ss.prep})
    if (!st) st = cuda_status(cudaStreamWaitEvent(x, ev, 0));
  return st;
}

int streams_join(const StreamSet& ss, cudaStream_t s, const cudaEvent_t* ev5) {
  // uploads end in prep already
  const cudaStream_t x[5] = {ss.down, ss.bp[0], ss.bp[1], ss.cnn, ss.prep};
  int st = LCT_OK;
  for (int i = 0; i < 5 && !st; ++i) {
    st = cuda_status(cudaEventRecord(ev5[i], x[i]));
    if (!st) st = cuda_status(cudaStreamWaitEvent(s, ev5[i], 0));
  }
  return st;
}

bool recon_streamable(const lct_recon* r) {
  return r->o.mode == LCT_MODE_SCAN && r->o.rebinner == LCT_REBIN_FAN2PAR &&
         r->o.preweight == LCT_PW_NONE && r->o.backprojector == LCT_BP_PAR;
}

constexpr long long kStreamPiece = 512;  // global views per upload / rebin / filter piece

int recon_run_streamed(lct_recon* r, const float* fan_host, long long skip, float* d_img,
                       float* d_out, float* image_host, cudaStream_t s, const StreamSet& ss) {
  const lct_geom& g = r->info.ctg;
  const lct_img& ig = r->info.ig;
  const int nb = r->info.n_blocks_run;
  const long long slab = (long long)kBlockSlices * ig.nx * ig.ny;
  const long long plane = r->plane;
  int st;
  const cudaStream_t sp = ss.prep;  // per-piece rebin / filter / pack
  (void)s;                          // the caller forks the set from s and joins it back
  // events: the caller's fork and join, per slab: views ready, backprojected, corrected;
  // per piece: uploaded, packed
  // + the first slab's short pieces (the pivot and at most 64 doublings up to a full piece)
  const long long n_pieces = r->g_count / kStreamPiece + nb + 2 + 64;
  const size_t n_ev = kForkJoinEvents + 3 * (size_t)nb + 2 * (size_t)n_pieces;
  while (r->sev.size() < n_ev) {
    cudaEvent_t e;
    if ((st = cuda_status(cudaEventCreateWithFlags(&e, cudaEventDisableTiming)))) return st;
    r->sev.push_back(e);
  }
  cudaEvent_t* ev_views = r->sev.data() + kForkJoinEvents;
  cudaEvent_t* ev_bp = ev_views + nb;
  cudaEvent_t* ev_cnn = ev_bp + nb;
  cudaEvent_t* ev_up = ev_cnn + nb;
  cudaEvent_t* ev_packed = ev_up + n_pieces;
  long long piece = 0;

  // fan views a range of global views reads (the scan rebin's column shifts, in FP64)
  const double smax = (((double)(g.ns - 1) - (double)g.ws) * (double)g.ds / (double)g.dso) /
                      (double)g.orbit;
  const long long shift_hi = (long long)std::floor(smax) + 1;
  std::vector<int> order(nb);
  std::vector<long long> gfirst(nb), gend(nb);
  for (int b = 0; b < nb; ++b) {
    order[b] = b;
    gfirst[b] = r->blocks[b].block_proj_start + g.add_projections;
    gend[b] = gfirst[b] + g.n_angle;
  }
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return gend[x] < gend[y]; });
  const int addr0 = r->o.addr == LCT_ADDR_CLAMP ? LCT_ADDR_CLAMP : LCT_ADDR_BORDER;
  const int packed = addr0;
  long long done = r->g_first, up = 0;  // global views rebinned so far; fan views uploaded
  std::vector<char> bp_done(nb, 0), cnn_done(nb, 0);
  auto download = [&](int b, const float* src, cudaEvent_t after) -> int {
    if (!image_host) return LCT_OK;
    int e = cuda_status(cudaStreamWaitEvent(ss.down, after, 0));
    if (!e)
      e = cuda_status(cudaMemcpyAsync(image_host + b * slab, src + b * slab, sizeof(float) * slab,
                                      cudaMemcpyDeviceToHost, ss.down));
    return e;
  };
  auto bp = [&](int b, int lo, int hi, int part, cudaStream_t sb) -> int {
    BpLaunch L;
    recon_bp_launch(r, b, b + 1, d_img, L);
    L.view_lo = lo;
    L.view_hi = hi;
    L.part = part;
    const int addr = block_addr(r, b);
    const int e = (r->quads && addr == packed) ? recon_bp_pairs(r, L, sb)
                                               : launch_bp_par(g, ig, L, sb);
    if (!e) r->launches++;
    return e;
  };
  for (int k = 0; k < nb; ++k) {
    const int b = order[k];
    cudaStream_t sb = ss.bp[k & 1];
    // the first slab is backprojected in parts as its views arrive (the others' windows are
    // complete by the time their turn comes); only the quad kernel carries parts
    const bool split = k == 0 && r->quads && block_addr(r, b) == packed;
    const long long slab_end = std::min(gend[b], r->g_first + r->g_count);
    int bp_lo = 0, parts = 0;
    while (slab_end > done) {
      long long target = std::min(slab_end, done + kStreamPiece);
      if (split) target = first_part_target(done, target, gfirst[b], g.n_proj_turn / 2);
      const long long need = std::min(r->fan_count, target - 1 + shift_hi + 1 - r->fan_first);
      if (piece >= n_pieces) return LCT_ERR_ARG;  // cannot happen: pieces are counted above
      if (need > up) {
        if ((st = cuda_status(cudaMemcpyAsync(r->d_fan + up * plane, fan_host + (skip + up) * plane,
                                              sizeof(float) * (need - up) * plane,
                                              cudaMemcpyHostToDevice, ss.up))))
          return st;
        up = need;
      }
      if ((st = cuda_status(cudaEventRecord(ev_up[piece], ss.up)))) return st;
      if ((st = cuda_status(cudaStreamWaitEvent(sp, ev_up[piece], 0)))) return st;
      const long long v0 = done - r->g_first, nv = target - done;
      float* par = r->d_par + v0 * plane;
      if ((st = launch_rebin_fan2par_scan(g, r->d_fan, r->fan_first, r->fan_count, par, done, nv,
                                          r->o.interp, addr0, sp)))
        return st;
      r->launches++;
      if (r->o.filter_mode != LCT_FILTER_FP32)
        st = tc_filter(g.ns, par, nv * g.nt, r->d_tc, r->tc_rows, r->o.filter_mode, sp);
      else
        st = launch_filter_rows(g.ns, r->d_h, par, nv * g.nt, LCT_FILTER_FP32, sp);
      if (st) return st;
      r->launches += filter_launches(r->o.filter_mode);
      if (r->quads) {
        if ((st = recon_pack(r, par, nv, v0, packed, sp))) return st;
        r->launches++;
      }
      done = target;
      if ((st = cuda_status(cudaEventRecord(ev_packed[piece], sp)))) return st;
      ++piece;
      // a pair starting at local view ia also reads its conjugate ia + half: a part takes the
      // pair starts whose conjugates are packed too
      const long long local = std::min<long long>(done - gfirst[b], g.n_angle);
      const int avail = (int)std::max<long long>(local - g.n_proj_turn / 2, 0);
      if (split && done < slab_end && avail > bp_lo) {
        if ((st = cuda_status(cudaStreamWaitEvent(sb, ev_packed[piece - 1], 0)))) return st;
        if ((st = bp(b, bp_lo, avail, parts ? kBpMiddle : kBpFirst, sb))) return st;
        bp_lo = avail;
        ++parts;
      }
    }
    // every view of the slab's window is packed
    if ((st = cuda_status(cudaEventRecord(ev_views[k], sp)))) return st;
    if ((st = cuda_status(cudaStreamWaitEvent(sb, ev_views[k], 0)))) return st;
    if ((st = parts ? bp(b, bp_lo, g.n_angle, kBpLast, sb) : bp(b, 0, 1 << 30, kBpWhole, sb)))
      return st;
    bp_done[b] = 1;
    if ((st = cuda_status(cudaEventRecord(ev_bp[b], sb)))) return st;
    if (!r->cnn) {
      if ((st = download(b, d_out, ev_bp[b]))) return st;
      continue;
    }
    // corrected slabs whose 5-slice inputs are now all backprojected (one stream: the network's
    // workspace is shared by its passes)
    for (int c = std::max(0, b - 1); c <= std::min(nb - 1, b + 1); ++c) {
      if (cnn_done[c] || !bp_done[c] || (c > 0 && !bp_done[c - 1]) || (c + 1 < nb && !bp_done[c + 1]))
        continue;
      for (int n = std::max(0, c - 1); n <= std::min(nb - 1, c + 1); ++n)
        if ((st = cuda_status(cudaStreamWaitEvent(ss.cnn, ev_bp[n], 0)))) return st;
      if ((st = cnn_infer_range(r->cnn, d_img, d_out, nb * kBlockSlices, c * kBlockSlices,
                                (c + 1) * kBlockSlices, r->cnn_bound, ss.cnn)))
        return st;
      r->launches += 9 * cnn_passes(r->cnn, kBlockSlices);
      cnn_done[c] = 1;
      if ((st = cuda_status(cudaEventRecord(ev_cnn[c], ss.cnn)))) return st;
      if ((st = download(c, d_out, ev_cnn[c]))) return st;
    }
  }
  return LCT_OK;
}

}  // namespace lct

LCT_API int lct_recon_run(lct_recon* r, const float* fan, int64_t fan_view0, int fan_on_device,
                          float* image, int image_on_device, lct_stream stream) {
  if (!r || !fan || !image) return LCT_ERR_ARG;
  if (fan_view0 < 0 || fan_view0 > r->fan_first + r->info.data_offset) return LCT_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const lct_img& ig = r->info.ig;
  const int nb = r->info.n_blocks_run;
  const long long off = r->info.data_offset;
  int st;
  if (r->bounded)  // rings: always the overlapped pipeline, from the run's first fan view
    return recon_run_bounded_ptr(r, fan + (r->fan_first + off - fan_view0) * r->plane,
                                 fan_on_device != 0, image, image_on_device != 0, s);
  r->launches = 0;
  r->streamed = false;
  if ((st = cuda_status(cudaEventRecord(r->ev[0], s)))) return st;

  // fan views needed by the run (the union of the blocks' windows)
  const float* d_fan;
  const long long skip = r->fan_first + off - fan_view0;  // views before the run's first
  if (!fan_on_device && recon_streamable(r)) {
    // host fan: copies overlapped with the compute; one span reported as backprojection
    float* d_out = image_on_device ? image : r->d_img;
    float* d_img = r->cnn ? r->d_plain : d_out;
    r->streamed = true;
    if (r->cnn && (st = cnn_reset_rejects(r->cnn, s))) return st;
    for (int i = 1; i < 4; ++i)
      if ((st = cuda_status(cudaEventRecord(r->ev[i], s)))) return st;
    if ((st = streams_create(r->ss))) return st;
    while (r->sev.size() < (size_t)kForkJoinEvents) {
      cudaEvent_t e;
      if ((st = cuda_status(cudaEventCreateWithFlags(&e, cudaEventDisableTiming)))) return st;
      r->sev.push_back(e);
    }
    // the other streams start after everything already queued on s (an earlier run included)
    if ((st = streams_fork(r->ss, s, r->sev[0]))) return st;
    // a pageable volume is downloaded once, after the pipeline: slab downloads into it would each
    // hold this thread until the slab is backprojected
    const bool host_slabs = !image_on_device && host_pinned(image);
    if ((st = recon_run_streamed(r, fan, skip, d_img, d_out, host_slabs ? image : nullptr, s,
                                 r->ss)))
      return st;
    if ((st = streams_join(r->ss, s, r->sev.data() + 1))) return st;
    if (!image_on_device && !host_slabs &&
        (st = cuda_status(cudaMemcpyAsync(image, d_out, sizeof(float) * nb * kBlockSlices *
                                                            (long long)ig.nx * ig.ny,
                                          cudaMemcpyDeviceToHost, s))))
      return st;
    if ((st = cuda_status(cudaEventRecord(r->ev[4], s)))) return st;
    if ((st = cuda_status(cudaEventRecord(r->ev[5], s)))) return st;
    if ((st = cuda_status(cudaEventSynchronize(r->ev[5])))) return st;
    for (int i = 0; i < 5; ++i) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, r->ev[i], r->ev[i + 1]);
      r->times[i] = ms;
    }
    r->cnn_ms = 0.f;  // interleaved with the backprojection: not separable
    return LCT_OK;
  }
  if (fan_on_device) {
    d_fan = fan + skip * r->plane;
  } else {
    if ((st = cuda_status(cudaMemcpyAsync(r->d_fan, fan + skip * r->plane,
                                          sizeof(float) * r->fan_count * r->plane,
                                          cudaMemcpyHostToDevice, s))))
      return st;
    d_fan = r->d_fan;
  }
  if ((st = cuda_status(cudaEventRecord(r->ev[1], s)))) return st;
  float* d_out = image_on_device ? image : r->d_img;
  float* d_img = r->cnn ? r->d_plain : d_out;  // backprojection target
  const long long slab = (long long)kBlockSlices * ig.nx * ig.ny;

  if (r->o.mode == LCT_MODE_BLOCK) {
    // stages interleave per block; the whole compute span is reported as backprojection
    cudaEventRecord(r->ev[2], s);
    cudaEventRecord(r->ev[3], s);
    if ((st = run_blocks(r, d_fan, d_img, s))) return st;
    cudaEventRecord(r->ev[4], s);
  } else {
    if ((st = recon_stage_rebin(r, d_fan, s))) return st;
    if ((st = cuda_status(cudaEventRecord(r->ev[2], s)))) return st;
    if ((st = recon_stage_filter(r, s))) return st;
    if ((st = cuda_status(cudaEventRecord(r->ev[3], s)))) return st;
    if ((st = recon_stage_bp(r, d_img, s))) return st;
    if ((st = cuda_status(cudaEventRecord(r->ev[4], s)))) return st;
  }
  if (r->cnn) {  // fused learned correction: plain volume -> gated corrected volume
    if ((st = cuda_status(cudaEventRecord(r->ev_cnn[0], s)))) return st;
    if ((st = lct_cnn_infer_volume(r->cnn, d_img, d_out, nb * kBlockSlices, r->cnn_bound, nullptr,
                                   stream)))
      return st;
    if ((st = cuda_status(cudaEventRecord(r->ev_cnn[1], s)))) return st;
    int ms = 0, ny = 0, nx = 0;
    lct_cnn_get_shape(r->cnn, &ms, &ny, &nx);
    r->launches += 1 + 9 * ((nb * kBlockSlices + ms - 1) / ms);  // memset + (prep + 8 convs) per pass
  }

  if (!image_on_device) {
    if ((st = cuda_status(cudaMemcpyAsync(image, r->d_img, sizeof(float) * nb * slab,
                                          cudaMemcpyDeviceToHost, s))))
      return st;
  }
  if ((st = cuda_status(cudaEventRecord(r->ev[5], s)))) return st;
  if ((st = cuda_status(cudaEventSynchronize(r->ev[5])))) return st;
  for (int i = 0; i < 5; ++i) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, r->ev[i], r->ev[i + 1]);
    r->times[i] = ms;
  }
  r->cnn_ms = 0.f;
  if (r->cnn) cudaEventElapsedTime(&r->cnn_ms, r->ev_cnn[0], r->ev_cnn[1]);
  return LCT_OK;
}

LCT_API int lct_recon_set_learned(lct_recon* r, lct_cnn* c, float bound) {
  if (!r || !(bound >= 0.f)) return LCT_ERR_ARG;
  if (r->bounded && c) return LCT_ERR_UNSUPPORTED;  // the network reads whole-volume neighbours
  if (!c) {
    r->cnn = nullptr;
    return LCT_OK;
  }
  int ms = 0, ny = 0, nx = 0;
  int st = lct_cnn_get_shape(c, &ms, &ny, &nx);
  if (st) return st;
  if (ny != r->info.ig.ny || nx != r->info.ig.nx) return LCT_ERR_ARG;
  const size_t img_elems =
      (size_t)r->info.n_blocks_run * kBlockSlices * r->info.ig.nx * r->info.ig.ny;
  if (!r->d_plain && (st = cuda_status(cudaMalloc(&r->d_plain, sizeof(float) * img_elems))))
    return st;
  for (auto& e : r->ev_cnn)
    if (!e && (st = cuda_status(cudaEventCreate(&e)))) return st;
  r->cnn = c;
  r->cnn_bound = bound;
  return LCT_OK;
}

LCT_API int lct_recon_learned_info(const lct_recon* r, float* ms, int64_t* rejected) {
  if (!r) return LCT_ERR_ARG;
  if (ms) *ms = r->cnn ? r->cnn_ms : 0.f;
  if (rejected) {
    *rejected = 0;
    if (r->cnn) return lct_cnn_last_rejected(r->cnn, rejected);
  }
  return LCT_OK;
}

LCT_API void lct_recon_destroy(lct_recon* r) { free_recon(r); }
