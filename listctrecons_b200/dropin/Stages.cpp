// Drop-in stage implementations for the reference program (ltldlzltl/LISTCTRecons).
//
// This file replaces the reference's CUDA/Rebiner.cu, CUDA/PreWeighting.cu, CUDA/Filter.cu and
// CUDA/Backprojector.cu: it defines the same member functions, declared by the reference's own
// unchanged headers (Include/Rebiner.h, PreWeighting.h, Filter.h, Backprojector.h), on top of
// the C ABI of liblct.so (include/lct.h).  Everything else of the reference -- FileParams,
// ReconData and its planner, the factory, FDKReconstructor, the reader and writer, main -- links
// unchanged, so the binary is a drop-in.
//
// Ownership is the reference's (Include/DataStructs.h:213-229): the rebinner allocates projGpu,
// the filter works on it in place and copies the filtered block to host `rebin`, the
// backprojector allocates imgGpu, writes the block into host `image` and frees both.  Stages print
// and return on errors like the reference; the last lct status is kept in lct_dropin_status().
//
// Sampling: the reference's texture semantics (LCT_INTERP_TEX8) with the legacy binding
// behaviour of its texture references (Clamp for the first bound block, Border afterwards:
// LCT_ADDR_LEGACY).  Environment switches: LCT_DROPIN_ADDR=border|clamp|legacy,
// LCT_DROPIN_INTERP=tex8|exact, LCT_DROPIN_FILTER=fp32|bf16x3|bf16x6,
// LCT_DROPIN_FILTERED_COPY=0 (skip the filtered block's copy to host `rebin`).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>

#include "Backprojector.h"
#include "Common.h"
#include "DataStructs.h"
#include "Filter.h"
#include "GPUMemoryCtrl.h"
#include "PreWeighting.h"
#include "Rebiner.h"
#include "lct.h"

namespace {

int g_last_status = LCT_OK;

int env_choice(const char* name, const char* const* names, const int* values, int n, int dflt) {
  const char* v = std::getenv(name);
  if (!v) return dflt;
  for (int i = 0; i < n; ++i)
    if (std::strcmp(v, names[i]) == 0) return values[i];
  return dflt;
}

int interp_mode() {
  static const char* n[] = {"tex8", "exact"};
  static const int v[] = {LCT_INTERP_TEX8, LCT_INTERP_EXACT};
  return env_choice("LCT_DROPIN_INTERP", n, v, 2, LCT_INTERP_TEX8);
}

int filter_mode() {
  static const char* n[] = {"fp32", "bf16x3", "bf16x6"};
  static const int v[] = {LCT_FILTER_FP32, LCT_FILTER_BF16X3, LCT_FILTER_BF16X6};
  return env_choice("LCT_DROPIN_FILTER", n, v, 3, LCT_FILTER_FP32);
}

// Addressing of the n-th bind of a stage's texture (legacy: attributes captured at bind time,
// Border assigned after the first bind: CUDA/Rebiner.cu:137-139, CUDA/Backprojector.cu:134-136)
int addr_for_bind(int& binds) {
  static const char* n[] = {"border", "clamp", "legacy"};
  static const int v[] = {LCT_ADDR_BORDER, LCT_ADDR_CLAMP, LCT_ADDR_LEGACY};
  const int mode = env_choice("LCT_DROPIN_ADDR", n, v, 3, LCT_ADDR_LEGACY);
  const int first = binds++ == 0;
  if (mode == LCT_ADDR_LEGACY) return first ? LCT_ADDR_CLAMP : LCT_ADDR_BORDER;
  return mode;
}

lct_geom to_geom(const CTGeom* c) {
  lct_geom g;
  g.orbit = c->orbit_();
  g.orbit_start = c->orbit_start();
  g.ns = c->ns_();
  g.nt = c->nt_();
  g.ws = c->ws_();
  g.wt = c->wt_();
  g.n_angle = c->n_angle();
  g.n_angle_add = c->n_angle_add();
  g.ds = c->ds_();
  g.dt = c->dt_();
  g.pitch = c->pitch_();
  g.source_z0 = c->source_z0();
  g.dso = c->dso_();
  g.n_proj_turn = c->n_proj_turn();
  g.z_dir = c->z_dir();
  g.add_projections = c->add_projections();
  return g;
}

lct_img to_img(const ImgGeom* i) {
  lct_img g;
  g.nx = i->nx_();
  g.ny = i->ny_();
  g.nz = i->nz_();
  g.wx = i->wx_();
  g.wy = i->wy_();
  g.wz = i->wz_();
  g.dx = i->dx_();
  g.dy = i->dy_();
  g.dz = i->dz_();
  return g;
}

bool ok(int st, const char* what) {
  g_last_status = st;
  if (st == LCT_OK) return true;
  std::cout << "[ERROR] " << what << ": " << lct_status_string(st) << std::endl;
  return false;
}

// The fan block on the device (the reference's 3-D texture array, one per rebin call).
GPUMemoryCtrl<float>& fan_buffer() {
  static GPUMemoryCtrl<float> buf;
  return buf;
}

// Shared body of the three rebinners: upload the block, allocate projGpu, run `kernel`.
template <class F>
void rebin_with(const ReconData* mr, int& binds, F kernel, const char* what) {
  CTGeom* ctg = mr->ctg_();
  CTDataGPU* dg = mr->data_gpu();
  const size_t nfan = (size_t)ctg->ns_() * ctg->nt_() * ctg->n_angle_add();
  GPUMemoryCtrl<float>& fan = fan_buffer();
  fan.free_memory();
  if (!fan.allocate_memory(nfan) || !fan.copy_from_CPU(mr->data_cpu()->proj_(), nfan)) {
    std::cout << "[ERROR] Could not copy img to device" << std::endl;
    g_last_status = LCT_ERR_ALLOC;
    return;
  }
  // CUDA/Rebiner.cu:142-144: the rebinner owns the projGpu allocation and uploads ctg
  dg->proj_gpu()->allocate_memory((size_t)ctg->ns_() * ctg->nt_() * ctg->n_angle());
  dg->ctg_gpu()->copy_from_CPU(ctg, 1);
  const lct_geom g = to_geom(ctg);
  if (!ok(kernel(&g, fan.get_pointer(), dg->proj_gpu()->get_pointer(), addr_for_bind(binds)), what))
    return;
  ok(cudaDeviceSynchronize() == cudaSuccess ? LCT_OK : LCT_ERR_CUDA, what);
  fan.free_memory();
  std::cout << "Rebin finished" << std::endl;
}

int g_binds_rebin = 0, g_binds_bp = 0;

}  // namespace

extern "C" int lct_dropin_status(void) { return g_last_status; }

void NullRebinerGPU::rebin(const ReconData* mr) {
  rebin_with(
      mr, g_binds_rebin,
      [](const lct_geom* g, const float* f, float* p, int addr) {
        return lct_rebin_null(g, f, p, addr, nullptr);
      },
      "lct_rebin_null");
}

void HelicalConeBeamFan2ParRebinerGPU::rebin(const ReconData* mr) {
  const int interp = interp_mode();
  rebin_with(
      mr, g_binds_rebin,
      [interp](const lct_geom* g, const float* f, float* p, int addr) {
        return lct_rebin_fan2par(g, f, p, interp, addr, nullptr);
      },
      "lct_rebin_fan2par");
}

void PiOriRebiner::rebin(const ReconData* mr) {
  const int interp = interp_mode();
  rebin_with(
      mr, g_binds_rebin,
      [interp](const lct_geom* g, const float* f, float* p, int addr) {
        return lct_rebin_pi_ori(g, f, p, interp, addr, nullptr);
      },
      "lct_rebin_pi_ori");
}

// CUDA/PreWeighting.cu:32-44: 1 on success, -1 on a CUDA error
int PiOriPreWeighting::weighting(const ReconData* mr) {
  const lct_geom g = to_geom(mr->ctg_());
  if (!ok(lct_weight_pi_ori(&g, mr->data_gpu()->proj_gpu()->get_pointer(), nullptr),
          "lct_weight_pi_ori"))
    return -1;
  return cudaDeviceSynchronize() == cudaSuccess ? 1 : -1;
}

// CUDA/Filter.cu:52-73: taps from the calculate_filter hook, in place, then D2H to `rebin`
void Filter::filter(const ReconData* mr) {
  CTGeom* ctg = mr->ctg_();
  CTDataGPU* dg = mr->data_gpu();
  const int ns = ctg->ns_();
  float* h = new float[2 * ns];
  calculate_filter(h, ctg);
  GPUMemoryCtrl<float> d_h;
  if (!d_h.allocate_memory(2 * (size_t)ns) || !d_h.copy_from_CPU(h, 2 * (size_t)ns)) {
    delete[] h;
    ok(LCT_ERR_ALLOC, "filter taps");
    return;
  }
  delete[] h;
  const long long rows = (long long)ctg->n_angle() * ctg->nt_();
  if (!ok(lct_filter_rows(ns, d_h.get_pointer(), dg->proj_gpu()->get_pointer(), rows, filter_mode(),
                          nullptr),
          "lct_filter_rows"))
    return;
  // the reference copies every filtered block to host `rebin` (CUDA/Filter.cu:69), which only its
  // writer's rebin.raw dump reads; LCT_DROPIN_FILTERED_COPY=0 skips that copy (rebin.raw then
  // holds zeros)
  const char* keep = std::getenv("LCT_DROPIN_FILTERED_COPY");
  if (!keep || std::strcmp(keep, "0") != 0)
    dg->proj_gpu()->copy_to_CPU(mr->data_cpu()->rebin_(), (size_t)ns * ctg->nt_() * ctg->n_angle());
  std::cout << "Filter finished" << std::endl;
}

// CUDA/Backprojector.cu:101-169 (and :252-307 for the PI-window variant)
template <class F>
static void backproject_with(const ReconData* mr, F kernel, const char* what) {
  CTGeom* ctg = mr->ctg_();
  ImgGeom* ig = mr->ig_();
  CTDataGPU* dg = mr->data_gpu();
  dg->img_gpu()->allocate_memory((size_t)ig->nx_() * ig->ny_() * ig->nz_());
  dg->betas_gpu()->copy_from_CPU(
      &(mr->data_cpu()->tube_angles()[mr->bi_()->block_proj_start() + ctg->add_projections()]),
      ctg->n_angle());
  dg->ig_gpu()->copy_from_CPU(ig, 1);
  const lct_geom g = to_geom(ctg);
  const lct_img im = to_img(ig);
  const int addr = addr_for_bind(g_binds_bp);
  if (ok(kernel(&g, &im, dg->betas_gpu()->get_pointer(), dg->proj_gpu()->get_pointer(),
                dg->img_gpu()->get_pointer(), addr),
         what) &&
      ok(cudaDeviceSynchronize() == cudaSuccess ? LCT_OK : LCT_ERR_CUDA, what)) {
    std::cout << "backprojection finished." << std::endl;
    const size_t n = (size_t)ig->nx_() * ig->ny_() * ig->nz_();
    dg->img_gpu()->copy_to_CPU(&mr->data_cpu()->image_()[n * mr->bi_()->block_idx()], n);
  }
  dg->proj_gpu()->free_memory();
  dg->img_gpu()->free_memory();
}

void HelicalConeBeamFanRebinBackprojectorGPU::backproject(const ReconData* mr) {
  const int interp = interp_mode();
  backproject_with(
      mr,
      [interp](const lct_geom* g, const lct_img* i, const float* b, const float* p, float* img,
               int addr) { return lct_backproject_par(g, i, b, p, img, interp, addr, nullptr); },
      "lct_backproject_par");
}

void PiOriBackprojectorGPU::backproject(const ReconData* mr) {
  const int interp = interp_mode();
  backproject_with(
      mr,
      [interp](const lct_geom* g, const lct_img* i, const float* b, const float* p, float* img,
               int addr) { return lct_backproject_pi_ori(g, i, b, p, img, interp, addr, nullptr); },
      "lct_backproject_pi_ori");
}
