// The whole-scan reconstructor behind the type name "Helicalfdkramprebinb200": a Reconstructor
// (Include/Reconstructor.h:15) whose reconstruct(const ReconData*) runs the scan-mode path of
// liblct.so over every block the reference's planner planned, instead of the per-block stage
// calls of FDKReconstructor::reconstruct (Src/Reconstructor.cpp:30-49).
//
//   * the plan is the reference's own: CTGeom, ImgGeom and ReconInfo of the ReconData and every
//     block's BlockInfo (walked with BlockInfo::update, as the reference's loop does), adopted
//     with lct_plan_adopt -- the same blocks, the same view windows;
//   * each fan view is read once from the DataInterpFile with 64-bit offsets (the reference reads
//     each block's window through an `int` offset, Src/DataReader.cpp:14), rebinned and filtered
//     once, and every slab backprojected from the shared filtered views;
//   * the volume lands in the ReconData's host image, as the reference's backprojector leaves it
//     (CUDA/Backprojector.cu:158), so RawImageWriter writes it unchanged.  The filtered block the
//     reference's Filter copies to host `rebin` does not exist in this flow: `rebin` stays zero.
//
// Defaults: exact interpolation, the BF16x6 tensor-core filter, border addressing, a bounded
// device footprint (lct_recon_create_bounded) fed by lct_recon_run_file's reader threads.  The
// recon's create, run and destroy times and its file I/O times are printed on one "[B200]" line.
// Environment switches, as for the stage drop-in: LCT_DROPIN_INTERP=tex8|exact,
// LCT_DROPIN_FILTER=fp32|bf16x3|bf16x6, LCT_DROPIN_ADDR=border|clamp|legacy.  LEGACY (the
// reference's clamped first block) needs the whole filtered views on the device: that run
// reads the fan window into pinned memory and uses lct_recon_create with lct_recon_run.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "DataStructs.h"
#include "Reconstructor.h"
#include "lct.h"

namespace {

int env_choice(const char* name, const char* const* names, const int* values, int n, int dflt) {
  const char* v = std::getenv(name);
  if (!v) return dflt;
  for (int i = 0; i < n; ++i)
    if (std::strcmp(v, names[i]) == 0) return values[i];
  return dflt;
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
  if (st == LCT_OK) return true;
  std::cout << "[ERROR] " << what << ": " << lct_status_string(st) << std::endl;
  return false;
}

// views [v0, v0 + n) of the raw file into dst (64-bit offsets)
int read_views(const std::string& path, long long v0, long long n, long long view_bytes, float* dst) {
  const int fd = ::open(path.c_str(), O_RDONLY);
  if (fd < 0) return LCT_ERR_IO;
  char* p = reinterpret_cast<char*>(dst);
  long long left = n * view_bytes, off = v0 * view_bytes;
  while (left > 0) {
    const ssize_t k = ::pread(fd, p, (size_t)(left < (1LL << 30) ? left : (1LL << 30)), (off_t)off);
    if (k <= 0) {
      ::close(fd);
      return LCT_ERR_IO;
    }
    p += k;
    off += k;
    left -= k;
  }
  ::close(fd);
  return LCT_OK;
}

class B200FDKReconstructor : public Reconstructor {
 public:
  void reconstruct(const ReconData* mr) override;
};

void B200FDKReconstructor::reconstruct(const ReconData* mr) {
  std::cout << "Start reconstruction (whole scan)..." << std::endl;
  const CTGeom* ctg = mr->ctg_();
  const ImgGeom* ig = mr->ig_();
  const ReconInfo* ri = mr->ri_();
  const int nb = ri->n_blocks();
  if (nb <= 0) {
    std::cout << "[ERROR] no blocks planned" << std::endl;
    return;
  }
  // every block's BlockInfo, in the order FDKReconstructor::reconstruct visits them
  std::vector<lct_block_info> blocks(nb);
  for (int b = 0; b < nb; ++b) {
    const BlockInfo* bi = mr->bi_();
    blocks[b].block_idx = bi->block_idx();
    blocks[b].block_proj_start = bi->block_proj_start();
    blocks[b].block_proj_end = bi->block_proj_end();
    blocks[b].block_start = bi->block_start();
    blocks[b].block_end = bi->block_end();
    blocks[b].block_slice_start = bi->block_slice_start();
    blocks[b].block_slice_end = bi->block_slice_end();
    mr->bi_()->update(ri, ctg, ig, mr->data_cpu());
  }
  lct_plan_info info;
  std::memset(&info, 0, sizeof(info));
  info.ctg = to_geom(ctg);
  info.ig = to_img(ig);
  info.n_readings = ri->n_readings();
  info.data_begin_pos = ri->data_begin_pos();
  info.data_end_pos = ri->data_end_pos();
  info.allow_begin = ri->allow_begin();
  info.allow_end = ri->allow_end();
  info.start_pos = ri->start_pos();
  info.end_pos = ri->end_pos();
  info.recon_start_pos = ri->recon_start_pos();
  info.recon_end_pos = ri->recon_end_pos();
  info.n_slices_recon = ri->n_slices_recon();
  info.n_slices_block = ri->n_slices_block();
  info.n_blocks = nb;
  info.data_offset = ri->data_offset();
  info.first_block = 0;
  info.n_blocks_run = nb;
  lct_plan* plan = nullptr;
  if (!ok(lct_plan_adopt(&info, blocks.data(), nb, mr->data_cpu()->tube_angles(),
                         mr->data_cpu()->table_positions(), &plan),
          "lct_plan_adopt"))
    return;

  lct_recon_opts o;
  lct_recon_opts_default(&o);
  o.mode = LCT_MODE_SCAN;
  o.filter_kind = LCT_FILTER_RAMLAK;  // RampFilterGPU (Src/Filter.cpp:8-20)
  {
    static const char* n[] = {"tex8", "exact"};
    static const int v[] = {LCT_INTERP_TEX8, LCT_INTERP_EXACT};
    o.interp = env_choice("LCT_DROPIN_INTERP", n, v, 2, LCT_INTERP_EXACT);
  }
  {
    static const char* n[] = {"fp32", "bf16x3", "bf16x6"};
    static const int v[] = {LCT_FILTER_FP32, LCT_FILTER_BF16X3, LCT_FILTER_BF16X6};
    o.filter_mode = env_choice("LCT_DROPIN_FILTER", n, v, 3, LCT_FILTER_BF16X6);
  }
  {
    static const char* n[] = {"border", "clamp", "legacy"};
    static const int v[] = {LCT_ADDR_BORDER, LCT_ADDR_CLAMP, LCT_ADDR_LEGACY};
    o.addr = env_choice("LCT_DROPIN_ADDR", n, v, 3, LCT_ADDR_BORDER);
  }
  const std::string path = mr->fi_()->in_file_dir() + mr->fi_()->data_file_name();
  float* image = mr->data_cpu()->image_();
  lct_recon* r = nullptr;
  using clk = std::chrono::steady_clock;
  const clk::time_point t0 = clk::now();
  clk::time_point t1 = t0;
  if (o.addr != LCT_ADDR_LEGACY) {
    if (ok(lct_recon_create_bounded(plan, &o, 0, &r), "lct_recon_create_bounded")) {
      t1 = clk::now();
      ok(lct_recon_run_file(r, path.c_str(), nullptr, image, nullptr), "lct_recon_run_file");
    }
  } else if (ok(lct_recon_create(plan, &o, &r), "lct_recon_create")) {
    t1 = clk::now();
    int64_t first = 0, count = 0;
    lct_recon_fan_range(r, &first, &count);
    const long long view_bytes = (long long)sizeof(float) * ctg->ns_() * ctg->nt_();
    float* fan = nullptr;
    if (ok(cudaHostAlloc((void**)&fan, (size_t)(count * view_bytes), cudaHostAllocDefault) ==
                   cudaSuccess
               ? LCT_OK
               : LCT_ERR_ALLOC,
           "pinned fan buffer") &&
        ok(read_views(path, first + info.data_offset, count, view_bytes, fan), "reading the fan"))
      ok(lct_recon_run(r, fan, first + info.data_offset, 0, image, 0, nullptr), "lct_recon_run");
    if (fan) cudaFreeHost(fan);
  }
  const clk::time_point t2 = clk::now();
  float io[3] = {0.f, 0.f, 0.f};
  if (r) lct_recon_io_times(r, io);
  if (r) lct_recon_destroy(r);
  lct_plan_destroy(plan);
  const clk::time_point t3 = clk::now();
  auto secs = [](clk::time_point a, clk::time_point b) {
    return std::chrono::duration<double>(b - a).count();
  };
  std::printf("[B200] create %.4f s, run %.4f s, destroy %.4f s; reads %.4f s (summed over the "
              "reader threads), waits for reads %.4f s, for the writer %.4f s\n",
              secs(t0, t1), secs(t1, t2), secs(t2, t3), io[0], io[1], io[2]);
  std::cout << "Reconstruction of " << nb << " blocks finished." << std::endl;
}

}  // namespace

Reconstructor* lct_make_b200_reconstructor() { return new B200FDKReconstructor(); }
