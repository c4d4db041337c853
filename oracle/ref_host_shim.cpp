/*
 * ref_host_shim.cpp -- TEST INFRASTRUCTURE ONLY (oracle side).
 *
 * A tiny command-line driver linked against the reference's own, unmodified host sources
 * (Src/DataStructs.cpp, Src/FileParams.cpp, Src/Filter.cpp) so that tests can pin the
 * product's planner and filter taps against the reference itself.
 *
 *   ref_plan plan <file.prm>      -> JSON: CTGeom, ImgGeom, ReconInfo and every BlockInfo
 *                                    (block 0 from ReconData::convert_from_file_params,
 *                                    blocks 1.. from BlockInfo::update), i.e. exactly what
 *                                    FDKReconstructor::reconstruct (Src/Reconstructor.cpp:33-48)
 *                                    would see.
 *   ref_plan taps <ns> <ds>       -> JSON: RampFilterGPU::calculate_filter (Src/Filter.cpp:8-20)
 *
 * The reference exits the process on invalid input (Src/FileParams.cpp:18-20,
 * Src/DataStructs.cpp:210-218), which is why this is a separate process and not a library.
 */
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "DataStructs.h"
#include "FileParams.h"
/* calculate_filter is a private virtual hook of the reference's Filter classes
   (Include/Filter.h:9,20); opening access here changes no layout. */
#define private public
#include "Filter.h"
#undef private

static void print_block(const BlockInfo* bi, int id) {
  std::printf(
      "{\"block_id\": %d, \"block_idx\": %d, \"block_proj_start\": %d, \"block_proj_end\": %d, "
      "\"block_start\": %.9g, \"block_end\": %.9g, \"block_slice_start\": %d, "
      "\"block_slice_end\": %d}",
      id, bi->block_idx(), bi->block_proj_start(), bi->block_proj_end(), bi->block_start(),
      bi->block_end(), bi->block_slice_start(), bi->block_slice_end());
}

static int do_plan(const char* prm) {
  FileParams fp{std::string(prm)};
  ReconData* mr = new ReconData(fp);
  const CTGeom* g = mr->ctg_();
  const ImgGeom* ig = mr->ig_();
  const ReconInfo* ri = mr->ri_();
  std::printf("{\"ctg\": {\"orbit\": %.9g, \"orbit_start\": %.9g, \"ns\": %d, \"nt\": %d, "
              "\"ws\": %.9g, \"wt\": %.9g, \"n_angle\": %d, \"n_angle_add\": %d, \"ds\": %.9g, "
              "\"dt\": %.9g, \"pitch\": %.9g, \"source_z0\": %.9g, \"dso\": %.9g, "
              "\"n_proj_turn\": %d, \"z_dir\": %d, \"add_projections\": %d},\n",
              g->orbit_(), g->orbit_start(), g->ns_(), g->nt_(), g->ws_(), g->wt_(),
              g->n_angle(), g->n_angle_add(), g->ds_(), g->dt_(), g->pitch_(), g->source_z0(),
              g->dso_(), g->n_proj_turn(), g->z_dir(), g->add_projections());
  std::printf("\"ig\": {\"nx\": %d, \"ny\": %d, \"nz\": %d, \"wx\": %.9g, \"wy\": %.9g, "
              "\"wz\": %.9g, \"dx\": %.9g, \"dy\": %.9g, \"dz\": %.9g},\n",
              ig->nx_(), ig->ny_(), ig->nz_(), ig->wx_(), ig->wy_(), ig->wz_(), ig->dx_(),
              ig->dy_(), ig->dz_());
  std::printf("\"ri\": {\"n_readings\": %d, \"data_begin_pos\": %.9g, \"data_end_pos\": %.9g, "
              "\"allow_begin\": %.9g, \"allow_end\": %.9g, \"start_pos\": %.9g, "
              "\"end_pos\": %.9g, \"recon_start_pos\": %.9g, \"recon_end_pos\": %.9g, "
              "\"n_slices_recon\": %d, \"n_slices_block\": %d, \"n_blocks\": %d, "
              "\"data_offset\": %d},\n",
              ri->n_readings(), ri->data_begin_pos(), ri->data_end_pos(), ri->allow_begin(),
              ri->allow_end(), ri->start_pos(), ri->end_pos(), ri->recon_start_pos(),
              ri->recon_end_pos(), ri->n_slices_recon(), ri->n_slices_block(), ri->n_blocks(),
              ri->data_offset());
  std::printf("\"blocks\": [");
  int nb = ri->n_blocks();
  for (int b = 0; b < nb; ++b) {
    if (b) std::printf(",\n");
    print_block(mr->bi_(), b);
    mr->bi_()->update(ri, g, ig, mr->data_cpu());
  }
  std::printf("]}\n");
  /* ReconData's destructor frees device buffers through the CUDA runtime; skip it so the
     shim also runs on a machine without a GPU. */
  return 0;
}

static int do_taps(int ns, float ds) {
  CTGeom g(0.f, 0.f, ns, 1, 1, 1, ds, 1.f, 0.f, 0.f, 1.f, 0.f, 1.f, 1, 1, 0);
  std::vector<float> h(2 * (size_t)ns);
  RampFilterGPU f;
  f.calculate_filter(h.data(), &g);
  std::printf("{\"ns\": %d, \"ds\": %.9g, \"h\": [", ns, ds);
  for (int i = 0; i < 2 * ns; ++i) std::printf(i ? ", %.9g" : "%.9g", h[i]);
  std::printf("]}\n");
  return 0;
}

int main(int argc, char** argv) {
  if (argc >= 3 && std::string(argv[1]) == "plan") return do_plan(argv[2]);
  if (argc >= 4 && std::string(argv[1]) == "taps")
    return do_taps(std::atoi(argv[2]), (float)std::atof(argv[3]));
  std::fprintf(stderr, "usage: ref_plan plan <prm> | ref_plan taps <ns> <ds>\n");
  return 2;
}
