// Planner: which fan views each 32-slice block reads and the block geometry.
//
// Restates ReconData::convert_from_file_params (Src/DataStructs.cpp:121-250) and
// BlockInfo::update (Src/DataStructs.cpp:77-108) with the reference's arithmetic types:
// every float expression is evaluated in float in the reference's order (the host build uses
// -ffp-contract=off), and the float-overload rounding functions (std::ceil(float) etc.) are
// the ones the reference's `using namespace std` selects.  Differences, all deliberate:
//   * errors are status codes instead of exit(1);
//   * array_search tests the bound before reading (the reference reads array[idx] first,
//     Src/DataStructs.cpp:17,22,27; results are identical whenever its read is in bounds);
//   * sizes are 64-bit and a block whose view window leaves the data is rejected (the
//     reference reads outside the file there, Src/DataReader.cpp:14);
//   * the optional MaxBlocks / FirstBlock keys select the blocks reconstructed.
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "lct_internal.h"

struct lct_plan {
  lct_scan_params p;
  std::vector<float> angles, zpos;
  lct_plan_info info;
  std::vector<lct_block_info> blocks;
};

namespace lct {

// Src/DataStructs.cpp:12-34
static int array_search(float key, const float* a, int n, int type) {
  int idx = 0;
  switch (type) {
    case -1:
      while (idx < n && key < a[idx]) idx++;
      break;
    case 0:
      while (idx < n && key != a[idx]) idx++;
      break;
    case 1:
      while (idx < n && key > a[idx]) idx++;
      break;
  }
  return idx;
}

static int sign_of(float num_over) { return (int)num_over; }

// int(fabs(d)/d) with the reference's fallback to 1 for a zero difference
static int direction(float d) {
  float q = std::fabs(d) / d;
  if (std::isnan(q)) return 1;
  int r = (int)q;
  if (r != 1 && r != -1) r = 1;
  return r;
}

static int plan_build(lct_plan& P) {
  const lct_scan_params& fp = P.p;
  if (fp.ns <= 0 || fp.nt <= 0 || fp.nx <= 0 || fp.ny <= 0 || fp.n_proj_turn < 2) return LCT_ERR_ARG;
  if (fp.readings < 101 || !(fp.ds > 0.f) || !(fp.dt > 0.f) || !(fp.dz > 0.f) || !(fp.dx > 0.f))
    return LCT_ERR_ARG;
  if (!(fp.r_src_to_iso > 0.f)) return LCT_ERR_ARG;
  const float* ta = P.angles.data();
  const float* tp = P.zpos.data();
  const int npt = fp.n_proj_turn;
  const int nsb = kBlockSlices;

  // :123
  const float mx = std::max(fp.central_channel, (float)fp.ns - fp.central_channel);
  const int add = (int)((double)(mx * fp.ds * (float)npt) / ((double)(2.0f * fp.r_src_to_iso) * kRefPi) + 10);

  // :169-176
  const float dd = tp[100] - tp[0];
  if (dd == 0.0f || !std::isfinite(dd)) return LCT_ERR_ARG;
  const int array_dir = sign_of(std::fabs(dd) / dd);
  const int z_dir = array_dir;
  const float orbit_start = ta[0];
  float orbit;
  if ((ta[1] < 1 && ta[0] > 6) || (ta[1] > 6 && ta[0] < 1))
    orbit = ta[2] - ta[1];
  else
    orbit = ta[1] - ta[0];
  const float source_z0 = -fp.pitch_value / 2.0f;

  // :179-218
  const float data_begin = tp[0];
  const float data_end = tp[fp.readings - 1];
  const float padding = fp.pitch_value * (float)(npt / 2 + add + 256) / (float)npt;
  const float allow_begin = data_begin + (float)array_dir * padding;
  const float allow_end = data_end - (float)array_dir * padding;
  float start_pos, end_pos;
  if (array_dir > 0) {
    start_pos = std::ceil(allow_begin + (float)(1 * array_dir));
    end_pos = std::floor(allow_end - (float)(1 * array_dir));
  } else {
    start_pos = std::floor(allow_begin + (float)(1 * array_dir));
    end_pos = std::ceil(allow_end - (float)(1 * array_dir));
  }
  const int recon_dir = direction(end_pos - start_pos);
  const float recon_start = start_pos - (float)recon_dir * fp.dz;
  float recon_end = end_pos + (float)recon_dir * fp.dz;
  const int n_req = (int)(std::floor(std::fabs(recon_end - recon_start) / fp.dz) + 1.0f);
  const int n_slices = (n_req - 1) - (n_req - 1) % nsb;
  recon_end = recon_start + (float)(recon_dir * (n_slices - 1)) * fp.dz;
  const int n_blocks = n_slices / nsb;
  if (((start_pos > allow_begin) && (start_pos > allow_end)) ||
      ((start_pos < allow_begin) && (start_pos < allow_end)))
    return LCT_ERR_RANGE;
  if (((end_pos > allow_begin) && (end_pos > allow_end)) ||
      ((end_pos < allow_begin) && (end_pos < allow_end)))
    return LCT_ERR_RANGE;

  // :222-240 block 0
  float block_start = recon_start;
  float block_end = block_start + (float)(recon_dir * (nsb - 1)) * fp.dz;
  int bps = array_search(block_start, tp, fp.readings, array_dir);
  int bpe = array_search(block_end, tp, fp.readings, array_dir);
  if (bps > bpe) {
    bps = bpe - npt / 2 - add;
    bpe = bps + npt / 2 + add;
  } else {
    bps = bps - npt / 2 - add;
    bpe = bpe + npt / 2 + add;
  }
  const int n_angle_add = bpe - bps + 100;
  const int n_angle = n_angle_add - 2 * add;
  if (n_angle <= 0) return LCT_ERR_RANGE;

  lct_plan_info& I = P.info;
  std::memset(&I, 0, sizeof(I));
  lct_geom& g = I.ctg;
  g.orbit = orbit;
  g.orbit_start = orbit_start;
  g.ns = fp.ns;
  g.nt = fp.nt;
  g.ws = fp.central_channel;
  g.wt = (fp.nt - 1) / 2.0f;
  g.n_angle = n_angle;
  g.n_angle_add = n_angle_add;
  g.ds = fp.ds;
  g.dt = fp.dt;
  g.pitch = fp.pitch_value;
  g.source_z0 = source_z0;
  g.dso = fp.r_src_to_iso;
  g.n_proj_turn = npt;
  g.z_dir = z_dir;
  g.add_projections = add;
  // ImgGeom(nx, ny, 32, dx, dx, dz, offX, offY, 0), Include/DataStructs.h:118-129
  lct_img& ig = I.ig;
  ig.nx = fp.nx;
  ig.ny = fp.ny;
  ig.nz = nsb;
  ig.dx = fp.dx;
  ig.dy = fp.dx;
  ig.dz = fp.dz;
  ig.wx = (fp.nx - 1) / 2.0f + fp.offset_x;
  ig.wy = (fp.ny - 1) / 2.0f + fp.offset_y;
  ig.wz = 0.0f;

  I.n_readings = fp.readings;
  I.data_begin_pos = data_begin;
  I.data_end_pos = data_end;
  I.allow_begin = allow_begin;
  I.allow_end = allow_end;
  I.start_pos = start_pos;
  I.end_pos = end_pos;
  I.recon_start_pos = recon_start;
  I.recon_end_pos = recon_end;
  I.n_slices_recon = n_slices;
  I.n_slices_block = nsb;
  I.n_blocks = n_blocks;
  I.data_offset = fp.data_offset;
  if (fp.first_block < 0 || (fp.first_block > 0 && fp.first_block >= n_blocks)) return LCT_ERR_RANGE;
  I.first_block = fp.first_block;
  const int left = n_blocks - fp.first_block;
  I.n_blocks_run = (fp.max_blocks > 0 && fp.max_blocks < left) ? fp.max_blocks : left;

  P.blocks.clear();
  lct_block_info b0;
  b0.block_idx = 0;
  b0.block_proj_start = bps;
  b0.block_proj_end = bpe;
  b0.block_start = block_start;
  b0.block_end = block_end;
  b0.block_slice_start = 0;
  b0.block_slice_end = nsb - 1;
  P.blocks.push_back(b0);
  // BlockInfo::update for blocks 1.. (:77-108)
  const int rdir = direction(end_pos - start_pos);
  for (int id = 1; id < n_blocks; ++id) {
    float bs = recon_start + (float)(rdir * id) * fp.dz * (float)nsb;
    float be = bs + (float)(rdir * (nsb - 1)) * fp.dz;
    int s = array_search(bs, tp, fp.readings, z_dir);
    int e = array_search(be, tp, fp.readings, z_dir);
    if (s > e)
      s = e - npt / 2 - add;
    else
      s = s - npt / 2 - add;
    lct_block_info b;
    b.block_idx = id;
    b.block_proj_start = s;
    b.block_proj_end = s + n_angle_add;
    b.block_start = bs;
    b.block_end = be;
    b.block_slice_start = nsb * id;
    b.block_slice_end = nsb * id + nsb - 1;
    P.blocks.push_back(b);
  }
  return LCT_OK;
}

}  // namespace lct

using namespace lct;

LCT_API int lct_plan_create(const lct_scan_params* p, const float* tube_angles,
                            const float* table_positions, lct_plan** out) {
  if (!p || !tube_angles || !table_positions || !out) return LCT_ERR_ARG;
  *out = nullptr;
  if (p->readings < 101) return LCT_ERR_ARG;
  lct_plan* P = new (std::nothrow) lct_plan;
  if (!P) return LCT_ERR_ALLOC;
  P->p = *p;
  P->angles.assign(tube_angles, tube_angles + p->readings);
  P->zpos.assign(table_positions, table_positions + p->readings);
  int st = plan_build(*P);
  if (st) {
    delete P;
    return st;
  }
  *out = P;
  return LCT_OK;
}

LCT_API int lct_plan_adopt(const lct_plan_info* info, const lct_block_info* blocks, int n_blocks,
                           const float* tube_angles, const float* table_positions,
                           lct_plan** out) {
  if (!info || !blocks || !tube_angles || !table_positions || !out) return LCT_ERR_ARG;
  *out = nullptr;
  int st = check_geom(&info->ctg);
  if (st) return st;
  if ((st = check_img(&info->ig))) return st;
  if (info->ig.nz != kBlockSlices || info->n_readings <= 0) return LCT_ERR_ARG;
  if (n_blocks <= 0 || n_blocks != info->n_blocks) return LCT_ERR_ARG;
  if (info->first_block < 0 || info->n_blocks_run <= 0 ||
      info->first_block + info->n_blocks_run > n_blocks)
    return LCT_ERR_ARG;
  // (the views a run reads are checked against the data by lct_recon_create, as for any plan)
  lct_plan* P = new (std::nothrow) lct_plan;
  if (!P) return LCT_ERR_ALLOC;
  std::memset(&P->p, 0, sizeof(P->p));
  P->p.ns = info->ctg.ns;
  P->p.nt = info->ctg.nt;
  P->p.ds = info->ctg.ds;
  P->p.dt = info->ctg.dt;
  P->p.pitch_value = info->ctg.pitch;
  P->p.nx = info->ig.nx;
  P->p.ny = info->ig.ny;
  P->p.dx = info->ig.dx;
  P->p.dz = info->ig.dz;
  P->p.readings = info->n_readings;
  P->p.data_offset = info->data_offset;
  P->p.r_src_to_iso = info->ctg.dso;
  P->p.central_channel = info->ctg.ws;
  P->p.n_proj_turn = info->ctg.n_proj_turn;
  P->p.first_block = info->first_block;
  P->p.max_blocks = info->n_blocks_run;
  P->angles.assign(tube_angles, tube_angles + info->n_readings);
  P->zpos.assign(table_positions, table_positions + info->n_readings);
  P->info = *info;
  P->blocks.assign(blocks, blocks + n_blocks);
  *out = P;
  return LCT_OK;
}

LCT_API int lct_plan_info_get(const lct_plan* plan, lct_plan_info* out) {
  if (!plan || !out) return LCT_ERR_ARG;
  *out = plan->info;
  return LCT_OK;
}

LCT_API int lct_plan_block(const lct_plan* plan, int b, lct_block_info* out) {
  if (!plan || !out || b < 0 || b >= (int)plan->blocks.size()) return LCT_ERR_ARG;
  *out = plan->blocks[b];
  return LCT_OK;
}

LCT_API void lct_plan_destroy(lct_plan* plan) { delete plan; }

// access for recon.cu
namespace lct {
const float* plan_angles(const lct_plan* p) { return p->angles.data(); }
const float* plan_zpos(const lct_plan* p) { return p->zpos.data(); }
const lct_scan_params& plan_params(const lct_plan* p) { return p->p; }
}  // namespace lct
