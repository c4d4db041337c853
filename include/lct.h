/*
 * lct.h -- C ABI of the B200-native helical cone-beam FDK hot path (liblct.so).
 *
 * Plain C types only: device pointers are `float*`/`double*` the caller owns, streams are
 * cudaStream_t passed as an opaque pointer, every function returns an lct status code
 * (LCT_OK == 0).  Kernels are asynchronous on the given stream unless stated otherwise.
 *
 * Each entry point names the reference interface it replaces (file:line within the reference
 * project ltldlzltl/LISTCTRecons).  The reference stage methods take a `const ReconData*` and
 * work on buffers owned by its CTDataGPU (Include/DataStructs.h:207-229); the drop-in glue
 * (listctrecons_b200/dropin/Stages.cpp) unpacks those buffers and calls the functions below.
 */
#ifndef LCT_H
#define LCT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------------------------
 * Status codes
 * ------------------------------------------------------------------------------------- */
#define LCT_OK 0
#define LCT_ERR_ARG 1         /* invalid argument or geometry */
#define LCT_ERR_CUDA 2        /* CUDA runtime error; lct_last_cuda_error() has the code */
#define LCT_ERR_ALLOC 3       /* device or host allocation failed */
#define LCT_ERR_RANGE 4       /* planner: reconstruction outside the data range
                                 (reference exits: Src/DataStructs.cpp:210-218) */
#define LCT_ERR_DEVICE 5      /* a kernel raised the device status word */
#define LCT_ERR_UNSUPPORTED 6 /* option not available for this geometry / build */
#define LCT_ERR_IO 7          /* file missing or short */
#define LCT_ERR_SCRATCH 8     /* larger than the fixed scratch of an allocation-free entry point */

typedef void* lct_stream; /* cudaStream_t; NULL = the legacy default stream */

/* Mirrors CTGeom (Include/DataStructs.h:15-107), field for field, same types. */
typedef struct lct_geom {
  float orbit, orbit_start; /* radians per view, angle of view 0 */
  int ns, nt;               /* detector columns, rows */
  float ws, wt;             /* central column, central row ((nt-1)/2) */
  int n_angle, n_angle_add; /* rebinned views per block, fan views per block */
  float ds, dt;             /* column / row spacing at iso (mm) */
  float pitch;              /* table feed per rotation (mm) -- the .prm "PitchValue" */
  float source_z0;          /* -pitch/2 */
  float dso;                /* source to iso (mm) */
  int n_proj_turn;          /* views per rotation */
  int z_dir;                /* +1 / -1, direction of couch positions */
  int add_projections;      /* extra fan views each side of a block */
} lct_geom;

/* Mirrors ImgGeom (Include/DataStructs.h:109-162). */
typedef struct lct_img {
  int nx, ny, nz;
  float wx, wy, wz; /* voxel index of the origin: (n-1)/2 + offset, wz = 0 */
  float dx, dy, dz;
} lct_img;

/* Interpolation: TEX8 reproduces the reference's texture sampling (its FP32 coordinate
   arithmetic, 8-bit-fraction linear weights); EXACT uses FP64 geometry tables and full
   FP32 weights. */
#define LCT_INTERP_TEX8 0
#define LCT_INTERP_EXACT 1

/* Addressing outside the detector: BORDER reads 0 (cudaAddressModeBorder, the mode the
   reference sets), CLAMP repeats the edge.  LEGACY (whole-pipeline option only) = CLAMP on
   the first block and BORDER afterwards, which is what the reference's legacy texture
   references did (attributes are captured at bind time and it assigns Border after the first
   bind: CUDA/Rebiner.cu:137-139, CUDA/Backprojector.cu:134-136). */
#define LCT_ADDR_BORDER 0
#define LCT_ADDR_CLAMP 1
#define LCT_ADDR_LEGACY 2

/* ---------------------------------------------------------------------------------------
 * Errors and device status
 * ------------------------------------------------------------------------------------- */
const char* lct_status_string(int status);
int lct_last_cuda_error(void); /* cudaError_t of the last LCT_ERR_CUDA, per thread */
/* Reads and clears the device status word that kernels raise on out-of-range work items
   (no trap, no assert).  Synchronous. */
int lct_device_status(int* code_out);
int lct_version(void);

/* ---------------------------------------------------------------------------------------
 * Stage 1 -- rebinning.  fan [n_angle_add][nt][ns] -> par [n_angle][nt][ns] (both device).
 * ------------------------------------------------------------------------------------- */
/* HelicalConeBeamFan2ParRebinerGPU::rebin + rebin_fan2par_kernel (CUDA/Rebiner.cu:82-154) */
int lct_rebin_fan2par(const lct_geom* g, const float* d_fan, float* d_par, int interp, int addr,
                      lct_stream stream);
/* The integer fan-view index and weight rebin_fan2par uses for every (ia, is), [n_angle][ns]
   (diagnostic; same device code as lct_rebin_fan2par). */
int lct_rebin_fan2par_index(const lct_geom* g, int interp, int32_t* d_idx, float* d_w,
                            lct_stream stream);
/* The scan-mode rebin (no reference counterpart as a whole-scan call; the per-view formula is
   rebin_fan2par_kernel's, CUDA/Rebiner.cu:92-100, with the column shift alpha(is)/orbit in FP64):
   global parallel views [g0, g0 + nviews) into d_par [nviews][nt][ns] from d_fan, whose view 0 is
   global fan view fan_first and which holds fan_count views.  width: 0 = four columns per thread
   (float4 rows) where the geometry allows, 1 = one column per thread, 4 = four or
   LCT_ERR_UNSUPPORTED; every width gives the same bits. */
int lct_rebin_fan2par_scan(const lct_geom* g, const float* d_fan, int64_t fan_first,
                           int64_t fan_count, float* d_par, int64_t g0, int64_t nviews, int interp,
                           int addr, int width, lct_stream stream);
/* NullRebinerGPU::rebin + rebin_null_kernel (CUDA/Rebiner.cu:13-80) */
int lct_rebin_null(const lct_geom* g, const float* d_fan, float* d_par, int addr,
                   lct_stream stream);
/* PiOriRebiner::rebin + rebin_pi_ori_kernel (CUDA/Rebiner.cu:156-233).  TEX8 samples the fan
   block through the texture unit as the reference does (its trilinear filter, a 3-D array bound
   for the call) and therefore synchronises the stream before returning; EXACT is asynchronous.
   (lct_recon in block mode keeps one such array for all its blocks and stays asynchronous.) */
int lct_rebin_pi_ori(const lct_geom* g, const float* d_fan, float* d_par, int interp, int addr,
                     lct_stream stream);

/* ---------------------------------------------------------------------------------------
 * Stage 2 -- pre-weighting, in place on par [n_angle][nt][ns].
 * ------------------------------------------------------------------------------------- */
/* PiOriPreWeighting::weighting + weighting_pi_ori_kernel (CUDA/PreWeighting.cu:8-44).
   (NULLPreWeighting, Include/PreWeighting.h:13-19, is a no-op and needs no entry point.) */
int lct_weight_pi_ori(const lct_geom* g, float* d_par, lct_stream stream);

/* ---------------------------------------------------------------------------------------
 * Stage 3 -- ramp filter.
 * ------------------------------------------------------------------------------------- */
#define LCT_FILTER_RAMLAK 0      /* RampFilterGPU::calculate_filter (Src/Filter.cpp:8-20) */
#define LCT_FILTER_SHEPP_LOGAN 1 /* Shepp-Logan kernel, same scaling convention */

/* Smooth window (Include/SmoothWindow.h is empty in the reference): a frequency window
   applied to the taps' response.  NONE leaves the taps bit-identical to the reference's. */
#define LCT_WINDOW_NONE 0
#define LCT_WINDOW_HANN 1
#define LCT_WINDOW_HAMMING 2
#define LCT_WINDOW_COSINE 3

/* Host: fills h[2*ns] (h[0] unused, h[ns] is the centre tap), FP64 evaluated, stored as
   float.  Replaces Filter::calculate_filter (Include/Filter.h:9, Src/Filter.cpp:8-20). */
int lct_filter_taps(int kind, int window, int ns, float ds, float* h);

#define LCT_FILTER_FP32 0  /* FP32 FMA in the reference's summation order (bit-exact) */
#define LCT_FILTER_BF16X3 1 /* Toeplitz GEMM on tcgen05, BF16 hi/lo split, FP32 accumulate */
#define LCT_FILTER_BF16X6 2 /* the same with 3-way splits and 6 products (FP32-level error) */

/* Filter::filter + filter_kernel (CUDA/Filter.cu:10-73): rows[r][is] <-
   sum_k h[is-k+ns] * rows[r][k] for r < nrows, in place (device pointers; d_h has 2*ns). */
int lct_filter_rows(int ns, const float* d_h, float* d_rows, int64_t nrows, int mode,
                    lct_stream stream);

/* ---------------------------------------------------------------------------------------
 * Stage 4 -- backprojection.  proj [n_angle][nt][ns] filtered (device), betas[n_angle]
 * (device, radians, float as in the reference), img [nz][ny][nx] (device).
 * ------------------------------------------------------------------------------------- */
/* HelicalConeBeamFanRebinBackprojectorGPU::backproject + backprojection_cbct_par_kernel
   (CUDA/Backprojector.cu:12-169; na1_half = n_proj_turn/2, dz per view = pitch/n_proj_turn).
   TEX8 takes the reference's own __cosf / __sinf of the view angle, EXACT FP64 trigonometry. */
int lct_backproject_par(const lct_geom* g, const lct_img* ig, const float* d_betas,
                        const float* d_proj, float* d_img, int interp, int addr,
                        lct_stream stream);
/* Host-side query, no launch: *out = 1 when lct_backproject_par (and the allocation-free
   variant below) take the quad path for this block -- nz <= 32 and every slice's view window a
   full rotation, which the reference planner's blocks always have -- else 0 (the general
   kernel, which needs no scratch). */
int lct_backproject_par_quad_path(const lct_geom* g, const lct_img* ig, int* out);
/* No counterpart in the reference.  lct_backproject_par for callers that cannot let the
   library allocate device memory (a host that budgets all device memory itself, an acquisition
   loop that must not stall or fail on an allocation, a plugin host with its own allocator): the
   quad-layout scratch comes from a fixed 64 MiB array in the library that every GPU loading it
   holds until exit, and nothing is allocated.  Blocks needing more than 64 MiB of scratch
   (n_angle*(nt+3)*(ns+3)*16 bytes) return LCT_ERR_SCRATCH before any launch.  All calls on a
   device share that array: calls that overlap on the GPU race.  Each call looks up the array's
   device address for the current device (a host-side lookup); the first call on a device may
   also load the library's device code there, so make it before any stream capture. */
int lct_backproject_par_noalloc(const lct_geom* g, const lct_img* ig, const float* d_betas,
                                const float* d_proj, float* d_img, int interp, int addr,
                                lct_stream stream);
/* PiOriBackprojectorGPU::backproject + backprojection_cbct_pi_ori_kernel
   (CUDA/Backprojector.cu:171-307).  TEX8 takes the reference's own __cosf / __sinf of the view
   angle, EXACT FP64 trigonometry; the walk stops at the last of the n_angle views. */
int lct_backproject_pi_ori(const lct_geom* g, const lct_img* ig, const float* d_betas,
                           const float* d_proj, float* d_img, int interp, int addr,
                           lct_stream stream);

/* ---------------------------------------------------------------------------------------
 * Planner -- ReconData::convert_from_file_params (Src/DataStructs.cpp:121-250) and
 * BlockInfo::update (Src/DataStructs.cpp:77-108), reproduced in the reference's FP32
 * arithmetic with 64-bit sizes.
 * ------------------------------------------------------------------------------------- */
/* The .prm keys that reach the path (Src/FileParams.cpp:10), plus one optional key. */
typedef struct lct_scan_params {
  int ns, nt;
  float ds, dt;
  float pitch_value; /* PitchValue: / TableFeed: */
  int nx, ny;
  float dx, dz;
  float offset_x, offset_y;
  int readings, view_offset, data_offset;
  float r_src_to_iso;
  float central_channel;
  int n_proj_turn;
  int max_blocks;  /* new optional key MaxBlocks: reconstruct at most N blocks (0 = all) */
  int first_block; /* new optional key FirstBlock: start at this block (0 = the first) */
} lct_scan_params;

typedef struct lct_plan_info {
  lct_geom ctg;
  lct_img ig;
  /* ReconInfo (Include/DataStructs.h:231-279) */
  int n_readings;
  float data_begin_pos, data_end_pos, allow_begin, allow_end, start_pos, end_pos;
  float recon_start_pos, recon_end_pos;
  int n_slices_recon, n_slices_block, n_blocks, data_offset;
  int first_block;  /* first block reconstructed */
  int n_blocks_run; /* blocks reconstructed: min(n_blocks - first_block, max_blocks) */
} lct_plan_info;

/* BlockInfo (Include/DataStructs.h:281-311) of one block. */
typedef struct lct_block_info {
  int block_idx;
  int block_proj_start, block_proj_end;
  float block_start, block_end;
  int block_slice_start, block_slice_end;
} lct_block_info;

typedef struct lct_plan lct_plan;

/* tube_angles / table_positions: `readings` floats each (the contents of ViewAngleFile and
   CouchPosFile after ViewOffset), copied. */
int lct_plan_create(const lct_scan_params* p, const float* tube_angles,
                    const float* table_positions, lct_plan** out);
/* A plan holding planner results computed elsewhere: a host that already planned with the
   reference's own code (ReconData::convert_from_file_params and BlockInfo::update,
   Src/DataStructs.cpp:77-250) passes its CTGeom / ImgGeom / ReconInfo as `info` and every
   block's BlockInfo, and runs exactly those blocks.  info->first_block and info->n_blocks_run
   select the blocks run; tube_angles / table_positions hold info->n_readings floats (after
   ViewOffset).  Copies everything. */
int lct_plan_adopt(const lct_plan_info* info, const lct_block_info* blocks, int n_blocks,
                   const float* tube_angles, const float* table_positions, lct_plan** out);
int lct_plan_info_get(const lct_plan* plan, lct_plan_info* out);
int lct_plan_block(const lct_plan* plan, int b, lct_block_info* out);
void lct_plan_destroy(lct_plan* plan);

/* ---------------------------------------------------------------------------------------
 * Whole reconstruction -- FDKReconstructor::reconstruct (Src/Reconstructor.cpp:30-49) with
 * the stages the factory builds (Src/ReconstructorAbstractFactory.cpp:11-33).
 * ------------------------------------------------------------------------------------- */
#define LCT_MODE_BLOCK 0 /* the reference's per-block flow (each block rebins/filters its own
                            view window), on device-resident data */
#define LCT_MODE_SCAN 1  /* each view is rebinned and filtered once; slabs backproject from
                            the shared filtered views (FP64 rebin tables) */

#define LCT_REBIN_FAN2PAR 0
#define LCT_REBIN_NULL 1
#define LCT_REBIN_PI_ORI 2
#define LCT_PW_NONE 0
#define LCT_PW_PI_ORI 1
#define LCT_BP_PAR 0
#define LCT_BP_PI_ORI 1

/* Backprojection samplers (scan and block modes with full view windows):
   QUADS    views repacked as 2x2 texel blocks, one 16-byte load per bilinear sample (either
            interpolation);
   TEXTURE  views in a 3-D texture, one hardware fetch per sample (TEX8 only: the reference's own
            fetch, CUDA/Backprojector.cu:85-86; QUADS otherwise);
   QUADS_TMA (EXACT only) the quads, with each view's tile footprint staged in shared memory by
            TMA before the samples read it (the same values: bit-identical to QUADS);
   AUTO     QUADS (on B200 the quad kernel's TEX8 path outran the texture fetch: 121 against
            137 ms on a 512^2 x 256 volume of 736 x 64 views). */
#define LCT_BP_SAMPLER_AUTO 0
#define LCT_BP_SAMPLER_QUADS 1
#define LCT_BP_SAMPLER_TEXTURE 2
#define LCT_BP_SAMPLER_QUADS_TMA 3

typedef struct lct_recon_opts {
  int mode;          /* LCT_MODE_* */
  int rebinner;      /* LCT_REBIN_* */
  int preweight;     /* LCT_PW_* */
  int filter_kind;   /* LCT_FILTER_RAMLAK / SHEPP_LOGAN */
  int window;        /* LCT_WINDOW_* */
  int filter_mode;   /* LCT_FILTER_FP32 / BF16X3 */
  int backprojector; /* LCT_BP_* */
  int interp;        /* LCT_INTERP_* */
  int addr;          /* LCT_ADDR_* */
  int bp_nz;         /* backprojection slices per thread: 4, 8, 16; 0 = default (8, or 4 when a
                        view stays active for few slices); -1 = autotune at create */
  int bp_minb;       /* backprojection CTAs per SM the register budget targets: 1-4 (0 = 4) */
  int bp_sampler;    /* LCT_BP_SAMPLER_*: how the backprojector samples the filtered views */
} lct_recon_opts;

void lct_recon_opts_default(lct_recon_opts* o);

typedef struct lct_recon lct_recon;

/* Allocates every device buffer the plan needs (no allocation happens in run). */
int lct_recon_create(const lct_plan* plan, const lct_recon_opts* opts, lct_recon** out);
/* Reconstructs blocks [first_block, first_block + n_blocks_run).  fan: [views][nt][ns] float
   holding fan views from `fan_view0` on (file view numbering, DataOffset included) and at
   least through the run's range (lct_recon_fan_range); host (pinned or pageable) or device.
   image: [n_blocks_run*32][ny][nx].  Returns after the image is complete (synchronous).
   Scan mode (fan->parallel rebin, no pre-weighting, parallel BP) with a HOST fan streams: fan
   views are uploaded in pieces on an internal copy stream while earlier pieces are rebinned,
   filtered and backprojected slab by slab, and each finished slab is downloaded on a second copy
   stream (pinned host buffers make the copies asynchronous; a pageable volume is downloaded
   once after the pipeline, or, for a bounded recon, copied out of pinned slabs by four threads,
   so the pipeline is never held by a copy into pageable memory).  The volume is bit-identical
   to the device-resident run. */
int lct_recon_run(lct_recon* r, const float* fan, int64_t fan_view0, int fan_on_device,
                  float* image, int image_on_device, lct_stream stream);
/* Bounded device memory (no reference counterpart for the bound; the reference bounds memory
   per 32-slice block by re-reading and re-rebinning each block's window, Src/DataReader.cpp:8-19,
   Src/Reconstructor.cpp:33-48).  Like lct_recon_create, but the fan views, the filtered views
   and the backprojector's quad views live in rings sized to the slab windows in flight, and a
   volume written to host memory or a file passes through a ring of four slabs, so the device
   footprint does not grow with the scan's length.  Each view is still uploaded, rebinned and
   filtered once, and the volume is bit-identical to lct_recon_create's.  Scan mode with the
   fan->parallel rebinner, no pre-weighting, the parallel backprojector and BORDER or CLAMP
   addressing (else LCT_ERR_UNSUPPORTED); no learned correction and no autotuning (bp_nz = -1
   means the default).  piece_views: views rebinned, filtered and packed per step (0 = 512).
   Runs: lct_recon_run (host or device fan, host or device volume) and lct_recon_run_file. */
int lct_recon_create_bounded(const lct_plan* plan, const lct_recon_opts* opts, int piece_views,
                             lct_recon** out);
/* Device memory a recon holds (buffers, rings, tensor-core filter operands), bytes. */
int lct_recon_device_bytes(const lct_recon* r, int64_t* bytes);
/* Whole scan from the reference's raw files: RawDataReader::readData (Src/DataReader.cpp:8-19)
   and RawImageWriter (Src/ImageWriter.cpp:9-43) for every block of the run, with 64-bit offsets.
   fan_path: the DataInterpFile, fan view v of the scan at byte (v + DataOffset) * nt * ns * 4;
   four reader threads read the run's views into pinned chunks (whole views, at most 16 MiB)
   that are uploaded as the pipeline needs them.  image_path (or NULL): the volume
   [n_blocks_run * 32][ny][nx] float32 is written there slab by slab; image (or NULL): host
   buffer for the volume, pinned or pageable.  At least one of the two.  A file, or a pageable
   buffer, is written from pinned slabs by four writer threads (both outputs from one download
   per slab); a pinned buffer alone is downloaded into directly.  Scan-mode recons as for
   lct_recon_create_bounded (bounded or not), no learned correction.  The recon's pinned staging
   (eight fan chunks, four slabs) is pinned slot by slot by the reader and writer threads on
   first use, overlapped with the run, and kept until lct_recon_destroy.  Synchronous;
   LCT_ERR_IO for a missing or short file. */
int lct_recon_run_file(lct_recon* r, const char* fan_path, const char* image_path, float* image,
                       lct_stream stream);
/* File I/O of the last lct_recon_run_file, seconds: s3[0] = time the reader threads spent in
   reads (summed over threads), s3[1] = time the pipeline waited for fan chunks not yet read,
   s3[2] = time it waited for a free slab slot of the writer.  Zeros before the first call. */
int lct_recon_io_times(const lct_recon* r, float* s3);
/* Backprojection autotuner (no reference counterpart): times the kernel's slices-per-thread x
   CTAs-per-SM variants on this recon's buffers, keeps the fastest in the recon, and caches it per
   geometry class for the process.  Synchronous; returns the choice. */
int lct_recon_autotune(lct_recon* r, int* nz, int* minb);
/* Device-side per-stage time of the last run (ms): h2d, rebin, filter, backproject, d2h.  A
   streamed run reports its whole overlapped span as backprojection and 0 for the others. */
int lct_recon_last_times(const lct_recon* r, float* ms5);
/* Fan views [first, first+count) the run reads (h2d bytes = count*nt*ns*4). */
int lct_recon_fan_range(const lct_recon* r, int64_t* first, int64_t* count);

typedef struct lct_recon_stats {
  int64_t voxel_updates;  /* sum over reconstructed voxels of (a_max - a_min): iterations of
                             CUDA/Backprojector.cu:46 the reference would run */
  int64_t h2d_bytes;      /* fan bytes a host-buffer run copies in */
  int64_t d2h_bytes;      /* image bytes a host-buffer run copies out */
  int64_t rebinned_views; /* parallel views rebinned and filtered per run */
  int launches;           /* kernels launched by the last run */
} lct_recon_stats;
int lct_recon_stats_get(const lct_recon* r, lct_recon_stats* out);
void lct_recon_destroy(lct_recon* r);

/* ---------------------------------------------------------------------------------------
 * Batched reconstruction of many independent scans (no reference counterpart): one CUDA-graph
 * launch per stage -- rebin, filter (+ quad pack), backprojection -- and the backprojection of
 * every scan in ONE persistent work-list kernel over (scan, slab, tile) items.  Each scan's
 * volume is bit-identical to its own lct_recon run with the same options.  Scan mode only.
 * ------------------------------------------------------------------------------------- */
typedef struct lct_batch lct_batch;
int lct_batch_create(const lct_plan* const* plans, int n_scans, const lct_recon_opts* opts,
                     lct_batch** out);
/* fans[i]: scan i's views from fan_view0[i] on (host or device, as fan_on_device says);
   images[i]: [n_blocks_run_i*32][ny][nx].  Synchronous.  Host fans stream: the scans' uploads,
   per-slab compute and downloads overlap on internal streams (same kernels per scan as the
   device-resident graphs, bit-identical volumes; last_times reports one span). */
int lct_batch_run(lct_batch* b, const float* const* fans, const int64_t* fan_view0,
                  int fan_on_device, float* const* images, int image_on_device, lct_stream stream);
/* Per-scan fan range and totals over the batch (voxel_updates, bytes, launches = graph and
   copy launches of the last run). */
int lct_batch_fan_range(const lct_batch* b, int scan, int64_t* first, int64_t* count);
int lct_batch_stats_get(const lct_batch* b, lct_recon_stats* total);
/* ms of the last run: upload, rebin graph, filter graph, backprojection graph, download */
int lct_batch_last_times(const lct_batch* b, float* ms5);
void lct_batch_destroy(lct_batch* b);

/* ---------------------------------------------------------------------------------------
 * Scan simulator (no reference counterpart): analytic helical fan-beam line integrals of
 * an ellipsoid phantom with Poisson noise.  Ellipsoid record = 16 doubles:
 * cx, cy, cz, ax, ay, az, rot[9] (row-major, ellipsoid frame -> world), mu (1/mm).
 * ------------------------------------------------------------------------------------- */
int lct_sim_project(const double* d_ellipsoids, int n_ellipsoids, int ns, int nt, float ds,
                    float dt, float ws, float wt, float dso, const double* d_angles,
                    const double* d_zpos, int64_t v0, int64_t v1, double i0, uint64_t seed,
                    float* d_fan, lct_stream stream);

/* Voxelised phantom on the GPU (training targets): mean attenuation over ss^3 sub-samples per
   voxel, d_out [nz][ny][nx], voxel (ix, iy, iz) centred at (x0 + ix dx, y0 + iy dy, z0 + iz dz).
   Asynchronous. */
int lct_voxelise(const double* d_ellipsoids, int n_ellipsoids, int nx, int ny, int nz, double x0,
                 double y0, double z0, double dx, double dy, double dz, int ss, float* d_out,
                 lct_stream stream);

/* ---------------------------------------------------------------------------------------
 * Learned 2.5D residual correction (no reference counterpart: the reference stops at the FDK
 * volume).  5 neighbouring slices of the calibrated FDK volume in, 8 zero-padded 3x3
 * convolutions (5->32, 6 x 32->32, 32->1) with ReLU between them, a residual r out:
 *   plain(z)     = calib * fdk(z)                       (calibrated plain FDK, phantom units)
 *   network in   = bf16(calib * in_scale * fdk(z-2..z+2))
 *   corrected(z) = plain(z) + r / in_scale   where |r / in_scale| <= bound, else plain(z)
 * BF16 weights and activations, FP32 accumulation, tcgen05 implicit-GEMM convolutions.
 * Parameters: 57,249 floats, for l = 0..7: W_l[cout][cin][3][3], then b_l[cout]
 * (FP32 master copy; Adam state on the device).
 * ------------------------------------------------------------------------------------- */
#define LCT_CNN_TRAIN 1 /* keep every activation and the deltas (training); else inference only */
typedef struct lct_cnn lct_cnn;
int lct_cnn_param_count(int64_t* n);
/* Workspace for up to max_slices slices of ny x nx; weights He-initialised from seed.
   Synchronous. */
int lct_cnn_create(int max_slices, int ny, int nx, int flags, uint64_t seed, lct_cnn** out);
/* Parameter copies (host or device pointers; synchronous: they wait for all work on the device
   first).  set_params resets the Adam state. */
int lct_cnn_set_params(lct_cnn* c, const float* params, int on_device);
int lct_cnn_get_params(const lct_cnn* c, float* params, int on_device);
int lct_cnn_get_grads(const lct_cnn* c, float* grads, int on_device);
int lct_cnn_set_scales(lct_cnn* c, float calib, float in_scale);
int lct_cnn_get_scales(const lct_cnn* c, float* calib, float* in_scale);
/* Training (LCT_CNN_TRAIN workspaces).  d_in5 [n][5][ny][nx]: FDK slices z-2..z+2 (raw FDK
   units); d_target [n][ny][nx]: phantom slices (phantom units).  forward writes the residual r
   (network units) to d_resid when non-null; backward (after forward on the same inputs)
   computes the gradient of mean((in_scale*plain + r - in_scale*target)^2); adam_step updates
   the FP32 master weights; train_step = forward + backward + adam_step(0.9, 0.999, 1e-8).
   Asynchronous on the stream. */
int lct_cnn_forward(lct_cnn* c, const float* d_in5, int n_slices, float* d_resid,
                    lct_stream stream);
int lct_cnn_backward(lct_cnn* c, const float* d_in5, const float* d_target, int n_slices,
                     lct_stream stream);
int lct_cnn_adam_step(lct_cnn* c, float lr, float beta1, float beta2, float eps,
                      lct_stream stream);
int lct_cnn_train_step(lct_cnn* c, const float* d_in5, const float* d_target, int n_slices,
                       float lr, lct_stream stream);
/* loss of the last backward pass (synchronous: waits for all work on the device) */
int lct_cnn_last_loss(const lct_cnn* c, double* loss);
/* Inference with the acceptance gate over a device volume d_vol [nz][ny][nx] (raw FDK) ->
   d_out (corrected, phantom units; must not alias d_vol), max_slices slices per pass, edge
   slices replicated.  n_rejected (host, may be NULL): voxels where the gate kept the plain
   value; when given, the call synchronises the stream. */
int lct_cnn_infer_volume(lct_cnn* c, const float* d_vol, float* d_out, int nz, float bound,
                         int64_t* n_rejected, lct_stream stream);
/* rejected-voxel count of the last infer_volume (synchronous: waits for all work on the device) */
int lct_cnn_last_rejected(const lct_cnn* c, int64_t* n);
int lct_cnn_get_shape(const lct_cnn* c, int* max_slices, int* ny, int* nx);
void lct_cnn_destroy(lct_cnn* c);

/* Fused learned correction in lct_recon_run (c = NULL turns it off; c is not owned and must
   outlive its use; its ny, nx must match the plan's image).  The run then backprojects into an
   internal plain volume and writes the gated corrected volume to `image`.  learned_info: ms of
   the correction in the last run (inside the backprojection -> download span of
   lct_recon_last_times) and its rejected-voxel count; either pointer may be NULL. */
int lct_recon_set_learned(lct_recon* r, lct_cnn* c, float bound);
int lct_recon_learned_info(const lct_recon* r, float* ms, int64_t* rejected);

#ifdef __cplusplus
}
#endif
#endif /* LCT_H */
