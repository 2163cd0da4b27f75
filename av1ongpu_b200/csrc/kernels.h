/*
 * kernels.h - the argument blocks of the frame-step kernels and their
 * launchers (kernels.cu). Host code fills these and launches on its stream.
 */
#ifndef AV1B_KERNELS_H
#define AV1B_KERNELS_H

#include <cuda_runtime.h>

#include "dev_common.cuh"
#include "dev_filters.cuh"
#include "filter_prep.cuh"

namespace av1b {

#define AV1B_STATUS_TIMEOUT 1   /* a dependency wait gave up */

/* Everything the reconstruction kernels read, by value. */
/* Done flags sit 128 bytes apart: the blocks in flight are neighbours in
 * coding order, and flags sharing lines would pile every poll of the frontier
 * onto a few L2 slices, slowing every other access there. */
#define AV1B_FLAG_STRIDE 32

/* Phase B: shared-memory scratch per warp (ints) - the residual image of a
 * block whose prediction and residual fuse (so blocks of up to this many
 * samples fuse) and, for filter intra (at most 32x32), its predictions at
 * offset 1024 - and the CTAs of four warps resident per SM. Blocks up to
 * 64x64 fuse: the unfused path reads the prediction back through L2, a
 * round trip a batch of samples that costs a 64x64 block tens of
 * microseconds on the dependency path, more than the halved residency (two
 * CTAs a SM instead of four) costs. */
#define AV1B_UNIT_SCRATCH 4096
/* superres: output samples of a row a CTA writes; loop restoration: the
 * columns of a tile */
#define AV1B_UP_OUT 512
#define AV1B_LR_TW 32
#define AV1B_UNIT_CTAS_PER_SM 2
/* deblocking: the edge records a warp takes at once in the batched form and
 * in a single stream's launch */
#define AV1B_DB_GROUP 8
#ifndef AV1B_DB_PLAIN
#define AV1B_DB_PLAIN 2
#endif

struct FrameArgs {
  Layout L;
  px_t* cur;                    /* the picture being reconstructed */
  px_t* const* slot_ptr;        /* device array: base of each reference slot */
  const BlockRec* blocks;
  int n_blocks;
  const TxRec* txs;
  const ObmcRec* obmc;
  const WarpRec* warps;
  const int* coef;
  const int* residual;
  const uint8_t* palette_map;
  const int* palette_colors;    /* 8 per palette block */
  unsigned* done;               /* per block, AV1B_FLAG_STRIDE apart: == epoch once
                                   reconstructed (phase B) */
  unsigned epoch;
  const int* units;             /* phase B block indices, chain after chain */
  const int* chains;            /* chain c is units[chains[c] .. chains[c + 1]) */
  int n_chains;
  const int* deps;              /* the phase B blocks each phase B block waits for */
  int units_inter;              /* some phase B block is an inter kind */
  int n_units;
  unsigned* queue;
  const int2* inter_tiles;      /* phase A: (block, x0 | y0 << 16) */
  int n_inter_tiles;
  int n_inter_simple;           /* the first ones: unmasked blocks (the lean kernel) */
  int n_inter_lmask;            /* the next ones: wedge and luma difference-weighted
                                   compounds (the lean kernel's masked build) */
  int n_inter_cmask;            /* the last ones: chroma tiles reading a luma mask */
  unsigned char* mask_pool;     /* blend masks of difference-weighted luma blocks */
  const int2* itx_jobs;         /* phase A: (block, transform); the transforms of
                                   phase B blocks compute their residual ahead */
  int n_itx;
  const int4* itx_batches;      /* (first job, jobs, log2 size class or 7 raw) */
  int n_itx_batches;
  int itx_class_first[8], itx_class_count[8];   /* the batches of each class */
  int* pre_res;                 /* residuals computed ahead (TxRec::pre_off) */
  int* status;
  int maxv;
  int scale_x, scale_y;
  unsigned long long wait_ns;   /* limit of one dependency wait */
  unsigned long long* trace;    /* null, or 4 per block: claimed, ready, published
                                   (globaltimer ns), last dependency */
};

struct LrArgs {
  int type[3];                  /* non-zero: the plane is restored */
  int unit_size[3], unit_rows[3], unit_cols[3], n_units[3];
  const LrUnitRec* units[3];
};

/* The film grain parameters the template kernel reads. */
struct GrainParamsDev {
  int seed, bitdepth, ss_x, ss_y;
  int num_y_points, num_cb_points, num_cr_points, chroma_scaling_from_luma;
  int ar_coeff_lag, ar_coeff_shift_minus_6, grain_scale_shift;
  int ar_y[24], ar_cb[25], ar_cr[25];
};

/* superres: per plane, the Q14 step and the phase of the first column */
struct UpscaleArgs {
  int step[3], initial[3];
};

struct RgbArgs {
  int m[8];
  int o[3];
};

cudaError_t set_kernel_attributes();
cudaError_t launch_selftest_wait(const unsigned* flag, int* status, unsigned long long limit_ns,
                                 cudaStream_t s);
/* stage 1: phase A prediction; 2: the inverse transforms (phase A residual
 * added, phase B residual computed ahead); 3: the dependency-scheduled
 * phase B. */
cudaError_t launch_recon_stage(int stage, const FrameArgs& a, int n_sm, cudaStream_t s);
cudaError_t launch_prep_filters(const av1b_deblock_edge* edges, int n_edges, const av1b_cdef_block* cdef,
                                int n_cdef, const Layout& L, int grid_w, int grid_n, DeblockRec* v,
                                DeblockRec* h, CdefRec* cdef_out, unsigned* extra, PrepOut* out,
                                cudaStream_t s);
cudaError_t launch_dequant(const DqRec* jobs, int n, const short* levels, const unsigned char* qm,
                           int* coef, int bit_depth, cudaStream_t s);
cudaError_t launch_deblock(px_t* pic, const DeblockRec* recs, int n, int sharpness, int bd,
                           int maxv, cudaStream_t s);
/* CDEF: the direction searches - every 8x8 luma block of a grid_w-wide grid
 * (grid_n cells) when `grid`, then the n_extra positions off the grid (x | y
 * << 16, results after the grid's) - then the filter of every record. */
cudaError_t launch_cdef(const px_t* src, px_t* dst, const CdefRec* recs, int n, int grid_w,
                        int grid_n, bool grid, const unsigned* extra_pos, int n_extra, int* search,
                        const Layout& L, cudaStream_t s);
/* border_rows: only the rows within two of a loop restoration stripe
 * boundary (for the pre-CDEF picture loop restoration reads). */
cudaError_t launch_upscale(const px_t* src, px_t* dst, const Layout& L, int maxv, bool border_rows,
                           cudaStream_t s);
cudaError_t launch_lr(const px_t* cdef, const px_t* curr, px_t* dst, const Layout& L,
                      const LrArgs& r, int maxv, bool copy_rest, cudaStream_t s);
cudaError_t launch_grain_template(GrainState* gs, const GrainParamsDev& prm, const uint16_t* orbit,
                                  const uint16_t* pos, cudaStream_t s);
cudaError_t launch_grain_blend(const px_t* src, px_t* dst, const Layout& L, const GrainState* gs,
                               const uint16_t* orbit, const uint16_t* pos, cudaStream_t s);
cudaError_t launch_nv12(const px_t* pic, uint8_t* out, const Layout& L, int pitch, cudaStream_t s);
/* NV12 of `pic` before film grain, the grain (state `gs`) applied while packing. */
cudaError_t launch_nv12_grain(const px_t* pic, uint8_t* out, const Layout& L, int pitch,
                              const GrainState* gs, const uint16_t* orbit, const uint16_t* pos,
                              cudaStream_t s);
cudaError_t launch_rgb(const px_t* pic, uint8_t* out, const Layout& L, const RgbArgs& m,
                       cudaStream_t s);

}  // namespace av1b

#endif
