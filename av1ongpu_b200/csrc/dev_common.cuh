/*
 * dev_common.cuh - shared device definitions: sample type, frame layout, job
 * records, and the scalar helpers every stage uses.
 *
 * All arithmetic is integer. Every rounding helper states which of the
 * specification's operators it is, because the two Round2 variants (and the
 * arithmetic shift) disagree on negative numbers and a decoder is bit exact
 * only if each call site uses the right one.
 */
#ifndef AV1B_DEV_COMMON_CUH
#define AV1B_DEV_COMMON_CUH

#include <cstdint>

#include "av1b_tables.h"

#define AV1B_DEV __device__ __forceinline__
#define AV1B_HD __host__ __device__ __forceinline__

namespace av1b {

typedef uint16_t px_t; /* one sample, 16 bits at every bit depth */

/* ---- scalar helpers --------------------------------------------------------- */
AV1B_HD int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* A strided walk over a row-major n-wide rectangle: element k = r * n + q,
 * from `start` in steps of `step`, with (r, q) advanced without a division
 * per step (step % n < n, so one carry suffices). */
struct StepWalk {
  int k, r, q, dr, dq, n;
  __device__ __forceinline__ StepWalk(int start, int step, int n_) : k(start), n(n_) {
    r = start / n;
    q = start - r * n;
    dr = step / n;
    dq = step - dr * n;
    dk = step;
  }
  __device__ __forceinline__ void next() {
    k += dk;
    r += dr;
    q += dq;
    if (q >= n) {
      q -= n;
      ++r;
    }
  }
  int dk;
};
AV1B_HD int mini(int a, int b) { return a < b ? a : b; }
AV1B_HD int maxi(int a, int b) { return a > b ? a : b; }
AV1B_HD int absi(int v) { return v < 0 ? -v : v; }
/* Round2(x, n) for n >= 1: (x + 2^(n-1)) >> n with an arithmetic shift. */
AV1B_HD int rnd2(int x, int n) { return (x + (1 << (n - 1))) >> n; }
/* Round2 that passes x through when n == 0. */
AV1B_HD int rnd2z(int x, int n) { return n == 0 ? x : (x + (1 << (n - 1))) >> n; }
AV1B_HD int rnd2ll(long long x, int n) { return (int)((x + (1LL << (n - 1))) >> n); }
AV1B_HD int rnd2llz(long long x, int n) { return n == 0 ? (int)x : (int)((x + (1LL << (n - 1))) >> n); }
/* Round2Signed: the rounding offset is applied to the magnitude. */
AV1B_HD int rnd2s(int x, int n) {
  if (n == 0) return x;
  return x >= 0 ? (x + (1 << (n - 1))) >> n : -((-x + (1 << (n - 1))) >> n);
}
/* (x + 2^(n-1) + sign) >> n: Round2Signed written with one shift (the form the
 * reference uses in its scaled prediction path, av1gpu_kernels.h:81-84). */
AV1B_HD int rnd2s_shift(int x, int n) { return (x + (1 << (n - 1)) + (x < 0 ? -1 : 0)) >> n; }
AV1B_HD int ilog2(int v) {
  int n = 0;
  while ((1 << n) < v) ++n;
  return n;
}
AV1B_HD int floor_log2(int v) {
  int n = 0;
  while (v > 1) {
    v >>= 1;
    ++n;
  }
  return n;
}

/* A sample of the picture being reconstructed, read through L2: another SM
 * wrote it and published it with a release flag. */
#ifdef __CUDACC__
__device__ __forceinline__ int ldpx(const px_t* p) { return (int)__ldcg(p); }
#endif

/* Sm_Weights for a block side of n; any n other than 4, 8, 16, 32 reads the
 * 64-sample table, as the reference's av1g_sm_weight does. */
__device__ __forceinline__ int sm_weight(int n, int i) {
  const int base = n == 4 ? 0 : (n == 8 ? 4 : (n == 16 ? 12 : (n == 32 ? 28 : 60)));
  return kSmWeights[base + i];
}

/* ---- frame layout --------------------------------------------------------------
 * One picture is one allocation with the three planes back to back. The
 * stride follows the display width (a superres frame is reconstructed narrow
 * and upscaled in place of the same rows) and is a multiple of 64 samples so
 * rows start on 128-byte lines. Blocks may overhang the coded picture by up
 * to 64 luma samples on the right and at the bottom, which the padding holds.
 */
struct PlaneGeom {
  int off;          /* sample offset of the plane in the picture buffer */
  int stride;       /* samples per row */
  int coded_w, coded_h;   /* the reconstructed (coded) plane */
  int out_w, out_h;       /* the display plane (after superres) */
  int grid_w, grid_h;     /* coded size rounded up to the 8x8 luma grid */
};

struct Layout {
  PlaneGeom p[3];
  int ss_x, ss_y, bit_depth;
  long long size; /* samples per picture */
};

/* ---- intra / unit records (phase B: dependency scheduled) ------------------- */
/* flags */
#define AV1B_U_INTRA 0          /* kind: intra transform block */
#define AV1B_U_INTERINTRA 1     /* kind: inter block with an intra blend */
#define AV1B_U_INTRABC 2        /* kind: intra block copy */

/* The per block record every reconstruction kernel reads. Fields a kind does
 * not use are zero. 128 bytes. */
struct BlockRec {
  short x, y, w, h;           /* plane samples */
  unsigned char plane, kind, is_inter, mode;
  signed char angle_delta, filter_type, cfl_alpha, fi_mode;   /* fi_mode -1: none */
  unsigned char have_left, have_above, have_ar, have_bl;      /* have_ar/bl: 0/1, 2 = derive */
  unsigned char lossless, residual_provided, palette, palette_size;
  int palette_off, palette_stride;
  int tx_first, tx_count;
  /* inter */
  int ref_slot[2];            /* device slot, -1: the picture being decoded */
  int mv[2][2];
  unsigned char filt, filt_v, compound, mask_kind;   /* compound: 0 none 1 avg 2 dist; mask 0/1 wedge/2 diffwtd */
  unsigned char w0, w1, mask_sign, ii_mode;
  unsigned char interintra, ii_wedge, wedge_dir, wedge_flip;
  signed char wedge_xoff, wedge_yoff, warp0, warp1;
  unsigned char mask_warp0, mask_warp1, phase_b;   /* phase_b: dependency scheduled */
  unsigned char fuse_res;     /* phase B: the transforms tile disjoint parts of the
                                 block, so prediction and residual add fuse */
  int warp_idx[2];            /* into the frame's warp model table, -1 none */
  int obmc_first, obmc_count;
  int palette_color_idx;      /* into the palette colour table */
  int dep_first, dep_count;   /* phase B: the blocks it waits for (frame's dep list) */
  /* a difference-weighted compound: 1 - a luma block that writes its blend
   * mask (a byte a sample, mask_w a row) at mask_off of the frame's mask
   * pool; 2 - a chroma block whose luma block is the same prediction, which
   * reads that mask instead of predicting the luma itself; 0 - neither */
  int mask_off;
  short mask_w;
  unsigned char mask_role, pad_mask;
};

/* One coded transform of a frame whose coefficients arrive as coded levels:
 * where its raster goes in the coefficient pool, where its levels start, and
 * its dequantiser. 32 bytes. */
struct DqRec {
  int coef_off;               /* the raster, (1 << alw) x (1 << alh) ints */
  int level_off;              /* first of `count` levels, in scan order */
  int count;                  /* min(eob, raster area) */
  int dc_step, ac_step;
  int qm_off;                 /* into the frame's QM pool, -1: no matrix */
  unsigned short scan_off;    /* into the scan table */
  unsigned short denom;       /* 1, 2 or 4 (the 32 and 64 point families) */
  unsigned char alw, alh;     /* log2 of the raster's width and height (2..5) */
  unsigned char pad[2];
};

/* One transform of a block: position relative to the block. 16 bytes. */
struct TxRec {
  int coef_off;               /* into the coefficient (or residual) pool */
  short x, y;
  short w, h;                 /* 4..64 for a transform; any size for raw residual */
  unsigned char log2w, log2h, type, row_shift;
  int pre_off;                /* >= 0: the residual is computed ahead, here in the
                                 precomputed residual buffer (w * h, row-major) */
};

/* One OBMC strip. */
struct ObmcRec {
  short pass, x, y, w, h;
  short filt, filt_v;
  int mv_x, mv_y;
  int ref_slot;
};

/* One global warp model with its shear (computed on the host per model). */
struct WarpRec {
  int params[6];
  int abcd[4];
};

}  // namespace av1b

#endif
