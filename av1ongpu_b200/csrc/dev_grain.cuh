/*
 * dev_grain.cuh - one sample of the film grain output process (7.18.3.5):
 * the noise sample computed on its own from the grain templates, scaled by
 * the plane's curve and added. Used by the no-allocation entry point
 * (noalloc.cu); the arithmetic is that of the decoder's k_grain_blend.
 *
 * The reference builds the whole noise image on the host (grain.cpp:70-198,
 * av1gpu_kernels.h:3201-3291): square blocks cut from the templates at a
 * random offset per block, stitched into 32-row stripes with a 2-column
 * overlap blend (1 at 4:2:0 chroma), the stripes blended over 2 rows (1). A
 * sample of that image depends only on the block that covers it, the block
 * before it, and the stripe above - and the random offset of a block is the
 * LFSR state a fixed number of steps after the stripe's seed, which the orbit
 * table gives directly. So each output sample evaluates its noise value here.
 */
#ifndef AV1B_DEV_GRAIN_CUH
#define AV1B_DEV_GRAIN_CUH

#include "dev_filters.cuh"

namespace av1b {

/* The stripe value of plane `p` at (row, col) of stripe `s` (the horizontal
 * half): the grain block that covers the column, blended with the previous
 * block at the two (one for subsampled chroma) overlap columns. */
__device__ __forceinline__ int grain_stripe(const GrainState* gs, const short* grain, int src_w, int sub_x, int sub_y,
                            int s, int row, int col, const uint16_t* orbit, const uint16_t* pos,
                            int gmin, int gmax) {
  unsigned st0 = (unsigned)gs->seed & 0xffffu;
  st0 ^= (unsigned)(((s * 37 + 178) & 255) << 8);
  st0 ^= (unsigned)((s * 173 + 105) & 255);
  st0 &= 0xffffu;
  const int bw_log = sub_x ? 4 : 5;
  const int k = col >> bw_log;
  const int j = col & ((1 << bw_log) - 1);
  auto sample = [&](int blk, int jj) {
    const int r = (lfsr_after(orbit, pos, st0, blk + 1) >> 8) & 255;
    const int ox = r >> 4, oy = r & 15;
    const int src_x = sub_x ? 6 + ox : 9 + ox * 2;
    const int src_y = sub_y ? 6 + oy : 9 + oy * 2;
    return (int)grain[(src_y + row) * src_w + src_x + jj];
  };
  int g = sample(k, j);
  if (gs->overlap && k > 0) {
    if (!sub_x && j < 2) {
      const int old = sample(k - 1, j + 32);
      g = clampi(rnd2z(j == 0 ? old * 27 + g * 17 : old * 17 + g * 27, 5), gmin, gmax);
    } else if (sub_x && j == 0) {
      const int old = sample(k - 1, 16);
      g = clampi(rnd2z(old * 23 + g * 22, 5), gmin, gmax);
    }
  }
  return g;
}


/* One output sample of plane p at (x, y): `orig` is its decoded value; for a
 * chroma sample l0 / l1 are the co-located luma sample and its right
 * neighbour (clamped to the luma width), both before grain. */
__device__ __forceinline__ int grain_sample(const GrainState* gs, const uint16_t* orbit,
                                            const uint16_t* pos, int p, int sub_x, int sub_y, int x,
                                            int y, int orig, int l0, int l1) {
  const int bd = gs->bitdepth;
  const bool active = p == 0 ? gs->num_points[0] > 0 : (gs->chroma_from_luma || gs->num_points[p] > 0);
  if (!active) return orig;
  const int gmin = -(128 << (bd - 8)), gmax = (256 << (bd - 8)) - 1 - (128 << (bd - 8));
  const short* grain = p == 0 ? gs->luma : (p == 1 ? gs->cb : gs->cr);
  const int src_w = p == 0 ? 82 : gs->chroma_w;
  /* vertical half: stripes of 32 (16) rows, blended with the stripe above */
  const int sh = 5 - sub_y;
  const int s = y >> sh, row = y - (s << sh);
  int n = grain_stripe(gs, grain, src_w, sub_x, sub_y, s, row, x, orbit, pos, gmin, gmax);
  if (gs->overlap && s > 0) {
    if (!sub_y && row < 2) {
      const int old = grain_stripe(gs, grain, src_w, sub_x, sub_y, s - 1, row + 32, x, orbit, pos,
                                   gmin, gmax);
      n = clampi(rnd2z(row == 0 ? old * 27 + n * 17 : old * 17 + n * 27, 5), gmin, gmax);
    } else if (sub_y && row == 0) {
      const int old = grain_stripe(gs, grain, src_w, sub_x, sub_y, s - 1, 16, x, orbit, pos, gmin,
                                   gmax);
      n = clampi(rnd2z(old * 23 + n * 22, 5), gmin, gmax);
    }
  }
  int index;
  if (p == 0) {
    index = orig;
  } else {
    int avg = l0;
    if (sub_x) avg = rnd2z(l0 + l1, 1);
    if (gs->chroma_from_luma) {
      index = avg;
    } else {
      const int comb = avg * (gs->luma_mult[p] - 128) + orig * (gs->mult[p] - 128);
      index = clampi((comb >> 6) + (gs->offset[p] - 256) * (1 << (bd - 8)), 0, (1 << bd) - 1);
    }
  }
  const int scaled = rnd2z(grain_scale_lut(gs->lut[p], index, bd) * n, gs->scaling_shift);
  return clampi(orig + scaled, gs->min_value, p == 0 ? gs->max_luma : gs->max_chroma);
}

}  // namespace av1b

#endif
