/*
 * wedge.h - the wedge master mask (specification 7.11.3.11,
 * initialise_wedge_mask_table), usable from host and device code: the host
 * needs it for the codebook's sign choice, the device for the mask itself.
 * Same construction as the reference's av1g_wedge_1d / _ob63 / _master
 * (av1gpu_kernels.h:1968-2003).
 */
#ifndef AV1B_WEDGE_H
#define AV1B_WEDGE_H

#if defined(__CUDACC__)
#define AV1B_WEDGE_FN __host__ __device__ __forceinline__
#else
#define AV1B_WEDGE_FN inline
#endif

namespace av1b {

/* The one dimensional templates: the two oblique rasters (even and odd rows)
 * and the vertical one, 0 below the ramp and 64 above it. */
AV1B_WEDGE_FN int wedge_1d(int which, int j) {
  const int even[8] = {1, 4, 11, 27, 46, 58, 62, 63};
  const int odd[8] = {1, 2, 6, 18, 37, 53, 60, 63};
  const int vertical[6] = {2, 7, 21, 43, 57, 62};
  if (which == 2) return j < 29 ? 0 : (j >= 35 ? 64 : vertical[j - 29]);
  if (j < 28) return 0;
  if (j >= 36) return 64;
  return which == 0 ? even[j - 28] : odd[j - 28];
}

/* The 63-degree raster: one step every two rows, odd rows one step ahead. */
AV1B_WEDGE_FN int wedge_ob63(int i, int j) {
  const int k = i >> 1;
  const int shift = (i & 1) ? (15 - k) : (16 - k);
  int c = j - shift;
  c = c < 0 ? 0 : (c > 63 ? 63 : c);
  return wedge_1d(i & 1, c);
}

/* MasterMask[dir][i][j]: 0 horizontal, 1 vertical, 2 oblique27, 3 oblique63,
 * 4 oblique117, 5 oblique153. */
AV1B_WEDGE_FN int wedge_master(int dir, int i, int j) {
  switch (dir) {
    case 0: return wedge_1d(2, i);
    case 1: return wedge_1d(2, j);
    case 2: return wedge_ob63(j, i);
    case 4: return 64 - wedge_ob63(i, 63 - j);
    case 5: return 64 - wedge_ob63(j, 63 - i);
    default: return wedge_ob63(i, j);
  }
}

}  // namespace av1b

#endif
