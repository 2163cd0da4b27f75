/*
 * plan_host.h - host-side helpers of the frame planner that read the
 * specification's tables (compiled by the host compiler, plan_host.cpp).
 */
#ifndef AV1B_PLAN_HOST_H
#define AV1B_PLAN_HOST_H

#include <cstdint>

namespace av1b {

/* setup_shear (7.11.3.6): alpha..delta of a global warp model. Returns false
 * when the shear is too steep (warpValid = 0). */
bool gm_setup_shear(const int32_t* params, int* alpha, int* beta, int* gamma, int* delta);

/* The wedge codebook entry of a luma block size: master mask direction, mask
 * origin and whether the block reads 64 - mask. False: no wedge at this size. */
bool wedge_entry(int block_w, int block_h, int wedge_index, int* dir, int* xoff, int* yoff,
                 int* flip);

/* scaling_lookup_initialization (7.18.3.4): the 256-entry curve of a plane. */
void grain_scaling_lut(int num_points, const int32_t* value, const int32_t* scaling, int* lut);

/* Sgr_Params[16][4] (r0, e0, r1, e1), for the host. */
const short* sgr_params_table();

/* The Q16 YUV -> RGB matrix with range offsets folded in. */
void color_matrix(int matrix, int range, int bit_depth, int m[8], int o[3]);

}  // namespace av1b

#endif
