/*
 * batch.h - the device descriptors of the batched form: one frame of each of
 * up to AV1B_BATCH_MAX independent streams decoded by one set of persistent
 * kernels (kernels.cu, "batched form"), and their launchers.
 *
 * A batched step is a fixed sequence of stage kernels, each launched once for
 * every stream of the step with a grid sized to the GPU (CTAs per SM times
 * the SM count, from the tuned configuration) rather than to the work. A
 * stage kernel takes work items from the step's device descriptors: the
 * per-stream arguments (StreamStep) and, per stage, the prefix sums of every
 * stream's item count, so item i belongs to the stream s with
 * pfx[s] <= i < pfx[s + 1]. Warp-level stages (prediction tiles, transform
 * batches, deblocking edges, dependency chains) claim items from a counter in
 * the header; CTA-level stages (filters on picture tiles) stride over them.
 * Nothing in the launch depends on the frames, so a step is one CUDA graph
 * replayed with new descriptors.
 */
#ifndef AV1B_BATCH_H
#define AV1B_BATCH_H

#include "kernels.h"

namespace av1b {

#define AV1B_BATCH_MAX 64

/* The stages of a batched step, in launch order. */
enum BatchStage {
  kBInterSimple, kBInterLeanMask, kBInter, kBInterMask,
  kBItx2, kBItx3, kBItx4, kBItx5, kBItx6, kBItx7,
  kBUnits,
  kBDeblockV, kBDeblockH,
  kBCopySnap, kBCdefSearch, kBCdef, kBCopyPost,
  kBUpscale, kBLr, kBCopyRef,
  kBGrainTemplate, kBGrain, kBNv12,
  kBStageCount
};

/* A copy stage moves a picture in items of this many bytes (a CTA each). */
#define AV1B_COPY_ITEM 16384

/* Per stream: what the filter chain of the frame reads and writes. Every
 * stage the frame does not need has no items. */
struct FilterArgs {
  int maxv, bd, sharpness;
  const DeblockRec* dbv;
  const DeblockRec* dbh;
  int n_dbv, n_dbh;
  /* CDEF: the searches (the grid when n_grid > 0, then the extra positions)
   * and the records */
  const px_t* cdef_src;
  px_t* cdef_dst;
  const CdefRec* cdef;
  int n_cdef, cdef_grid_w, cdef_grid_n, cdef_n_grid, n_cdef_extra;
  const unsigned* cdef_extra;
  int* cdef_search;
  /* copies: the snapshot before CDEF, the one after it, the reference store */
  const px_t* copy_src[3];
  px_t* copy_dst[3];
  long long copy_items[3];        /* AV1B_COPY_ITEM pieces (the bytes are a multiple of 16) */
  long long copy_bytes[3];
  /* superres: up to two passes (the rows loop restoration reads from the
   * pre-CDEF picture, then the picture) */
  const px_t* up_src[2];
  px_t* up_dst[2];
  int up_border[2], up_rows0[2], up_segs[2], up_items[2];
  UpscaleArgs up;
  /* loop restoration */
  const px_t* lr_cdef;
  const px_t* lr_curr;
  px_t* lr_dst;
  int lr_copy_rest, lr_tiles, lr_stripes;
  LrArgs lr;
  /* film grain: templates from the parameters, then the blend cur -> disp */
  int grain;
  const int* gs_src;              /* the plan's grain constants (GrainState from lut on) */
  GrainState* gs;
  GrainParamsDev gp;
  const uint16_t* orbit;
  const uint16_t* pos;
  const px_t* grain_src;
  px_t* grain_dst;
  int grain_xblocks, grain_rows;
  /* NV12 output (null: none), packed from nv12_src; with fuse_grain the
   * grain of the packed samples is computed while packing and grain_dst is
   * not written */
  uint8_t* nv12;
  const px_t* nv12_src;
  int nv12_pitch, nv12_xblocks, nv12_rows, fuse_grain;
};

struct StreamStep {
  FrameArgs a;
  FilterArgs f;
};

/* The step's header: stream count, item prefix sums per stage, the claim
 * counters (zeroed at the start of every step) and the merged chain order of
 * the dependency-scheduled phase: (stream, chain) pairs, each stream's chains
 * in its own claim order, streams interleaved by chain depth (aligned at the
 * ends of their dependency paths). */
struct BatchHeader {
  int n;
  int pfx[kBStageCount][AV1B_BATCH_MAX + 1];
  unsigned claim[kBStageCount];
  int n_chain_order;
  const int2* chain_order;
};

/* CTAs per SM of each persistent stage kernel, the items a warp claims at
 * once, the build of the full prediction kernel (the autotuner's knobs);
 * fuse_grain_nv12: the grain of a frame whose output is only its NV12 pack
 * is applied inside the pack. */
struct BatchTuning {
  int ctas_per_sm[kBStageCount];
  int claim_chunk;
  int fuse_grain_nv12;
  int inter_variant;              /* the build of the full prediction kernel: 0 / 1 */
};

cudaError_t set_batch_kernel_attributes();
/* The most CTAs of a stage's kernel one SM holds (its registers, shared
 * memory and block size), at least 1. */
int batch_stage_max_ctas(int stage);
/* Queues the stage kernels of one batched step on `s` (and the grain
 * templates on `side`, joined before the blend). `steps` and `hdr` are
 * device memory the caller filled; `units_inter`: some stream's phase B has
 * inter blocks. */
cudaError_t launch_batch_step(const StreamStep* steps, BatchHeader* hdr, const BatchTuning& t,
                              int n_sm, bool units_inter, cudaStream_t s, cudaStream_t side,
                              cudaEvent_t fork, cudaEvent_t join, cudaEvent_t* prof = nullptr);

}  // namespace av1b

#endif
