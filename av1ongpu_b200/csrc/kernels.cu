/*
 * kernels.cu - the sm_100a kernels of one frame step.
 *
 * Reconstruction runs in two phases. Phase A is everything that reads only
 * reference pictures: the inter prediction of every inter block (one warp per
 * 16x8 tile), then every inverse transform (one warp per transform) - added
 * to the picture for inter blocks, left in a buffer for the rest. Phase B is
 * the dependency-scheduled rest: intra blocks, inter-intra blocks and intra
 * block copies, by a persistent kernel whose warps claim blocks from a device
 * queue, wait for the blocks whose samples they read and add the residual
 * computed ahead. What each block waits for comes from the planner, which
 * resolves the reference's owner grids and edge scans (engine.cpp:719-924)
 * into a short list per block and orders the claims by dependency depth: the
 * host launches nothing per wave.
 *
 * Waiting is safe without a cooperative launch: a block only ever waits on
 * blocks claimed before it, each by a warp that is already running (or has
 * finished it), so the first unfinished block in claim order always has
 * everything it needs. Every wait is bounded (one second of globaltimer); on
 * expiry the kernel records AV1B_STATUS_TIMEOUT in the status word and
 * carries on, and the host fails the frame.
 */
#include <cuda_runtime.h>

#include "dev_common.cuh"
#include "dev_filters.cuh"
#include "dev_inter.cuh"
#include "dev_intra.cuh"
#include "dev_itx.cuh"
#include "kernels.h"
#include "batch.h"

namespace av1b {

/* ---- helpers --------------------------------------------------------------------- */
__device__ __forceinline__ unsigned ld_relaxed(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ const px_t* ref_plane(const FrameArgs& a, int slot, int plane) {
  const px_t* base = slot >= 0 ? a.slot_ptr[slot] : a.cur;
  return base + a.L.p[plane].off;
}

/* Builds the resolved inter job of a block. */
__device__ void make_inter_job(const FrameArgs& a, const BlockRec& b, InterJob* j) {
  const int p = b.plane;
  const PlaneGeom& g = a.L.p[p];
  j->x = b.x;
  j->y = b.y;
  j->w = b.w;
  j->h = b.h;
  j->plane = p;
  j->ctx.sub_x = p > 0 ? a.L.ss_x : 0;
  j->ctx.sub_y = p > 0 ? a.L.ss_y : 0;
  j->ctx.bitdepth = a.L.bit_depth;
  if (b.kind == AV1B_U_INTRABC) {
    /* a block copy reads this frame: the 4-rounded coded size, unscaled */
    j->ctx.ref_w = ((a.L.p[0].coded_w + 3) & ~3) >> j->ctx.sub_x;
    j->ctx.ref_h = ((a.L.p[0].coded_h + 3) & ~3) >> j->ctx.sub_y;
    j->ctx.scale_x = AV1B_SCALE_ONE;
    j->ctx.scale_y = AV1B_SCALE_ONE;
  } else {
    j->ctx.ref_w = g.out_w;
    j->ctx.ref_h = g.out_h;
    j->ctx.scale_x = a.scale_x;
    j->ctx.scale_y = a.scale_y;
  }
  j->ref[0] = ref_plane(a, b.ref_slot[0], p);
  j->ref[1] = ref_plane(a, b.ref_slot[1], p);
  j->ref_stride = g.stride;
  for (int r = 0; r < 2; ++r) {
    j->mv[r][0] = b.mv[r][0];
    j->mv[r][1] = b.mv[r][1];
  }
  j->filt = b.filt;
  j->filt_v = b.filt_v;
  j->compound = b.compound;
  j->w0 = b.w0;
  j->w1 = b.w1;
  j->mask_kind = b.mask_kind;
  j->mask_sign = b.mask_sign;
  j->wedge_dir = b.wedge_dir;
  j->wedge_xoff = b.wedge_xoff;
  j->wedge_yoff = b.wedge_yoff;
  j->wedge_flip = b.wedge_flip;
  j->warp[0] = b.warp0;
  j->warp[1] = b.warp1;
  j->mask_warp[0] = b.mask_warp0;
  j->mask_warp[1] = b.mask_warp1;
  j->model[0] = a.warps + (b.warp_idx[0] >= 0 ? b.warp_idx[0] : 0);
  j->model[1] = a.warps + (b.warp_idx[1] >= 0 ? b.warp_idx[1] : 0);
  j->luma_ref[0] = ref_plane(a, b.ref_slot[0], 0);
  j->luma_ref[1] = ref_plane(a, b.ref_slot[1], 0);
  j->luma_stride = a.L.p[0].stride;
  j->luma_x = b.x << (p > 0 ? a.L.ss_x : 0);
  j->luma_y = b.y << (p > 0 ? a.L.ss_y : 0);
  j->luma_ref_w = a.L.p[0].out_w;
  j->luma_ref_h = a.L.p[0].out_h;
  j->interintra = b.interintra;
  j->ii_mode = b.ii_mode;
  j->ii_wedge = b.ii_wedge;
  j->have_left = b.have_left;
  j->have_above = b.have_above;
  j->max_x = g.grid_w - 1;
  j->max_y = g.grid_h - 1;
  j->cur = a.cur + g.off + b.y * g.stride + b.x;
  j->cur_stride = g.stride;
  j->obmc = a.obmc + b.obmc_first;
  j->obmc_count = b.obmc_count;
  for (int k = 0; k < 8; ++k)
    j->obmc_ref[k] = k < b.obmc_count ? ref_plane(a, a.obmc[b.obmc_first + k].ref_slot, p) : j->ref[0];
  j->maxv = a.maxv;
}

/* ---- phase A ------------------------------------------------------------------------ */

/* The compound mask of a block the lean kernel predicts, its fields read
 * once into registers (the mask pool's byte stores could alias the block
 * record, so fields read from it would be loaded again after every store). */
struct LeanMask {
  int kind, sign, role, off, mw, dir, xoff, yoff, flip;
  __device__ __forceinline__ explicit LeanMask(const BlockRec& b)
      : kind(b.compound ? b.mask_kind : 0), sign(b.mask_sign), role(b.mask_role), off(b.mask_off),
        mw(b.mask_w), dir(b.wedge_dir), xoff(b.wedge_xoff), yoff(b.wedge_yoff), flip(b.wedge_flip) {}
};

/* The mask (0..64) of sample (x, y): a wedge (a chroma sample averages the
 * luma positions it covers), a luma difference-weighted mask from the two
 * predictions - written to the mask pool when chroma blocks read it - or a
 * chroma difference-weighted mask read from the pool its luma block wrote. */
__device__ __forceinline__ int lean_mask(const FrameArgs& a, const LeanMask& k, int plane, int sub_x,
                                         int sub_y, int bitdepth, int x, int y, int v0, int v1) {
  if (k.kind == 2 && plane == 0) {
    const int sh = 7 - (bitdepth >= 12 ? 5 : 3) + (bitdepth - 8);
    const int m = diffwtd_m(absi(v0 - v1), sh, k.sign);
    if (k.role == 1) a.mask_pool[k.off + y * k.mw + x] = static_cast<unsigned char>(m);
    return m;
  }
  const int nx = sub_x + 1, ny = sub_y + 1;
  int sum = 0;
  for (int jj = 0; jj < ny; ++jj)
    for (int ii = 0; ii < nx; ++ii) {
      const int lx = (x << sub_x) + ii, ly = (y << sub_y) + jj;
      if (k.kind == 1) {
        const int m = wedge_px(k.dir, k.xoff, k.yoff, k.flip, ly, lx);
        sum += k.sign ? 64 - m : m;
      } else {
        sum += a.mask_pool[k.off + ly * k.mw + lx];
      }
    }
  const int n = nx * ny;
  return n == 1 ? sum : (n == 2 ? (sum + 1) >> 1 : (sum + 2) >> 2);
}

/* Inter prediction of the phase A blocks but inter-intra ones and chroma
 * blocks of difference-weighted compounds without a luma mask to read (they
 * take the full kernel): one warp per 16x8 tile, each reference through
 * mc_rect or, for a globally warped one, warp_block8, then the blend, then
 * the OBMC strips in order, each neighbour's prediction of the strip through
 * mc_rect. It carries none of the full kernel's state, so it runs with a
 * fraction of its registers and many more warps in flight. Two builds: the
 * average and distance-weighted blends (MASK false: translation, global
 * warp and OBMC blocks, almost every tile), and the masked blends (MASK
 * true: wedge and difference-weighted compounds) - the mask code in the
 * first build slows its tiles by a fifth. */
template <bool MASK>
__device__ __forceinline__ void inter_simple_tile(const FrameArgs& a, int tile, McScratch& scr,
                                                  int (&pred)[2][8 * 16], int lane) {
  const int2 t = a.inter_tiles[tile];
  const BlockRec& b = a.blocks[t.x];
  const int p = b.plane;
  const PlaneGeom& g = a.L.p[p];
  InterCtx c;
  c.sub_x = p > 0 ? a.L.ss_x : 0;
  c.sub_y = p > 0 ? a.L.ss_y : 0;
  c.ref_w = g.out_w;
  c.ref_h = g.out_h;
  c.bitdepth = a.L.bit_depth;
  c.scale_x = a.scale_x;
  c.scale_y = a.scale_y;
  const int x0 = t.y & 0xffff, y0 = t.y >> 16;
  const int tw = mini(16, b.w - x0), th = mini(8, b.h - y0);
  /* k / tw for the tile's k < 128 as a multiply and a shift (exact there) */
  const int tmul = (65536 + tw - 1) / tw;
  const int nref = b.compound ? 2 : 1;
  for (int r = 0; r < nref; ++r) {
    int* pr = pred[r];
    const px_t* ref = ref_plane(a, b.ref_slot[r], p);
    if (r == 0 ? b.warp0 : b.warp1) {
      /* one or two whole 8x8 warp blocks (x0 is a multiple of 16, y0 of 8) */
      const WarpRec& m = a.warps[b.warp_idx[r] >= 0 ? b.warp_idx[r] : 0];
      for (int bx = 0; bx < tw; bx += 8)
        warp_block8(c.sub_x, c.sub_y, c.ref_w, c.ref_h, m, ref, g.stride, b.x, b.y, x0 + bx, y0,
                    c.bitdepth, b.compound != 0, scr, pr + bx, 16, mini(8, tw - bx), th, lane);
      continue;
    }
    if (!mc_rect(c, ref, g.stride, b.x, b.y, b.w, b.h, b.mv[r][0], b.mv[r][1], b.filt, b.filt_v,
                 b.compound != 0, x0, y0, tw, th, scr, pr, lane)) {
      for (int k = lane; k < tw * th; k += 32) {
        const int yy = k / tw, xx = k - yy * tw;
        pr[yy * 16 + xx] = mc_tap(c, ref, g.stride, b.x, b.y, b.w, b.h, b.mv[r][0], b.mv[r][1],
                                  b.filt, b.filt_v, x0 + xx, y0 + yy, b.compound != 0);
      }
      __syncwarp();
    }
  }
  px_t* dst = a.cur + g.off + (b.y + y0) * g.stride + b.x + x0;
  const int post = 7 - (c.bitdepth >= 12 ? 5 : 3);
  int acc[4];
  if constexpr (MASK) {
    const LeanMask mk(b);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int k = lane + 32 * q;
      if (k >= tw * th) continue;
      const int yy = (k * tmul) >> 16, xx = k - yy * tw;
      const int v0 = pred[0][yy * 16 + xx], v1 = pred[1][yy * 16 + xx];
      const int m = lean_mask(a, mk, p, c.sub_x, c.sub_y, c.bitdepth, x0 + xx, y0 + yy, v0, v1);
      acc[q] = clampi((m * v0 + (64 - m) * v1 + (1 << (5 + post))) >> (6 + post), 0, a.maxv);
    }
  } else {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int k = lane + 32 * q;
      if (k >= tw * th) continue;
      const int yy = (k * tmul) >> 16, xx = k - yy * tw;
      const int v0 = pred[0][yy * 16 + xx];
      int out = v0;
      if (b.compound == 1) {
        out = (v0 + pred[1][yy * 16 + xx] + (1 << post)) >> (1 + post);
      } else if (b.compound) {
        out = (b.w0 * v0 + b.w1 * pred[1][yy * 16 + xx] + (1 << (3 + post))) >> (4 + post);
      }
      acc[q] = clampi(out, 0, a.maxv);
    }
  }
  __syncwarp();
  /* OBMC: the strips in order, each blended onto the samples it covers */
  for (int kk = 0; kk < b.obmc_count; ++kk) {
    const ObmcRec& o = a.obmc[b.obmc_first + kk];
    const int ix0 = maxi(o.x, x0), ix1 = mini(o.x + o.w, x0 + tw);
    const int iy0 = maxi(o.y, y0), iy1 = mini(o.y + o.h, y0 + th);
    if (ix0 >= ix1 || iy0 >= iy1) continue;
    int* tmp = pred[0];
    const px_t* oref = ref_plane(a, o.ref_slot, p);
    const bool ok = mc_rect(c, oref, g.stride, b.x + o.x, b.y + o.y, o.w, o.h, o.mv_x, o.mv_y, o.filt,
                            o.filt_v, 0, ix0 - o.x, iy0 - o.y, ix1 - ix0, iy1 - iy0, scr, tmp,
                            lane);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int k = lane + 32 * q;
      if (k >= tw * th) continue;
      const int yy = (k * tmul) >> 16, xx = k - yy * tw;
      const int x = x0 + xx, y = y0 + yy;
      if (x < ix0 || x >= ix1 || y < iy0 || y >= iy1) continue;
      const int pv = ok ? tmp[(y - iy0) * 16 + x - ix0]
                        : mc_tap(c, oref, g.stride, b.x + o.x, b.y + o.y, o.w, o.h, o.mv_x, o.mv_y,
                                 o.filt, o.filt_v, x - o.x, y - o.y, 0);
      acc[q] = obmc_blend(o, x - o.x, y - o.y, acc[q], pv, a.maxv);
    }
    __syncwarp();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int k = lane + 32 * q;
    if (k < tw * th) {
      const int yy = (k * tmul) >> 16, xx = k - yy * tw;
      dst[yy * g.stride + xx] = (px_t)acc[q];
    }
  }
}

/* Tiles [first, end) of the lean kernel's: the unmasked tiles listed first;
 * the masked build takes the wedge and luma difference-weighted tiles listed
 * next and (a launch of their own, after the luma tiles that write the
 * masks) the chroma tiles that read a luma mask, listed last. */
template <bool MASK>
__global__ void __launch_bounds__(128) k_inter_simple(const __grid_constant__ FrameArgs a, int first,
                                                      int end) {
  __shared__ McScratch scr[4];
  __shared__ int pred[4][2][8 * 16];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int warp = first + blockIdx.x * 4 + wib;
  if (warp >= end) return;
  inter_simple_tile<MASK>(a, warp, scr[wib], pred[wib], lane);
}

/* Inter prediction of phase A blocks: one warp per 16x8 tile. Translation
 * predictions (and OBMC strips) go through mc_rect, warped ones through
 * warp_block8; the composition and the OBMC blends run per sample on
 * registers. A chroma tile whose compound mask is difference-weighted takes
 * its mask from the luma predictions of the area it covers (up to 32x16
 * luma samples), computed the same separable way into shared memory. */
__device__ __forceinline__ void inter_full_tile(const FrameArgs& a, int tile, McScratch& scr,
                                                int (&pred)[2][8 * 16],
                                                int (&lpred)[2][4 * 8 * 16], int lane) {
  const int2 t = a.inter_tiles[tile];
  const BlockRec& b = a.blocks[t.x];
  InterJob j;
  make_inter_job(a, b, &j);
  const int x0 = t.y & 0xffff, y0 = t.y >> 16;
  const int tw = mini(16, b.w - x0), th = mini(8, b.h - y0);
  /* k / tw for the tile's k < 128 as a multiply and a shift (exact there) */
  const int tmul = (65536 + tw - 1) / tw;
  const PlaneGeom& g = a.L.p[b.plane];
  px_t* dst = a.cur + g.off + (b.y + y0) * g.stride + b.x + x0;
  if (j.interintra) {
    /* inter-intra reads this frame: scheduled with the dependency phase */
    for (int k = lane; k < tw * th; k += 32) {
      const int yy = k / tw, xx = k - yy * tw;
      int v = inter_core(j, x0 + xx, y0 + yy);
      v = inter_finish(j, x0 + xx, y0 + yy, v, 0);
      dst[yy * g.stride + xx] = (px_t)v;
    }
    return;
  }
  const int nref = j.compound ? 2 : 1;
  for (int r = 0; r < nref; ++r) {
    int* pr = pred[r];
    if (j.warp[r]) {
      /* the tile is one or two whole 8x8 warp blocks (x0 is a multiple of
       * 16, y0 of 8) */
      for (int bx = 0; bx < tw; bx += 8)
        warp_block8(j.ctx.sub_x, j.ctx.sub_y, j.ctx.ref_w, j.ctx.ref_h, *j.model[r], j.ref[r],
                    j.ref_stride, j.x, j.y, x0 + bx, y0, j.ctx.bitdepth, j.compound != 0, scr,
                    pr + bx, 16, mini(8, tw - bx), th, lane);
      continue;
    }
    const bool ok = mc_rect(j.ctx, j.ref[r], j.ref_stride, j.x, j.y, j.w, j.h, j.mv[r][0],
                            j.mv[r][1], j.filt, j.filt_v, j.compound != 0, x0, y0, tw, th, scr,
                            pr, lane);
    if (!ok) {
      for (int k = lane; k < tw * th; k += 32) {
        const int yy = k / tw, xx = k - yy * tw;
        pr[yy * 16 + xx] = inter_ref(j, r, x0 + xx, y0 + yy);
      }
      __syncwarp();
    }
  }
  const bool luma_mask = j.compound && j.mask_kind == 2 && b.plane > 0;
  /* the luma block is the same prediction and has written its mask */
  const bool shared_mask = luma_mask && b.mask_role == 2;
  if (luma_mask && !shared_mask) {
    InterCtx l;
    l.sub_x = l.sub_y = 0;
    l.ref_w = j.luma_ref_w;
    l.ref_h = j.luma_ref_h;
    l.bitdepth = j.ctx.bitdepth;
    l.scale_x = j.ctx.scale_x;
    l.scale_y = j.ctx.scale_y;
    const int lx0 = x0 << j.ctx.sub_x, ly0 = y0 << j.ctx.sub_y;
    const int lw = tw << j.ctx.sub_x, lh = th << j.ctx.sub_y;
    const int ew = j.w << j.ctx.sub_x, eh = j.h << j.ctx.sub_y;
    for (int r = 0; r < 2; ++r)
      for (int qy = 0; qy < lh; qy += 8)
        for (int qx = 0; qx < lw; qx += 16) {
          int* out = lpred[r] + ((qy >> 3) * 2 + (qx >> 4)) * 128;
          const int rw = mini(16, lw - qx), rh = mini(8, lh - qy);
          if (j.mask_warp[r]) {
            for (int bx = 0; bx < rw; bx += 8)
              warp_block8(0, 0, j.luma_ref_w, j.luma_ref_h, *j.model[r], j.luma_ref[r],
                          j.luma_stride, j.luma_x, j.luma_y, lx0 + qx + bx, ly0 + qy,
                          j.ctx.bitdepth, 1, scr, out + bx, 16, mini(8, rw - bx), rh, lane);
          } else if (!mc_rect(l, j.luma_ref[r], j.luma_stride, j.luma_x, j.luma_y, ew, eh,
                              j.mv[r][0], j.mv[r][1], j.filt, j.filt_v, 1, lx0 + qx, ly0 + qy, rw,
                              rh, scr, out, lane)) {
            for (int k = lane; k < rw * rh; k += 32) {
              const int yy = k / rw, xx = k - yy * rw;
              out[yy * 16 + xx] = mc_tap(l, j.luma_ref[r], j.luma_stride, j.luma_x, j.luma_y, ew,
                                         eh, j.mv[r][0], j.mv[r][1], j.filt, j.filt_v,
                                         lx0 + qx + xx, ly0 + qy + yy, 1);
            }
            __syncwarp();
          }
        }
  }
  int acc[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int k = lane + 32 * q;
    if (k < tw * th) {
      const int yy = (k * tmul) >> 16, xx = k - yy * tw;
      const int v0 = pred[0][yy * 16 + xx], v1 = nref > 1 ? pred[1][yy * 16 + xx] : 0;
      if (luma_mask) {
        /* the chroma sample's mask: the mean over the luma samples it covers,
         * from the luma block's mask or from the luma predictions */
        const int sh = 7 - (j.ctx.bitdepth >= 12 ? 5 : 3) + (j.ctx.bitdepth - 8);
        const int nx = j.ctx.sub_x + 1, ny = j.ctx.sub_y + 1;
        int sum = 0;
        for (int jj = 0; jj < ny; ++jj)
          for (int ii = 0; ii < nx; ++ii) {
            const int lx = (xx << j.ctx.sub_x) + ii, ly = (yy << j.ctx.sub_y) + jj;
            if (shared_mask) {
              const int bx = (x0 << j.ctx.sub_x) + lx, by = (y0 << j.ctx.sub_y) + ly;
              sum += a.mask_pool[b.mask_off + by * b.mask_w + bx];
            } else {
              const int idx = ((ly >> 3) * 2 + (lx >> 4)) * 128 + (ly & 7) * 16 + (lx & 15);
              sum += diffwtd_m(absi(lpred[0][idx] - lpred[1][idx]), sh, j.mask_sign);
            }
          }
        const int n = nx * ny;
        const int m = n == 1 ? sum : (n == 2 ? (sum + 1) >> 1 : (sum + 2) >> 2);
        acc[q] = blend_mask(j, v0, v1, m);
      } else {
        acc[q] = inter_compose(j, x0 + xx, y0 + yy, v0, v1);
        if (b.mask_role == 1) {
          /* the mask its chroma blocks read (the one inter_compose blends with) */
          const int sh = 7 - (j.ctx.bitdepth >= 12 ? 5 : 3) + (j.ctx.bitdepth - 8);
          a.mask_pool[b.mask_off + (y0 + yy) * b.mask_w + x0 + xx] =
              static_cast<unsigned char>(diffwtd_m(absi(v0 - v1), sh, j.mask_sign));
        }
      }
    }
  }
  __syncwarp();
  for (int kk = 0; kk < j.obmc_count; ++kk) {
    const ObmcRec& c = j.obmc[kk];
    const int ix0 = maxi(c.x, x0), ix1 = mini(c.x + c.w, x0 + tw);
    const int iy0 = maxi(c.y, y0), iy1 = mini(c.y + c.h, y0 + th);
    if (ix0 >= ix1 || iy0 >= iy1) continue;
    int* tmp = pred[0];
    const bool ok = mc_rect(j.ctx, j.obmc_ref[kk], j.ref_stride, j.x + c.x, j.y + c.y, c.w, c.h,
                            c.mv_x, c.mv_y, c.filt, c.filt_v, 0, ix0 - c.x, iy0 - c.y, ix1 - ix0,
                            iy1 - iy0, scr, tmp, lane);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int k = lane + 32 * q;
      if (k >= tw * th) continue;
      const int yy = (k * tmul) >> 16, xx = k - yy * tw;
      const int x = x0 + xx, y = y0 + yy;
      if (x < ix0 || x >= ix1 || y < iy0 || y >= iy1) continue;
      const int pv = ok ? tmp[(y - iy0) * 16 + x - ix0]
                        : mc_tap(j.ctx, j.obmc_ref[kk], j.ref_stride, j.x + c.x, j.y + c.y, c.w,
                                 c.h, c.mv_x, c.mv_y, c.filt, c.filt_v, x - c.x, y - c.y, 0);
      acc[q] = obmc_blend(c, x - c.x, y - c.y, acc[q], pv, j.maxv);
    }
    __syncwarp();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int k = lane + 32 * q;
    if (k < tw * th) {
      const int yy = (k * tmul) >> 16, xx = k - yy * tw;
      dst[yy * g.stride + xx] = (px_t)acc[q];
    }
  }
}

/* Tiles [first, end) of the full kernel's (between the lean kernel's two
 * ranges). */
__global__ void __launch_bounds__(128, 4) k_inter(const __grid_constant__ FrameArgs a, int first, int end) {
  __shared__ McScratch scr[4];
  __shared__ int pred[4][2][8 * 16];
  __shared__ int lpred[4][2][4 * 8 * 16];   /* luma predictions, four 16x8 quarters */
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int warp = first + blockIdx.x * 4 + wib;
  if (warp >= end) return;
  inter_full_tile(a, warp, scr[wib], pred[wib], lpred[wib], lane);
}

/* Adds one transform's residual (or a raw residual block) to the picture. */
template <bool CG>
__device__ void apply_tx(const FrameArgs& a, const BlockRec& b, const TxRec& tx, int* tmp,
                         int lane) {
  const PlaneGeom& g = a.L.p[b.plane];
  px_t* dst = a.cur + g.off + (b.y + tx.y) * g.stride + b.x + tx.x;
  if (b.residual_provided || tx.pre_off >= 0) {
    const int* res = b.residual_provided ? a.residual + tx.coef_off : a.pre_res + tx.pre_off;
    for (int k = lane; k < tx.w * tx.h; k += 32) {
      const int yy = k / tx.w, xx = k - yy * tx.w;
      px_t* q = dst + yy * g.stride + xx;
      const int old = CG ? (int)__ldcg(q) : (int)*q;
      *q = (px_t)clampi(old + res[yy * tx.w + xx], 0, a.maxv);
    }
    __syncwarp();
    return;
  }
  ItxParams p;
  p.lw = tx.log2w;
  p.lh = tx.log2h;
  p.type = tx.type;
  p.lossless = b.lossless;
  p.row_shift = tx.row_shift;
  p.bitdepth = a.L.bit_depth;
  itx_warp<CG>(p, a.coef + tx.coef_off, tmp, dst, g.stride, a.maxv, lane);
}

/* Dequantisation on the device: a frame's coded levels, in scan order, into
 * the raster the inverse transforms read (the reference front end's
 * dequantise_tile fill, dequant.hpp:317-345, with dequantise_level,
 * dequant.hpp:94-106). One warp per coded transform: the raster is cleared
 * with vector stores, then the lanes place the levels through the scan. It
 * runs on the planner's upload stream right after the levels arrive, so it
 * overlaps the frames still decoding; the rasters it writes are what the
 * ITX kernels read next, mostly out of L2. */
__global__ void __launch_bounds__(256) k_dequant(const DqRec* __restrict__ jobs, int n,
                                                 const short* __restrict__ levels,
                                                 const unsigned char* __restrict__ qm,
                                                 int* __restrict__ coef, int bit_depth) {
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= n) return;
  const DqRec r = jobs[j];
  const int area = 1 << (r.alw + r.alh);
  int* raster = coef + r.coef_off;
  if ((r.coef_off & 3) == 0) {
    int4* v = reinterpret_cast<int4*>(raster);
    for (int k = lane; k < (area >> 2); k += 32) v[k] = make_int4(0, 0, 0, 0);
  } else {
    for (int k = lane; k < area; k += 32) raster[k] = 0;
  }
  __syncwarp();
  const short* lv = levels + r.level_off;
  const unsigned short* scan = kScans + r.scan_off;
  const unsigned char* m = r.qm_off >= 0 ? qm + r.qm_off : nullptr;
  const int hi = (1 << (7 + bit_depth)) - 1, lo = -(1 << (7 + bit_depth));
  for (int i = lane; i < r.count; i += 32) {
    const int level = lv[i];
    const int pos = scan[i];
    if (level == 0 || pos >= area) continue;
    int step = pos == 0 ? r.dc_step : r.ac_step;
    if (m) step = (step * m[pos] + 16) >> 5;
    const long long prod = static_cast<long long>(level) * step;
    const unsigned mag = static_cast<unsigned>((prod < 0 ? -prod : prod) & 0xFFFFFF);
    const int scaled = static_cast<int>(mag / r.denom);
    raster[pos] = clampi(prod < 0 ? -scaled : scaled, lo, hi);
  }
}

cudaError_t launch_dequant(const DqRec* jobs, int n, const short* levels, const unsigned char* qm,
                           int* coef, int bit_depth, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_dequant<<<(n + 7) / 8, 256, 0, s>>>(jobs, n, levels, qm, coef, bit_depth);
  return cudaGetLastError();
}

/* Inverse transforms, in batches of one size class: a warp runs 32 / S
 * transforms whose longer side is S (S = 4, 8, 16, 32; one of 64), one lane
 * group of S lanes each, so a 4x4 transform no longer leaves 28 lanes idle.
 * One launch per class (CLS = log2 S), each instantiating only its class's
 * transform lengths: the small classes, most of the transforms, run with a
 * fraction of the registers of the 64-point ones and so with many more warps
 * in flight. The planner sorts the transforms by class, shape and type, so
 * the groups of a warp mostly take the same path. Those of phase A blocks add
 * into the picture; those of phase B blocks leave their residual in the
 * precomputed buffer, so the dependency-scheduled kernel only predicts and
 * adds (the residual does not depend on the prediction). Raw residual blocks
 * (class 7) add with the whole warp. */
/* Scratch ints a warp of class CLS needs. */
template <int CLS>
struct ItxScratch {
  static constexpr int S = 1 << (CLS < 7 ? CLS : 5);
  static constexpr int PER_WARP = CLS >= 6 ? 4096 : 32 * S;
};

/* One batch of class CLS (`bt`: first job, jobs, class) with the warp's
 * scratch `wsm`. */
template <int CLS>
__device__ __forceinline__ void itx_batch(const FrameArgs& a, const int4 bt, int* wsm, int lane) {
  constexpr int S = ItxScratch<CLS>::S, STEP = S < 32 ? S : 32;
  if constexpr (CLS == 7) {
    const int2 t = a.itx_jobs[bt.x];
    apply_tx<false>(a, a.blocks[t.x], a.txs[t.y], wsm, lane);
  } else {
    const int g = lane / STEP, sub = lane - g * STEP;
    const bool active = g < bt.y;
    const int2 t = a.itx_jobs[bt.x + (active ? g : 0)];
    const BlockRec& b = a.blocks[t.x];
    const TxRec& tx = a.txs[t.y];
    ItxParams p;
    p.lw = tx.log2w;
    p.lh = tx.log2h;
    p.type = tx.type;
    p.lossless = b.lossless;
    p.row_shift = tx.row_shift;
    p.bitdepth = a.L.bit_depth;
    int* tmp = wsm + (S <= 32 ? g * S * S : 0);
    const PlaneGeom& gm = a.L.p[b.plane];
    px_t* dst = a.cur + gm.off + (b.y + tx.y) * gm.stride + b.x + tx.x;
    int* res = tx.pre_off >= 0 ? a.pre_res + tx.pre_off : nullptr;
    itx_group_cls<CLS, false>(p, a.coef + tx.coef_off, tmp, dst, gm.stride, a.maxv, res, sub, STEP,
                              active);
  }
}

template <int CLS>
__global__ void __launch_bounds__(128) k_itx(const __grid_constant__ FrameArgs a, int first,
                                             int count) {
  extern __shared__ int smem[];
  const int wib = threadIdx.x >> 5;
  const int bi = blockIdx.x * (blockDim.x >> 5) + wib;
  const int lane = threadIdx.x & 31;
  if (bi >= count) return;
  itx_batch<CLS>(a, a.itx_batches[first + bi], smem + wib * ItxScratch<CLS>::PER_WARP, lane);
}

template <int CLS>
static cudaError_t launch_itx_class(const FrameArgs& a, cudaStream_t s) {
  const int first = a.itx_class_first[CLS], count = a.itx_class_count[CLS];
  if (count <= 0) return cudaSuccess;
  constexpr int per_warp = CLS == 7 || CLS >= 6 ? 4096 : 32 * (1 << CLS);
  k_itx<CLS><<<(count + 3) / 4, 128, 4 * per_warp * sizeof(int), s>>>(a, first, count);
  return cudaGetLastError();
}

/* ---- phase B -------------------------------------------------------------------------- */

/* How a dependency wait polls: with AV1B_POLL_ACQUIRE every poll is an
 * acquire load (the load that sees the flag orders what follows, no separate
 * fence); without, relaxed polls and one acquire fence once the flag is seen.
 * Between polls the warp sleeps, backing off to AV1B_POLL_PAUSE_MAX ns (0: no
 * sleep). Acquire polls take about 6 % off the dependency-scheduled phase
 * (the fence after a relaxed poll is a round trip of its own on the path).
 * Shorter pauses gain nothing on one stream, and with many streams' chains
 * waiting at once (a batched key frame-set) 64 ns pauses saw occasional
 * steps of twice the usual time, 256 ns none. */
#ifndef AV1B_POLL_ACQUIRE
#define AV1B_POLL_ACQUIRE 1
#endif
#ifndef AV1B_POLL_PAUSE_MAX
#define AV1B_POLL_PAUSE_MAX 256
#endif

__device__ __forceinline__ bool flag_seen(const unsigned* flag, unsigned want) {
#if AV1B_POLL_ACQUIRE
  return ld_acquire(flag) == want;
#else
  if (ld_relaxed(flag) != want) return false;
  fence_acq_rel();
  return true;
#endif
}

/* Waits until *flag == want, for at most limit_ns of globaltimer. Once any
 * wait has given up (AV1B_STATUS_TIMEOUT in *status), nothing waits any more:
 * the frame has failed and the kernel only has to run to its end. The status
 * word and the clock are read every 16th poll. */
__device__ bool bounded_wait(const unsigned* flag, unsigned want, int* status,
                             unsigned long long limit_ns) {
  if (flag_seen(flag, want)) return true;
  const unsigned long long t0 = global_ns();
  unsigned pause = AV1B_POLL_PAUSE_MAX < 32 ? AV1B_POLL_PAUSE_MAX : 32;
  for (unsigned it = 1;; ++it) {
    if (flag_seen(flag, want)) return true;
    if ((it & 15) == 0) {
      if (ld_relaxed(reinterpret_cast<const unsigned*>(status)) & AV1B_STATUS_TIMEOUT) return false;
      if (global_ns() - t0 > limit_ns) {
        atomicOr(status, AV1B_STATUS_TIMEOUT);
        return false;
      }
    }
    if (AV1B_POLL_PAUSE_MAX > 0) __nanosleep(pause);
    if (pause < AV1B_POLL_PAUSE_MAX) pause <<= 1;
  }
}

/* Waits until block `o` is reconstructed. Returns false on timeout. */
__device__ bool wait_block(const FrameArgs& a, int o) {
  return bounded_wait(a.done + (size_t)o * AV1B_FLAG_STRIDE, a.epoch, a.status, a.wait_ns);
}

/* A wait on a flag nothing sets: the failure-detection self test. */
__global__ void k_selftest_wait(const unsigned* flag, int* status, unsigned long long limit_ns) {
  if (threadIdx.x == 0) bounded_wait(flag, 1u, status, limit_ns);
}

cudaError_t launch_selftest_wait(const unsigned* flag, int* status, unsigned long long limit_ns,
                                 cudaStream_t s) {
  k_selftest_wait<<<1, 32, 0, s>>>(flag, status, limit_ns);
  return cudaGetLastError();
}

/* The persistent dependency-scheduled kernel: each warp claims chains of
 * blocks in the planner's order (chains start in order of dependency depth)
 * and runs a chain's blocks one after another: for each it waits for the
 * blocks its list names - except the one before it in the chain, its own
 * work - and reconstructs. Everything that does not depend on other blocks - the
 * block record, its dependency list, its residual - is loaded before the
 * wait. Shared memory per warp: three edge buffers and a 64x64 scratch (the
 * block's residual image, or the transform scratch). */
/* Adds a phase B transform's residual - precomputed by k_itx, or the raw
 * residual of a residual-provided block - to the reconstructed prediction
 * (read back through L2). No transform code here: the kernel stays small. */
__device__ void add_residual_cg(const FrameArgs& a, const BlockRec& b, const TxRec& tx, int lane) {
  const PlaneGeom& g = a.L.p[b.plane];
  px_t* dst = a.cur + g.off + (b.y + tx.y) * g.stride + b.x + tx.x;
  const int* res = b.residual_provided ? a.residual + tx.coef_off : a.pre_res + tx.pre_off;
  /* four samples a lane at a time, every load before any store: the loads
   * read the picture the stores write, so the compiler cannot overlap one
   * sample's load with another's store by itself */
  const int n = tx.w * tx.h;
  for (int k0 = lane; k0 < n; k0 += 4 * 32) {
    int v[4];
    int o[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int k = k0 + 32 * q;
      if (k < n) {
        const int yy = k / tx.w, xx = k - yy * tx.w;
        o[q] = yy * g.stride + xx;
        v[q] = (int)__ldcg(dst + o[q]) + res[k];
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (k0 + 32 * q < n) dst[o[q]] = (px_t)clampi(v[q], 0, a.maxv);
  }
  __syncwarp();
}

/* INTER: the frame has phase B inter blocks (inter-intra, intra block copy);
 * a frame of intra blocks only (every key frame) runs the instantiation
 * without the inter prediction code, a much smaller kernel. */
/* Runs chain `c` of the frame: its blocks one after another, each after the
 * blocks it waits for. `edges` and `tmp` are the warp's shared memory. */
template <bool INTER>
__device__ __forceinline__ void run_chain(const FrameArgs& a, int c, int* edges, int* tmp,
                                          int lane) {
  {
    const int u_end = a.chains[c + 1];
    int prev = -1;
    /* the next block's record is loaded while this one runs: in a chain the
     * next block usually starts as soon as this one is published (not in
     * the kernel with inter prediction, whose registers it would spill) */
    int bi_next = a.units[a.chains[c]];
    BlockRec b_next = a.blocks[bi_next];
    for (int u = a.chains[c]; u < u_end; ++u) {
      const int bi = bi_next;
      const BlockRec b = INTER ? a.blocks[bi] : b_next;
      if (u + 1 < u_end) {
        bi_next = a.units[u + 1];
        if (!INTER) b_next = a.blocks[bi_next];
      }
      const int p = b.plane;
      const PlaneGeom& g = a.L.p[p];
      const bool fused = b.kind == AV1B_U_INTRA && b.fuse_res;

      /* the residual image, copied asynchronously: it arrives while the
       * block waits and reads its edges (intra_predict waits for it) */
      if (fused) {
        const int n = b.w * b.h;
        for (int k = lane; k < n; k += 32) tmp[k] = 0;
        __syncwarp();
        for (int t = 0; t < b.tx_count; ++t) {
          const TxRec tx = a.txs[b.tx_first + t];
          const int* src = b.residual_provided ? a.residual + tx.coef_off : a.pre_res + tx.pre_off;
          for (int k = lane; k < tx.w * tx.h; k += 32) {
            const int yy = k / tx.w, xx = k - yy * tx.w;
            const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(tmp + (tx.y + yy) * b.w + tx.x + xx));
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src + k) : "memory");
          }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
      }

      /* the blocks this one reads from: each lane's acquire load of a done flag
       * orders the samples that block published before that lane's later
       * reads, and the warp barrier extends the order to every lane (all
       * picture reads go through L2, never a stale L1 line) */
      unsigned long long t_claim = 0;
      if (a.trace) t_claim = global_ns();
      /* the block before this one in the chain is this warp's own work, already
       * ordered by the warp barrier that ended it */
      for (int k = lane; k < b.dep_count; k += 32) {
        const int o = a.deps[b.dep_first + k];
        if (o != prev) wait_block(a, o);
      }
      __syncwarp();
      if (a.trace) {
        /* the dependency published last (its record was written before its
         * flag, so the acquire above made it visible) */
        unsigned long long last = 0, who = ~0ull;
        for (int k = lane; k < b.dep_count; k += 32) {
          const int o = a.deps[b.dep_first + k];
          const unsigned long long t = __ldcg(a.trace + 4 * (size_t)o + 2);
          if (t >= last) {
            last = t;
            who = static_cast<unsigned long long>(o);
          }
        }
        for (int s = 16; s > 0; s >>= 1) {
          const unsigned long long lo = __shfl_down_sync(0xffffffffu, last, s);
          const unsigned long long wo = __shfl_down_sync(0xffffffffu, who, s);
          if (lo > last) {
            last = lo;
            who = wo;
          }
        }
        if (lane == 0) {
          a.trace[4 * (size_t)bi + 0] = t_claim;
          a.trace[4 * (size_t)bi + 1] = global_ns();
          a.trace[4 * (size_t)bi + 3] = who;
        }
      }

      px_t* dst = a.cur + g.off + b.y * g.stride + b.x;
      if (b.kind == AV1B_U_INTRA) {
        IntraJob j;
        j.x = b.x;
        j.y = b.y;
        j.w = b.w;
        j.h = b.h;
        j.mode = b.mode;
        j.angle = b.angle_delta;
        j.bitdepth = a.L.bit_depth;
        j.maxv = a.maxv;
        j.have_left = b.have_left;
        j.have_above = b.have_above;
        j.have_ar = b.have_ar;
        j.have_bl = b.have_bl;
        j.filter_type = b.filter_type;
        j.filter_intra = b.fi_mode >= 0;
        j.fi_mode = b.fi_mode >= 0 ? b.fi_mode : 0;
        j.cfl_alpha = b.cfl_alpha;
        j.max_x = g.grid_w - 1;
        j.max_y = g.grid_h - 1;
        j.ss_x = a.L.ss_x;
        j.ss_y = a.L.ss_y;
        j.palette = b.palette;
        j.palette_off = b.palette_off;
        j.palette_stride = b.palette_stride;
        /* filter intra (at most 32x32) keeps its predictions after the
         * residual image: tmp[1024 ..] */
        intra_predict(j, dst, g.stride, a.cur + a.L.p[0].off, a.L.p[0].stride, a.palette_map,
                      a.palette_colors + 8 * b.palette_color_idx, edges, lane,
                      fused ? tmp : nullptr, tmp + 1024, fused);
      } else if constexpr (INTER) {
        InterJob j;
        make_inter_job(a, b, &j);
        int dc = 0;
        if (b.interintra && b.ii_mode == 0) dc = ii_dc(j);
        for (int k = lane; k < b.w * b.h; k += 32) {
          const int yy = k / b.w, xx = k - yy * b.w;
          int v = b.kind == AV1B_U_INTRABC ? inter_core<true>(j, xx, yy) : inter_core(j, xx, yy);
          v = inter_finish(j, xx, yy, v, dc);
          dst[yy * g.stride + xx] = (px_t)v;
        }
      }
      __syncwarp();
      if (!fused)
        for (int t = 0; t < b.tx_count; ++t) add_residual_cg(a, b, a.txs[b.tx_first + t], lane);

      /* publish: the barrier orders every lane's stores before lane 0's
       * release, whose fence (cumulative) makes them visible at GPU scope to
       * any warp that acquires the flag */
      __syncwarp();
      if (a.trace && lane == 0) a.trace[4 * (size_t)bi + 2] = global_ns();
      if (lane == 0) st_release(a.done + (size_t)bi * AV1B_FLAG_STRIDE, a.epoch);
      prev = bi;
    }
  }
}

template <bool INTER>
__global__ void __launch_bounds__(128, AV1B_UNIT_CTAS_PER_SM) k_units(const __grid_constant__ FrameArgs a) {
  extern __shared__ int smem[];
  const int wib = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  int* edges = smem + wib * (3 * AV1B_EDGE_LEN + AV1B_UNIT_SCRATCH);
  int* tmp = edges + 3 * AV1B_EDGE_LEN;
  for (;;) {
    int c = 0;
    if (lane == 0) c = atomicAdd(a.queue, 1);
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= a.n_chains) break;
    run_chain<INTER>(a, c, edges, tmp, lane);
  }
}

/* ---- deblocking ---------------------------------------------------------------------- */
/* Deblocks records recs[0 .. m), m <= AV1B_DB_GROUP, with the warp's lanes
 * spread over their samples: most edges are 4 or 8 samples long, so a warp
 * per edge would leave three lanes of four idle. Lane j < m holds record j;
 * an inclusive scan of the lengths maps each sample to its record, whose
 * fields the sample's lane takes by shuffle, and the warp steps 32 samples at
 * a time. The edges of one pass never filter the same sample (a filter is
 * never longer than the transforms on its sides), so their samples run in
 * any order. */
template <int G = AV1B_DB_GROUP>
__device__ __forceinline__ void deblock_group(px_t* pic, const DeblockRec* recs, int m, int sharpness,
                                              int bd, int maxv, int lane) {
  DeblockRec r{};
  int len = 0;
  if (lane < m) {
    r = recs[lane];
    len = r.len;
  }
  int cum = len;
#pragma unroll
  for (int o = 1; o < G; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, cum, o);
    if (lane >= o) cum += v;
  }
  const int total = __shfl_sync(0xffffffffu, cum, G - 1);
  const int fc = r.filter_size | (r.chroma << 8);
  for (int base = 0; base < total; base += 32) {
    const int t = base + lane;
    int j = 0;
#pragma unroll
    for (int q = 0; q < G - 1; ++q) j += __shfl_sync(0xffffffffu, cum, q) <= t;
    const int start = __shfl_sync(0xffffffffu, cum - len, j);
    const int p_off = __shfl_sync(0xffffffffu, r.p_off, j);
    const int across = __shfl_sync(0xffffffffu, r.across, j);
    const int along = __shfl_sync(0xffffffffu, r.along, j);
    const int level = __shfl_sync(0xffffffffu, static_cast<int>(r.level), j);
    const int fcj = __shfl_sync(0xffffffffu, fc, j);
    if (t < total)
      deblock_px(pic + p_off + (t - start) * along, across, level, sharpness, fcj & 255, fcj >> 8, bd,
                 maxv);
  }
}

/* A warp per G records. */
template <int G>
__global__ void k_deblock(px_t* pic, const DeblockRec* recs, int n, int sharpness, int bd,
                          int maxv) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const long long r0 = static_cast<long long>(warp) * G;
  if (r0 >= n) return;
  deblock_group<G>(pic, recs + r0, mini(G, n - static_cast<int>(r0)), sharpness, bd, maxv, lane);
}

/* ---- CDEF ------------------------------------------------------------------------------ */
/* CDEF direction search (av1gpu_kernels.h:2601-2660), one thread per 8x8 luma
 * block: the 90 partial sums of the eight directions stay in registers (the
 * loops unroll, so every bin index is a constant). The result packs
 * (variance << 3) | direction. Threads [0, n_grid) search the cells of the
 * 8x8 grid (result index = cell), the rest the listed positions off the grid
 * (result index grid_n + k). Chroma blocks read the search of their luma
 * block, so each luma block is searched once. */
__device__ __forceinline__ void cdef_search_one(const px_t* __restrict__ src, int grid_w, int grid_n,
                                                int n_grid, const unsigned* __restrict__ pos,
                                                int* out, const Layout& L, int t) {
  int x, y, o;
  if (t < n_grid) {
    y = (t / grid_w) << 3;
    x = (t - (t / grid_w) * grid_w) << 3;
    o = t;
  } else {
    const unsigned q = pos[t - n_grid];
    x = q & 0xffff;
    y = q >> 16;
    o = grid_n + (t - n_grid);
  }
  const int stride = L.p[0].stride, cs = L.bit_depth - 8;
  const px_t* b = src + L.p[0].off + y * stride + x;
  int p0[15] = {}, p1[11] = {}, p2[8] = {}, p3[11] = {}, p4[15] = {}, p5[11] = {}, p6[8] = {},
      p7[11] = {};
  const bool vec = ((L.p[0].off + y * stride + x) & 7) == 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    int v[8];
    if (vec) {
      const uint4 w = __ldg(reinterpret_cast<const uint4*>(b + i * stride));
      const unsigned u[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        v[2 * k] = u[k] & 0xffff;
        v[2 * k + 1] = u[k] >> 16;
      }
    } else {
#pragma unroll
      for (int j = 0; j < 8; ++j) v[j] = b[i * stride + j];
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int s = (v[j] >> cs) - 128;
      p0[i + j] += s;
      p1[i + j / 2] += s;
      p2[i] += s;
      p3[3 + i - j / 2] += s;
      p4[7 + i - j] += s;
      p5[3 - i / 2 + j] += s;
      p6[j] += s;
      p7[i / 2 + j] += s;
    }
  }
  const int div[9] = {0, 840, 420, 280, 210, 168, 140, 120, 105};
  int cost[8];
  cost[2] = cost[6] = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    cost[2] += p2[i] * p2[i];
    cost[6] += p6[i] * p6[i];
  }
  cost[2] *= div[8];
  cost[6] *= div[8];
  cost[0] = p0[7] * p0[7] * div[8];
  cost[4] = p4[7] * p4[7] * div[8];
#pragma unroll
  for (int i = 0; i < 7; ++i) {
    cost[0] += (p0[i] * p0[i] + p0[14 - i] * p0[14 - i]) * div[i + 1];
    cost[4] += (p4[i] * p4[i] + p4[14 - i] * p4[14 - i]) * div[i + 1];
  }
  int* odd[4] = {p1, p3, p5, p7};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int* pt = odd[k];
    int c = 0;
#pragma unroll
    for (int j = 0; j < 5; ++j) c += pt[3 + j] * pt[3 + j];
    c *= div[8];
#pragma unroll
    for (int j = 0; j < 3; ++j) c += (pt[j] * pt[j] + pt[10 - j] * pt[10 - j]) * div[2 * j + 2];
    cost[2 * k + 1] = c;
  }
  int best = 0, d = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i)
    if (cost[i] > best) {
      best = cost[i];
      d = i;
    }
  int opp = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i)
    if (i == ((d + 4) & 7)) opp = cost[i];
  out[o] = (((best - opp) >> 10) << 3) | d;
}

__global__ void __launch_bounds__(128) k_cdef_search(const px_t* __restrict__ src, int grid_w,
                                                     int grid_n, int n_grid,
                                                     const unsigned* __restrict__ pos, int n_extra,
                                                     int* out, const __grid_constant__ Layout L) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_grid + n_extra) return;
  cdef_search_one(src, grid_w, grid_n, n_grid, pos, out, L, t);
}

__constant__ signed char kCdefDirs[8][2][2] = {
    {{-1, 1}, {-2, 2}}, {{0, 1}, {-1, 2}}, {{0, 1}, {0, 2}}, {{0, 1}, {1, 2}},
    {{1, 1}, {2, 2}},   {{1, 0}, {2, 1}},  {{1, 0}, {2, 0}}, {{1, 0}, {2, -1}},
};
__constant__ unsigned char kCdefUvDir[2][2][8] = {{{0, 1, 2, 3, 4, 5, 6, 7}, {1, 2, 2, 2, 3, 4, 6, 0}},
                                                  {{7, 0, 2, 4, 5, 6, 6, 6}, {0, 1, 2, 3, 4, 5, 6, 7}}};

/* CDEF filter (av1gpu_kernels.h:2662-2775), one half-warp per block: the
 * block and its 2-sample halo staged in shared memory, then 4 samples a lane
 * (luma 8x8) or 1 (4:2:0 chroma 4x4), so chroma blocks leave no lane idle.
 * Everything per block is resolved once before the sample loop: the tap
 * offsets of the three directions, each strength's damping shift (the
 * constrain function's floor_log2), and whether every tap of the block lies
 * inside the plane (then no per-tap bound checks). */
__device__ __forceinline__ int cdef_cst(int diff, int th, int sh) {
  const int m = absi(diff);
  const int v = clampi(th - (m >> sh), 0, m);
  return diff < 0 ? -v : v;
}

/* The same with the hardware's three-input and add-min-relu integer
 * instructions (max(min(th - s, m), 0) is the clamp of th - s to [0, m] for
 * m >= 0). */
__device__ __forceinline__ int cdef_cst3(int diff, int th, int sh) {
  const int m = absi(diff);
  const int v = __viaddmin_s32_relu(th, -(m >> sh), m);
  return diff < 0 ? -v : v;
}

template <bool EDGE>
__device__ __forceinline__ void cdef_samples(const int* win, px_t* d, int stride, int w, int h,
                                             int hl, int x0, int y0, int pw, int ph,
                                             const int (&oy)[6], const int (&ox)[6], int pri,
                                             int psh, int sec, int ssh, int pt0, int pt1,
                                             int maxv) {
  for (int k = hl; k < w * h; k += 16) {
    const int i = k >> (w == 8 ? 3 : (w == 4 ? 2 : 1)), j = k & (w - 1);
    if (EDGE && (y0 + i >= ph || x0 + j >= pw)) continue;
    const int x = win[(i + 2) * 12 + j + 2];
    int sum = 0, lo = x, hi = x;
    if (!EDGE) {
      /* every tap lies in the plane: both taps of a direction at once */
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        const int tap = q == 0 ? pt0 : (q == 1 ? pt1 : (q & 1 ? 1 : 2));
        const int th = q < 2 ? pri : sec, sh = q < 2 ? psh : ssh;
        const int o = oy[q] * 12 + ox[q];
        const int va = win[(i + 2) * 12 + j + 2 - o], vb = win[(i + 2) * 12 + j + 2 + o];
        if (th) sum += tap * (cdef_cst3(va - x, th, sh) + cdef_cst3(vb - x, th, sh));
        lo = __vimin3_s32(lo, va, vb);
        hi = __vimax3_s32(hi, va, vb);
      }
      d[i * stride + j] = (px_t)clampi(clampi(x + ((8 + sum - (sum < 0)) >> 4), lo, hi), 0, maxv);
      continue;
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const int tap = q == 0 ? pt0 : (q == 1 ? pt1 : (q & 1 ? 1 : 2));
      const int th = q < 2 ? pri : sec, sh = q < 2 ? psh : ssh;
#pragma unroll
      for (int sg = -1; sg <= 1; sg += 2) {
        const int dy = sg * oy[q], dx = sg * ox[q];
        if (EDGE) {
          const int px = x0 + j + dx, py = y0 + i + dy;
          if (px < 0 || px >= pw || py < 0 || py >= ph) continue;
        }
        const int v = win[(i + 2 + dy) * 12 + j + 2 + dx];
        if (th) sum += tap * cdef_cst(v - x, th, sh);
        lo = mini(lo, v);
        hi = maxi(hi, v);
      }
    }
    d[i * stride + j] = (px_t)clampi(clampi(x + ((8 + sum - (sum < 0)) >> 4), lo, hi), 0, maxv);
  }
}

/* One CDEF record by a half-warp (lanes `hmask`, this thread `hl`) with its
 * 12x12 window `win` in shared memory. */
__device__ __forceinline__ void cdef_record(const px_t* __restrict__ src, px_t* dst,
                                            const CdefRec& r, const int* __restrict__ search,
                                            const Layout& L, int* win, int hl, unsigned hmask) {
  const int p = r.plane;
  const bool uv = p > 0;
  const PlaneGeom& g = L.p[p];
  const int bd = L.bit_depth, maxv = (1 << bd) - 1, cs = bd - 8;
  const int w = uv ? (8 >> L.ss_x) : 8, h = uv ? (8 >> L.ss_y) : 8;
  const int pw = g.grid_w, ph = g.grid_h;
  /* the block and its halo; rows and columns above or left of the buffer
   * clamp into it (taps outside the plane are never used) */
  for (StepWalk wk(hl, 16, w + 4); wk.k < (h + 4) * (w + 4); wk.next()) {
    const int i = wk.r, j = wk.q;
    const int y = maxi(r.y - 2 + i, 0), x = maxi(r.x - 2 + j, 0);
    win[i * 12 + j] = src[g.off + y * g.stride + x];
  }
  int pri = r.pri << cs, sec = r.sec << cs;
  const int damping = r.damping + cs - (uv ? 1 : 0);
  int dir = r.dir;
  if (dir < 0) {
    const int sr = search[r.search];
    const int ydir = sr & 7, var = sr >> 3;
    if (uv) {
      dir = pri == 0 ? 0 : kCdefUvDir[L.ss_x][L.ss_y][ydir];
    } else {
      const int vs = (var >> 6) ? mini(floor_log2(var >> 6), 12) : 0;
      dir = pri == 0 ? 0 : ydir;
      pri = var ? ((pri * (4 + vs) + 8) >> 4) : 0;
    }
  }
  __syncwarp(hmask);
  px_t* d = dst + g.off + r.y * g.stride + r.x;
  if (pri == 0 && sec == 0) {
    for (int k = hl; k < w * h; k += 16) {
      const int i = k / w, j = k - i * w;
      if (r.y + i < ph && r.x + j < pw) d[i * g.stride + j] = (px_t)win[(i + 2) * 12 + j + 2];
    }
    return;
  }
  const int ts = (pri >> cs) & 1;
  const int pt0 = ts ? 3 : 4, pt1 = ts ? 3 : 2;
  const int psh = pri ? maxi(0, damping - floor_log2(pri)) : 0;
  const int ssh = sec ? maxi(0, damping - floor_log2(sec)) : 0;
  /* taps: primary (dir) k = 0, 1; secondary (dir - 2, dir + 2) k = 0, 1 */
  int oy[6], ox[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const int dd = q < 2 ? dir : (q < 4 ? (dir + 6) & 7 : (dir + 2) & 7);
    const int t = q & 1;
    oy[q] = kCdefDirs[dd][t][0];
    ox[q] = kCdefDirs[dd][t][1];
  }
  const bool interior = r.x >= 2 && r.y >= 2 && r.x + w + 2 <= pw && r.y + h + 2 <= ph;
  if (interior)
    cdef_samples<false>(win, d, g.stride, w, h, hl, r.x, r.y, pw, ph, oy, ox, pri, psh, sec, ssh,
                        pt0, pt1, maxv);
  else
    cdef_samples<true>(win, d, g.stride, w, h, hl, r.x, r.y, pw, ph, oy, ox, pri, psh, sec, ssh,
                       pt0, pt1, maxv);
}

__global__ void __launch_bounds__(128) k_cdef(const px_t* __restrict__ src, px_t* dst,
                                              const CdefRec* recs, int n,
                                              const int* __restrict__ search,
                                              const __grid_constant__ Layout L) {
  __shared__ int sw[8][12 * 12];
  const int hw = threadIdx.x >> 4, hl = threadIdx.x & 15;
  const unsigned hmask = 0xffffu << (threadIdx.x & 16);
  const int ri = blockIdx.x * 8 + hw;
  if (ri >= n) return;
  const CdefRec r = recs[ri];
  cdef_record(src, dst, r, search, L, sw[hw], hl, hmask);
}

/* ---- superres ------------------------------------------------------------------------- */
/* One CTA of 128 threads per 512 output samples of a row, a thread per 4
 * (CTAs of half that, 64 threads, took 11 % longer: twice the CTAs,
 * each staging the taps and its span). The source span those outputs read (a
 * superres step is at most one source sample, so at most 512 + 8 samples) is
 * staged in shared memory once, with
 * the clamp to the coded row applied while staging, and the 8-tap phases
 * beside it; each output then reads its taps there. Grid rows: the luma
 * rows, then the chroma rows with plane 1's segments and plane 2's side by
 * side. `border_rows`: only the rows within two of a loop restoration stripe
 * boundary (the rows the restoration reads from the pre-CDEF picture,
 * av1gpu_kernels.h:2832-2845); the reference upscales the whole pre-CDEF
 * picture and reads only these. */
#define AV1B_UP_SPAN 544
/* One CTA item (segment xb of grid row yb): the caller has filled `taps`
 * (the 64 filter phases); the body stages the source span, meets the CTA
 * barrier and writes. Early returns are either uniform over the CTA or after
 * its last barrier. */
__device__ __forceinline__ void upscale_item(const px_t* __restrict__ src, px_t* dst, const Layout& L,
                                             const UpscaleArgs& u, int maxv, int border_rows,
                                             int rows0, int xb, int yb, const short* taps,
                                             px_t* span) {
  int y = yb, p = 0;
  if (y >= rows0) {
    y -= rows0;
    const int xb1 = (L.p[1].out_w + AV1B_UP_OUT - 1) / AV1B_UP_OUT;
    p = 1;
    if (xb >= xb1) {
      xb -= xb1;
      p = 2;
    }
  }
  const PlaneGeom& g = L.p[p];
  if (border_rows) {
    const int sub_y = p > 0 ? L.ss_y : 0;
    const int b = (64 * (y / 4 + 1) - 8) >> sub_y;
    y = b - 2 + (y & 3);
    if (y < 0) return;
  }
  const int xs = xb * AV1B_UP_OUT;
  if (y >= g.out_h || xs >= g.out_w) return;  /* uniform over the CTA */
  const px_t* row = src + g.off + y * g.stride;
  px_t* out = dst + g.off + y * g.stride;
  const int last = g.coded_w - 1;
  const int step = u.step[p], init = u.initial[p] - (1 << 14);
  const int xe = min(xs + AV1B_UP_OUT, g.out_w) - 1;
  const int p0 = (init + xs * step) >> 14;
  const int n = ((init + xe * step) >> 14) - p0 + 8;
  const bool staged = n <= AV1B_UP_SPAN;
  if (staged)
    for (int i = threadIdx.x; i < n; i += blockDim.x) span[i] = row[clampi(p0 - 3 + i, 0, last)];
  __syncthreads();
  const int x0 = xs + threadIdx.x * 4;
  if (x0 > xe) return;
  int o[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int x = min(x0 + q, xe);  /* past the row's end: a repeat, not stored */
    const int sx = init + x * step;
    const int px = sx >> 14;
    const int4 fv = *reinterpret_cast<const int4*>(taps + ((sx & ((1 << 14) - 1)) >> 8) * 8);
    const int f[8] = {(short)fv.x, fv.x >> 16, (short)fv.y, fv.y >> 16,
                      (short)fv.z, fv.z >> 16, (short)fv.w, fv.w >> 16};
    int sum = 0;
    if (staged) {
      const px_t* sp = span + (px - p0);
#pragma unroll
      for (int k = 0; k < 8; ++k) sum += (int)sp[k] * f[k];
    } else {
#pragma unroll
      for (int k = 0; k < 8; ++k) sum += (int)row[clampi(px + k - 3, 0, last)] * f[k];
    }
    o[q] = clampi(rnd2(sum, 7), 0, maxv);
  }
  if (x0 + 3 <= xe && (reinterpret_cast<uintptr_t>(out) & 7) == 0) {
    uint2 v;
    v.x = (unsigned)o[0] | ((unsigned)o[1] << 16);
    v.y = (unsigned)o[2] | ((unsigned)o[3] << 16);
    *reinterpret_cast<uint2*>(out + x0) = v;
  } else {
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (x0 + q <= xe) out[x0 + q] = (px_t)o[q];
  }
}

__global__ void __launch_bounds__(128) k_upscale(const px_t* __restrict__ src, px_t* dst,
                                                const __grid_constant__ Layout L,
                                                const __grid_constant__ UpscaleArgs u, int maxv,
                                                int border_rows, int rows0) {
  __shared__ __align__(16) short taps[512];
  __shared__ px_t span[AV1B_UP_SPAN];
  for (int i = threadIdx.x; i < 512; i += blockDim.x) taps[i] = kUpscaleFilter[i];
  upscale_item(src, dst, L, u, maxv, border_rows, rows0, blockIdx.x, blockIdx.y, taps, span);
}

/* ---- loop restoration --------------------------------------------------------------------- */
/* Loop restoration by tiles: one CTA per (plane, stripe piece, 32 columns).
 * A stripe piece is the rows of one 64-row luma stripe (offset by 8), so every
 * sample of the tile reads through the same stripe mapping (get_source_sample,
 * av1gpu_kernels.h:2832-2845), and a 32-column tile lies in one restoration
 * unit (units are 32..256 wide; the last one of a row extends to the edge).
 * The source window (3 samples of margin) is staged in shared memory once.
 * Wiener runs as a horizontal pass into an intermediate (rounded and clipped
 * like the reference's) and a vertical pass. Self-guided computes A and B of
 * every box position the tile needs once - the reference recomputes them nine
 * times per output sample (av1gpu_kernels.h:2928-2970) - then projects. */
#define AV1B_LR_MAXR 64
#define AV1B_LR_WR (AV1B_LR_MAXR + 6)
#define AV1B_LR_WC (AV1B_LR_TW + 6)
#define AV1B_LR_AR (AV1B_LR_MAXR + 2)
#define AV1B_LR_AC (AV1B_LR_TW + 2)

/* A and B of one self-guided box position (i, j) from its box sums `sq`
 * (squares) and `sb` (samples). */
__device__ __forceinline__ void sgr_ab(unsigned sq, int sb, int bd, int n, long long mtable, int one_over_n,
                                       const short* xbyx1, int* a_out, int* b_out) {
  const long long sa = rnd2llz(static_cast<long long>(sq), 2 * (bd - 8));
  const long long sbs = rnd2z(sb, bd - 8);
  long long pv = sa * n - sbs * sbs;
  if (pv < 0) pv = 0;
  const int z = rnd2ll(pv * mtable, 20);
  const int a2 = xbyx1[mini(z, 255)];
  const long long b2 = (long long)(256 - a2) * sb * one_over_n;
  *a_out = a2;
  *b_out = rnd2ll(b2, 12);
}

/* The box sums of a self-guided pass of radius RAD, register blocked: a
 * thread takes one column and LR_G box positions STEP rows apart (the first
 * pass of radius 2 keeps every other row, the second of radius 1 every row),
 * sums each window row it needs across the box once, and adds those row sums
 * down each box - (2 RAD + 1) (STEP (LR_G - 1) + 2 RAD + 1) loads for LR_G
 * positions instead of (2 RAD + 1)^2 each. Positions i = first, first + STEP,
 * ... below `ar` and columns below `ac`; window rows below `wr` are read. */
#define AV1B_LR_G 4
template <int RAD, int STEP>
__device__ __forceinline__ void sgr_box_pass(const int* win, int* a_out, int* b_out, int first, int ar,
                                             int ac, int wr, int bd, int n, long long mtable,
                                             int one_over_n, const short* xbyx1) {
  constexpr int NR = STEP * (AV1B_LR_G - 1) + 2 * RAD + 1;
  const int rows = ar > first ? (ar - first + STEP - 1) / STEP : 0;
  const int groups = (rows + AV1B_LR_G - 1) / AV1B_LR_G;
  for (int it = threadIdx.x; it < groups * ac; it += blockDim.x) {
    const int g = it / ac, j = it - g * ac;
    const int i0 = first + g * AV1B_LR_G * STEP;
    int hs[NR];
    unsigned hq[NR];
#pragma unroll
    for (int t = 0; t < NR; ++t) {
      const int row = i0 + 2 - RAD + t;
      int sum = 0;
      unsigned sq = 0;
      if (row < wr) {
        const int* w = win + row * AV1B_LR_WC + j + 2 - RAD;
#pragma unroll
        for (int dx = 0; dx <= 2 * RAD; ++dx) {
          const int c = w[dx];
          sum += c;
          sq += static_cast<unsigned>(c * c);
        }
      }
      hs[t] = sum;
      hq[t] = sq;
    }
#pragma unroll
    for (int k = 0; k < AV1B_LR_G; ++k) {
      const int i = i0 + k * STEP;
      if (i < ar) {
        int sb = 0;
        unsigned sq = 0;   /* at most 25 * 4095^2 */
#pragma unroll
        for (int t = 0; t <= 2 * RAD; ++t) {
          sb += hs[k * STEP + t];
          sq += hq[k * STEP + t];
        }
        sgr_ab(sq, sb, bd, n, mtable, one_over_n, xbyx1, a_out + i * AV1B_LR_AC + j,
               b_out + i * AV1B_LR_AC + j);
      }
    }
  }
}

/* Shared memory of one loop restoration tile. */
struct LrSmem {
  int win[AV1B_LR_WR * AV1B_LR_WC];
  int aux[2][2][AV1B_LR_AR * AV1B_LR_AC];  /* Wiener: aux[0][0] = intermediate */
  short xbyx1[256];   /* a2 = ((z << 8) + z / 2) / (z + 1), by z */
};

/* One tile (bx, stripe, bz). Early returns are uniform over the CTA or after
 * its last barrier. */
__device__ __forceinline__ void lr_tile_item(const px_t* __restrict__ cdef,
                                             const px_t* __restrict__ curr, px_t* dst,
                                             const Layout& L, const LrArgs& r, int maxv,
                                             int copy_rest, int bx, int stripe, int bz,
                                             LrSmem& sm) {
  int* win = sm.win;
  auto& aux = sm.aux;
  short* xbyx1 = sm.xbyx1;
  /* grid z: luma, then chroma with plane 1's tiles and plane 2's side by side */
  int p = bz;
  if (p > 0) {
    const int t1 = (L.p[1].out_w + AV1B_LR_TW - 1) / AV1B_LR_TW;
    if (bx >= t1) {
      bx -= t1;
      p = 2;
    }
  }
  const PlaneGeom& g = L.p[p];
  const int sub_y = p > 0 ? L.ss_y : 0;
  const int x0 = bx * AV1B_LR_TW;
  if (x0 >= g.out_w) return;
  /* the stripe piece */
  const int s0 = (-8 + stripe * 64) >> sub_y;
  const int s1 = s0 + (64 >> sub_y) - 1;
  const int y0 = maxi(s0, 0), y1 = mini(g.out_h, s1 + 1);
  if (y0 >= y1) return;
  const int tw = mini(AV1B_LR_TW, g.out_w - x0), th = y1 - y0;
  LrUnitRec u{};
  if (r.type[p]) {
    const int us = r.unit_size[p];
    const int urow = mini(r.unit_rows[p] - 1, ((((y0 << sub_y) + 8) >> sub_y) / us));
    const int ucol = mini(r.unit_cols[p] - 1, x0 / us);
    const int idx = urow * r.unit_cols[p] + ucol;
    if (idx < r.n_units[p]) u = r.units[p][idx];
  }
  if (u.type != 1 && u.type != 2) {
    /* not restored: with `copy_rest` (the source is not the destination's
     * own content) the tile passes through */
    if (copy_rest)
      for (StepWalk wk(threadIdx.x, blockDim.x, tw); wk.k < th * tw; wk.next())
        dst[g.off + (y0 + wk.r) * g.stride + x0 + wk.q] = cdef[g.off + (y0 + wk.r) * g.stride + x0 + wk.q];
    return;
  }
  const int wr = th + 6, wc = tw + 6;
  const px_t* pc = cdef + g.off;
  const px_t* pp = curr + g.off;
  /* source window: rows y0-3 .., columns x0-3 .. */
  for (StepWalk wk(threadIdx.x, blockDim.x, wc); wk.k < wr * wc; wk.next()) {
    const int i = wk.r, j = wk.q;
    const int x = clampi(x0 - 3 + j, 0, g.out_w - 1);
    const int y = clampi(y0 - 3 + i, 0, g.out_h - 1);
    int v;
    if (y < s0) v = pp[maxi(y, s0 - 2) * g.stride + x];
    else if (y > s1) v = pp[mini(y, s1 + 2) * g.stride + x];
    else v = pc[y * g.stride + x];
    win[i * AV1B_LR_WC + j] = v;
  }
  __syncthreads();
  const int bd = L.bit_depth;
  px_t* out = dst + g.off + y0 * g.stride + x0;
  if (u.type == 1) {
    const int r0 = bd == 12 ? 5 : 3, r1 = bd == 12 ? 9 : 11;
    const int offset = 1 << (bd + 7 - r0 - 1);
    const int limit = (1 << (bd + 1 + 7 - r0)) - 1;
    int ht[7], vt[7];
    for (int t = 0; t < 3; ++t) {
      ht[t] = ht[6 - t] = u.hf[t];
      vt[t] = vt[6 - t] = u.vf[t];
    }
    ht[3] = 128 - 2 * (u.hf[0] + u.hf[1] + u.hf[2]);
    vt[3] = 128 - 2 * (u.vf[0] + u.vf[1] + u.vf[2]);
    /* the intermediate has up to 70 rows: it spans aux[0][0] and aux[0][1] */
    static_assert(AV1B_LR_WR * AV1B_LR_AC <= 2 * AV1B_LR_AR * AV1B_LR_AC, "Wiener intermediate");
    int* mid = &aux[0][0][0];
    for (StepWalk wk(threadIdx.x, blockDim.x, tw); wk.k < wr * tw; wk.next()) {
      const int i = wk.r, j = wk.q;
      const int* w = win + i * AV1B_LR_WC + j;
      int acc = 0;
#pragma unroll
      for (int t = 0; t < 7; ++t) acc += ht[t] * w[t];
      mid[i * AV1B_LR_AC + j] = clampi(rnd2(acc, r0), -offset, limit - offset);
    }
    __syncthreads();
    for (StepWalk wk(threadIdx.x, blockDim.x, tw); wk.k < th * tw; wk.next()) {
      const int i = wk.r, j = wk.q;
      int acc = 0;
#pragma unroll
      for (int t = 0; t < 7; ++t) acc += vt[t] * mid[(i + t) * AV1B_LR_AC + j];
      out[i * g.stride + j] = (px_t)clampi(rnd2(acc, r1), 0, maxv);
    }
    return;
  }
  /* self-guided: A and B of both passes on rows y0-1 .. y1, columns x0-1 .. */
  for (int z = threadIdx.x; z < 256; z += blockDim.x)
    xbyx1[z] = static_cast<short>(z >= 255 ? 256 : (z == 0 ? 1 : ((z << 8) + (z / 2)) / (z + 1)));
  __syncthreads();
  const int ar = th + 2, ac = tw + 2;
  /* unrolled: the unit record stays in registers (indexed by a loop
   * variable it would live in local memory) */
#pragma unroll
  for (int pass = 0; pass < 2; ++pass) {
    const int rad = u.r[pass];
    if (rad == 0) continue;
    const int n = (2 * rad + 1) * (2 * rad + 1);
    const long long n2e = (long long)n * n * u.e[pass];
    const long long mtable = ((1LL << 20) + n2e / 2) / n2e;
    const int one_over_n = ((1 << 12) + (n / 2)) / n;
    /* the first pass keeps the odd rows of the picture only */
    if (pass == 0 && rad == 2) {
      sgr_box_pass<2, 2>(win, aux[0][0], aux[0][1], y0 & 1, ar, ac, wr, bd, n, mtable, one_over_n, xbyx1);
      continue;
    }
    if (pass == 1 && rad == 1) {
      sgr_box_pass<1, 1>(win, aux[1][0], aux[1][1], 0, ar, ac, wr, bd, n, mtable, one_over_n, xbyx1);
      continue;
    }
    for (StepWalk wk(threadIdx.x, blockDim.x, ac); wk.k < ar * ac; wk.next()) {
      const int i = wk.r, j = wk.q;
      /* the first pass reads odd rows only */
      if (pass == 0 && !((y0 - 1 + i) & 1)) continue;
      unsigned sq = 0;   /* at most 25 * 4095^2 */
      int sb = 0;
      for (int dy = -rad; dy <= rad; ++dy) {
        const int* w = win + (i + 2 + dy) * AV1B_LR_WC + j + 2;
        for (int dx = -rad; dx <= rad; ++dx) {
          const int c = w[dx];
          sq += static_cast<unsigned>(c * c);
          sb += c;
        }
      }
      sgr_ab(sq, sb, bd, n, mtable, one_over_n, xbyx1, &aux[pass][0][i * AV1B_LR_AC + j],
             &aux[pass][1][i * AV1B_LR_AC + j]);
    }
  }
  __syncthreads();
  const int w0 = u.xqd[0], w1 = u.xqd[1], w2 = 128 - w0 - w1;
  for (StepWalk wk(threadIdx.x, blockDim.x, tw); wk.k < th * tw; wk.next()) {
    const int i = wk.r, j = wk.q;
    const int y = y0 + i;
    const int v = win[(i + 3) * AV1B_LR_WC + j + 3];
    int flt[2] = {0, 0};
#pragma unroll
    for (int pass = 0; pass < 2; ++pass) {
      if (u.r[pass] == 0) continue;
      int a = 0, b = 0;
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          int wgt;
          if (pass == 0) wgt = ((y + dy) & 1) ? (dx == 0 ? 6 : 5) : 0;
          else wgt = (dx == 0 || dy == 0) ? 4 : 3;
          if (!wgt) continue;
          const int o = (i + 1 + dy) * AV1B_LR_AC + j + 1 + dx;
          a += wgt * aux[pass][0][o];
          b += wgt * aux[pass][1][o];
        }
      const int shift = (pass == 0 && (y & 1)) ? 4 : 5;
      flt[pass] = rnd2ll((long long)a * v + b, 8 + shift - 4);
    }
    const int vs = v << 4;
    long long t = (long long)w1 * vs;
    t += (long long)w0 * (u.r[0] ? flt[0] : vs);
    t += (long long)w2 * (u.r[1] ? flt[1] : vs);
    out[i * g.stride + j] = (px_t)clampi(rnd2ll(t, 11), 0, maxv);
  }
}

__global__ void __launch_bounds__(256) k_lr_tile(const px_t* __restrict__ cdef,
                                                 const px_t* __restrict__ curr, px_t* dst,
                                                 const __grid_constant__ Layout L,
                                                 const __grid_constant__ LrArgs r, int maxv,
                                                 int copy_rest) {
  __shared__ LrSmem sm;
  lr_tile_item(cdef, curr, dst, L, r, maxv, copy_rest, blockIdx.x, blockIdx.y, blockIdx.z, sm);
}

/* ---- film grain ------------------------------------------------------------------------------- */

/* Generates the three grain templates (7.18.3.3): Gaussian noise from the LFSR
 * (every draw independent through the orbit table), then the auto-regressive
 * filter as a wavefront: sample (x, y) depends on rows above within +-lag
 * columns and on the lag samples to its left, so t = x + 4y orders it
 * (lag <= 3). One block: the Gaussian fill on all its threads, the filters
 * of the three templates on its first warps, luma and chroma in the same
 * steps. */

/* Luma rows the auto-regressive filter runs (3 .. 72 of the 82x73
 * template), a thread each. */
constexpr int kGrainLumaRows = 70;

/* The step by which the chroma wavefront trails the luma one: a chroma
 * sample (x, y) of step x + 4y + delay reads the luma samples it averages
 * (columns ((x - 3) << ss_x) + 3 .. + ss_x, rows likewise), whose own step
 * X + 4Y is at most delay - 1 before it; the lag grows with x (y) when
 * ss_x (ss_y) doubles the luma coordinate, largest at the template's last
 * column (row). */
__host__ __device__ __forceinline__ int grain_chroma_delay(int ss_x, int ss_y, int cw, int ch) {
  return (ss_x ? cw - 6 : 0) + 4 * (ss_y ? ch - 3 : 0) + 1;
}

/* The auto-regressive filters of the three templates (7.18.3.3) with lag
 * LAG, by wavefront: sample (x, y) reads the LAG rows above within +-LAG
 * columns and the LAG samples to its left, so the steps t = x + 4y order
 * it, and the samples of one step are independent. Thread tid <
 * kGrainLumaRows takes luma row 3 + tid; thread kGrainLumaRows + i takes
 * chroma item i (plane i & 1, row i >> 1), its wavefront `delay` steps
 * behind (grain_chroma_delay) so that every luma sample it reads is final.
 * All `nthreads` threads (a multiple of 32) meet a named barrier after each
 * step. */
template <int LAG>
__device__ void grain_ar(const GrainParamsDev& prm, short* luma, short* cb, short* cr, int cw, int ch,
                         bool chroma, int arshift, int gmin, int gmax, int tid, int nthreads) {
  constexpr int NT = 2 * LAG * (LAG + 1);   /* taps before the sample itself */
  constexpr int W = 82, H = 73;
  const bool do_luma = prm.num_y_points > 0;
  const int sx = prm.ss_x, sy = prm.ss_y;
  const int delay = chroma && do_luma ? grain_chroma_delay(sx, sy, cw, ch) : 0;
  const bool luma_thread = tid < kGrainLumaRows;
  const int ci = tid - kGrainLumaRows;
  const int plane = ci & 1;
  /* this thread's row of its template, and its work */
  const int y = luma_thread ? 3 + tid : ci >> 1;
  const bool mine = luma_thread ? do_luma : (chroma && ci >= 0 && ci < 2 * ch && y >= 3);
  short* gp = luma_thread ? luma : (plane ? cr : cb);
  const int gw = luma_thread ? W : cw;
  const int off = luma_thread ? 0 : delay;
  int co[NT + 1];
  {
    const int* cp = luma_thread ? prm.ar_y : (plane ? prm.ar_cr : prm.ar_cb);
#pragma unroll
    for (int i = 0; i <= NT; ++i) co[i] = (luma_thread && i == NT) ? 0 : cp[i];
  }
  const int tl = do_luma ? (W - 4) + 4 * (H - 1) : 0;
  const int tc = chroma ? (cw - 4) + 4 * (ch - 1) + delay : 0;
  const int tmax = tl > tc ? tl : tc;
  for (int t = 3 + 4 * 3; t <= tmax; ++t) {
    const int x = t - off - 4 * y;
    if (mine && x >= 3 && x < gw - 3) {
      int sum = 0, k = 0;
#pragma unroll
      for (int dr = -LAG; dr <= 0; ++dr)
#pragma unroll
        for (int dc = -LAG; dc <= LAG; ++dc) {
          if (dr == 0 && dc == 0) break;
          sum += gp[(y + dr) * gw + x + dc] * co[k++];
        }
      if (!luma_thread && do_luma) {
        const int lx = ((x - 3) << sx) + 3, ly = ((y - 3) << sy) + 3;
        int acc = 0;
        for (int i = 0; i <= sy; ++i)
          for (int j = 0; j <= sx; ++j) acc += luma[(ly + i) * W + lx + j];
        sum += rnd2z(acc, sx + sy) * co[NT];
      }
      gp[y * gw + x] = (short)clampi(gp[y * gw + x] + rnd2z(sum, arshift), gmin, gmax);
    }
    asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
  }
}

/* The templates live in shared memory while the auto-regressive wavefront
 * runs (hundreds of dependent steps: every tap a shared-memory read, not a
 * global one) and are written out at the end. */
struct GrainTemplateSmem {
  short luma[82 * 73], cb[82 * 73], cr[82 * 73];
};

/* Every thread of the CTA runs it (the filters on its first five warps);
 * it has no early return. */
__device__ __forceinline__ void grain_template_body(GrainState* gs, const GrainParamsDev& prm,
                                                    const uint16_t* orbit, const uint16_t* pos,
                                                    GrainTemplateSmem& sm) {
  short* s_luma = sm.luma;
  short* s_cb = sm.cb;
  short* s_cr = sm.cr;
  const int tid = threadIdx.x;
  const int bd = prm.bitdepth;
  const int shift = 12 - bd + prm.grain_scale_shift;
  const int gmin = -(128 << (bd - 8)), gmax = (256 << (bd - 8)) - 1 - (128 << (bd - 8));
  const int cw = gs->chroma_w, ch = gs->chroma_h;
  short* luma = s_luma;
  short* cb = s_cb;
  short* cr = s_cr;
  /* Gaussian fill */
  for (int k = tid; k < 82 * 73; k += blockDim.x) {
    int g = 0;
    if (prm.num_y_points > 0) {
      const int st = lfsr_after(orbit, pos, (unsigned)prm.seed & 0xffffu, k + 1);
      g = kGaussianSequence[(st >> 5) & 2047];
    }
    luma[k] = (short)rnd2z(g, shift);
  }
  const bool chroma = prm.chroma_scaling_from_luma || prm.num_cb_points > 0 || prm.num_cr_points > 0;
  if (chroma) {
    const bool acb = prm.num_cb_points > 0 || prm.chroma_scaling_from_luma;
    const bool acr = prm.num_cr_points > 0 || prm.chroma_scaling_from_luma;
    for (int k = tid; k < cw * ch; k += blockDim.x) {
      int g0 = 0, g1 = 0;
      if (acb) g0 = kGaussianSequence[(lfsr_after(orbit, pos, ((unsigned)prm.seed ^ 0xb524u) & 0xffffu, k + 1) >> 5) & 2047];
      if (acr) g1 = kGaussianSequence[(lfsr_after(orbit, pos, ((unsigned)prm.seed ^ 0x49d8u) & 0xffffu, k + 1) >> 5) & 2047];
      cb[k] = (short)rnd2z(g0, shift);
      cr[k] = (short)rnd2z(g1, shift);
    }
  }
  __syncthreads();
  const int arshift = prm.ar_coeff_shift_minus_6 + 6;
  /* the auto-regressive filters on the first warps (a step of a wavefront
   * has at most 70 luma and 146 chroma samples, one a thread: 96 threads for
   * luma alone, up to 224 with chroma), a named barrier between steps; the
   * lag as a constant, so a sample's taps are independent loads */
  const int ar_threads = ((kGrainLumaRows + (chroma ? 2 * ch : 0)) + 31) & ~31;
  if (tid < ar_threads) {
    switch (prm.ar_coeff_lag) {
      case 0: grain_ar<0>(prm, luma, cb, cr, cw, ch, chroma, arshift, gmin, gmax, tid, ar_threads); break;
      case 1: grain_ar<1>(prm, luma, cb, cr, cw, ch, chroma, arshift, gmin, gmax, tid, ar_threads); break;
      case 2: grain_ar<2>(prm, luma, cb, cr, cw, ch, chroma, arshift, gmin, gmax, tid, ar_threads); break;
      default: grain_ar<3>(prm, luma, cb, cr, cw, ch, chroma, arshift, gmin, gmax, tid, ar_threads); break;
    }
  }
  __syncthreads();
  for (int k = tid; k < 82 * 73; k += blockDim.x) gs->luma[k] = luma[k];
  if (chroma)
    for (int k = tid; k < cw * ch; k += blockDim.x) {
      gs->cb[k] = cb[k];
      gs->cr[k] = cr[k];
    }
}

__global__ void __launch_bounds__(256) k_grain_template(GrainState* gs, GrainParamsDev prm,
                                                        const uint16_t* orbit,
                                                        const uint16_t* pos) {
  __shared__ GrainTemplateSmem sm;
  grain_template_body(gs, prm, orbit, pos, sm);
}

/* The stripe values of plane `p` (7.18.3.5, the horizontal half: the grain
 * block that covers the column, blended with the previous block at the two -
 * one for subsampled chroma - overlap columns) of four samples
 * x0 .. x0 + 3 of one row, x0 a multiple of 4: they lie in one grain block,
 * whose random offset is computed once; only a group starting a block has
 * overlap columns. */
__device__ __forceinline__ void grain_stripe4(const GrainState* gs, const short* grain, int src_w,
                                              int sub_x, int sub_y, int s, int row, int x0,
                                              const uint16_t* orbit, const uint16_t* pos, int gmin,
                                              int gmax, bool overlap, int n[4]) {
  unsigned st0 = (unsigned)gs->seed & 0xffffu;
  st0 ^= (unsigned)(((s * 37 + 178) & 255) << 8);
  st0 ^= (unsigned)((s * 173 + 105) & 255);
  st0 &= 0xffffu;
  const int bw_log = sub_x ? 4 : 5;
  const int k = x0 >> bw_log, j0 = x0 & ((1 << bw_log) - 1);
  auto block_row = [&](int blk) {
    const int r = (lfsr_after(orbit, pos, st0, blk + 1) >> 8) & 255;
    const int ox = r >> 4, oy = r & 15;
    const int src_x = sub_x ? 6 + ox : 9 + ox * 2;
    const int src_y = sub_y ? 6 + oy : 9 + oy * 2;
    return grain + (src_y + row) * src_w + src_x;
  };
  const short* cur = block_row(k) + j0;
#pragma unroll
  for (int q = 0; q < 4; ++q) n[q] = cur[q];
  if (overlap && k > 0 && j0 == 0) {
    const short* prev = block_row(k - 1);
    if (!sub_x) {
      n[0] = clampi(rnd2z((int)prev[32] * 27 + n[0] * 17, 5), gmin, gmax);
      n[1] = clampi(rnd2z((int)prev[33] * 17 + n[1] * 27, 5), gmin, gmax);
    } else {
      n[0] = clampi(rnd2z((int)prev[16] * 23 + n[0] * 22, 5), gmin, gmax);
    }
  }
}

/* Film grain blend, out of place: `src` is the decoded picture (luma read
 * before any grain), `dst` gets the output picture. One thread per four
 * samples of a row (8-byte loads and stores; a chroma group reads its luma as
 * one 8- or 16-byte load); the arithmetic per sample is that of
 * 7.18.3.5 (the no-allocation entry point's grain_sample is the same per
 * sample). Grid rows are the luma rows, then the chroma rows
 * with plane 1's groups and plane 2's side by side, so a chroma row of
 * 4:2:0 fills a grid row as a luma row does. */
/* The film grain output of four samples x0 .. x0 + 3 (x0 a multiple of 4) of
 * row y of plane p, from their decoded values `orig` (7.18.3.5); `src` is the
 * picture before grain (a chroma sample reads its luma there), `vec` whether
 * it is 16-byte aligned. */
__device__ __forceinline__ void grain_group4(const px_t* __restrict__ src, const Layout& L,
                                             const GrainState* gs, const uint16_t* orbit,
                                             const uint16_t* pos, int p, int y, int x0, bool vec,
                                             const int (&orig)[4], int (&out)[4]) {
  const int bd = gs->bitdepth;
#pragma unroll
  for (int q = 0; q < 4; ++q) out[q] = orig[q];
  const bool active = p == 0 ? gs->num_points[0] > 0 : (gs->chroma_from_luma || gs->num_points[p] > 0);
  if (active) {
    const int sub_x = p ? L.ss_x : 0, sub_y = p ? L.ss_y : 0;
    const int gmin = -(128 << (bd - 8)), gmax = (256 << (bd - 8)) - 1 - (128 << (bd - 8));
    const short* grain = p == 0 ? gs->luma : (p == 1 ? gs->cb : gs->cr);
    const int src_w = p == 0 ? 82 : gs->chroma_w;
    const bool overlap = gs->overlap != 0;
    /* vertical half: stripes of 32 (16) rows, blended with the stripe above */
    const int sh = 5 - sub_y;
    const int s = y >> sh, row = y - (s << sh);
    int n[4];
    grain_stripe4(gs, grain, src_w, sub_x, sub_y, s, row, x0, orbit, pos, gmin, gmax, overlap, n);
    if (overlap && s > 0) {
      if (!sub_y && row < 2) {
        int old[4];
        grain_stripe4(gs, grain, src_w, sub_x, sub_y, s - 1, row + 32, x0, orbit, pos, gmin, gmax,
                      overlap, old);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          n[q] = clampi(rnd2z(row == 0 ? old[q] * 27 + n[q] * 17 : old[q] * 17 + n[q] * 27, 5), gmin,
                        gmax);
      } else if (sub_y && row == 0) {
        int old[4];
        grain_stripe4(gs, grain, src_w, sub_x, sub_y, s - 1, 16, x0, orbit, pos, gmin, gmax, overlap,
                      old);
#pragma unroll
        for (int q = 0; q < 4; ++q) n[q] = clampi(rnd2z(old[q] * 23 + n[q] * 22, 5), gmin, gmax);
      }
    }
    int index[4];
    if (p == 0) {
#pragma unroll
      for (int q = 0; q < 4; ++q) index[q] = orig[q];
    } else {
      /* the co-located luma sample and its right neighbour (clamped to the
       * luma width), before grain */
      const PlaneGeom& gl = L.p[0];
      const int ly = y << L.ss_y, lx0 = x0 << L.ss_x;
      const px_t* lrow = src + gl.off + ly * gl.stride;
      int lum[8];
      if (vec && L.ss_x) {
        const uint4 v = *reinterpret_cast<const uint4*>(lrow + lx0);
        lum[0] = v.x & 0xffff;
        lum[1] = v.x >> 16;
        lum[2] = v.y & 0xffff;
        lum[3] = v.y >> 16;
        lum[4] = v.z & 0xffff;
        lum[5] = v.z >> 16;
        lum[6] = v.w & 0xffff;
        lum[7] = v.w >> 16;
      } else if (vec) {
        const uint2 v = *reinterpret_cast<const uint2*>(lrow + lx0);
        lum[0] = v.x & 0xffff;
        lum[1] = v.x >> 16;
        lum[2] = v.y & 0xffff;
        lum[3] = v.y >> 16;
        lum[4] = lum[5] = lum[6] = lum[7] = 0;
      } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) lum[q] = (L.ss_x || q < 4) ? lrow[min(lx0 + q, gl.out_w - 1)] : 0;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        int avg;
        if (L.ss_x) {
          const int lx = lx0 + 2 * q;
          const int l0 = lum[2 * q];
          const int l1 = lx + 1 < gl.out_w ? lum[2 * q + 1] : l0;
          avg = rnd2z(l0 + l1, 1);
        } else {
          avg = lum[q];
        }
        if (gs->chroma_from_luma) {
          index[q] = avg;
        } else {
          const int comb = avg * (gs->luma_mult[p] - 128) + orig[q] * (gs->mult[p] - 128);
          index[q] = clampi((comb >> 6) + (gs->offset[p] - 256) * (1 << (bd - 8)), 0, (1 << bd) - 1);
        }
      }
    }
    const int hi = p == 0 ? gs->max_luma : gs->max_chroma;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int scaled = rnd2z(grain_scale_lut(gs->lut[p], index[q], bd) * n[q], gs->scaling_shift);
      out[q] = clampi(orig[q] + scaled, gs->min_value, hi);
    }
  }
}

/* One thread's four samples: group gi of grid row y (no barrier). */
__device__ __forceinline__ void grain_blend_item(const px_t* __restrict__ src, px_t* dst,
                                                 const Layout& L, const GrainState* gs,
                                                 const uint16_t* orbit, const uint16_t* pos,
                                                 int gi, int y) {
  int p = 0;
  if (y >= L.p[0].out_h) {
    y -= L.p[0].out_h;
    const int g1 = (L.p[1].out_w + 3) >> 2;
    p = 1;
    if (gi >= g1) {
      gi -= g1;
      p = 2;
    }
  }
  const PlaneGeom& g = L.p[p];
  const int x0 = gi * 4;
  if (x0 >= g.out_w || y >= g.out_h) return;
  const int idx = g.off + y * g.stride + x0;
  const bool vec = ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0;
  const int nq = min(4, g.out_w - x0);
  int orig[4];
  if (vec) {
    const uint2 v = *reinterpret_cast<const uint2*>(src + idx);
    orig[0] = v.x & 0xffff;
    orig[1] = v.x >> 16;
    orig[2] = v.y & 0xffff;
    orig[3] = v.y >> 16;
  } else {
#pragma unroll
    for (int q = 0; q < 4; ++q) orig[q] = q < nq ? src[idx + q] : 0;
  }
  int out[4];
  grain_group4(src, L, gs, orbit, pos, p, y, x0, vec, orig, out);
  if (vec && nq == 4) {
    uint2 v;
    v.x = (unsigned)out[0] | ((unsigned)out[1] << 16);
    v.y = (unsigned)out[2] | ((unsigned)out[3] << 16);
    *reinterpret_cast<uint2*>(dst + idx) = v;
  } else {
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (q < nq) dst[idx + q] = (px_t)out[q];
  }
}

__global__ void k_grain_blend(const px_t* __restrict__ src, px_t* dst,
                              const __grid_constant__ Layout L,
                              const GrainState* gs, const uint16_t* orbit, const uint16_t* pos) {
  grain_blend_item(src, dst, L, gs, orbit, pos, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y);
}

/* ---- output packing ---------------------------------------------------------------------------- */

/* NV12: one thread per 8 output bytes of a `pitch`-byte row; rows [0, h) are
 * luma, then (h + 1) / 2 rows of interleaved Cb, Cr. Padding is zero.
 *
 * The reference packs a copy of the picture gathered row by row at the
 * *coded* width into a display-sized frame that starts out zero
 * (cpu_backend.cpp:576-584), so for a superres frame every sample right of the
 * coded width packs as 0. This kernel reproduces that byte for byte. */
/* One thread's eight bytes at byte x0 of NV12 row `row` (no barrier). */
__device__ __forceinline__ void nv12_item(const px_t* __restrict__ pic, uint8_t* out, const Layout& L,
                                          int pitch, int x0, int row) {
  if (x0 >= pitch) return;
  const int w = L.p[0].out_w, h = L.p[0].out_h;
  const int shift = L.bit_depth - 8;
  uint8_t v[8];
  if (row < h) {
    const px_t* src = pic + L.p[0].off + row * L.p[0].stride;
    const int lim = mini(w, L.p[0].coded_w);
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = x0 + k < lim ? (uint8_t)(src[x0 + k] >> shift) : 0;
  } else {
    const int cr = row - h;
    const int cw = (w + 1) >> 1;
    const int ccw = L.p[1].coded_w;
    const px_t* u = pic + L.p[1].off + cr * L.p[1].stride;
    const px_t* vv = pic + L.p[2].off + cr * L.p[2].stride;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int x = x0 + k;
      v[k] = (x < 2 * cw && (x >> 1) < ccw) ? (uint8_t)(((x & 1) ? vv[x >> 1] : u[x >> 1]) >> shift) : 0;
    }
  }
  uint8_t* d = out + (size_t)row * pitch + x0;
  if (x0 + 8 <= pitch && ((reinterpret_cast<uintptr_t>(d) & 7) == 0)) {
    uint2 pk;
    pk.x = v[0] | (v[1] << 8) | (v[2] << 16) | ((unsigned)v[3] << 24);
    pk.y = v[4] | (v[5] << 8) | (v[6] << 16) | ((unsigned)v[7] << 24);
    *reinterpret_cast<uint2*>(d) = pk;
  } else {
    for (int k = 0; k < 8 && x0 + k < pitch; ++k) d[k] = v[k];
  }
}

__global__ void k_nv12(const px_t* __restrict__ pic, uint8_t* out, const __grid_constant__ Layout L,
                       int pitch) {
  nv12_item(pic, out, L, pitch, (blockIdx.x * blockDim.x + threadIdx.x) * 8, blockIdx.y);
}

/* NV12 with the film grain of the packed samples applied while packing:
 * eight bytes of row `row` at byte x0, from the picture before grain. The
 * same arithmetic per sample as grain_blend_item followed by nv12_item. */
__device__ __forceinline__ void nv12_grain_item(const px_t* __restrict__ pic, uint8_t* out,
                                                const Layout& L, int pitch, int x0, int row,
                                                const GrainState* gs, const uint16_t* orbit,
                                                const uint16_t* pos) {
  if (x0 >= pitch) return;
  const int w = L.p[0].out_w, h = L.p[0].out_h;
  const int shift = L.bit_depth - 8;
  const bool vec = (reinterpret_cast<uintptr_t>(pic) & 15) == 0;
  uint8_t v[8];
  if (row < h) {
    const px_t* src = pic + L.p[0].off + row * L.p[0].stride;
    const int lim = mini(w, L.p[0].coded_w);
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int xs = x0 + 4 * half;
      int orig[4] = {0, 0, 0, 0}, o[4] = {0, 0, 0, 0};
      if (xs < lim) {
#pragma unroll
        for (int q = 0; q < 4; ++q) orig[q] = xs + q < w ? src[xs + q] : 0;
        grain_group4(pic, L, gs, orbit, pos, 0, row, xs, vec, orig, o);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) v[4 * half + q] = xs + q < lim ? (uint8_t)(o[q] >> shift) : 0;
    }
  } else {
    const int cr = row - h;
    const int cw = (w + 1) >> 1;
    const int ccw = L.p[1].coded_w;
    const int cx0 = x0 >> 1;
    int ou[4] = {0, 0, 0, 0}, ov[4] = {0, 0, 0, 0};
    if (cx0 < mini(cw, ccw)) {
      const px_t* u = pic + L.p[1].off + cr * L.p[1].stride;
      const px_t* vv = pic + L.p[2].off + cr * L.p[2].stride;
      int origu[4], origv[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        origu[q] = cx0 + q < L.p[1].out_w ? u[cx0 + q] : 0;
        origv[q] = cx0 + q < L.p[2].out_w ? vv[cx0 + q] : 0;
      }
      grain_group4(pic, L, gs, orbit, pos, 1, cr, cx0, vec, origu, ou);
      grain_group4(pic, L, gs, orbit, pos, 2, cr, cx0, vec, origv, ov);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int x = x0 + k;
      const int c = (x >> 1) - cx0;
      v[k] = (x < 2 * cw && (x >> 1) < ccw) ? (uint8_t)(((x & 1) ? ov[c] : ou[c]) >> shift) : 0;
    }
  }
  uint8_t* d = out + (size_t)row * pitch + x0;
  if (x0 + 8 <= pitch && ((reinterpret_cast<uintptr_t>(d) & 7) == 0)) {
    uint2 pk;
    pk.x = v[0] | (v[1] << 8) | (v[2] << 16) | ((unsigned)v[3] << 24);
    pk.y = v[4] | (v[5] << 8) | (v[6] << 16) | ((unsigned)v[7] << 24);
    *reinterpret_cast<uint2*>(d) = pk;
  } else {
    for (int k = 0; k < 8 && x0 + k < pitch; ++k) d[k] = v[k];
  }
}

/* NV12 of a picture whose film grain was not applied yet (its decode read
 * nothing back): the grain of each packed sample is computed while packing,
 * and the display picture is not written. */
__global__ void k_nv12_grain(const px_t* __restrict__ pic, uint8_t* out,
                             const __grid_constant__ Layout L, int pitch, const GrainState* gs,
                             const uint16_t* orbit, const uint16_t* pos) {
  nv12_grain_item(pic, out, L, pitch, (blockIdx.x * blockDim.x + threadIdx.x) * 8, blockIdx.y, gs,
                  orbit, pos);
}

__global__ void k_rgb(const px_t* __restrict__ pic, uint8_t* out, const __grid_constant__ Layout L,
                      const __grid_constant__ RgbArgs m) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const int w = L.p[0].out_w;
  if (x >= w) return;
  /* zero right of the coded width, as in the reference's gathered frame */
  const int yy = x < L.p[0].coded_w ? pic[L.p[0].off + y * L.p[0].stride + x] : 0;
  const int cx = x >> L.ss_x;
  const int ci = (y >> L.ss_y) * L.p[1].stride + cx;
  const int uu = cx < L.p[1].coded_w ? pic[L.p[1].off + ci] : 0;
  const int vv = cx < L.p[2].coded_w ? pic[L.p[2].off + ci] : 0;
  const int r = (m.m[0] * yy + m.m[1] * vv + m.o[0]) >> 16;
  const int g = (m.m[2] * yy + m.m[3] * uu + m.m[4] * vv + m.o[1]) >> 16;
  const int b = (m.m[5] * yy + m.m[6] * uu + m.o[2]) >> 16;
  uint8_t* d = out + ((size_t)y * w + x) * 3;
  d[0] = (uint8_t)clampi(r, 0, 255);
  d[1] = (uint8_t)clampi(g, 0, 255);
  d[2] = (uint8_t)clampi(b, 0, 255);
}

/* ---- launchers ------------------------------------------------------------------------------------ */
static inline unsigned cdiv(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

cudaError_t launch_recon_stage(int stage, const FrameArgs& a, int n_sm, cudaStream_t s) {
  switch (stage) {
    case 1:
      if (a.n_inter_tiles > 0)
      {
        if (a.n_inter_simple > 0)
          k_inter_simple<false><<<cdiv(a.n_inter_simple, 4), 128, 0, s>>>(a, 0, a.n_inter_simple);
        const int lm_end = a.n_inter_simple + a.n_inter_lmask;
        if (a.n_inter_lmask > 0)
          k_inter_simple<true><<<cdiv(a.n_inter_lmask, 4), 128, 0, s>>>(a, a.n_inter_simple, lm_end);
        /* the full kernel's tiles, then the chroma tiles that read the masks
         * the luma tiles wrote */
        const int cm_first = a.n_inter_tiles - a.n_inter_cmask;
        if (cm_first > lm_end) k_inter<<<cdiv(cm_first - lm_end, 4), 128, 0, s>>>(a, lm_end, cm_first);
        if (a.n_inter_cmask > 0)
          k_inter_simple<true><<<cdiv(a.n_inter_cmask, 4), 128, 0, s>>>(a, cm_first, a.n_inter_tiles);
      }
      break;
    case 2:
      if (a.n_itx_batches > 0) {
        cudaError_t e;
        if ((e = launch_itx_class<2>(a, s)) != cudaSuccess || (e = launch_itx_class<3>(a, s)) != cudaSuccess ||
            (e = launch_itx_class<4>(a, s)) != cudaSuccess || (e = launch_itx_class<5>(a, s)) != cudaSuccess ||
            (e = launch_itx_class<6>(a, s)) != cudaSuccess || (e = launch_itx_class<7>(a, s)) != cudaSuccess)
          return e;
      }
      break;
    default:
      if (a.n_units > 0) {
        const size_t smem = 4 * (3 * AV1B_EDGE_LEN + AV1B_UNIT_SCRATCH) * sizeof(int);
        const int grid = AV1B_UNIT_CTAS_PER_SM * n_sm;
        if (a.units_inter) k_units<true><<<grid, 128, smem, s>>>(a);
        else k_units<false><<<grid, 128, smem, s>>>(a);
      }
      break;
  }
  return cudaGetLastError();
}

/* A frame's deblocking edges and CDEF blocks, converted where the caller's
 * lists were uploaded: one thread per record validates and converts it
 * (prep_edge / prep_cdef, the checks the host planner runs too). Edges are
 * compacted into the V and H lists with one atomic per warp: the edges of one
 * direction are independent, so their order in a list does not matter. A CDEF
 * block off the 8x8 search grid gets a search of its own, listed after the
 * grid. `out` (zeroed by the caller) gets the counts and the invalid flag. */
__global__ void __launch_bounds__(256) k_prep_filters(
    const av1b_deblock_edge* __restrict__ de, int nde, const av1b_cdef_block* __restrict__ cb,
    int ncb, const Layout L, int grid_w, int grid_n, DeblockRec* __restrict__ v,
    DeblockRec* __restrict__ h, CdefRec* __restrict__ cdef, unsigned* __restrict__ extra,
    PrepOut* __restrict__ out) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool is_edge = i < nde, is_cdef = !is_edge && i < static_cast<long long>(nde) + ncb;
  int code = kPrepSkip, vert = 0, off_grid = 0;
  DeblockRec er{};
  CdefRec cr{};
  unsigned pos = 0;
  if (is_edge) {
    code = prep_edge(L, de[i], &er, &vert);
  } else if (is_cdef) {
    const av1b_cdef_block& c = cb[i - nde];
    code = prep_cdef(L, c, grid_w, &cr, &off_grid);
    if (code == kPrepOk && off_grid) {
      const int sx = c.plane ? L.ss_x : 0, sy = c.plane ? L.ss_y : 0;
      pos = static_cast<unsigned>(c.x << sx) | (static_cast<unsigned>(c.y << sy) << 16);
    }
  }
  const bool ok = code == kPrepOk;
  const unsigned mv = __ballot_sync(0xffffffffu, is_edge && ok && vert);
  const unsigned mh = __ballot_sync(0xffffffffu, is_edge && ok && !vert);
  const unsigned me = __ballot_sync(0xffffffffu, is_cdef && ok && off_grid);
  const unsigned mg = __ballot_sync(0xffffffffu, is_cdef && ok && !off_grid && cr.dir < 0);
  const unsigned mb = __ballot_sync(0xffffffffu, code >= kPrepErrFirst);
  unsigned bv = 0, bh = 0, be = 0;
  if (lane == 0) {
    if (mv) bv = atomicAdd(&out->n_v, __popc(mv));
    if (mh) bh = atomicAdd(&out->n_h, __popc(mh));
    if (me) be = atomicAdd(&out->n_extra, __popc(me));
    if (mg) atomicOr(&out->any_grid, 1u);
    if (mb) atomicOr(&out->bad, 1u);
  }
  bv = __shfl_sync(0xffffffffu, bv, 0);
  bh = __shfl_sync(0xffffffffu, bh, 0);
  be = __shfl_sync(0xffffffffu, be, 0);
  const unsigned below = (1u << lane) - 1u;
  if (is_edge && ok) {
    if (vert)
      v[bv + __popc(mv & below)] = er;
    else
      h[bh + __popc(mh & below)] = er;
  } else if (is_cdef && ok) {
    if (off_grid) {
      const unsigned k = be + __popc(me & below);
      cr.search = grid_n + static_cast<int>(k);
      extra[k] = pos;
    }
    cdef[i - nde] = cr;
  }
}

cudaError_t launch_prep_filters(const av1b_deblock_edge* edges, int n_edges, const av1b_cdef_block* cdef,
                                int n_cdef, const Layout& L, int grid_w, int grid_n, DeblockRec* v,
                                DeblockRec* h, CdefRec* cdef_out, unsigned* extra, PrepOut* out,
                                cudaStream_t s) {
  const long long n = static_cast<long long>(n_edges) + n_cdef;
  if (n <= 0) return cudaSuccess;
  k_prep_filters<<<cdiv(n, 256), 256, 0, s>>>(edges, n_edges, cdef, n_cdef, L, grid_w, grid_n, v, h,
                                              cdef_out, extra, out);
  return cudaGetLastError();
}

cudaError_t launch_deblock(px_t* pic, const DeblockRec* recs, int n, int sharpness, int bd, int maxv,
                           cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_deblock<AV1B_DB_PLAIN><<<cdiv(cdiv(n, AV1B_DB_PLAIN) * 32, 256), 256, 0, s>>>(pic, recs, n, sharpness, bd,
                                                                                  maxv);
  return cudaGetLastError();
}

cudaError_t launch_cdef(const px_t* src, px_t* dst, const CdefRec* recs, int n, int grid_w,
                        int grid_n, bool grid, const unsigned* extra_pos, int n_extra, int* search,
                        const Layout& L, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int n_grid = grid ? grid_n : 0;
  if (n_grid + n_extra > 0)
    k_cdef_search<<<cdiv(n_grid + n_extra, 128), 128, 0, s>>>(src, grid_w, grid_n, n_grid, extra_pos,
                                                               n_extra, search, L);
  k_cdef<<<cdiv(n, 8), 128, 0, s>>>(src, dst, recs, n, search, L);
  return cudaGetLastError();
}

cudaError_t launch_upscale(const px_t* src, px_t* dst, const Layout& L, int maxv, bool border_rows,
                           cudaStream_t s) {
  UpscaleArgs u;
  for (int p = 0; p < 3; ++p) superres_params(L.p[p].coded_w, L.p[p].out_w, &u.step[p], &u.initial[p]);
  /* grid rows: the luma rows, then the chroma rows (planes 1 and 2 side by side) */
  const int rows0 = border_rows ? 4 * ((L.p[0].out_h + 8) / 64 + 1) : L.p[0].out_h;
  const int rows1 = L.p[1].out_h > 0 ? (border_rows ? rows0 : L.p[1].out_h) : 0;
  const int segs = maxi(cdiv(L.p[0].out_w, AV1B_UP_OUT), 2 * cdiv(L.p[1].out_w, AV1B_UP_OUT));
  k_upscale<<<dim3(segs, rows0 + rows1), 128, 0, s>>>(src, dst, L, u, maxv, border_rows ? 1 : 0, rows0);
  return cudaGetLastError();
}

cudaError_t launch_lr(const px_t* cdef, const px_t* curr, px_t* dst, const Layout& L,
                      const LrArgs& r, int maxv, bool copy_rest, cudaStream_t s) {
  const int stripes = (L.p[0].out_h + 8 + 63) / 64;
  const int tiles = maxi(cdiv(L.p[0].out_w, AV1B_LR_TW), 2 * cdiv(L.p[1].out_w, AV1B_LR_TW));
  k_lr_tile<<<dim3(tiles, stripes, 2), 256, 0, s>>>(cdef, curr, dst, L, r, maxv, copy_rest ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_grain_template(GrainState* gs, const GrainParamsDev& prm, const uint16_t* orbit,
                                  const uint16_t* pos, cudaStream_t s) {
  k_grain_template<<<1, 256, 0, s>>>(gs, prm, orbit, pos);
  return cudaGetLastError();
}

cudaError_t launch_grain_blend(const px_t* src, px_t* dst, const Layout& L, const GrainState* gs,
                               const uint16_t* orbit, const uint16_t* pos, cudaStream_t s) {
  /* grid rows: the luma rows, then the chroma rows (planes 1 and 2 side by side) */
  const int groups = maxi(cdiv(L.p[0].out_w, 4), 2 * cdiv(L.p[1].out_w, 4));
  const int rows = L.p[0].out_h + L.p[1].out_h;
  k_grain_blend<<<dim3(cdiv(groups, 128), rows), 128, 0, s>>>(src, dst, L, gs, orbit, pos);
  return cudaGetLastError();
}

cudaError_t launch_nv12(const px_t* pic, uint8_t* out, const Layout& L, int pitch, cudaStream_t s) {
  const int rows = L.p[0].out_h + (L.p[0].out_h + 1) / 2;
  k_nv12<<<dim3(cdiv(cdiv(pitch, 8), 128), rows), 128, 0, s>>>(pic, out, L, pitch);
  return cudaGetLastError();
}

cudaError_t launch_nv12_grain(const px_t* pic, uint8_t* out, const Layout& L, int pitch,
                              const GrainState* gs, const uint16_t* orbit, const uint16_t* pos,
                              cudaStream_t s) {
  const int rows = L.p[0].out_h + (L.p[0].out_h + 1) / 2;
  k_nv12_grain<<<dim3(cdiv(cdiv(pitch, 8), 128), rows), 128, 0, s>>>(pic, out, L, pitch, gs, orbit, pos);
  return cudaGetLastError();
}

cudaError_t launch_rgb(const px_t* pic, uint8_t* out, const Layout& L, const RgbArgs& m,
                       cudaStream_t s) {
  k_rgb<<<dim3(cdiv(L.p[0].out_w, 128), L.p[0].out_h), 128, 0, s>>>(pic, out, L, m);
  return cudaGetLastError();
}

/* Loads every kernel of this file now. With lazy module loading (the CUDA
 * 12 default) a kernel's first launch loads its code, and a load waits for
 * the kernels already running; decoder creation loading them all keeps that
 * wait out of every frame. */
template <class K>
static cudaError_t load_kernel(K k) {
  cudaFuncAttributes fa;
  return cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(k));
}

static cudaError_t load_all_kernels() {
  cudaError_t e;
  if ((e = load_kernel(k_inter_simple<false>)) != cudaSuccess ||
      (e = load_kernel(k_inter_simple<true>)) != cudaSuccess || (e = load_kernel(k_inter)) != cudaSuccess ||
      (e = load_kernel(k_itx<2>)) != cudaSuccess || (e = load_kernel(k_itx<3>)) != cudaSuccess ||
      (e = load_kernel(k_itx<4>)) != cudaSuccess || (e = load_kernel(k_itx<5>)) != cudaSuccess ||
      (e = load_kernel(k_itx<6>)) != cudaSuccess || (e = load_kernel(k_itx<7>)) != cudaSuccess ||
      (e = load_kernel(k_units<true>)) != cudaSuccess || (e = load_kernel(k_units<false>)) != cudaSuccess ||
      (e = load_kernel(k_selftest_wait)) != cudaSuccess || (e = load_kernel(k_deblock<AV1B_DB_PLAIN>)) != cudaSuccess ||
      (e = load_kernel(k_cdef_search)) != cudaSuccess || (e = load_kernel(k_cdef)) != cudaSuccess ||
      (e = load_kernel(k_upscale)) != cudaSuccess || (e = load_kernel(k_lr_tile)) != cudaSuccess ||
      (e = load_kernel(k_grain_template)) != cudaSuccess || (e = load_kernel(k_grain_blend)) != cudaSuccess ||
      (e = load_kernel(k_nv12)) != cudaSuccess || (e = load_kernel(k_nv12_grain)) != cudaSuccess ||
      (e = load_kernel(k_rgb)) != cudaSuccess ||
      (e = load_kernel(k_dequant)) != cudaSuccess || (e = load_kernel(k_prep_filters)) != cudaSuccess)
    return e;
  return cudaSuccess;
}

cudaError_t set_kernel_attributes() {
  {
    const cudaError_t e = load_all_kernels();
    if (e != cudaSuccess) return e;
  }
  cudaError_t e = cudaFuncSetAttribute(k_units<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       4 * (3 * AV1B_EDGE_LEN + AV1B_UNIT_SCRATCH) * (int)sizeof(int));
  if (e != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_units<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                4 * (3 * AV1B_EDGE_LEN + AV1B_UNIT_SCRATCH) * (int)sizeof(int))) != cudaSuccess)
    return e;
  /* phase B's picture reads bypass L1: the SM's memory goes to shared memory,
   * so AV1B_UNIT_CTAS_PER_SM CTAs fit */
  if ((e = cudaFuncSetAttribute(k_units<true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared)) != cudaSuccess ||
      (e = cudaFuncSetAttribute(k_units<false>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared)) != cudaSuccess)
    return e;
  /* the two classes whose scratch passes the 48 KB default */
  if ((e = cudaFuncSetAttribute(k_itx<6>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                4 * 4096 * (int)sizeof(int))) != cudaSuccess)
    return e;
  return cudaFuncSetAttribute(k_itx<7>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              4 * 4096 * (int)sizeof(int));
}

/* ---- batched form: the stage kernels of many streams ------------------------------------- */
#include "batch_kernels.cuh"

}  // namespace av1b
