/*
 * dev_inter.cuh - inter prediction arithmetic (specification 7.11.3).
 *
 * Each function computes one output sample with the reference's arithmetic
 * (av1gpu_kernels.h:1689-2326):
 *   - two-stage separable 8-tap interpolation with InterRound0 / InterRound1
 *     (1756-1786), the 4-tap rows for 4-sample extents (1696-1701);
 *   - the scaled path of reference scaling / superres, positions in 1/1024
 *     (1809-1857);
 *   - global warp with the per-8x8 projection and alpha..delta shear
 *     (1919-1958);
 *   - wedge and difference-weighted masks (1968-2068), OBMC taper
 *     (2076-2100), inter-intra taper and edges (2120-2205);
 *   - the composition order: references, compound / mask blend, clip,
 *     inter-intra, OBMC strips in order (2207-2326).
 * mc_rect is the separable form of the translation cases for a warp's tile,
 * with the reference window in shared memory; the per-sample forms serve the
 * warped references and the blocks of the dependency-scheduled phase.
 */
#ifndef AV1B_DEV_INTER_CUH
#define AV1B_DEV_INTER_CUH

#include "dev_common.cuh"
#include "wedge.h"

namespace av1b {

#define AV1B_SCALE_ONE (1 << 14)

struct InterCtx {
  int sub_x, sub_y;
  int ref_w, ref_h;   /* visible reference plane size: the clamp */
  int bitdepth;
  int scale_x, scale_y;
};

AV1B_HD int filt_row(int cls, int extent) {
  if (extent > 4) return cls;
  if (cls == 0 || cls == 2) return 4; /* regular, sharp -> 4-tap regular */
  if (cls == 1) return 5;             /* smooth -> 4-tap smooth */
  return cls;
}

AV1B_DEV int subpel(int row, int phase, int tap) { return kSubpelFilters[(row * 16 + phase) * 8 + tap]; }

/* A reference sample, clamped to the visible plane. CG: the reference is the
 * picture being decoded (intra block copy), read through L2. */
template <bool CG = false>
AV1B_DEV int fetch(const px_t* p, int stride, int x, int y, int x1, int y1) {
  x = clampi(x, 0, x1);
  y = clampi(y, 0, y1);
  if (CG) return (int)__ldcg(p + y * stride + x);
  return (int)__ldg(p + y * stride + x);
}

AV1B_DEV void rounds(int bitdepth, int compound, int* r0, int* r1) {
  *r0 = bitdepth >= 12 ? 5 : 3;
  *r1 = compound ? 7 : 11;
  if (bitdepth >= 12 && !compound) *r1 -= 2;
}

/* One sample, unscaled. (x, y) are relative to the patch origin. */
template <bool CG = false>
AV1B_DEV int mc_unscaled(const InterCtx& c, const px_t* ref, int stride, int base_x, int base_y,
                         int ew, int eh, int mvx, int mvy, int filt, int filt_v, int x, int y,
                         int compound) {
  const int mx = mvx * 2, my = mvy * 2;
  const int xs = mx >> (4 + c.sub_x), xf = (mx >> c.sub_x) & 15;
  const int ys = my >> (4 + c.sub_y), yf = (my >> c.sub_y) & 15;
  const int ax = base_x + x + xs, ay = base_y + y + ys;
  const int fh = filt_row(filt, ew), fv = filt_row(filt_v, eh);
  int r0, r1;
  rounds(c.bitdepth, compound, &r0, &r1);
  int acc = 0;
  for (int j = 0; j < 8; ++j) {
    int row = 0;
    for (int i = 0; i < 8; ++i)
      row += fetch<CG>(ref, stride, ax - 3 + i, ay - 3 + j, c.ref_w - 1, c.ref_h - 1) *
             subpel(fh, xf, i);
    acc += ((row + (1 << (r0 - 1))) >> r0) * subpel(fv, yf, j);
  }
  return (acc + (1 << (r1 - 1))) >> r1;
}

/* The scaled position of sample (x, y) of a patch: integer sample and 1/16
 * phase per axis (7.11.3.3). */
AV1B_DEV void scaled_pos(const InterCtx& c, int base_x, int base_y, int mvx, int mvy, int x, int y,
                         int* cx, int* cy, int* xf, int* yf) {
  const int ox = (base_x << 4) + ((2 * mvx) >> c.sub_x) + 8;
  const int oy = (base_y << 4) + ((2 * mvy) >> c.sub_y) + 8;
  const int bx = ox * c.scale_x - (8 << 14);
  const int by = oy * c.scale_y - (8 << 14);
  const int sx = rnd2s_shift(bx, 14 + 4 - 10) + (1 << (10 - 4 - 1));
  const int sy = rnd2s_shift(by, 14 + 4 - 10) + (1 << (10 - 4 - 1));
  const int stx = rnd2s_shift(c.scale_x, 14 - 10);
  const int sty = rnd2s_shift(c.scale_y, 14 - 10);
  const int px = sx + stx * x, py = sy + sty * y;
  *cx = px >> 10;
  *cy = py >> 10;
  *xf = (px & 1023) >> 6;
  *yf = (py & 1023) >> 6;
}

template <bool CG = false>
AV1B_DEV int mc_scaled(const InterCtx& c, const px_t* ref, int stride, int base_x, int base_y,
                       int ew, int eh, int mvx, int mvy, int filt, int filt_v, int x, int y,
                       int compound) {
  int cx, cy, xf, yf;
  scaled_pos(c, base_x, base_y, mvx, mvy, x, y, &cx, &cy, &xf, &yf);
  const int fh = filt_row(filt, ew), fv = filt_row(filt_v, eh);
  int r0, r1;
  rounds(c.bitdepth, compound, &r0, &r1);
  int acc = 0;
  for (int j = 0; j < 8; ++j) {
    int row = 0;
    for (int i = 0; i < 8; ++i)
      row += fetch<CG>(ref, stride, cx - 3 + i, cy - 3 + j, c.ref_w - 1, c.ref_h - 1) *
             subpel(fh, xf, i);
    acc += ((row + (1 << (r0 - 1))) >> r0) * subpel(fv, yf, j);
  }
  return (acc + (1 << (r1 - 1))) >> r1;
}

template <bool CG = false>
AV1B_DEV int mc_tap(const InterCtx& c, const px_t* ref, int stride, int base_x, int base_y, int ew,
                    int eh, int mvx, int mvy, int filt, int filt_v, int x, int y, int compound) {
  if (c.scale_x == AV1B_SCALE_ONE && c.scale_y == AV1B_SCALE_ONE)
    return mc_unscaled<CG>(c, ref, stride, base_x, base_y, ew, eh, mvx, mvy, filt, filt_v, x, y,
                           compound);
  return mc_scaled<CG>(c, ref, stride, base_x, base_y, ew, eh, mvx, mvy, filt, filt_v, x, y, compound);
}

/* Separable motion compensation of a rectangle of a patch, for one warp.
 * Every output sample of a translation (unscaled or scaled) prediction is
 * the vertical 8-tap filter over intermediate rows, each the horizontal
 * 8-tap filter of one reference row rounded by InterRound0; the intermediate
 * at (reference row, output column) is the same for every output sample that
 * reads it. So the reference window is staged in shared memory once, the
 * intermediate rows computed once, then the vertical pass - the same integers
 * as the per-sample form above (mc_unscaled / mc_scaled), 16 multiplies a
 * sample instead of 64.
 * The rectangle is (rx, ry) .. + (rw <= 16, rh <= 8) in patch coordinates;
 * `out` receives rh rows of 16. Returns false, with nothing written, when the
 * window does not fit the scratch (a reference scaled by more than 2:1). */
#define AV1B_MC_WR 24
#define AV1B_MC_WC 40
struct McScratch {
  int win[AV1B_MC_WR * AV1B_MC_WC];
  int mid[AV1B_MC_WR * 16];
  int4 ht[16][2], vt[8][2];   /* the taps of each output column, of each output row */
  int cx[16], xf[16], cy[8], yf[8];
};

template <bool CG = false>
AV1B_DEV bool mc_rect(const InterCtx& c, const px_t* ref, int stride, int base_x, int base_y,
                      int ew, int eh, int mvx, int mvy, int filt, int filt_v, int compound, int rx,
                      int ry, int rw, int rh, McScratch& s, int* out, int lane) {
  const bool unscaled = c.scale_x == AV1B_SCALE_ONE && c.scale_y == AV1B_SCALE_ONE;
  if (lane < rw || (lane >= 16 && lane - 16 < rh)) {
    const int k = lane & 15;
    int px, py, fx, fy;
    if (unscaled) {
      const int mx = mvx * 2, my = mvy * 2;
      px = base_x + rx + k + (mx >> (4 + c.sub_x));
      fx = (mx >> c.sub_x) & 15;
      py = base_y + ry + k + (my >> (4 + c.sub_y));
      fy = (my >> c.sub_y) & 15;
    } else {
      scaled_pos(c, base_x, base_y, mvx, mvy, rx + k, ry + k, &px, &py, &fx, &fy);
    }
    if (lane < 16) {
      s.cx[k] = px;
      s.xf[k] = fx;
    } else {
      s.cy[k] = py;
      s.yf[k] = fy;
    }
  }
  __syncwarp();
  const int cbase = s.cx[0] - 3, rbase = s.cy[0] - 3;
  const int ncols = s.cx[rw - 1] + 5 - cbase, nrows = s.cy[rh - 1] + 5 - rbase;
  if (ncols > AV1B_MC_WC || nrows > AV1B_MC_WR) {
    __syncwarp();
    return false;
  }
  if (cbase >= 0 && rbase >= 0 && cbase + ncols <= c.ref_w && rbase + nrows <= c.ref_h) {
    /* the window lies inside the reference (no sample clamps): four samples
     * a load from the 8-byte boundary at or left of it - the rows of a plane
     * start on 128-byte boundaries and run a border past the picture, so the
     * load never leaves the row; samples left or right of the window are
     * dropped */
    const int a0 = cbase & ~3;
    const int groups = (cbase + ncols - a0 + 3) >> 2;
    StepWalk wk(lane, 32, groups);
    for (int k = lane; k < nrows * groups; k += 32, wk.next()) {
      const uint2* src =
          reinterpret_cast<const uint2*>(ref + (rbase + wk.r) * stride + a0 + 4 * wk.q);
      const uint2 v = CG ? __ldcg(src) : __ldg(src);
      const int vals[4] = {static_cast<int>(v.x & 0xffff), static_cast<int>(v.x >> 16),
                           static_cast<int>(v.y & 0xffff), static_cast<int>(v.y >> 16)};
      const int q0 = a0 + 4 * wk.q - cbase;
      int* row = s.win + wk.r * AV1B_MC_WC;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (q0 + j >= 0 && q0 + j < ncols) row[q0 + j] = vals[j];
    }
  } else {
    StepWalk wk(lane, 32, ncols);
    for (int k = lane; k < nrows * ncols; k += 32, wk.next())
      s.win[wk.r * AV1B_MC_WC + wk.q] =
          fetch<CG>(ref, stride, cbase + wk.q, rbase + wk.r, c.ref_w - 1, c.ref_h - 1);
  }
  const int fh = filt_row(filt, ew), fv = filt_row(filt_v, eh);
  /* each column's and each row's taps, once */
  if (lane < rw) {
    const short* f = kSubpelFilters + (fh * 16 + s.xf[lane]) * 8;
    s.ht[lane][0] = make_int4(f[0], f[1], f[2], f[3]);
    s.ht[lane][1] = make_int4(f[4], f[5], f[6], f[7]);
  } else if (lane >= 16 && lane - 16 < rh) {
    const short* f = kSubpelFilters + (fv * 16 + s.yf[lane - 16]) * 8;
    s.vt[lane - 16][0] = make_int4(f[0], f[1], f[2], f[3]);
    s.vt[lane - 16][1] = make_int4(f[4], f[5], f[6], f[7]);
  }
  __syncwarp();
  int r0, r1;
  rounds(c.bitdepth, compound, &r0, &r1);
  {
    StepWalk wk(lane, 32, rw);
    for (int k = lane; k < nrows * rw; k += 32, wk.next()) {
      const int* w = s.win + wk.r * AV1B_MC_WC + s.cx[wk.q] - 3 - cbase;
      const int4 ta = s.ht[wk.q][0], tb = s.ht[wk.q][1];
      const int sum = w[0] * ta.x + w[1] * ta.y + w[2] * ta.z + w[3] * ta.w + w[4] * tb.x +
                      w[5] * tb.y + w[6] * tb.z + w[7] * tb.w;
      s.mid[wk.r * 16 + wk.q] = (sum + (1 << (r0 - 1))) >> r0;
    }
  }
  __syncwarp();
  {
    StepWalk wk(lane, 32, rw);
    for (int k = lane; k < rh * rw; k += 32, wk.next()) {
      const int* m = s.mid + (s.cy[wk.r] - 3 - rbase) * 16 + wk.q;
      const int4 ta = s.vt[wk.r][0], tb = s.vt[wk.r][1];
      const int acc = m[0] * ta.x + m[16] * ta.y + m[32] * ta.z + m[48] * ta.w + m[64] * tb.x +
                      m[80] * tb.y + m[96] * tb.z + m[112] * tb.w;
      out[wk.r * 16 + wk.q] = (acc + (1 << (r1 - 1))) >> r1;
    }
  }
  __syncwarp();
  return true;
}

AV1B_DEV int warp_offs(int v) {
  const int offs = (v + (1 << 9)) >> 10;
  return clampi(offs + 64, 0, 192);
}

/* One globally warped sample (7.11.3.5), (x, y) relative to the block. */
template <bool CG = false>
AV1B_DEV int warp_tap(int sub_x, int sub_y, int ref_w, int ref_h, const WarpRec& m,
                      const px_t* ref, int stride, int base_x, int base_y, int x, int y,
                      int bitdepth, int compound) {
  const int i8 = y >> 3, j8 = x >> 3;
  const int i1 = (y & 7) - 4, i2 = (x & 7) - 4;
  const long long src_x = (long long)((base_x + j8 * 8 + 4) << sub_x);
  const long long src_y = (long long)((base_y + i8 * 8 + 4) << sub_y);
  const long long dst_x = (long long)m.params[2] * src_x + (long long)m.params[3] * src_y + m.params[0];
  const long long dst_y = (long long)m.params[4] * src_x + (long long)m.params[5] * src_y + m.params[1];
  const long long x4 = dst_x >> sub_x, y4 = dst_y >> sub_y;
  const int ix4 = (int)(x4 >> 16), sx4 = (int)(x4 & 0xffff);
  const int iy4 = (int)(y4 >> 16), sy4 = (int)(y4 & 0xffff);
  int r0, r1;
  rounds(bitdepth, compound, &r0, &r1);
  const int offs_y = warp_offs(sy4 + m.abcd[2] * i2 + m.abcd[3] * i1);
  int acc = 0;
  for (int k = 0; k < 8; ++k) {
    const int row = i1 - 3 + k;
    const int offs_x = warp_offs(sx4 + m.abcd[0] * i2 + m.abcd[1] * row);
    const int ry = iy4 + row;
    int s = 0;
    for (int t = 0; t < 8; ++t)
      s += kWarpedFilters[offs_x * 8 + t] *
           fetch<CG>(ref, stride, ix4 + i2 - 3 + t, ry, ref_w - 1, ref_h - 1);
    acc += ((s + (1 << (r0 - 1))) >> r0) * kWarpedFilters[offs_y * 8 + k];
  }
  return (acc + (1 << (r1 - 1))) >> r1;
}

/* One 8x8 block of a globally warped prediction, for one warp, separable
 * like the reference's per-block warp (av1gpu_kernels.h:1919-1958): the
 * 15x15 reference window around the block's projected centre staged in
 * shared memory, the horizontal 8-tap filter (its phase from alpha and beta)
 * for the 15 rows x 8 columns the block reads, rounded by InterRound0, then
 * the vertical filter (phase from gamma and delta) - the same integers as
 * warp_tap, which computes them again for every output sample. (bx, by): the
 * 8x8 block's offset in the prediction block; out: rows of `out_stride`. */
template <bool CG = false>
AV1B_DEV void warp_block8(int sub_x, int sub_y, int ref_w, int ref_h, const WarpRec& m,
                          const px_t* ref, int stride, int base_x, int base_y, int bx, int by,
                          int bitdepth, int compound, McScratch& s, int* out, int out_stride,
                          int ow, int oh, int lane) {
  const long long src_x = (long long)((base_x + bx + 4) << sub_x);
  const long long src_y = (long long)((base_y + by + 4) << sub_y);
  const long long dst_x = (long long)m.params[2] * src_x + (long long)m.params[3] * src_y + m.params[0];
  const long long dst_y = (long long)m.params[4] * src_x + (long long)m.params[5] * src_y + m.params[1];
  const long long x4 = dst_x >> sub_x, y4 = dst_y >> sub_y;
  const int ix4 = (int)(x4 >> 16), sx4 = (int)(x4 & 0xffff);
  const int iy4 = (int)(y4 >> 16), sy4 = (int)(y4 & 0xffff);
  int r0, r1;
  rounds(bitdepth, compound, &r0, &r1);
  /* window rows iy4 - 7 .. iy4 + 7, columns ix4 - 7 .. ix4 + 7 */
  for (int k = lane; k < 15 * 15; k += 32) {
    const int r = k / 15, c = k - r * 15;
    s.win[r * 16 + c] = fetch<CG>(ref, stride, ix4 - 7 + c, iy4 - 7 + r, ref_w - 1, ref_h - 1);
  }
  __syncwarp();
  /* H[r][c]: row r - 7, column offset i2 = c - 4 */
  for (int k = lane; k < 15 * 8; k += 32) {
    const int r = k >> 3, c = k & 7;
    const int offs_x = warp_offs(sx4 + m.abcd[0] * (c - 4) + m.abcd[1] * (r - 7));
    const short* f = kWarpedFilters + offs_x * 8;
    const int* w = s.win + r * 16 + c;
    int sum = 0;
#pragma unroll
    for (int t = 0; t < 8; ++t) sum += f[t] * w[t];
    s.mid[r * 8 + c] = (sum + (1 << (r0 - 1))) >> r0;
  }
  __syncwarp();
  for (int k = lane; k < 64; k += 32) {
    const int i = k >> 3, j = k & 7;
    if (i >= oh || j >= ow) continue;
    const int offs_y = warp_offs(sy4 + m.abcd[2] * (j - 4) + m.abcd[3] * (i - 4));
    const short* f = kWarpedFilters + offs_y * 8;
    int acc = 0;
#pragma unroll
    for (int t = 0; t < 8; ++t) acc += f[t] * s.mid[(i + t) * 8 + j];
    out[i * out_stride + j] = (acc + (1 << (r1 - 1))) >> r1;
  }
  __syncwarp();
}

/* ---- masks ------------------------------------------------------------------- */

AV1B_DEV int wedge_px(int dir, int xoff, int yoff, int flip, int i, int j) {
  const int m = wedge_master(dir, clampi(yoff + i, 0, 63), clampi(xoff + j, 0, 63));
  return flip ? 64 - m : m;
}

AV1B_DEV int diffwtd_m(int d, int sh, int sign) {
  d = (d + (1 << (sh - 1))) >> sh;
  d = clampi(38 + (d >> 4), 0, 64);
  return sign ? 64 - d : d;
}

AV1B_DEV int obmc_mask(int length, int index) {
  switch (length) {
    case 2: {
      const unsigned char m[2] = {45, 64};
      return m[index];
    }
    case 4: {
      const unsigned char m[4] = {39, 50, 59, 64};
      return m[index];
    }
    case 8: {
      const unsigned char m[8] = {36, 42, 48, 53, 57, 61, 64, 64};
      return m[index];
    }
    case 16: {
      const unsigned char m[16] = {34, 37, 40, 43, 46, 49, 52, 54, 56, 58, 60, 61, 64, 64, 64, 64};
      return m[index];
    }
    default: {
      const unsigned char m[32] = {33, 35, 36, 38, 40, 41, 43, 44, 45, 47, 48, 50, 51, 52, 53, 55,
                                   56, 57, 58, 59, 60, 60, 61, 62, 64, 64, 64, 64, 64, 64, 64, 64};
      return m[index];
    }
  }
}

/* ---- one inter block, resolved ------------------------------------------------ */
struct InterJob {
  int x, y, w, h, plane;
  InterCtx ctx;
  const px_t* ref[2];       /* this plane of each reference (or of this picture) */
  int ref_stride;
  int mv[2][2];
  int filt, filt_v;
  int compound;             /* 0 none, 1 average, 2 distance, 3 wedge, 4 diffwtd */
  int w0, w1;
  int mask_kind, mask_sign; /* 0 none, 1 wedge, 2 difference weighted */
  int wedge_dir, wedge_xoff, wedge_yoff, wedge_flip;
  int warp[2], mask_warp[2];
  const WarpRec* model[2];
  /* chroma difference weighted mask: the luma planes of both references */
  const px_t* luma_ref[2];
  int luma_stride, luma_x, luma_y, luma_ref_w, luma_ref_h;
  /* inter-intra */
  int interintra, ii_mode, ii_wedge;
  int have_left, have_above, max_x, max_y;
  const px_t* cur;          /* this plane of the picture being decoded, block origin */
  int cur_stride;
  /* OBMC */
  const ObmcRec* obmc;
  int obmc_count;
  const px_t* obmc_ref[8];
  int maxv;
};

template <bool CG = false>
AV1B_DEV int mask_luma_diff(const InterJob& b, int lx, int ly, int ew, int eh) {
  InterCtx l;
  l.sub_x = 0;
  l.sub_y = 0;
  l.ref_w = b.luma_ref_w;
  l.ref_h = b.luma_ref_h;
  l.bitdepth = b.ctx.bitdepth;
  l.scale_x = b.ctx.scale_x;
  l.scale_y = b.ctx.scale_y;
  int v[2];
  for (int r = 0; r < 2; ++r)
    v[r] = b.mask_warp[r]
               ? warp_tap<CG>(0, 0, b.luma_ref_w, b.luma_ref_h, *b.model[r], b.luma_ref[r],
                              b.luma_stride, b.luma_x, b.luma_y, lx, ly, b.ctx.bitdepth, 1)
               : mc_tap<CG>(l, b.luma_ref[r], b.luma_stride, b.luma_x, b.luma_y, ew, eh, b.mv[r][0],
                        b.mv[r][1], b.filt, b.filt_v, lx, ly, 1);
  return v[0] - v[1];
}

AV1B_DEV int ii_above(const InterJob& b, int i) {
  const int mid = 1 << (b.ctx.bitdepth - 1);
  if (!b.have_above) return b.have_left ? ldpx(b.cur - 1) : mid - 1;
  if (b.x + i > b.max_x) i = b.max_x - b.x;
  return ldpx(b.cur - b.cur_stride + i);
}

AV1B_DEV int ii_left(const InterJob& b, int i) {
  const int mid = 1 << (b.ctx.bitdepth - 1);
  if (!b.have_left) return b.have_above ? ldpx(b.cur - b.cur_stride) : mid + 1;
  if (b.y + i > b.max_y) i = b.max_y - b.y;
  return ldpx(b.cur + i * b.cur_stride - 1);
}

AV1B_DEV int ii_dc(const InterJob& b) {
  int s = 0;
  if (b.have_above && b.have_left) {
    for (int k = 0; k < b.w; ++k) s += ii_above(b, k);
    for (int k = 0; k < b.h; ++k) s += ii_left(b, k);
    return (s + ((b.w + b.h) >> 1)) / (b.w + b.h);
  }
  if (b.have_left) {
    for (int k = 0; k < b.h; ++k) s += ii_left(b, k);
    return (s + (b.h >> 1)) >> ilog2(b.h);
  }
  if (b.have_above) {
    for (int k = 0; k < b.w; ++k) s += ii_above(b, k);
    return (s + (b.w >> 1)) >> ilog2(b.w);
  }
  return 1 << (b.ctx.bitdepth - 1);
}

AV1B_DEV int ii_sample(const InterJob& b, int x, int y, int dc) {
  if (b.ii_mode == 1) return ii_above(b, x);
  if (b.ii_mode == 2) return ii_left(b, y);
  if (b.ii_mode == 3) {
    const int wy = sm_weight(b.h, y), wx = sm_weight(b.w, x);
    return rnd2(wy * ii_above(b, x) + (256 - wy) * ii_left(b, b.h - 1) + wx * ii_left(b, y) +
                    (256 - wx) * ii_above(b, b.w - 1), 9);
  }
  return dc;
}

AV1B_DEV int ii_mask(const InterJob& b, int x, int y) {
  if (b.ii_wedge) {
    const int ny = b.ctx.sub_y + 1, nx = b.ctx.sub_x + 1;
    int sum = 0;
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        sum += wedge_px(b.wedge_dir, b.wedge_xoff, b.wedge_yoff, b.wedge_flip,
                        (y << b.ctx.sub_y) + j, (x << b.ctx.sub_x) + i);
    const int n = nx * ny;
    return n == 1 ? sum : (n == 2 ? (sum + 1) >> 1 : (sum + 2) >> 2);
  }
  if (b.ii_mode == 0) return 32;
  const int scale = 128 / maxi(b.w, b.h);
  int k = 0;
  if (b.ii_mode == 1) k = y * scale;
  else if (b.ii_mode == 2) k = x * scale;
  else k = mini(x, y) * scale;
  return kIiWeights[mini(k, 127)];
}

/* The composition of the block's two predictions `v0`, `v1` (or one) at
 * (x, y): average, distance weights or a mask, then the clip. */
/* The compound blend of two predictions with mask value m (0..64), clipped. */
AV1B_DEV int blend_mask(const InterJob& b, int v0, int v1, int m) {
  const int post = 7 - (b.ctx.bitdepth >= 12 ? 5 : 3);
  return clampi((m * v0 + (64 - m) * v1 + (1 << (5 + post))) >> (6 + post), 0, b.maxv);
}

template <bool CG = false>
AV1B_DEV int inter_compose(const InterJob& b, int x, int y, int v0, int v1) {
  int out = v0;
  if (b.compound) {
    const int round0 = b.ctx.bitdepth >= 12 ? 5 : 3;
    const int post = 7 - round0;
    if (b.mask_kind != 0) {
      const int sh = post + (b.ctx.bitdepth - 8);
      const int ny = b.ctx.sub_y + 1, nx = b.ctx.sub_x + 1;
      int sum = 0;
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const int lx = (x << b.ctx.sub_x) + i, ly = (y << b.ctx.sub_y) + j;
          int m;
          if (b.mask_kind == 1) {
            m = wedge_px(b.wedge_dir, b.wedge_xoff, b.wedge_yoff, b.wedge_flip, ly, lx);
            if (b.mask_sign) m = 64 - m;
          } else if (b.plane == 0) {
            m = diffwtd_m(absi(v0 - v1), sh, b.mask_sign);
          } else {
            m = diffwtd_m(absi(mask_luma_diff<CG>(b, lx, ly, b.w << b.ctx.sub_x, b.h << b.ctx.sub_y)),
                          sh, b.mask_sign);
          }
          sum += m;
        }
      const int n = nx * ny;
      const int m = n == 1 ? sum : (n == 2 ? (sum + 1) >> 1 : (sum + 2) >> 2);
      out = (m * v0 + (64 - m) * v1 + (1 << (5 + post))) >> (6 + post);
    } else if (b.compound == 1) {
      out = (v0 + v1 + (1 << post)) >> (1 + post);
    } else {
      out = (b.w0 * v0 + b.w1 * v1 + (1 << (3 + post))) >> (4 + post);
    }
  }
  return clampi(out, 0, b.maxv);
}

/* One reference's prediction of sample (x, y), per sample. */
template <bool CG = false>
AV1B_DEV int inter_ref(const InterJob& b, int r, int x, int y) {
  const int compound = b.compound != 0;
  return b.warp[r] ? warp_tap<CG>(b.ctx.sub_x, b.ctx.sub_y, b.ctx.ref_w, b.ctx.ref_h, *b.model[r],
                                  b.ref[r], b.ref_stride, b.x, b.y, x, y, b.ctx.bitdepth, compound)
                   : mc_tap<CG>(b.ctx, b.ref[r], b.ref_stride, b.x, b.y, b.w, b.h, b.mv[r][0],
                                b.mv[r][1], b.filt, b.filt_v, x, y, compound);
}

/* The block's prediction before inter-intra and OBMC, clipped. */
template <bool CG = false>
AV1B_DEV int inter_core(const InterJob& b, int x, int y) {
  const int v0 = inter_ref<CG>(b, 0, x, y);
  const int v1 = b.compound ? inter_ref<CG>(b, 1, x, y) : 0;
  return inter_compose<CG>(b, x, y, v0, v1);
}

AV1B_DEV int obmc_blend(const ObmcRec& c, int j, int i, int out, int pred, int maxv) {
  const int m = c.pass == 0 ? obmc_mask(c.h, i) : obmc_mask(c.w, j);
  pred = clampi(pred, 0, maxv);
  return (m * out + (64 - m) * pred + 32) >> 6;
}

/* Inter-intra and OBMC on top of a clipped prediction `out`. */
AV1B_DEV int inter_finish(const InterJob& b, int x, int y, int out, int ii_dc_value) {
  if (b.interintra) {
    const int m = ii_mask(b, x, y);
    const int intra = ii_sample(b, x, y, ii_dc_value);
    out = (m * intra + (64 - m) * out + 32) >> 6;
  }
  for (int k = 0; k < b.obmc_count; ++k) {
    const ObmcRec& c = b.obmc[k];
    if (x < c.x || x >= c.x + c.w || y < c.y || y >= c.y + c.h) continue;
    const int j = x - c.x, i = y - c.y;
    const int pred = mc_tap(b.ctx, b.obmc_ref[k], b.ref_stride, b.x + c.x, b.y + c.y, c.w, c.h,
                            c.mv_x, c.mv_y, c.filt, c.filt_v, j, i, 0);
    out = obmc_blend(c, j, i, out, pred, b.maxv);
  }
  return out;
}

}  // namespace av1b

#endif
