/*
 * dev_filters.cuh - the in-loop filters and the output process, per sample or
 * per block, with the reference's arithmetic:
 *   - deblocking: thresholds, filter mask, flat masks, narrow filter4 and the
 *     wide 6/8/14-tap filters (av1gpu_kernels.h:2422-2554);
 *   - CDEF: direction search, variance-adjusted strength, constrain and the
 *     primary / secondary taps clipped to the taps' range (2601-2775);
 *   - superres upscaling (2375-2402);
 *   - loop restoration: stripe-aware source, Wiener, self-guided (2832-2970);
 *   - film grain: scaling LUT interpolation and the blend (3295-3365), with the
 *     noise synthesis of src/core/grain.cpp and av1gpu_kernels.h:3057-3291
 *     re-derived so that any noise sample can be computed on its own (see
 *     grain_noise below);
 *   - NV12 and RGB packing (3379-3417).
 */
#ifndef AV1B_DEV_FILTERS_CUH
#define AV1B_DEV_FILTERS_CUH

#include "dev_common.cuh"

namespace av1b {

/* ---- deblocking ---------------------------------------------------------------- */
struct DeblockRec {
  int p_off;        /* sample p1 of the first position, picture offset */
  int across;       /* step across the edge (1 vertical, stride horizontal) */
  int along;        /* step along the edge */
  short len, level;
  unsigned char filter_size, chroma, pad0, pad1;
};

AV1B_DEV int f4clamp(int v, int bd) { return clampi(v, -(1 << (bd - 1)), (1 << (bd - 1)) - 1); }

/* One sample position of an edge; `b` points at p1. */
/* The wide filters (6-tap chroma, 8-tap and 16-tap luma): `N` samples each
 * side written, taps of weight 2 within `N2` of the centre, a 2^LOG2N sum.
 * One build per filter, so the sample and output arrays stay in registers. */
template <int N, int N2, int LOG2N>
AV1B_DEV void deblock_wide(px_t* b, int s, int maxv) {
  int v[2 * N + 2];
#pragma unroll
  for (int k = -(N + 1); k <= N; ++k) v[k + N + 1] = b[(2 + k) * s];
  int out[2 * N];
#pragma unroll
  for (int i = -N; i < N; ++i) {
    int t = 0;
#pragma unroll
    for (int j = -N; j <= N; ++j) {
      const int tap = clampi(i + j, -(N + 1), N);
      t += v[tap + N + 1] * (absi(j) <= N2 ? 2 : 1);
    }
    out[i + N] = rnd2(t, LOG2N);
  }
#pragma unroll
  for (int i = -N; i < N; ++i) b[(2 + i) * s] = (px_t)clampi(out[i + N], 0, maxv);
}

AV1B_DEV void deblock_px(px_t* b, int s, int level, int sharpness, int filter_size, int chroma,
                         int bd, int maxv) {
  if (level == 0) return;
  const int shift = bd - 8;
  const int mid = 0x80 << shift;
  const int p1 = b[0], p0 = b[s], q0 = b[2 * s], q1 = b[3 * s];
  const int flen = filter_size == 4 ? 4 : (chroma ? 6 : (filter_size == 8 ? 8 : 16));
  const int sh = sharpness > 4 ? 2 : (sharpness > 0 ? 1 : 0);
  int limit = level >> sh;
  if (limit < 1) limit = 1;
  if (sharpness > 0 && limit > 9 - sharpness) limit = 9 - sharpness;
  const int blimit = 2 * (level + 2) + limit;
  const int thresh = level >> 4;
  const int lim = limit << shift, blim = blimit << shift, thr = thresh << shift, flat = 1 << shift;
  const bool hev = absi(p1 - p0) > thr || absi(q1 - q0) > thr;
  bool bad = absi(p1 - p0) > lim || absi(q1 - q0) > lim ||
             absi(p0 - q0) * 2 + absi(p1 - q1) / 2 > blim;
  if (flen >= 6) {
    const int p2 = b[-s], q2 = b[4 * s];
    bad = bad || absi(p2 - p1) > lim || absi(q2 - q1) > lim;
  }
  if (flen >= 8) {
    const int p3 = b[-2 * s], q3 = b[5 * s];
    bad = bad || absi(p3 - (int)b[-s]) > lim || absi(q3 - (int)b[4 * s]) > lim;
  }
  if (bad) return;
  bool flat1 = true, flat2 = true;
  if (filter_size >= 8) {
    bool m = absi(p1 - p0) > flat || absi(q1 - q0) > flat || absi((int)b[-s] - p0) > flat ||
             absi((int)b[4 * s] - q0) > flat;
    if (flen >= 8) m = m || absi((int)b[-2 * s] - p0) > flat || absi((int)b[5 * s] - q0) > flat;
    flat1 = !m;
  }
  if (filter_size >= 16) {
    const bool m = absi((int)b[-5 * s] - p0) > flat || absi((int)b[8 * s] - q0) > flat ||
                   absi((int)b[-4 * s] - p0) > flat || absi((int)b[7 * s] - q0) > flat ||
                   absi((int)b[-3 * s] - p0) > flat || absi((int)b[6 * s] - q0) > flat;
    flat2 = !m;
  }
  if (filter_size == 4 || !flat1) {
    const int ps1 = p1 - mid, ps0 = p0 - mid, qs0 = q0 - mid, qs1 = q1 - mid;
    int f = hev ? f4clamp(ps1 - qs1, bd) : 0;
    f = f4clamp(f + 3 * (qs0 - ps0), bd);
    const int f1 = f4clamp(f + 4, bd) >> 3;
    const int f2 = f4clamp(f + 3, bd) >> 3;
    b[2 * s] = (px_t)clampi(f4clamp(qs0 - f1, bd) + mid, 0, maxv);
    b[s] = (px_t)clampi(f4clamp(ps0 + f2, bd) + mid, 0, maxv);
    if (!hev) {
      const int f3 = rnd2(f1, 1);
      b[3 * s] = (px_t)clampi(f4clamp(qs1 - f3, bd) + mid, 0, maxv);
      b[0] = (px_t)clampi(f4clamp(ps1 + f3, bd) + mid, 0, maxv);
    }
    return;
  }
  /* log2n 4: n 6, n2 1; log2n 3: n 2, n2 1 (chroma) or n 3, n2 0 (luma) */
  const int log2n = (filter_size == 8 || !flat2) ? 3 : 4;
  if (log2n == 4) deblock_wide<6, 1, 4>(b, s, maxv);
  else if (chroma) deblock_wide<2, 1, 3>(b, s, maxv);
  else deblock_wide<3, 0, 3>(b, s, maxv);
}

/* ---- CDEF -------------------------------------------------------------------- */
struct CdefRec {
  short x, y;                 /* plane samples */
  unsigned char plane, pri, sec, damping;
  signed char dir, pad0, pad1, pad2;
  int search;                 /* direction search result to use when dir < 0 */
};

AV1B_DEV int cdef_constrain(int diff, int threshold, int damping) {
  if (!threshold) return 0;
  const int adj = maxi(0, damping - floor_log2(threshold));
  const int mag = absi(diff);
  const int m = clampi(threshold - (mag >> adj), 0, mag);
  return diff < 0 ? -m : m;
}

/* ---- superres ------------------------------------------------------------------- */
AV1B_HD void superres_params(int down_w, int up_w, int* step, int* initial) {
  const int s = ((down_w << 14) + (up_w / 2)) / up_w;
  const int err = up_w * s - (down_w << 14);
  const int sub = (-((up_w - down_w) << 13) + (up_w / 2)) / up_w + (1 << 7) - err / 2;
  *step = s;
  *initial = sub & ((1 << 14) - 1);
}

/* ---- loop restoration --------------------------------------------------------------- */
struct LrUnitRec {
  int type;                     /* 1 Wiener, 2 self guided */
  int vf[3], hf[3];             /* Wiener coded coefficients */
  int r[2], e[2], xqd[2];       /* self guided */
};

/* ---- film grain ------------------------------------------------------------------ */

/* The frame's grain state on the device: templates, per-plane constants and
 * the scaling tables. */
struct GrainState {
  short luma[73 * 82];
  short cb[73 * 82];      /* chroma templates are chroma_w x chroma_h: 44x38 at */
  short cr[73 * 82];      /* 4:2:0, up to 82x73 at 4:4:4                        */
  int lut[3][256];
  int seed;
  int bitdepth, overlap, scaling_shift;
  int num_points[3];
  int chroma_from_luma;
  int mult[3], luma_mult[3], offset[3];
  int min_value, max_luma, max_chroma;
  int chroma_w, chroma_h;
};

/* get_random_number's 16-bit LFSR has period 65535 over the non-zero states,
 * so the state after n steps from s is orbit[(pos[s] + n) mod 65535]. */
AV1B_DEV int lfsr_after(const uint16_t* orbit, const uint16_t* pos, unsigned state, unsigned n) {
  if (state == 0) return 0;
  return orbit[(pos[state] + n) % 65535u];
}

AV1B_DEV int grain_scale_lut(const int* lut, int index, int bd) {
  const int shift = bd - 8;
  const int x = shift > 0 ? (index >> shift) : index;
  if (bd == 8 || x >= 255) return lut[x > 255 ? 255 : x];
  const int rem = index - (x << shift);
  const int a = lut[x], b = lut[x + 1];
  return a + rnd2z((b - a) * rem, shift);
}

/* ---- output ------------------------------------------------------------------------- */
AV1B_HD size_t nv12_bytes(int w, int h, int ss_x, int ss_y, size_t pitch) {
  if (w <= 0 || h <= 0) return 0;
  if (ss_x != 1 || ss_y != 1) return 0;
  const size_t crow = 2 * ((static_cast<size_t>(w) + 1) / 2);
  if ((pitch & 1) != 0 || pitch < crow) return 0;
  return pitch * (static_cast<size_t>(h) + (static_cast<size_t>(h) + 1) / 2);
}

}  // namespace av1b

#endif
