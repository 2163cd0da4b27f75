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
  const int log2n = (filter_size == 8 || !flat2) ? 3 : 4;
  const int n = log2n == 4 ? 6 : (chroma ? 2 : 3);
  const int n2 = (log2n == 3 && !chroma) ? 0 : 1;
  int v[14];
  for (int k = -(n + 1); k <= n; ++k) v[k + 7] = b[(2 + k) * s];
  int out[12];
  for (int i = -n; i < n; ++i) {
    int t = 0;
    for (int j = -n; j <= n; ++j) {
      const int tap = clampi(i + j, -(n + 1), n);
      t += v[tap + 7] * (absi(j) <= n2 ? 2 : 1);
    }
    out[i + n] = rnd2(t, log2n);
  }
  for (int i = -n; i < n; ++i) b[(2 + i) * s] = (px_t)clampi(out[i + n], 0, maxv);
}

/* ---- CDEF -------------------------------------------------------------------- */
struct CdefRec {
  short x, y;                 /* plane samples */
  unsigned char plane, pri, sec, damping;
  signed char dir, pad0, pad1, pad2;
};

AV1B_DEV void cdef_direction(const px_t* luma, int stride, int bd, int* dir_out, int* var_out) {
  int partial[8][15];
  int cost[8];
  for (int i = 0; i < 8; ++i) {
    cost[i] = 0;
    for (int j = 0; j < 15; ++j) partial[i][j] = 0;
  }
  const int shift = bd - 8;
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 8; ++j) {
      const int x = ((int)luma[i * stride + j] >> shift) - 128;
      partial[0][i + j] += x;
      partial[1][i + j / 2] += x;
      partial[2][i] += x;
      partial[3][3 + i - j / 2] += x;
      partial[4][7 + i - j] += x;
      partial[5][3 - i / 2 + j] += x;
      partial[6][j] += x;
      partial[7][i / 2 + j] += x;
    }
  const int div[9] = {0, 840, 420, 280, 210, 168, 140, 120, 105};
  for (int i = 0; i < 8; ++i) {
    cost[2] += partial[2][i] * partial[2][i];
    cost[6] += partial[6][i] * partial[6][i];
  }
  cost[2] *= div[8];
  cost[6] *= div[8];
  for (int i = 0; i < 7; ++i) {
    cost[0] += (partial[0][i] * partial[0][i] + partial[0][14 - i] * partial[0][14 - i]) * div[i + 1];
    cost[4] += (partial[4][i] * partial[4][i] + partial[4][14 - i] * partial[4][14 - i]) * div[i + 1];
  }
  cost[0] += partial[0][7] * partial[0][7] * div[8];
  cost[4] += partial[4][7] * partial[4][7] * div[8];
  for (int i = 1; i < 8; i += 2) {
    for (int j = 0; j < 5; ++j) cost[i] += partial[i][3 + j] * partial[i][3 + j];
    cost[i] *= div[8];
    for (int j = 0; j < 3; ++j)
      cost[i] += (partial[i][j] * partial[i][j] + partial[i][10 - j] * partial[i][10 - j]) *
                 div[2 * j + 2];
  }
  int best = 0, d = 0;
  for (int i = 0; i < 8; ++i)
    if (cost[i] > best) {
      best = cost[i];
      d = i;
    }
  *dir_out = d;
  *var_out = (best - cost[(d + 4) & 7]) >> 10;
}

AV1B_DEV int cdef_constrain(int diff, int threshold, int damping) {
  if (!threshold) return 0;
  const int adj = maxi(0, damping - floor_log2(threshold));
  const int mag = absi(diff);
  const int m = clampi(threshold - (mag >> adj), 0, mag);
  return diff < 0 ? -m : m;
}

/* Cdef_Directions: (dy, dx) of the first and second tap along each of the
 * eight directions. */
AV1B_DEV void cdef_dir_offsets(int dir, int k, int* dy, int* dx) {
  const signed char t[8][2][2] = {
      {{-1, 1}, {-2, 2}}, {{0, 1}, {-1, 2}}, {{0, 1}, {0, 2}}, {{0, 1}, {1, 2}},
      {{1, 1}, {2, 2}},   {{1, 0}, {2, 1}},  {{1, 0}, {2, 0}}, {{1, 0}, {2, -1}},
  };
  *dy = t[dir][k][0];
  *dx = t[dir][k][1];
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

struct LrSrc {
  const px_t* cdef;   /* plane origin of the CDEF (and superres) output */
  const px_t* curr;   /* plane origin of the deblocked picture (upscaled) */
  int stride;
  int w, h;           /* visible plane size */
  int s0, s1;         /* stripe rows, inclusive */
};

AV1B_DEV int lr_src(const LrSrc& s, int x, int y) {
  x = clampi(x, 0, s.w - 1);
  y = clampi(y, 0, s.h - 1);
  if (y < s.s0) return s.curr[maxi(y, s.s0 - 2) * s.stride + x];
  if (y > s.s1) return s.curr[mini(y, s.s1 + 2) * s.stride + x];
  return s.cdef[y * s.stride + x];
}

AV1B_DEV int lr_wiener(const LrSrc& s, const LrUnitRec& u, int bd, int x, int y) {
  const int r0 = bd == 12 ? 5 : 3, r1 = bd == 12 ? 9 : 11;
  const int offset = 1 << (bd + 7 - r0 - 1);
  const int limit = (1 << (bd + 1 + 7 - r0)) - 1;
  int vt[7], ht[7];
  for (int t = 0; t < 3; ++t) {
    vt[t] = vt[6 - t] = u.vf[t];
    ht[t] = ht[6 - t] = u.hf[t];
  }
  vt[3] = 128 - 2 * (u.vf[0] + u.vf[1] + u.vf[2]);
  ht[3] = 128 - 2 * (u.hf[0] + u.hf[1] + u.hf[2]);
  int sum = 0;
  for (int t = 0; t < 7; ++t) {
    int acc = 0;
    for (int k = 0; k < 7; ++k) acc += ht[k] * lr_src(s, x + k - 3, y + t - 3);
    sum += vt[t] * clampi(rnd2(acc, r0), -offset, limit - offset);
  }
  return rnd2(sum, r1);
}

/* A and B of the box filter centred on (x, y) (7.17.3). */
AV1B_DEV void sgr_ab(const LrSrc& s, int bd, int x, int y, int r, int eps, int* a_out, int* b_out) {
  const int n = (2 * r + 1) * (2 * r + 1);
  const long long n2e = (long long)n * n * eps;
  const long long mtable = ((1LL << 20) + n2e / 2) / n2e;
  long long sa = 0, sb = 0;
  for (int dy = -r; dy <= r; ++dy)
    for (int dx = -r; dx <= r; ++dx) {
      const int c = lr_src(s, x + dx, y + dy);
      sa += (long long)c * c;
      sb += c;
    }
  const long long b_sum = sb;
  sa = rnd2llz(sa, 2 * (bd - 8));
  sb = rnd2llz(sb, bd - 8);
  long long p = sa * n - sb * sb;
  if (p < 0) p = 0;
  const int z = rnd2ll(p * mtable, 20);
  int a2;
  if (z >= 255) a2 = 256;
  else if (z == 0) a2 = 1;
  else a2 = ((z << 8) + (z / 2)) / (z + 1);
  const int one_over_n = ((1 << 12) + (n / 2)) / n;
  const long long b2 = (long long)(256 - a2) * b_sum * one_over_n;
  *a_out = a2;
  *b_out = rnd2ll(b2, 12);
}

AV1B_DEV int lr_sgr(const LrSrc& s, const LrUnitRec& u, int bd, int x, int y) {
  const int v = lr_src(s, x, y);
  const int w0 = u.xqd[0], w1 = u.xqd[1], w2 = 128 - w0 - w1;
  int flt[2];
  for (int pass = 0; pass < 2; ++pass) {
    const int r = u.r[pass];
    if (r == 0) {
      flt[pass] = 0;
      continue;
    }
    int a = 0, b = 0;
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        int wgt;
        if (pass == 0) wgt = ((y + dy) & 1) ? (dx == 0 ? 6 : 5) : 0;
        else wgt = (dx == 0 || dy == 0) ? 4 : 3;
        if (!wgt) continue;
        int a2, b2;
        sgr_ab(s, bd, x + dx, y + dy, r, u.e[pass], &a2, &b2);
        a += wgt * a2;
        b += wgt * b2;
      }
    const int shift = (pass == 0 && (y & 1)) ? 4 : 5;
    flt[pass] = rnd2ll((long long)a * v + b, 8 + shift - 4);
  }
  const int us = v << 4;
  long long t = (long long)w1 * us;
  t += (long long)w0 * (u.r[0] ? flt[0] : us);
  t += (long long)w2 * (u.r[1] ? flt[1] : us);
  return rnd2ll(t, 4 + 7);
}

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
