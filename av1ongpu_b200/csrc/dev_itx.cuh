/*
 * dev_itx.cuh - the AV1 inverse transforms (specification 7.13.2-7.13.3).
 *
 * The 1-D transforms are the specification's butterfly networks: a bit exact
 * decoder has to perform the same rotations (B) and clipped Hadamard steps
 * (H) in the same order, because each rounds. The step lists below follow
 * the specification's inverse DCT / ADST array processes; they are the same
 * steps the reference's av1g_idct / av1g_adst8 / av1g_adst16 take
 * (av1gpu_kernels.h:521-790), written here as compile-time unrolled loops over
 * a register array: every index is a constant after unrolling, so a 64-point
 * row lives in 64 registers and never touches local memory.
 *
 * Products are formed in 64 bits and rounded back (Round2(x, 12)), which is
 * what the reference does (av1gpu_kernels.h:495-508) so that an out-of-range
 * coefficient gives the same wrapped result on every backend.
 *
 * The 2-D transform of one block is done by one warp: lanes take rows for the
 * first pass (results to shared memory, clamped to the column range) and
 * columns for the second, which adds the residual to the prediction with the
 * flips applied at the add (av1gpu_kernels.h:869-930).
 */
#ifndef AV1B_DEV_ITX_CUH
#define AV1B_DEV_ITX_CUH

#include "dev_common.cuh"

namespace av1b {

AV1B_DEV int cos128(int angle) {
  const int a = angle & 255;
  if (a <= 64) return kCos128[a];
  if (a <= 128) return -kCos128[128 - a];
  if (a <= 192) return -kCos128[a - 128];
  return kCos128[256 - a];
}
AV1B_DEV int sin128(int angle) { return cos128(angle - 64); }

AV1B_HD constexpr int brev(int bits, int x) {
  int r = 0;
  for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1) << (bits - 1 - i);
  return r;
}

/* B(a, b, angle, flip) */
template <int N>
AV1B_DEV void rot(int (&t)[N], int a, int b, int angle, bool flip) {
  const long long c = cos128(angle), s = sin128(angle);
  const long long ta = t[a], tb = t[b];
  const int x = rnd2ll(ta * c - tb * s, 12);
  const int y = rnd2ll(ta * s + tb * c, 12);
  t[a] = flip ? y : x;
  t[b] = flip ? x : y;
}

/* H(a, b, flip, r): sum and difference clipped to r bits; with flip the
 * difference is b - a and lands in a. */
template <int N>
AV1B_DEV void had(int (&t)[N], int a, int b, bool flip, int lo, int hi) {
  const int x = t[a], y = t[b];
  const int sum = clampi(x + y, lo, hi);
  const int dif = clampi(flip ? y - x : x - y, lo, hi);
  t[a] = flip ? dif : sum;
  t[b] = flip ? sum : dif;
}

/* Inverse DCT array process for 2^n points, n = 2..6. */
template <int n, int N>
AV1B_DEV void idct(int (&t)[N], int lo, int hi) {
  constexpr int L = 1 << n;
  {
    int c[L];
#pragma unroll
    for (int i = 0; i < L; ++i) c[i] = t[brev(n, i)];
#pragma unroll
    for (int i = 0; i < L; ++i) t[i] = c[i];
  }
  if constexpr (n == 6) {
#pragma unroll
    for (int i = 0; i < 16; ++i) rot(t, 32 + i, 63 - i, 63 - 4 * brev(4, i), false);
  }
  if constexpr (n >= 5) {
#pragma unroll
    for (int i = 0; i < 8; ++i) rot(t, 16 + i, 31 - i, 6 + (brev(3, 7 - i) << 3), false);
  }
  if constexpr (n == 6) {
#pragma unroll
    for (int i = 0; i < 16; ++i) had(t, 32 + i * 2, 33 + i * 2, i & 1, lo, hi);
  }
  if constexpr (n >= 4) {
#pragma unroll
    for (int i = 0; i < 4; ++i) rot(t, 8 + i, 15 - i, 12 + (brev(2, 3 - i) << 4), false);
  }
  if constexpr (n >= 5) {
#pragma unroll
    for (int i = 0; i < 8; ++i) had(t, 16 + 2 * i, 17 + 2 * i, i & 1, lo, hi);
  }
  if constexpr (n == 6) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j)
        rot(t, 62 - i * 4 - j, 33 + i * 4 + j, 60 - 16 * brev(2, i) + 64 * j, true);
  }
  if constexpr (n >= 3) {
#pragma unroll
    for (int i = 0; i < 2; ++i) rot(t, 4 + i, 7 - i, 56 - 32 * i, false);
  }
  if constexpr (n >= 4) {
#pragma unroll
    for (int i = 0; i < 4; ++i) had(t, 8 + 2 * i, 9 + 2 * i, i & 1, lo, hi);
  }
  if constexpr (n >= 5) {
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j)
        rot(t, 30 - 4 * i - j, 17 + 4 * i + j, 24 + (j << 6) + ((1 - i) << 5), true);
  }
  if constexpr (n == 6) {
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) had(t, 32 + i * 4 + j, 35 + i * 4 - j, i & 1, lo, hi);
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) rot(t, 2 * i, 2 * i + 1, 32 + 16 * i, i == 0);
  if constexpr (n >= 3) {
#pragma unroll
    for (int i = 0; i < 2; ++i) had(t, 4 + 2 * i, 5 + 2 * i, i, lo, hi);
  }
  if constexpr (n >= 4) {
#pragma unroll
    for (int i = 0; i < 2; ++i) rot(t, 14 - i, 9 + i, 48 + 64 * i, true);
  }
  if constexpr (n >= 5) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) had(t, 16 + 4 * i + j, 19 + 4 * i - j, i & 1, lo, hi);
  }
  if constexpr (n == 6) {
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
        rot(t, 61 - i * 8 - j, 34 + i * 8 + j, 56 - i * 32 + (j >> 1) * 64, true);
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) had(t, i, 3 - i, false, lo, hi);
  if constexpr (n >= 3) rot(t, 6, 5, 32, true);
  if constexpr (n >= 4) {
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) had(t, 8 + 4 * i + j, 11 + 4 * i - j, i, lo, hi);
  }
  if constexpr (n >= 5) {
#pragma unroll
    for (int i = 0; i < 4; ++i) rot(t, 29 - i, 18 + i, 48 + (i >> 1) * 64, true);
  }
  if constexpr (n == 6) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) had(t, 32 + 8 * i + j, 39 + 8 * i - j, i & 1, lo, hi);
  }
  if constexpr (n >= 3) {
#pragma unroll
    for (int i = 0; i < 4; ++i) had(t, i, 7 - i, false, lo, hi);
  }
  if constexpr (n >= 4) {
#pragma unroll
    for (int i = 0; i < 2; ++i) rot(t, 13 - i, 10 + i, 32, true);
  }
  if constexpr (n >= 5) {
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) had(t, 16 + i * 8 + j, 23 + i * 8 - j, i, lo, hi);
  }
  if constexpr (n == 6) {
#pragma unroll
    for (int i = 0; i < 8; ++i) rot(t, 59 - i, 36 + i, i < 4 ? 48 : 112, true);
  }
  if constexpr (n >= 4) {
#pragma unroll
    for (int i = 0; i < 8; ++i) had(t, i, 15 - i, false, lo, hi);
  }
  if constexpr (n >= 5) {
#pragma unroll
    for (int i = 0; i < 4; ++i) rot(t, 27 - i, 20 + i, 32, true);
  }
  if constexpr (n == 6) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      had(t, 32 + i, 47 - i, false, lo, hi);
      had(t, 48 + i, 63 - i, true, lo, hi);
    }
  }
  if constexpr (n >= 5) {
#pragma unroll
    for (int i = 0; i < 16; ++i) had(t, i, 31 - i, false, lo, hi);
  }
  if constexpr (n == 6) {
#pragma unroll
    for (int i = 0; i < 8; ++i) rot(t, 55 - i, 40 + i, 32, true);
#pragma unroll
    for (int i = 0; i < 32; ++i) had(t, i, 63 - i, false, lo, hi);
  }
}

/* ADST input permutation: even outputs take the mirrored inputs. */
template <int n, int N>
AV1B_DEV void adst_in(int (&t)[N]) {
  constexpr int L = 1 << n;
  int c[L];
#pragma unroll
  for (int i = 0; i < L; ++i) c[i] = t[(i & 1) ? (i - 1) : (L - i - 1)];
#pragma unroll
  for (int i = 0; i < L; ++i) t[i] = c[i];
}

/* ADST output permutation (a Gray-code reordering) with alternating signs. */
template <int n, int N>
AV1B_DEV void adst_out(int (&t)[N]) {
  constexpr int L = 1 << n;
  int c[L];
#pragma unroll
  for (int i = 0; i < L; ++i) c[i] = t[i];
#pragma unroll
  for (int i = 0; i < L; ++i) {
    const int a = (i >> 3) & 1;
    const int b = ((i >> 2) & 1) ^ ((i >> 3) & 1);
    const int cc = ((i >> 1) & 1) ^ ((i >> 2) & 1);
    const int d = (i & 1) ^ ((i >> 1) & 1);
    const int idx = ((d << 3) | (cc << 2) | (b << 1) | a) >> (4 - n);
    t[i] = (i & 1) ? -c[idx] : c[idx];
  }
}

template <int N>
AV1B_DEV void adst4(int (&t)[N]) {
  const long long s0a = (long long)AV1B_SINPI_1_9 * t[0];
  const long long s1a = (long long)AV1B_SINPI_2_9 * t[0];
  const long long s2a = (long long)AV1B_SINPI_3_9 * t[1];
  const long long s3a = (long long)AV1B_SINPI_4_9 * t[2];
  const long long s4 = (long long)AV1B_SINPI_1_9 * t[2];
  const long long s5 = (long long)AV1B_SINPI_2_9 * t[3];
  const long long s6 = (long long)AV1B_SINPI_4_9 * t[3];
  const int a7 = t[0] - t[2];
  const int b7 = a7 + t[3];
  const long long s0 = s0a + s3a + s5;
  const long long s1 = s1a - s4 - s6;
  const long long s3 = s2a;
  const long long s2 = (long long)AV1B_SINPI_3_9 * b7;
  t[0] = rnd2ll(s0 + s3, 12);
  t[1] = rnd2ll(s1 + s3, 12);
  t[2] = rnd2ll(s2, 12);
  t[3] = rnd2ll(s0 + s1 - s3, 12);
}

template <int N>
AV1B_DEV void adst8(int (&t)[N], int lo, int hi) {
  adst_in<3>(t);
#pragma unroll
  for (int i = 0; i < 4; ++i) rot(t, 2 * i, 2 * i + 1, 60 - 16 * i, true);
#pragma unroll
  for (int i = 0; i < 4; ++i) had(t, i, 4 + i, false, lo, hi);
#pragma unroll
  for (int i = 0; i < 2; ++i) rot(t, 4 + 3 * i, 5 + i, 48 - 32 * i, true);
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) had(t, 4 * j + i, 2 + 4 * j + i, false, lo, hi);
#pragma unroll
  for (int i = 0; i < 2; ++i) rot(t, 2 + 4 * i, 3 + 4 * i, 32, true);
  adst_out<3>(t);
}

template <int N>
AV1B_DEV void adst16(int (&t)[N], int lo, int hi) {
  adst_in<4>(t);
#pragma unroll
  for (int i = 0; i < 8; ++i) rot(t, 2 * i, 2 * i + 1, 62 - 8 * i, true);
#pragma unroll
  for (int i = 0; i < 8; ++i) had(t, i, 8 + i, false, lo, hi);
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    rot(t, 8 + 2 * i, 9 + 2 * i, 56 - 32 * i, true);
    rot(t, 13 + 2 * i, 12 + 2 * i, 8 + 32 * i, true);
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) had(t, 8 * j + i, 4 + 8 * j + i, false, lo, hi);
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) rot(t, 4 + 8 * j + 3 * i, 5 + 8 * j + i, 48 - 32 * i, true);
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) had(t, 4 * j + i, 2 + 4 * j + i, false, lo, hi);
#pragma unroll
  for (int i = 0; i < 4; ++i) rot(t, 2 + 4 * i, 3 + 4 * i, 32, true);
  adst_out<4>(t);
}

/* The identity transforms rescale to the Q12 convention of the others. */
template <int n, int N>
AV1B_DEV void iidentity(int (&t)[N]) {
  constexpr int L = 1 << n;
#pragma unroll
  for (int i = 0; i < L; ++i) {
    if constexpr (n == 2) t[i] = rnd2ll((long long)t[i] * 5793, 12);
    else if constexpr (n == 3) t[i] = t[i] * 2;
    else if constexpr (n == 4) t[i] = rnd2ll((long long)t[i] * 11586, 12);
    else t[i] = t[i] * 4;
  }
}

/* Inverse Walsh-Hadamard (lossless), in place on t[0..3]. */
template <int N>
AV1B_DEV void iwht4(int (&t)[N], int shift) {
  int a = t[0] >> shift, c = t[1] >> shift, d = t[2] >> shift, b = t[3] >> shift;
  a += c;
  d -= b;
  const int e = (a - d) >> 1;
  b = e - b;
  c = e - c;
  a -= b;
  d += c;
  t[0] = a;
  t[1] = b;
  t[2] = c;
  t[3] = d;
}

/* 1-D kinds */
enum : int { kTxDct = 0, kTxAdst = 1, kTxIdtx = 2 };

/* Per transform type: column kind, row kind, flip up-down, flip left-right.
 * The first name of a type is the vertical (column) transform. */
AV1B_HD int tx_col_kind(int type) {
  /* DCT_*: 0 2 5 10; ADST-like: 1 3 4 6 7 8 12 14; identity: 9 11 13 15 */
  const unsigned dct = (1u << 0) | (1u << 2) | (1u << 5) | (1u << 10);
  const unsigned adst = (1u << 1) | (1u << 3) | (1u << 4) | (1u << 6) | (1u << 7) | (1u << 8) |
                        (1u << 12) | (1u << 14);
  return (dct >> type) & 1 ? kTxDct : ((adst >> type) & 1 ? kTxAdst : kTxIdtx);
}
AV1B_HD int tx_row_kind(int type) {
  const unsigned dct = (1u << 0) | (1u << 1) | (1u << 4) | (1u << 11);
  const unsigned adst = (1u << 2) | (1u << 3) | (1u << 5) | (1u << 6) | (1u << 7) | (1u << 8) |
                        (1u << 13) | (1u << 15);
  return (dct >> type) & 1 ? kTxDct : ((adst >> type) & 1 ? kTxAdst : kTxIdtx);
}
AV1B_HD bool tx_flip_ud(int type) { return type == 4 || type == 6 || type == 8 || type == 14; }
AV1B_HD bool tx_flip_lr(int type) { return type == 5 || type == 6 || type == 7 || type == 15; }

/* Transform_Row_Shift for a w x h transform (log2 sizes). */
AV1B_HD int tx_row_shift(int lw, int lh) {
  /* 4x4 0, 8x8 1, 16x16 2, 32x32 2, 64x64 2, 4x8 0, 8x4 0, 8x16 1, 16x8 1,
   * 16x32 1, 32x16 1, 32x64 1, 64x32 1, 4x16 1, 16x4 1, 8x32 2, 32x8 2,
   * 16x64 2, 64x16 2 */
  const int key = lw * 8 + lh;
  switch (key) {
    case 2 * 8 + 2: return 0;
    case 3 * 8 + 3: return 1;
    case 4 * 8 + 4: case 5 * 8 + 5: case 6 * 8 + 6: return 2;
    case 2 * 8 + 3: case 3 * 8 + 2: return 0;
    case 3 * 8 + 4: case 4 * 8 + 3: return 1;
    case 4 * 8 + 5: case 5 * 8 + 4: return 1;
    case 5 * 8 + 6: case 6 * 8 + 5: return 1;
    case 2 * 8 + 4: case 4 * 8 + 2: return 1;
    case 3 * 8 + 5: case 5 * 8 + 3: return 2;
    case 4 * 8 + 6: case 6 * 8 + 4: return 2;
    default: return 0;
  }
}

template <int n, int N>
AV1B_DEV void tx1d(int (&t)[N], int kind, int lo, int hi) {
  if (kind == kTxDct) {
    idct<n>(t, lo, hi);
  } else if (kind == kTxAdst) {
    if constexpr (n == 2) adst4(t);
    else if constexpr (n == 3) adst8(t, lo, hi);
    else adst16(t, lo, hi); /* the reference runs 16 points for every n >= 4 */
  } else {
    iidentity<n < 5 ? n : 5>(t); /* and scales 32 points by 4 for every n >= 5 */
  }
}

/* ---- the two passes --------------------------------------------------------- */

/* Parameters of one 2-D transform. */
struct ItxParams {
  int lw, lh;       /* log2 sizes */
  int type;
  int lossless;
  int row_shift;
  int bitdepth;
};

/* Pass 1 for row `y`: coefficients (raster, min(w,32) wide, rows >= 32 are
 * zero) -> tmp[y * w + j], clamped to the column range. */
template <int LW>
AV1B_DEV void itx_row(const ItxParams& p, const int* __restrict__ coef, int y, int* tmp) {
  constexpr int W = 1 << LW;
  constexpr int CS = W < 32 ? W : 32;
  int t[W];
  const int col_bits = maxi(p.bitdepth + 6, 16);
  const int clo = -(1 << (col_bits - 1)), chi = (1 << (col_bits - 1)) - 1;
  if (y >= 32) {
#pragma unroll
    for (int j = 0; j < W; ++j) tmp[y * W + j] = 0;
    return;
  }
  const int* row = coef + y * CS;
  if ((reinterpret_cast<uintptr_t>(row) & 15) == 0) {
    /* a 16-byte aligned row (every row of a raster that starts aligned):
     * four coefficients a load */
#pragma unroll
    for (int j = 0; j < CS; j += 4) {
      const int4 v = *reinterpret_cast<const int4*>(row + j);
      t[j] = v.x;
      t[j + 1] = v.y;
      t[j + 2] = v.z;
      t[j + 3] = v.w;
    }
#pragma unroll
    for (int j = CS; j < W; ++j) t[j] = 0;
  } else {
#pragma unroll
    for (int j = 0; j < W; ++j) t[j] = j < CS ? row[j] : 0;
  }
  if (absi(LW - p.lh) == 1) {
#pragma unroll
    for (int j = 0; j < W; ++j) t[j] = rnd2ll((long long)t[j] * 2896, 12);
  }
  if (p.lossless) {
    if constexpr (LW == 2) iwht4(t, 2);
  } else {
    const int rb = p.bitdepth + 8;
    tx1d<LW>(t, tx_row_kind(p.type), -(1 << (rb - 1)), (1 << (rb - 1)) - 1);
  }
#pragma unroll
  for (int j = 0; j < W; ++j) {
    const int r = p.lossless ? t[j] : rnd2z(t[j], p.row_shift);
    tmp[y * W + j] = clampi(r, clo, chi);
  }
}

/* Pass 2 for column `x`: tmp -> residual, added to dst with the flips. */
template <int LH, bool CG>
AV1B_DEV void itx_col_add(const ItxParams& p, const int* tmp, int x, px_t* dst, int stride,
                          int maxv, int* res = nullptr) {
  constexpr int H = 1 << LH;
  const int W = 1 << p.lw;
  int t[H];
#pragma unroll
  for (int i = 0; i < H; ++i) t[i] = tmp[i * W + x];
  if (p.lossless) {
    if constexpr (LH == 2) iwht4(t, 0);
  } else {
    const int cb = maxi(p.bitdepth + 6, 16);
    tx1d<LH>(t, tx_col_kind(p.type), -(1 << (cb - 1)), (1 << (cb - 1)) - 1);
  }
  const bool fud = tx_flip_ud(p.type), flr = tx_flip_lr(p.type);
  const int xx = flr ? W - 1 - x : x;
#pragma unroll
  for (int i = 0; i < H; ++i) {
    const int r = p.lossless ? t[i] : rnd2(t[i], 4);
    const int yy = fud ? H - 1 - i : i;
    if (res) {
      res[yy * W + xx] = r;
      continue;
    }
    px_t* q = dst + yy * stride + xx;
    const int old = CG ? (int)__ldcg(q) : (int)*q;
    *q = (px_t)clampi(old + r, 0, maxv);
  }
}

AV1B_DEV void itx_row_dispatch(const ItxParams& p, const int* coef, int y, int* tmp) {
  switch (p.lw) {
    case 2: itx_row<2>(p, coef, y, tmp); break;
    case 3: itx_row<3>(p, coef, y, tmp); break;
    case 4: itx_row<4>(p, coef, y, tmp); break;
    case 5: itx_row<5>(p, coef, y, tmp); break;
    default: itx_row<6>(p, coef, y, tmp); break;
  }
}

template <bool CG>
AV1B_DEV void itx_col_dispatch(const ItxParams& p, const int* tmp, int x, px_t* dst, int stride,
                               int maxv, int* res = nullptr) {
  switch (p.lh) {
    case 2: itx_col_add<2, CG>(p, tmp, x, dst, stride, maxv, res); break;
    case 3: itx_col_add<3, CG>(p, tmp, x, dst, stride, maxv, res); break;
    case 4: itx_col_add<4, CG>(p, tmp, x, dst, stride, maxv, res); break;
    case 5: itx_col_add<5, CG>(p, tmp, x, dst, stride, maxv, res); break;
    default: itx_col_add<6, CG>(p, tmp, x, dst, stride, maxv, res); break;
  }
}

/* The whole 2-D transform + add, by one warp. `tmp` is warp-private shared
 * memory of at least w * h ints; `dst` is the block's top-left sample. CG:
 * read the prediction back through L2 (the dependency-scheduled kernel, where
 * neighbouring samples are written by other SMs). */
template <bool CG>
AV1B_DEV void itx_warp(const ItxParams& p, const int* __restrict__ coef, int* tmp, px_t* dst,
                       int stride, int maxv, int lane) {
  const int w = 1 << p.lw, h = 1 << p.lh;
  for (int y = lane; y < h; y += 32) itx_row_dispatch(p, coef, y, tmp);
  __syncwarp();
  for (int x = lane; x < w; x += 32) itx_col_dispatch<CG>(p, tmp, x, dst, stride, maxv);
  __syncwarp();
}

/* One transform by a group of `step` lanes of a warp (`sub`: this lane's
 * index in the group), several groups - several transforms of one size class
 * - per warp. Every lane of the warp takes both barriers, active or not.
 * `res` non-null: the residual goes there (w * h, row-major) instead of into
 * the picture. */
template <bool CG>
AV1B_DEV void itx_group(const ItxParams& p, const int* __restrict__ coef, int* tmp, px_t* dst,
                        int stride, int maxv, int* res, int sub, int step, bool active) {
  const int w = 1 << p.lw, h = 1 << p.lh;
  if (active)
    for (int y = sub; y < h; y += step) itx_row_dispatch(p, coef, y, tmp);
  __syncwarp();
  if (active)
    for (int x = sub; x < w; x += step) itx_col_dispatch<CG>(p, tmp, x, dst, stride, maxv, res);
  __syncwarp();
}

/* The same for transforms whose longer side is 1 << CLS: only the three
 * lengths that class holds (CLS - 2 .. CLS, the 4:1 shapes included) are
 * instantiated, so a kernel for the small classes is not sized for the
 * 64-point transforms' registers. */
template <int LO, int HI>
AV1B_DEV void itx_row_range(const ItxParams& p, const int* coef, int y, int* tmp) {
  if constexpr (LO < HI) {
    if (p.lw == LO) {
      itx_row<LO>(p, coef, y, tmp);
      return;
    }
    itx_row_range<LO + 1, HI>(p, coef, y, tmp);
  } else {
    itx_row<HI>(p, coef, y, tmp);
  }
}

template <int LO, int HI, bool CG>
AV1B_DEV void itx_col_range(const ItxParams& p, const int* tmp, int x, px_t* dst, int stride, int maxv,
                            int* res) {
  if constexpr (LO < HI) {
    if (p.lh == LO) {
      itx_col_add<LO, CG>(p, tmp, x, dst, stride, maxv, res);
      return;
    }
    itx_col_range<LO + 1, HI, CG>(p, tmp, x, dst, stride, maxv, res);
  } else {
    itx_col_add<HI, CG>(p, tmp, x, dst, stride, maxv, res);
  }
}

template <int CLS, bool CG>
AV1B_DEV void itx_group_cls(const ItxParams& p, const int* __restrict__ coef, int* tmp, px_t* dst,
                            int stride, int maxv, int* res, int sub, int step, bool active) {
  constexpr int LO = CLS - 2 > 2 ? CLS - 2 : 2;
  const int w = 1 << p.lw, h = 1 << p.lh;
  if (active)
    for (int y = sub; y < h; y += step) itx_row_range<LO, CLS>(p, coef, y, tmp);
  __syncwarp();
  if (active)
    for (int x = sub; x < w; x += step) itx_col_range<LO, CLS, CG>(p, tmp, x, dst, stride, maxv, res);
  __syncwarp();
}

/* The 2-D transform alone: the residual (before the add and the clip) into
 * `res`, w * h row-major. */
AV1B_DEV void itx_warp_residual(const ItxParams& p, const int* __restrict__ coef, int* tmp, int* res,
                                int lane) {
  const int w = 1 << p.lw, h = 1 << p.lh;
  for (int y = lane; y < h; y += 32) itx_row_dispatch(p, coef, y, tmp);
  __syncwarp();
  for (int x = lane; x < w; x += 32) itx_col_dispatch<false>(p, tmp, x, nullptr, 0, 0, res);
  __syncwarp();
}

}  // namespace av1b

#endif
