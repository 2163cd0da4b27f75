/*
 * plan_host.cpp - host helpers of the frame planner (see plan_host.h).
 *
 * Each one restates a step of the reference's host tables code:
 *   gm_setup_shear     - src/core/tables.cpp:444-470 (spec 7.11.3.6/7.11.3.7)
 *   wedge_entry        - src/core/tables.cpp:578-616 (spec 7.11.3.11)
 *   grain_scaling_lut  - kernels/av1gpu_kernels.h:3157-3188 (spec 7.18.3.4)
 *   color_matrix       - src/core/tables.cpp:481-535
 */
#include "plan_host.h"

#include <cstdlib>

#include "av1b_tables.h"
#include "wedge.h"

namespace av1b {
namespace {

int floor_log2_host(int v) {
  int n = 0;
  while ((1 << (n + 1)) <= v) ++n;
  return n;
}

int round2_signed(int v, int n) {
  const int r = (1 << n) >> 1;
  return v >= 0 ? (v + r) >> n : -((-v + r) >> n);
}

long long round2_signed64(long long v, int n) {
  const long long r = 1LL << (n - 1);
  return v >= 0 ? (v + r) >> n : -((-v + r) >> n);
}

int clip16(long long v) { return v < -32768 ? -32768 : (v > 32767 ? 32767 : static_cast<int>(v)); }

}  // namespace

bool gm_setup_shear(const int32_t* m, int* alpha, int* beta, int* gamma, int* delta) {
  const int alpha0 = clip16(static_cast<long long>(m[2]) - 65536);
  const int beta0 = clip16(m[3]);
  /* resolve_divisor(m[2]): 1/d as a Q14 table entry and a shift */
  const int d = m[2];
  const int ad = d < 0 ? -d : d;
  const int n = floor_log2_host(ad);
  const int e = ad - (1 << n);
  const int f = n > 8 ? (e + (1 << ((n - 8) - 1))) >> (n - 8) : e << (8 - n);
  const int div_shift = n + 14;
  const long long div_factor = d < 0 ? -kDivLut[f] : kDivLut[f];
  const long long v = static_cast<long long>(m[4]) * 65536;
  const int gamma0 = clip16(round2_signed64(v * div_factor, div_shift));
  const long long w = static_cast<long long>(m[3]) * m[4];
  const int delta0 = clip16(static_cast<long long>(m[5]) - round2_signed64(w * div_factor, div_shift) - 65536);
  *alpha = round2_signed(alpha0, 6) * 64;
  *beta = round2_signed(beta0, 6) * 64;
  *gamma = round2_signed(gamma0, 6) * 64;
  *delta = round2_signed(delta0, 6) * 64;
  if (4 * std::abs(*alpha) + 7 * std::abs(*beta) >= 65536) return false;
  if (4 * std::abs(*gamma) + 4 * std::abs(*delta) >= 65536) return false;
  return true;
}

bool wedge_entry(int bw, int bh, int index, int* dir, int* xoff, int* yoff, int* flip) {
  if (index < 0 || index >= 16 || bw < 8 || bh < 8 || bw > 32 || bh > 32) return false;
  const int shape = bh > bw ? 0 : (bh < bw ? 1 : 2);
  const unsigned char* c = kWedgeCodebook + (shape * 16 + index) * 3;
  *dir = c[0];
  *xoff = 32 - ((c[1] * bw) >> 3);
  *yoff = 32 - ((c[2] * bh) >> 3);
  /* the sign is chosen from the mean of the first row and first column */
  int sum = 0;
  for (int i = 0; i < bw; ++i) sum += wedge_master(*dir, *yoff, *xoff + i);
  for (int i = 1; i < bh; ++i) sum += wedge_master(*dir, *yoff + i, *xoff);
  const int n = bw + bh - 1;
  *flip = ((sum + n / 2) / n) < 32 ? 1 : 0;
  return true;
}

void grain_scaling_lut(int num, const int32_t* value, const int32_t* scaling, int* lut) {
  if (num <= 0) {
    for (int x = 0; x < 256; ++x) lut[x] = 0;
    return;
  }
  for (int x = 0; x < value[0]; ++x) lut[x] = scaling[0];
  for (int i = 0; i + 1 < num; ++i) {
    const int dy = scaling[i + 1] - scaling[i];
    const int dx = value[i + 1] - value[i];
    const int delta = dy * ((65536 + (dx >> 1)) / dx);
    for (int x = 0; x < dx; ++x) lut[value[i] + x] = scaling[i] + ((x * delta + 32768) >> 16);
  }
  for (int x = value[num - 1]; x < 256; ++x) lut[x] = scaling[num - 1];
}

const short* sgr_params_table() { return kSgrParams; }

void color_matrix(int matrix, int range, int bd, int m[8], int o[3]) {
  const int shift = bd - 8;
  const int y_off = range == 0 ? (16 << shift) : 0;
  const int c_off = range == 0 ? (128 << shift) : (1 << (bd - 1));
  const int half = 1 << 15;
  for (int i = 0; i < 8; ++i) m[i] = 0;
  if (matrix == 3) { /* identity: the planes are G, B, R already */
    m[0] = 65536;
    m[2] = 65536;
    m[5] = 65536;
    o[0] = o[1] = o[2] = 0;
    return;
  }
  if (matrix == 2) { /* BT.2020 */
    m[0] = 76293; m[1] = 109969; m[2] = 76293; m[3] = -12255; m[4] = -42598; m[5] = 76293;
    m[6] = 121634;
  } else { /* BT.709, also used for BT.601 as the reference does */
    m[0] = 76293; m[1] = 117504; m[2] = 76293; m[3] = -13926; m[4] = -34937; m[5] = 76293;
    m[6] = 138412;
  }
  o[0] = half - m[0] * y_off - m[1] * c_off;
  o[1] = half - m[2] * y_off - m[3] * c_off - m[4] * c_off;
  o[2] = half - m[5] * y_off - m[6] * c_off;
}

}  // namespace av1b
