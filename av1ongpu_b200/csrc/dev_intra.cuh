/*
 * dev_intra.cuh - intra prediction of one transform block by one warp
 * (specification 7.11.2).
 *
 * The reference predicts a row per thread and gathers and filters the whole
 * edge again in every thread (av1_cuda.cu:70-117). Here the warp gathers the
 * block's two edges once into shared memory, runs the edge filter and the
 * upsampler with one lane per edge sample, and then predicts the block with
 * one lane per output sample. The arithmetic of every step is the
 * reference's (av1gpu_kernels.h:1108-1677):
 *   - edge gather and the stand-in values for missing neighbours (1108-1151);
 *   - corner fix, edge filter strength and upsampling selection (1193-1239,
 *     1452-1481);
 *   - directional, smooth, Paeth, DC, recursive filter, palette and
 *     chroma-from-luma predictors (1245-1447, 1578-1677).
 * Reads of the picture being reconstructed go through L2 (ld.cg), because
 * another SM produced them and published them with a release flag.
 */
#ifndef AV1B_DEV_INTRA_CUH
#define AV1B_DEV_INTRA_CUH

#include "dev_common.cuh"

namespace av1b {

#define AV1B_EDGE_LEN 288
#define AV1B_EDGE_OFF 16

/* Everything the intra predictor needs for one block, resolved. */
struct IntraJob {
  int x, y, w, h;
  int mode, angle, bitdepth, maxv;
  int have_left, have_above, have_ar, have_bl;
  int filter_type;     /* -1: the sequence disables the intra edge filter */
  int filter_intra, fi_mode;
  int cfl_alpha;
  int max_x, max_y;
  int ss_x, ss_y;
  int palette, palette_off, palette_stride;
};


AV1B_DEV int edge_strength(int w, int h, int filter_type, int delta) {
  const int d = absi(delta);
  const int blk = w + h;
  int s = 0;
  if (filter_type == 0) {
    if (blk <= 8) {
      if (d >= 56) s = 1;
    } else if (blk <= 16) {
      if (d >= 40) s = 1;
    } else if (blk <= 24) {
      if (d >= 8) s = 1;
      if (d >= 16) s = 2;
      if (d >= 32) s = 3;
    } else if (blk <= 32) {
      s = 1;
      if (d >= 4) s = 2;
      if (d >= 32) s = 3;
    } else {
      s = 3;
    }
  } else {
    if (blk <= 8) {
      if (d >= 40) s = 1;
      if (d >= 64) s = 2;
    } else if (blk <= 16) {
      if (d >= 20) s = 1;
      if (d >= 48) s = 2;
    } else if (blk <= 24) {
      if (d >= 4) s = 3;
    } else {
      s = 3;
    }
  }
  return s;
}

AV1B_DEV int upsample_sel(int w, int h, int filter_type, int delta) {
  const int d = absi(delta);
  if (d <= 0 || d >= 40) return 0;
  return filter_type == 0 ? (w + h <= 16) : (w + h <= 8);
}

/* Gathers AboveRow[-1 .. w+h-1] and LeftCol[-1 .. w+h-1]. `p` is the block's
 * top-left sample in the plane. */
AV1B_DEV void intra_edges(const IntraJob& j, const px_t* p, int stride, int* above, int* left,
                          int lane) {
  const int n = j.w + j.h;
  const int mid = 1 << (j.bitdepth - 1);
  const int alimit = mini(j.max_x, j.x + (j.have_ar ? 2 * j.w : j.w) - 1);
  const int llimit = mini(j.max_y, j.y + (j.have_bl ? 2 * j.h : j.h) - 1);
  /* every load of the edges (at most 128 + 128 samples and the corner) is
   * issued before any is used: one round trip to L2, not one per sample */
  int a[4], l[4], c = mid;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int i = lane + 32 * q;
    a[q] = mid - 1;
    l[q] = mid + 1;
    if (i < n) {
      if (!j.have_above) a[q] = j.have_left ? ldpx(p - 1) : mid - 1;
      else a[q] = ldpx(p - stride + (mini(j.x + i, alimit) - j.x));
      if (!j.have_left) l[q] = j.have_above ? ldpx(p - stride) : mid + 1;
      else l[q] = ldpx(p + (mini(j.y + i, llimit) - j.y) * stride - 1);
    }
  }
  if (lane == 0) {
    if (j.have_above && j.have_left) c = ldpx(p - stride - 1);
    else if (j.have_above) c = ldpx(p - stride);
    else if (j.have_left) c = ldpx(p - 1);
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int i = lane + 32 * q;
    if (i < n) {
      above[i] = a[q];
      left[i] = l[q];
    }
  }
  if (lane == 0) {
    above[-1] = c;
    left[-1] = c;
  }
  __syncwarp();
}

/* The 5-tap intra edge filter over buf[-1 .. sz-2] (entry i-1 is edge sample
 * i; sample 0, the corner, is read but not written). */
AV1B_DEV void edge_filter(int* buf, int sz, int strength, int* tmp, int lane) {
  if (strength <= 0) return;
  for (int i = lane; i < sz; i += 32) tmp[i] = buf[i - 1];
  __syncwarp();
  const short* k = kEdgeKernel + (strength - 1) * 5;
  for (int i = 1 + lane; i < sz; i += 32) {
    int s = 0;
#pragma unroll
    for (int t = 0; t < 5; ++t) s += k[t] * tmp[clampi(i - 2 + t, 0, sz - 1)];
    buf[i - 1] = (s + 8) >> 4;
  }
  __syncwarp();
}

/* Doubles the edge resolution: buf[-2 .. 2*num-2]. */
AV1B_DEV void edge_upsample(int* buf, int num, int maxv, int* dup, int lane) {
  /* dup[k] = buf[k-2] for k = 1..num+1, with both ends repeated */
  for (int k = lane; k < num + 3; k += 32) {
    int v;
    if (k == 0) v = buf[-1];
    else if (k == num + 2) v = buf[num - 1];
    else v = buf[k - 2];
    dup[k] = v;
  }
  __syncwarp();
  if (lane == 0) buf[-2] = dup[0];
  for (int i = lane; i < num; i += 32) {
    int s = -dup[i] + 9 * dup[i + 1] + 9 * dup[i + 2] - dup[i + 3];
    buf[2 * i - 1] = clampi(rnd2(s, 4), 0, maxv);
    buf[2 * i] = dup[i + 2];
  }
  __syncwarp();
}

AV1B_DEV int warp_sum(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
AV1B_DEV long long warp_sum64(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

/* DC of whichever edges exist. */
AV1B_DEV int intra_dc(const IntraJob& j, const int* above, const int* left, int lane) {
  int s = 0;
  if (j.have_above)
    for (int k = lane; k < j.w; k += 32) s += above[k];
  if (j.have_left)
    for (int k = lane; k < j.h; k += 32) s += left[k];
  s = warp_sum(s);
  if (j.have_above && j.have_left) return (s + ((j.w + j.h) >> 1)) / (j.w + j.h);
  if (j.have_left) return (s + (j.h >> 1)) >> ilog2(j.h);
  if (j.have_above) return (s + (j.w >> 1)) >> ilog2(j.w);
  return 1 << (j.bitdepth - 1);
}

/* One directional sample (the reference's av1g_intra_directional_row). */
AV1B_DEV int dir_sample(const int* above, const int* left, int w, int h, int pangle, int dx,
                        int dy, int ua, int ul, int i, int jj) {
  if (pangle < 90) {
    const int max_base = (w + h - 1) << ua;
    const int idx = (i + 1) * dx;
    const int base = (idx >> (6 - ua)) + (jj << ua);
    const int shift = ((idx << ua) >> 1) & 0x1F;
    if (base < max_base) return rnd2(above[base] * (32 - shift) + above[base + 1] * shift, 5);
    return above[max_base];
  }
  if (pangle > 90 && pangle < 180) {
    int idx = (jj << 6) - (i + 1) * dx;
    int base = idx >> (6 - ua);
    if (base >= -(1 << ua)) {
      const int shift = ((idx * (1 << ua)) >> 1) & 0x1F;
      return rnd2(above[base] * (32 - shift) + above[base + 1] * shift, 5);
    }
    idx = (i << 6) - (jj + 1) * dy;
    base = idx >> (6 - ul);
    const int shift = ((idx * (1 << ul)) >> 1) & 0x1F;
    return rnd2(left[base] * (32 - shift) + left[base + 1] * shift, 5);
  }
  if (pangle > 180) {
    const int idx = (jj + 1) * dy;
    const int base = (idx >> (6 - ul)) + (i << ul);
    const int shift = ((idx << ul) >> 1) & 0x1F;
    return rnd2(left[base] * (32 - shift) + left[base + 1] * shift, 5);
  }
  return pangle == 90 ? above[jj] : left[i];
}

/* Predicts one intra block into `dst` (the block's top-left sample in its
 * plane, global memory). `plane` points at the plane origin (for CFL's luma,
 * `luma` at the luma plane origin). `scratch` is warp-private shared memory of
 * 3 * AV1B_EDGE_LEN ints. */
/* Waits for the asynchronous copies this thread issued (cp.async), then
 * for the warp: every lane's copies are in shared memory. */
AV1B_DEV void async_copies_done() {
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncwarp();
}

AV1B_DEV void intra_predict(const IntraJob& j, px_t* dst, int stride, const px_t* luma,
                            int luma_stride, const uint8_t* palette_map,
                            const int* palette_colors, int* scratch, int lane,
                            const int* res = nullptr, int* fi_pred = nullptr,
                            bool res_in_flight = false) {
  /* `res_in_flight`: the caller's residual image is still arriving by
   * asynchronous copies; it is waited for after the edges are read (the two
   * fetches overlap), before the first sample is written */
  const int w = j.w, h = j.h, n = w * h;
  const int lw = ilog2(w);
  /* the reconstructed sample: the prediction plus, when the caller fused the
   * residual in (`res`, the block's residual, w x h row-major), that residual,
   * clipped - what adding the transforms afterwards gives */
  auto put = [&](int i, int jj, int v) {
    if (res) v = clampi(v + res[i * w + jj], 0, j.maxv);
    dst[i * stride + jj] = (px_t)v;
  };
  if (j.palette) {
    if (res_in_flight) async_copies_done();
    const uint8_t* map = palette_map + j.palette_off;
    for (int k = lane; k < n; k += 32) {
      const int i = k >> lw, jj = k & (w - 1);
      put(i, jj, palette_colors[map[i * j.palette_stride + jj]]);
    }
    return;
  }
  int* above = scratch + AV1B_EDGE_OFF;
  int* left = scratch + AV1B_EDGE_LEN + AV1B_EDGE_OFF;
  int* tmp = scratch + 2 * AV1B_EDGE_LEN;
  intra_edges(j, dst, stride, above, left, lane);
  if (res_in_flight) async_copies_done();

  if (j.mode == 13 && fi_pred && n <= 1024) {
    /* chroma from luma, each sample's luma value read once: kept in the
     * filter-intra buffer (unused by a CFL block) between the average and the
     * prediction. The (up to four) luma samples of a chroma sample are read
     * from neighbouring positions clamped to the block: every load of an
     * iteration is issued before any is used (one round trip to L2, not one
     * per sample), four iterations at a time. */
    const int dc = intra_dc(j, above, left, lane);
    const int sx = j.ss_x, sy = j.ss_y;
    const int lxl = ((j.x + w) << sx) - (1 << sx);
    const int lyl = ((j.y + h) << sy) - (1 << sy);
    long long sum = 0;
#pragma unroll 2
    for (int k = lane; k < n; k += 32) {
      const int i = k >> lw, jj = k & (w - 1);
      const int ly = mini((j.y + i) << sy, lyl), lx = mini((j.x + jj) << sx, lxl);
      const px_t* p0 = luma + ly * luma_stride + lx;
      const px_t* p1 = p0 + (sy ? luma_stride : 0);
      const int v00 = ldpx(p0), v01 = ldpx(p0 + sx), v10 = ldpx(p1), v11 = ldpx(p1 + sx);
      /* the sum of the 1, 2 or 4 samples the subsampling averages, scaled to 8x */
      int t;
      if (sx && sy) t = (v00 + v01 + v10 + v11) << 1;
      else if (sx) t = (v00 + v01) << 2;
      else if (sy) t = (v00 + v10) << 2;
      else t = v00 << 3;
      fi_pred[k] = t;
      sum += t;
    }
    sum = warp_sum64(sum);
    const int shift = lw + ilog2(h);
    const int avg = (int)((sum + (1LL << (shift - 1))) >> shift);
    __syncwarp();
    for (int k = lane; k < n; k += 32) {
      const int i = k >> lw, jj = k & (w - 1);
      put(i, jj, clampi(dc + rnd2s(j.cfl_alpha * (fi_pred[k] - avg), 6), 0, j.maxv));
    }
    return;
  }
  if (j.mode == 13) { /* chroma from luma */
    const int dc = intra_dc(j, above, left, lane);
    const int sx = j.ss_x, sy = j.ss_y;
    const int lxl = ((j.x + w) << sx) - (1 << sx);
    const int lyl = ((j.y + h) << sy) - (1 << sy);
    long long sum = 0;
    for (int k = lane; k < n; k += 32) {
      const int i = k >> lw, jj = k & (w - 1);
      const int ly = mini((j.y + i) << sy, lyl), lx = mini((j.x + jj) << sx, lxl);
      int t = 0;
      for (int a = 0; a <= sy; ++a)
        for (int b = 0; b <= sx; ++b) t += ldpx(luma + (ly + a) * luma_stride + lx + b);
      sum += t << (3 - sx - sy);
    }
    sum = warp_sum64(sum);
    const int shift = lw + ilog2(h);
    const int avg = (int)((sum + (1LL << (shift - 1))) >> shift);
    for (int k = lane; k < n; k += 32) {
      const int i = k >> lw, jj = k & (w - 1);
      const int ly = mini((j.y + i) << sy, lyl), lx = mini((j.x + jj) << sx, lxl);
      int t = 0;
      for (int a = 0; a <= sy; ++a)
        for (int b = 0; b <= sx; ++b) t += ldpx(luma + (ly + a) * luma_stride + lx + b);
      const int v = t << (3 - sx - sy);
      put(i, jj, clampi(dc + rnd2s(j.cfl_alpha * (v - avg), 6), 0, j.maxv));
    }
    return;
  }

  if (j.filter_intra && w >= 4 && h >= 2) {
    /* recursive filter: 4x2 cells along anti-diagonals; a cell reads the row
     * above it (cells up-left and up) and the column left of it - the
     * predictions of this block, kept in `fi_pred` (w x h, shared memory) so
     * the recursion never round-trips through global memory; the block is
     * written (with its residual when fused) once every cell is done */
    const int cw = w >> 2, ch = h >> 1;
    const signed char* taps = kFilterIntraTaps + j.fi_mode * 56;
    for (int d = 0; d < cw + ch - 1; ++d) {
      const int c0 = maxi(0, d - (ch - 1)), c1 = mini(d, cw - 1);
      const int cells = c1 - c0 + 1;
      for (int k = lane; k < cells * 8; k += 32) {
        const int j4 = c0 + (k >> 3), i2 = d - j4;
        const int pos = k & 7, i1 = pos >> 2, j1 = pos & 3;
        int pv[7];
        for (int t = 0; t < 5; ++t) {
          if (i2 == 0) pv[t] = above[(j4 << 2) + t - 1];
          else if (j4 == 0 && t == 0) pv[t] = left[(i2 << 1) - 1];
          else pv[t] = fi_pred[((i2 << 1) - 1) * w + (j4 << 2) + t - 1];
        }
        for (int t = 5; t < 7; ++t) {
          if (j4 == 0) pv[t] = left[(i2 << 1) + t - 5];
          else pv[t] = fi_pred[((i2 << 1) + t - 5) * w + (j4 << 2) - 1];
        }
        int pr = 0;
        for (int t = 0; t < 7; ++t) pr += taps[pos * 7 + t] * pv[t];
        fi_pred[((i2 << 1) + i1) * w + (j4 << 2) + j1] = clampi(rnd2(pr, 4), 0, j.maxv);
      }
      __syncwarp();
    }
    for (int k = lane; k < n; k += 32) {
      const int i = k >> lw, jj = k & (w - 1);
      put(i, jj, fi_pred[k]);
    }
    return;
  }

  const int mode = j.mode;
  if (mode >= 1 && mode <= 8) {
    const int pangle = kModeAngle[mode] + j.angle * 3;
    int ua = 0, ul = 0;
    if (j.filter_type >= 0 && pangle != 90 && pangle != 180) {
      if (pangle > 90 && pangle < 180 && w + h >= 24) {
        if (lane == 0) {
          const int c = rnd2(left[0] * 5 + above[-1] * 6 + above[0] * 5, 4);
          above[-1] = c;
          left[-1] = c;
        }
        __syncwarp();
      }
      if (j.have_above) {
        const int s = edge_strength(w, h, j.filter_type, pangle - 90);
        const int num = mini(w, j.max_x - j.x + 1) + (pangle < 90 ? h : 0) + 1;
        edge_filter(above, num, s, tmp, lane);
      }
      if (j.have_left) {
        const int s = edge_strength(w, h, j.filter_type, pangle - 180);
        const int num = mini(h, j.max_y - j.y + 1) + (pangle > 180 ? w : 0) + 1;
        edge_filter(left, num, s, tmp, lane);
      }
      ua = upsample_sel(w, h, j.filter_type, pangle - 90);
      if (ua) edge_upsample(above, w + (pangle < 90 ? h : 0), j.maxv, tmp, lane);
      ul = upsample_sel(w, h, j.filter_type, pangle - 180);
      if (ul) edge_upsample(left, h + (pangle > 180 ? w : 0), j.maxv, tmp, lane);
    }
    int dx = 0, dy = 0;
    if (pangle < 90) dx = kDrDeriv[pangle];
    else if (pangle > 90 && pangle < 180) dx = kDrDeriv[180 - pangle];
    if (pangle > 90 && pangle < 180) dy = kDrDeriv[pangle - 90];
    else if (pangle > 180) dy = kDrDeriv[270 - pangle];
    for (int k = lane; k < n; k += 32) {
      const int i = k >> lw, jj = k & (w - 1);
      const int v = dir_sample(above, left, w, h, pangle, dx, dy, ua, ul, i, jj);
      put(i, jj, clampi(v, 0, j.maxv));
    }
    return;
  }
  if (mode >= 9 && mode <= 11 && w >= 32) {
    /* wide blocks: a lane keeps its column's above sample and weight and
     * walks down the rows */
    const int bl = left[h - 1], tr = above[w - 1];
    for (int c = lane; c < w; c += 32) {
      const int av = above[c], wx = sm_weight(w, c);
      for (int i = 0; i < h; ++i) {
        int pred;
        if (mode == 9) {
          const int wy = sm_weight(h, i);
          pred = rnd2(wy * av + (256 - wy) * bl + wx * left[i] + (256 - wx) * tr, 9);
        } else if (mode == 10) {
          const int wy = sm_weight(h, i);
          pred = rnd2(wy * av + (256 - wy) * bl, 8);
        } else {
          pred = rnd2(wx * left[i] + (256 - wx) * tr, 8);
        }
        put(i, c, clampi(pred, 0, j.maxv));
      }
    }
    return;
  }
  if (mode >= 9 && mode <= 11) {
    for (int k = lane; k < n; k += 32) {
      const int i = k >> lw, jj = k & (w - 1);
      int pred;
      if (mode == 9) {
        const int wy = sm_weight(h, i), wx = sm_weight(w, jj);
        pred = rnd2(wy * above[jj] + (256 - wy) * left[h - 1] + wx * left[i] +
                        (256 - wx) * above[w - 1], 9);
      } else if (mode == 10) {
        const int wy = sm_weight(h, i);
        pred = rnd2(wy * above[jj] + (256 - wy) * left[h - 1], 8);
      } else {
        const int wx = sm_weight(w, jj);
        pred = rnd2(wx * left[i] + (256 - wx) * above[w - 1], 8);
      }
      put(i, jj, clampi(pred, 0, j.maxv));
    }
    return;
  }
  if (mode == 12) {
    const int tl = above[-1];
    for (int k = lane; k < n; k += 32) {
      const int i = k >> lw, jj = k & (w - 1);
      const int base = above[jj] + left[i] - tl;
      const int pl = absi(base - left[i]), pt = absi(base - above[jj]), ptl = absi(base - tl);
      const int v = (pl <= pt && pl <= ptl) ? left[i] : (pt <= ptl ? above[jj] : tl);
      put(i, jj, clampi(v, 0, j.maxv));
    }
    return;
  }
  const int dc = clampi(intra_dc(j, above, left, lane), 0, j.maxv);
  for (int k = lane; k < n; k += 32) {
    const int i = k >> lw, jj = k & (w - 1);
    put(i, jj, dc);
  }
}

}  // namespace av1b

#endif
