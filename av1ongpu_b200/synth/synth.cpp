/*
 * synth.cpp - seeded synthetic FrameSyntax for the benchmark workloads.
 *
 * The reference measures its decoder on a synthetic clip (src/core/synthetic.cpp)
 * that only exercises DC intra, full-pel motion and one transform size. The
 * workloads here exercise every tool of the reconstruction path instead: a
 * random partition tree per superblock, every transform size and legal type,
 * all intra modes with edge filtering and upsampling, chroma from luma,
 * palette, filter intra, compound / wedge / difference-weighted prediction,
 * OBMC, global warp, deblocking, CDEF, loop restoration, superres and film
 * grain. Everything is integer arithmetic on a splitmix64 stream, so a seed
 * gives the same bytes on every machine.
 *
 * Validity rules the reference assumes but does not check (its kernels would
 * otherwise compute something undefined or order dependent) and which this
 * generator respects:
 *   - ADST / FLIPADST only when both sides are <= 16 (av1gpu_kernels.h:746-754
 *     runs the 16-point ADST for every length >= 16); 32-point sides use
 *     DCT_DCT or IDTX; 64-point sides DCT_DCT only;
 *   - intra blocks are one BlockSyntax per transform block (<= 64x64);
 *   - deblocking edges of one direction never touch the samples another edge
 *     of that direction reads (the CPU backend filters them in parallel,
 *     cpu_backend.cpp:346-356): the filter size is capped by the transform
 *     sizes on both sides;
 *   - CDEF direction is detected (dir = -1), pri 0..15, sec in {0,1,2,4};
 *   - global warp models pass the shear validity test (tables.cpp:444).
 *
 * A synthetic frame lists its references as frame *distances* (1 = previous
 * frame); the caller maps them to its own slot ids (av1b_blob_set_refs).
 *
 * The generator is a library of its own (libav1synth.so, include/av1b_synth.h),
 * apart from the decoder: a process that only needs the workload - the timed
 * CPU reference, a tool writing fixtures - loads no decoder code.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/av1b_synth.h"
#include "flat_syntax.hpp"

namespace av1b {
namespace {

enum Tool : int {
  kToolTx64 = 1 << 0,        /* 64-point transforms                       */
  kToolAllTypes = 1 << 1,    /* all 16 transform types + identity         */
  kToolCfl = 1 << 2,
  kToolPalette = 1 << 3,
  kToolFilterIntra = 1 << 4,
  kToolCompound = 1 << 5,    /* average and distance compound             */
  kToolMasks = 1 << 6,       /* wedge and difference weighted compound    */
  kToolObmc = 1 << 7,
  kToolWarp = 1 << 8,        /* global warped motion                      */
  kToolLr = 1 << 9,          /* loop restoration                          */
  kToolGrain = 1 << 10,
  kToolInterIntra = 1 << 11,
  kToolIntraBc = 1 << 12,
  kToolLossless = 1 << 13,
  kToolResidual = 1 << 14,   /* residual_provided blocks                  */
  kToolEdgeVariants = 1 << 15, /* filter_type and sharpness variations    */
  kToolNoDeblock = 1 << 16,  /* leave the deblocking edge list empty      */
  kToolNoCdef = 1 << 17,     /* leave the CDEF block list empty           */
};

constexpr int kToolsAll = kToolTx64 | kToolAllTypes | kToolCfl | kToolPalette |
                          kToolFilterIntra | kToolCompound | kToolMasks | kToolObmc |
                          kToolWarp | kToolLr | kToolGrain | kToolEdgeVariants;

struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  /* uniform in [lo, hi] */
  int range(int lo, int hi) {
    return lo + static_cast<int>(next() % static_cast<uint64_t>(hi - lo + 1));
  }
  /* true with probability num/den */
  bool chance(int num, int den) { return static_cast<int>(next() % den) < num; }
};

struct Params {
  int width = 0, height = 0, coded_width = 0, bit_depth = 8, sb = 64;
  int tools = 0;
  int key_interval = 30;
  int max_refs = 1;
};

struct Tile {
  int plane, x, y, w, h;
};

class Generator {
 public:
  Generator(const Params& p, uint64_t seed, int frame_index)
      : P(p), rng(seed * 0x100000001B3ull + static_cast<uint64_t>(frame_index) * 7919u + 17u) {
    key = (frame_index % std::max(1, P.key_interval)) == 0;
    const int since_key = frame_index % std::max(1, P.key_interval);
    nrefs = key ? 0 : std::min(P.max_refs, since_key);
    cw = P.coded_width > 0 ? P.coded_width : P.width;
    grid_w[0] = (cw + 7) & ~7;
    grid_h[0] = (P.height + 7) & ~7;
    grid_w[1] = grid_w[2] = grid_w[0] >> 1;
    grid_h[1] = grid_h[2] = grid_h[0] >> 1;
    maxv = (1 << P.bit_depth) - 1;
    lossless = (P.tools & kToolLossless) != 0;
  }

  void run(FlatSyntax* out) {
    f = out;
    frame_header();
    for (int y = 0; y < grid_h[0]; y += P.sb)
      for (int x = 0; x < grid_w[0]; x += P.sb) partition(x, y, P.sb);
    deblock_edges();
    cdef_blocks();
    if (P.tools & kToolNoDeblock) f->deblock.clear();
    if (P.tools & kToolNoCdef) f->cdef.clear();
    if (P.tools & kToolLr) restoration();
    if (P.tools & kToolGrain) film_grain();
  }

 private:
  Params P;
  Rng rng;
  FlatSyntax* f = nullptr;
  bool key = true, lossless = false;
  int nrefs = 0, cw = 0, maxv = 255;
  int grid_w[3] = {0, 0, 0}, grid_h[3] = {0, 0, 0};
  int gm[3][6] = {{0}};
  std::vector<Tile> tiles;

  bool has(int tool) const { return (P.tools & tool) != 0; }

  void frame_header() {
    av1b_frame_syntax& h = f->hdr;
    h.width = P.width;
    h.coded_width = P.coded_width > 0 && P.coded_width != P.width ? P.coded_width : 0;
    h.height = P.height;
    h.bit_depth = P.bit_depth;
    h.ss_x = 1;
    h.ss_y = 1;
    h.base_q_idx = rng.range(20, 200);
    h.sharpness = has(kToolEdgeVariants) ? rng.range(0, 7) : 0;
    h.enable_intra_edge_filter = 1;
    h.color_matrix = 1; /* BT.709 */
    h.color_range = 0;
    for (int i = 0; i < nrefs; ++i) f->reference_slots.push_back(i + 1);
    for (int r = 0; r < 3; ++r) {
      /* small affine models: scale and rotation within +-2 %, translation
       * within +-64 luma samples, all at WARPEDMODEL_PREC_BITS = 16 */
      gm[r][0] = rng.range(-64 * 65536, 64 * 65536);
      gm[r][1] = rng.range(-64 * 65536, 64 * 65536);
      gm[r][2] = 65536 + rng.range(-1310, 1310);
      gm[r][3] = rng.range(-1310, 1310);
      gm[r][4] = rng.range(-1310, 1310);
      gm[r][5] = 65536 + rng.range(-1310, 1310);
    }
  }

  /* ---- partition ------------------------------------------------------ */
  void partition(int x, int y, int s) {
    if (x >= grid_w[0] || y >= grid_h[0]) return;
    const bool crosses = x + s > grid_w[0] || y + s > grid_h[0];
    const bool can_split = s > 8;
    if (can_split && (crosses || rng.chance(1, 2))) {
      const int h = s / 2;
      partition(x, y, h);
      partition(x + h, y, h);
      partition(x, y + h, h);
      partition(x + h, y + h, h);
      return;
    }
    coding_block(x, y, s);
  }

  void coding_block(int x, int y, int s) {
    const bool intra = key || rng.chance(1, 10);
    if (intra) {
      if (key && has(kToolIntraBc) && y >= 64 && s <= 32 && rng.chance(1, 8)) {
        intrabc_block(x, y, s);
        return;
      }
      intra_block(x, y, s);
    } else {
      inter_block(x, y, s);
    }
  }

  /* ---- transforms and coefficients ---------------------------------- */
  int max_tx() const { return has(kToolTx64) ? 64 : 32; }

  /* Picks a transform tiling of a w x h region: returns the tile size. */
  void pick_tx(int w, int h, int* tw, int* th) {
    if (lossless) {
      *tw = *th = 4;
      return;
    }
    int t = std::min(std::min(w, h), max_tx());
    const int drop = rng.range(0, 2);
    for (int i = 0; i < drop && t > 4; ++i) t >>= 1;
    *tw = *th = t;
    const int shape = rng.range(0, 5);
    if (shape == 1 && t >= 8 && t <= 64) *th = t / 2;        /* 2:1 wide   */
    if (shape == 2 && t >= 8 && t <= 64) *tw = t / 2;        /* 1:2 tall   */
    if (shape == 3 && t >= 16 && t <= 64) *th = t / 4;       /* 4:1 wide   */
    if (shape == 4 && t >= 16 && t <= 64) *tw = t / 4;       /* 1:4 tall   */
    if (*tw > w) *tw = w;
    if (*th > h) *th = h;
  }

  int pick_type(int w, int h) {
    const int m = std::max(w, h);
    if (m == 64) return 0;
    if (m == 32) return (has(kToolAllTypes) && rng.chance(1, 6)) ? 9 : 0;
    if (has(kToolAllTypes)) {
      if (rng.chance(2, 5)) return 0;
      return rng.range(0, 15);
    }
    /* 70 % DCT_DCT, 30 % an ADST mix */
    if (rng.chance(7, 10)) return 0;
    static const int mix[3] = {1, 2, 3};
    return mix[rng.range(0, 2)];
  }

  /* Laplacian magnitude with scale 64, from an integer uniform. */
  int laplace() {
    const double u = (static_cast<double>(rng.next() >> 11) + 0.5) / 9007199254740992.0;
    int m = static_cast<int>(-64.0 * std::log(u));
    return m < 1 ? 1 : m;
  }

  /* Appends one transform's coefficient raster; returns eob (0 = no residual). */
  int fill_coefficients(const av1b_transform& t, int bd) {
    const int cw_ = std::min(t.w, 32), ch = std::min(t.h, 32);
    const int area = cw_ * ch;
    const size_t base = f->coefficients.size();
    f->coefficients.resize(base + area, 0);
    int* r = f->coefficients.data() + base;
    const int limit = (1 << (7 + bd)) - 1;
    if (lossless) {
      /* small residuals so the WHT round trip stays in range */
      int nz = 0;
      for (int i = 0; i < area; ++i)
        if (rng.chance(1, 3)) {
          r[i] = rng.range(-96, 96);
          nz += r[i] != 0;
        }
      return nz;
    }
    /* about 10 % of the raster, concentrated on the low diagonals */
    int target = std::max(1, area / 10 + rng.range(-area / 40, area / 40));
    int nz = 0;
    const int diag_max = cw_ + ch - 2;
    for (int k = 0; k < target; ++k) {
      int d = 0;
      const int spread = std::max(1, (cw_ + ch) / 6);
      while (d < diag_max && rng.chance(spread, spread + 1)) ++d;
      /* a position on anti-diagonal d */
      const int c0 = std::max(0, d - (ch - 1)), c1 = std::min(d, cw_ - 1);
      const int c = rng.range(c0, c1);
      const int row = d - c;
      int v = laplace();
      if (rng.chance(1, 2)) v = -v;
      v = std::max(-limit, std::min(limit, v));
      if (r[row * cw_ + c] == 0) ++nz;
      r[row * cw_ + c] = v;
    }
    return nz;
  }

  /* Adds the transforms of a w x h region at (x, y) of `plane` (all with
   * residual or none) to block `b`; returns whether any were added. */
  void add_transforms(av1b_block* b, int plane, int w, int h, bool with_residual, bool record,
                      int forced_tw = 0, int forced_th = 0) {
    int tw, th;
    if (forced_tw) {
      tw = forced_tw;
      th = forced_th;
    } else {
      pick_tx(w, h, &tw, &th);
    }
    b->tx_first = static_cast<int32_t>(f->transforms.size());
    b->tx_count = 0;
    for (int ty = 0; ty < h; ty += th)
      for (int tx = 0; tx < w; tx += tw) {
        if (record) tiles.push_back(Tile{plane, b->x + tx, b->y + ty, tw, th});
        if (!with_residual) continue;
        av1b_transform t;
        std::memset(&t, 0, sizeof(t));
        t.x = tx;
        t.y = ty;
        t.w = tw;
        t.h = th;
        t.tx_type = lossless ? 0 : pick_type(tw, th);
        t.coef_offset = static_cast<int32_t>(f->coefficients.size());
        t.denominator = 1;
        t.qm_off = -1;
        t.qindex = f->hdr.base_q_idx;
        t.eob = fill_coefficients(t, b->bit_depth);
        f->transforms.push_back(t);
        ++b->tx_count;
      }
  }

  av1b_block new_block(int plane, int x, int y, int w, int h) {
    av1b_block b;
    std::memset(&b, 0, sizeof(b));
    b.x = x;
    b.y = y;
    b.w = w;
    b.h = h;
    b.plane = plane;
    b.bit_depth = P.bit_depth;
    b.have_left = x > 0;
    b.have_above = y > 0;
    b.have_above_right = -1;
    b.have_below_left = -1;
    b.ref[0] = b.ref[1] = -1;
    b.blend[0] = b.blend[1] = 8;
    b.lossless = lossless ? 1 : 0;
    return b;
  }

  /* ---- intra ------------------------------------------------------------ */
  void intra_block(int x, int y, int s) {
    const bool palette = has(kToolPalette) && s <= 64 && rng.chance(1, 10);
    const bool filter_intra = !palette && has(kToolFilterIntra) && s <= 32 && rng.chance(1, 7);
    const int fi_mode = rng.range(0, 4);
    for (int plane = 0; plane < 3; ++plane) {
      const int sub = plane ? 1 : 0;
      const int px = x >> sub, py = y >> sub, ps = s >> sub;
      /* this plane's palette and colour map */
      int colors[8] = {0};
      int pal_size = 0;
      size_t pal_base = 0;
      if (palette) {
        pal_size = rng.range(2, 8);
        for (int i = 0; i < pal_size; ++i) colors[i] = rng.range(0, maxv);
        std::sort(colors, colors + pal_size);
        pal_base = f->palette_map.size();
        f->palette_map.resize(pal_base + static_cast<size_t>(ps) * ps);
        uint8_t* map = f->palette_map.data() + pal_base;
        int run = rng.range(0, pal_size - 1);
        for (int i = 0; i < ps * ps; ++i) {
          if (rng.chance(1, 4)) run = rng.range(0, pal_size - 1);
          map[i] = static_cast<uint8_t>(run);
        }
      }
      const bool cfl = plane > 0 && !palette && has(kToolCfl) && ps <= 32 && rng.chance(1, 4);
      const int cfl_alpha = rng.range(-16, 16);
      int tw, th;
      pick_tx(ps, ps, &tw, &th);
      if (cfl) tw = th = std::min(ps, 32);
      for (int ty = 0; ty < ps; ty += th)
        for (int tx = 0; tx < ps; tx += tw) {
          av1b_block b = new_block(plane, px + tx, py + ty, tw, th);
          b.is_intra = 1;
          b.mode = rng.range(0, 12);
          if (b.mode >= 1 && b.mode <= 8) b.angle_delta = rng.range(-3, 3);
          b.filter_type = has(kToolEdgeVariants) ? rng.range(0, 1) : 0;
          if (cfl) {
            b.mode = 13;
            b.cfl_alpha = cfl_alpha;
          }
          if (filter_intra && plane == 0) {
            b.use_filter_intra = 1;
            b.filter_intra_mode = fi_mode;
            b.mode = 0;
          }
          if (palette) {
            b.use_palette = 1;
            b.mode = 0;
            b.palette_size = pal_size;
            for (int i = 0; i < 8; ++i) b.palette[i] = colors[i];
            b.palette_off = static_cast<int32_t>(pal_base + static_cast<size_t>(ty) * ps + tx);
            b.palette_stride = ps;
          }
          const bool residual = rng.chance(4, 5);
          add_transforms(&b, plane, tw, th, residual, true, tw, th);
          f->blocks.push_back(b);
        }
    }
  }

  /* Intra block copy: an inter-shaped block that copies an already decoded
   * region of this frame (at least one superblock row above). */
  void intrabc_block(int x, int y, int s) {
    /* the source lies entirely in the superblock rows above this one, which
     * are decoded before any block of this row */
    const int top = y & ~(P.sb - 1);
    if (top - s < 0) {
      intra_block(x, y, s);
      return;
    }
    const int sy = rng.range(0, (top - s) / 8) * 8;
    const int sx = std::max(0, std::min(grid_w[0] - s, x + rng.range(-8, 8) * 8));
    const int mvx = (sx - x) * 8, mvy = (sy - y) * 8;
    for (int plane = 0; plane < 3; ++plane) {
      const int sub = plane ? 1 : 0;
      av1b_block b = new_block(plane, x >> sub, y >> sub, s >> sub, s >> sub);
      b.is_intra = 0;
      b.intrabc = 1;
      b.mv[0][0] = mvx;
      b.mv[0][1] = mvy;
      b.filter = b.filter_v = 3; /* bilinear */
      add_transforms(&b, plane, b.w, b.h, rng.chance(1, 2), true);
      f->blocks.push_back(b);
    }
  }

  /* ---- inter ------------------------------------------------------------ */
  void inter_block(int x, int y, int s) {
    const bool compound = has(kToolCompound) && nrefs >= 2 && rng.chance(3, 10);
    int comp_type = 0;
    if (compound) {
      const bool masks_ok = has(kToolMasks);
      const int r = rng.range(0, masks_ok ? 3 : 1);
      comp_type = r + 1; /* 1 avg, 2 dist, 3 wedge, 4 diffwtd */
      if (comp_type == 3 && (s < 8 || s > 32)) comp_type = 4;
    }
    const bool obmc = !compound && has(kToolObmc) && (x > 0 || y > 0) && rng.chance(1, 5);
    const bool interintra = !compound && !obmc && has(kToolInterIntra) && s >= 8 && s <= 32 &&
                            rng.chance(1, 6);
    const bool ii_wedge = interintra && rng.chance(1, 3);
    const int ii_mode = rng.range(0, 3);
    int ref0 = rng.range(0, nrefs - 1), ref1 = -1;
    if (compound) {
      ref1 = rng.range(0, nrefs - 2);
      if (ref1 >= ref0) ++ref1;
    }
    int mv[2][2];
    for (int i = 0; i < 2; ++i)
      for (int k = 0; k < 2; ++k) mv[i][k] = rng.range(-512, 512);
    const int filt = rng.range(0, 3), filt_v = rng.range(0, 3);
    const bool warp0 = has(kToolWarp) && rng.chance(1, 4);
    const bool warp1 = compound && has(kToolWarp) && rng.chance(1, 4);
    static const int kDist[8][2] = {{9, 7}, {11, 5}, {12, 4}, {13, 3},
                                    {7, 9}, {5, 11}, {4, 12}, {3, 13}};
    const int dist = rng.range(0, 7);
    const int wedge_index = rng.range(0, 15), mask_sign = rng.range(0, 1);
    const bool skip = rng.chance(3, 10);
    /* the OBMC strips of the luma block; chroma halves them */
    struct Strip {
      int pass, x, y, w, h, mvx, mvy, filt, filt_v, ref;
    };
    std::vector<Strip> strips;
    if (obmc) {
      const int ov = std::min(s / 2, 32);
      if (y > 0) {
        const int n = s >= 32 ? (rng.chance(1, 2) ? 4 : 2) : 1;
        const int sw = std::max(8, s / n);
        for (int i = 0; i * sw < s; ++i)
          strips.push_back(Strip{0, i * sw, 0, sw, ov, rng.range(-512, 512), rng.range(-512, 512),
                                 rng.range(0, 3), rng.range(0, 3), rng.range(0, nrefs - 1)});
      }
      if (x > 0) {
        const int n = s >= 32 ? (rng.chance(1, 2) ? 4 : 2) : 1;
        const int sh = std::max(8, s / n);
        for (int i = 0; i * sh < s; ++i)
          strips.push_back(Strip{1, 0, i * sh, ov, sh, rng.range(-512, 512), rng.range(-512, 512),
                                 rng.range(0, 3), rng.range(0, 3), rng.range(0, nrefs - 1)});
      }
    }
    int tw = 0, th = 0;
    pick_tx(std::min(s, 64), std::min(s, 64), &tw, &th);
    for (int plane = 0; plane < 3; ++plane) {
      const int sub = plane ? 1 : 0;
      av1b_block b = new_block(plane, x >> sub, y >> sub, s >> sub, s >> sub);
      b.is_intra = 0;
      b.ref[0] = ref0;
      b.ref[1] = ref1;
      for (int i = 0; i < 2; ++i) {
        b.mv[i][0] = mv[i][0];
        b.mv[i][1] = mv[i][1];
      }
      b.filter = filt;
      b.filter_v = filt_v;
      b.compound = comp_type;
      if (comp_type == 2) {
        b.blend[0] = kDist[dist][0];
        b.blend[1] = kDist[dist][1];
      }
      if (comp_type == 3 || comp_type == 4) {
        b.wedge_index = wedge_index;
        b.mask_sign = mask_sign;
      }
      /* the luma region decides the difference weighted mask; a chroma
       * region below 8x8 is predicted from its vector */
      const bool big = b.w >= 8 && b.h >= 8;
      b.warp[0] = warp0 && big;
      b.warp[1] = warp1 && big;
      b.mask_warp[0] = warp0;
      b.mask_warp[1] = warp1;
      for (int k = 0; k < 6; ++k) {
        b.warp_params[0][k] = gm[ref0][k];
        if (ref1 >= 0) b.warp_params[1][k] = gm[ref1][k];
      }
      b.motion_mode = obmc ? 1 : 0;
      if (interintra) {
        b.interintra = 1;
        b.interintra_mode = ii_mode;
        b.interintra_wedge = ii_wedge ? 1 : 0;
        b.wedge_index = wedge_index;
      }
      b.obmc_first = static_cast<int32_t>(f->obmc.size());
      for (const Strip& st : strips) {
        av1b_obmc o;
        o.pass = st.pass;
        o.x = st.x >> sub;
        o.y = st.y >> sub;
        o.w = st.w >> sub;
        o.h = st.h >> sub;
        o.mv[0] = st.mvx;
        o.mv[1] = st.mvy;
        o.filter = st.filt;
        o.filter_v = st.filt_v;
        o.ref = st.ref;
        f->obmc.push_back(o);
      }
      b.obmc_count = static_cast<int32_t>(strips.size());
      const bool residual_provided = has(kToolResidual) && !skip && rng.chance(1, 8);
      if (residual_provided) {
        b.residual_provided = 1;
        add_residual(&b);
      } else if (skip) {
        /* a skipped block still has its prediction edges deblocked */
        const int e = std::min(b.w, 64 >> sub);
        add_transforms(&b, plane, b.w, b.h, false, true, e, std::min(b.h, 64 >> sub));
      } else {
        const int ptw = std::max(4, tw >> sub), pth = std::max(4, th >> sub);
        add_transforms(&b, plane, b.w, b.h, true, true, std::min(ptw, b.w), std::min(pth, b.h));
      }
      f->blocks.push_back(b);
    }
  }

  /* Raw residual samples for a residual_provided block: one "transform" per
   * 16x16 region whose pool holds w*h residual samples. */
  void add_residual(av1b_block* b) {
    const int t = std::min(16, b->w);
    b->tx_first = static_cast<int32_t>(f->transforms.size());
    b->tx_count = 0;
    for (int ty = 0; ty < b->h; ty += t)
      for (int tx = 0; tx < b->w; tx += t) {
        tiles.push_back(Tile{b->plane, b->x + tx, b->y + ty, t, t});
        av1b_transform o;
        std::memset(&o, 0, sizeof(o));
        o.x = tx;
        o.y = ty;
        o.w = t;
        o.h = t;
        o.coef_offset = static_cast<int32_t>(f->residual.size());
        o.eob = 1;
        o.denominator = 1;
        o.qm_off = -1;
        for (int i = 0; i < t * t; ++i) f->residual.push_back(rng.range(-40, 40));
        f->transforms.push_back(o);
        ++b->tx_count;
      }
  }

  /* ---- deblocking --------------------------------------------------------- */
  void deblock_edges() {
    int level[4];
    for (int i = 0; i < 4; ++i) level[i] = rng.range(0, 63);
    for (int plane = 0; plane < 3; ++plane) {
      const int cw4 = (grid_w[plane] + 3) / 4, ch4 = (grid_h[plane] + 3) / 4;
      std::vector<uint8_t> tw(static_cast<size_t>(cw4) * ch4, 0), th(tw.size(), 0);
      for (const Tile& t : tiles) {
        if (t.plane != plane) continue;
        for (int y = t.y; y < t.y + t.h && y < grid_h[plane]; y += 4)
          for (int x = t.x; x < t.x + t.w && x < grid_w[plane]; x += 4) {
            tw[(y / 4) * cw4 + x / 4] = static_cast<uint8_t>(std::min(t.w, 64));
            th[(y / 4) * cw4 + x / 4] = static_cast<uint8_t>(std::min(t.h, 64));
          }
      }
      auto size_of = [&](int m) {
        if (plane) return m >= 8 ? 8 : 4;
        return m >= 16 ? 16 : (m >= 8 ? 8 : 4);
      };
      for (const Tile& t : tiles) {
        if (t.plane != plane) continue;
        if (t.x >= grid_w[plane] || t.y >= grid_h[plane]) continue;
        const int len_v = std::min(t.h, grid_h[plane] - t.y);
        const int len_h = std::min(t.w, grid_w[plane] - t.x);
        if (t.x > 0 && len_v > 0) {
          int m = t.w;
          for (int y = t.y; y < t.y + len_v; y += 4) m = std::min(m, (int)tw[(y / 4) * cw4 + (t.x - 4) / 4]);
          av1b_deblock_edge e{plane, t.x, t.y, 1, len_v, plane == 0 ? level[0] : level[1 + plane],
                              size_of(m)};
          f->deblock.push_back(e);
        }
        if (t.y > 0 && len_h > 0) {
          int m = t.h;
          for (int x = t.x; x < t.x + len_h; x += 4) m = std::min(m, (int)th[((t.y - 4) / 4) * cw4 + x / 4]);
          av1b_deblock_edge e{plane, t.x, t.y, 0, len_h, plane == 0 ? level[1] : level[1 + plane],
                              size_of(m)};
          f->deblock.push_back(e);
        }
      }
    }
  }

  /* ---- CDEF --------------------------------------------------------------- */
  void cdef_blocks() {
    static const int kSec[4] = {0, 1, 2, 4};
    const int damping = rng.range(3, 6);
    int preset[8][4];
    for (int i = 0; i < 8; ++i) {
      preset[i][0] = rng.range(0, 15);
      preset[i][1] = kSec[rng.range(0, 3)];
      preset[i][2] = rng.range(0, 15);
      preset[i][3] = kSec[rng.range(0, 3)];
    }
    for (int fy = 0; fy < grid_h[0]; fy += 64)
      for (int fx = 0; fx < grid_w[0]; fx += 64) {
        if (rng.chance(1, 10)) continue;
        const int idx = rng.range(0, 7);
        for (int y = fy; y < std::min(fy + 64, grid_h[0]); y += 8)
          for (int x = fx; x < std::min(fx + 64, grid_w[0]); x += 8) {
            if (rng.chance(3, 20)) continue;
            f->cdef.push_back(av1b_cdef_block{0, x, y, preset[idx][0], preset[idx][1], damping, -1});
            for (int p = 1; p < 3; ++p)
              f->cdef.push_back(
                  av1b_cdef_block{p, x >> 1, y >> 1, preset[idx][2], preset[idx][3], damping, -1});
          }
      }
  }

  /* ---- loop restoration ---------------------------------------------------- */
  void restoration() {
    for (int p = 0; p < 3; ++p) {
      const int sub = p ? 1 : 0;
      const int pw = (P.width + sub) >> sub, ph = (P.height + sub) >> sub;
      const int cols = std::max((pw + 32) >> 6, 1), rows = std::max((ph + 32) >> 6, 1);
      f->hdr.restoration_type[p] = 1; /* switchable: every unit picks */
      f->hdr.restoration_unit_log2[p] = 6;
      f->hdr.restoration_unit_cols[p] = cols;
      f->restoration[p].resize(static_cast<size_t>(cols) * rows);
      for (auto& u : f->restoration[p]) {
        std::memset(&u, 0, sizeof(u));
        if (rng.chance(1, 2)) {
          u.type = 2; /* RESTORE_WIENER in the reference's numbering (av1gpu.hpp:372-377) */
          for (int pass = 0; pass < 2; ++pass) {
            u.wiener[pass][0] = p ? 0 : rng.range(-5, 10);
            u.wiener[pass][1] = rng.range(-23, 8);
            u.wiener[pass][2] = rng.range(-17, 46);
          }
        } else {
          u.type = 3; /* RESTORE_SGRPROJ */
          u.sgr_set = rng.range(0, 15);
          u.sgr_xqd[0] = rng.range(-96, 31);
          u.sgr_xqd[1] = rng.range(-32, 95);
          if (u.sgr_set >= 10 && u.sgr_set <= 13) u.sgr_xqd[0] = 0;
          if (u.sgr_set >= 14) u.sgr_xqd[1] = std::max(-32, std::min(95, 128 - u.sgr_xqd[0]));
        }
      }
    }
  }

  /* ---- film grain --------------------------------------------------------- */
  void points(int n, int32_t* value, int32_t* scaling) {
    int v = rng.range(0, 40);
    for (int i = 0; i < n; ++i) {
      value[i] = std::min(255, v);
      scaling[i] = rng.range(0, 160);
      v += rng.range(8, std::max(9, 215 / std::max(1, n)));
    }
    /* strictly increasing and inside 0..255 */
    for (int i = 1; i < n; ++i)
      if (value[i] <= value[i - 1]) value[i] = value[i - 1] + 1;
    for (int i = n - 1; i >= 0; --i)
      if (value[i] > 255 - (n - 1 - i)) value[i] = 255 - (n - 1 - i);
  }

  void film_grain() {
    av1b_film_grain& g = f->hdr.grain;
    std::memset(&g, 0, sizeof(g));
    g.apply = 1;
    g.seed = rng.range(0, 65535);
    g.num_y_points = rng.range(2, 10);
    points(g.num_y_points, g.point_y_value, g.point_y_scaling);
    g.chroma_scaling_from_luma = rng.chance(1, 4);
    if (!g.chroma_scaling_from_luma) {
      g.num_cb_points = rng.range(0, 6);
      g.num_cr_points = rng.range(1, 6);
      points(g.num_cb_points, g.point_cb_value, g.point_cb_scaling);
      points(g.num_cr_points, g.point_cr_value, g.point_cr_scaling);
    }
    g.grain_scaling_minus_8 = rng.range(0, 3);
    g.ar_coeff_lag = 3;
    for (int i = 0; i < 24; ++i) g.ar_coeffs_y[i] = rng.range(-24, 24);
    for (int i = 0; i < 25; ++i) {
      g.ar_coeffs_cb[i] = rng.range(-24, 24);
      g.ar_coeffs_cr[i] = rng.range(-24, 24);
    }
    g.ar_coeff_shift_minus_6 = rng.range(0, 3);
    g.grain_scale_shift = rng.range(0, 1);
    g.cb_mult = rng.range(100, 160);
    g.cb_luma_mult = rng.range(100, 200);
    g.cb_offset = rng.range(200, 320);
    g.cr_mult = rng.range(100, 160);
    g.cr_luma_mult = rng.range(100, 200);
    g.cr_offset = rng.range(200, 320);
    g.overlap_flag = rng.range(0, 1);
    g.clip_to_restricted_range = rng.range(0, 1);
  }
};

Params config_params(int config, int scale) {
  Params p;
  auto scaled = [scale](int v) { return std::max(16, ((v / std::max(1, scale)) + 1) & ~1); };
  switch (config) {
    case 1: /* 1280x720 8-bit, 1 key + inter frames from one reference */
      p.width = scaled(1280);
      p.height = scaled(720);
      p.bit_depth = 8;
      p.sb = 64;
      p.tools = 0;
      p.key_interval = 1 << 30;
      p.max_refs = 1;
      break;
    case 2: /* 1920x1080 10-bit, every tool, key frame every 30 */
      p.width = scaled(1920);
      p.height = scaled(1080);
      p.bit_depth = 10;
      p.sb = 64;
      p.tools = kToolsAll;
      p.key_interval = 30;
      p.max_refs = 3;
      break;
    case 3: /* coded 2880x2160 superres to 3840x2160 10-bit, 128x128 superblocks */
      p.width = scaled(3840);
      p.coded_width = scaled(2880);
      p.height = scaled(2160);
      p.bit_depth = 10;
      p.sb = 128;
      p.tools = kToolsAll;
      p.key_interval = 30;
      p.max_refs = 3;
      break;
    default:
      break;
  }
  return p;
}

}  // namespace

/* Builds one synthetic frame. */
bool synth_frame(const Params& p, uint64_t seed, int frame_index, FlatSyntax* out) {
  if (p.width <= 0 || p.height <= 0 || (p.width & 1) || (p.height & 1)) return false;
  Generator g(p, seed, frame_index);
  g.run(out);
  return true;
}

}  // namespace av1b

extern "C" {

static int synth_to_blob(const av1b::Params& p, uint64_t seed, int frame_index, uint8_t** blob,
                         size_t* len) {
  if (!blob || !len) return AV1B_ERR_ARG;
  av1b::FlatSyntax fs;
  if (!av1b::synth_frame(p, seed, frame_index, &fs)) return AV1B_ERR_ARG;
  std::vector<uint8_t> bytes;
  av1b::write_blob(fs.view(), &bytes);
  void* mem = nullptr;
  if (posix_memalign(&mem, 64, bytes.size() ? bytes.size() : 64) != 0) return AV1B_ERR_NOMEM;
  std::memcpy(mem, bytes.data(), bytes.size());
  *blob = static_cast<uint8_t*>(mem);
  *len = bytes.size();
  return AV1B_OK;
}

int av1s_synth_frame(int config, int scale, uint64_t seed, int frame_index, uint8_t** blob,
                     size_t* len) {
  const av1b::Params p = av1b::config_params(config, scale);
  if (p.width <= 0) return AV1B_ERR_ARG;
  return synth_to_blob(p, seed, frame_index, blob, len);
}

int av1s_synth_frame_refs(int width, int height, int coded_width, int bit_depth, int sb_size,
                          int tools, int max_refs, uint64_t seed, int frame_index, int key_interval,
                          uint8_t** blob, size_t* len) {
  av1b::Params p;
  p.width = width;
  p.height = height;
  p.coded_width = coded_width;
  p.bit_depth = bit_depth;
  p.sb = sb_size == 128 ? 128 : 64;
  p.tools = tools;
  p.key_interval = key_interval > 0 ? key_interval : (1 << 30);
  p.max_refs = max_refs;
  if (bit_depth != 8 && bit_depth != 10 && bit_depth != 12) return AV1B_ERR_ARG;
  if (max_refs < 1 || max_refs > 3) return AV1B_ERR_ARG;
  return synth_to_blob(p, seed, frame_index, blob, len);
}

int av1s_synth_frame_ex(int width, int height, int coded_width, int bit_depth, int sb_size,
                        int tools, uint64_t seed, int frame_index, int key_interval,
                        uint8_t** blob, size_t* len) {
  return av1s_synth_frame_refs(width, height, coded_width, bit_depth, sb_size, tools,
                               (tools & (1 << 5)) ? 3 : 1, seed, frame_index, key_interval, blob,
                               len);
}

void av1s_blob_free(uint8_t* blob) { free(blob); }

}  // extern "C"
