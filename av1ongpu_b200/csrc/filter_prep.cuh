/*
 * filter_prep.cuh - the deblocking edge and CDEF block records of a frame,
 * validated and converted from the caller's av1b_deblock_edge /
 * av1b_cdef_block (the reference's DeblockEdge / CdefBlock,
 * av1gpu.hpp:436-462).
 *
 * One definition for both sides: the device converts a frame's lists where
 * they were uploaded (k_prep_filters, one thread per record), and the host
 * planner runs the same checks, in order, only to name the first invalid
 * record when the device found one.
 */
#ifndef AV1B_FILTER_PREP_CUH
#define AV1B_FILTER_PREP_CUH

#include "../../include/av1b.h"
#include "dev_common.cuh"
#include "dev_filters.cuh"

namespace av1b {

/* Rows of plane p in the picture buffer (its padding included). */
AV1B_HD int layout_rows(const Layout& L, int p) {
  return static_cast<int>(((p < 2 ? L.p[p + 1].off : L.size) - L.p[p].off) / L.p[p].stride);
}

/* Outcomes of a record: converted, skipped (an edge the filter leaves
 * alone), or the index of the reason it is invalid in kPrepMessages. */
enum { kPrepOk = 0, kPrepSkip = 1, kPrepErrFirst = 2 };

static const char* const kPrepMessages[] = {
    "", "",
    "deblock plane out of range",
    "deblock level out of range",
    "deblock filter size must be 4, 8 or 16",
    "deblock edge reaches outside the picture",
    "CDEF plane out of range",
    "CDEF block outside the picture",
    "CDEF parameters out of range",
};

/* A deblocking edge: its record and direction (1 vertical: the V pass). */
AV1B_HD int prep_edge(const Layout& L, const av1b_deblock_edge& e, DeblockRec* r, int* vertical) {
  if (e.plane < 0 || e.plane > 2) return 2;
  if (e.length <= 0 || e.level == 0) return kPrepSkip;
  if (e.level < 0 || e.level > 63) return 3;
  if (e.filter_size != 4 && e.filter_size != 8 && e.filter_size != 16) return 4;
  const PlaneGeom& g = L.p[e.plane];
  const int rows = layout_rows(L, e.plane);
  /* how far the filter reaches across the edge: p6..q6 at most */
  const int reach = e.filter_size == 16 ? 7 : (e.filter_size == 4 ? 2 : 4);
  r->len = static_cast<short>(e.length);
  r->level = static_cast<short>(e.level);
  r->filter_size = static_cast<unsigned char>(e.filter_size);
  r->chroma = e.plane != 0;
  r->pad0 = r->pad1 = 0;
  *vertical = e.vertical ? 1 : 0;
  if (e.vertical) {
    if (e.x - reach < 0 || e.x + reach > g.stride || e.y < 0 || e.y + e.length > rows) return 5;
    r->p_off = g.off + e.y * g.stride + e.x - 2;
    r->across = 1;
    r->along = g.stride;
  } else {
    if (e.y - reach < 0 || e.y + reach > rows || e.x < 0 || e.x + e.length > g.stride) return 5;
    r->p_off = g.off + (e.y - 2) * g.stride + e.x;
    r->across = g.stride;
    r->along = 1;
  }
  return kPrepOk;
}

/* A CDEF block. A block whose direction is searched (dir -1) reads the
 * search of its 8x8 luma block from the frame's grid (`search` = the grid
 * cell); one at a luma position off the 8x8 grid needs a search of its own,
 * which the caller lists and points `search` at (*off_grid = 1). */
AV1B_HD int prep_cdef(const Layout& L, const av1b_cdef_block& c, int grid_w, CdefRec* r,
                      int* off_grid) {
  *off_grid = 0;
  if (c.plane < 0 || c.plane > 2) return 6;
  const int sx = c.plane ? L.ss_x : 0, sy = c.plane ? L.ss_y : 0;
  const int bw = 8 >> sx, bh = 8 >> sy;
  const PlaneGeom& g = L.p[c.plane];
  if (c.x < 0 || c.y < 0 || c.x + bw + 2 > g.stride || c.y + bh + 2 > layout_rows(L, c.plane) ||
      (c.x << sx) + 8 > L.p[0].stride || (c.y << sy) + 8 > layout_rows(L, 0))
    return 7;
  if (c.dir < -1 || c.dir > 7 || c.pri_strength < 0 || c.pri_strength > 255 ||
      c.sec_strength < 0 || c.sec_strength > 255 || c.damping < 0 || c.damping > 63)
    return 8;
  r->x = static_cast<short>(c.x);
  r->y = static_cast<short>(c.y);
  r->plane = static_cast<unsigned char>(c.plane);
  r->pri = static_cast<unsigned char>(c.pri_strength);
  r->sec = static_cast<unsigned char>(c.sec_strength);
  r->damping = static_cast<unsigned char>(c.damping);
  r->dir = static_cast<signed char>(c.dir);
  r->pad0 = r->pad1 = r->pad2 = 0;
  r->search = -1;
  if (c.dir < 0) {
    const int lx = c.x << sx, ly = c.y << sy;
    if ((lx | ly) & 7)
      *off_grid = 1;
    else
      r->search = (ly >> 3) * grid_w + (lx >> 3);
  }
  return kPrepOk;
}

/* What k_prep_filters reports back: the V and H edge counts, the searches
 * off the grid, whether any block reads the grid, and whether some record
 * was invalid. */
struct PrepOut {
  unsigned n_v, n_h, n_extra, any_grid, bad;
  unsigned pad[3];
};

}  // namespace av1b

#endif  // AV1B_FILTER_PREP_CUH
