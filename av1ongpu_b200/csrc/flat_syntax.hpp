/*
 * flat_syntax.hpp - an owning container for av1b_frame_syntax, its byte image
 * ("blob"), and conversions to and from a C++ FrameSyntax.
 *
 * The C++ conversions are templates over the FrameSyntax type so that the
 * same code serves this library's av1gpu::FrameSyntax and any other struct
 * with the reference's field names (include/av1gpu/av1gpu.hpp:187-537 of the
 * reference library).
 *
 * Blob layout (little endian, every array 16-byte aligned so that a view can
 * point into the buffer without copying):
 *   u32 magic "AV1B", u32 version, u32 reserved, u32 n_refs,
 *   i32 ref_slots[8]                      (patchable in place)
 *   scalar prefix of av1b_frame_syntax    (everything before reference_slots)
 *   for each array, in the order below: u64 count, padding, elements
 */
#ifndef AV1B_FLAT_SYNTAX_HPP
#define AV1B_FLAT_SYNTAX_HPP

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <vector>

#include "../../include/av1b.h"

namespace av1b {

constexpr uint32_t kBlobMagic = 0x42315641u; /* "AV1B" */
constexpr uint32_t kBlobVersion = 1;
constexpr int kBlobMaxRefs = 8;
constexpr size_t kScalarBytes = offsetof(av1b_frame_syntax, reference_slots);
constexpr size_t kBlobHeader = 16 + 4 * kBlobMaxRefs;

struct FlatSyntax {
  av1b_frame_syntax hdr;  /* scalars; the pointers are filled by view() */
  std::vector<int32_t> reference_slots;
  std::vector<av1b_block> blocks;
  std::vector<av1b_transform> transforms;
  std::vector<av1b_obmc> obmc;
  std::vector<int32_t> coefficients;
  std::vector<int32_t> residual;
  std::vector<int16_t> levels;
  std::vector<uint8_t> qm_pool;
  std::vector<uint8_t> palette_map;
  std::vector<av1b_deblock_edge> deblock;
  std::vector<av1b_cdef_block> cdef;
  std::vector<av1b_restoration_unit> restoration[3];

  FlatSyntax() { std::memset(&hdr, 0, sizeof(hdr)); }

  av1b_frame_syntax view() const {
    av1b_frame_syntax v = hdr;
    v.reference_slots = reference_slots.data();
    v.n_reference_slots = reference_slots.size();
    v.blocks = blocks.data();
    v.n_blocks = blocks.size();
    v.transforms = transforms.data();
    v.n_transforms = transforms.size();
    v.obmc = obmc.data();
    v.n_obmc = obmc.size();
    v.coefficients = coefficients.data();
    v.n_coefficients = coefficients.size();
    v.residual = residual.data();
    v.n_residual = residual.size();
    v.levels = levels.data();
    v.n_levels = levels.size();
    v.qm_pool = qm_pool.data();
    v.n_qm_pool = qm_pool.size();
    v.palette_map = palette_map.data();
    v.n_palette_map = palette_map.size();
    v.deblock = deblock.data();
    v.n_deblock = deblock.size();
    v.cdef = cdef.data();
    v.n_cdef = cdef.size();
    for (int p = 0; p < 3; ++p) {
      v.restoration[p] = restoration[p].data();
      v.n_restoration[p] = restoration[p].size();
    }
    return v;
  }
};

namespace detail {

inline size_t align16(size_t v) { return (v + 15) & ~static_cast<size_t>(15); }

struct Writer {
  std::vector<uint8_t>* out;
  void put(const void* p, size_t n) {
    const uint8_t* b = static_cast<const uint8_t*>(p);
    out->insert(out->end(), b, b + n);
  }
  void pad() { out->resize(align16(out->size()), 0); }
  template <class T>
  void array(const T* data, size_t count) {
    const uint64_t c = count;
    put(&c, sizeof(c));
    pad();
    if (count) put(data, count * sizeof(T));
    pad();
  }
};

struct Reader {
  const uint8_t* base;
  size_t len, pos;
  bool ok = true;
  template <class T>
  const T* array(size_t* count) {
    if (pos + 8 > len) { ok = false; return nullptr; }
    uint64_t c;
    std::memcpy(&c, base + pos, 8);
    pos = align16(pos + 8);
    const size_t bytes = static_cast<size_t>(c) * sizeof(T);
    if (c > (uint64_t)len || pos + bytes > len) { ok = false; return nullptr; }
    const T* p = reinterpret_cast<const T*>(base + pos);
    pos = align16(pos + bytes);
    *count = static_cast<size_t>(c);
    return c ? p : nullptr;
  }
};

}  // namespace detail

/* Serializes a view into a blob. */
inline void write_blob(const av1b_frame_syntax& v, std::vector<uint8_t>* out) {
  out->clear();
  detail::Writer w{out};
  const uint32_t head[4] = {kBlobMagic, kBlobVersion, 0,
                            static_cast<uint32_t>(v.n_reference_slots)};
  w.put(head, sizeof(head));
  int32_t refs[kBlobMaxRefs];
  for (int i = 0; i < kBlobMaxRefs; ++i)
    refs[i] = i < (int)v.n_reference_slots ? v.reference_slots[i] : -1;
  w.put(refs, sizeof(refs));
  w.put(&v, kScalarBytes);
  w.pad();
  w.array(v.blocks, v.n_blocks);
  w.array(v.transforms, v.n_transforms);
  w.array(v.obmc, v.n_obmc);
  w.array(v.coefficients, v.n_coefficients);
  w.array(v.residual, v.n_residual);
  w.array(v.levels, v.n_levels);
  w.array(v.qm_pool, v.n_qm_pool);
  w.array(v.palette_map, v.n_palette_map);
  w.array(v.deblock, v.n_deblock);
  w.array(v.cdef, v.n_cdef);
  for (int p = 0; p < 3; ++p) w.array(v.restoration[p], v.n_restoration[p]);
}

/* Points a view into a blob. Returns false on a malformed buffer. The
 * reference slot list points into the blob's patchable header. */
inline bool view_blob(const uint8_t* blob, size_t len, av1b_frame_syntax* v) {
  if (!blob || len < kBlobHeader + kScalarBytes) return false;
  uint32_t head[4];
  std::memcpy(head, blob, sizeof(head));
  if (head[0] != kBlobMagic || head[1] != kBlobVersion || head[3] > kBlobMaxRefs) return false;
  if ((reinterpret_cast<uintptr_t>(blob) & 15) != 0) return false;
  std::memcpy(v, blob + kBlobHeader, kScalarBytes);
  v->reference_slots = reinterpret_cast<const int32_t*>(blob + 16);
  v->n_reference_slots = head[3];
  detail::Reader r{blob, len, detail::align16(kBlobHeader + kScalarBytes)};
  v->blocks = r.array<av1b_block>(&v->n_blocks);
  v->transforms = r.array<av1b_transform>(&v->n_transforms);
  v->obmc = r.array<av1b_obmc>(&v->n_obmc);
  v->coefficients = r.array<int32_t>(&v->n_coefficients);
  v->residual = r.array<int32_t>(&v->n_residual);
  v->levels = r.array<int16_t>(&v->n_levels);
  v->qm_pool = r.array<uint8_t>(&v->n_qm_pool);
  v->palette_map = r.array<uint8_t>(&v->n_palette_map);
  v->deblock = r.array<av1b_deblock_edge>(&v->n_deblock);
  v->cdef = r.array<av1b_cdef_block>(&v->n_cdef);
  for (int p = 0; p < 3; ++p)
    v->restoration[p] = r.array<av1b_restoration_unit>(&v->n_restoration[p]);
  return r.ok;
}

inline bool blob_set_refs(uint8_t* blob, size_t len, const int32_t* slots, int n) {
  if (!blob || len < kBlobHeader || n < 0 || n > kBlobMaxRefs) return false;
  uint32_t head[4];
  std::memcpy(head, blob, sizeof(head));
  if (head[0] != kBlobMagic) return false;
  head[3] = static_cast<uint32_t>(n);
  std::memcpy(blob, head, sizeof(head));
  for (int i = 0; i < kBlobMaxRefs; ++i) {
    const int32_t s = i < n ? slots[i] : -1;
    std::memcpy(blob + 16 + 4 * i, &s, 4);
  }
  return true;
}

/* ---- C++ FrameSyntax <-> view ---------------------------------------------
 * FS is any struct with the reference's FrameSyntax field names. */

template <class FS>
void cpp_from_view(const av1b_frame_syntax& v, FS* s) {
  using Block = typename decltype(s->blocks)::value_type;
  using Tx = typename decltype(Block().transforms)::value_type;
  using Obmc = typename decltype(Block().obmc)::value_type;
  using Edge = typename decltype(s->deblock)::value_type;
  using Cdef = typename decltype(s->cdef)::value_type;
  using Unit = typename std::remove_reference<decltype(s->restoration[0])>::type::value_type;
  using Mode = decltype(Block().mode);
  using FiMode = decltype(Block().filter_intra_mode);
  using Filt = decltype(Block().filter);
  using Comp = decltype(Block().compound);
  using TxType = decltype(Tx().tx_type);
  using Matrix = decltype(s->color.matrix);
  using Range = decltype(s->color.range);

  s->width = v.width;
  s->coded_width = v.coded_width;
  s->height = v.height;
  s->bit_depth = v.bit_depth;
  s->ss_x = v.ss_x;
  s->ss_y = v.ss_y;
  s->base_q_idx = v.base_q_idx;
  s->sharpness = v.sharpness;
  s->enable_intra_edge_filter = v.enable_intra_edge_filter != 0;
  s->color.matrix = static_cast<Matrix>(v.color_matrix);
  s->color.range = static_cast<Range>(v.color_range);
  for (int i = 0; i < 7; ++i) {
    s->reference_width[i] = v.reference_width[i];
    s->reference_height[i] = v.reference_height[i];
  }
  for (int p = 0; p < 3; ++p) {
    s->restoration_type[p] = v.restoration_type[p];
    s->restoration_unit_log2[p] = v.restoration_unit_log2[p];
    s->restoration_unit_cols[p] = v.restoration_unit_cols[p];
  }
  s->reference_slots.assign(v.reference_slots, v.reference_slots + v.n_reference_slots);

  s->blocks.resize(v.n_blocks);
  for (size_t i = 0; i < v.n_blocks; ++i) {
    const av1b_block& a = v.blocks[i];
    Block& b = s->blocks[i];
    b.x = a.x; b.y = a.y; b.w = a.w; b.h = a.h;
    b.plane = a.plane;
    b.bit_depth = a.bit_depth;
    b.is_intra = a.is_intra != 0;
    b.intrabc = a.intrabc != 0;
    b.mode = static_cast<Mode>(a.mode);
    b.have_left = a.have_left != 0;
    b.have_above = a.have_above != 0;
    b.have_above_right = a.have_above_right;
    b.have_below_left = a.have_below_left;
    b.angle_delta = a.angle_delta;
    b.filter_type = a.filter_type;
    b.use_filter_intra = a.use_filter_intra != 0;
    b.filter_intra_mode = static_cast<FiMode>(a.filter_intra_mode);
    b.cfl_alpha = a.cfl_alpha;
    b.lossless = a.lossless != 0;
    b.use_palette = a.use_palette != 0;
    b.palette_size = a.palette_size;
    for (int k = 0; k < 8; ++k) b.palette[k] = a.palette[k];
    b.palette_off = a.palette_off;
    b.palette_stride = a.palette_stride;
    for (int k = 0; k < 2; ++k) {
      b.ref[k] = a.ref[k];
      b.mv[k][0] = a.mv[k][0];
      b.mv[k][1] = a.mv[k][1];
      b.blend[k] = a.blend[k];
      b.warp[k] = a.warp[k] != 0;
      b.mask_warp[k] = a.mask_warp[k] != 0;
      for (int j = 0; j < 6; ++j) b.warp_params[k][j] = a.warp_params[k][j];
    }
    b.filter = static_cast<Filt>(a.filter);
    b.filter_v = static_cast<Filt>(a.filter_v);
    b.motion_mode = a.motion_mode;
    b.compound = static_cast<Comp>(a.compound);
    b.wedge_index = a.wedge_index;
    b.mask_sign = a.mask_sign;
    b.interintra = a.interintra != 0;
    b.interintra_mode = a.interintra_mode;
    b.interintra_wedge = a.interintra_wedge != 0;
    b.residual_provided = a.residual_provided != 0;
    b.transforms.resize(a.tx_count > 0 ? a.tx_count : 0);
    for (int k = 0; k < a.tx_count; ++k) {
      const av1b_transform& t = v.transforms[a.tx_first + k];
      Tx& o = b.transforms[k];
      o.x = t.x; o.y = t.y; o.w = t.w; o.h = t.h;
      o.coef_offset = t.coef_offset;
      o.eob = t.eob;
      o.tx_type = static_cast<TxType>(t.tx_type);
      o.level_offset = t.level_offset;
      o.qindex = t.qindex;
      o.dc_step = t.dc_step;
      o.ac_step = t.ac_step;
      o.denominator = t.denominator;
      o.qm_off = t.qm_off;
    }
    b.obmc.resize(a.obmc_count > 0 ? a.obmc_count : 0);
    for (int k = 0; k < a.obmc_count; ++k) {
      const av1b_obmc& c = v.obmc[a.obmc_first + k];
      Obmc& o = b.obmc[k];
      o.pass = c.pass; o.x = c.x; o.y = c.y; o.w = c.w; o.h = c.h;
      o.mv[0] = c.mv[0];
      o.mv[1] = c.mv[1];
      o.filter = static_cast<Filt>(c.filter);
      o.filter_v = static_cast<Filt>(c.filter_v);
      o.ref = c.ref;
    }
  }
  s->coefficients.assign(v.coefficients, v.coefficients + v.n_coefficients);
  s->residual.assign(v.residual, v.residual + v.n_residual);
  s->levels.assign(v.levels, v.levels + v.n_levels);
  s->qm_pool.assign(v.qm_pool, v.qm_pool + v.n_qm_pool);
  s->palette_map.assign(v.palette_map, v.palette_map + v.n_palette_map);
  s->deblock.resize(v.n_deblock);
  for (size_t i = 0; i < v.n_deblock; ++i) {
    const av1b_deblock_edge& e = v.deblock[i];
    Edge& o = s->deblock[i];
    o.plane = e.plane; o.x = e.x; o.y = e.y;
    o.vertical = e.vertical != 0;
    o.length = e.length;
    o.level = e.level;
    o.filter_size = e.filter_size;
  }
  s->cdef.resize(v.n_cdef);
  for (size_t i = 0; i < v.n_cdef; ++i) {
    const av1b_cdef_block& c = v.cdef[i];
    Cdef& o = s->cdef[i];
    o.plane = c.plane; o.x = c.x; o.y = c.y;
    o.pri_strength = c.pri_strength;
    o.sec_strength = c.sec_strength;
    o.damping = c.damping;
    o.dir = c.dir;
  }
  for (int p = 0; p < 3; ++p) {
    s->restoration[p].resize(v.n_restoration[p]);
    for (size_t i = 0; i < v.n_restoration[p]; ++i) {
      const av1b_restoration_unit& u = v.restoration[p][i];
      Unit& o = s->restoration[p][i];
      o.type = u.type;
      for (int a = 0; a < 2; ++a)
        for (int k = 0; k < 3; ++k) o.wiener[a][k] = u.wiener[a][k];
      o.sgr_set = u.sgr_set;
      o.sgr_xqd[0] = u.sgr_xqd[0];
      o.sgr_xqd[1] = u.sgr_xqd[1];
    }
  }
  const av1b_film_grain& g = v.grain;
  auto& d = s->grain;
  d.apply = g.apply != 0;
  d.seed = g.seed;
  d.num_y_points = g.num_y_points;
  d.chroma_scaling_from_luma = g.chroma_scaling_from_luma != 0;
  d.num_cb_points = g.num_cb_points;
  d.num_cr_points = g.num_cr_points;
  for (int i = 0; i < 16; ++i) {
    d.point_y_value[i] = g.point_y_value[i];
    d.point_y_scaling[i] = g.point_y_scaling[i];
    d.point_cb_value[i] = g.point_cb_value[i];
    d.point_cb_scaling[i] = g.point_cb_scaling[i];
    d.point_cr_value[i] = g.point_cr_value[i];
    d.point_cr_scaling[i] = g.point_cr_scaling[i];
  }
  d.grain_scaling_minus_8 = g.grain_scaling_minus_8;
  d.ar_coeff_lag = g.ar_coeff_lag;
  for (int i = 0; i < 24; ++i) d.ar_coeffs_y[i] = g.ar_coeffs_y[i];
  for (int i = 0; i < 25; ++i) {
    d.ar_coeffs_cb[i] = g.ar_coeffs_cb[i];
    d.ar_coeffs_cr[i] = g.ar_coeffs_cr[i];
  }
  d.ar_coeff_shift_minus_6 = g.ar_coeff_shift_minus_6;
  d.grain_scale_shift = g.grain_scale_shift;
  d.cb_mult = g.cb_mult;
  d.cb_luma_mult = g.cb_luma_mult;
  d.cb_offset = g.cb_offset;
  d.cr_mult = g.cr_mult;
  d.cr_luma_mult = g.cr_luma_mult;
  d.cr_offset = g.cr_offset;
  d.overlap_flag = g.overlap_flag != 0;
  d.clip_to_restricted_range = g.clip_to_restricted_range != 0;
}

template <class FS>
void view_from_cpp(const FS& s, FlatSyntax* f) {
  av1b_frame_syntax& h = f->hdr;
  std::memset(&h, 0, sizeof(h));
  h.width = s.width;
  h.coded_width = s.coded_width;
  h.height = s.height;
  h.bit_depth = s.bit_depth;
  h.ss_x = s.ss_x;
  h.ss_y = s.ss_y;
  h.base_q_idx = s.base_q_idx;
  h.sharpness = s.sharpness;
  h.enable_intra_edge_filter = s.enable_intra_edge_filter ? 1 : 0;
  h.color_matrix = static_cast<int>(s.color.matrix);
  h.color_range = static_cast<int>(s.color.range);
  for (int i = 0; i < 7; ++i) {
    h.reference_width[i] = s.reference_width[i];
    h.reference_height[i] = s.reference_height[i];
  }
  for (int p = 0; p < 3; ++p) {
    h.restoration_type[p] = s.restoration_type[p];
    h.restoration_unit_log2[p] = s.restoration_unit_log2[p];
    h.restoration_unit_cols[p] = s.restoration_unit_cols[p];
  }
  f->reference_slots.assign(s.reference_slots.begin(), s.reference_slots.end());
  f->blocks.resize(s.blocks.size());
  f->transforms.clear();
  f->obmc.clear();
  for (size_t i = 0; i < s.blocks.size(); ++i) {
    const auto& b = s.blocks[i];
    av1b_block& a = f->blocks[i];
    std::memset(&a, 0, sizeof(a));
    a.x = b.x; a.y = b.y; a.w = b.w; a.h = b.h;
    a.plane = b.plane;
    a.bit_depth = b.bit_depth;
    a.is_intra = b.is_intra;
    a.intrabc = b.intrabc;
    a.mode = static_cast<int>(b.mode);
    a.have_left = b.have_left;
    a.have_above = b.have_above;
    a.have_above_right = b.have_above_right;
    a.have_below_left = b.have_below_left;
    a.angle_delta = b.angle_delta;
    a.filter_type = b.filter_type;
    a.use_filter_intra = b.use_filter_intra;
    a.filter_intra_mode = static_cast<int>(b.filter_intra_mode);
    a.cfl_alpha = b.cfl_alpha;
    a.lossless = b.lossless;
    a.use_palette = b.use_palette;
    a.palette_size = b.palette_size;
    for (int k = 0; k < 8; ++k) a.palette[k] = b.palette[k];
    a.palette_off = b.palette_off;
    a.palette_stride = b.palette_stride;
    for (int k = 0; k < 2; ++k) {
      a.ref[k] = b.ref[k];
      a.mv[k][0] = b.mv[k][0];
      a.mv[k][1] = b.mv[k][1];
      a.blend[k] = b.blend[k];
      a.warp[k] = b.warp[k];
      a.mask_warp[k] = b.mask_warp[k];
      for (int j = 0; j < 6; ++j) a.warp_params[k][j] = b.warp_params[k][j];
    }
    a.filter = static_cast<int>(b.filter);
    a.filter_v = static_cast<int>(b.filter_v);
    a.motion_mode = b.motion_mode;
    a.compound = static_cast<int>(b.compound);
    a.wedge_index = b.wedge_index;
    a.mask_sign = b.mask_sign;
    a.interintra = b.interintra;
    a.interintra_mode = b.interintra_mode;
    a.interintra_wedge = b.interintra_wedge;
    a.residual_provided = b.residual_provided;
    a.tx_first = static_cast<int32_t>(f->transforms.size());
    a.tx_count = static_cast<int32_t>(b.transforms.size());
    for (const auto& t : b.transforms) {
      av1b_transform o;
      o.x = t.x; o.y = t.y; o.w = t.w; o.h = t.h;
      o.coef_offset = t.coef_offset;
      o.eob = t.eob;
      o.tx_type = static_cast<int>(t.tx_type);
      o.level_offset = t.level_offset;
      o.qindex = t.qindex;
      o.dc_step = t.dc_step;
      o.ac_step = t.ac_step;
      o.denominator = t.denominator;
      o.qm_off = t.qm_off;
      f->transforms.push_back(o);
    }
    a.obmc_first = static_cast<int32_t>(f->obmc.size());
    a.obmc_count = static_cast<int32_t>(b.obmc.size());
    for (const auto& c : b.obmc) {
      av1b_obmc o;
      o.pass = c.pass; o.x = c.x; o.y = c.y; o.w = c.w; o.h = c.h;
      o.mv[0] = c.mv[0];
      o.mv[1] = c.mv[1];
      o.filter = static_cast<int>(c.filter);
      o.filter_v = static_cast<int>(c.filter_v);
      o.ref = c.ref;
      f->obmc.push_back(o);
    }
  }
  f->coefficients.assign(s.coefficients.begin(), s.coefficients.end());
  f->residual.assign(s.residual.begin(), s.residual.end());
  f->levels.assign(s.levels.begin(), s.levels.end());
  f->qm_pool.assign(s.qm_pool.begin(), s.qm_pool.end());
  f->palette_map.assign(s.palette_map.begin(), s.palette_map.end());
  f->deblock.resize(s.deblock.size());
  for (size_t i = 0; i < s.deblock.size(); ++i) {
    const auto& e = s.deblock[i];
    f->deblock[i] = av1b_deblock_edge{e.plane, e.x, e.y, e.vertical ? 1 : 0,
                                      e.length, e.level, e.filter_size};
  }
  f->cdef.resize(s.cdef.size());
  for (size_t i = 0; i < s.cdef.size(); ++i) {
    const auto& c = s.cdef[i];
    f->cdef[i] = av1b_cdef_block{c.plane, c.x, c.y, c.pri_strength, c.sec_strength,
                                 c.damping, c.dir};
  }
  for (int p = 0; p < 3; ++p) {
    f->restoration[p].resize(s.restoration[p].size());
    for (size_t i = 0; i < s.restoration[p].size(); ++i) {
      const auto& u = s.restoration[p][i];
      av1b_restoration_unit& o = f->restoration[p][i];
      o.type = u.type;
      for (int a = 0; a < 2; ++a)
        for (int k = 0; k < 3; ++k) o.wiener[a][k] = u.wiener[a][k];
      o.sgr_set = u.sgr_set;
      o.sgr_xqd[0] = u.sgr_xqd[0];
      o.sgr_xqd[1] = u.sgr_xqd[1];
    }
  }
  const auto& d = s.grain;
  av1b_film_grain& g = h.grain;
  g.apply = d.apply;
  g.seed = d.seed;
  g.num_y_points = d.num_y_points;
  g.chroma_scaling_from_luma = d.chroma_scaling_from_luma;
  g.num_cb_points = d.num_cb_points;
  g.num_cr_points = d.num_cr_points;
  for (int i = 0; i < 16; ++i) {
    g.point_y_value[i] = d.point_y_value[i];
    g.point_y_scaling[i] = d.point_y_scaling[i];
    g.point_cb_value[i] = d.point_cb_value[i];
    g.point_cb_scaling[i] = d.point_cb_scaling[i];
    g.point_cr_value[i] = d.point_cr_value[i];
    g.point_cr_scaling[i] = d.point_cr_scaling[i];
  }
  g.grain_scaling_minus_8 = d.grain_scaling_minus_8;
  g.ar_coeff_lag = d.ar_coeff_lag;
  for (int i = 0; i < 24; ++i) g.ar_coeffs_y[i] = d.ar_coeffs_y[i];
  for (int i = 0; i < 25; ++i) {
    g.ar_coeffs_cb[i] = d.ar_coeffs_cb[i];
    g.ar_coeffs_cr[i] = d.ar_coeffs_cr[i];
  }
  g.ar_coeff_shift_minus_6 = d.ar_coeff_shift_minus_6;
  g.grain_scale_shift = d.grain_scale_shift;
  g.cb_mult = d.cb_mult;
  g.cb_luma_mult = d.cb_luma_mult;
  g.cb_offset = d.cb_offset;
  g.cr_mult = d.cr_mult;
  g.cr_luma_mult = d.cr_luma_mult;
  g.cr_offset = d.cr_offset;
  g.overlap_flag = d.overlap_flag;
  g.clip_to_restricted_range = d.clip_to_restricted_range;
}

}  // namespace av1b

#endif  // AV1B_FLAT_SYNTAX_HPP
