/*
 * ref_shim.cpp - a C entry surface over the reference's own CPU backend.
 *
 * TEST INFRASTRUCTURE ONLY. This file is compiled together with the
 * reference's sources (src/core/*.cpp, src/backends/cpu/cpu_backend.cpp) by
 * oracle/Makefile into oracle/_ref/libav1ref.so, with the reference namespace
 * renamed to av1ref so it can share a process with this repository's library.
 * Only tests/, the smoke check and bench.py's CPU baseline load it; nothing
 * in the product links it.
 *
 * Every call goes through the reference's public API: av1gpu::Decoder
 * (include/av1gpu/av1gpu.hpp:615-787) created with BackendKind::Cpu, which is
 * EngineDecoder over CpuBackend (engine.cpp:1509-1558, cpu_backend.cpp:645).
 * Frames arrive as the serialized av1b_frame_syntax blobs this repository's
 * tests and benchmark use, and are rebuilt into the reference's FrameSyntax
 * field by field (av1ongpu_b200/csrc/flat_syntax.hpp).
 */
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#if defined(_OPENMP)
#include <omp.h>
#endif

#include "av1gpu/av1gpu.hpp"
#include "av1gpu_kernels.h"
#include "flat_syntax.hpp"
#include "frontend/coef_model.hpp"
#include "frontend/dequant.hpp"

namespace {

struct RefDecoder {
  std::unique_ptr<av1gpu::Decoder> dec;
  av1gpu::Frame out;
  std::string error;
};

}  // namespace

extern "C" {

__attribute__((visibility("default"))) void av1ref_set_threads(int n) {
#if defined(_OPENMP)
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

__attribute__((visibility("default"))) int av1ref_max_threads(void) {
#if defined(_OPENMP)
  return omp_get_max_threads();
#else
  return 1;
#endif
}

__attribute__((visibility("default"))) void* av1ref_create(void) {
  av1gpu::BackendOptions opt;
  opt.kind = av1gpu::BackendKind::Cpu;
  opt.allow_cpu_fallback = true;
  std::string err;
  auto* r = new RefDecoder;
  r->dec = av1gpu::Decoder::create(opt, &err);
  if (!r->dec) {
    delete r;
    return nullptr;
  }
  return r;
}

__attribute__((visibility("default"))) void av1ref_destroy(void* h) {
  delete static_cast<RefDecoder*>(h);
}

/* Decodes one serialized frame. keep != 0: Decoder::decode_reference, the
 * return value is the slot; keep == 0: Decoder::decode, the return value is -1
 * on success. -2 means failure (av1ref_error has the message). When `out` is
 * not null the display planes are packed into it, plane after plane, each
 * plane_width * plane_height uint16 samples; `out_len` is its size in
 * samples. */
__attribute__((visibility("default"))) int av1ref_decode(void* h, const uint8_t* blob,
                                                         size_t len, int keep, uint16_t* out,
                                                         size_t out_len) {
  RefDecoder* r = static_cast<RefDecoder*>(h);
  av1b_frame_syntax view;
  if (!r || !av1b::view_blob(blob, len, &view)) return -2;
  av1gpu::FrameSyntax syntax;
  av1b::cpp_from_view(view, &syntax);
  int slot = -1;
  r->error.clear();
  if (keep) {
    slot = r->dec->decode_reference(syntax, &r->out, &r->error);
    if (slot < 0) return -2;
  } else {
    if (!r->dec->decode(syntax, &r->out, &r->error)) return -2;
  }
  if (out) {
    size_t pos = 0;
    for (int p = 0; p < 3; ++p) {
      const int pw = r->out.plane_width(p), ph = r->out.plane_height(p);
      if (pos + static_cast<size_t>(pw) * ph > out_len) return -2;
      for (int y = 0; y < ph; ++y) {
        std::memcpy(out + pos, r->out.plane(p) + static_cast<size_t>(y) * r->out.stride[p],
                    sizeof(uint16_t) * pw);
        pos += pw;
      }
    }
  }
  return slot;
}

__attribute__((visibility("default"))) const char* av1ref_error(void* h) {
  return h ? static_cast<RefDecoder*>(h)->error.c_str() : "";
}

__attribute__((visibility("default"))) void av1ref_release(void* h, int slot) {
  if (h) static_cast<RefDecoder*>(h)->dec->release_reference(slot);
}

__attribute__((visibility("default"))) int av1ref_to_nv12(void* h, int slot, size_t pitch,
                                                          uint8_t* out, size_t out_len) {
  RefDecoder* r = static_cast<RefDecoder*>(h);
  std::vector<uint8_t> bytes;
  if (!r || !r->dec->to_nv12(slot, pitch, &bytes, &r->error)) return -2;
  if (bytes.size() > out_len) return -2;
  std::memcpy(out, bytes.data(), bytes.size());
  return static_cast<int>(bytes.size());
}

__attribute__((visibility("default"))) int av1ref_to_rgb(void* h, int slot, int matrix,
                                                         int range, uint8_t* out,
                                                         size_t out_len) {
  RefDecoder* r = static_cast<RefDecoder*>(h);
  std::vector<uint8_t> bytes;
  if (!r || !r->dec->to_rgb(slot, static_cast<av1gpu::ColorMatrix>(matrix),
                            static_cast<av1gpu::ColorRange>(range), &bytes, &r->error))
    return -2;
  if (bytes.size() > out_len) return -2;
  std::memcpy(out, bytes.data(), bytes.size());
  return static_cast<int>(bytes.size());
}

/* DecodeStats of the last decode: reconstruct, filter, total milliseconds. */
__attribute__((visibility("default"))) void av1ref_stats(void* h, double* ms3, int* waves) {
  const av1gpu::DecodeStats& s = static_cast<RefDecoder*>(h)->dec->stats();
  ms3[0] = s.reconstruct_ms;
  ms3[1] = s.filter_ms;
  ms3[2] = s.total_ms;
  *waves = s.waves;
}

/* One 2-D inverse transform plus residual add, through the reference's
 * av1g_itx_row / av1g_itx_col_add (av1gpu_kernels.h:869-930), the way the CPU
 * backend runs a job (cpu_backend.cpp:319-325). `dst` is w*h samples, row
 * major, updated in place. */
__attribute__((visibility("default"))) void av1ref_itx(int w, int h, int tx_type, int lossless,
                                                       int row_shift, int bitdepth,
                                                       const int32_t* coef, uint16_t* dst) {
  Av1gItxJob job;
  std::memset(&job, 0, sizeof(job));
  job.coef_off = 0;
  job.tmp_off = 0;
  job.dst_off = 0;
  job.dst_stride = w;
  job.w = w;
  job.h = h;
  job.tx_type = tx_type;
  job.eob = 1;
  job.row_shift = row_shift;
  job.lossless = lossless;
  job.bitdepth = bitdepth;
  std::vector<int> tmp(static_cast<size_t>(w) * h + 64, 0);
  const int maxv = (1 << bitdepth) - 1;
  for (int y = 0; y < h; ++y) av1g_itx_row(&job, coef, tmp.data(), y);
  for (int x = 0; x < w; ++x) av1g_itx_col_add(&job, tmp.data(), dst, x, maxv);
}

/* The array lengths of a serialized frame, in av1b_frame_syntax order: blocks,
 * transforms, obmc, coefficients, residual, levels, qm_pool, palette_map,
 * deblock, cdef, and the restoration units of all three planes. Returns 11,
 * or -1 for a malformed blob. */
__attribute__((visibility("default"))) int av1ref_blob_counts(const uint8_t* blob, size_t len,
                                                              uint64_t* out) {
  av1b_frame_syntax v;
  if (!av1b::view_blob(blob, len, &v)) return -1;
  const size_t n[11] = {v.n_blocks,   v.n_transforms,   v.n_obmc,           v.n_coefficients,
                        v.n_residual, v.n_levels,       v.n_qm_pool,        v.n_palette_map,
                        v.n_deblock,  v.n_cdef,         v.n_restoration[0] + v.n_restoration[1] +
                                                            v.n_restoration[2]};
  for (int i = 0; i < 11; ++i) out[i] = n[i];
  return 11;
}

/* Test support for device dequantisation. From a frame that carries coded
 * levels, two serialized frames: `with_qm` is the frame with a quantiser
 * matrix pool (4096 bytes of values 1..255 drawn from `seed`; seed 0: all 32,
 * the identity) and a matrix on every transform that has levels, at a seeded
 * offset; `expanded` is that
 * same frame with the coefficient rasters the reference front end's host fill
 * builds from those levels (dequant.hpp:317-345, through its own coef_scan
 * and dequantise_level) and no levels. The caller frees both with
 * av1ref_free. Returns 0, or -1 for a malformed blob. */
__attribute__((visibility("default"))) int av1ref_dequant_pair(const uint8_t* blob, size_t len,
                                                               uint32_t seed, uint8_t** with_qm,
                                                               size_t* with_qm_len,
                                                               uint8_t** expanded,
                                                               size_t* expanded_len) {
  namespace fe = av1gpu::frontend;
  av1b_frame_syntax v;
  if (!av1b::view_blob(blob, len, &v)) return -1;
  std::vector<uint8_t> qm(4096);
  uint32_t x = seed * 2654435761u + 1;
  for (uint8_t& b : qm) {
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    b = seed ? static_cast<uint8_t>(1 + x % 255) : 32;
  }
  std::vector<av1b_transform> txs(v.transforms, v.transforms + v.n_transforms);
  size_t pool = 0;
  for (av1b_transform& t : txs) {
    const int aw = t.w < 32 ? t.w : 32, ah = t.h < 32 ? t.h : 32;
    pool = std::max(pool, static_cast<size_t>(t.coef_offset) + static_cast<size_t>(aw) * ah);
    if (t.eob <= 0) continue;
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    t.qm_off = static_cast<int32_t>(x % (4096 - aw * ah + 1));
  }
  std::vector<int32_t> coef(pool + 64, 0);
  for (const av1b_transform& t : txs) {
    if (t.eob <= 0) continue;
    fe::TxSize size;
    for (size.lw = 0; (4 << size.lw) < t.w; ++size.lw) {}
    for (size.lh = 0; (4 << size.lh) < t.h; ++size.lh) {}
    const fe::TxSize adjusted = fe::adjusted_tx_size(size);
    const int area = (4 << adjusted.lw) * (4 << adjusted.lh);
    const fe::ScanOrder scan = fe::coef_scan(adjusted, t.tx_type);
    const int count = t.eob < scan.count ? t.eob : scan.count;
    for (int i = 0; i < count; ++i) {
      const int pos = scan.at(i);
      if (pos < 0 || pos >= area) continue;
      const int level = v.levels[t.level_offset + i];
      if (level == 0) continue;
      int step = pos == 0 ? t.dc_step : t.ac_step;
      step = (step * qm[t.qm_off + pos] + 16) >> 5;
      coef[t.coef_offset + pos] = fe::dequantise_level(level, step, t.denominator, v.bit_depth);
    }
  }
  av1b_frame_syntax a = v;
  a.transforms = txs.data();
  a.qm_pool = qm.data();
  a.n_qm_pool = qm.size();
  av1b_frame_syntax b = a;
  b.levels = nullptr;
  b.n_levels = 0;
  b.coefficients = coef.data();
  b.n_coefficients = coef.size();
  std::vector<uint8_t> out_a, out_b;
  av1b::write_blob(a, &out_a);
  av1b::write_blob(b, &out_b);
  *with_qm = static_cast<uint8_t*>(std::malloc(out_a.size()));
  *expanded = static_cast<uint8_t*>(std::malloc(out_b.size()));
  std::memcpy(*with_qm, out_a.data(), out_a.size());
  std::memcpy(*expanded, out_b.data(), out_b.size());
  *with_qm_len = out_a.size();
  *expanded_len = out_b.size();
  return 0;
}

__attribute__((visibility("default"))) void av1ref_free(void* p) { std::free(p); }

/* Test support for stage-by-stage comparisons: a copy of a serialized frame
 * without some of its in-loop stages. `drop` bit 0: the deblocking edges,
 * bit 1: the CDEF blocks, bit 2: loop restoration (types and units), bit 3:
 * film grain. The caller frees the copy with av1ref_free. Returns 0, or -1
 * for a malformed blob. */
__attribute__((visibility("default"))) int av1ref_strip(const uint8_t* blob, size_t len, int drop,
                                                        uint8_t** out, size_t* out_len) {
  av1b_frame_syntax v;
  if (!av1b::view_blob(blob, len, &v)) return -1;
  if (drop & 1) v.n_deblock = 0;
  if (drop & 2) v.n_cdef = 0;
  if (drop & 4)
    for (int p = 0; p < 3; ++p) {
      v.restoration_type[p] = 0;
      v.n_restoration[p] = 0;
    }
  if (drop & 8) v.grain.apply = 0;
  std::vector<uint8_t> bytes;
  av1b::write_blob(v, &bytes);
  *out = static_cast<uint8_t*>(std::malloc(bytes.size()));
  std::memcpy(*out, bytes.data(), bytes.size());
  *out_len = bytes.size();
  return 0;
}

/* Test support for the error paths: a copy of a serialized frame with one
 * record made invalid. `what` 1: deblocking edge `index` gets level 99;
 * 2: edge `index` reaches outside the picture; 3: CDEF block `index` gets
 * direction 9; 4: the luma restoration unit size becomes 8 samples (log2 3);
 * 5: film grain is switched on with a seed out of range. The caller frees the
 * copy with av1ref_free. Returns 0, or -1 for a malformed blob or index. */
__attribute__((visibility("default"))) int av1ref_corrupt(const uint8_t* blob, size_t len, int what,
                                                          size_t index, uint8_t** out,
                                                          size_t* out_len) {
  av1b_frame_syntax v;
  if (!av1b::view_blob(blob, len, &v)) return -1;
  std::vector<av1b_deblock_edge> edges(v.deblock, v.deblock + v.n_deblock);
  std::vector<av1b_cdef_block> cdef(v.cdef, v.cdef + v.n_cdef);
  if ((what == 1 || what == 2) && index >= edges.size()) return -1;
  if (what == 3 && index >= cdef.size()) return -1;
  if (what == 1 || what == 2) edges[index].length = std::max(edges[index].length, 4);
  if (what == 1) edges[index].level = 99;
  if (what == 2) {
    edges[index].x = -64;
    edges[index].vertical = 1;
    edges[index].level = 10;
  }
  if (what == 3) cdef[index].dir = 9;
  if (what == 4) {
    v.restoration_type[0] = 1;
    v.restoration_unit_log2[0] = 3;
  }
  if (what == 5) {
    v.grain.apply = 1;
    v.grain.seed = -1;
  }
  v.deblock = edges.data();
  v.cdef = cdef.data();
  std::vector<uint8_t> bytes;
  av1b::write_blob(v, &bytes);
  *out = static_cast<uint8_t*>(std::malloc(bytes.size()));
  std::memcpy(*out, bytes.data(), bytes.size());
  *out_len = bytes.size();
  return 0;
}

/* FNV-1a 64 over `n` bytes, seeded with `h` (0xcbf29ce484222325 to start): the
 * frame hash of the reference's stream tests (tools/av1gpu_decode.cpp:131-140),
 * chainable so a picture can be hashed plane by plane. */
__attribute__((visibility("default"))) uint64_t av1ref_fnv1a64(uint64_t h, const uint8_t* p,
                                                               size_t n) {
  for (size_t i = 0; i < n; ++i) {
    h ^= p[i];
    h *= 0x100000001b3ull;
  }
  return h;
}

}  // extern "C"
