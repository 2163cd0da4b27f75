/*
 * stream_dump.cpp - real-stream replay fixtures for the parity tests.
 *
 * TEST INFRASTRUCTURE ONLY. Built by oracle/Makefile (target `streams`) from
 * the reference's own front end and CPU backend, compiled where they lie; the
 * binary and what it writes stay under oracle/_ref/. Nothing in the product
 * links or runs it.
 *
 *   stream_dump IN.ivf --frames N [--yuv16] --hashes IN.hash -o OUT.av1s
 *
 * It decodes the stream the way the reference's decode tool does
 * (tools/av1gpu_decode.cpp:383-785): the OBU walk, the frame and tile headers,
 * the tile decoder, the dequantiser and the planner of src/frontend produce one
 * FrameSyntax per coded frame, and the reference CPU Decoder
 * (av1gpu::Decoder, BackendKind::Cpu) reconstructs it, with the tool's
 * reference pool: the AV1 slots a frame refreshes but does not read are
 * released before it is decoded (av1gpu_decode.cpp:681-702), the refreshed
 * slots take the new picture afterwards (768-781), and a show_existing_frame
 * re-emits a picture decoded earlier (506-518). Every shown picture is hashed
 * (FNV-1a 64 over 8-bit planar samples, or 16-bit little endian ones with
 * --yuv16; av1gpu_decode.cpp:131-140, factory.cpp:194-233) and checked against
 * the stream's recorded hash list; a mismatch or a short output is an error,
 * so a fixture is only written when the reference itself decodes the stream
 * bit exactly.
 *
 * The fixture records every Decoder call in call order, with each frame as
 * this repository's serialized av1b_frame_syntax blob (the reference slots in
 * the blob are the CPU decoder's slot numbers; a replay maps them onto its own
 * decoder's), plus the expected hash list:
 *
 *   header  "AV1S", u32 version (1), u32 flags (bit 0: 16-bit hashes),
 *           u32 n_hashes, u32 n_events, u32 reserved[3], u64 hashes[n_hashes]
 *   event   u32 kind, i32 a, i32 b, u32 reserved, u64 len, then len bytes
 *     kind 1 decode_reference: a = the slot it returned, b = 1 when the
 *            picture is shown, the bytes are the blob
 *     kind 2 release_reference: a = the slot
 *     kind 3 show_existing_frame: a = the index (in decode order, from 0) of
 *            the decode whose picture is shown again
 *
 * With --levels the frames are planned the way the reference pipeline plans
 * them for a device dequantiser (the planner overload that moves the coded
 * levels into the syntax, reconstruct.hpp:1033-1040): the blobs carry
 * `levels` with the per-transform steps and QM offsets, and an empty
 * coefficient pool, which is what dequant.hpp:200-210's levels_only leaves
 * (the offsets are the same prefix sums either way). The reference CPU
 * backend only reads a dequantised pool, so the pool is still built for its
 * decode and the hash check, and dropped from the recorded blob.
 */
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "av1gpu/av1gpu.hpp"
#include "frontend/dequant.hpp"
#include "frontend/headers.hpp"
#include "frontend/tile_decoder.hpp"

/* reconstruct.hpp:1029 and :1039 pass `std::move(quant)` to a function that
 * takes `DequantisedTile&`, which only MSVC accepts. An overload taking the
 * rvalue, declared before the header is read, is what those two calls resolve
 * to under GCC; it forwards to the header's own function unchanged. */
namespace av1gpu {
namespace frontend {
struct ReferenceInfo;
bool plan_from_tile_impl(const SequenceHeader& seq, const FrameHeader& frame,
                         const TileDecodeResult& tile, TileDecodeResult* levels_from,
                         DequantisedTile&& quant, FrameSyntax* out, std::string* error,
                         const ReferenceInfo* refs);
}  // namespace frontend
}  // namespace av1gpu

#include "frontend/ivf.hpp"
#include "frontend/obu.hpp"
#include "frontend/reconstruct.hpp"
#include "frontend/tiles.hpp"

#include "flat_syntax.hpp"

namespace av1gpu {
namespace frontend {
bool plan_from_tile_impl(const SequenceHeader& seq, const FrameHeader& frame,
                         const TileDecodeResult& tile, TileDecodeResult* levels_from,
                         DequantisedTile&& quant, FrameSyntax* out, std::string* error,
                         const ReferenceInfo* refs) {
  DequantisedTile& pool = quant;
  return plan_from_tile_impl(seq, frame, tile, levels_from, pool, out, error, refs);
}
}  // namespace frontend
}  // namespace av1gpu

namespace {

using namespace av1gpu;
using namespace av1gpu::frontend;

struct Args {
  std::string input, hashes, output;
  int frames = -1;
  bool yuv16 = false;
  bool levels = false;
};

enum EventKind : uint32_t { kDecode = 1, kRelease = 2, kShowExisting = 3 };

struct Recorder {
  std::vector<uint8_t> bytes;
  uint32_t events = 0;

  void put(const void* p, size_t n) {
    const uint8_t* b = static_cast<const uint8_t*>(p);
    bytes.insert(bytes.end(), b, b + n);
  }
  void event(uint32_t kind, int32_t a, int32_t b, const std::vector<uint8_t>* payload) {
    const uint32_t reserved = 0;
    const uint64_t len = payload ? payload->size() : 0;
    put(&kind, 4);
    put(&a, 4);
    put(&b, 4);
    put(&reserved, 4);
    put(&len, 8);
    if (len) put(payload->data(), len);
    ++events;
  }
};

bool load(const std::string& path, std::vector<uint8_t>* out) {
  std::FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  uint8_t buf[1 << 16];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) out->insert(out->end(), buf, buf + n);
  const bool bad = std::ferror(f) != 0;
  std::fclose(f);
  return !bad;
}

/* "frame N: 0x..." lines; '#' comments and anything else are skipped. */
bool load_hashes(const std::string& path, std::vector<uint64_t>* out) {
  std::FILE* f = std::fopen(path.c_str(), "r");
  if (!f) return false;
  char line[512];
  while (std::fgets(line, sizeof(line), f)) {
    unsigned long long index = 0, h = 0;
    const char* p = line;
    while (*p == ' ' || *p == '\t') ++p;
    if (std::sscanf(p, "frame %llu: 0x%llx", &index, &h) == 2) out->push_back(h);
  }
  std::fclose(f);
  return true;
}

uint64_t picture_hash(const Frame& pic, bool yuv16) {
  std::vector<uint8_t> bytes;
  if (yuv16)
    frame_to_yuv16(pic, &bytes);
  else
    frame_to_yuv8(pic, &bytes);
  uint64_t h = 0xcbf29ce484222325ull;
  for (uint8_t b : bytes) {
    h ^= b;
    h *= 0x100000001b3ull;
  }
  return h;
}

int run(const Args& args) {
  std::vector<uint8_t> file;
  std::string error;
  if (!load(args.input, &file)) {
    std::fprintf(stderr, "stream_dump: cannot read %s\n", args.input.c_str());
    return 2;
  }
  std::vector<uint64_t> expected;
  if (!load_hashes(args.hashes, &expected) || expected.empty()) {
    std::fprintf(stderr, "stream_dump: no hashes in %s\n", args.hashes.c_str());
    return 2;
  }

  std::vector<IvfFrame> units;
  IvfReader reader;
  if (!reader.open(file, &error)) {
    std::fprintf(stderr, "stream_dump: %s\n", error.c_str());
    return 1;
  }
  IvfFrame unit;
  while (reader.next(&unit, &error)) {
    units.push_back(unit);
    if (args.frames >= 0 && static_cast<int>(units.size()) >= args.frames) break;
  }
  if (!error.empty()) {
    std::fprintf(stderr, "stream_dump: %s\n", error.c_str());
    return 1;
  }

  BackendOptions options;
  options.kind = BackendKind::Cpu;
  options.allow_cpu_fallback = true;
  std::unique_ptr<Decoder> decoder = Decoder::create(options, &error);
  if (!decoder) {
    std::fprintf(stderr, "stream_dump: %s\n", error.c_str());
    return 1;
  }

  Recorder rec;
  std::vector<uint64_t> got;
  SequenceHeader seq;
  bool have_seq = false;
  RefPool refs;
  int pool_slot[8];
  int pool_decode[8];
  Frame pool_picture[8];
  for (int i = 0; i < 8; ++i) pool_slot[i] = pool_decode[i] = -1;
  int decodes = 0;

  auto release_if_unused = [&](int slot) {
    if (slot < 0) return;
    for (int i = 0; i < 8; ++i)
      if (pool_slot[i] == slot) return;
    decoder->release_reference(slot);
    rec.event(kRelease, slot, 0, nullptr);
  };

  for (size_t index = 0; index < units.size(); ++index) {
    std::vector<Obu> obus;
    if (!split_obus(units[index].payload.data(), units[index].payload.size(), &obus, &error)) {
      std::fprintf(stderr, "stream_dump: unit %zu: %s\n", index, error.c_str());
      return 1;
    }
    for (const Obu& obu : obus) {
      if (obu.type == ObuType::SequenceHeader) {
        if (parse_sequence_header(obu.data, obu.size, &seq, &error) == ParseStatus::Invalid) {
          std::fprintf(stderr, "stream_dump: %s\n", error.c_str());
          return 1;
        }
        have_seq = true;
        continue;
      }
      if (obu.type != ObuType::FrameHeader && obu.type != ObuType::Frame &&
          obu.type != ObuType::RedundantFrameHeader)
        continue;
      if (!have_seq) {
        std::fprintf(stderr, "stream_dump: frame before any sequence header\n");
        return 1;
      }
      FrameHeader frame;
      const ParseStatus parsed =
          parse_frame_header(seq, obu.data, obu.size, &frame, &error, &refs);
      if (parsed == ParseStatus::Invalid) {
        std::fprintf(stderr, "stream_dump: unit %zu: %s\n", index, error.c_str());
        return 1;
      }
      if (parsed == ParseStatus::Unsupported) {
        /* the decode tool skips such a frame as well; the hash check below
         * then fails, so no fixture is written for the stream */
        std::fprintf(stderr, "stream_dump: unit %zu: %s\n", index, error.c_str());
        refresh_ref_pool(frame, &refs);
        continue;
      }
      if (frame.show_existing_frame) {
        const int which = frame.existing_frame_idx;
        if (which < 0 || which >= 8 || pool_decode[which] < 0) {
          std::fprintf(stderr, "stream_dump: unit %zu shows an empty slot\n", index);
          return 1;
        }
        rec.event(kShowExisting, pool_decode[which], 0, nullptr);
        got.push_back(picture_hash(pool_picture[which], args.yuv16));
        continue;
      }

      TileGroup group;
      if (parse_tile_group(seq, frame, obu.data, obu.size, &group, &error) != ParseStatus::Ok ||
          !tile_group_is_complete(frame, group)) {
        std::fprintf(stderr, "stream_dump: unit %zu: tile group: %s\n", index, error.c_str());
        return 1;
      }
      TileDecodeResult decoded;
      if (decode_tiles(seq, frame, &refs, group.tiles.data(), group.tiles.size(), obu.data,
                       obu.size, &decoded, &error) != ParseStatus::Ok) {
        std::fprintf(stderr, "stream_dump: unit %zu: tile: %s\n", index,
                     decoded.stop_reason.empty() ? error.c_str() : decoded.stop_reason.c_str());
        return 1;
      }
      DequantisedTile quant;
      dequantise_tile(frame, seq.bit_depth, decoded, &quant);

      ReferenceInfo info;
      for (int i = 0; i < 7; ++i) {
        const int which = frame.ref_frame_idx[i];
        if (which < 0 || which >= 8 || !refs.slots[which].valid) continue;
        info.slot[i] = pool_slot[which];
        info.width[i] = refs.slots[which].width;
        info.height[i] = refs.slots[which].height;
        info.upscaled_width[i] = refs.slots[which].upscaled_width > 0
                                     ? refs.slots[which].upscaled_width
                                     : refs.slots[which].width;
      }

      FrameSyntax syntax;
      bool planned;
      if (args.levels) {
        /* the coded levels move into the syntax: keep what the reference pool
         * refresh below still reads */
        auto ref_mvs = decoded.ref_mvs;
        auto cdf = decoded.cdf;
        auto seg_map = decoded.seg_map;
        planned = plan_from_tile(seq, frame, std::move(decoded), std::move(quant), &syntax,
                                 &error, &info);
        decoded.ref_mvs = ref_mvs;
        decoded.cdf = cdf;
        decoded.seg_map = seg_map;
      } else {
        const TileDecodeResult& tile = decoded;
        planned = plan_from_tile(seq, frame, tile, std::move(quant), &syntax, &error, &info);
      }
      if (!planned) {
        std::fprintf(stderr, "stream_dump: unit %zu: plan: %s\n", index, error.c_str());
        return 1;
      }

      for (int i = 0; i < 8; ++i) {
        if (!(frame.refresh_frame_flags & (1 << i))) continue;
        bool read = false;
        for (int j = 0; j < 7; ++j) read = read || frame.ref_frame_idx[j] == i;
        if (read) continue;
        const int freed = pool_slot[i];
        pool_slot[i] = -1;
        pool_decode[i] = -1;
        release_if_unused(freed);
      }

      av1b::FlatSyntax flat;
      av1b::view_from_cpp(syntax, &flat);
      /* the reference CPU backend reads the dequantised pool, so it is built
       * for the hash check; a device-dequantiser frame travels without it */
      if (args.levels) flat.coefficients.clear();
      std::vector<uint8_t> blob;
      av1b::write_blob(flat.view(), &blob);

      Frame picture;
      const int slot = decoder->decode_reference(syntax, &picture, &error);
      if (slot < 0) {
        std::fprintf(stderr, "stream_dump: unit %zu: decode: %s\n", index, error.c_str());
        return 1;
      }
      rec.event(kDecode, slot, frame.show_frame ? 1 : 0, &blob);
      const int this_decode = decodes++;
      if (frame.show_frame) got.push_back(picture_hash(picture, args.yuv16));

      bool kept = false;
      for (int i = 0; i < 8; ++i) {
        if (!(frame.refresh_frame_flags & (1 << i))) continue;
        const int previous = pool_slot[i];
        pool_slot[i] = -1;
        release_if_unused(previous);
        pool_slot[i] = slot;
        pool_decode[i] = this_decode;
        pool_picture[i] = picture;
        kept = true;
      }
      if (!kept) release_if_unused(slot);
      refresh_ref_pool(frame, &refs, decoded.ref_mvs, decoded.cdf, decoded.seg_map);
    }
  }

  size_t bad = got.size() == expected.size() ? 0 : 1;
  for (size_t i = 0; i < got.size() && i < expected.size(); ++i) {
    if (got[i] != expected[i]) {
      if (bad < 4)
        std::fprintf(stderr, "stream_dump: frame %zu: 0x%016llx, expected 0x%016llx\n", i,
                     static_cast<unsigned long long>(got[i]),
                     static_cast<unsigned long long>(expected[i]));
      ++bad;
    }
  }
  if (bad) {
    std::fprintf(stderr, "stream_dump: %s: %zu shown frame(s), %zu hash(es), %zu mismatch(es)\n",
                 args.input.c_str(), got.size(), expected.size(), bad);
    return 1;
  }

  std::vector<uint8_t> out;
  const uint32_t head[8] = {0x53315641u /* "AV1S" */, 1, args.yuv16 ? 1u : 0u,
                            static_cast<uint32_t>(expected.size()), rec.events, 0, 0, 0};
  out.resize(sizeof(head) + expected.size() * 8);
  std::memcpy(out.data(), head, sizeof(head));
  std::memcpy(out.data() + sizeof(head), expected.data(), expected.size() * 8);
  out.insert(out.end(), rec.bytes.begin(), rec.bytes.end());
  std::FILE* f = std::fopen(args.output.c_str(), "wb");
  if (!f || std::fwrite(out.data(), 1, out.size(), f) != out.size()) {
    std::fprintf(stderr, "stream_dump: cannot write %s\n", args.output.c_str());
    if (f) std::fclose(f);
    return 2;
  }
  std::fclose(f);
  std::printf("%s: %d decode(s), %zu shown frame(s) bit exact, %zu bytes\n", args.input.c_str(),
              decodes, got.size(), out.size());
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  Args args;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--frames" && i + 1 < argc)
      args.frames = std::atoi(argv[++i]);
    else if (a == "--hashes" && i + 1 < argc)
      args.hashes = argv[++i];
    else if (a == "-o" && i + 1 < argc)
      args.output = argv[++i];
    else if (a == "--yuv16")
      args.yuv16 = true;
    else if (a == "--levels")
      args.levels = true;
    else if (!a.empty() && a[0] != '-')
      args.input = a;
    else {
      std::fprintf(stderr, "usage: stream_dump IN.ivf --frames N [--yuv16] [--levels] "
                           "--hashes IN.hash -o OUT.av1s\n");
      return 2;
    }
  }
  if (args.input.empty() || args.hashes.empty() || args.output.empty()) {
    std::fprintf(stderr, "stream_dump: IN.ivf, --hashes and -o are required\n");
    return 2;
  }
  return run(args);
}
