/*
 * api_client.cpp - a client of the av1gpu::Decoder C++ API, written the way a
 * user of the reference library writes one: create, decode_reference into
 * reference slots, release, to_nv12 and the split nv12_pack_begin / wait /
 * release, plan_frame / decode_reference_planned.
 * The frames come from the workload generator as serialized syntax and are
 * rebuilt into av1gpu::FrameSyntax. Output: the decoded planes and NV12 bytes
 * of every frame, appended to a binary file the test compares with the oracle.
 *
 *   api_client <out.bin> <width> <height> <coded_width> <bitdepth> <sb> <tools> <seed> <frames>
 */
#include <cstdio>
#include <cstdlib>
#include <map>
#include <string>
#include <vector>

#include "av1b.h"
#include "av1b_synth.h"
#include "av1gpu/av1gpu.hpp"
#include "flat_syntax.hpp"

int main(int argc, char** argv) {
  if (argc < 10) return 2;
  FILE* out = std::fopen(argv[1], "wb");
  const int w = std::atoi(argv[2]), h = std::atoi(argv[3]), cw = std::atoi(argv[4]);
  const int bd = std::atoi(argv[5]), sb = std::atoi(argv[6]), tools = std::atoi(argv[7]);
  const unsigned long long seed = std::strtoull(argv[8], nullptr, 10);
  const int frames = std::atoi(argv[9]);
  std::string err;
  av1gpu::BackendOptions opt;
  opt.kind = av1gpu::BackendKind::CUDA;
  std::unique_ptr<av1gpu::Decoder> dec = av1gpu::Decoder::create(opt, &err);
  if (!dec) {
    std::fprintf(stderr, "create: %s\n", err.c_str());
    return 1;
  }
  std::map<int, int> slot_of;
  for (int k = 0; k < frames; ++k) {
    uint8_t* blob = nullptr;
    size_t len = 0;
    if (av1s_synth_frame_ex(w, h, cw, bd, sb, tools, seed, k, 30, &blob, &len) != 0) return 1;
    av1b_frame_syntax view;
    av1b_syntax_view(blob, len, &view);
    av1gpu::FrameSyntax s;
    av1b::cpp_from_view(view, &s);
    for (int& r : s.reference_slots) r = slot_of[k - r];  /* distances -> slots */
    av1gpu::Frame frame;
    int slot;
    if (k % 2 == 0) {
      slot = dec->decode_reference(s, &frame, &err);
    } else {
      /* the pipelined form: reserve, plan, decode the plan */
      slot = dec->reserve_reference();
      void* plan = nullptr;
      if (!dec->plan_frame(std::move(s), &plan, &err)) {
        std::fprintf(stderr, "plan: %s\n", err.c_str());
        return 1;
      }
      slot = dec->decode_reference_planned(plan, slot, &frame, &err);
    }
    av1s_blob_free(blob);
    if (slot < 0) {
      std::fprintf(stderr, "decode %d: %s\n", k, err.c_str());
      return 1;
    }
    slot_of[k] = slot;
    for (int p = 0; p < 3; ++p)
      for (int y = 0; y < frame.plane_height(p); ++y)
        std::fwrite(frame.plane(p) + static_cast<size_t>(y) * frame.stride[p], 2,
                    frame.plane_width(p), out);
    std::vector<uint8_t> nv12;
    const size_t pitch = (w + 63) & ~63;
    if (k % 2 == 0) {
      if (!dec->to_nv12(slot, pitch, &nv12, &err)) {
        std::fprintf(stderr, "to_nv12: %s\n", err.c_str());
        return 1;
      }
    } else {
      /* the split pack, the way a pipeline's output stage uses it */
      if (!dec->packs_nv12_on_device()) return 1;
      const int handle = dec->nv12_pack_begin(slot, pitch, &err);
      if (handle < 0 || !dec->nv12_pack_wait(handle, &nv12, &err)) {
        std::fprintf(stderr, "nv12_pack: %s\n", err.c_str());
        return 1;
      }
      dec->nv12_pack_release(handle);
    }
    std::fwrite(nv12.data(), 1, nv12.size(), out);
    if (k >= 3) dec->release_reference(slot_of[k - 3]);
  }
  std::fclose(out);
  std::printf("ok %d frames\n", frames);
  return 0;
}
