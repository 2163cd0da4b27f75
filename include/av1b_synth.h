/*
 * av1b_synth.h - the seeded synthetic workload generator (libav1synth.so).
 *
 * The reference measures its decoder on a synthetic clip made by its own
 * encoder (src/core/synthetic.cpp, driven by tools/av1gpu_bench.cpp:113-147).
 * This generator replaces it for the benchmark configurations: every tool of
 * the reconstruction path, from a seed, as serialized FrameSyntax blobs
 * (the byte image av1b_syntax_view reads, include/av1b.h). It is a library of
 * its own, apart from the decoder, so that a process that only needs the
 * workload - the timed CPU reference, a tool writing fixtures - maps no
 * decoder code.
 *
 * A frame lists its references as frame *distances* (1 = the previous frame);
 * the caller rewrites them into its own slot ids (av1b_blob_set_refs, or the
 * blob header directly: u32 magic, version, reserved, count, then eight int32
 * slots at byte 16). Buffers are owned by the library: release them with
 * av1s_blob_free.
 */
#ifndef AV1B_SYNTH_H
#define AV1B_SYNTH_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define AV1S_API __attribute__((visibility("default")))
#else
#define AV1S_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Frame `frame_index` of workload `config` (1: 1280x720 8-bit, one reference;
 * 2: 1920x1080 10-bit, every tool, key frame every 30; 3: coded 2880x2160
 * superres to 3840x2160 10-bit, 128x128 superblocks, every tool), its picture
 * size divided by `scale` (1 = full size). */
AV1S_API int av1s_synth_frame(int config, int scale, uint64_t seed, int frame_index, uint8_t** blob,
                              size_t* len);
/* A frame of any geometry: `tools` is a mask of the generator's tool bits
 * (compound prediction among them selects up to three references), a key
 * frame every `key_interval` frames (0: only the first). */
AV1S_API int av1s_synth_frame_ex(int width, int height, int coded_width, int bit_depth, int sb_size,
                                 int tools, uint64_t seed, int frame_index, int key_interval,
                                 uint8_t** blob, size_t* len);
/* The same with the number of reference slots an inter frame draws from set
 * explicitly (1..3). */
AV1S_API int av1s_synth_frame_refs(int width, int height, int coded_width, int bit_depth,
                                   int sb_size, int tools, int max_refs, uint64_t seed,
                                   int frame_index, int key_interval, uint8_t** blob, size_t* len);
AV1S_API void av1s_blob_free(uint8_t* blob);

#ifdef __cplusplus
}
#endif

#endif /* AV1B_SYNTH_H */
