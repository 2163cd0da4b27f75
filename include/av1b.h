/*
 * av1b.h - the C ABI of the B200 AV1 reconstruction backend.
 *
 * The reference library (trprkkk/AV1onGPU) exposes its reconstruction path as
 * the C++ class av1gpu::Decoder (include/av1gpu/av1gpu.hpp:615-787) fed with
 * av1gpu::FrameSyntax (av1gpu.hpp:476-537). It ships no foreign-function
 * binding. This header is the binding a non-C++ caller (ctypes, cgo, JNI,
 * N-API) would use: every entry point maps one Decoder method, takes plain
 * pointers and sizes, never throws and returns AV1B_OK or a negative code.
 * The C++ class in include/av1gpu/av1gpu.hpp is implemented on top of it in
 * the same shared library.
 *
 * FrameSyntax crosses the boundary as av1b_frame_syntax: the scalar fields of
 * the reference struct plus (pointer, count) pairs for each of its vectors.
 * The per-block vectors (BlockSyntax::transforms, BlockSyntax::obmc) are
 * flattened into frame-wide arrays addressed by (first, count) in each block,
 * which is the layout the device upload wants anyway.
 *
 * Thread safety: one decoder is driven by one thread at a time; different
 * decoders may be used from different threads.
 */
#ifndef AV1B_H
#define AV1B_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define AV1B_API __attribute__((visibility("default")))
#else
#define AV1B_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define AV1B_OK 0
#define AV1B_ERR_ARG (-1)        /* a null pointer, a bad size or slot     */
#define AV1B_ERR_CUDA (-2)       /* a CUDA call failed                     */
#define AV1B_ERR_NOMEM (-3)      /* the HBM budget or the slot pool is out */
#define AV1B_ERR_SYNTAX (-4)     /* the frame syntax is inconsistent        */
#define AV1B_ERR_TIMEOUT (-5)    /* a device-side dependency wait gave up   */
#define AV1B_ERR_UNSUPPORTED (-6)
#define AV1B_ERR_NO_DEVICE (-7)  /* no CUDA device: there is no CPU fallback */

/* TransformBlock (av1gpu.hpp:187-208). */
typedef struct av1b_transform {
  int32_t x, y, w, h;
  int32_t coef_offset;
  int32_t eob;
  int32_t tx_type;
  int32_t level_offset, qindex;
  int32_t dc_step, ac_step, denominator, qm_off;
} av1b_transform;

/* ObmcCandidate (av1gpu.hpp:215-225). */
typedef struct av1b_obmc {
  int32_t pass, x, y, w, h;
  int32_t mv[2];
  int32_t filter, filter_v;
  int32_t ref;
} av1b_obmc;

/* BlockSyntax (av1gpu.hpp:229-342), booleans as 0/1 ints, the two vectors as
 * ranges of the frame-wide transform and OBMC arrays. */
typedef struct av1b_block {
  int32_t x, y, w, h, plane, bit_depth;
  int32_t is_intra, intrabc;
  int32_t mode;
  int32_t have_left, have_above, have_above_right, have_below_left;
  int32_t angle_delta, filter_type;
  int32_t use_filter_intra, filter_intra_mode;
  int32_t cfl_alpha;
  int32_t lossless;
  int32_t use_palette, palette_size, palette[8], palette_off, palette_stride;
  int32_t ref[2];
  int32_t mv[2][2];
  int32_t filter, filter_v;
  int32_t motion_mode, compound;
  int32_t blend[2];
  int32_t wedge_index, mask_sign;
  int32_t interintra, interintra_mode, interintra_wedge;
  int32_t warp[2];
  int32_t warp_params[2][6];
  int32_t mask_warp[2];
  int32_t residual_provided;
  int32_t tx_first, tx_count;     /* into av1b_frame_syntax::transforms */
  int32_t obmc_first, obmc_count; /* into av1b_frame_syntax::obmc       */
} av1b_block;

/* DeblockEdge (av1gpu.hpp:347-358). */
typedef struct av1b_deblock_edge {
  int32_t plane, x, y, vertical, length, level, filter_size;
} av1b_deblock_edge;

/* CdefBlock (av1gpu.hpp:361-369). */
typedef struct av1b_cdef_block {
  int32_t plane, x, y, pri_strength, sec_strength, damping, dir;
} av1b_cdef_block;

/* RestorationUnit (av1gpu.hpp:418-426). */
typedef struct av1b_restoration_unit {
  int32_t type;
  int32_t wiener[2][3];
  int32_t sgr_set;
  int32_t sgr_xqd[2];
} av1b_restoration_unit;

/* FilmGrainParams (av1gpu.hpp:434-468). */
typedef struct av1b_film_grain {
  int32_t apply, seed;
  int32_t num_y_points, point_y_value[16], point_y_scaling[16];
  int32_t chroma_scaling_from_luma;
  int32_t num_cb_points, point_cb_value[16], point_cb_scaling[16];
  int32_t num_cr_points, point_cr_value[16], point_cr_scaling[16];
  int32_t grain_scaling_minus_8;
  int32_t ar_coeff_lag;
  int32_t ar_coeffs_y[24], ar_coeffs_cb[25], ar_coeffs_cr[25];
  int32_t ar_coeff_shift_minus_6, grain_scale_shift;
  int32_t cb_mult, cb_luma_mult, cb_offset;
  int32_t cr_mult, cr_luma_mult, cr_offset;
  int32_t overlap_flag, clip_to_restricted_range;
} av1b_film_grain;

/* FrameSyntax (av1gpu.hpp:476-537): the scalars and one (pointer, count) per
 * vector. Nothing is retained after the call that takes it returns.
 *
 * Coefficients arrive one of two ways. A frame with n_levels == 0 brings its
 * dequantised rasters in `coefficients` (TransformBlock::coef_offset). A frame
 * with coded levels (n_levels > 0, as the reference front end leaves them with
 * its levels_only dequantiser, dequant.hpp:200-210) is dequantised on the
 * device from `levels` (level_offset, eob), the per-transform dc_step,
 * ac_step, denominator and qm_off into `qm_pool`; its `coefficients`, if
 * any, are then not read - the reference engine's device-dequantiser path
 * (engine.cpp:386, 655-670). */
typedef struct av1b_frame_syntax {
  int32_t width, coded_width, height, bit_depth, ss_x, ss_y;
  int32_t base_q_idx, sharpness, enable_intra_edge_filter;
  int32_t color_matrix, color_range;
  int32_t reference_width[7], reference_height[7];
  int32_t restoration_type[3], restoration_unit_log2[3], restoration_unit_cols[3];
  av1b_film_grain grain;

  const int32_t* reference_slots;          size_t n_reference_slots;
  const av1b_block* blocks;                size_t n_blocks;
  const av1b_transform* transforms;        size_t n_transforms;
  const av1b_obmc* obmc;                   size_t n_obmc;
  const int32_t* coefficients;             size_t n_coefficients;
  const int32_t* residual;                 size_t n_residual;
  const int16_t* levels;                   size_t n_levels;
  const uint8_t* qm_pool;                  size_t n_qm_pool;
  const uint8_t* palette_map;              size_t n_palette_map;
  const av1b_deblock_edge* deblock;        size_t n_deblock;
  const av1b_cdef_block* cdef;             size_t n_cdef;
  const av1b_restoration_unit* restoration[3];
  size_t n_restoration[3];
} av1b_frame_syntax;

/* Frame (av1gpu.hpp:77-109) as three caller-owned planes of uint16 samples.
 * `stride` is in samples. Plane sizes follow Frame::plane_width/height. */
typedef struct av1b_planes {
  uint16_t* plane[3];
  int32_t stride[3];
} av1b_planes;

/* DecodeStats (av1gpu.hpp:544-552). */
typedef struct av1b_stats {
  int32_t blocks, waves, kernel_launches;
  double reconstruct_ms, filter_ms, readback_ms, total_ms;
} av1b_stats;

typedef struct av1b_decoder av1b_decoder;

/* --- serialized syntax (a flat byte image of av1b_frame_syntax) ------------
 * A test fixture, a file, or a process boundary carries a frame as one byte
 * buffer. av1b_syntax_view points a view at such a buffer without copying. The
 * buffer must stay alive and unmodified while the view is used. */
AV1B_API int av1b_syntax_view(const uint8_t* blob, size_t len, av1b_frame_syntax* out);

/* --- decoder lifetime: Decoder::create (engine.cpp:1509-1558) -------------- */
/* `device` is the CUDA ordinal. `hbm_budget_bytes` caps what the decoder may
 * allocate (0: no cap). A missing device is an error (AV1B_ERR_NO_DEVICE):
 * there is no CPU path in this library. */
AV1B_API int av1b_decoder_create(int device, size_t hbm_budget_bytes, av1b_decoder** out);
/* The same with the decoder's host planning resources set: `planners` frames
 * planned at once (1..8; 0: 3) by `planner_threads` host threads each
 * (0: all cores but one, at most 16). A process decoding many streams - the
 * batched and served forms - gives each decoder one or two planners of a few
 * threads, so the streams' planners together do not oversubscribe the host. */
typedef struct av1b_decoder_options {
  int32_t planners;
  int32_t planner_threads;
} av1b_decoder_options;
AV1B_API int av1b_decoder_create_ex(int device, size_t hbm_budget_bytes,
                                    const av1b_decoder_options* options, av1b_decoder** out);
AV1B_API int av1b_decoder_destroy(av1b_decoder* dec);
/* Decoder::reset (engine.cpp:65-71): drops every slot. */
AV1B_API int av1b_decoder_reset(av1b_decoder* dec);

/* --- decode: Decoder::decode_reference / decode (av1gpu.hpp:635-636, 733) --
 * Decodes `syntax` and keeps the picture resident in a reference slot when
 * `keep_reference` is non-zero (its id goes to *out_slot, else -1). `out` may be
 * null (no read back); otherwise the display picture, film grain included, is
 * copied into the caller's planes. `error` (nullable, `error_len` bytes)
 * receives a message on failure. */
AV1B_API int av1b_decode(av1b_decoder* dec, const av1b_frame_syntax* syntax, int keep_reference,
                const av1b_planes* out, int* out_slot, char* error, size_t error_len);

/* The same for a serialized frame (see av1b_syntax_view). */
AV1B_API int av1b_decode_blob(av1b_decoder* dec, const uint8_t* blob, size_t len, int keep_reference,
                     const av1b_planes* out, int* out_slot, char* error, size_t error_len);

/* --- pipelined form: Decoder::plan_frame / decode_reference_planned /
 * discard_frame_plan (av1gpu.hpp:670-712). A plan holds one frame's validated
 * device records and coefficient pools, already uploaded into device memory it
 * owns, so a pipeline can plan frame N+1 while frame N runs and the decode
 * itself is device work only. The reference slots a plan reads must be held
 * (decoded, or reserved and decoded before the plan is decoded). */
typedef struct av1b_plan av1b_plan;
AV1B_API int av1b_plan_frame(av1b_decoder* dec, const av1b_frame_syntax* syntax, av1b_plan** out);
/* Decodes a plan into `slot` (a reserved or held slot; -1: the lowest free
 * slot when `keep_reference`, none otherwise). `wait` == 0 returns once the
 * work is queued on the decoder's stream: call av1b_sync before reading
 * anything the frame produced on the host. The plan can be decoded again. */
AV1B_API int av1b_decode_planned(av1b_decoder* dec, av1b_plan* plan, int slot, int keep_reference,
                                 const av1b_planes* out, int* out_slot, int wait);
AV1B_API int av1b_plan_free(av1b_decoder* dec, av1b_plan* plan);
/* What a planned frame holds: its geometry and the work each stage has, as
 * the planner counted it (the reference's DecodeStats, av1gpu.hpp:544-552,
 * counts blocks and waves; a benchmark needs the samples each kernel touches
 * to state its algorithmic bytes). Phase B is the dependency-scheduled part
 * (intra, inter-intra and intra block copy blocks), in `chains` chains of
 * dependency depth `depth`; phase A inter blocks are predicted from
 * reference pictures only, `inter_ref_samples` counting a compound block's
 * two predictions. */
typedef struct av1b_plan_info {
  int32_t width, height, coded_width, bit_depth;
  int64_t blocks, phase_b_blocks, chains, phase_b_samples;
  int64_t inter_tiles, inter_samples, inter_ref_samples;
  int64_t transforms, tx_samples, coef_samples;
  int64_t deblock_edges[2];      /* vertical, horizontal */
  int64_t cdef_blocks, lr_units;
  int32_t depth, upscaled, restored, grain;
} av1b_plan_info;
AV1B_API int av1b_plan_stats(const av1b_plan* plan, av1b_plan_info* out);

/* Waits for queued work and reports a device-side failure of the last frame. */
AV1B_API int av1b_sync(av1b_decoder* dec);

/* The device memory a decoder needs for a stream of this geometry with
 * `n_slots` reference slots and `plans` plans alive at once (planned ahead,
 * in flight, or kept for reuse: a decoder keeps up to 8 freed plans) - an
 * upper bound for frames whose blocks are 4x4 or larger - and what a decoder
 * holds now against its budget. A server admitting streams by HBM sizes
 * each stream's decoder budget with the first and checks the second. */
AV1B_API size_t av1b_stream_hbm_estimate(int width, int height, int coded_width, int bit_depth,
                                         int ss_x, int ss_y, int n_slots, int plans);
AV1B_API int av1b_decoder_memory(av1b_decoder* dec, size_t* allocated, size_t* budget);

/* Decoder::reserve_reference / decode_reference_reserved (av1gpu.hpp:645-661). */
AV1B_API int av1b_reserve_reference(av1b_decoder* dec, int* out_slot);
AV1B_API int av1b_decode_reserved(av1b_decoder* dec, const av1b_frame_syntax* syntax, int slot,
                         const av1b_planes* out, char* error, size_t error_len);

/* Decoder::release_reference (av1gpu.hpp:736). */
AV1B_API int av1b_release_reference(av1b_decoder* dec, int slot);

/* Decoder::to_nv12 (av1gpu.hpp:745-746): packs `slot` on the device into
 * `pitch`-byte rows and copies the bytes to `dst` (host, `dst_len` bytes).
 * The slot of the frame decoded last packs the picture after film grain; an
 * older slot packs its stored picture, which is the one before film grain
 * (the reference CPU backend's gather(), cpu_backend.cpp:557-570). */
AV1B_API int av1b_to_nv12(av1b_decoder* dec, int slot, size_t pitch, uint8_t* dst, size_t dst_len);
/* Same, but `dst` is device memory: the zero-copy end of the path. */
AV1B_API int av1b_to_nv12_device(av1b_decoder* dec, int slot, size_t pitch, void* dst_device,
                        size_t dst_len);
/* Decoder::nv12_pack_begin / nv12_pack_wait / nv12_pack_release
 * (av1gpu.hpp:748-772): the pack split so the read back leaves the decoding
 * thread. begin packs `slot` on the device (the picture to_nv12 would give)
 * and starts its copy into page-locked memory on a side stream, so the next
 * frame's decode overlaps it; it returns a handle. wait blocks until the
 * bytes are there and copies them to `dst` (may be null), and/or points
 * `*data` at the page-locked bytes, valid until release; `*bytes` is their
 * count. Up to eight packs are outstanding; begin returns AV1B_ERR_NOMEM
 * while all are held. */
AV1B_API int av1b_nv12_pack_begin(av1b_decoder* dec, int slot, size_t pitch, int* out_handle);
AV1B_API int av1b_nv12_pack_wait(av1b_decoder* dec, int handle, uint8_t* dst, size_t dst_len,
                                 const uint8_t** data, size_t* bytes);
AV1B_API int av1b_nv12_pack_release(av1b_decoder* dec, int handle);
/* The byte count to_nv12 produces (factory.cpp:236-244's nv12_buffer_size):
 * 0 for a frame that is not 4:2:0, an odd pitch or a pitch below a chroma row. */
AV1B_API size_t av1b_nv12_size(int width, int height, int ss_x, int ss_y, size_t pitch);

/* Decoder::to_rgb (av1gpu.hpp:739-740): RGB24, width*height*3 bytes. */
AV1B_API int av1b_to_rgb(av1b_decoder* dec, int slot, int matrix, int range, uint8_t* dst,
                size_t dst_len);

/* Decoder::stats (av1gpu.hpp:630). */
AV1B_API int av1b_get_stats(av1b_decoder* dec, av1b_stats* out);

/* The device status word: non-zero after a device-side wait gave up or a
 * bounds check refused an access. Reading clears it. */
AV1B_API int av1b_poll_status(av1b_decoder* dec, int* status);

/* Device pointer and layout of a slot's planes (for callers that hand the
 * picture on without a host copy). The planes hold the picture once the work
 * queued on the decoder's stream (av1b_decoder_stream) up to this call has
 * run - the display picture of a frame whose film grain was left to its
 * outputs is made here, on that stream - so a reader orders itself after
 * that stream (an event on it, or av1b_sync). */
AV1B_API int av1b_slot_planes_device(av1b_decoder* dec, int slot, uint16_t* plane_ptr[3],
                            int32_t stride[3]);

/* The message of the last failed call on this decoder (empty if none). The
 * pointer stays valid until the next call on the decoder. */
AV1B_API const char* av1b_last_error(av1b_decoder* dec);

/* The limit of one device-side dependency wait (default 1 s). A wait that runs
 * out sets the status word; the frame then fails with AV1B_ERR_TIMEOUT and
 * every later wait of the frame gives up at once, so a broken frame ends in
 * about one limit instead of hanging the device. */
AV1B_API int av1b_set_wait_limit(av1b_decoder* dec, long long limit_ns);
/* Failure-detection self test: one device wait on a flag nothing ever sets,
 * bounded by `limit_ns`. Fills the resulting status word (1: the wait gave up)
 * and the elapsed device time. */
AV1B_API int av1b_selftest_wait(av1b_decoder* dec, long long limit_ns, int* status,
                                double* elapsed_ms);

/* The integer-ALU roof of `device`: 32-bit operations per second of
 * independent adds (kind 0) or multiply-adds (kind 1, one instruction each),
 * measured by a short kernel on every SM. The per-stage report divides each
 * stage's counted operations by it, beside its bytes by the HBM bandwidth.
 * No counterpart in the reference. */
AV1B_API int av1b_int_peak(int device, int kind, double* ops_per_s);
/* The floor of one step of the dependency-scheduled phase's critical path:
 * the median one-way time, in ns, of a flag handed between warps on two SMs
 * by a release store and acquire polls (the publication and wait that phase
 * uses), over 16 SM pairs and 8 places of the flag in memory, measured by a
 * short cooperative kernel. No counterpart in the reference. */
AV1B_API int av1b_handoff_peak(int device, double* one_way_ns);

/* Per-stage device timing: with profiling on, every launch (and device copy)
 * is bracketed by CUDA events on the decoder's stream, and the elapsed times
 * are summed per stage at each synchronisation. av1b_profile returns 1 and
 * fills the stage's name, total milliseconds and launch count, 0 past the last
 * stage. Switching profiling on or off clears the totals. */
AV1B_API int av1b_set_profiling(av1b_decoder* dec, int on);
AV1B_API int av1b_profile(av1b_decoder* dec, int stage, const char** name, double* total_ms,
                          long long* count);

/* Trace of the dependency-scheduled phase: with tracing on, each frame
 * records, per phase B block, the device time (globaltimer ns) it was
 * claimed, the time its dependencies were all met, the time it was
 * published, and which dependency was published last (-1: none). After a
 * decode, av1b_unit_trace copies the last frame's records - four uint64 per
 * block of the frame, indexed by block, zero for blocks outside phase B -
 * into `out` (room for `cap` uint64) and sets *n to the count. */
AV1B_API int av1b_set_unit_trace(av1b_decoder* dec, int on);
AV1B_API int av1b_unit_trace(av1b_decoder* dec, uint64_t* out, size_t cap, size_t* n);

/* Whether frames planned from now on let a chroma block of a difference-
 * weighted compound read the blend mask its luma block wrote when that block
 * is the same prediction (on by default), instead of predicting the luma it
 * covers itself. Both give the same samples; off, every such chroma tile
 * takes the full prediction kernel (tests compare the two paths). No
 * counterpart in the reference. */
AV1B_API int av1b_set_shared_masks(av1b_decoder* dec, int on);

/* CUDA stream the decoder runs on (a cudaStream_t), so a caller can order its
 * own work after a decode without a host synchronisation. */
AV1B_API void* av1b_decoder_stream(av1b_decoder* dec);

/* --- batched form: many streams' frames in one step -------------------------
 * No counterpart in the reference, which decodes one stream per Decoder
 * (its nearest mechanism: the per-frame graph capture of its CUDA backend,
 * src/backends/cuda/cuda_backend.cpp:1212-1227). A batch runs one planned
 * frame of each of up to AV1B_BATCH_MAX independent streams - each stream its
 * own decoder, with its own geometry, bit depth, reference slots and
 * planners, all on the batch's device - as one step: persistent kernels, one
 * per stage for all the streams, take the frames' work from device
 * descriptors, and the step is replayed as a CUDA graph. Each stream's
 * output is the same as decoding its frame alone (av1b_decode_planned).
 *
 * av1b_batch_decode queues frame i of the step as plans[i] decoded by
 * decoders[i] into slots[i] (a reserved or held slot, -1: the lowest free
 * one; the slot gets the picture as av1b_decode_planned with keep_reference
 * does), and, when nv12_device[i] is non-null, its NV12 pack into that device
 * buffer (nv12_pitch[i] bytes a row, nv12_len[i] bytes of room;
 * av1b_nv12_size). out_slots[i] (nullable) gets the slot. A decoder appears
 * at most once a step. The call returns when the step is queued on the
 * batch's stream; the decoders' own streams are ordered after it, so their
 * later calls see the step's results. av1b_batch_sync waits for the step and
 * reports the first failed stream. */
#define AV1B_BATCH_MAX 64
typedef struct av1b_batch av1b_batch;
/* The step's launch shape: CTAs per SM of each stage kernel (0: keep the
 * current value; stages in launch order, 23 of them), the work items a warp
 * claims at once, whether the film grain of a stream whose only output is
 * its NV12 pack is applied inside the pack (its display picture is then made
 * when an output call asks for it), and whether steps replay as a CUDA graph. */
typedef struct av1b_batch_config {
  int32_t ctas_per_sm[24];
  int32_t claim_chunk;
  int32_t fuse_grain_nv12;
  int32_t use_graph;
  int32_t inter_variant;    /* the build of the full prediction kernel (0: fewer CTAs, more registers) */
} av1b_batch_config;
AV1B_API int av1b_batch_create(int device, av1b_batch** out);
AV1B_API int av1b_batch_destroy(av1b_batch* batch);
AV1B_API int av1b_batch_decode(av1b_batch* batch, int n, av1b_decoder* const* decoders,
                               av1b_plan* const* plans, const int* slots, int* out_slots,
                               uint8_t* const* nv12_device, const size_t* nv12_pitch,
                               const size_t* nv12_len);
AV1B_API int av1b_batch_sync(av1b_batch* batch);
AV1B_API int av1b_batch_get_config(av1b_batch* batch, av1b_batch_config* out);
AV1B_API int av1b_batch_set_config(av1b_batch* batch, const av1b_batch_config* config);
/* The autotuner: picks the launch shape for a set of streams by timing the
 * given step (decoded again and again: its slots must not be among the
 * slots its frames read) with each candidate - CTAs per SM per stage group,
 * the claim size, the build of the full prediction kernel, the grain-in-pack
 * fusion - by coordinate descent, `reps`
 * timed steps each. The result is kept in `cache_path` (nullable), one line
 * per signature of the step (GPU, SM count, each stream's geometry, bit
 * depth and tools), and a later call with the same signature takes it from
 * there without timing (*best_ms = -1). The batch keeps the result. */
AV1B_API int av1b_batch_autotune(av1b_batch* batch, int n, av1b_decoder* const* decoders,
                                 av1b_plan* const* plans, const int* slots,
                                 uint8_t* const* nv12_device, const size_t* nv12_pitch,
                                 const size_t* nv12_len, const char* cache_path, int reps,
                                 av1b_batch_config* out, double* best_ms);
AV1B_API const char* av1b_batch_last_error(av1b_batch* batch);
/* Per-stage device time of batched steps: with profiling on, steps launch
 * without the graph, each stage bracketed by CUDA events, and
 * av1b_batch_profile gives stage `stage`'s summed milliseconds (in launch
 * order, 0..22; the grain templates run beside the others) and the steps
 * timed. Switching profiling clears the sums. */
AV1B_API int av1b_batch_set_profiling(av1b_batch* batch, int on);
AV1B_API int av1b_batch_profile(av1b_batch* batch, int stage, double* total_ms, long long* steps);
/* The CUDA stream the batch's steps run on (a cudaStream_t). */
AV1B_API void* av1b_batch_stream(av1b_batch* batch);

/* --- served form: a request loop over many streams --------------------------
 * No counterpart in the reference (its nearest mechanisms: the pipelined
 * plan / decode API, av1gpu.hpp:656-689, and its DirectShow filter's job
 * loop for one stream, dsfilter/decode_core.hpp:47-68). A server admits
 * streams by the device memory their decoder needs (their HBM budget is
 * reserved at av1b_server_open, which refuses with AV1B_ERR_NOMEM when it
 * does not fit; av1b_server_close returns it), plans frame requests on host
 * threads as they arrive, and runs the planned frames of all streams in
 * batched steps (av1b_batch_*) as they become ready: continuous batching, one
 * frame a stream a step, at most max_inflight steps queued on the GPU.
 *
 * A request is a serialized FrameSyntax (av1b_syntax_view) whose
 * reference_slots hold frame *distances* within its stream (1 = the
 * previous frame submitted on it, at most max_refs); the server maps them to
 * the stream's device slots. A stream's first frame reads no reference. The
 * server reads the caller's bytes in place, never writing them (streams may
 * share a buffer): they must stay unchanged until the frame's result has
 * been polled.
 * Results come back through av1b_server_poll in completion order: the
 * frame's arrival and device-completion times on the host clock (ms since
 * the server started) and their difference, and its NV12 pack in device
 * memory (a ring of eight buffers a stream: valid until eight more frames
 * of the stream complete). `status` is a failure of the frame's planning or
 * launch; a device-side failure surfaces at av1b_server_drain, which waits
 * for every submitted frame and checks every decoder. */
typedef struct av1b_server av1b_server;
typedef struct av1b_server_options {
  int32_t device;
  int32_t max_batch;        /* frames a step (1..64; 0: 64) */
  int32_t max_inflight;     /* steps queued on the GPU at once (1..8; 0: 2); while one is
                               queued, the next waits up to batch_wait_us for a quarter of
                               the open streams to have a frame ready */
  int32_t planner_threads;  /* requests planned at once (0: cores / 2) */
  int32_t decoder_threads;  /* host threads planning one request (0: one per 0.7 million
                               samples of the stream's frames, 1..6) */
  int32_t batch_wait_us;    /* (0: 1000; negative: no wait) */
  size_t hbm_budget;        /* device memory the streams may hold (0: 90 % of the free memory) */
} av1b_server_options;
typedef struct av1b_stream_desc {
  int32_t width, height, coded_width, bit_depth, ss_x, ss_y;
  int32_t max_refs;         /* reference frames a frame may read (1..7) */
  int32_t nv12_pitch;       /* 0: no NV12 output */
} av1b_stream_desc;
typedef struct av1b_server_result {
  int32_t stream_id, status, slot, batch_size;
  uint64_t tag, frame_index;
  int64_t step;
  double arrival_ms, done_ms, latency_ms;
  double planned_ms;        /* when the frame's plan was ready (host clock) */
  const uint8_t* nv12_device;
  size_t nv12_bytes;
} av1b_server_result;
typedef struct av1b_server_stats {
  uint64_t submitted, completed, steps, stepped_frames;
  size_t hbm_used, hbm_budget;
  int32_t streams;
  double now_ms;
  double plan_ms;           /* host time planning requests, summed over planner threads */
  double launch_ms;         /* host time queueing steps (av1b_batch_decode) */
} av1b_server_stats;
AV1B_API int av1b_server_create(const av1b_server_options* options, av1b_server** out);
AV1B_API int av1b_server_destroy(av1b_server* server);
AV1B_API int av1b_server_open(av1b_server* server, const av1b_stream_desc* desc, int* stream_id,
                              size_t* hbm_bytes);
AV1B_API int av1b_server_close(av1b_server* server, int stream_id);
AV1B_API int av1b_server_submit(av1b_server* server, int stream_id, const uint8_t* blob, size_t len,
                                uint64_t tag);
AV1B_API int av1b_server_poll(av1b_server* server, av1b_server_result* out, int max, int wait_ms,
                              int* n);
AV1B_API int av1b_server_drain(av1b_server* server, int timeout_ms);
AV1B_API int av1b_server_get_stats(av1b_server* server, av1b_server_stats* out);
/* The server's batch (an av1b_batch*), e.g. to set or tune its launch shape. */
AV1B_API void* av1b_server_batch(av1b_server* server);

/* --- film grain without allocation -----------------------------------------
 * No counterpart in the reference: its film grain runs inside decode only.
 * For callers that cannot allocate device memory where they need a frame's
 * grain - a display callback re-showing a reference slot (which holds the
 * picture before grain) under a real-time deadline, where cudaMalloc/cudaFree
 * may synchronize the device, or a host that fixes its device memory at
 * start-up. It applies `syntax`'s film grain (syntax->grain, its size, bit
 * depth, subsampling and colour matrix; nothing else of the syntax is read) to
 * the picture in `src` and writes the output picture to `dst`: three device
 * planes each, strides in samples, queued on `stream` (a cudaStream_t of the
 * current device, 0 for the default stream; a stream of another device is
 * refused with AV1B_ERR_ARG). Without grain (apply == 0) it copies src to
 * dst. The output planes must not share a byte with any input plane or with
 * each other (AV1B_ERR_ARG): grain is not applied in place, because a chroma
 * sample's grain reads the input luma that an in-place write would already
 * have changed.
 *
 * It allocates nothing. Its scratch is a file-scope device array of
 * AV1B_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until
 * exit; pictures above AV1B_NOALLOC_MAX_DIM samples on a side are refused
 * (AV1B_ERR_ARG). The first call on a device sets the scratch up (resolves its
 * address, builds the grain LFSR tables, and waits for that): make it before
 * any stream capture. Calls share the scratch, so calls that overlap on the
 * GPU race; serialize them. */
#define AV1B_NOALLOC_SCRATCH_BYTES 301312
#define AV1B_NOALLOC_MAX_DIM 16384
AV1B_API int av1b_apply_film_grain_noalloc(const av1b_frame_syntax* syntax,
                                           const uint16_t* const src[3], const int32_t src_stride[3],
                                           uint16_t* const dst[3], const int32_t dst_stride[3],
                                           void* stream);

/* --- a serialized frame's reference slot list ----------------------------- */
/* Rewrites the reference slot list of a serialized frame in place. */
AV1B_API int av1b_blob_set_refs(uint8_t* blob, size_t len, const int32_t* slots, int n);
/* Reads the reference slot list (distances for a synthetic frame). */
AV1B_API int av1b_blob_get_refs(const uint8_t* blob, size_t len, int32_t* slots, int max_n);

#ifdef __cplusplus
}
#endif

#endif /* AV1B_H */
