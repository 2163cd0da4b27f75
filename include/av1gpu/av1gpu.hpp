/*
 * av1gpu.hpp - the C++ API of the B200 AV1 reconstruction backend.
 *
 * Drop-in for the reference library's public header (trprkkk/AV1onGPU,
 * include/av1gpu/av1gpu.hpp): the same namespace, types, members, defaults
 * and virtual methods, so code written against the reference compiles and
 * links against libav1b.so unchanged. The declarations have to be alike -
 * that is what makes it a drop-in - the implementation behind them
 * (av1ongpu_b200/csrc/api.cpp) is this library's: every decode runs on the
 * CUDA device through the C ABI in av1b.h.
 *
 * Differences a caller can observe:
 *   - BackendKind::Cpu and BackendKind::OpenCL are refused by Decoder::create
 *     (there is one backend, CUDA on sm_100a, and no CPU fallback).
 */
#ifndef AV1GPU_AV1GPU_HPP
#define AV1GPU_AV1GPU_HPP

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#if defined(__GNUC__)
#define AV1GPU_API __attribute__((visibility("default")))
#else
#define AV1GPU_API
#endif

namespace av1gpu {

enum class ColorMatrix : int { Bt601 = 0, Bt709 = 1, Bt2020 = 2, Identity = 3 };
enum class ColorRange : int { Limited = 0, Full = 1 };
enum class BackendKind : int { Auto = 0, Cpu = 1, OpenCL = 2, CUDA = 3 };

/* "cpu" / "opencl" / "cuda" / "auto" */
AV1GPU_API const char* to_string(BackendKind kind);
AV1GPU_API BackendKind backend_kind_from_string(const std::string& name);

struct FrameGeometry {
  int width = 0;
  int height = 0;
  int bit_depth = 8;
  int ss_x = 1;
  int ss_y = 1;
};

/* A decoded picture on the host: three planes of 16-bit samples whatever the
 * bit depth, rows 32-sample aligned. */
class AV1GPU_API Frame {
 public:
  Frame() = default;
  Frame(int width, int height, int bit_depth = 8, int ss_x = 1, int ss_y = 1) {
    allocate(width, height, bit_depth, ss_x, ss_y);
  }
  /* (Re)allocates the planes, all samples zero. */
  void allocate(int width, int height, int bit_depth, int ss_x, int ss_y);
  /* True when the frame has this geometry and room for it. */
  bool matches(int width, int height, int bit_depth, int ss_x, int ss_y) const;
  void fill(uint16_t value);
  int plane_width(int plane) const;
  int plane_height(int plane) const;
  int max_value() const { return (1 << bit_depth) - 1; }
  bool empty() const { return width <= 0 || height <= 0; }
  uint16_t* plane(int p) { return storage[p].data(); }
  const uint16_t* plane(int p) const { return storage[p].data(); }

  int width = 0;
  int height = 0;
  int bit_depth = 8;
  int ss_x = 1;
  int ss_y = 1;
  int stride[3] = {0, 0, 0};
  std::vector<uint16_t> storage[3];
};

/* Intra modes in the specification's numbering, chroma from luma as 13. */
enum class PredictionMode : int {
  Dc = 0, Vertical = 1, Horizontal = 2, D45 = 3, D135 = 4, D113 = 5, D157 = 6, D203 = 7,
  D67 = 8, Smooth = 9, SmoothVertical = 10, SmoothHorizontal = 11, Paeth = 12,
  ChromaFromLuma = 13,
};

/* TxType: the vertical transform is named first. */
enum class TransformType : int {
  DctDct = 0, AdstDct = 1, DctAdst = 2, AdstAdst = 3, FlipadstDct = 4, DctFlipadst = 5,
  FlipadstFlipadst = 6, AdstFlipadst = 7, FlipadstAdst = 8, Idtx = 9, VDct = 10, HDct = 11,
  VAdst = 12, HAdst = 13, VFlipadst = 14, HFlipadst = 15,
};

enum class FilterIntraMode : int { Dc = 0, V = 1, H = 2, D157 = 3, Paeth = 4 };
enum class FilterType : int { Regular = 0, Smooth = 1, Sharp = 2, Bilinear = 3 };
enum class CompoundType : int { None = 0, Average = 1, Distance = 2, Wedge = 3, DiffWtd = 4 };

/* One transform of a block; its dequantised coefficients are a raster of
 * min(w,32) x min(h,32) at FrameSyntax::coefficients[coef_offset]. */
struct TransformBlock {
  int x = 0;
  int y = 0;
  int w = 0;
  int h = 0;
  int coef_offset = 0;
  int eob = 0; /* 0: no residual */
  TransformType tx_type = TransformType::DctDct;
  int level_offset = 0;
  int qindex = 0;
  int dc_step = 0;
  int ac_step = 0;
  int denominator = 1;
  int qm_off = -1;
};

/* An OBMC strip of an inter block, relative to the block. */
struct ObmcCandidate {
  int pass = 0; /* 0 above, 1 left */
  int x = 0;
  int y = 0;
  int w = 0;
  int h = 0;
  int mv[2] = {0, 0};
  FilterType filter = FilterType::Regular;
  FilterType filter_v = FilterType::Regular;
  int ref = -1;
};

/* One prediction block of one plane. */
struct BlockSyntax {
  int x = 0;
  int y = 0;
  int w = 0;
  int h = 0;
  int plane = 0;
  int bit_depth = 8;

  bool is_intra = true;
  bool intrabc = false;

  PredictionMode mode = PredictionMode::Dc;
  bool have_left = true;
  bool have_above = true;
  int have_above_right = -1; /* -1: derived from what is decoded before this block */
  int have_below_left = -1;
  int angle_delta = 0;
  int filter_type = 0;
  bool use_filter_intra = false;
  FilterIntraMode filter_intra_mode = FilterIntraMode::Dc;
  int cfl_alpha = 0;

  bool lossless = false;

  bool use_palette = false;
  int palette_size = 0;
  int palette[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int palette_off = 0;
  int palette_stride = 0;

  int ref[2] = {-1, -1};
  int mv[2][2] = {{0, 0}, {0, 0}};
  FilterType filter = FilterType::Regular;
  FilterType filter_v = FilterType::Regular;
  int motion_mode = 0;
  CompoundType compound = CompoundType::None;
  int blend[2] = {8, 8};
  int wedge_index = 0;
  int mask_sign = 0;
  bool interintra = false;
  int interintra_mode = 0;
  bool interintra_wedge = false;
  bool warp[2] = {false, false};
  int32_t warp_params[2][6] = {{0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0}};
  bool mask_warp[2] = {false, false};
  std::vector<ObmcCandidate> obmc;

  bool residual_provided = false;

  std::vector<TransformBlock> transforms;
};

/* A deblocking edge segment: (x, y) is q0, `length` samples along the edge. */
struct DeblockEdge {
  int plane = 0;
  int x = 0;
  int y = 0;
  bool vertical = true;
  int length = 0;
  int level = 0;
  int filter_size = 8;
};

/* An 8x8 CDEF block (chroma blocks in their own plane's samples). */
struct CdefBlock {
  int plane = 0;
  int x = 0;
  int y = 0;
  int pri_strength = 0;
  int sec_strength = 0;
  int damping = 3;
  int dir = 0;
};

/* FrameRestorationType. */
enum RestorationType {
  kRestoreNone = 0,
  kRestoreSwitchable = 1,
  kRestoreWiener = 2,
  kRestoreSgrproj = 3,
};

constexpr int kWienerTaps = 3;
constexpr int kSgrParamsBits = 4;
constexpr int kSgrProjPrjBits = 7;
constexpr int kSgrProjRstBits = 4;
constexpr int kSgrProjMtableBits = 20;
constexpr int kSgrProjSgrBits = 8;
constexpr int kSgrProjRecipBits = 12;
constexpr int kSgrProjSubexpK = 4;
constexpr int kWienerTapsMin[3] = {-5, -23, -17};
constexpr int kWienerTapsMax[3] = {10, 8, 46};
constexpr int kWienerTapsK[3] = {1, 2, 3};
constexpr int kSgrXqdMin[2] = {-96, -32};
constexpr int kSgrXqdMax[2] = {31, 95};
constexpr int kWienerTapsMid[3] = {3, -7, 15};
constexpr int kSgrXqdMid[2] = {-32, 31};
/* Sgr_Params: (r0, e0, r1, e1) per set. */
constexpr int kSgrParams[16][4] = {
    {2, 12, 1, 4},  {2, 15, 1, 6},  {2, 18, 1, 8},  {2, 21, 1, 9},  {2, 24, 1, 10}, {2, 29, 1, 11},
    {2, 36, 1, 12}, {2, 45, 1, 13}, {2, 56, 1, 14}, {2, 68, 1, 15}, {0, 0, 1, 5},   {0, 0, 1, 8},
    {0, 0, 1, 11},  {0, 0, 1, 14},  {2, 30, 0, 0},  {2, 75, 0, 0},
};

/* One loop restoration unit. `type` 2 selects the Wiener filter and any other
 * non-zero value the self-guided one, as the reference engine interprets it. */
struct RestorationUnit {
  int type = 0;
  int wiener[2][3] = {{0, 0, 0}, {0, 0, 0}};
  int sgr_set = 0;
  int sgr_xqd[2] = {0, 0};
};

/* film_grain_params(); ar_coeffs_* are signed (coded value - 128). */
struct FilmGrainParams {
  bool apply = false;
  int seed = 0;
  int num_y_points = 0;
  int point_y_value[16] = {0};
  int point_y_scaling[16] = {0};
  bool chroma_scaling_from_luma = false;
  int num_cb_points = 0;
  int point_cb_value[16] = {0};
  int point_cb_scaling[16] = {0};
  int num_cr_points = 0;
  int point_cr_value[16] = {0};
  int point_cr_scaling[16] = {0};
  int grain_scaling_minus_8 = 0;
  int ar_coeff_lag = 0;
  int ar_coeffs_y[24] = {0};
  int ar_coeffs_cb[25] = {0};
  int ar_coeffs_cr[25] = {0};
  int ar_coeff_shift_minus_6 = 0;
  int grain_scale_shift = 0;
  int cb_mult = 0;
  int cb_luma_mult = 0;
  int cb_offset = 0;
  int cr_mult = 0;
  int cr_luma_mult = 0;
  int cr_offset = 0;
  bool overlap_flag = false;
  bool clip_to_restricted_range = false;
};

struct ColorSyntax {
  ColorMatrix matrix = ColorMatrix::Bt709;
  ColorRange range = ColorRange::Limited;
};

/* Everything one frame's reconstruction needs. */
struct FrameSyntax {
  int width = 0;
  int coded_width = 0; /* 0: not superres */
  int height = 0;
  int bit_depth = 8;
  int ss_x = 1;
  int ss_y = 1;
  int base_q_idx = 0;
  int sharpness = 0;
  bool enable_intra_edge_filter = true;

  std::vector<int> reference_slots;
  int reference_width[7] = {0, 0, 0, 0, 0, 0, 0};
  int reference_height[7] = {0, 0, 0, 0, 0, 0, 0};

  std::vector<BlockSyntax> blocks;

  std::vector<int32_t> coefficients;
  std::vector<int32_t> residual;
  std::vector<int16_t> levels;
  std::vector<uint8_t> qm_pool;
  std::vector<uint8_t> palette_map;

  std::vector<DeblockEdge> deblock;
  std::vector<CdefBlock> cdef;

  int restoration_type[3] = {0, 0, 0};
  int restoration_unit_log2[3] = {0, 0, 0};
  int restoration_unit_cols[3] = {0, 0, 0};
  std::vector<RestorationUnit> restoration[3];

  FilmGrainParams grain;
  ColorSyntax color;
};

/* Device timings of the last frame, milliseconds. */
struct DecodeStats {
  int blocks = 0;
  int waves = 0;
  int kernel_launches = 0;
  double reconstruct_ms = 0.0;
  double filter_ms = 0.0;
  double readback_ms = 0.0;
  double total_ms = 0.0;
};

struct DeviceInfo {
  BackendKind kind = BackendKind::Cpu;
  std::string name;
  std::string vendor;
  std::string version;
  std::string detail;
  bool available = false;
  bool unified_memory = false;
  uint64_t global_mem = 0;
  int compute_units = 0;
};

struct BackendOptions {
  BackendKind kind = BackendKind::Auto;
  int device_index = 0;
  /* Kept for source compatibility; this library has no CPU backend to fall
   * back to, so a missing device is always an error. */
  bool allow_cpu_fallback = true;
  bool verbose = false;
};

AV1GPU_API std::vector<DeviceInfo> enumerate_devices();
AV1GPU_API std::string build_info();

struct Psnr {
  double y = 0.0;
  double u = 0.0;
  double v = 0.0;
};

AV1GPU_API Psnr frame_psnr(const Frame& a, const Frame& b);
AV1GPU_API void frame_to_yuv8(const Frame& frame, std::vector<uint8_t>* out);
AV1GPU_API void frame_to_yuv16(const Frame& frame, std::vector<uint8_t>* out);
/* NV12 at `pitch` bytes per row, padding zero; false for a frame that is not
 * 4:2:0, an odd pitch, or a pitch narrower than a chroma row. */
AV1GPU_API bool frame_to_nv12(const Frame& frame, size_t pitch, std::vector<uint8_t>* out);

class AV1GPU_API Decoder {
 public:
  static std::unique_ptr<Decoder> create(const BackendOptions& options,
                                         std::string* error = nullptr);
  virtual ~Decoder();
  Decoder(const Decoder&) = delete;
  Decoder& operator=(const Decoder&) = delete;

  virtual const DeviceInfo& device() const = 0;
  virtual const BackendOptions& options() const = 0;
  virtual const DecodeStats& stats() const = 0;

  /* Decodes into a device-resident reference slot; -1 on failure. */
  virtual int decode_reference(const FrameSyntax& syntax, Frame* out,
                               std::string* error = nullptr) = 0;

  virtual int decode_reference_reserved(const FrameSyntax& syntax, int slot, Frame* out,
                                        std::string* error = nullptr, bool read_back = true) {
    (void)read_back;
    (void)syntax;
    (void)slot;
    (void)out;
    if (error) *error = "reserved-slot decode is not supported";
    return -1;
  }

  virtual int reserve_reference() { return -1; }

  virtual bool plan_frame(const FrameSyntax& syntax, void** plan, std::string* error = nullptr,
                          std::atomic<bool>* cancel = nullptr) {
    (void)syntax;
    (void)plan;
    (void)cancel;
    if (error) *error = "pre-planning is not supported";
    return false;
  }

  virtual bool plan_frame(FrameSyntax&& syntax, void** plan, std::string* error = nullptr,
                          std::atomic<bool>* cancel = nullptr) {
    return plan_frame(static_cast<const FrameSyntax&>(syntax), plan, error, cancel);
  }

  virtual int decode_reference_planned(void* plan, int slot, Frame* out,
                                       std::string* error = nullptr, bool read_back = true) {
    (void)plan;
    (void)slot;
    (void)out;
    (void)read_back;
    if (error) *error = "pre-planned decode is not supported";
    return -1;
  }

  virtual void discard_frame_plan(void* plan) { (void)plan; }
  virtual bool supports_preplanning() const { return false; }
  virtual bool dequantises_on_device() const { return false; }
  virtual bool packs_nv12_on_device() const { return false; }

  /* Decode and drop the device copy. */
  virtual bool decode(const FrameSyntax& syntax, Frame* out, std::string* error = nullptr);

  virtual void release_reference(int slot) = 0;

  virtual bool to_rgb(int slot, ColorMatrix matrix, ColorRange range, std::vector<uint8_t>* rgb,
                      std::string* error = nullptr) = 0;

  virtual bool to_nv12(int slot, size_t pitch, std::vector<uint8_t>* nv12,
                       std::string* error = nullptr) = 0;

  virtual int nv12_pack_begin(int slot, size_t pitch, std::string* error = nullptr) {
    (void)slot;
    (void)pitch;
    (void)error;
    return -1;
  }

  virtual bool nv12_pack_wait(int handle, std::vector<uint8_t>* nv12,
                              std::string* error = nullptr) {
    (void)handle;
    (void)nv12;
    (void)error;
    return false;
  }

  virtual void nv12_pack_release(int handle) { (void)handle; }

  virtual void hold_output(bool hold) { (void)hold; }

  virtual void reset() = 0;

 protected:
  Decoder() = default;
};

AV1GPU_API std::unique_ptr<Decoder> create_best_decoder(const BackendOptions& options,
                                                        std::string* error = nullptr);

} /* namespace av1gpu */

#endif /* AV1GPU_AV1GPU_HPP */
