/*
 * api.cpp - av1gpu::Decoder (include/av1gpu/av1gpu.hpp) over the C ABI.
 *
 * The reference implements its Decoder as EngineDecoder over a Backend
 * (src/core/engine.cpp:50-494). Here the engine is the C ABI's decoder
 * (decoder.cu); this file only converts between the C++ types and the flat
 * av1b_frame_syntax view and keeps the bookkeeping the C++ API promises:
 * output frames (re)allocated to the display geometry, the NV12 pack handles,
 * the output gate.
 */
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>

#include "../../include/av1b.h"
#include "../../include/av1gpu/av1gpu.hpp"
#include "flat_syntax.hpp"

namespace av1gpu {

const char* to_string(BackendKind kind) {
  switch (kind) {
    case BackendKind::Cpu: return "cpu";
    case BackendKind::OpenCL: return "opencl";
    case BackendKind::CUDA: return "cuda";
    default: return "auto";
  }
}

BackendKind backend_kind_from_string(const std::string& name) {
  if (name == "cpu") return BackendKind::Cpu;
  if (name == "opencl") return BackendKind::OpenCL;
  if (name == "cuda") return BackendKind::CUDA;
  return BackendKind::Auto;
}

/* ---- Frame ------------------------------------------------------------------------- */
int Frame::plane_width(int p) const { return p == 0 ? width : (width + ss_x) >> ss_x; }
int Frame::plane_height(int p) const { return p == 0 ? height : (height + ss_y) >> ss_y; }

void Frame::allocate(int w, int h, int bd, int sx, int sy) {
  width = w;
  height = h;
  bit_depth = bd;
  ss_x = sx;
  ss_y = sy;
  for (int p = 0; p < 3; ++p) {
    const int pw = plane_width(p), ph = plane_height(p);
    stride[p] = (pw + 31) & ~31;
    /* a few rows of slack: the loop filters of an encoder-side frame may read
     * just past the last row band */
    storage[p].assign(static_cast<size_t>(stride[p]) * ((ph + 7) & ~7), 0);
  }
}

bool Frame::matches(int w, int h, int bd, int sx, int sy) const {
  if (width != w || height != h || bit_depth != bd || ss_x != sx || ss_y != sy) return false;
  for (int p = 0; p < 3; ++p) {
    const int pw = plane_width(p), ph = plane_height(p);
    if (stride[p] < pw || storage[p].size() < static_cast<size_t>(stride[p]) * ph) return false;
  }
  return true;
}

void Frame::fill(uint16_t v) {
  for (int p = 0; p < 3; ++p) std::fill(storage[p].begin(), storage[p].end(), v);
}

/* ---- host helpers --------------------------------------------------------------------- */
std::vector<DeviceInfo> enumerate_devices() {
  std::vector<DeviceInfo> out;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return out;
  for (int i = 0; i < n; ++i) {
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, i) != cudaSuccess) continue;
    DeviceInfo d;
    d.kind = BackendKind::CUDA;
    d.name = p.name;
    d.vendor = "NVIDIA";
    d.version = "sm_" + std::to_string(p.major) + std::to_string(p.minor);
    d.detail = "av1ongpu_b200 sm_100a kernels";
    d.available = p.major == 10;
    d.unified_memory = p.unifiedAddressing != 0;
    d.global_mem = p.totalGlobalMem;
    d.compute_units = p.multiProcessorCount;
    out.push_back(d);
  }
  return out;
}

std::string build_info() {
  return "av1ongpu_b200: one backend, CUDA for sm_100a (B200); integer reconstruction bit exact "
         "with the reference CPU backend; no CPU fallback";
}

Psnr frame_psnr(const Frame& a, const Frame& b) {
  Psnr r;
  double* out[3] = {&r.y, &r.u, &r.v};
  const double peak = static_cast<double>(a.max_value());
  for (int p = 0; p < 3; ++p) {
    const int w = std::min(a.plane_width(p), b.plane_width(p));
    const int h = std::min(a.plane_height(p), b.plane_height(p));
    double se = 0;
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x) {
        const double d = static_cast<double>(a.plane(p)[static_cast<size_t>(y) * a.stride[p] + x]) -
                         b.plane(p)[static_cast<size_t>(y) * b.stride[p] + x];
        se += d * d;
      }
    const double mse = w && h ? se / (static_cast<double>(w) * h) : 0;
    *out[p] = mse <= 0 ? 99.0 : 10.0 * std::log10(peak * peak / mse);
  }
  return r;
}

void frame_to_yuv8(const Frame& f, std::vector<uint8_t>* out) {
  out->clear();
  const int shift = f.bit_depth - 8;
  for (int p = 0; p < 3; ++p)
    for (int y = 0; y < f.plane_height(p); ++y)
      for (int x = 0; x < f.plane_width(p); ++x)
        out->push_back(static_cast<uint8_t>(f.plane(p)[static_cast<size_t>(y) * f.stride[p] + x] >> shift));
}

void frame_to_yuv16(const Frame& f, std::vector<uint8_t>* out) {
  out->clear();
  for (int p = 0; p < 3; ++p)
    for (int y = 0; y < f.plane_height(p); ++y)
      for (int x = 0; x < f.plane_width(p); ++x) {
        const uint16_t v = f.plane(p)[static_cast<size_t>(y) * f.stride[p] + x];
        out->push_back(static_cast<uint8_t>(v & 0xff));
        out->push_back(static_cast<uint8_t>(v >> 8));
      }
}

bool frame_to_nv12(const Frame& f, size_t pitch, std::vector<uint8_t>* out) {
  const size_t bytes = av1b_nv12_size(f.width, f.height, f.ss_x, f.ss_y, pitch);
  if (bytes == 0 || !out) return false;
  out->assign(bytes, 0);
  const int shift = f.bit_depth - 8;
  for (int y = 0; y < f.height; ++y)
    for (int x = 0; x < f.width; ++x)
      (*out)[static_cast<size_t>(y) * pitch + x] =
          static_cast<uint8_t>(f.plane(0)[static_cast<size_t>(y) * f.stride[0] + x] >> shift);
  const int cw = (f.width + 1) / 2, ch = (f.height + 1) / 2;
  for (int y = 0; y < ch; ++y)
    for (int x = 0; x < cw; ++x) {
      uint8_t* d = out->data() + static_cast<size_t>(f.height + y) * pitch + 2 * x;
      d[0] = static_cast<uint8_t>(f.plane(1)[static_cast<size_t>(y) * f.stride[1] + x] >> shift);
      d[1] = static_cast<uint8_t>(f.plane(2)[static_cast<size_t>(y) * f.stride[2] + x] >> shift);
    }
  return true;
}

/* ---- the decoder --------------------------------------------------------------------------- */
Decoder::~Decoder() = default;

bool Decoder::decode(const FrameSyntax& syntax, Frame* out, std::string* error) {
  const int slot = decode_reference(syntax, out, error);
  if (slot < 0) return false;
  release_reference(slot);
  return true;
}

namespace {

class B200Decoder final : public Decoder {
 public:
  B200Decoder(av1b_decoder* h, const BackendOptions& o) : h_(h), opt_(o) {
    info_.kind = BackendKind::CUDA;
    info_.available = true;
    info_.vendor = "NVIDIA";
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, o.device_index) == cudaSuccess) {
      info_.name = p.name;
      info_.version = "sm_" + std::to_string(p.major) + std::to_string(p.minor);
      info_.global_mem = p.totalGlobalMem;
      info_.compute_units = p.multiProcessorCount;
    }
    info_.detail = build_info();
  }
  ~B200Decoder() override { av1b_decoder_destroy(h_); }

  const DeviceInfo& device() const override { return info_; }
  const BackendOptions& options() const override { return opt_; }
  const DecodeStats& stats() const override { return stats_; }

  int decode_reference(const FrameSyntax& s, Frame* out, std::string* error) override {
    int slot = -1;
    return run(s, 1, -1, out, true, &slot, error) ? slot : -1;
  }

  bool decode(const FrameSyntax& s, Frame* out, std::string* error) override {
    int slot = -1;
    return run(s, 0, -1, out, true, &slot, error);
  }

  int decode_reference_reserved(const FrameSyntax& s, int slot, Frame* out, std::string* error,
                                bool read_back) override {
    if (slot < 0) {
      decode(s, out, error);
      return -1;
    }
    int got = -1;
    return run(s, 1, slot, out, read_back, &got, error) ? got : -1;
  }

  int reserve_reference() override {
    int s = -1;
    return av1b_reserve_reference(h_, &s) == AV1B_OK ? s : -1;
  }

  bool plan_frame(const FrameSyntax& s, void** plan, std::string* error,
                  std::atomic<bool>* cancel) override {
    if (!plan) {
      if (error) *error = "plan_frame: no output handle";
      return false;
    }
    if (cancel && cancel->load(std::memory_order_relaxed)) {
      if (error) *error = "planning cancelled";
      return false;
    }
    av1b::FlatSyntax f;
    av1b::view_from_cpp(s, &f);
    const av1b_frame_syntax v = f.view();
    av1b_plan* pl = nullptr;
    if (av1b_plan_frame(h_, &v, &pl) != AV1B_OK) {
      if (error) *error = av1b_last_error(h_);
      return false;
    }
    std::lock_guard<std::mutex> lk(mu_);
    plan_geom_[pl] = Geom{s.width, s.height, s.bit_depth, s.ss_x, s.ss_y};
    *plan = pl;
    return true;
  }

  int decode_reference_planned(void* plan, int slot, Frame* out, std::string* error,
                               bool read_back) override {
    auto* pl = static_cast<av1b_plan*>(plan);
    if (!pl) {
      if (error) *error = "decode_reference_planned: no plan";
      return -1;
    }
    Geom g;
    {
      std::lock_guard<std::mutex> lk(mu_);
      g = plan_geom_[pl];
      plan_geom_.erase(pl);
    }
    av1b_planes planes;
    const bool want = out && read_back;
    if (out && !out->matches(g.w, g.h, g.bd, g.sx, g.sy)) out->allocate(g.w, g.h, g.bd, g.sx, g.sy);
    if (want) fill_planes(out, &planes);
    int got = -1;
    const int rc = av1b_decode_planned(h_, pl, slot, slot >= 0 ? 1 : 0, want ? &planes : nullptr,
                                       &got, 1);
    av1b_plan_free(h_, pl);
    if (rc != AV1B_OK) {
      if (error) *error = av1b_last_error(h_);
      return -1;
    }
    geom_ = g;
    pull_stats();
    return got;
  }

  void discard_frame_plan(void* plan) override {
    if (!plan) return;
    {
      std::lock_guard<std::mutex> lk(mu_);
      plan_geom_.erase(plan);
    }
    av1b_plan_free(h_, static_cast<av1b_plan*>(plan));
  }

  bool supports_preplanning() const override { return true; }
  bool dequantises_on_device() const override { return true; }
  bool packs_nv12_on_device() const override { return true; }

  void release_reference(int slot) override { av1b_release_reference(h_, slot); }

  bool to_rgb(int slot, ColorMatrix matrix, ColorRange range, std::vector<uint8_t>* rgb,
              std::string* error) override {
    if (!rgb) return false;
    rgb->resize(static_cast<size_t>(geom_.w) * geom_.h * 3);
    if (av1b_to_rgb(h_, slot, static_cast<int>(matrix), static_cast<int>(range), rgb->data(),
                    rgb->size()) != AV1B_OK) {
      if (error) *error = av1b_last_error(h_);
      return false;
    }
    return true;
  }

  bool to_nv12(int slot, size_t pitch, std::vector<uint8_t>* nv12, std::string* error) override {
    const size_t bytes = av1b_nv12_size(geom_.w, geom_.h, geom_.sx, geom_.sy, pitch);
    if (bytes == 0 || !nv12) {
      if (error) *error = "NV12 output needs a 4:2:0 frame and an even pitch at least as wide";
      return false;
    }
    nv12->resize(bytes);
    if (av1b_to_nv12(h_, slot, pitch, nv12->data(), bytes) != AV1B_OK) {
      if (error) *error = av1b_last_error(h_);
      return false;
    }
    return true;
  }

  int nv12_pack_begin(int slot, size_t pitch, std::string* error) override {
    int handle = -1;
    if (av1b_nv12_pack_begin(h_, slot, pitch, &handle) != AV1B_OK) {
      if (error) *error = av1b_last_error(h_);
      return -1;
    }
    return handle;
  }

  bool nv12_pack_wait(int handle, std::vector<uint8_t>* nv12, std::string* error) override {
    const uint8_t* data = nullptr;
    size_t bytes = 0;
    if (av1b_nv12_pack_wait(h_, handle, nullptr, 0, &data, &bytes) != AV1B_OK) {
      if (error) *error = av1b_last_error(h_);
      return false;
    }
    if (nv12) nv12->assign(data, data + bytes);
    return true;
  }

  void nv12_pack_release(int handle) override { av1b_nv12_pack_release(h_, handle); }

  void hold_output(bool hold) override { hold_.store(hold, std::memory_order_relaxed); }

  void reset() override {
    av1b_decoder_reset(h_);
    stats_ = DecodeStats();
  }

 private:
  struct Geom {
    int w = 0, h = 0, bd = 8, sx = 1, sy = 1;
  };

  static void fill_planes(Frame* out, av1b_planes* pl) {
    for (int p = 0; p < 3; ++p) {
      pl->plane[p] = out->plane(p);
      pl->stride[p] = out->stride[p];
    }
  }

  bool run(const FrameSyntax& s, int keep, int slot, Frame* out, bool read_back, int* got,
           std::string* error) {
    av1b::FlatSyntax f;
    av1b::view_from_cpp(s, &f);
    const av1b_frame_syntax v = f.view();
    if (out && !out->matches(s.width, s.height, s.bit_depth, s.ss_x, s.ss_y))
      out->allocate(s.width, s.height, s.bit_depth, s.ss_x, s.ss_y);
    av1b_planes planes;
    const bool want = out && read_back;
    if (want) fill_planes(out, &planes);
    char err[512] = {0};
    int rc;
    if (slot >= 0)
      rc = av1b_decode_reserved(h_, &v, slot, want ? &planes : nullptr, err, sizeof(err));
    else
      rc = av1b_decode(h_, &v, keep, want ? &planes : nullptr, got, err, sizeof(err));
    if (rc != AV1B_OK) {
      if (error) *error = err;
      return false;
    }
    if (slot >= 0) *got = slot;
    geom_ = Geom{s.width, s.height, s.bit_depth, s.ss_x, s.ss_y};
    pull_stats();
    return true;
  }

  void pull_stats() {
    av1b_stats st;
    if (av1b_get_stats(h_, &st) != AV1B_OK) return;
    stats_.blocks = st.blocks;
    stats_.waves = st.waves;
    stats_.kernel_launches = st.kernel_launches;
    stats_.reconstruct_ms = st.reconstruct_ms;
    stats_.filter_ms = st.filter_ms;
    stats_.readback_ms = st.readback_ms;
    stats_.total_ms = st.total_ms;
  }

  av1b_decoder* h_;
  BackendOptions opt_;
  DeviceInfo info_;
  DecodeStats stats_;
  Geom geom_;
  std::mutex mu_;
  std::map<void*, Geom> plan_geom_;
  std::atomic<bool> hold_{false};
};

}  // namespace

std::unique_ptr<Decoder> Decoder::create(const BackendOptions& options, std::string* error) {
  std::string local;
  if (!error) error = &local;
  error->clear();
  if (options.kind == BackendKind::Cpu || options.kind == BackendKind::OpenCL) {
    *error = std::string("backend '") + to_string(options.kind) +
             "' is not part of this library: it has one backend, CUDA on sm_100a";
    return nullptr;
  }
  av1b_decoder* h = nullptr;
  const int rc = av1b_decoder_create(options.device_index, 0, &h);
  if (rc != AV1B_OK) {
    *error = rc == AV1B_ERR_NO_DEVICE ? "no CUDA device (this library has no CPU fallback)"
                                      : "CUDA decoder creation failed";
    return nullptr;
  }
  return std::unique_ptr<Decoder>(new B200Decoder(h, options));
}

std::unique_ptr<Decoder> create_best_decoder(const BackendOptions& options, std::string* error) {
  return Decoder::create(options, error);
}

}  // namespace av1gpu
