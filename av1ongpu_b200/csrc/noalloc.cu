/*
 * noalloc.cu - film grain synthesis for callers that cannot allocate.
 *
 * Some callers of this library cannot call cudaMalloc at the point where they
 * want a frame's film grain: a player's display callback that re-shows a
 * reference slot (the slot holds the picture before grain) under a real-time
 * deadline, where cudaMalloc / cudaFree may synchronize the whole device; a
 * host application that fixes its device memory at start-up and forbids any
 * later allocation. av1b_apply_film_grain_noalloc serves them: the caller
 * passes the input picture and the output planes (device memory it owns), and
 * the call allocates nothing - no cudaMalloc, no cudaFree, no allocating
 * library routine.
 *
 * Its scratch - the grain templates and scaling tables of the frame, and the
 * two 65536-entry tables of the grain LFSR - lives in the file-scope array
 * below, g_noalloc_scratch, of AV1B_NOALLOC_SCRATCH_BYTES (about 300 KB).
 * Every GPU that loads the library holds it until the process exits. The
 * scratch does not grow with the picture; pictures up to
 * AV1B_NOALLOC_MAX_DIM samples on a side are accepted, larger ones refused.
 *
 * The array's name in host code is a host-side stand-in, not a device
 * address. The first call on each device resolves the address with
 * cudaGetSymbolAddress (with that device current), builds the LFSR tables in
 * the scratch and waits for that, once; make that first call before any
 * stream capture. Every call shares the scratch and leaves the last call's
 * contents in it (each call rewrites the templates and tables it reads before
 * reading them), so calls that overlap on the GPU - two streams, or two host
 * threads - race: serialize them.
 */
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/av1b.h"
#include "dev_grain.cuh"
#include "kernels.h"

namespace av1b {
namespace {

constexpr size_t kGrainBytes = (sizeof(GrainState) + 255) & ~static_cast<size_t>(255);
constexpr size_t kTableBytes = 65536 * sizeof(uint16_t);
constexpr size_t kScratchBytes = kGrainBytes + 2 * kTableBytes;
static_assert(kScratchBytes == AV1B_NOALLOC_SCRATCH_BYTES, "scratch size of av1b.h");

/* The scratch: [GrainState][LFSR orbit][LFSR position]. */
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct DeviceScratch {
  bool ready = false;
  unsigned char* ptr = nullptr;
};
std::mutex g_mu;
DeviceScratch g_dev[64];

/* Walks the grain LFSR once from state 1: orbit[k] is the state after k
 * steps, pos[s] the step at which state s occurs (period 65535). */
__global__ void k_lfsr_tables(uint16_t* orbit, uint16_t* pos) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  unsigned s = 1;
  for (unsigned k = 0; k < 65535; ++k) {
    orbit[k] = static_cast<uint16_t>(s);
    pos[s] = static_cast<uint16_t>(k);
    const unsigned bit = ((s >> 0) ^ (s >> 1) ^ (s >> 3) ^ (s >> 12)) & 1u;
    s = (s >> 1) | (bit << 15);
  }
  orbit[65535] = 0;
  pos[0] = 0;
}

struct GrainSetup {
  av1b_film_grain f;
  int bitdepth, ss_x, ss_y, identity;
};

__device__ void lut_of(int num, const int32_t* value, const int32_t* scaling, int* lut) {
  if (num <= 0) {
    for (int x = 0; x < 256; ++x) lut[x] = 0;
    return;
  }
  for (int x = 0; x < value[0]; ++x) lut[x] = scaling[0];
  for (int i = 0; i + 1 < num; ++i) {
    const int dy = scaling[i + 1] - scaling[i];
    const int dx = value[i + 1] - value[i];
    const int delta = dy * ((65536 + (dx >> 1)) / dx);
    for (int x = 0; x < dx; ++x) lut[value[i] + x] = scaling[i] + ((x * delta + 32768) >> 16);
  }
  for (int x = value[num - 1]; x < 256; ++x) lut[x] = scaling[num - 1];
}

/* The frame's grain constants and scaling tables (scaling_lookup_initialization,
 * the clip range), written into the scratch's GrainState. */
__global__ void k_grain_prepare(GrainState* gs, GrainSetup s) {
  const av1b_film_grain& f = s.f;
  const int t = threadIdx.x;
  const bool chroma = f.chroma_scaling_from_luma || f.num_cb_points > 0 || f.num_cr_points > 0;
  if (t == 0) lut_of(f.num_y_points, f.point_y_value, f.point_y_scaling, gs->lut[0]);
  if (t == 1) {
    if (!chroma) for (int x = 0; x < 256; ++x) gs->lut[1][x] = 0;
    else if (f.chroma_scaling_from_luma) lut_of(f.num_y_points, f.point_y_value, f.point_y_scaling, gs->lut[1]);
    else lut_of(f.num_cb_points, f.point_cb_value, f.point_cb_scaling, gs->lut[1]);
  }
  if (t == 2) {
    if (!chroma) for (int x = 0; x < 256; ++x) gs->lut[2][x] = 0;
    else if (f.chroma_scaling_from_luma) lut_of(f.num_y_points, f.point_y_value, f.point_y_scaling, gs->lut[2]);
    else lut_of(f.num_cr_points, f.point_cr_value, f.point_cr_scaling, gs->lut[2]);
  }
  if (t == 3) {
    const int bd = s.bitdepth, maxv = (1 << bd) - 1;
    gs->seed = f.seed;
    gs->bitdepth = bd;
    gs->overlap = f.overlap_flag ? 1 : 0;
    gs->scaling_shift = f.grain_scaling_minus_8 + 8;
    gs->num_points[0] = f.num_y_points;
    gs->num_points[1] = f.num_cb_points;
    gs->num_points[2] = f.num_cr_points;
    gs->chroma_from_luma = f.chroma_scaling_from_luma ? 1 : 0;
    gs->mult[1] = f.cb_mult;
    gs->luma_mult[1] = f.cb_luma_mult;
    gs->offset[1] = f.cb_offset;
    gs->mult[2] = f.cr_mult;
    gs->luma_mult[2] = f.cr_luma_mult;
    gs->offset[2] = f.cr_offset;
    gs->min_value = 0;
    gs->max_luma = maxv;
    gs->max_chroma = maxv;
    if (f.clip_to_restricted_range) {
      gs->min_value = 16 << (bd - 8);
      gs->max_luma = 235 << (bd - 8);
      gs->max_chroma = s.identity ? gs->max_luma : (240 << (bd - 8));
    }
    gs->chroma_w = s.ss_x ? 44 : 82;
    gs->chroma_h = s.ss_y ? 38 : 73;
  }
}

struct PlaneArgs {
  const uint16_t* src[3];
  int src_stride[3];
  uint16_t* dst[3];
  int dst_stride[3];
  int w[3], h[3];
  int ss_x, ss_y;
};

/* The blend over three separately allocated planes (the decoder's k_grain_blend
 * over caller planes): one thread per sample. */
__global__ void k_grain_blend_planes(PlaneArgs a, const GrainState* gs, const uint16_t* orbit,
                                     const uint16_t* pos) {
  const int p = blockIdx.z;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= a.w[p] || y >= a.h[p]) return;
  const int orig = a.src[p][static_cast<size_t>(y) * a.src_stride[p] + x];
  int l0 = 0, l1 = 0;
  if (p > 0) {
    const int ly = y << a.ss_y, lx = x << a.ss_x;
    const int nx = lx + 1 < a.w[0] ? lx + 1 : a.w[0] - 1;
    const uint16_t* row = a.src[0] + static_cast<size_t>(ly) * a.src_stride[0];
    l0 = row[lx];
    l1 = row[nx];
  }
  a.dst[p][static_cast<size_t>(y) * a.dst_stride[p] + x] = static_cast<uint16_t>(
      grain_sample(gs, orbit, pos, p, p ? a.ss_x : 0, p ? a.ss_y : 0, x, y, orig, l0, l1));
}

/* Resolves this device's scratch address and builds the LFSR tables, once. */
int device_scratch(unsigned char** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return AV1B_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceScratch& d = g_dev[dev];
  if (!d.ready) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return AV1B_ERR_CUDA;
    unsigned char* base = static_cast<unsigned char*>(p);
    k_lfsr_tables<<<1, 32>>>(reinterpret_cast<uint16_t*>(base + kGrainBytes),
                             reinterpret_cast<uint16_t*>(base + kGrainBytes + kTableBytes));
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
      return AV1B_ERR_CUDA;
    d.ptr = base;
    d.ready = true;
  }
  *out = d.ptr;
  return AV1B_OK;
}

/* The bytes a plane of w x h samples at `stride` spans: [lo, hi). */
struct Span {
  uintptr_t lo, hi;
};
Span plane_span(const void* base, int stride, int w, int h) {
  const uintptr_t lo = reinterpret_cast<uintptr_t>(base);
  return Span{lo, lo + (static_cast<uintptr_t>(h - 1) * stride + w) * sizeof(uint16_t)};
}
bool overlap(const Span& a, const Span& b) { return a.lo < b.hi && b.lo < a.hi; }

bool grain_params_ok(const av1b_film_grain& f) {
  if (f.seed < 0 || f.seed > 65535 || f.ar_coeff_lag < 0 || f.ar_coeff_lag > 3 ||
      f.num_y_points < 0 || f.num_y_points > 16 || f.num_cb_points < 0 || f.num_cb_points > 16 ||
      f.num_cr_points < 0 || f.num_cr_points > 16 || f.grain_scaling_minus_8 < 0 ||
      f.grain_scaling_minus_8 > 3 || f.ar_coeff_shift_minus_6 < 0 || f.ar_coeff_shift_minus_6 > 3 ||
      f.grain_scale_shift < 0 || f.grain_scale_shift > 3)
    return false;
  const int32_t* v[3] = {f.point_y_value, f.point_cb_value, f.point_cr_value};
  const int n[3] = {f.num_y_points, f.num_cb_points, f.num_cr_points};
  for (int p = 0; p < 3; ++p)
    for (int i = 0; i < n[p]; ++i)
      if (v[p][i] < 0 || v[p][i] > 255 || (i > 0 && v[p][i] <= v[p][i - 1])) return false;
  return true;
}

}  // namespace
}  // namespace av1b

using namespace av1b;

extern "C" int av1b_apply_film_grain_noalloc(const av1b_frame_syntax* s, const uint16_t* const src[3],
                                             const int32_t src_stride[3], uint16_t* const dst[3],
                                             const int32_t dst_stride[3], void* stream) {
  if (!s || !src || !dst || !src_stride || !dst_stride) return AV1B_ERR_ARG;
  if (s->width <= 0 || s->height <= 0 || s->width > AV1B_NOALLOC_MAX_DIM ||
      s->height > AV1B_NOALLOC_MAX_DIM)
    return AV1B_ERR_ARG; /* beyond the stated maximum of this entry point */
  if (s->bit_depth != 8 && s->bit_depth != 10 && s->bit_depth != 12) return AV1B_ERR_ARG;
  if (s->ss_x < 0 || s->ss_x > 1 || s->ss_y < 0 || s->ss_y > 1 || (s->ss_y && !s->ss_x))
    return AV1B_ERR_ARG;
  PlaneArgs a{};
  a.ss_x = s->ss_x;
  a.ss_y = s->ss_y;
  for (int p = 0; p < 3; ++p) {
    a.w[p] = p ? (s->width + s->ss_x) >> s->ss_x : s->width;
    a.h[p] = p ? (s->height + s->ss_y) >> s->ss_y : s->height;
    if (!src[p] || !dst[p] || src_stride[p] < a.w[p] || dst_stride[p] < a.w[p]) return AV1B_ERR_ARG;
    a.src[p] = src[p];
    a.dst[p] = dst[p];
    a.src_stride[p] = src_stride[p];
    a.dst_stride[p] = dst_stride[p];
  }
  /* The blend of a chroma sample reads the co-located luma of the input
   * while other blocks write the output: an output plane that shares bytes
   * with any input plane (in-place grain) or with another output plane would
   * make the result depend on the order the GPU runs the blocks in. */
  for (int p = 0; p < 3; ++p) {
    const Span d = plane_span(dst[p], dst_stride[p], a.w[p], a.h[p]);
    for (int q = 0; q < 3; ++q) {
      if (overlap(d, plane_span(src[q], src_stride[q], a.w[q], a.h[q]))) return AV1B_ERR_ARG;
      if (q != p && overlap(d, plane_span(dst[q], dst_stride[q], a.w[q], a.h[q]))) return AV1B_ERR_ARG;
    }
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  /* the scratch resolved below is the current device's: a stream of another
   * device could not reach it */
  if (st != nullptr) {
    int cur = -1, sdev = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cudaStreamGetDevice(st, &sdev) != cudaSuccess)
      return AV1B_ERR_CUDA;
    if (sdev != cur) return AV1B_ERR_ARG;
  }
  if (!s->grain.apply) {
    /* no grain: the output picture is the input */
    for (int p = 0; p < 3; ++p)
      if (cudaMemcpy2DAsync(dst[p], static_cast<size_t>(dst_stride[p]) * 2, src[p],
                            static_cast<size_t>(src_stride[p]) * 2, static_cast<size_t>(a.w[p]) * 2,
                            a.h[p], cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return AV1B_ERR_CUDA;
    return AV1B_OK;
  }
  if (!grain_params_ok(s->grain)) return AV1B_ERR_SYNTAX;
  unsigned char* base = nullptr;
  int rc = device_scratch(&base);
  if (rc) return rc;
  GrainState* gs = reinterpret_cast<GrainState*>(base);
  const uint16_t* orbit = reinterpret_cast<const uint16_t*>(base + kGrainBytes);
  const uint16_t* pos = reinterpret_cast<const uint16_t*>(base + kGrainBytes + kTableBytes);

  GrainSetup su;
  su.f = s->grain;
  su.bitdepth = s->bit_depth;
  su.ss_x = s->ss_x;
  su.ss_y = s->ss_y;
  su.identity = s->color_matrix == 3;
  k_grain_prepare<<<1, 32, 0, st>>>(gs, su);
  GrainParamsDev g;
  std::memset(&g, 0, sizeof(g));
  const av1b_film_grain& f = s->grain;
  g.seed = f.seed;
  g.bitdepth = s->bit_depth;
  g.ss_x = s->ss_x;
  g.ss_y = s->ss_y;
  g.num_y_points = f.num_y_points;
  g.num_cb_points = f.num_cb_points;
  g.num_cr_points = f.num_cr_points;
  g.chroma_scaling_from_luma = f.chroma_scaling_from_luma ? 1 : 0;
  g.ar_coeff_lag = f.ar_coeff_lag;
  g.ar_coeff_shift_minus_6 = f.ar_coeff_shift_minus_6;
  g.grain_scale_shift = f.grain_scale_shift;
  for (int i = 0; i < 24; ++i) g.ar_y[i] = f.ar_coeffs_y[i];
  for (int i = 0; i < 25; ++i) {
    g.ar_cb[i] = f.ar_coeffs_cb[i];
    g.ar_cr[i] = f.ar_coeffs_cr[i];
  }
  if (launch_grain_template(gs, g, orbit, pos, st) != cudaSuccess) return AV1B_ERR_CUDA;
  const dim3 grid((a.w[0] + 127) / 128, a.h[0], 3);
  k_grain_blend_planes<<<grid, 128, 0, st>>>(a, gs, orbit, pos);
  return cudaGetLastError() == cudaSuccess ? AV1B_OK : AV1B_ERR_CUDA;
}
