/*
 * decoder.cu - the host engine behind the C ABI (include/av1b.h).
 *
 * It replaces the reference's EngineDecoder + CudaBackend pair
 * (src/core/engine.cpp, src/backends/cuda/cuda_backend.cpp) with one object:
 *
 *   plan    FrameSyntax -> compact device records, O(blocks), no wavefront:
 *           BlockRec per block, TxRec per coded transform, OBMC strips, warp
 *           models, edge / CDEF / restoration records, grain constants; every
 *           offset is validated here so no kernel can address outside its
 *           buffers;
 *   upload  one pinned staging arena -> one device arena per frame, plus the
 *           coefficient and residual pools;
 *   run     the frame step on one CUDA stream: reconstruction (phase A, then
 *           the dependency-scheduled phase B), deblock V then H, CDEF,
 *           superres, loop restoration, reference store, film grain;
 *   output  the display picture back to the caller, or NV12 / RGB packed on
 *           the device.
 *
 * Slot semantics follow the reference CPU backend (cpu_backend.cpp:93-553):
 * a slot holds the picture before film grain; the frame decoded last is also
 * kept after film grain, and that is what the output calls of its slot read.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "../../include/av1b.h"
#include "flat_syntax.hpp"
#include "dev_inter.cuh"
#include "dev_itx.cuh"
#include "kernels.h"
#include "batch.h"
#include "work_pool.hpp"
#include "plan_host.h"

namespace av1b {
namespace {

constexpr int kSlots = 32;       /* reference slots, as the reference's pools */
constexpr int kPadLuma = 128;    /* right/bottom border for block overhang */

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

}  // namespace
}  // namespace av1b

using namespace av1b;

namespace av1b {
namespace {
struct PlanScratch;
struct PlanLists;
}
}  // namespace av1b

struct av1b_decoder {
  int device = 0;
  cudaStream_t stream = nullptr;
  int n_sm = 148;
  size_t budget = 0, allocated = 0;
  std::mutex mu;                 /* one decode, output or slot call at a time */
  /* Planning runs outside `mu` (a pipeline plans frames N+1, N+2 on their
   * own threads while frame N runs), on one of a few planners - each a host
   * thread pool, scratch, record lists and an upload stream - taken one
   * plan_frame at a time (planner_mu / planner_cv). slot_mu guards the slot
   * table planners read, err_mu the error text, alloc_mu the HBM account.
   * Lock order: mu, a planner, slot_mu / alloc_mu / err_mu. */
  std::mutex planner_mu, slot_mu, err_mu, alloc_mu, prof_mu;
  std::condition_variable planner_cv;
  struct Planner {
    av1b::WorkPool* pool = nullptr;
    av1b::PlanScratch* scratch = nullptr;
    av1b::PlanLists* lists = nullptr;  /* the record lists (page-locked) */
    cudaStream_t upload = nullptr;     /* its uploads, overlapping frames in flight */
    bool busy = false;
  };
  std::vector<Planner> planners;
  /* freed plans kept with their buffers for the next av1b_plan_frame */
  std::mutex plan_pool_mu;
  std::vector<struct av1b_plan*> plan_pool;
  /* The largest capacity any planner's record list (elements) and any plan's
   * arena and filter buffer (bytes) has needed. A planner or plan that has
   * not held so large a frame grows to it when it is next taken, so the
   * growth - a page-locked allocation stalls every CUDA call of the process,
   * a device free waits for the device - happens once, early in a stream
   * (after its first key frame), not whenever a planner or plan first meets
   * a key frame. Guarded by hw_mu. */
  std::mutex hw_mu;
  size_t list_hw[32] = {};
  size_t arena_hw = 0, filt_hw = 0;

  /* geometry of the pictures currently allocated */
  bool have_geom = false;
  int width = 0, height = 0, coded_width = 0, bit_depth = 8, ss_x = 1, ss_y = 1;
  Layout L{};

  /* pictures */
  DevBuf cur, snap, lr_pre_up, lr_cdef, disp;
  DevBuf cdef_search;             /* CDEF direction search results */
  DevBuf pre_res;                 /* phase B residuals computed ahead */
  DevBuf mask_pool;               /* difference-weighted luma masks chroma tiles read */
  bool disp_is_cur = true;
  /* a batched step applied the last frame's film grain inside its NV12 pack:
   * the display picture is made from cur when an output call asks for it */
  bool disp_pending = false;
  cudaEvent_t ev_batch = nullptr;   /* a batched step's wait on this decoder's stream */
  /* a batched step ran this decoder's frame on the batch's stream: the
   * decoder's own stream joins it (waits for ev_after_batch) only when a call
   * next queues work there, so back-to-back batched steps never wait on it */
  bool batch_pending = false;
  cudaEvent_t ev_after_batch = nullptr;
  DevBuf slot_buf[kSlots];
  bool slot_used[kSlots] = {false};
  bool slot_valid[kSlots] = {false};
  int slot_width[kSlots] = {0}, slot_height[kSlots] = {0}, slot_bd[kSlots] = {0};
  DevBuf slot_ptr_dev;
  int last_slot = -1;
  bool have_last = false;

  /* per-frame buffers */
  DevBuf arena, coef, residual, done, status_q, nv12, rgb;
  unsigned epoch = 0;

  /* film grain */
  DevBuf grain_state, orbit, pos;
  bool grain_tables = false;

  av1b_stats stats{};
  bool stats_pending = false;
  std::string err;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  /* a side stream for work that depends only on the frame's parameters (the
   * film grain templates), joined before its consumer */
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaEvent_t ev_block = nullptr;  /* blocking-sync event: host waits on the stream */
  int* status_host = nullptr;          /* pinned */
  void* slot_ptr_host[32] = {nullptr};
  struct av1b_plan* own_plan = nullptr;

  /* split NV12 packs (av1b_nv12_pack_begin / wait / release): each entry a
   * device buffer the pack kernel writes on the decoder's stream and a
   * page-locked one the copy stream reads it back into, so the read back
   * overlaps the next frame's decode. pack_mu guards the table; a wait does
   * not hold `mu`. */
  struct Pack {
    DevBuf dev;
    uint8_t* host = nullptr;
    size_t host_cap = 0, bytes = 0;
    cudaEvent_t packed = nullptr, copied = nullptr;
    int handle = -1;               /* -1: free */
  };
  std::mutex pack_mu;
  std::vector<Pack> packs;
  int next_pack = 0;
  cudaStream_t copy_stream = nullptr;

  /* chroma blocks of difference-weighted compounds read their luma block's
   * mask when it is the same prediction (av1b_set_shared_masks) */
  std::atomic<bool> share_masks{true};

  /* optional trace of phase B (av1b_set_unit_trace): 4 uint64 per block */
  bool tracing = false;
  DevBuf trace;
  size_t trace_n = 0;

  /* optional per-stage device timing (CUDA events on the decoder's stream) */
  unsigned long long wait_ns = 1000000000ull;   /* one dependency wait: 1 s */
  bool profiling = false;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  std::vector<std::pair<int, size_t>> marks;   /* (stage, index of its start event) */
  double prof_ms[24] = {0};
  long long prof_n[24] = {0};
};

namespace av1b {
namespace {

int fail(av1b_decoder* d, int code, const std::string& msg) {
  std::lock_guard<std::mutex> lk(d->err_mu);
  d->err = msg;
  return code;
}

int cuda_fail(av1b_decoder* d, cudaError_t e, const char* what) {
  std::lock_guard<std::mutex> lk(d->err_mu);
  d->err = std::string(what) + ": " + cudaGetErrorString(e);
  return AV1B_ERR_CUDA;
}

void clear_err(av1b_decoder* d) {
  std::lock_guard<std::mutex> lk(d->err_mu);
  d->err.clear();
}

/* Waits for the decoder's stream without spinning a core (the planner pool
 * and a planning thread share the host). Called with the decoder lock. */
cudaError_t wait_stream(av1b_decoder* d) {
  const cudaError_t e = cudaEventRecord(d->ev_block, d->stream);
  return e != cudaSuccess ? e : cudaEventSynchronize(d->ev_block);
}

/* Orders the decoder's stream after its last batched step (see
 * batch_pending). Called with the decoder lock, before queueing work. */
void join_batch(av1b_decoder* d) {
  if (d->batch_pending) {
    cudaStreamWaitEvent(d->stream, d->ev_after_batch, 0);
    d->batch_pending = false;
  }
}

#define CK(call, what)                                     \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return cuda_fail(d, e_, what);  \
  } while (0)

/* Makes `b` hold at least `bytes`; when it has to grow, it takes `room`
 * bytes if that is more (and the HBM budget allows), so buffers whose need
 * varies frame to frame grow once rather than at every larger frame - each
 * cudaFree waits for the whole device. */
int dev_ensure(av1b_decoder* d, DevBuf& b, size_t bytes, size_t room = 0) {
  if (bytes == 0) bytes = 256;
  if (b.cap >= bytes) return AV1B_OK;
  size_t want = align_up(bytes + bytes / 8, 1 << 16);
  {
    std::lock_guard<std::mutex> lk(d->alloc_mu);
    const size_t roomy = align_up(room, 1 << 16);
    if (roomy > want && (!d->budget || d->allocated - b.cap + roomy <= d->budget)) want = roomy;
    if (d->budget && d->allocated - b.cap + want > d->budget)
      return fail(d, AV1B_ERR_NOMEM, "decoder HBM budget exhausted");
    d->allocated -= b.cap;
  }
  if (b.p) {
    cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
  }
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, want);
  if (e != cudaSuccess) return cuda_fail(d, e, "cudaMalloc");
  b.p = p;
  b.cap = want;
  std::lock_guard<std::mutex> lk(d->alloc_mu);
  d->allocated += want;
  return AV1B_OK;
}

void dev_release(av1b_decoder* d, DevBuf& b) {
  if (b.p) {
    cudaFree(b.p);
    std::lock_guard<std::mutex> lk(d->alloc_mu);
    d->allocated -= b.cap;
  }
  b.p = nullptr;
  b.cap = 0;
}

Layout make_layout(int width, int height, int coded_width, int bd, int ss_x, int ss_y) {
  Layout L{};
  L.ss_x = ss_x;
  L.ss_y = ss_y;
  L.bit_depth = bd;
  long long size = 0;
  for (int p = 0; p < 3; ++p) {
    const int sx = p ? ss_x : 0, sy = p ? ss_y : 0;
    PlaneGeom& g = L.p[p];
    g.out_w = (width + sx) >> sx;
    g.out_h = (height + sy) >> sy;
    g.coded_w = (coded_width + sx) >> sx;
    g.coded_h = g.out_h;
    g.grid_w = ((coded_width + 7) & ~7) >> sx;
    g.grid_h = ((height + 7) & ~7) >> sy;
    const int padx = kPadLuma >> sx, pady = kPadLuma >> sy;
    g.stride = static_cast<int>(align_up(static_cast<size_t>(std::max(g.out_w, g.grid_w) + padx), 64));
    g.off = static_cast<int>(size);
    size += static_cast<long long>(g.stride) * (std::max(g.out_h, g.grid_h) + pady);
    size = align_up(size, 64);
  }
  L.size = size;
  return L;
}

int plane_rows(const Layout& L, int p) {
  return static_cast<int>(((p < 2 ? L.p[p + 1].off : L.size) - L.p[p].off) / L.p[p].stride);
}

/* (Re)allocates the pictures for a geometry. Slots keep their contents and
 * their own geometry tag; a frame may only reference slots of its size. */
int ensure_geometry(av1b_decoder* d, const av1b_frame_syntax& s, int coded_width) {
  if (d->have_geom && d->width == s.width && d->height == s.height &&
      d->coded_width == coded_width && d->bit_depth == s.bit_depth && d->ss_x == s.ss_x &&
      d->ss_y == s.ss_y)
    return AV1B_OK;
  const Layout L = make_layout(s.width, s.height, coded_width, s.bit_depth, s.ss_x, s.ss_y);
  const bool same_pictures = d->have_geom && L.size == d->L.size && d->width == s.width &&
                             d->height == s.height && d->bit_depth == s.bit_depth &&
                             d->ss_x == s.ss_x && d->ss_y == s.ss_y;
  const size_t bytes = static_cast<size_t>(L.size) * sizeof(px_t);
  int rc;
  if ((rc = dev_ensure(d, d->cur, bytes)) || (rc = dev_ensure(d, d->snap, bytes)) ||
      (rc = dev_ensure(d, d->disp, bytes)))
    return rc;
  if (!same_pictures) {
    /* a different display geometry: the slots' pictures are unusable */
    std::lock_guard<std::mutex> lk(d->slot_mu);
    for (int i = 0; i < kSlots; ++i) d->slot_valid[i] = false;
  }
  d->L = L;
  d->width = s.width;
  d->height = s.height;
  d->coded_width = coded_width;
  d->bit_depth = s.bit_depth;
  d->ss_x = s.ss_x;
  d->ss_y = s.ss_y;
  d->have_geom = true;
  d->have_last = false;
  return AV1B_OK;
}

int init_grain_tables(av1b_decoder* d) {
  if (d->grain_tables) return AV1B_OK;
  int rc;
  if ((rc = dev_ensure(d, d->orbit, 65536 * 2)) || (rc = dev_ensure(d, d->pos, 65536 * 2)) ||
      (rc = dev_ensure(d, d->grain_state, sizeof(GrainState))))
    return rc;
  std::vector<uint16_t> orbit(65536, 0), pos(65536, 0);
  unsigned s = 1;
  for (unsigned k = 0; k < 65535; ++k) {
    orbit[k] = static_cast<uint16_t>(s);
    pos[s] = static_cast<uint16_t>(k);
    const unsigned bit = ((s >> 0) ^ (s >> 1) ^ (s >> 3) ^ (s >> 12)) & 1u;
    s = (s >> 1) | (bit << 15);
  }
  CK(cudaMemcpy(d->orbit.p, orbit.data(), 65536 * 2, cudaMemcpyHostToDevice), "orbit upload");
  CK(cudaMemcpy(d->pos.p, pos.data(), 65536 * 2, cudaMemcpyHostToDevice), "pos upload");
  d->grain_tables = true;
  return AV1B_OK;
}

/* ---- the planner ------------------------------------------------------------------------- */

/* Page-locked host memory for the plan's record lists, so they upload
 * straight from where the planner wrote them (no staging copy). A plan keeps
 * its lists between frames, so allocations stop once the sizes settle. */
template <class T>
struct PinnedAlloc {
  using value_type = T;
  PinnedAlloc() = default;
  template <class U>
  PinnedAlloc(const PinnedAlloc<U>&) {}
  T* allocate(size_t n) {
    void* p = nullptr;
    if (cudaHostAlloc(&p, std::max<size_t>(n, 1) * sizeof(T), cudaHostAllocDefault) != cudaSuccess)
      throw std::bad_alloc();
    return static_cast<T*>(p);
  }
  void deallocate(T* p, size_t) { cudaFreeHost(p); }
  /* resize() leaves new elements uninitialised: every list is written in
   * full by the planner, and zeroing megabytes first is serial work */
  template <class U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <class U, class... Args>
  void construct(U* p, Args&&... args) {
    ::new (static_cast<void*>(p)) U(std::forward<Args>(args)...);
  }
  template <class U>
  bool operator==(const PinnedAlloc<U>&) const { return true; }
  template <class U>
  bool operator!=(const PinnedAlloc<U>&) const { return false; }
};
template <class T>
using pvec = std::vector<T, PinnedAlloc<T>>;

/* The record lists a plan builds, in page-locked host memory so they upload
 * from where the planner wrote them. One set per planner: a planner plans one
 * frame at a time and a plan's uploads finish before plan_frame returns, so
 * its lists are free again then. Their capacity is kept, and grown to the
 * largest any planner has needed when the planner is next taken - no
 * page-locked allocation, which stalls every CUDA call of the process, in the
 * steady state. */
struct PlanLists {
  pvec<BlockRec> blocks;
  pvec<TxRec> txs;
  pvec<ObmcRec> obmc;
  pvec<WarpRec> warps;
  pvec<int> palette_colors;
  pvec<int> units;                /* phase B blocks, chain after chain */
  pvec<int> chains;               /* where each chain starts in `units`, and the end */
  pvec<int> deps;                 /* per phase B block (dep_first, dep_count): the
                                     phase B blocks it waits for */
  pvec<int2> inter_tiles;
  pvec<int2> itx_jobs;            /* sorted by size class, then shape and type */
  pvec<int4> itx_batches;         /* (first job, jobs, log2 class or 7 = raw) */
  pvec<LrUnitRec> lr_units[3];
  pvec<DqRec> dq;                 /* coded transforms to dequantise (levels frames) */
};

/* Calls f(index, list) for every list of R. */
template <class F>
void each_list(PlanLists& R, F&& f) {
  int i = 0;
  f(i++, R.blocks);
  f(i++, R.txs);
  f(i++, R.obmc);
  f(i++, R.warps);
  f(i++, R.palette_colors);
  f(i++, R.units);
  f(i++, R.chains);
  f(i++, R.deps);
  f(i++, R.inter_tiles);
  f(i++, R.itx_jobs);
  f(i++, R.itx_batches);
  for (int p = 0; p < 3; ++p) f(i++, R.lr_units[p]);
  f(i++, R.dq);
}

/* One planned frame's constants and record counts (its records live in
 * device memory, uploaded from the PlanLists). */
/* Sizes a page-locked list, growing it with half again as much room: a
 * page-locked allocation stalls every CUDA call of the process, so lists
 * grow rarely and early (the key frame's lists are the largest). */
template <class V>
void sized(V& v, size_t n) {
  if (n > v.capacity()) v.reserve(n + n / 2);
  v.resize(n);
}

struct Plan {
  PlanLists* R = nullptr;         /* while planning: the lists being built */
  size_t n_tiles_simple = 0;      /* unmasked inter tiles (the lean kernel, listed first) */
  size_t n_tiles_lmask = 0;       /* masked tiles the lean kernel takes (listed next) */
  size_t n_tiles_cmask = 0;       /* chroma tiles reading a luma block's mask (listed last) */
  size_t mask_pool = 0;           /* bytes of the difference-weighted luma masks */
  size_t n_blocks = 0, n_units = 0, n_chains = 0, n_tiles = 0, n_itx = 0, n_itxb = 0, n_dbv = 0, n_dbh = 0,
         n_cdef = 0,
         n_cdef_search = 0;
  int unit_depth = 0;             /* dependency depth of the frame */
  /* chains by the depth of their first block: chains [depth_first[k],
   * depth_first[k + 1]) start at depth k (a batched step interleaves the
   * streams' chains by it) */
  std::vector<int> depth_first;
  bool units_inter = false;       /* some phase B block is an inter kind */
  int itx_class_first[8] = {0}, itx_class_count[8] = {0};  /* batches per class */
  int cdef_grid_w = 0, cdef_grid_n = 0;  /* the grid of 8x8 luma searches */
  bool cdef_search_any = false;          /* some record reads the grid */
  LrArgs lr{};
  bool use_lr = false;
  size_t coef_pool = 0, residual_pool = 0;
  size_t pre_res_pool = 0;        /* ints of residual computed ahead (phase B) */
  size_t n_dq = 0;                /* transforms the device dequantises */
  size_t unit_samples = 0, inter_samples = 0, inter_ref_samples = 0, tx_samples = 0,
         coef_samples = 0;        /* work counts, summed over the planner's pieces */
  int scale_x = AV1B_SCALE_ONE, scale_y = AV1B_SCALE_ONE;
  bool upscaled = false;
  bool grain = false;
  GrainParamsDev gp{};
  GrainState gs_tail;   /* only the constants after the templates are used */
};

/* What the planner reads of the decoder: the frame's layout and the state of
 * the reference slots, copied under the slot lock when planning starts, so a
 * frame can be planned on another thread while earlier frames run. */
struct PlanCtx {
  Layout L;
  bool slot_used[kSlots], slot_valid[kSlots];
  int slot_width[kSlots], slot_height[kSlots];
  WorkPool* pool = nullptr;
  struct PlanScratch* scratch = nullptr;
  /* the frame carries coded levels: the device builds the coefficient
   * rasters from them (and the frame's coefficient array is not read) */
  bool levels = false;
  size_t n_levels = 0, n_qm = 0;
  bool share_masks = true;        /* plan_shared_masks runs */
};

/* The first error one piece of the planner met. */
struct PlanErr {
  int code = AV1B_OK;
  std::string msg;
  int set(int c, const char* m) {
    if (code == AV1B_OK) {
      code = c;
      msg = m;
    }
    return c;
  }
};

/* Maps a block's reference index to a device slot. At planning time a slot
 * only has to be held or reserved (a pipeline plans a frame before the frame
 * it references has been decoded); execute_plan checks that it holds a
 * picture of this size by the time the plan runs. */
int resolve_slot(const PlanCtx& c, PlanErr& e, const av1b_frame_syntax& s, int ref, int* slot) {
  *slot = -1;
  if (ref < 0 || ref >= static_cast<int>(s.n_reference_slots)) return AV1B_OK;
  const int sl = s.reference_slots[ref];
  if (sl < 0 || sl >= kSlots) return AV1B_OK;
  if (!c.slot_used[sl])
    return e.set(AV1B_ERR_SYNTAX, "a block references a slot that is neither held nor reserved");
  if (c.slot_valid[sl] && (c.slot_width[sl] != s.width || c.slot_height[sl] != s.height))
    return e.set(AV1B_ERR_SYNTAX,
                 "engine: reference scaling between pictures of different sizes is not supported");
  *slot = sl;
  return AV1B_OK;
}

bool pow2_in(int v, int lo, int hi) { return v >= lo && v <= hi && (v & (v - 1)) == 0; }

/* The records of the blocks of one piece of the frame. List indices in the
 * block records (tx_first, obmc_first, palette_color_idx, warp_idx - 1 based
 * - and pre_off) are local to the piece until build_plan adds the piece's
 * offsets. */
struct BlockOut {
  std::vector<TxRec> txs;
  std::vector<ObmcRec> obmc;
  std::vector<WarpRec> warps;
  std::vector<int> palette_colors;
  std::vector<int> units;
  std::vector<int2> inter_tiles, inter_tiles_mask, inter_tiles_full;
  std::vector<int2> itx_jobs;
  std::vector<DqRec> dq;
  size_t pre_res_pool = 0, coef_end = 0, res_end = 0;
  /* work counts (av1b_plan_stats): samples of phase B blocks, of phase A
   * inter blocks (and of their reference reads, two for a compound block),
   * of transforms, and the coefficient raster samples the transforms read */
  size_t unit_samples = 0, inter_samples = 0, inter_ref_samples = 0, tx_samples = 0,
         coef_samples = 0;
  uint8_t* is_b = nullptr;        /* the frame's phase B flags, by block */
  /* the owner-cell grids (cells of 1 << cell[p] samples, owner_w x owner_h),
   * filled as the blocks convert */
  int* owner[3] = {nullptr, nullptr, nullptr};
  int owner_w[3] = {0, 0, 0}, owner_h[3] = {0, 0, 0}, cell[3] = {2, 2, 2};
  uint8_t unaligned[3] = {0, 0, 0};  /* a block of the plane off its owner-cell grid */
  PlanErr err;
  void clear() {
    unaligned[0] = unaligned[1] = unaligned[2] = 0;
    txs.clear();
    dq.clear();
    obmc.clear();
    warps.clear();
    palette_colors.clear();
    units.clear();
    inter_tiles.clear();
    inter_tiles_mask.clear();
    inter_tiles_full.clear();
    itx_jobs.clear();
    pre_res_pool = coef_end = res_end = 0;
    unit_samples = inter_samples = inter_ref_samples = tx_samples = coef_samples = 0;
    err = PlanErr();
  }
};

/* The dequantiser of one coded transform of a levels frame, as the reference
 * front end's dequantise_tile reads it (dequant.hpp:317-345): the raster is
 * the adjusted size (each side at most 32), the levels are min(eob, area) in
 * the scan of the transform's class (coef_model.hpp:190-219: vertical 1-D
 * types the row scan, horizontal ones the column scan, falling back to the
 * diagonal scan of the size), and the matrix, when there is one, is read
 * whatever the type. */
int plan_dequant(const PlanCtx& ctx, const av1b_transform& t, const TxRec& x, BlockOut* O) {
  DqRec q{};
  q.alw = static_cast<unsigned char>(std::min<int>(x.log2w, 5));
  q.alh = static_cast<unsigned char>(std::min<int>(x.log2h, 5));
  const int area = 1 << (q.alw + q.alh);
  const int cls = (t.tx_type == 10 || t.tx_type == 12 || t.tx_type == 14)   ? 2
                  : (t.tx_type == 11 || t.tx_type == 13 || t.tx_type == 15) ? 1
                                                                            : 0;
  const int key = (q.alw - 2) * 4 + (q.alh - 2);
  int so = kScanOffset[cls * 16 + key];
  if (so < 0) so = kScanOffset[key];
  if (so < 0) so = 0;
  q.count = std::min(t.eob, area);
  if (t.level_offset < 0 || static_cast<size_t>(t.level_offset) + q.count > ctx.n_levels)
    return O->err.set(AV1B_ERR_SYNTAX, "transform levels outside the frame's level list");
  if (so + q.count > AV1B_SCAN_ENTRIES)
    return O->err.set(AV1B_ERR_SYNTAX, "transform size without a coefficient scan");
  if (t.denominator < 1 || t.denominator > 4 || t.dc_step < 0 || t.dc_step > (1 << 20) ||
      t.ac_step < 0 || t.ac_step > (1 << 20))
    return O->err.set(AV1B_ERR_SYNTAX, "dequantiser step or denominator out of range");
  if (t.qm_off >= 0 && static_cast<size_t>(t.qm_off) + area > ctx.n_qm)
    return O->err.set(AV1B_ERR_SYNTAX, "quantiser matrix outside the frame's pool");
  q.coef_off = t.coef_offset;
  q.level_off = t.level_offset;
  q.dc_step = t.dc_step;
  q.ac_step = t.ac_step;
  q.qm_off = t.qm_off >= 0 ? t.qm_off : -1;
  q.scan_off = static_cast<unsigned short>(so);
  q.denom = static_cast<unsigned short>(t.denominator);
  O->dq.push_back(q);
  return AV1B_OK;
}

int plan_block(const PlanCtx& ctx, const av1b_frame_syntax& s, size_t bi, BlockRec& r, BlockOut* O) {
  const Layout& L = ctx.L;
  const av1b_block& b = s.blocks[bi];
  std::memset(&r, 0, sizeof(r));
  if (b.plane < 0 || b.plane > 2) return O->err.set(AV1B_ERR_SYNTAX, "block plane out of range");
  const PlaneGeom& g = L.p[b.plane];
  const int rows = plane_rows(L, b.plane);
  if (b.x < 0 || b.y < 0 || b.w < 1 || b.h < 1 || b.w > 128 || b.h > 128 ||
      b.x + b.w > g.stride || b.y + b.h > rows)
    return O->err.set(AV1B_ERR_SYNTAX, "block outside the picture and its border");
  r.x = static_cast<short>(b.x);
  r.y = static_cast<short>(b.y);
  r.w = static_cast<short>(b.w);
  r.h = static_cast<short>(b.h);
  r.plane = static_cast<unsigned char>(b.plane);
  r.have_left = b.have_left && b.x > 0;
  r.have_above = b.have_above && b.y > 0;
  r.lossless = b.lossless ? 1 : 0;
  r.residual_provided = b.residual_provided ? 1 : 0;
  r.warp_idx[0] = r.warp_idx[1] = 0;
  r.ref_slot[0] = r.ref_slot[1] = -1;
  if (b.is_intra) {
    if (!pow2_in(b.w, 2, 64) || !pow2_in(b.h, 2, 64))
      return O->err.set(AV1B_ERR_SYNTAX, "an intra block must be 2..64 samples per side");
    if (b.mode < 0 || b.mode > 13) return O->err.set(AV1B_ERR_SYNTAX, "intra mode out of range");
    if (b.angle_delta < -3 || b.angle_delta > 3)
      return O->err.set(AV1B_ERR_SYNTAX, "angle delta out of range");
    r.kind = AV1B_U_INTRA;
    r.is_inter = 0;
    r.phase_b = 1;
    r.mode = static_cast<unsigned char>(b.mode);
    r.angle_delta = static_cast<signed char>(b.angle_delta);
    /* negative: no edge filtering at all; any other non-zero value selects
     * the second strength table (av1gpu_kernels.h:1195-1239, 1459) */
    r.filter_type = static_cast<signed char>(
        !s.enable_intra_edge_filter || b.filter_type < 0 ? -1 : (b.filter_type ? 1 : 0));
    const bool fi = b.use_filter_intra && b.plane == 0;
    if (fi && (b.filter_intra_mode < 0 || b.filter_intra_mode > 4))
      return O->err.set(AV1B_ERR_SYNTAX, "filter intra mode out of range");
    if (fi && (b.w > 32 || b.h > 32))
      return O->err.set(AV1B_ERR_SYNTAX, "filter intra on a block larger than 32x32");
    r.fi_mode = static_cast<signed char>(fi ? b.filter_intra_mode : -1);
    r.cfl_alpha = static_cast<signed char>(std::max(-128, std::min(127, b.cfl_alpha)));
    r.have_ar = b.have_above_right >= 0 ? (b.have_above_right != 0) : 2;
    r.have_bl = b.have_below_left >= 0 ? (b.have_below_left != 0) : 2;
    if (b.use_palette) {
      if (b.palette_off < 0 || b.palette_stride < b.w ||
          static_cast<size_t>(b.palette_off) + static_cast<size_t>(b.h - 1) * b.palette_stride + b.w >
              s.n_palette_map)
        return O->err.set(AV1B_ERR_SYNTAX, "palette map outside the frame's pool");
      for (int i = 0; i < b.h; ++i)
        for (int j = 0; j < b.w; ++j)
          if (s.palette_map[b.palette_off + i * b.palette_stride + j] > 7)
            return O->err.set(AV1B_ERR_SYNTAX, "palette index above 7");
      r.palette = 1;
      r.palette_off = b.palette_off;
      r.palette_stride = b.palette_stride;
      r.palette_color_idx = static_cast<int>(O->palette_colors.size() / 8);
      for (int k = 0; k < 8; ++k) O->palette_colors.push_back(b.palette[k]);
    }
  } else {
    r.kind = b.intrabc ? AV1B_U_INTRABC : (b.interintra ? AV1B_U_INTERINTRA : 0);
    r.is_inter = 1;
    r.phase_b = (b.intrabc || b.interintra) ? 1 : 0;
    if (b.filter < 0 || b.filter > 3 || b.filter_v < 0 || b.filter_v > 3)
      return O->err.set(AV1B_ERR_SYNTAX, "interpolation filter out of range");
    if (b.compound < 0 || b.compound > 4) return O->err.set(AV1B_ERR_SYNTAX, "compound type out of range");
    int rc;
    if (b.intrabc) {
      r.ref_slot[0] = r.ref_slot[1] = -1;
    } else {
      if ((rc = resolve_slot(ctx, O->err, s, b.ref[0], &r.ref_slot[0]))) return rc;
      if (r.ref_slot[0] < 0) return O->err.set(AV1B_ERR_SYNTAX, "an inter block without a reference");
      if (b.compound) {
        if ((rc = resolve_slot(ctx, O->err, s, b.ref[1], &r.ref_slot[1]))) return rc;
        if (r.ref_slot[1] < 0)
          return O->err.set(AV1B_ERR_SYNTAX, "a compound block without a second reference");
      }
    }
    for (int k = 0; k < 2; ++k) {
      r.mv[k][0] = b.mv[k][0];
      r.mv[k][1] = b.mv[k][1];
    }
    r.filt = static_cast<unsigned char>(b.filter);
    r.filt_v = static_cast<unsigned char>(b.filter_v);
    r.compound = static_cast<unsigned char>(b.compound);
    r.w0 = static_cast<unsigned char>(b.blend[0]);
    r.w1 = static_cast<unsigned char>(b.blend[1]);
    const int lw = b.w << (b.plane > 0 ? s.ss_x : 0), lh = b.h << (b.plane > 0 ? s.ss_y : 0);
    if (b.compound == 3 || b.compound == 4) {
      r.mask_kind = b.compound == 3 ? 1 : 2;
      r.mask_sign = b.mask_sign ? 1 : 0;
      if (b.compound == 3) {
        int dir, xo, yo, fl;
        if (!wedge_entry(lw, lh, b.wedge_index, &dir, &xo, &yo, &fl))
          return O->err.set(AV1B_ERR_SYNTAX, "engine: a wedge on a block size that has none");
        r.wedge_dir = static_cast<unsigned char>(dir);
        r.wedge_xoff = static_cast<signed char>(xo);
        r.wedge_yoff = static_cast<signed char>(yo);
        r.wedge_flip = static_cast<unsigned char>(fl);
      }
    }
    if (b.interintra) {
      if (!pow2_in(b.w, 2, 64) || !pow2_in(b.h, 2, 64) || b.interintra_mode < 0 ||
          b.interintra_mode > 3)
        return O->err.set(AV1B_ERR_SYNTAX, "inter-intra block shape or mode out of range");
      r.interintra = 1;
      r.ii_mode = static_cast<unsigned char>(b.interintra_mode);
      if (b.interintra_wedge) {
        int dir, xo, yo, fl;
        if (!wedge_entry(lw, lh, b.wedge_index, &dir, &xo, &yo, &fl))
          return O->err.set(AV1B_ERR_SYNTAX, "engine: an inter/intra wedge on a block size that has none");
        r.ii_wedge = 1;
        r.wedge_dir = static_cast<unsigned char>(dir);
        r.wedge_xoff = static_cast<signed char>(xo);
        r.wedge_yoff = static_cast<signed char>(yo);
        r.wedge_flip = static_cast<unsigned char>(fl);
      }
    }
    /* global warp: a model whose shear is invalid keeps the warp flag with
     * an all-zero model, exactly as the reference engine leaves its job
     * (engine.cpp:1172-1193) */
    for (int k = 0; k < 2; ++k) {
      const bool w = b.warp[k] != 0, mw = b.mask_warp[k] != 0;
      if (k == 0) {
        r.warp0 = w;
        r.mask_warp0 = mw;
      } else {
        r.warp1 = w;
        r.mask_warp1 = mw;
      }
      if (!w && !mw) continue;
      WarpRec m{};
      int al, be, ga, de;
      if (gm_setup_shear(b.warp_params[k], &al, &be, &ga, &de)) {
        for (int j = 0; j < 6; ++j) m.params[j] = b.warp_params[k][j];
        m.abcd[0] = al;
        m.abcd[1] = be;
        m.abcd[2] = ga;
        m.abcd[3] = de;
      }
      r.warp_idx[k] = static_cast<int>(O->warps.size()) + 1;
      O->warps.push_back(m);
    }
    r.obmc_first = static_cast<int>(O->obmc.size());
    r.obmc_count = 0;
    if (b.obmc_count > 0) {
      if (b.obmc_first < 0 || static_cast<size_t>(b.obmc_first) + b.obmc_count > s.n_obmc)
        return O->err.set(AV1B_ERR_SYNTAX, "OBMC range outside the frame's list");
      for (int k = 0; k < b.obmc_count && k < 8; ++k) {
        const av1b_obmc& c = s.obmc[b.obmc_first + k];
        ObmcRec o{};
        o.pass = static_cast<short>(c.pass);
        o.x = static_cast<short>(c.x);
        o.y = static_cast<short>(c.y);
        o.w = static_cast<short>(c.w);
        o.h = static_cast<short>(c.h);
        const int len = c.pass == 0 ? c.h : c.w;
        if (c.w < 1 || c.h < 1 || c.x < 0 || c.y < 0 || !(len == 2 || len == 4 || len == 8 ||
                                                          len == 16 || len == 32))
          return O->err.set(AV1B_ERR_SYNTAX, "OBMC strip shape out of range");
        if (c.filter < 0 || c.filter > 3 || c.filter_v < 0 || c.filter_v > 3)
          return O->err.set(AV1B_ERR_SYNTAX, "OBMC filter out of range");
        o.filt = static_cast<short>(c.filter);
        o.filt_v = static_cast<short>(c.filter_v);
        o.mv_x = c.mv[0];
        o.mv_y = c.mv[1];
        if ((rc = resolve_slot(ctx, O->err, s, c.ref, &o.ref_slot))) return rc;
        if (o.ref_slot < 0) return O->err.set(AV1B_ERR_SYNTAX, "an OBMC strip without a reference");
        O->obmc.push_back(o);
        ++r.obmc_count;
      }
    }
  }
  /* transforms */
  r.tx_first = static_cast<int>(O->txs.size());
  r.tx_count = 0;
  if (b.tx_count > 0) {
    if (b.tx_first < 0 || static_cast<size_t>(b.tx_first) + b.tx_count > s.n_transforms)
      return O->err.set(AV1B_ERR_SYNTAX, "transform range outside the frame's list");
    for (int k = 0; k < b.tx_count; ++k) {
      const av1b_transform& t = s.transforms[b.tx_first + k];
      if (t.eob <= 0) continue;
      if (t.coef_offset < 0 || t.x < 0 || t.y < 0 || b.x + t.x + t.w > g.stride ||
          b.y + t.y + t.h > rows)
        return O->err.set(AV1B_ERR_SYNTAX, "transform outside the picture and its border");
      TxRec x{};
      x.coef_off = t.coef_offset;
      x.x = static_cast<short>(t.x);
      x.y = static_cast<short>(t.y);
      x.w = static_cast<short>(t.w);
      x.h = static_cast<short>(t.h);
      if (b.residual_provided) {
        if (t.w < 1 || t.h < 1 || t.w > 128 || t.h > 128)
          return O->err.set(AV1B_ERR_SYNTAX, "residual block size out of range");
        O->res_end = std::max(O->res_end, static_cast<size_t>(t.coef_offset) + static_cast<size_t>(t.w) * t.h);
      } else {
        if (!pow2_in(t.w, 4, 64) || !pow2_in(t.h, 4, 64) || t.tx_type < 0 || t.tx_type > 15)
          return O->err.set(AV1B_ERR_SYNTAX, "transform size or type out of range");
        if (b.lossless && (t.w != 4 || t.h != 4))
          return O->err.set(AV1B_ERR_SYNTAX, "a lossless transform must be 4x4");
        x.log2w = static_cast<unsigned char>(__builtin_ctz(t.w));
        x.log2h = static_cast<unsigned char>(__builtin_ctz(t.h));
        x.type = static_cast<unsigned char>(t.tx_type);
        x.row_shift = static_cast<unsigned char>(b.lossless ? 0 : tx_row_shift(x.log2w, x.log2h));
        O->coef_end = std::max(O->coef_end, static_cast<size_t>(t.coef_offset) + static_cast<size_t>(t.w) * t.h);
        if (ctx.levels) {
          int rc;
          if ((rc = plan_dequant(ctx, t, x, O))) return rc;
        }
      }
      x.pre_off = -1;
      if (r.phase_b && !b.residual_provided) {
        x.pre_off = static_cast<int>(O->pre_res_pool);
        O->pre_res_pool += static_cast<size_t>(t.w) * t.h;
      }
      if (!r.phase_b || x.pre_off >= 0)
        O->itx_jobs.push_back(make_int2(static_cast<int>(bi), static_cast<int>(O->txs.size())));
      O->txs.push_back(x);
      ++r.tx_count;
      O->tx_samples += static_cast<size_t>(t.w) * t.h;
      O->coef_samples += b.residual_provided ? static_cast<size_t>(t.w) * t.h
                                             : static_cast<size_t>(std::min(t.w, 32)) * std::min(t.h, 32);
    }
  }
  if (r.phase_b) {
    O->units.push_back(static_cast<int>(bi));
    O->unit_samples += static_cast<size_t>(b.w) * b.h;
  } else {
    O->inter_samples += static_cast<size_t>(b.w) * b.h;
    O->inter_ref_samples += static_cast<size_t>(b.w) * b.h * (r.compound ? 2 : 1);
    /* the lean prediction kernel takes every block but inter-intra ones
     * and the chroma of difference-weighted compounds, whose masks come from
     * luma predictions (those of them that read the luma block's mask return
     * to the lean kernel, last): unmasked blocks (translation or global warp,
     * OBMC, average or distance compound) in one build, wedge and luma
     * difference-weighted compounds in the masked one */
    const bool full = r.interintra || (r.mask_kind == 2 && r.plane > 0);
    auto& tiles = full ? O->inter_tiles_full : (r.mask_kind ? O->inter_tiles_mask : O->inter_tiles);
    for (int y0 = 0; y0 < b.h; y0 += 8)
      for (int x0 = 0; x0 < b.w; x0 += 16)
        tiles.push_back(make_int2(static_cast<int>(bi), x0 | (y0 << 16)));
  }
  /* for the dependency schedule: owner cells are 4 samples, 2 in a chroma
   * plane whose axis is subsampled (plane 1 keyed on ss_x, plane 2 on ss_y) */
  const int p = b.plane, cs = O->cell[p], oc = 1 << cs;
  if ((b.x | b.y | b.w | b.h) & (oc - 1)) O->unaligned[p] = 1;
  O->is_b[bi] = r.phase_b;
  /* the block's owner cells. A plane whose blocks are not all on the cell
   * grid is filled again, serially and in coding order, once every block is
   * converted; this piece stops filling it as soon as it meets such a block.
   * Blocks of other pieces may still write cells such a block shares at the
   * same moment (the only cells two threads write at once: blocks of valid
   * syntax on the grid do not overlap), and the serial pass overwrites all of
   * them before anything reads the grid. */
  if (O->unaligned[p]) return AV1B_OK;
  const int cx0 = b.x >> cs, cy0 = b.y >> cs;
  const int cx1 = std::min((b.x + b.w + oc - 1) >> cs, O->owner_w[p]);
  const int cy1 = std::min((b.y + b.h + oc - 1) >> cs, O->owner_h[p]);
  int* o = O->owner[p];
  if (cx0 < cx1)  /* a block right of the grid (in the border) owns no cell */
    for (int y = cy0; y < cy1; ++y)
      std::fill(o + static_cast<size_t>(y) * O->owner_w[p] + cx0, o + static_cast<size_t>(y) * O->owner_w[p] + cx1,
              static_cast<int>(bi));
  return AV1B_OK;
}


/* The planner's per-piece outputs, kept between frames for their capacity. */
struct PlanScratch {
  std::vector<BlockOut> blocks;
  std::vector<int> owner[3];
  std::vector<std::vector<int>> unit_deps;
  std::vector<int> dep_count, dep_first;
  std::vector<int> chain_id, chain_len, height, crit, best;
  std::vector<uint64_t> head_key;
  std::vector<int> units_coding, ui_of, udepth, udeps;
  std::vector<uint8_t> is_b;
  std::vector<uint16_t> itx_key;
  std::vector<int> itx_hist;
  std::vector<int2> itx_unsorted;  /* the blocks' transform jobs, before plan_itx sorts them */
};

/* Splits [0, n) into pieces of at least `min_piece` for the pool. */
int pieces_for(size_t n, const PlanCtx& c, size_t min_piece) {
  if (n == 0) return 0;
  const size_t most = static_cast<size_t>(c.pool ? 4 * c.pool->threads() : 1);
  return static_cast<int>(std::max<size_t>(1, std::min(most, n / min_piece)));
}
inline size_t piece_begin(size_t n, int pieces, int i) { return n * i / pieces; }

/* The dependency-scheduled (phase B) blocks: what each waits for, and the
 * order the device claims them in.
 *
 * A block waits for the blocks that own the samples it reads from this
 * picture - its left column and above row (extended below-left / above-right
 * when a directional mode reads there and that part was decoded before it),
 * the corner, an intra block copy's source, CFL's co-located luma - as the
 * reference's owner grids (square cells of 4 luma samples, 2 for a chroma
 * plane whose axis is subsampled; plane 1 keyed on ss_x and plane 2 on ss_y,
 * engine.cpp:737-741) and already_decoded (engine.cpp:784-793) define them.
 * Blocks of the parallel phase are complete before any of these run, so only
 * phase B owners are kept: a short deduplicated list per block, resolved here
 * once instead of by owner lookups on the device's critical path. The
 * above-right / below-left availability the reference derives the same way is
 * resolved here too.
 *
 * The claim order is by dependency depth (1 + the deepest block waited for),
 * coding order within a depth. Every block a block waits for is shallower, so
 * it is claimed earlier - by a warp that is running it or will - and every
 * depth runs as one wide wave. */
int plan_units(av1b_decoder* d, const PlanCtx& c, Plan* P) {
  const Layout& L = c.L;
  P->R->deps.clear();
  P->n_chains = 0;
  P->depth_first.clear();
  P->R->chains.clear();
  if (P->R->units.empty()) return AV1B_OK;
  PlanScratch& S = *c.scratch;
  int sh[3], cw[3], ch[3];
  for (int p = 0; p < 3; ++p) {
    sh[p] = p == 0 ? 2 : (p == 1 ? (L.ss_x ? 1 : 2) : (L.ss_y ? 1 : 2));
    cw[p] = (L.p[p].grid_w + (1 << sh[p]) - 1) >> sh[p];
    ch[p] = (L.p[p].grid_h + (1 << sh[p]) - 1) >> sh[p];
  }
  /* the owner grids were filled as the blocks converted (build_plan) */
  const size_t nb = P->R->blocks.size();
  const std::vector<uint8_t>& is_b = S.is_b;
  /* the cells of [x0, x1] x [y0, y1] inside the plane's grid, row by row
   * from the cell holding (x0, y0) (the device's wait_rect / decoded_before
   * walk): `f(owner)` for each cell whose owner differs from the one of the
   * cell before it. Every caller ignores -1 (no owner: outside the grid, or
   * no block) and a repeat of the owner it was just given, so neither
   * changes what it collects. */
  auto each_cell = [&](int p, int x0, int x1, int y0, int y1, auto&& f) {
    const int s = sh[p], w = cw[p];
    const int cx0 = std::max(x0 >> s, 0), cx1 = std::min(x1 >> s, w - 1);
    const int cy0 = std::max(y0 >> s, 0), cy1 = std::min(y1 >> s, ch[p] - 1);
    const int* o = S.owner[p].data();
    int last = -1;
    for (int cy = cy0; cy <= cy1; ++cy) {
      const int* row = o + static_cast<size_t>(cy) * w;
      for (int cx = cx0; cx <= cx1; ++cx)
        if (row[cx] != last) {
          last = row[cx];
          f(last);
        }
    }
  };
  static const int kAngle[9] = {0, 90, 180, 45, 135, 113, 157, 203, 67};
  const size_t nu = P->R->units.size();
  const int pieces = pieces_for(nu, c, 256);
  std::vector<std::vector<int>>& pdeps = S.unit_deps;
  if (pdeps.size() < static_cast<size_t>(pieces)) pdeps.resize(pieces);
  std::vector<int>& dep_count = S.dep_count;
  dep_count.assign(nu, 0);
  std::vector<int>& ui_of = S.ui_of;  /* a phase B block's unit index */
  ui_of.resize(nb);
  std::vector<uint8_t> inter_piece(pieces, 0);
  c.pool->run(pieces, [&](int pi) {
    std::vector<int>& out = pdeps[pi];
    out.clear();
    std::vector<int> mine;
    for (size_t ui = piece_begin(nu, pieces, pi); ui < piece_begin(nu, pieces, pi + 1); ++ui) {
      const int bi = P->R->units[ui];
      BlockRec& b = P->R->blocks[bi];
      ui_of[bi] = static_cast<int>(ui);
      if (b.kind != AV1B_U_INTRA) inter_piece[pi] = 1;
      const int p = b.plane, oc = 1 << sh[p];
      mine.clear();
      /* neighbouring cells mostly share an owner: skip the repeat at once */
      auto wait_on = [&](int o) {
        if (o >= 0 && o < bi && is_b[o] && (mine.empty() || mine.back() != o)) mine.push_back(o);
      };
      int har = b.have_ar, hbl = b.have_bl;
      if (b.kind == AV1B_U_INTRA) {
        if (har == 2) {
          bool ok = true;
          each_cell(p, b.x + b.w, b.x + 2 * b.w - 1, b.y - 1, b.y - 1,
                    [&](int o) { if (o >= 0 && o >= bi) ok = false; });
          har = b.y > 0 && ok;
        }
        if (hbl == 2) {
          bool ok = true;
          each_cell(p, b.x - 1, b.x - 1, b.y + b.h, b.y + 2 * b.h - 1,
                    [&](int o) { if (o >= 0 && o >= bi) ok = false; });
          hbl = b.x > 0 && ok;
        }
      } else {
        har = hbl = 0;
      }
      b.have_ar = static_cast<unsigned char>(har);
      b.have_bl = static_cast<unsigned char>(hbl);
      if (b.kind == AV1B_U_INTRA || b.interintra) {
        int left_y1 = b.y + b.h - 1, above_x1 = b.x + b.w - 1;
        if (b.kind == AV1B_U_INTRA && !b.palette) {
          if (b.mode >= 1 && b.mode <= 8) {
            const int pangle = kAngle[b.mode] + 3 * b.angle_delta;
            if (pangle < 90 && har) above_x1 = b.x + 2 * b.w - 1;
            if (pangle > 180 && hbl) left_y1 = b.y + 2 * b.h - 1;
          }
        } else if (b.kind == AV1B_U_INTRA) {
          above_x1 = b.x - 1;
          left_y1 = b.y - 1;
        }
        if (left_y1 >= (b.y & ~(oc - 1))) each_cell(p, b.x - 1, b.x - 1, b.y, left_y1, wait_on);
        if (above_x1 >= (b.x & ~(oc - 1))) each_cell(p, b.x, above_x1, b.y - 1, b.y - 1, wait_on);
        if (above_x1 >= b.x || left_y1 >= b.y) each_cell(p, b.x - 1, b.x - 1, b.y - 1, b.y - 1, wait_on);
      }
      if (b.kind == AV1B_U_INTRABC) {
        const int sx_ = p > 0 ? L.ss_x : 0, sy_ = p > 0 ? L.ss_y : 0;
        const int sx = b.x + (b.mv[0][0] >> (3 + sx_));
        const int sy = b.y + (b.mv[0][1] >> (3 + sy_));
        const int x1 = std::min(sx + b.w, L.p[p].grid_w), y1 = std::min(sy + b.h, L.p[p].grid_h);
        if (x1 > std::max(sx, 0) && y1 > std::max(sy, 0))
          each_cell(p, std::max(sx, 0), x1 - 1, std::max(sy, 0), y1 - 1, wait_on);
      }
      if (b.kind == AV1B_U_INTRA && b.mode == 13 && !b.palette)
        each_cell(0, b.x << L.ss_x, (b.x + b.w - 1) << L.ss_x, b.y << L.ss_y,
                  (b.y + b.h - 1) << L.ss_y, wait_on);
      if (mine.size() > 24) {
        std::sort(mine.begin(), mine.end());
      } else {
        for (size_t x = 1; x < mine.size(); ++x)  /* short lists: insertion sort */
          for (size_t y = x; y > 0 && mine[y - 1] > mine[y]; --y) std::swap(mine[y - 1], mine[y]);
      }
      mine.erase(std::unique(mine.begin(), mine.end()), mine.end());
      /* prediction and residual fuse when the transforms cover disjoint parts
       * of the block (each sample then gets at most one residual) */
      b.fuse_res = 0;
      if (b.kind == AV1B_U_INTRA && b.w * b.h <= AV1B_UNIT_SCRATCH && b.tx_count <= 1) {
        /* none or one transform: disjoint by itself once it lies in the block */
        bool ok = true;
        if (b.tx_count == 1) {
          const TxRec& x = P->R->txs[b.tx_first];
          ok = x.x >= 0 && x.y >= 0 && x.x + x.w <= b.w && x.y + x.h <= b.h;
        }
        b.fuse_res = ok ? 1 : 0;
      } else if (b.kind == AV1B_U_INTRA && b.w * b.h <= AV1B_UNIT_SCRATCH) {
        bool ok = true, grid4 = true;
        for (int t = 0; t < b.tx_count && ok; ++t) {
          const TxRec& x = P->R->txs[b.tx_first + t];
          if (x.x < 0 || x.y < 0 || x.x + x.w > b.w || x.y + x.h > b.h) ok = false;
          if ((x.x | x.y | x.w | x.h) & 3) grid4 = false;
        }
        if (ok && grid4) {
          /* 4x4 cells of the block (at most 16 x 16) */
          uint64_t cov[4] = {0, 0, 0, 0};
          for (int t = 0; t < b.tx_count && ok; ++t) {
            const TxRec& x = P->R->txs[b.tx_first + t];
            for (int cy = x.y >> 2; cy < (x.y + x.h) >> 2 && ok; ++cy)
              for (int cx = x.x >> 2; cx < (x.x + x.w) >> 2; ++cx) {
                const int bit = cy * 16 + cx;
                if (cov[bit >> 6] >> (bit & 63) & 1) {
                  ok = false;
                  break;
                }
                cov[bit >> 6] |= 1ull << (bit & 63);
              }
          }
        } else if (ok) {
          for (int t = 0; t < b.tx_count && ok; ++t) {
            const TxRec& x = P->R->txs[b.tx_first + t];
            for (int u = 0; u < t && ok; ++u) {
              const TxRec& y = P->R->txs[b.tx_first + u];
              if (x.x < y.x + y.w && y.x < x.x + x.w && x.y < y.y + y.h && y.y < x.y + x.h) ok = false;
            }
            if (t > 64) ok = false;
          }
        }
        b.fuse_res = ok ? 1 : 0;
      }
      dep_count[ui] = static_cast<int>(mine.size());
      out.insert(out.end(), mine.begin(), mine.end());
    }
  });
  /* the lists back to back for the device (block indices), and as unit
   * indices for the passes below */
  {
    size_t total = 0;
    for (size_t ui = 0; ui < nu; ++ui) total += static_cast<size_t>(dep_count[ui]);
    if (total > static_cast<size_t>(INT32_MAX)) return fail(d, AV1B_ERR_SYNTAX, "frame too large");
  }
  std::vector<int>& first = S.dep_first;  /* where each unit's list starts, and the end */
  first.resize(nu + 1);
  first[0] = 0;
  for (size_t ui = 0; ui < nu; ++ui) first[ui + 1] = first[ui] + dep_count[ui];
  sized(P->R->deps, first[nu]);
  std::vector<int>& udeps = S.udeps;
  udeps.resize(first[nu]);
  c.pool->run(pieces, [&](int pi) {
    const size_t u0 = piece_begin(nu, pieces, pi), u1 = piece_begin(nu, pieces, pi + 1);
    std::copy(pdeps[pi].begin(), pdeps[pi].end(), P->R->deps.begin() + first[u0]);
    for (size_t k = first[u0]; k < first[u1]; ++k) udeps[k] = ui_of[pdeps[pi][k - first[u0]]];
    for (size_t ui = u0; ui < u1; ++ui) {
      BlockRec& b = P->R->blocks[P->R->units[ui]];
      b.dep_first = static_cast<int>(first[ui]);
      b.dep_count = dep_count[ui];
    }
  });
  /* chains: a warp claims a chain and runs its blocks in order, so a block
   * whose deepest dependency is the block before it in its chain waits on
   * its own warp's work instead of a flag published on another SM.
   *
   * A block's depth is 1 + the deepest block it waits for, and that block
   * (the latest in coding order of equally deep ones) is its candidate
   * predecessor. Of the blocks naming the same candidate, the one with the
   * longest path still ahead of it (its height; the first in order of depth,
   * then coding order, of equal ones) gets it, so chains follow the critical
   * path. It joins the candidate's chain - as its next block: no other block
   * can take that place - when every other block it waits for lies in that
   * chain or in one started earlier; otherwise it starts a chain. Chains are
   * ordered by their first block, by depth then coding order, and claimed in
   * that order, so every wait across chains is on a chain claimed before: the
   * warp holding the earliest unfinished chain always progresses. A chain's
   * blocks are in coding order, which is also their order of depth.
   *
   * Every dependency precedes its dependant in coding order, so each pass is
   * one sweep over the units in coding order (or its reverse, for heights). */
  std::vector<int>& U = S.units_coding;
  U.assign(P->R->units.begin(), P->R->units.end());
  std::vector<int>& ud = S.udepth;
  std::vector<int>& critv = S.crit;
  ud.resize(nu);
  critv.resize(nu);
  int max_depth = 0;
  for (size_t u = 0; u < nu; ++u) {
    /* (depth, unit) of the deepest dependency, the latest of equally deep
     * ones, as one 64-bit key: the maximum, without branches */
    uint64_t key = 0;
    for (size_t j = first[u]; j < first[u + 1]; ++j) {
      const int o = udeps[j];
      key = std::max(key, (static_cast<uint64_t>(ud[o]) << 32) | static_cast<uint32_t>(o + 1));
    }
    const int cr = static_cast<int>(static_cast<uint32_t>(key)) - 1;
    critv[u] = cr;
    ud[u] = static_cast<int>(key >> 32) + 1;
    max_depth = std::max(max_depth, ud[u]);
  }
  std::vector<int>& height = S.height;
  std::vector<int>& best = S.best;
  height.assign(nu, 0);
  best.assign(nu, -1);
  for (size_t k = nu; k-- > 0;) {
    const int u = static_cast<int>(k);  /* every block waiting for u is done: its height is final */
    for (size_t j = first[u]; j < first[u + 1]; ++j) {
      const int o = udeps[j];
      height[o] = std::max(height[o], height[u] + 1);
    }
    const int cr = critv[u];
    if (cr >= 0) {
      const int bu = best[cr];  /* later in coding order than u */
      if (bu < 0 || height[u] > height[bu] || (height[u] == height[bu] && ud[u] <= ud[bu])) best[cr] = u;
    }
  }
  /* each block's chain, as the (depth, unit) key of its first block */
  std::vector<uint64_t>& hk = S.head_key;
  hk.resize(nu);
  std::vector<int> count(max_depth + 2, 0);
  for (size_t u = 0; u < nu; ++u) {
    const int cr = critv[u];
    const uint64_t own = (static_cast<uint64_t>(ud[u]) << 32) | static_cast<uint32_t>(u);
    uint64_t h = own;
    if (cr >= 0 && best[cr] == static_cast<int>(u)) {
      const uint64_t hc = hk[cr];
      bool ok = true;
      for (size_t j = first[u]; j < first[u + 1]; ++j) ok &= hk[udeps[j]] <= hc;
      if (ok) h = hc;
    }
    hk[u] = h;
    if (h == own) ++count[ud[u] + 1];
  }
  for (int k = 0; k <= max_depth; ++k) count[k + 1] += count[k];
  const size_t nch = static_cast<size_t>(count[max_depth + 1]);
  P->depth_first.assign(count.begin(), count.end());
  std::vector<int>& cid = S.chain_id;  /* each block's chain, in claim order */
  std::vector<int>& clen = S.chain_len;
  cid.resize(nu);
  clen.assign(nch + 1, 0);
  for (size_t u = 0; u < nu; ++u) {
    const int hu = static_cast<int>(static_cast<uint32_t>(hk[u]));
    cid[u] = hu == static_cast<int>(u) ? count[ud[u]]++ : cid[hu];
    ++clen[cid[u] + 1];
  }
  sized(P->R->chains, nch + 1);
  for (size_t k = 0; k < nch; ++k) clen[k + 1] += clen[k];
  for (size_t k = 0; k <= nch; ++k) P->R->chains[k] = clen[k];
  for (size_t u = 0; u < nu; ++u) P->R->units[clen[cid[u]]++] = U[u];
  P->n_chains = nch;
  P->unit_depth = max_depth;
  P->units_inter = false;
  for (int pi = 0; pi < pieces; ++pi)
    if (inter_piece[pi]) P->units_inter = true;
  return AV1B_OK;
}

/* Orders the inverse transforms for the batched kernel: by size class (the
 * longer side, 4 .. 64; raw residual blocks last), then shape and type, so
 * the lane groups of a warp mostly run the same code; then cuts each class
 * into batches of 32 / class transforms (one for 64 and raw). */
void plan_itx(const PlanCtx& c, Plan* P) {
  PlanLists& R = *P->R;
  PlanScratch& S = *c.scratch;
  const std::vector<int2>& jobs = S.itx_unsorted;
  const size_t n = jobs.size();
  R.itx_batches.clear();
  for (int k = 0; k < 8; ++k) P->itx_class_first[k] = P->itx_class_count[k] = 0;
  if (n == 0) return;
  /* keys: the 25 shapes (log2 sides 2..6) ranked by class (the longer side),
   * then width, then height; 16 types each; raw residual blocks last */
  struct ShapeRank {
    unsigned char rank[5][5], cls[25];
    ShapeRank() {
      int r = 0;
      for (int cl = 2; cl <= 6; ++cl)
        for (int lw = 2; lw <= 6; ++lw)
          for (int lh = 2; lh <= 6; ++lh)
            if (std::max(lw, lh) == cl) {
              rank[lw - 2][lh - 2] = static_cast<unsigned char>(r);
              cls[r++] = static_cast<unsigned char>(cl);
            }
    }
  };
  static const ShapeRank shapes;
  constexpr int kRaw = 25 * 16, kKeys = kRaw + 1;
  std::vector<uint16_t>& key = S.itx_key;
  key.resize(n);
  /* a parallel counting sort: keys and per-piece histograms, offsets per
   * (key, piece), then every piece scatters its own jobs into the list that
   * is uploaded */
  const int pieces = pieces_for(n, c, 4096);
  std::vector<int>& hist = S.itx_hist;
  hist.assign(static_cast<size_t>(kKeys) * pieces, 0);
  c.pool->run(pieces, [&](int pi) {
    int* h = hist.data() + static_cast<size_t>(pi) * kKeys;
    for (size_t i = piece_begin(n, pieces, pi); i < piece_begin(n, pieces, pi + 1); ++i) {
      const int2 j = jobs[i];
      const TxRec& t = R.txs[j.y];
      int k = kRaw;
      if (!R.blocks[j.x].residual_provided) k = shapes.rank[t.log2w - 2][t.log2h - 2] * 16 + t.type;
      key[i] = static_cast<uint16_t>(k);
      ++h[k];
    }
  });
  /* offsets; and each class's range of the sorted list (its keys are
   * contiguous: ranks ascend with the class) */
  int run = 0;
  int cls_begin[8], cls_end[8];
  for (int k = 0; k < 8; ++k) cls_begin[k] = cls_end[k] = -1;
  for (int k = 0; k < kKeys; ++k) {
    const int cl = k == kRaw ? 7 : shapes.cls[k >> 4];
    if (cls_begin[cl] < 0) cls_begin[cl] = run;
    for (int pi = 0; pi < pieces; ++pi) {
      int& h = hist[static_cast<size_t>(pi) * kKeys + k];
      const int c0 = h;
      h = run;
      run += c0;
    }
    cls_end[cl] = run;
  }
  c.pool->run(pieces, [&](int pi) {
    int* h = hist.data() + static_cast<size_t>(pi) * kKeys;
    for (size_t i = piece_begin(n, pieces, pi); i < piece_begin(n, pieces, pi + 1); ++i)
      R.itx_jobs[h[key[i]]++] = jobs[i];
  });
  /* batches: runs of 32 / S jobs of one class (one job for the 64-point
   * class and for raw residual blocks), one launch per class */
  int nb = 0;
  for (int cl = 2; cl < 8; ++cl) {
    if (cls_begin[cl] < 0 || cls_end[cl] <= cls_begin[cl]) continue;
    const int per = cl >= 6 ? 1 : 32 >> cl;
    P->itx_class_first[cl] = nb;
    P->itx_class_count[cl] = (cls_end[cl] - cls_begin[cl] + per - 1) / per;
    nb += P->itx_class_count[cl];
  }
  sized(R.itx_batches, nb);
  c.pool->run(6, [&](int k) {
    const int cl = k + 2;
    if (P->itx_class_count[cl] == 0) return;
    const int per = cl >= 6 ? 1 : 32 >> cl;
    int4* out = R.itx_batches.data() + P->itx_class_first[cl];
    for (int b = 0, i = cls_begin[cl]; i < cls_end[cl]; ++b, i += per)
      out[b] = make_int4(i, std::min(per, cls_end[cl] - i), cl, 0);
  });
}

/* Stages the profiler reports (av1b_profile). */
enum Stage {
  kStOwner, kStInter, kStItx, kStUnits, kStDeblockV, kStDeblockH, kStCdef, kStUpscale, kStLr,
  kStGrainTemplate, kStGrainBlend, kStNv12, kStRgb, kStCopy,
  /* host time of plan_frame: records, the wait for the staging buffer, the
   * copy into it; and the parts of the records: blocks, the dependency
   * schedule, the transform batches, the filter lists, film grain */
  kStPlanHost, kStWaitHost, kStStageHost, kStPlanBlocks, kStPlanUnits, kStPlanItx, kStPlanFilters,
  kStPlanGrain, kStageCount
};
static_assert(kStageCount <= 24, "profile table");
const char* const kStageNames[kStageCount] = {
    "owner", "inter", "itx", "units", "deblock_v", "deblock_h", "cdef", "upscale", "lr",
    "grain_template", "grain_blend", "nv12", "rgb", "copy", "plan_host", "wait_host", "stage_host",
    "blocks_host", "units_host", "itx_host", "filters_host", "grain_host"};

/* Host time since `t0` into a host stage, when profiling. */
void host_mark(av1b_decoder* d, int stage, std::chrono::steady_clock::time_point t0) {
  if (!d->profiling) return;
  std::lock_guard<std::mutex> lk(d->prof_mu);
  d->prof_ms[stage] +=
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  d->prof_n[stage] += 1;
}

/* The first invalid deblocking edge or CDEF block of a frame, in list order
 * (edges first): the device conversion only reports that there is one. The
 * lists are checked in pieces on the pool; the earliest piece's first invalid
 * record is the one a single pass in order meets. */
int filter_records_error(av1b_decoder* d, const PlanCtx& c, const av1b_frame_syntax& s) {
  struct List {
    size_t n;
    std::function<int(size_t)> check;
  };
  const List lists[2] = {
      {s.n_deblock,
       [&](size_t i) {
         DeblockRec r;
         int vertical;
         return prep_edge(c.L, s.deblock[i], &r, &vertical);
       }},
      {s.n_cdef, [&](size_t i) {
         CdefRec r;
         int off_grid;
         return prep_cdef(c.L, s.cdef[i], c.L.p[0].stride >> 3, &r, &off_grid);
       }}};
  for (const List& l : lists) {
    const int pieces = pieces_for(l.n, c, 4096);
    std::vector<int> first(pieces, kPrepOk);
    c.pool->run(pieces, [&](int i) {
      for (size_t k = piece_begin(l.n, pieces, i); k < piece_begin(l.n, pieces, i + 1); ++k) {
        const int code = l.check(k);
        if (code >= kPrepErrFirst) {
          first[i] = code;
          break;
        }
      }
    });
    for (int i = 0; i < pieces; ++i)
      if (first[i] >= kPrepErrFirst) return fail(d, AV1B_ERR_SYNTAX, kPrepMessages[first[i]]);
  }
  return AV1B_OK;
}

/* A chroma block of a difference-weighted compound blends with a mask made
 * from the luma predictions of the area it covers. When the luma block there
 * is that very prediction - the same position and size, references, motion,
 * filters, warp models (compared by value) and mask sign - its tiles write
 * the mask (a byte a luma sample, in the frame's mask pool) and the chroma
 * block's tiles read it, instead of predicting the luma again (two
 * references, up to four 16x8 areas each, per chroma tile). Any other chroma
 * block predicts the luma itself. The chroma tiles that read a mask go last
 * in the tile list: they run after every luma tile (a launch, or a stage, of
 * their own). */
void plan_shared_masks(const PlanCtx& c, Plan* P) {
  const Layout& L = c.L;
  PlanLists& R = *P->R;
  PlanScratch& S = *c.scratch;
  P->mask_pool = 0;
  P->n_tiles_cmask = 0;
  if (!c.share_masks) return;
  const size_t nt = R.inter_tiles.size();
  const size_t full0 = P->n_tiles_simple + P->n_tiles_lmask;
  if (nt == full0) return;
  const int ow = static_cast<int>((L.p[0].grid_w + 3) >> 2);
  const int oh = static_cast<int>((L.p[0].grid_h + 3) >> 2);
  if (S.owner[0].size() < static_cast<size_t>(ow) * oh) return;
  size_t pool = 0;
  bool any = false;
  for (size_t i = full0; i < nt; ++i) {
    const int bi = R.inter_tiles[i].x;
    BlockRec& b = R.blocks[bi];
    if (b.plane == 0 || b.mask_role || b.mask_kind != 2 || !b.compound || b.interintra) continue;
    const int lx = b.x << L.ss_x, ly = b.y << L.ss_y;
    if ((lx | ly) & 3 || (lx >> 2) >= ow || (ly >> 2) >= oh) continue;
    const int li = S.owner[0][static_cast<size_t>(ly >> 2) * ow + (lx >> 2)];
    if (li < 0) continue;
    BlockRec& l = R.blocks[li];
    bool same = l.plane == 0 && l.is_inter && !l.phase_b && l.x == lx && l.y == ly &&
                l.w == (b.w << L.ss_x) && l.h == (b.h << L.ss_y) && l.compound && l.mask_kind == 2 &&
                l.mask_sign == b.mask_sign && l.filt == b.filt && l.filt_v == b.filt_v;
    for (int r = 0; r < 2 && same; ++r) {
      const int lw = r ? l.warp1 : l.warp0, cw = r ? b.mask_warp1 : b.mask_warp0;
      same = l.ref_slot[r] == b.ref_slot[r] && l.mv[r][0] == b.mv[r][0] && l.mv[r][1] == b.mv[r][1] &&
             lw == cw;
      /* warped: the same model (each block has an entry of its own) */
      if (same && lw) {
        const int li_w = l.warp_idx[r] >= 0 ? l.warp_idx[r] : 0, bi_w = b.warp_idx[r] >= 0 ? b.warp_idx[r] : 0;
        same = li_w < static_cast<int>(R.warps.size()) && bi_w < static_cast<int>(R.warps.size()) &&
               std::memcmp(&R.warps[li_w], &R.warps[bi_w], sizeof(WarpRec)) == 0;
      }
    }
    if (!same) continue;
    if (l.mask_role != 1) {
      if (pool + static_cast<size_t>(l.w) * l.h > static_cast<size_t>(INT32_MAX)) continue;
      l.mask_role = 1;
      l.mask_off = static_cast<int>(pool);
      l.mask_w = l.w;
      pool += static_cast<size_t>(l.w) * l.h;
    }
    b.mask_role = 2;
    b.mask_off = l.mask_off;
    b.mask_w = l.w;
    any = true;
  }
  if (!any) return;
  P->mask_pool = pool;
  /* the tiles reading a mask to the end, the others in their order */
  auto first = R.inter_tiles.begin() + static_cast<std::ptrdiff_t>(full0);
  auto mid = std::stable_partition(first, R.inter_tiles.end(),
                                   [&](const int2& t) { return R.blocks[t.x].mask_role != 2; });
  P->n_tiles_cmask = static_cast<size_t>(R.inter_tiles.end() - mid);
}

/* Validates a frame and builds its device records. The blocks, deblocking
 * edges and CDEF blocks are converted in pieces on the pool; each piece stops
 * at its first invalid record and the error of the earliest piece is the one
 * reported, so the result - records and error alike - is the one a single
 * pass in order gives. */
int build_plan(av1b_decoder* d, const PlanCtx& c, const av1b_frame_syntax& s, Plan* P) {
  const Layout& L = c.L;
  const int bd = s.bit_depth;
  int rc_units;
  auto tp = std::chrono::steady_clock::now();
  auto phase = [&](int stage) {
    host_mark(d, stage, tp);
    tp = std::chrono::steady_clock::now();
  };
  sized(P->R->blocks, s.n_blocks);
  for (int i = 0; i < 7; ++i) {
    const int rw = s.reference_width[i] > 0 ? s.reference_width[i] : s.width;
    const int rh = s.reference_height[i] > 0 ? s.reference_height[i] : s.height;
    if (rw != s.width || rh != s.height)
      return fail(d, AV1B_ERR_UNSUPPORTED,
                  "engine: reference scaling between pictures of different sizes is not supported");
  }
  P->upscaled = L.p[0].coded_w != L.p[0].out_w;
  P->scale_x = P->scale_y = AV1B_SCALE_ONE;
  if (P->upscaled) {
    const int fw = L.p[0].coded_w, fh = L.p[0].coded_h;
    P->scale_x = ((s.width << 14) + (fw / 2)) / fw;
    P->scale_y = ((s.height << 14) + (fh / 2)) / fh;
  }
  size_t coef_end = 0, res_end = 0;
  {
    const size_t nb = s.n_blocks;
    const int pieces = pieces_for(nb, c, 512);
    std::vector<BlockOut>& outs = c.scratch->blocks;
    if (outs.size() < static_cast<size_t>(pieces)) outs.resize(pieces);
    /* the dependency schedule's owner-cell grids (plan_units): square cells
     * of 4 luma samples, 2 in a chroma plane whose axis is subsampled (plane
     * 1 keyed on ss_x, plane 2 on ss_y: engine.cpp:737-741), cleared here and
     * filled as the blocks convert */
    PlanScratch& S = *c.scratch;
    int cell[3], ow[3], oh[3];
    for (int p = 0; p < 3; ++p) {
      cell[p] = p == 0 ? 2 : ((p == 1 ? L.ss_x : L.ss_y) ? 1 : 2);
      ow[p] = (L.p[p].grid_w + (1 << cell[p]) - 1) >> cell[p];
      oh[p] = (L.p[p].grid_h + (1 << cell[p]) - 1) >> cell[p];
      S.owner[p].resize(static_cast<size_t>(ow[p]) * oh[p]);
    }
    c.pool->run(3 * 8, [&](int i) {
      std::vector<int>& o = S.owner[i / 8];
      std::fill(o.begin() + piece_begin(o.size(), 8, i % 8), o.begin() + piece_begin(o.size(), 8, i % 8 + 1), -1);
    });
    S.is_b.resize(nb);
    c.pool->run(pieces, [&](int i) {
      BlockOut* O = &outs[i];
      O->clear();
      O->is_b = S.is_b.data();
      for (int p = 0; p < 3; ++p) {
        O->owner[p] = S.owner[p].data();
        O->owner_w[p] = ow[p];
        O->owner_h[p] = oh[p];
        O->cell[p] = cell[p];
      }
      for (size_t bi = piece_begin(nb, pieces, i); bi < piece_begin(nb, pieces, i + 1); ++bi)
        if (plan_block(c, s, bi, P->R->blocks[bi], O)) break;
    });
    for (int i = 0; i < pieces; ++i)
      if (outs[i].err.code) return fail(d, outs[i].err.code, outs[i].err.msg);
    /* later blocks overwrite earlier ones where cells overlap: a plane whose
     * blocks are not all on the cell grid is filled again, in coding order */
    for (int p = 0; p < 3; ++p) {
      bool aligned = true;
      for (int i = 0; i < pieces; ++i)
        if (outs[i].unaligned[p]) aligned = false;
      if (aligned) continue;
      std::fill(S.owner[p].begin(), S.owner[p].end(), -1);
      const int oc = 1 << cell[p];
      int* o = S.owner[p].data();
      for (size_t bi = 0; bi < nb; ++bi) {
        const BlockRec& b = P->R->blocks[bi];
        if (b.plane != p) continue;
        const int cx0 = b.x >> cell[p], cy0 = b.y >> cell[p];
        const int cx1 = std::min((b.x + b.w + oc - 1) >> cell[p], ow[p]);
        const int cy1 = std::min((b.y + b.h + oc - 1) >> cell[p], oh[p]);
        if (cx0 < cx1)
          for (int y = cy0; y < cy1; ++y)
            std::fill(o + static_cast<size_t>(y) * ow[p] + cx0, o + static_cast<size_t>(y) * ow[p] + cx1,
                      static_cast<int>(bi));
      }
    }
    /* piece offsets into the frame's lists */
    std::vector<size_t> o_tx(pieces + 1, 0), o_obmc(pieces + 1, 0), o_warp(pieces + 1, 0),
        o_pal(pieces + 1, 0), o_unit(pieces + 1, 0), o_tile(pieces + 1, 0), o_tilem(pieces + 1, 0),
        o_tilef(pieces + 1, 0),
        o_itx(pieces + 1, 0), o_pre(pieces + 1, 0), o_dq(pieces + 1, 0);
    for (int i = 0; i < pieces; ++i) {
      const BlockOut& O = outs[i];
      o_tx[i + 1] = o_tx[i] + O.txs.size();
      o_obmc[i + 1] = o_obmc[i] + O.obmc.size();
      o_warp[i + 1] = o_warp[i] + O.warps.size();
      o_pal[i + 1] = o_pal[i] + O.palette_colors.size();
      o_unit[i + 1] = o_unit[i] + O.units.size();
      o_tile[i + 1] = o_tile[i] + O.inter_tiles.size();
      o_tilem[i + 1] = o_tilem[i] + O.inter_tiles_mask.size();
      o_tilef[i + 1] = o_tilef[i] + O.inter_tiles_full.size();
      o_itx[i + 1] = o_itx[i] + O.itx_jobs.size();
      o_pre[i + 1] = o_pre[i] + O.pre_res_pool;
      o_dq[i + 1] = o_dq[i] + O.dq.size();
      coef_end = std::max(coef_end, O.coef_end);
      res_end = std::max(res_end, O.res_end);
    }
    P->unit_samples = P->inter_samples = P->inter_ref_samples = P->tx_samples = P->coef_samples = 0;
    for (int i = 0; i < pieces; ++i) {
      P->unit_samples += outs[i].unit_samples;
      P->inter_samples += outs[i].inter_samples;
      P->inter_ref_samples += outs[i].inter_ref_samples;
      P->tx_samples += outs[i].tx_samples;
      P->coef_samples += outs[i].coef_samples;
    }
    if (o_pre[pieces] > static_cast<size_t>(INT32_MAX) || o_tx[pieces] > static_cast<size_t>(INT32_MAX))
      return fail(d, AV1B_ERR_SYNTAX, "frame too large");
    sized(P->R->txs, o_tx[pieces]);
    sized(P->R->obmc, o_obmc[pieces]);
    sized(P->R->warps, 1 + o_warp[pieces]);
    P->R->warps[0] = WarpRec{};
    sized(P->R->palette_colors, o_pal[pieces]);
    sized(P->R->units, o_unit[pieces]);
    /* the lean kernel's unmasked tiles, its masked ones, then the rest */
    sized(P->R->inter_tiles, o_tile[pieces] + o_tilem[pieces] + o_tilef[pieces]);
    P->n_tiles_simple = o_tile[pieces];
    P->n_tiles_lmask = o_tilem[pieces];
    c.scratch->itx_unsorted.resize(o_itx[pieces]);
    sized(P->R->itx_jobs, o_itx[pieces]);
    sized(P->R->dq, o_dq[pieces]);
    P->n_dq = o_dq[pieces];
    P->pre_res_pool = o_pre[pieces];
    c.pool->run(pieces, [&](int i) {
      const BlockOut& O = outs[i];
      const int dtx = static_cast<int>(o_tx[i]), dob = static_cast<int>(o_obmc[i]);
      const int dwp = static_cast<int>(o_warp[i]), dpal = static_cast<int>(o_pal[i] / 8);
      const int dpre = static_cast<int>(o_pre[i]);
      for (size_t bi = piece_begin(nb, pieces, i); bi < piece_begin(nb, pieces, i + 1); ++bi) {
        BlockRec& r = P->R->blocks[bi];
        r.tx_first += dtx;
        if (r.is_inter) r.obmc_first += dob;
        if (r.palette) r.palette_color_idx += dpal;
        for (int k = 0; k < 2; ++k)
          if (r.warp_idx[k] > 0) r.warp_idx[k] += dwp;
      }
      for (size_t k = 0; k < O.txs.size(); ++k) {
        TxRec x = O.txs[k];
        if (x.pre_off >= 0) x.pre_off += dpre;
        P->R->txs[o_tx[i] + k] = x;
      }
      std::copy(O.obmc.begin(), O.obmc.end(), P->R->obmc.begin() + o_obmc[i]);
      std::copy(O.warps.begin(), O.warps.end(), P->R->warps.begin() + 1 + o_warp[i]);
      std::copy(O.palette_colors.begin(), O.palette_colors.end(), P->R->palette_colors.begin() + o_pal[i]);
      std::copy(O.units.begin(), O.units.end(), P->R->units.begin() + o_unit[i]);
      std::copy(O.inter_tiles.begin(), O.inter_tiles.end(), P->R->inter_tiles.begin() + o_tile[i]);
      std::copy(O.inter_tiles_mask.begin(), O.inter_tiles_mask.end(),
                P->R->inter_tiles.begin() + o_tile[pieces] + o_tilem[i]);
      std::copy(O.inter_tiles_full.begin(), O.inter_tiles_full.end(),
                P->R->inter_tiles.begin() + o_tile[pieces] + o_tilem[pieces] + o_tilef[i]);
      for (size_t k = 0; k < O.itx_jobs.size(); ++k) {
        int2 j = O.itx_jobs[k];
        j.y += dtx;
        c.scratch->itx_unsorted[o_itx[i] + k] = j;
      }
      std::copy(O.dq.begin(), O.dq.end(), P->R->dq.begin() + o_dq[i]);
    });
  }
  plan_shared_masks(c, P);
  phase(kStPlanBlocks);
  if ((rc_units = plan_units(d, c, P))) return rc_units;
  phase(kStPlanUnits);
  plan_itx(c, P);
  phase(kStPlanItx);

  /* the pools read past the caller's arrays as zeros, like the reference's
   * padded plan pools (engine.cpp:665-674) */
  P->coef_pool = c.levels ? coef_end + 64 : std::max(coef_end + 64, s.n_coefficients);
  P->residual_pool = std::max(res_end + 64, s.n_residual);

  /* deblocking edges and CDEF blocks: converted on the device where they
   * are uploaded (plan_frame, k_prep_filters) */
  if (s.sharpness < 0 || s.sharpness > 7) return fail(d, AV1B_ERR_SYNTAX, "sharpness out of range");
  P->cdef_grid_w = L.p[0].stride >> 3;
  P->cdef_grid_n = P->cdef_grid_w * (plane_rows(L, 0) >> 3);
  /* an error found after them still reports an invalid filter record first,
   * as it comes earlier in the frame's validation order */
  auto fail_late = [&](int code, const char* msg) {
    const int rc = filter_records_error(d, c, s);
    return rc ? rc : fail(d, code, msg);
  };

  /* loop restoration */
  P->use_lr = false;
  std::memset(&P->lr, 0, sizeof(P->lr));
  for (int p = 0; p < 3; ++p) {
    P->R->lr_units[p].clear();
    if (s.restoration_type[p] == 0) continue;
    const int sub_y = p ? L.ss_y : 0;
    if (s.restoration_unit_log2[p] < 5 || s.restoration_unit_log2[p] > 8)
      return fail_late(AV1B_ERR_SYNTAX, "restoration unit size out of range");
    const int us = 1 << s.restoration_unit_log2[p];
    const int fh = (s.height + (sub_y ? 1 << (sub_y - 1) : 0)) >> sub_y;
    P->lr.type[p] = 1;
    P->lr.unit_size[p] = us;
    P->lr.unit_rows[p] = std::max((fh + (us >> 1)) / us, 1);
    P->lr.unit_cols[p] = std::max(s.restoration_unit_cols[p], 1);
    P->lr.n_units[p] = static_cast<int>(s.n_restoration[p]);
    for (size_t i = 0; i < s.n_restoration[p]; ++i) {
      const av1b_restoration_unit& u = s.restoration[p][i];
      LrUnitRec o{};
      /* the reference engine's mapping (engine.cpp:1417-1455): type 2 is the
       * Wiener filter, any other non-zero type the self-guided one */
      o.type = u.type == 0 ? 0 : (u.type == 2 ? 1 : 2);
      for (int k = 0; k < 3; ++k) {
        o.vf[k] = u.wiener[0][k];
        o.hf[k] = u.wiener[1][k];
      }
      const short* sp = sgr_params_table() + (u.sgr_set & 15) * 4;
      o.r[0] = sp[0];
      o.e[0] = sp[1];
      o.r[1] = sp[2];
      o.e[1] = sp[3];
      o.xqd[0] = u.sgr_xqd[0];
      o.xqd[1] = u.sgr_xqd[1];
      P->R->lr_units[p].push_back(o);
    }
    P->use_lr = true;
  }

  phase(kStPlanFilters);

  /* film grain */
  P->grain = s.grain.apply != 0;
  if (P->grain) {
    const av1b_film_grain& f = s.grain;
    if (f.seed < 0 || f.seed > 65535 || f.ar_coeff_lag < 0 || f.ar_coeff_lag > 3 ||
        f.num_y_points < 0 || f.num_y_points > 16 || f.num_cb_points < 0 || f.num_cb_points > 16 ||
        f.num_cr_points < 0 || f.num_cr_points > 16 || f.grain_scaling_minus_8 < 0 ||
        f.grain_scaling_minus_8 > 3 || f.ar_coeff_shift_minus_6 < 0 || f.ar_coeff_shift_minus_6 > 3 ||
        f.grain_scale_shift < 0 || f.grain_scale_shift > 3)
      return fail_late(AV1B_ERR_SYNTAX, "film grain parameters out of range");
    auto check_points = [&](int n, const int32_t* v) {
      for (int i = 0; i < n; ++i) {
        if (v[i] < 0 || v[i] > 255) return false;
        if (i > 0 && v[i] <= v[i - 1]) return false;
      }
      return true;
    };
    if (!check_points(f.num_y_points, f.point_y_value) ||
        !check_points(f.num_cb_points, f.point_cb_value) ||
        !check_points(f.num_cr_points, f.point_cr_value))
      return fail_late(AV1B_ERR_SYNTAX, "film grain points must increase strictly within 0..255");
    GrainParamsDev& g = P->gp;
    std::memset(&g, 0, sizeof(g));
    g.seed = f.seed;
    g.bitdepth = bd;
    g.ss_x = s.ss_x;
    g.ss_y = s.ss_y;
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
    GrainState& t = P->gs_tail;
    const bool chroma = f.chroma_scaling_from_luma || f.num_cb_points > 0 || f.num_cr_points > 0;
    grain_scaling_lut(f.num_y_points, f.point_y_value, f.point_y_scaling, t.lut[0]);
    if (chroma) {
      if (f.chroma_scaling_from_luma) {
        grain_scaling_lut(f.num_y_points, f.point_y_value, f.point_y_scaling, t.lut[1]);
        grain_scaling_lut(f.num_y_points, f.point_y_value, f.point_y_scaling, t.lut[2]);
      } else {
        grain_scaling_lut(f.num_cb_points, f.point_cb_value, f.point_cb_scaling, t.lut[1]);
        grain_scaling_lut(f.num_cr_points, f.point_cr_value, f.point_cr_scaling, t.lut[2]);
      }
    } else {
      std::memset(t.lut[1], 0, sizeof(t.lut[1]));
      std::memset(t.lut[2], 0, sizeof(t.lut[2]));
    }
    t.seed = f.seed;
    t.bitdepth = bd;
    t.overlap = f.overlap_flag ? 1 : 0;
    t.scaling_shift = f.grain_scaling_minus_8 + 8;
    t.num_points[0] = f.num_y_points;
    t.num_points[1] = f.num_cb_points;
    t.num_points[2] = f.num_cr_points;
    t.chroma_from_luma = f.chroma_scaling_from_luma ? 1 : 0;
    t.mult[1] = f.cb_mult;
    t.luma_mult[1] = f.cb_luma_mult;
    t.offset[1] = f.cb_offset;
    t.mult[2] = f.cr_mult;
    t.luma_mult[2] = f.cr_luma_mult;
    t.offset[2] = f.cr_offset;
    const int maxv = (1 << bd) - 1;
    t.min_value = 0;
    t.max_luma = maxv;
    t.max_chroma = maxv;
    if (f.clip_to_restricted_range) {
      t.min_value = 16 << (bd - 8);
      t.max_luma = 235 << (bd - 8);
      t.max_chroma = s.color_matrix == 3 ? t.max_luma : (240 << (bd - 8));
    }
    t.chroma_w = s.ss_x ? 44 : 82;
    t.chroma_h = s.ss_y ? 38 : 73;
  }
  phase(kStPlanGrain);
  return AV1B_OK;
}

/* ---- the frame step ------------------------------------------------------------------------ */

/* Reserves room for `v` in the staging arena; returns its offset. */
template <class V>
size_t stage_put(size_t* off, const V& v) {
  const size_t o = *off;
  *off = align_up(o + v.size() * sizeof(typename V::value_type), 256);
  return o;
}

cudaEvent_t pool_event(av1b_decoder* d) {
  if (d->ev_used == d->ev_pool.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    d->ev_pool.push_back(e);
  }
  return d->ev_pool[d->ev_used++];
}

/* Runs `launch`; with profiling on, brackets it with two events. */
template <class F>
cudaError_t timed(av1b_decoder* d, int stage, F launch, cudaStream_t on = nullptr) {
  if (!d->profiling) return launch();
  if (!on) on = d->stream;
  const size_t i0 = d->ev_used;
  cudaEvent_t a = pool_event(d);
  cudaEvent_t b = pool_event(d);
  if (!a || !b) return cudaErrorMemoryAllocation;
  cudaEventRecord(a, on);
  const cudaError_t e = launch();
  cudaEventRecord(b, on);
  d->marks.push_back(std::make_pair(stage, i0));
  return e;
}

/* After a synchronisation: folds the recorded stage times into the totals. */
void collect_profile(av1b_decoder* d) {
  for (const auto& m : d->marks) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, d->ev_pool[m.second], d->ev_pool[m.second + 1]) == cudaSuccess) {
      d->prof_ms[m.first] += ms;
      d->prof_n[m.first] += 1;
    }
  }
  d->marks.clear();
  d->ev_used = 0;
}

int check_header(av1b_decoder* d, const av1b_frame_syntax& s) {
  if (s.width <= 0 || s.height <= 0) return fail(d, AV1B_ERR_SYNTAX, "frame has no size");
  if (s.bit_depth != 8 && s.bit_depth != 10 && s.bit_depth != 12)
    return fail(d, AV1B_ERR_SYNTAX, "bit depth must be 8, 10 or 12");
  if (s.ss_x < 0 || s.ss_x > 1 || s.ss_y < 0 || s.ss_y > 1 || (s.ss_y && !s.ss_x))
    return fail(d, AV1B_ERR_SYNTAX, "unsupported chroma subsampling");
  if (s.width > 16384 || s.height > 16384) return fail(d, AV1B_ERR_SYNTAX, "frame too large");
  if ((s.n_blocks && !s.blocks) || (s.n_transforms && !s.transforms) || (s.n_obmc && !s.obmc) ||
      (s.n_coefficients && !s.coefficients) || (s.n_residual && !s.residual) ||
      (s.n_levels && !s.levels) || (s.n_qm_pool && !s.qm_pool) ||
      (s.n_palette_map && !s.palette_map) || (s.n_deblock && !s.deblock) || (s.n_cdef && !s.cdef) ||
      (s.n_reference_slots && !s.reference_slots) ||
      (s.n_restoration[0] && !s.restoration[0]) || (s.n_restoration[1] && !s.restoration[1]) ||
      (s.n_restoration[2] && !s.restoration[2]))
    return fail(d, AV1B_ERR_ARG, "a syntax array with a length but no data");
  return AV1B_OK;
}

}  // namespace
}  // namespace av1b

/* A planned frame: the validated device records of one FrameSyntax, already
 * uploaded into device memory the plan owns (the reference's FramePlan,
 * backend.hpp:140-206, which stays on the host there). */
struct av1b_plan {
  int width = 0, height = 0, coded_width = 0, bit_depth = 8, ss_x = 1, ss_y = 1;
  int sharpness = 0, color_matrix = 1;
  av1b::Layout L{};
  av1b::Plan P;                   /* host copy of the counts and constants */
  av1b::DevBuf arena, coef, residual;
  av1b::DevBuf dqsrc;             /* a levels frame's levels, then its QM pool */
  /* the caller's deblocking edges and CDEF blocks as uploaded, and the
   * records k_prep_filters makes of them (offsets o_de_raw .. o_prep) */
  av1b::DevBuf filt;
  av1b::PrepOut* prep_host = nullptr;   /* page-locked copy of the counts */
  /* ready: the uploads are done; done: the last frame that read this plan has
   * finished on the device (a plan is re-planned only after that) */
  cudaEvent_t ready = nullptr, done = nullptr;
  bool in_flight = false;
  size_t o_blocks = 0, o_txs = 0, o_obmc = 0, o_warps = 0, o_pal = 0, o_units = 0, o_deps = 0;
  size_t o_chains = 0;
  size_t o_tiles = 0, o_itx = 0, o_itxb = 0, o_dbv = 0, o_dbh = 0, o_cdef = 0, o_lr[3] = {0, 0, 0};
  size_t o_map = 0, o_cdef_search = 0, o_dq = 0, o_de_raw = 0, o_cb_raw = 0, o_prep = 0;
  size_t o_gs = 0;                /* the film grain constants and scaling tables */
  int slots_read[kSlots + 1];     /* the reference slots the frame reads, -1 ended */
  int n_blocks = 0;
  bool owned_by_decoder = false;
};

namespace av1b {
namespace {

/* Plans `s` into `pl`: validation, records, and the upload of records and
 * coefficient pools into the plan's device memory, on the upload stream. It
 * takes neither the decoder's lock nor its stream, so a pipeline plans frame
 * N+1 while frame N runs. It returns once the uploads are done: the caller's
 * arrays are free again. */
int plan_frame(av1b_decoder* d, const av1b_frame_syntax& s, av1b_plan* pl) {
  /* a free planner, held for this call */
  av1b_decoder::Planner* pn = nullptr;
  {
    std::unique_lock<std::mutex> lk(d->planner_mu);
    d->planner_cv.wait(lk, [&] {
      for (auto& q : d->planners)
        if (!q.busy) return true;
      return false;
    });
    for (auto& q : d->planners)
      if (!q.busy) {
        pn = &q;
        break;
      }
    pn->busy = true;
  }
  struct Release {
    av1b_decoder* d;
    av1b_decoder::Planner* pn;
    ~Release() {
      {
        std::lock_guard<std::mutex> lk(d->planner_mu);
        pn->busy = false;
      }
      d->planner_cv.notify_one();
    }
  } release{d, pn};
  int rc;
  if ((rc = check_header(d, s))) return rc;
  const int coded_width = (s.coded_width <= 0 || s.coded_width > s.width) ? s.width : s.coded_width;
  PlanCtx c;
  c.L = make_layout(s.width, s.height, coded_width, s.bit_depth, s.ss_x, s.ss_y);
  {
    std::lock_guard<std::mutex> lk(d->slot_mu);
    for (int i = 0; i < kSlots; ++i) {
      c.slot_used[i] = d->slot_used[i];
      c.slot_valid[i] = d->slot_valid[i];
      c.slot_width[i] = d->slot_width[i];
      c.slot_height[i] = d->slot_height[i];
    }
  }
  c.pool = pn->pool;
  c.scratch = pn->scratch;
  /* a frame that carries its coded levels is dequantised on the device, the
   * reference engine's device-dequantiser path (engine.cpp:386, 655-670):
   * its coefficient array, if it has one too, is not uploaded */
  c.levels = s.n_levels > 0;
  c.n_levels = s.n_levels;
  c.n_qm = s.n_qm_pool;
  c.share_masks = d->share_masks.load();
  const size_t n_coef = c.levels ? 0 : s.n_coefficients;
  if (!pl->ready) {
    /* blocking-sync events: a waiting planner sleeps instead of spinning on
     * a core the planner pool or the decoding thread could use */
    CK(cudaEventCreateWithFlags(&pl->ready, cudaEventDisableTiming | cudaEventBlockingSync), "event");
    CK(cudaEventCreateWithFlags(&pl->done, cudaEventDisableTiming | cudaEventBlockingSync), "event");
  }
  if (!pl->prep_host)
    CK(cudaHostAlloc(reinterpret_cast<void**>(&pl->prep_host), sizeof(PrepOut), cudaHostAllocDefault),
       "page-locked counts");
  if (pl->in_flight) {
    CK(cudaEventSynchronize(pl->done), "plan reuse wait");
    pl->in_flight = false;
  }
  Plan& P = pl->P;
  P.R = pn->lists;
  {
    /* grow to the largest frame planned so far (a failed growth is left to
     * the planning that needs it, which reports it) */
    size_t hw[32], arena_hw, filt_hw;
    {
      std::lock_guard<std::mutex> lk(d->hw_mu);
      std::copy(d->list_hw, d->list_hw + 32, hw);
      arena_hw = d->arena_hw;
      filt_hw = d->filt_hw;
    }
    try {
      each_list(*P.R, [&](int i, auto& v) {
        if (v.capacity() < hw[i]) v.reserve(hw[i]);
      });
    } catch (const std::bad_alloc&) {
    }
    auto pre_grow = [&](DevBuf& b, size_t bytes) {
      if (b.cap >= bytes) return;
      {
        std::lock_guard<std::mutex> lk(d->alloc_mu);
        if (d->budget && d->allocated - b.cap + align_up(bytes + bytes / 8, 1 << 16) > d->budget) return;
      }
      dev_ensure(d, b, bytes);
    };
    pre_grow(pl->arena, arena_hw);
    pre_grow(pl->filt, filt_hw);
  }
  cudaStream_t st = pn->upload;
  /* the caller's coefficients and raw residuals go up first, while the
   * records are built */
  /* a frame's coefficients never outnumber its samples: a plan's pool is
   * made that large on first use, whatever frame it first holds */
  if ((rc = dev_ensure(d, pl->coef, (n_coef + 64) * sizeof(int),
                       (static_cast<size_t>(c.L.size) + 64) * sizeof(int))) ||
      (rc = dev_ensure(d, pl->residual, (s.n_residual + 64) * sizeof(int))))
    return rc;
  if (n_coef)
    CK(cudaMemcpyAsync(pl->coef.p, s.coefficients, n_coef * sizeof(int),
                       cudaMemcpyHostToDevice, st), "coefficient upload");
  const size_t qm_at = align_up(s.n_levels * sizeof(int16_t), 256);
  if (c.levels) {
    const size_t bytes = qm_at + s.n_qm_pool + 64;
    if ((rc = dev_ensure(d, pl->dqsrc, bytes, bytes + bytes / 2))) return rc;
    CK(cudaMemcpyAsync(pl->dqsrc.p, s.levels, s.n_levels * sizeof(int16_t), cudaMemcpyHostToDevice,
                       st), "level upload");
    if (s.n_qm_pool)
      CK(cudaMemcpyAsync(static_cast<uint8_t*>(pl->dqsrc.p) + qm_at, s.qm_pool, s.n_qm_pool,
                         cudaMemcpyHostToDevice, st), "quantiser matrix upload");
  }
  /* the deblocking edges and CDEF blocks go up as they are and are converted
   * on the device while the host plans the rest */
  {
    const size_t nde = s.n_deblock, ncb = s.n_cdef;
    size_t fo = 0;
    auto room = [&](size_t bytes) {
      const size_t o = fo;
      fo = align_up(fo + bytes, 256);
      return o;
    };
    pl->o_de_raw = room(nde * sizeof(av1b_deblock_edge));
    pl->o_cb_raw = room(ncb * sizeof(av1b_cdef_block));
    pl->o_dbv = room(nde * sizeof(DeblockRec));
    pl->o_dbh = room(nde * sizeof(DeblockRec));
    pl->o_cdef = room(ncb * sizeof(CdefRec));
    pl->o_cdef_search = room(ncb * sizeof(unsigned));
    pl->o_prep = room(sizeof(PrepOut));
    if ((rc = dev_ensure(d, pl->filt, fo, fo + fo / 2))) {
      cudaStreamSynchronize(st);
      return rc;
    }
    {
      std::lock_guard<std::mutex> lk(d->hw_mu);
      d->filt_hw = std::max(d->filt_hw, fo);  /* the bytes needed, not the capacity: no runaway */
    }
    uint8_t* fl = static_cast<uint8_t*>(pl->filt.p);
    if (nde)
      CK(cudaMemcpyAsync(fl + pl->o_de_raw, s.deblock, nde * sizeof(av1b_deblock_edge),
                         cudaMemcpyHostToDevice, st), "deblock edge upload");
    if (ncb)
      CK(cudaMemcpyAsync(fl + pl->o_cb_raw, s.cdef, ncb * sizeof(av1b_cdef_block),
                         cudaMemcpyHostToDevice, st), "CDEF block upload");
    CK(cudaMemsetAsync(fl + pl->o_prep, 0, sizeof(PrepOut), st), "count reset");
    const int grid_w = c.L.p[0].stride >> 3;
    CK(launch_prep_filters(reinterpret_cast<const av1b_deblock_edge*>(fl + pl->o_de_raw),
                           static_cast<int>(nde),
                           reinterpret_cast<const av1b_cdef_block*>(fl + pl->o_cb_raw),
                           static_cast<int>(ncb), c.L, grid_w, grid_w * (plane_rows(c.L, 0) >> 3),
                           reinterpret_cast<DeblockRec*>(fl + pl->o_dbv),
                           reinterpret_cast<DeblockRec*>(fl + pl->o_dbh),
                           reinterpret_cast<CdefRec*>(fl + pl->o_cdef),
                           reinterpret_cast<unsigned*>(fl + pl->o_cdef_search),
                           reinterpret_cast<PrepOut*>(fl + pl->o_prep), st),
       "filter record launch");
    CK(cudaMemcpyAsync(pl->prep_host, fl + pl->o_prep, sizeof(PrepOut), cudaMemcpyDeviceToHost, st),
       "count read back");
  }
  if (s.n_residual)
    CK(cudaMemcpyAsync(pl->residual.p, s.residual, s.n_residual * sizeof(int),
                       cudaMemcpyHostToDevice, st), "residual upload");
  auto t0 = std::chrono::steady_clock::now();
  try {
    rc = build_plan(d, c, s, &P);
  } catch (const std::bad_alloc&) {
    rc = fail(d, AV1B_ERR_NOMEM, "host memory exhausted while planning");
  }
  if (rc) {
    cudaStreamSynchronize(st);  /* nothing in flight reads the caller's arrays */
    return rc;
  }
  {
    std::lock_guard<std::mutex> lk(d->hw_mu);
    each_list(*P.R, [&](int i, auto& v) { d->list_hw[i] = std::max(d->list_hw[i], v.capacity()); });
  }
  host_mark(d, kStPlanHost, t0);
  P.n_blocks = P.R->blocks.size();
  P.n_units = P.R->units.size();
  P.n_tiles = P.R->inter_tiles.size();
  P.n_itx = P.R->itx_jobs.size();
  P.n_itxb = P.R->itx_batches.size();
  pl->L = c.L;
  pl->width = s.width;
  pl->height = s.height;
  pl->coded_width = coded_width;
  pl->bit_depth = s.bit_depth;
  pl->ss_x = s.ss_x;
  pl->ss_y = s.ss_y;
  pl->sharpness = s.sharpness;
  pl->color_matrix = s.color_matrix;
  pl->n_blocks = static_cast<int>(s.n_blocks);
  {
    bool used[kSlots] = {false};
    for (const BlockRec& b : P.R->blocks)
      for (int k = 0; k < 2; ++k)
        if (b.ref_slot[k] >= 0) used[b.ref_slot[k]] = true;
    for (const ObmcRec& o : P.R->obmc)
      if (o.ref_slot >= 0) used[o.ref_slot] = true;
    int n = 0;
    for (int i = 0; i < kSlots; ++i)
      if (used[i]) pl->slots_read[n++] = i;
    pl->slots_read[n] = -1;
  }
  size_t off = 0;
  pl->o_blocks = stage_put(&off, P.R->blocks);
  pl->o_txs = stage_put(&off, P.R->txs);
  pl->o_obmc = stage_put(&off, P.R->obmc);
  pl->o_warps = stage_put(&off, P.R->warps);
  pl->o_pal = stage_put(&off, P.R->palette_colors);
  pl->o_units = stage_put(&off, P.R->units);
  pl->o_chains = stage_put(&off, P.R->chains);
  pl->o_deps = stage_put(&off, P.R->deps);
  pl->o_tiles = stage_put(&off, P.R->inter_tiles);
  pl->o_itx = stage_put(&off, P.R->itx_jobs);
  pl->o_itxb = stage_put(&off, P.R->itx_batches);
  for (int p = 0; p < 3; ++p) pl->o_lr[p] = stage_put(&off, P.R->lr_units[p]);
  pl->o_dq = stage_put(&off, P.R->dq);
  const size_t gs_tail = offsetof(GrainState, lut);
  pl->o_gs = off;
  off = align_up(off + (sizeof(GrainState) - gs_tail), 256);
  pl->o_map = off;
  off = align_up(off + s.n_palette_map + 64, 256);
  const size_t total = off;
  if ((rc = dev_ensure(d, pl->arena, total, total + total / 2))) {
    cudaStreamSynchronize(st);
    return rc;
  }
  {
    std::lock_guard<std::mutex> lk(d->hw_mu);
    d->arena_hw = std::max(d->arena_hw, total);
  }
  /* the record lists upload from where the planner wrote them (page-locked) */
  t0 = std::chrono::steady_clock::now();
  uint8_t* ar = static_cast<uint8_t*>(pl->arena.p);
  auto put = [&](size_t o, const auto& v) -> cudaError_t {
    const size_t bytes = v.size() * sizeof(v[0]);
    return bytes ? cudaMemcpyAsync(ar + o, v.data(), bytes, cudaMemcpyHostToDevice, st) : cudaSuccess;
  };
  CK(put(pl->o_blocks, P.R->blocks), "record upload");
  CK(put(pl->o_txs, P.R->txs), "record upload");
  CK(put(pl->o_obmc, P.R->obmc), "record upload");
  CK(put(pl->o_warps, P.R->warps), "record upload");
  CK(put(pl->o_pal, P.R->palette_colors), "record upload");
  CK(put(pl->o_units, P.R->units), "record upload");
  CK(put(pl->o_chains, P.R->chains), "record upload");
  CK(put(pl->o_deps, P.R->deps), "record upload");
  CK(put(pl->o_tiles, P.R->inter_tiles), "record upload");
  CK(put(pl->o_itx, P.R->itx_jobs), "record upload");
  CK(put(pl->o_itxb, P.R->itx_batches), "record upload");
  for (int p = 0; p < 3; ++p) CK(put(pl->o_lr[p], P.R->lr_units[p]), "record upload");
  CK(put(pl->o_dq, P.R->dq), "record upload");
  /* the grain constants: from the plan's own memory (its upload is waited
   * for before plan_frame returns), copied into the decoder's grain state on
   * the device when the frame runs */
  if (P.grain)
    CK(cudaMemcpyAsync(ar + pl->o_gs, reinterpret_cast<const uint8_t*>(&P.gs_tail) + gs_tail,
                       sizeof(GrainState) - gs_tail, cudaMemcpyHostToDevice, st), "grain constants upload");
  if (s.n_palette_map)
    CK(cudaMemcpyAsync(ar + pl->o_map, s.palette_map, s.n_palette_map, cudaMemcpyHostToDevice, st),
       "palette map upload");
  CK(cudaMemsetAsync(ar + pl->o_map + s.n_palette_map, 0, 64, st), "palette map pad");
  host_mark(d, kStStageHost, t0);

  /* the pools read past the caller's arrays as zeros; a pool longer than the
   * early copy's buffer is copied again into a larger one */
  const size_t coef_cap = pl->coef.cap / sizeof(int), res_cap = pl->residual.cap / sizeof(int);
  if (P.coef_pool > coef_cap || P.residual_pool > res_cap) {
    CK(cudaStreamSynchronize(st), "upload sync");
    if ((rc = dev_ensure(d, pl->coef, P.coef_pool * sizeof(int))) ||
        (rc = dev_ensure(d, pl->residual, P.residual_pool * sizeof(int))))
      return rc;
    if (n_coef)
      CK(cudaMemcpyAsync(pl->coef.p, s.coefficients, n_coef * sizeof(int),
                         cudaMemcpyHostToDevice, st), "coefficient upload");
    if (s.n_residual)
      CK(cudaMemcpyAsync(pl->residual.p, s.residual, s.n_residual * sizeof(int),
                         cudaMemcpyHostToDevice, st), "residual upload");
  }
  if (c.levels) {
    /* every raster a transform reads is written whole by the dequantiser */
    const uint8_t* src = static_cast<const uint8_t*>(pl->dqsrc.p);
    CK(launch_dequant(reinterpret_cast<const DqRec*>(ar + pl->o_dq), static_cast<int>(P.n_dq),
                      reinterpret_cast<const short*>(src), s.n_qm_pool ? src + qm_at : nullptr,
                      static_cast<int*>(pl->coef.p), s.bit_depth, st),
       "dequantiser launch");
  } else if (P.coef_pool > n_coef) {
    CK(cudaMemsetAsync(static_cast<int*>(pl->coef.p) + n_coef, 0,
                       (P.coef_pool - n_coef) * sizeof(int), st), "coefficient pad");
  }
  if (P.residual_pool > s.n_residual)
    CK(cudaMemsetAsync(static_cast<int*>(pl->residual.p) + s.n_residual, 0,
                       (P.residual_pool - s.n_residual) * sizeof(int), st), "residual pad");
  CK(cudaEventRecord(pl->ready, st), "event");
  t0 = std::chrono::steady_clock::now();
  CK(cudaEventSynchronize(pl->ready), "upload wait");
  host_mark(d, kStWaitHost, t0);
  const PrepOut po = *pl->prep_host;
  if (po.bad) {
    rc = filter_records_error(d, c, s);
    return rc ? rc : fail(d, AV1B_ERR_SYNTAX, "invalid deblocking edge or CDEF block");
  }
  P.n_dbv = po.n_v;
  P.n_dbh = po.n_h;
  P.n_cdef = s.n_cdef;
  P.n_cdef_search = po.n_extra;
  P.cdef_search_any = po.any_grid != 0;
  P.R = nullptr;
  return AV1B_OK;
}

/* Runs a planned frame on the device: reconstruction, filters, reference
 * store, film grain, and (with `out`) the read back. `sync`: wait for the
 * frame and check its status word before returning. */
int finish_frame(av1b_decoder* d);

/* One frame step's arguments: the destination slot, the reconstruction
 * kernels' FrameArgs and (in a batched step) the filter chain's FilterArgs. */
struct StepPrep {
  int slot = -1;
  int keep = 0;
  int launches = 0;
  /* the frame's film grain is applied when an output call asks for it (its
   * decode reads nothing back): the NV12 pack of the frame then applies it
   * while packing, and no display picture is written */
  bool defer_grain = false;
  FrameArgs a{};
  FilterArgs f{};
};

int fill_filter_args(av1b_decoder* d, av1b_plan* pl, StepPrep* sp);

/* The host side of a frame step before anything is launched: the
 * destination slot, the buffers the frame needs, the done flags, claim
 * counter and status word (reset on the decoder's stream), the slot table,
 * and the arguments. In a batched step (`batched`) the film grain constants
 * are uploaded on the decoder's stream as well, and the filter chain's
 * arguments are filled for the batched kernels. Called with the decoder's
 * lock held. */
int prepare_step(av1b_decoder* d, av1b_plan* pl, int keep, int forced_slot, bool batched,
                 StepPrep* sp, cudaStream_t st) {
  int rc;
  av1b_frame_syntax hdr{};
  hdr.width = pl->width;
  hdr.height = pl->height;
  hdr.bit_depth = pl->bit_depth;
  hdr.ss_x = pl->ss_x;
  hdr.ss_y = pl->ss_y;
  if ((rc = ensure_geometry(d, hdr, pl->coded_width))) return rc;
  if (std::memcmp(&d->L, &pl->L, sizeof(Layout)) != 0)
    return fail(d, AV1B_ERR_ARG, "a plan of another picture layout");
  for (int i = 0; pl->slots_read[i] >= 0; ++i) {
    const int sl = pl->slots_read[i];
    if (!d->slot_used[sl] || !d->slot_valid[sl] || d->slot_width[sl] != pl->width ||
        d->slot_height[sl] != pl->height)
      return fail(d, AV1B_ERR_SYNTAX, "a planned frame reads a slot that holds no picture of its size");
  }
  const Plan& P = pl->P;
  const Layout& L = d->L;
  const int maxv = (1 << pl->bit_depth) - 1;
  cudaEvent_t* ev = d->ev;

  /* the destination slot */
  int slot = -1;
  if (keep) {
    if (forced_slot >= 0) {
      if (forced_slot >= kSlots || !d->slot_used[forced_slot])
        return fail(d, AV1B_ERR_ARG, "invalid reserved slot");
      slot = forced_slot;
    } else {
      for (int i = 0; i < kSlots; ++i)
        if (!d->slot_used[i]) {
          slot = i;
          break;
        }
      if (slot < 0) return fail(d, AV1B_ERR_NOMEM, "reference pool exhausted");
    }
    if ((rc = dev_ensure(d, d->slot_buf[slot], static_cast<size_t>(L.size) * sizeof(px_t)))) return rc;
  }
  const size_t pic_bytes = static_cast<size_t>(L.size) * sizeof(px_t);
  if (P.pre_res_pool && (rc = dev_ensure(d, d->pre_res, P.pre_res_pool * sizeof(int)))) return rc;
  if (P.mask_pool && (rc = dev_ensure(d, d->mask_pool, P.mask_pool))) return rc;
  if ((P.cdef_search_any || (P.n_cdef_search != 0)) &&
      (rc = dev_ensure(d, d->cdef_search, (P.cdef_grid_n + P.n_cdef_search) * sizeof(int))))
    return rc;
  if (P.use_lr) {
    if ((rc = dev_ensure(d, d->lr_cdef, pic_bytes)) ||
        (P.upscaled && (rc = dev_ensure(d, d->lr_pre_up, pic_bytes))))
      return rc;
  }
  if (P.grain && (rc = init_grain_tables(d))) return rc;

  /* the plan's uploads (done when plan_frame returned; the wait orders them
   * on this stream) */
  CK(cudaStreamWaitEvent(st, pl->ready, 0), "upload order");

  /* slot pointer table, uploaded when a slot buffer moved */
  {
    px_t* ptrs[kSlots];
    for (int i = 0; i < kSlots; ++i) ptrs[i] = static_cast<px_t*>(d->slot_buf[i].p);
    if ((rc = dev_ensure(d, d->slot_ptr_dev, sizeof(ptrs)))) return rc;
    if (std::memcmp(ptrs, d->slot_ptr_host, sizeof(ptrs)) != 0) {
      std::memcpy(d->slot_ptr_host, ptrs, sizeof(ptrs));
      CK(cudaMemcpyAsync(d->slot_ptr_dev.p, d->slot_ptr_host, sizeof(ptrs), cudaMemcpyHostToDevice, st),
         "slot table upload");
    }
  }
  uint8_t* ar = static_cast<uint8_t*>(pl->arena.p);

  /* done flags, queue and status */
  FrameArgs& a = sp->a;
  a.L = L;
  const size_t done_bytes =
      static_cast<size_t>(pl->n_blocks) * AV1B_FLAG_STRIDE * sizeof(unsigned) + 256;
  if (d->done.cap < done_bytes) {
    if ((rc = dev_ensure(d, d->done, done_bytes))) return rc;
    CK(cudaMemsetAsync(d->done.p, 0, d->done.cap, st), "done reset");
  }
  ++d->epoch;
  if (d->epoch == 0) {
    CK(cudaMemsetAsync(d->done.p, 0, d->done.cap, st), "done reset");
    d->epoch = 1;
  }
  if (!d->status_q.p) {
    if ((rc = dev_ensure(d, d->status_q, 256))) return rc;
    CK(cudaMemsetAsync(d->status_q.p, 0, 256, st), "status reset");
  }
  /* the claim counter restarts every frame; the status word is sticky until
   * finish_frame has read it, so frames queued without a wait are covered */
  if (!batched)   /* a batched step claims chains from its own counter */
    CK(cudaMemsetAsync(d->status_q.p, 0, sizeof(unsigned), st), "queue reset");

  a.cur = static_cast<px_t*>(d->cur.p);
  a.slot_ptr = static_cast<px_t* const*>(d->slot_ptr_dev.p);
  a.blocks = reinterpret_cast<const BlockRec*>(ar + pl->o_blocks);
  a.n_blocks = static_cast<int>(P.n_blocks);
  a.txs = reinterpret_cast<const TxRec*>(ar + pl->o_txs);
  a.obmc = reinterpret_cast<const ObmcRec*>(ar + pl->o_obmc);
  a.warps = reinterpret_cast<const WarpRec*>(ar + pl->o_warps);
  a.coef = static_cast<const int*>(pl->coef.p);
  a.residual = static_cast<const int*>(pl->residual.p);
  a.palette_map = ar + pl->o_map;
  a.palette_colors = reinterpret_cast<const int*>(ar + pl->o_pal);
  a.done = static_cast<unsigned*>(d->done.p);
  a.epoch = d->epoch;
  a.units = reinterpret_cast<const int*>(ar + pl->o_units);
  a.n_units = static_cast<int>(P.n_units);
  a.chains = reinterpret_cast<const int*>(ar + pl->o_chains);
  a.n_chains = static_cast<int>(P.n_chains);
  a.deps = reinterpret_cast<const int*>(ar + pl->o_deps);
  a.units_inter = P.units_inter ? 1 : 0;
  a.queue = static_cast<unsigned*>(d->status_q.p);
  a.trace = nullptr;
  if (d->tracing) {
    const size_t bytes = static_cast<size_t>(pl->n_blocks) * 4 * sizeof(unsigned long long) + 64;
    if ((rc = dev_ensure(d, d->trace, bytes))) return rc;
    CK(cudaMemsetAsync(d->trace.p, 0, bytes, st), "trace reset");
    a.trace = static_cast<unsigned long long*>(d->trace.p);
    d->trace_n = static_cast<size_t>(pl->n_blocks) * 4;
  }
  a.status = reinterpret_cast<int*>(static_cast<uint8_t*>(d->status_q.p) + 64);
  a.inter_tiles = reinterpret_cast<const int2*>(ar + pl->o_tiles);
  a.n_inter_tiles = static_cast<int>(P.n_tiles);
  a.n_inter_simple = static_cast<int>(P.n_tiles_simple);
  a.n_inter_lmask = static_cast<int>(P.n_tiles_lmask);
  a.n_inter_cmask = static_cast<int>(P.n_tiles_cmask);
  a.mask_pool = static_cast<unsigned char*>(d->mask_pool.p);
  a.itx_jobs = reinterpret_cast<const int2*>(ar + pl->o_itx);
  a.n_itx = static_cast<int>(P.n_itx);
  a.itx_batches = reinterpret_cast<const int4*>(ar + pl->o_itxb);
  a.n_itx_batches = static_cast<int>(P.n_itxb);
  for (int k = 0; k < 8; ++k) {
    a.itx_class_first[k] = P.itx_class_first[k];
    a.itx_class_count[k] = P.itx_class_count[k];
  }
  a.pre_res = static_cast<int*>(d->pre_res.p);
  a.maxv = maxv;
  a.scale_x = P.scale_x;
  a.scale_y = P.scale_y;
  a.wait_ns = d->wait_ns;
  sp->slot = slot;
  sp->keep = keep;
  if (batched) {
    a.trace = nullptr;
    if ((rc = fill_filter_args(d, pl, sp))) return rc;
  }
  return AV1B_OK;
}

/* The single-stream launch sequence of a prepared frame step on the
 * decoder's stream (the grain templates on its side stream). */
int launch_step_plain(av1b_decoder* d, av1b_plan* pl, StepPrep* sp) {
  const Plan& P = pl->P;
  const Layout& L = d->L;
  const int maxv = (1 << pl->bit_depth) - 1;
  cudaStream_t st = d->stream;
  cudaEvent_t* ev = d->ev;
  const FrameArgs& a = sp->a;
  const int keep = sp->keep, slot = sp->slot;
  const size_t pic_bytes = static_cast<size_t>(L.size) * sizeof(px_t);
  uint8_t* ar = static_cast<uint8_t*>(pl->arena.p);
  int launches = 0;
  if (P.grain) {
    /* the grain templates depend only on the parameters: build them on the
     * side stream while the picture is reconstructed. The fork point orders
     * them after the previous frame's blend, which read the same state. */
    GrainState* gsd = static_cast<GrainState*>(d->grain_state.p);
    const size_t tail = offsetof(GrainState, lut);
    CK(cudaEventRecord(d->ev_fork, st), "fork");
    CK(cudaStreamWaitEvent(d->aux, d->ev_fork, 0), "fork wait");
    CK(cudaMemcpyAsync(reinterpret_cast<uint8_t*>(gsd) + tail, ar + pl->o_gs, sizeof(GrainState) - tail,
                       cudaMemcpyDeviceToDevice, d->aux), "grain constants");
    CK(timed(d, kStGrainTemplate, [&] {
         return launch_grain_template(gsd, P.gp, static_cast<const uint16_t*>(d->orbit.p),
                                      static_cast<const uint16_t*>(d->pos.p), d->aux);
       }, d->aux), "film grain template");
    CK(cudaEventRecord(d->ev_join, d->aux), "join");
    ++launches;
  }
  CK(cudaEventRecord(ev[0], st), "event");
  for (int stage = 1; stage < 4; ++stage) {
    const bool any =
        stage == 1 ? a.n_inter_tiles > 0 : (stage == 2 ? a.n_itx_batches > 0 : a.n_units > 0);
    if (!any) continue;
    CK(timed(d, kStOwner + stage, [&] { return launch_recon_stage(stage, a, d->n_sm, st); }),
       "reconstruction launch");
    /* the kernels each stage launches (launch_recon_stage): prediction up
     * to four (the lean kernel's unmasked and masked tiles, the full
     * kernel's, the chroma tiles reading luma masks), one transform kernel
     * a size class present, one dependency-scheduled kernel */
    if (stage == 1) {
      const int lm_end = a.n_inter_simple + a.n_inter_lmask, cm_first = a.n_inter_tiles - a.n_inter_cmask;
      launches += (a.n_inter_simple > 0) + (a.n_inter_lmask > 0) + (cm_first > lm_end) + (a.n_inter_cmask > 0);
    } else if (stage == 2) {
      for (int c = 2; c <= 7; ++c) launches += a.itx_class_count[c] > 0;
    } else {
      ++launches;
    }
  }
  CK(cudaEventRecord(ev[1], st), "event");

  /* ---- filters --------------------------------------------------------------------------- */
  px_t* cur = a.cur;
  const uint8_t* fl = static_cast<const uint8_t*>(pl->filt.p);
  if ((P.n_dbv != 0))
    CK(timed(d, kStDeblockV, [&] {
         return launch_deblock(cur, reinterpret_cast<const DeblockRec*>(fl + pl->o_dbv),
                               static_cast<int>(P.n_dbv), pl->sharpness, pl->bit_depth,
                               maxv, st);
       }), "deblock V");
  if ((P.n_dbh != 0))
    CK(timed(d, kStDeblockH, [&] {
         return launch_deblock(cur, reinterpret_cast<const DeblockRec*>(fl + pl->o_dbh),
                               static_cast<int>(P.n_dbh), pl->sharpness, pl->bit_depth,
                               maxv, st);
       }), "deblock H");
  launches += ((P.n_dbv != 0)) + ((P.n_dbh != 0));
  /* One snapshot of the deblocked picture serves CDEF (its source, CDEF
   * writes the picture) and loop restoration (the pre-CDEF rows of its
   * stripe boundaries); with superres the upscaled picture goes out of place
   * into the restoration's source buffer, so it needs no snapshot of its own */
  px_t* snap = static_cast<px_t*>(d->snap.p);
  if ((P.n_cdef != 0) || P.use_lr)
    CK(timed(d, kStCopy, [&] {
         return cudaMemcpyAsync(snap, cur, pic_bytes, cudaMemcpyDeviceToDevice, st);
       }), "deblocked snapshot");
  if ((P.n_cdef != 0)) {
    CK(timed(d, kStCdef, [&] {
         return launch_cdef(snap, cur, reinterpret_cast<const CdefRec*>(fl + pl->o_cdef),
                            static_cast<int>(P.n_cdef), P.cdef_grid_w, P.cdef_grid_n,
                            P.cdef_search_any,
                            reinterpret_cast<const unsigned*>(fl + pl->o_cdef_search),
                            static_cast<int>(P.n_cdef_search),
                            static_cast<int*>(d->cdef_search.p), L, st);
       }), "CDEF");
    /* the direction searches, when any record reads them, then the filter */
    launches += 1 + ((P.cdef_search_any ? P.cdef_grid_n : 0) + static_cast<int>(P.n_cdef_search) > 0);
  }
  px_t* lr_cdef = static_cast<px_t*>(d->lr_cdef.p);
  const px_t* lr_curr = snap;
  if (P.upscaled) {
    if (P.use_lr) {
      CK(timed(d, kStUpscale, [&] {
           return launch_upscale(snap, static_cast<px_t*>(d->lr_pre_up.p), L, maxv, true, st);
         }), "superres (pre-CDEF)");
      CK(timed(d, kStUpscale, [&] { return launch_upscale(cur, lr_cdef, L, maxv, false, st); }),
         "superres");
      launches += 2;
      lr_curr = static_cast<px_t*>(d->lr_pre_up.p);
    } else {
      CK(timed(d, kStCopy, [&] {
           return cudaMemcpyAsync(snap, cur, pic_bytes, cudaMemcpyDeviceToDevice, st);
         }), "superres snapshot");
      CK(timed(d, kStUpscale, [&] { return launch_upscale(snap, cur, L, maxv, false, st); }),
         "superres");
      ++launches;
    }
  } else if (P.use_lr) {
    CK(timed(d, kStCopy, [&] {
         return cudaMemcpyAsync(lr_cdef, cur, pic_bytes, cudaMemcpyDeviceToDevice, st);
       }), "LR snapshot");
  }
  if (P.use_lr) {
    LrArgs lr = P.lr;
    for (int p = 0; p < 3; ++p) lr.units[p] = reinterpret_cast<const LrUnitRec*>(ar + pl->o_lr[p]);
    /* with superres the restoration's source is the upscaled picture, not
     * the picture's own content: tiles it does not restore pass through */
    CK(timed(d, kStLr, [&] { return launch_lr(lr_cdef, lr_curr, cur, L, lr, maxv, P.upscaled, st); }),
       "loop restoration");
    ++launches;
  }
  if (keep)
    CK(timed(d, kStCopy, [&] {
         return cudaMemcpyAsync(d->slot_buf[slot].p, cur, pic_bytes, cudaMemcpyDeviceToDevice, st);
       }), "reference store");
  const px_t* display = cur;
  d->disp_is_cur = true;
  d->disp_pending = false;
  if (P.grain) {
    GrainState* gsd = static_cast<GrainState*>(d->grain_state.p);
    CK(cudaStreamWaitEvent(st, d->ev_join, 0), "join wait");
    if (sp->defer_grain) {
      d->disp_pending = true;
    } else {
      CK(timed(d, kStGrainBlend, [&] {
           return launch_grain_blend(cur, static_cast<px_t*>(d->disp.p), L, gsd,
                                     static_cast<const uint16_t*>(d->orbit.p),
                                     static_cast<const uint16_t*>(d->pos.p), st);
         }), "film grain blend");
      launches += 1;
    }
    display = static_cast<px_t*>(d->disp.p);
    d->disp_is_cur = false;
  }
  CK(cudaEventRecord(ev[2], st), "event");
  sp->launches = launches;
  return AV1B_OK;
}

/* After the launches of a frame step: the read back into `out`, the status
 * word's copy, the stats, the plan's done event and the slot bookkeeping, on
 * the decoder's stream - which first waits for `after` when the step ran on
 * another stream (a batched step). Called with the decoder's lock held. */
int commit_step(av1b_decoder* d, av1b_plan* pl, StepPrep* sp, const av1b_planes* out, int* out_slot,
                bool sync, cudaStream_t batch_stream) {
  const Layout& L = d->L;
  /* a batched step's status copy and plan event go on the batch's stream */
  cudaStream_t st = batch_stream ? batch_stream : d->stream;
  const FrameArgs& a = sp->a;
  const int keep = sp->keep, slot = sp->slot;
  const int launches = sp->launches;
  const px_t* display = d->disp_is_cur ? static_cast<const px_t*>(d->cur.p)
                                       : static_cast<const px_t*>(d->disp.p);

  /* ---- read back ---------------------------------------------------------------------------- */
  if (out) {
    for (int p = 0; p < 3; ++p) {
      const PlaneGeom& g = L.p[p];
      if (!out->plane[p] || out->stride[p] < g.out_w)
        return fail(d, AV1B_ERR_ARG, "output plane missing or too narrow");
      CK(cudaMemcpy2DAsync(out->plane[p], static_cast<size_t>(out->stride[p]) * sizeof(px_t),
                           display + g.off, static_cast<size_t>(g.stride) * sizeof(px_t),
                           static_cast<size_t>(g.out_w) * sizeof(px_t), g.out_h,
                           cudaMemcpyDeviceToHost, st), "read back");
    }
  }
  CK(cudaMemcpyAsync(d->status_host, a.status, sizeof(int), cudaMemcpyDeviceToHost, st), "status read");
  d->stats.blocks = pl->n_blocks;
  d->stats.waves = 0;
  d->stats.kernel_launches = launches;
  d->stats_pending = launches > 0;   /* a batched step times itself */
  CK(cudaEventRecord(pl->done, st), "event");
  pl->in_flight = true;
  if (batch_stream) {
    if (!d->ev_after_batch)
      CK(cudaEventCreateWithFlags(&d->ev_after_batch, cudaEventDisableTiming), "event");
    CK(cudaEventRecord(d->ev_after_batch, batch_stream), "event");
    d->batch_pending = true;
  }
  if (keep) {
    std::lock_guard<std::mutex> lk(d->slot_mu);
    d->slot_used[slot] = true;
    d->slot_valid[slot] = true;
    d->slot_width[slot] = pl->width;
    d->slot_height[slot] = pl->height;
    d->slot_bd[slot] = pl->bit_depth;
  }
  d->last_slot = slot;
  d->have_last = true;
  if (out_slot) *out_slot = slot;
  if (sync) return finish_frame(d);
  return AV1B_OK;
}

int execute_plan(av1b_decoder* d, av1b_plan* pl, int keep, int forced_slot, const av1b_planes* out,
                 int* out_slot, bool sync) {
  StepPrep sp;
  sp.defer_grain = out == nullptr;
  int rc;
  join_batch(d);
  if ((rc = prepare_step(d, pl, keep, forced_slot, false, &sp, d->stream)) ||
      (rc = launch_step_plain(d, pl, &sp)))
    return rc;
  return commit_step(d, pl, &sp, out, out_slot, sync, nullptr);
}

/* Frees a plan's buffers and events once no frame reads it any more. */
void release_plan(av1b_decoder* d, av1b_plan* pl) {
  if (pl->in_flight) cudaEventSynchronize(pl->done);
  dev_release(d, pl->arena);
  dev_release(d, pl->coef);
  dev_release(d, pl->residual);
  dev_release(d, pl->dqsrc);
  dev_release(d, pl->filt);
  if (pl->prep_host) cudaFreeHost(pl->prep_host);
  if (pl->ready) cudaEventDestroy(pl->ready);
  if (pl->done) cudaEventDestroy(pl->done);
  delete pl;
}

/* Returns a plan to the decoder's pool (its buffers stay allocated for the
 * next plan), or frees it when the pool is full. */
void recycle_plan(av1b_decoder* d, av1b_plan* pl) {
  {
    std::lock_guard<std::mutex> lk(d->plan_pool_mu);
    if (d->plan_pool.size() < 8) {
      d->plan_pool.push_back(pl);
      return;
    }
  }
  release_plan(d, pl);
}

/* Waits for the frame in flight and checks its status word. */
int finish_frame(av1b_decoder* d) {
  CK(wait_stream(d), "frame sync");
  collect_profile(d);
  if (d->stats_pending) {
    float ms_recon = 0, ms_filter = 0;
    cudaEventElapsedTime(&ms_recon, d->ev[0], d->ev[1]);
    cudaEventElapsedTime(&ms_filter, d->ev[1], d->ev[2]);
    d->stats.reconstruct_ms = ms_recon;
    d->stats.filter_ms = ms_filter;
    d->stats.readback_ms = 0;
    d->stats.total_ms = ms_recon + ms_filter;
    d->stats_pending = false;
  }
  if (*d->status_host & AV1B_STATUS_TIMEOUT) {
    *d->status_host = 0;
    CK(cudaMemset(static_cast<uint8_t*>(d->status_q.p) + 64, 0, sizeof(int)), "status clear");
    return fail(d, AV1B_ERR_TIMEOUT, "a device-side dependency wait timed out");
  }
  return AV1B_OK;
}

int run_frame(av1b_decoder* d, const av1b_frame_syntax& s, int keep, int forced_slot,
              const av1b_planes* out, int* out_slot) {
  int rc = plan_frame(d, s, d->own_plan);
  if (rc) return rc;
  return execute_plan(d, d->own_plan, keep, forced_slot, out, out_slot, true);
}

/* The picture an output call of `slot` reads: the display picture of the
 * frame decoded last for its slot (or a negative slot), else the stored one. */
int picture_of(av1b_decoder* d, int slot, const px_t** pic) {
  if (slot < 0 || slot == d->last_slot) {
    if (!d->have_last) return fail(d, AV1B_ERR_ARG, "no frame to convert");
    if (d->disp_pending) {
      /* the output picture of a frame whose grain a batched step applied
       * inside its NV12 pack: the blend from the frame's own grain state */
      CK(launch_grain_blend(static_cast<const px_t*>(d->cur.p), static_cast<px_t*>(d->disp.p), d->L,
                            static_cast<const GrainState*>(d->grain_state.p),
                            static_cast<const uint16_t*>(d->orbit.p),
                            static_cast<const uint16_t*>(d->pos.p), d->stream),
         "film grain blend");
      d->disp_pending = false;
    }
    *pic = d->disp_is_cur ? static_cast<const px_t*>(d->cur.p) : static_cast<const px_t*>(d->disp.p);
    return AV1B_OK;
  }
  if (slot >= kSlots || !d->slot_used[slot] || !d->slot_valid[slot])
    return fail(d, AV1B_ERR_ARG, "invalid reference slot");
  *pic = static_cast<const px_t*>(d->slot_buf[slot].p);
  return AV1B_OK;
}

void copy_error(const av1b_decoder* d, char* error, size_t len) {
  if (!error || !len) return;
  std::lock_guard<std::mutex> lk(const_cast<av1b_decoder*>(d)->err_mu);
  std::snprintf(error, len, "%s", d->err.c_str());
}

}  // namespace
}  // namespace av1b

/* ---- C ABI ---------------------------------------------------------------------------------------- */
extern "C" {

int av1b_decoder_create(int device, size_t hbm_budget_bytes, av1b_decoder** out) {
  return av1b_decoder_create_ex(device, hbm_budget_bytes, nullptr, out);
}

int av1b_decoder_create_ex(int device, size_t hbm_budget_bytes, const av1b_decoder_options* opt,
                           av1b_decoder** out) {
  if (!out) return AV1B_ERR_ARG;
  if (opt && (opt->planners < 0 || opt->planners > 8 || opt->planner_threads < 0 ||
              opt->planner_threads > 64))
    return AV1B_ERR_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return AV1B_ERR_NO_DEVICE;
  if (device < 0 || device >= n) return AV1B_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return AV1B_ERR_CUDA;
  auto* d = new av1b_decoder;
  d->device = device;
  d->budget = hbm_budget_bytes;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) d->n_sm = prop.multiProcessorCount;
  bool ok = cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) == cudaSuccess &&
            set_kernel_attributes() == cudaSuccess &&
            cudaHostAlloc(reinterpret_cast<void**>(&d->status_host), 64, cudaHostAllocDefault) == cudaSuccess;
  for (int i = 0; ok && i < 3; ++i) ok = cudaEventCreate(&d->ev[i]) == cudaSuccess;
  ok = ok && cudaStreamCreateWithFlags(&d->aux, cudaStreamNonBlocking) == cudaSuccess &&
       cudaEventCreateWithFlags(&d->ev_fork, cudaEventDisableTiming) == cudaSuccess &&
       cudaEventCreateWithFlags(&d->ev_join, cudaEventDisableTiming) == cudaSuccess &&
       cudaEventCreateWithFlags(&d->ev_block, cudaEventDisableTiming | cudaEventBlockingSync) ==
           cudaSuccess;
  if (!ok) {
    av1b_decoder_destroy(d);
    return AV1B_ERR_CUDA;
  }
  *d->status_host = 0;
  {
    /* three planners: one plan at a time uses all cores but the one left to
     * the thread that drives the device; plans at once share them (a key
     * frame's plan takes several inter frames' time, and the other planners
     * keep the device fed meanwhile) */
    const unsigned hc = std::thread::hardware_concurrency();
#ifdef AV1B_PLANNER_THREADS
    int threads = AV1B_PLANNER_THREADS;
    (void)hc;
#else
    int threads = static_cast<int>(std::min(16u, std::max(2u, hc) - 1));
#endif
#ifndef AV1B_PLANNERS
#define AV1B_PLANNERS 3
#endif
    int planners = AV1B_PLANNERS;
    if (opt && opt->planner_threads > 0) threads = opt->planner_threads;
    if (opt && opt->planners > 0) planners = opt->planners;
    d->planners.resize(planners);
    /* the planners' uploads and record conversions at the highest stream
     * priority: a plan waits for them, and on a busy GPU (a batched step's
     * persistent kernels) their few CTAs then go first */
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    for (auto& q : d->planners) {
      q.pool = new WorkPool(threads);
      q.scratch = new PlanScratch;
      q.lists = new PlanLists;
      if (cudaStreamCreateWithPriority(&q.upload, cudaStreamNonBlocking, prio_hi) != cudaSuccess) {
        av1b_decoder_destroy(d);
        return AV1B_ERR_CUDA;
      }
    }
  }
  d->own_plan = new av1b_plan;
  d->own_plan->owned_by_decoder = true;
  *out = d;
  return AV1B_OK;
}

int av1b_decoder_destroy(av1b_decoder* d) {
  if (!d) return AV1B_ERR_ARG;
  cudaSetDevice(d->device);
  if (d->stream) {
    join_batch(d);
    cudaStreamSynchronize(d->stream);
  }
  if (d->own_plan) release_plan(d, d->own_plan);
  for (av1b_plan* pl : d->plan_pool) release_plan(d, pl);
  d->plan_pool.clear();
  for (auto& q : d->planners) {
    if (q.upload) {
      cudaStreamSynchronize(q.upload);
      cudaStreamDestroy(q.upload);
    }
    delete q.pool;
    delete q.scratch;
    delete q.lists;
  }
  d->planners.clear();
  for (int i = 0; i < 3; ++i)
    if (d->ev[i]) cudaEventDestroy(d->ev[i]);
  if (d->aux) {
    cudaStreamSynchronize(d->aux);
    cudaStreamDestroy(d->aux);
  }
  if (d->ev_fork) cudaEventDestroy(d->ev_fork);
  if (d->ev_join) cudaEventDestroy(d->ev_join);
  if (d->ev_block) cudaEventDestroy(d->ev_block);
  if (d->ev_batch) cudaEventDestroy(d->ev_batch);
  if (d->ev_after_batch) cudaEventDestroy(d->ev_after_batch);
  if (d->status_host) cudaFreeHost(d->status_host);
  for (auto& k : d->packs) {
    if (k.copied) cudaEventSynchronize(k.copied);
    if (k.host) cudaFreeHost(k.host);
    if (k.packed) cudaEventDestroy(k.packed);
    if (k.copied) cudaEventDestroy(k.copied);
    dev_release(d, k.dev);
  }
  d->packs.clear();
  if (d->copy_stream) cudaStreamDestroy(d->copy_stream);
  DevBuf* bufs[] = {&d->cur, &d->snap, &d->lr_pre_up, &d->lr_cdef, &d->disp,
                    &d->slot_ptr_dev, &d->arena, &d->coef, &d->residual, &d->done,
                    &d->status_q, &d->nv12, &d->rgb,
                    &d->grain_state, &d->orbit, &d->pos, &d->cdef_search, &d->pre_res, &d->mask_pool,
                    &d->trace};
  for (DevBuf* b : bufs) dev_release(d, *b);
  for (int i = 0; i < kSlots; ++i) dev_release(d, d->slot_buf[i]);
  if (d->stream) cudaStreamDestroy(d->stream);
  delete d;
  return AV1B_OK;
}

int av1b_decoder_reset(av1b_decoder* d) {
  if (!d) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(d->mu);
  join_batch(d);
  std::lock_guard<std::mutex> slk(d->slot_mu);
  for (int i = 0; i < kSlots; ++i) {
    d->slot_used[i] = false;
    d->slot_valid[i] = false;
  }
  d->last_slot = -1;
  d->have_last = false;
  d->stats = av1b_stats{};
  return AV1B_OK;
}

int av1b_decode(av1b_decoder* d, const av1b_frame_syntax* syntax, int keep_reference,
                const av1b_planes* out, int* out_slot, char* error, size_t error_len) {
  if (!d || !syntax) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->device);
  if (out_slot) *out_slot = -1;
  clear_err(d);
  const int rc = run_frame(d, *syntax, keep_reference ? 1 : 0, -1, out, out_slot);
  if (rc) copy_error(d, error, error_len);
  return rc;
}

int av1b_decode_blob(av1b_decoder* d, const uint8_t* blob, size_t len, int keep_reference,
                     const av1b_planes* out, int* out_slot, char* error, size_t error_len) {
  av1b_frame_syntax v;
  if (!d) return AV1B_ERR_ARG;
  if (!view_blob(blob, len, &v)) {
    fail(d, AV1B_ERR_ARG, "malformed serialized frame");
    copy_error(d, error, error_len);
    return AV1B_ERR_ARG;
  }
  return av1b_decode(d, &v, keep_reference, out, out_slot, error, error_len);
}

/* Planning takes no decoder lock: it may run on its own thread while frames
 * decode (see plan_frame). */
int av1b_plan_frame(av1b_decoder* d, const av1b_frame_syntax* syntax, av1b_plan** out) {
  if (!d || !syntax || !out) return AV1B_ERR_ARG;
  cudaSetDevice(d->device);
  *out = nullptr;
  av1b_plan* pl = nullptr;
  {
    std::lock_guard<std::mutex> lk(d->plan_pool_mu);
    if (!d->plan_pool.empty()) {
      pl = d->plan_pool.back();
      d->plan_pool.pop_back();
    }
  }
  if (!pl) pl = new av1b_plan;
  const int rc = plan_frame(d, *syntax, pl);
  if (rc) {
    recycle_plan(d, pl);
    return rc;
  }
  *out = pl;
  return AV1B_OK;
}

int av1b_plan_free(av1b_decoder* d, av1b_plan* pl) {
  if (!d) return AV1B_ERR_ARG;
  if (!pl) return AV1B_OK;
  cudaSetDevice(d->device);
  recycle_plan(d, pl);
  return AV1B_OK;
}

int av1b_decode_planned(av1b_decoder* d, av1b_plan* pl, int slot, int keep_reference,
                        const av1b_planes* out, int* out_slot, int wait) {
  if (!d || !pl) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->device);
  clear_err(d);
  if (out_slot) *out_slot = -1;
  return execute_plan(d, pl, keep_reference ? 1 : 0, slot, out, out_slot, wait != 0);
}

int av1b_plan_stats(const av1b_plan* pl, av1b_plan_info* out) {
  if (!pl || !out) return AV1B_ERR_ARG;
  const Plan& P = pl->P;
  std::memset(out, 0, sizeof(*out));
  out->width = pl->width;
  out->height = pl->height;
  out->coded_width = pl->coded_width;
  out->bit_depth = pl->bit_depth;
  out->blocks = static_cast<int64_t>(P.n_blocks);
  out->phase_b_blocks = static_cast<int64_t>(P.n_units);
  out->chains = static_cast<int64_t>(P.n_chains);
  out->depth = P.unit_depth;
  out->phase_b_samples = static_cast<int64_t>(P.unit_samples);
  out->inter_tiles = static_cast<int64_t>(P.n_tiles);
  out->inter_samples = static_cast<int64_t>(P.inter_samples);
  out->inter_ref_samples = static_cast<int64_t>(P.inter_ref_samples);
  out->transforms = static_cast<int64_t>(P.n_itx);
  out->tx_samples = static_cast<int64_t>(P.tx_samples);
  out->coef_samples = static_cast<int64_t>(P.coef_samples);
  out->deblock_edges[0] = static_cast<int64_t>(P.n_dbv);
  out->deblock_edges[1] = static_cast<int64_t>(P.n_dbh);
  out->cdef_blocks = static_cast<int64_t>(P.n_cdef);
  for (int p = 0; p < 3; ++p) out->lr_units += P.lr.type[p] ? P.lr.n_units[p] : 0;
  out->upscaled = P.upscaled ? 1 : 0;
  out->restored = P.use_lr ? 1 : 0;
  out->grain = P.grain ? 1 : 0;
  return AV1B_OK;
}

size_t av1b_stream_hbm_estimate(int width, int height, int coded_width, int bit_depth, int ss_x,
                                 int ss_y, int n_slots, int plans) {
  if (width <= 0 || height <= 0 || n_slots < 0 || plans < 0) return 0;
  const Layout L = make_layout(width, height, coded_width > 0 ? coded_width : width, bit_depth, ss_x,
                               ss_y);
  const size_t pic = static_cast<size_t>(L.size) * sizeof(px_t);
  const int cw = coded_width > 0 ? coded_width : width;
  const size_t nc = static_cast<size_t>(cw) * height +
                    2 * static_cast<size_t>((cw + ss_x) >> ss_x) * ((height + ss_y) >> ss_y);
  /* every buffer as dev_ensure sizes it: an eighth of room, 64 KB granules */
  auto rounded = [](size_t b) { return align_up(b + b / 8, size_t(1) << 16); };
  /* pictures: the one reconstructed, the snapshot, the display picture, the
   * two loop restoration sources, and the reference slots; per sample: the
   * phase B residuals (4 B), the done flags (128 B a block, blocks of 16
   * samples or more) and the difference-weighted luma masks (1 B); per plan:
   * its five buffers - records, coefficient pool, residuals, levels, filter
   * lists - at most 10 B a coded sample in all; the grain tables and small
   * buffers, 2 MB */
  return (5 + static_cast<size_t>(n_slots)) * rounded(pic) + rounded(4 * nc) + rounded(8 * nc) +
         rounded(nc) + static_cast<size_t>(plans) * (5 * (size_t(1) << 16) + rounded(10 * nc)) +
         (size_t(2) << 20);
}

int av1b_decoder_memory(av1b_decoder* d, size_t* allocated, size_t* budget) {
  if (!d) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(d->alloc_mu);
  if (allocated) *allocated = d->allocated;
  if (budget) *budget = d->budget;
  return AV1B_OK;
}

int av1b_sync(av1b_decoder* d) {
  if (!d) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(d->mu);
  join_batch(d);
  cudaSetDevice(d->device);
  return finish_frame(d);
}

int av1b_reserve_reference(av1b_decoder* d, int* out_slot) {
  if (!d || !out_slot) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(d->mu);
  *out_slot = -1;
  std::lock_guard<std::mutex> slk(d->slot_mu);
  for (int i = 0; i < kSlots; ++i)
    if (!d->slot_used[i]) {
      d->slot_used[i] = true;
      d->slot_valid[i] = false;
      *out_slot = i;
      return AV1B_OK;
    }
  return AV1B_ERR_NOMEM;
}

int av1b_decode_reserved(av1b_decoder* d, const av1b_frame_syntax* syntax, int slot,
                         const av1b_planes* out, char* error, size_t error_len) {
  if (!d || !syntax) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(d->mu);
  cudaSetDevice(d->device);
  clear_err(d);
  int got = -1;
  const int rc = run_frame(d, *syntax, slot >= 0 ? 1 : 0, slot, out, &got);
  if (rc) copy_error(d, error, error_len);
  return rc;
}

int av1b_release_reference(av1b_decoder* d, int slot) {
  if (!d) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(d->mu);
  std::lock_guard<std::mutex> slk(d->slot_mu);
  if (slot >= 0 && slot < kSlots) {
    d->slot_used[slot] = false;
    d->slot_valid[slot] = false;
  }
  return AV1B_OK;
}

size_t av1b_nv12_size(int width, int height, int ss_x, int ss_y, size_t pitch) {
  return nv12_bytes(width, height, ss_x, ss_y, pitch);
}

/* Packs `slot` as NV12 into device memory on the decoder's stream: the
 * frame decoded last whose grain is still to be applied goes through the
 * pack that applies it; any other picture through the plain pack. */
int launch_pack(av1b_decoder* d, int slot, uint8_t* target, size_t pitch) {
  if ((slot < 0 || slot == d->last_slot) && d->have_last && d->disp_pending) {
    CK(timed(d, kStNv12, [&] {
         return launch_nv12_grain(static_cast<const px_t*>(d->cur.p), target, d->L,
                                  static_cast<int>(pitch),
                                  static_cast<const GrainState*>(d->grain_state.p),
                                  static_cast<const uint16_t*>(d->orbit.p),
                                  static_cast<const uint16_t*>(d->pos.p), d->stream);
       }), "NV12 pack with film grain");
    return AV1B_OK;
  }
  const px_t* pic = nullptr;
  const int rc = picture_of(d, slot, &pic);
  if (rc) return rc;
  CK(timed(d, kStNv12, [&] { return launch_nv12(pic, target, d->L, static_cast<int>(pitch), d->stream); }),
     "NV12 pack");
  return AV1B_OK;
}

static int to_nv12_impl(av1b_decoder* d, int slot, size_t pitch, uint8_t* dst, size_t dst_len,
                        bool device_dst) {
  if (!d || !dst) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(d->mu);
  join_batch(d);
  cudaSetDevice(d->device);
  int rc;
  {
    /* the slot check of picture_of, before any buffer is sized */
    const bool last = slot < 0 || slot == d->last_slot;
    if (last ? !d->have_last : (slot >= kSlots || !d->slot_used[slot] || !d->slot_valid[slot]))
      return fail(d, AV1B_ERR_ARG, last ? "no frame to convert" : "invalid reference slot");
  }
  const size_t bytes = nv12_bytes(d->width, d->height, d->ss_x, d->ss_y, pitch);
  if (bytes == 0 || pitch > (1u << 30))
    return fail(d, AV1B_ERR_ARG, "NV12 output needs a 4:2:0 frame and an even pitch at least as wide");
  if (dst_len < bytes) return fail(d, AV1B_ERR_ARG, "NV12 destination too small");
  uint8_t* target = dst;
  if (!device_dst) {
    if ((rc = dev_ensure(d, d->nv12, bytes))) return rc;
    target = static_cast<uint8_t*>(d->nv12.p);
  }
  if ((rc = launch_pack(d, slot, target, pitch))) return rc;
  if (!device_dst) {
    CK(cudaMemcpyAsync(dst, target, bytes, cudaMemcpyDeviceToHost, d->stream), "NV12 read back");
    CK(wait_stream(d), "NV12 sync");
    collect_profile(d);
  }
  /* the device variant stays queued on the decoder's stream */
  return AV1B_OK;
}

int av1b_to_nv12(av1b_decoder* d, int slot, size_t pitch, uint8_t* dst, size_t dst_len) {
  return to_nv12_impl(d, slot, pitch, dst, dst_len, false);
}

int av1b_to_nv12_device(av1b_decoder* d, int slot, size_t pitch, void* dst_device, size_t dst_len) {
  return to_nv12_impl(d, slot, pitch, static_cast<uint8_t*>(dst_device), dst_len, true);
}

/* The split pack. Up to eight packs are outstanding at once: a caller that
 * holds more gets AV1B_ERR_NOMEM until it releases one. */
constexpr int kMaxPacks = 8;

int av1b_nv12_pack_begin(av1b_decoder* d, int slot, size_t pitch, int* out_handle) {
  if (!d || !out_handle) return AV1B_ERR_ARG;
  *out_handle = -1;
  std::lock_guard<std::mutex> lk(d->mu);
  join_batch(d);
  cudaSetDevice(d->device);
  int rc;
  {
    /* the slot check of picture_of, without making a pending display picture */
    const bool last = slot < 0 || slot == d->last_slot;
    if (last ? !d->have_last : (slot >= kSlots || !d->slot_used[slot] || !d->slot_valid[slot]))
      return fail(d, AV1B_ERR_ARG, last ? "no frame to convert" : "invalid reference slot");
  }
  const size_t bytes = nv12_bytes(d->width, d->height, d->ss_x, d->ss_y, pitch);
  if (bytes == 0 || pitch > (1u << 30))
    return fail(d, AV1B_ERR_ARG, "NV12 output needs a 4:2:0 frame and an even pitch at least as wide");
  std::lock_guard<std::mutex> pk(d->pack_mu);
  if (!d->copy_stream)
    CK(cudaStreamCreateWithFlags(&d->copy_stream, cudaStreamNonBlocking), "copy stream");
  av1b_decoder::Pack* e = nullptr;
  for (auto& k : d->packs)
    if (k.handle < 0) {
      e = &k;
      break;
    }
  if (!e) {
    if (d->packs.size() >= static_cast<size_t>(kMaxPacks))
      return fail(d, AV1B_ERR_NOMEM, "every NV12 pack entry is in use; release one first");
    if (d->packs.empty()) d->packs.reserve(kMaxPacks);
    d->packs.emplace_back();
    e = &d->packs.back();
    CK(cudaEventCreateWithFlags(&e->packed, cudaEventDisableTiming), "event");
    CK(cudaEventCreateWithFlags(&e->copied, cudaEventDisableTiming | cudaEventBlockingSync), "event");
  }
  if ((rc = dev_ensure(d, e->dev, bytes))) return rc;
  if (e->host_cap < bytes) {
    if (e->host) cudaFreeHost(e->host);
    e->host = nullptr;
    e->host_cap = 0;
    CK(cudaHostAlloc(reinterpret_cast<void**>(&e->host), bytes, cudaHostAllocDefault),
       "page-locked NV12 buffer");
    e->host_cap = bytes;
  }
  uint8_t* dev = static_cast<uint8_t*>(e->dev.p);
  if ((rc = launch_pack(d, slot, dev, pitch))) return rc;
  CK(cudaEventRecord(e->packed, d->stream), "event");
  CK(cudaStreamWaitEvent(d->copy_stream, e->packed, 0), "copy stream wait");
  CK(cudaMemcpyAsync(e->host, dev, bytes, cudaMemcpyDeviceToHost, d->copy_stream), "NV12 read back");
  CK(cudaEventRecord(e->copied, d->copy_stream), "event");
  e->bytes = bytes;
  e->handle = d->next_pack = (d->next_pack + 1) & 0x3fffffff;
  *out_handle = e->handle;
  return AV1B_OK;
}

int av1b_nv12_pack_wait(av1b_decoder* d, int handle, uint8_t* dst, size_t dst_len,
                        const uint8_t** data, size_t* bytes) {
  if (!d || handle < 0) return AV1B_ERR_ARG;
  cudaEvent_t ev = nullptr;
  const uint8_t* host = nullptr;
  size_t n = 0;
  {
    std::lock_guard<std::mutex> pk(d->pack_mu);
    for (auto& k : d->packs)
      if (k.handle == handle) {
        ev = k.copied;
        host = k.host;
        n = k.bytes;
      }
  }
  if (!ev) return fail(d, AV1B_ERR_ARG, "unknown NV12 pack handle");
  if (dst && dst_len < n) return fail(d, AV1B_ERR_ARG, "NV12 destination too small");
  cudaSetDevice(d->device);
  CK(cudaEventSynchronize(ev), "NV12 pack wait");
  /* the entry stays ours until release: its bytes do not change */
  if (dst) std::memcpy(dst, host, n);
  if (data) *data = host;
  if (bytes) *bytes = n;
  return AV1B_OK;
}

int av1b_nv12_pack_release(av1b_decoder* d, int handle) {
  if (!d || handle < 0) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> pk(d->pack_mu);
  for (auto& k : d->packs)
    if (k.handle == handle) {
      /* a pack released unwaited still finishes before its buffers are reused */
      cudaSetDevice(d->device);
      cudaEventSynchronize(k.copied);
      k.handle = -1;
      return AV1B_OK;
    }
  return fail(d, AV1B_ERR_ARG, "unknown NV12 pack handle");
}

int av1b_to_rgb(av1b_decoder* d, int slot, int matrix, int range, uint8_t* dst, size_t dst_len) {
  if (!d || !dst) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(d->mu);
  join_batch(d);
  cudaSetDevice(d->device);
  const px_t* pic = nullptr;
  int rc = picture_of(d, slot, &pic);
  if (rc) return rc;
  const size_t bytes = static_cast<size_t>(d->width) * d->height * 3;
  if (dst_len < bytes) return fail(d, AV1B_ERR_ARG, "RGB destination too small");
  if ((rc = dev_ensure(d, d->rgb, bytes))) return rc;
  RgbArgs m{};
  color_matrix(matrix, range, d->bit_depth, m.m, m.o);
  CK(timed(d, kStRgb, [&] { return launch_rgb(pic, static_cast<uint8_t*>(d->rgb.p), d->L, m, d->stream); }),
     "RGB pack");
  CK(cudaMemcpyAsync(dst, d->rgb.p, bytes, cudaMemcpyDeviceToHost, d->stream), "RGB read back");
  CK(wait_stream(d), "RGB sync");
  collect_profile(d);
  return AV1B_OK;
}

int av1b_get_stats(av1b_decoder* d, av1b_stats* out) {
  if (!d || !out) return AV1B_ERR_ARG;
  *out = d->stats;
  return AV1B_OK;
}

int av1b_poll_status(av1b_decoder* d, int* status) {
  if (!d || !status) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(d->mu);
  join_batch(d);
  cudaSetDevice(d->device);
  /* the status word of the frames whose work has finished: its copy into
   * page-locked memory is queued after each frame */
  const cudaError_t q = cudaStreamQuery(d->stream);
  if (q != cudaSuccess && q != cudaErrorNotReady) return cuda_fail(d, q, "status poll");
  *status = *static_cast<volatile int*>(d->status_host);
  if (q == cudaSuccess && *status) {
    *d->status_host = 0;
    CK(cudaMemsetAsync(static_cast<uint8_t*>(d->status_q.p) + 64, 0, sizeof(int), d->stream), "status clear");
  }
  return AV1B_OK;
}

int av1b_slot_planes_device(av1b_decoder* d, int slot, uint16_t* plane_ptr[3], int32_t stride[3]) {
  if (!d || !plane_ptr || !stride) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(d->mu);
  join_batch(d);
  const px_t* pic = nullptr;
  const int rc = picture_of(d, slot, &pic);
  if (rc) return rc;
  for (int p = 0; p < 3; ++p) {
    plane_ptr[p] = const_cast<px_t*>(pic) + d->L.p[p].off;
    stride[p] = d->L.p[p].stride;
  }
  return AV1B_OK;
}

void* av1b_decoder_stream(av1b_decoder* d) { return d ? d->stream : nullptr; }

int av1b_set_wait_limit(av1b_decoder* d, long long limit_ns) {
  if (!d || limit_ns <= 0) return AV1B_ERR_ARG;
  d->wait_ns = static_cast<unsigned long long>(limit_ns);
  return AV1B_OK;
}

int av1b_selftest_wait(av1b_decoder* d, long long limit_ns, int* status, double* elapsed_ms) {
  if (!d || !status || limit_ns <= 0 || limit_ns > 10000000000LL) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(d->mu);
  join_batch(d);
  cudaSetDevice(d->device);
  DevBuf mem;
  int rc = dev_ensure(d, mem, 256);
  if (rc) return rc;
  CK(cudaMemsetAsync(mem.p, 0, 256, d->stream), "selftest reset");
  CK(cudaEventRecord(d->ev[0], d->stream), "event");
  CK(launch_selftest_wait(static_cast<const unsigned*>(mem.p),
                          reinterpret_cast<int*>(static_cast<uint8_t*>(mem.p) + 64),
                          static_cast<unsigned long long>(limit_ns), d->stream), "selftest launch");
  CK(cudaEventRecord(d->ev[1], d->stream), "event");
  int st = 0;
  CK(cudaMemcpyAsync(&st, static_cast<uint8_t*>(mem.p) + 64, sizeof(int), cudaMemcpyDeviceToHost,
                     d->stream), "selftest status");
  CK(cudaStreamSynchronize(d->stream), "selftest sync");
  float ms = 0;
  cudaEventElapsedTime(&ms, d->ev[0], d->ev[1]);
  dev_release(d, mem);
  *status = st;
  if (elapsed_ms) *elapsed_ms = ms;
  return AV1B_OK;
}

int av1b_set_shared_masks(av1b_decoder* d, int on) {
  if (!d) return AV1B_ERR_ARG;
  d->share_masks.store(on != 0);
  return AV1B_OK;
}

int av1b_set_unit_trace(av1b_decoder* d, int on) {
  if (!d) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(d->mu);
  d->tracing = on != 0;
  d->trace_n = 0;
  return AV1B_OK;
}

int av1b_unit_trace(av1b_decoder* d, uint64_t* out, size_t cap, size_t* n) {
  if (!d || !n) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(d->mu);
  join_batch(d);
  cudaSetDevice(d->device);
  *n = d->trace_n;
  if (!out || d->trace_n == 0) return AV1B_OK;
  if (cap < d->trace_n) return fail(d, AV1B_ERR_ARG, "trace buffer too small");
  CK(cudaStreamSynchronize(d->stream), "trace sync");
  CK(cudaMemcpy(out, d->trace.p, d->trace_n * sizeof(uint64_t), cudaMemcpyDeviceToHost), "trace read");
  return AV1B_OK;
}

int av1b_set_profiling(av1b_decoder* d, int on) {
  if (!d) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(d->mu);
  d->profiling = on != 0;
  for (int i = 0; i < kStageCount; ++i) {
    d->prof_ms[i] = 0;
    d->prof_n[i] = 0;
  }
  return AV1B_OK;
}

int av1b_profile(av1b_decoder* d, int stage, const char** name, double* total_ms, long long* count) {
  if (!d || stage < 0) return AV1B_ERR_ARG;
  if (stage >= kStageCount) return 0;
  if (name) *name = kStageNames[stage];
  if (total_ms) *total_ms = d->prof_ms[stage];
  if (count) *count = d->prof_n[stage];
  return 1;
}

const char* av1b_last_error(av1b_decoder* d) { return d ? d->err.c_str() : ""; }

}  // extern "C"

/* ---- batched form: many streams' frames in one step -------------------------------------- */
#include "batch_runtime.cuh"
