/*
 * batch_runtime.cuh - the batched form's host runtime: one frame of each of
 * many independent streams (each an av1b_decoder with its own reference
 * slots, pictures and planners) decoded as one step by the persistent stage
 * kernels of batch_kernels.cuh, replayed as a CUDA graph; and the autotuner
 * that picks the step's launch shape. Part of decoder.cu's translation unit
 * (included at its end): a step prepares every stream's frame with the same
 * code as a single-stream decode (prepare_step / commit_step).
 *
 * The reference decodes one stream per Decoder and captures its frame step
 * as a graph (src/backends/cuda/cuda_backend.cpp:1212-1227); it has no form
 * that decodes several streams in one launch.
 */

namespace av1b {
namespace {

/* The filter chain of a prepared frame step, for the batched kernels: the
 * same buffers, in the same order, as launch_step_plain uses. */
int fill_filter_args(av1b_decoder* d, av1b_plan* pl, StepPrep* sp) {
  const Plan& P = pl->P;
  const Layout& L = d->L;
  FilterArgs& f = sp->f;
  f = FilterArgs{};
  const size_t pic_bytes = static_cast<size_t>(L.size) * sizeof(px_t);
  const uint8_t* ar = static_cast<const uint8_t*>(pl->arena.p);
  const uint8_t* fl = static_cast<const uint8_t*>(pl->filt.p);
  px_t* cur = static_cast<px_t*>(d->cur.p);
  px_t* snap = static_cast<px_t*>(d->snap.p);
  px_t* lr_cdef = static_cast<px_t*>(d->lr_cdef.p);
  px_t* lr_pre_up = static_cast<px_t*>(d->lr_pre_up.p);
  f.bd = pl->bit_depth;
  f.maxv = (1 << pl->bit_depth) - 1;
  f.sharpness = pl->sharpness;
  f.dbv = reinterpret_cast<const DeblockRec*>(fl + pl->o_dbv);
  f.dbh = reinterpret_cast<const DeblockRec*>(fl + pl->o_dbh);
  f.n_dbv = static_cast<int>(P.n_dbv);
  f.n_dbh = static_cast<int>(P.n_dbh);
  auto set_copy = [&](int k, const px_t* src, px_t* dst) {
    f.copy_src[k] = src;
    f.copy_dst[k] = dst;
    f.copy_bytes[k] = static_cast<long long>(pic_bytes);
    f.copy_items[k] = static_cast<long long>((pic_bytes + AV1B_COPY_ITEM - 1) / AV1B_COPY_ITEM);
  };
  if (P.n_cdef != 0 || P.use_lr) set_copy(0, cur, snap);
  if (P.n_cdef != 0) {
    f.cdef_src = snap;
    f.cdef_dst = cur;
    f.cdef = reinterpret_cast<const CdefRec*>(fl + pl->o_cdef);
    f.n_cdef = static_cast<int>(P.n_cdef);
    f.cdef_grid_w = P.cdef_grid_w;
    f.cdef_grid_n = P.cdef_grid_n;
    f.cdef_n_grid = P.cdef_search_any ? P.cdef_grid_n : 0;
    f.cdef_extra = reinterpret_cast<const unsigned*>(fl + pl->o_cdef_search);
    f.n_cdef_extra = static_cast<int>(P.n_cdef_search);
    f.cdef_search = static_cast<int*>(d->cdef_search.p);
  }
  const px_t* lr_curr = snap;
  if (P.upscaled) {
    for (int p = 0; p < 3; ++p) superres_params(L.p[p].coded_w, L.p[p].out_w, &f.up.step[p], &f.up.initial[p]);
    auto set_pass = [&](int k, const px_t* src, px_t* dst, bool border) {
      const int rows0 = border ? 4 * ((L.p[0].out_h + 8) / 64 + 1) : L.p[0].out_h;
      const int rows1 = L.p[1].out_h > 0 ? (border ? rows0 : L.p[1].out_h) : 0;
      const int segs = std::max((L.p[0].out_w + AV1B_UP_OUT - 1) / AV1B_UP_OUT,
                                2 * ((L.p[1].out_w + AV1B_UP_OUT - 1) / AV1B_UP_OUT));
      f.up_src[k] = src;
      f.up_dst[k] = dst;
      f.up_border[k] = border ? 1 : 0;
      f.up_rows0[k] = rows0;
      f.up_segs[k] = segs;
      f.up_items[k] = segs * (rows0 + rows1);
    };
    if (P.use_lr) {
      set_pass(0, snap, lr_pre_up, true);
      set_pass(1, cur, lr_cdef, false);
      lr_curr = lr_pre_up;
    } else {
      set_copy(1, cur, snap);
      set_pass(1, snap, cur, false);
    }
  } else if (P.use_lr) {
    set_copy(1, cur, lr_cdef);
  }
  if (P.use_lr) {
    f.lr = P.lr;
    for (int p = 0; p < 3; ++p) f.lr.units[p] = reinterpret_cast<const LrUnitRec*>(ar + pl->o_lr[p]);
    f.lr_cdef = lr_cdef;
    f.lr_curr = lr_curr;
    f.lr_dst = cur;
    f.lr_copy_rest = P.upscaled ? 1 : 0;
    f.lr_tiles = std::max((L.p[0].out_w + AV1B_LR_TW - 1) / AV1B_LR_TW,
                          2 * ((L.p[1].out_w + AV1B_LR_TW - 1) / AV1B_LR_TW));
    f.lr_stripes = (L.p[0].out_h + 8 + 63) / 64;
  }
  if (sp->keep) set_copy(2, cur, static_cast<px_t*>(d->slot_buf[sp->slot].p));
  d->disp_is_cur = true;
  d->disp_pending = false;
  if (P.grain) {
    GrainState* gsd = static_cast<GrainState*>(d->grain_state.p);
    /* the constants are copied from the plan by the template kernel */
    f.gs_src = reinterpret_cast<const int*>(ar + pl->o_gs);
    f.grain = 1;
    f.gs = gsd;
    f.gp = P.gp;
    f.orbit = static_cast<const uint16_t*>(d->orbit.p);
    f.pos = static_cast<const uint16_t*>(d->pos.p);
    f.grain_src = cur;
    f.grain_dst = static_cast<px_t*>(d->disp.p);
    const int groups = std::max((L.p[0].out_w + 3) / 4, 2 * ((L.p[1].out_w + 3) / 4));
    f.grain_xblocks = (groups + 127) / 128;
    f.grain_rows = L.p[0].out_h + L.p[1].out_h;
    d->disp_is_cur = false;
  }
  return AV1B_OK;
}

}  // namespace
}  // namespace av1b

struct av1b_batch {
  int device = 0, n_sm = 148;
  cudaStream_t stream = nullptr, side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr, done = nullptr, t0 = nullptr, t1 = nullptr;
  av1b::StreamStep* d_steps = nullptr;
  av1b::BatchHeader* d_hdr = nullptr;
  int2* d_chains = nullptr;
  size_t chains_cap = 0;
  /* page-locked staging of a step's descriptors, a ring so that the host
   * fills one while earlier steps' copies are in flight */
  struct Staging {
    uint8_t* host = nullptr;
    size_t cap = 0;
    cudaEvent_t used = nullptr;
    bool pending = false;
  };
  Staging ring[4];
  int ring_next = 0;
  av1b::BatchTuning tuning{};
  bool use_graph = true;
  struct Graph {
    std::string key;
    cudaGraphExec_t exec = nullptr;
  };
  std::vector<Graph> graphs;
  std::vector<av1b_decoder*> last;   /* the decoders of the last step */
  /* per-stage timing (av1b_batch_set_profiling): a set of events a step,
   * summed when the batch is synchronized */
  bool profiling = false;
  std::vector<std::vector<cudaEvent_t>> prof_free, prof_pending;
  double prof_ms[av1b::kBStageCount] = {0};
  long long prof_n = 0;
  std::mutex mu;
  std::string err;
};

namespace av1b {
namespace {

int bfail(av1b_batch* b, int code, const std::string& msg) {
  b->err = msg;
  return code;
}

int bcuda(av1b_batch* b, cudaError_t e, const char* what) {
  b->err = std::string(what) + ": " + cudaGetErrorString(e);
  return AV1B_ERR_CUDA;
}

#define BCK(call, what)                                    \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return bcuda(b, e_, what);      \
  } while (0)

static_assert(kBStageCount <= static_cast<int>(sizeof(av1b_batch_config::ctas_per_sm) / sizeof(int32_t)),
              "the public launch-shape array holds every stage");

/* Launch shapes before tuning: CTAs per SM of each stage kernel. */
void default_tuning(BatchTuning* t) {
  static const int ctas[kBStageCount] = {
      4, 4, 4, 4,           /* prediction: lean unmasked, lean masked, full, chroma
                               tiles reading luma masks */
      4, 4, 4, 4, 2, 2,     /* transforms by class */
      AV1B_UNIT_CTAS_PER_SM,
      8, 8,                 /* deblocking */
      4, 8, 8, 4,           /* snapshot, CDEF searches, CDEF, post-CDEF copy */
      16, 4, 4,             /* superres, restoration, reference store */
      2, 8, 8};             /* grain templates, grain blend, NV12 */
  for (int k = 0; k < kBStageCount; ++k) t->ctas_per_sm[k] = ctas[k];
  t->claim_chunk = 1;
  t->fuse_grain_nv12 = 0;
  t->inter_variant = 0;
  /* never more CTAs an SM than the kernel's resources let one SM hold */
  for (int k = 0; k < kBStageCount; ++k) t->ctas_per_sm[k] = std::min(t->ctas_per_sm[k], batch_stage_max_ctas(k));
}

std::string tuning_key(const BatchTuning& t, bool units_inter) {
  std::string k = units_inter ? "i" : "n";
  char buf[16];
  for (int s = 0; s < kBStageCount; ++s) {
    std::snprintf(buf, sizeof(buf), ",%d", t.ctas_per_sm[s]);
    k += buf;
  }
  std::snprintf(buf, sizeof(buf), ";%d;%d", t.claim_chunk, t.inter_variant);
  return k + buf;
}

/* The step's graph for the tuning and kernel choice, captured on first use. */
int step_graph(av1b_batch* b, bool units_inter, cudaGraphExec_t* out) {
  const std::string key = tuning_key(b->tuning, units_inter);
  for (const auto& g : b->graphs)
    if (g.key == key) {
      *out = g.exec;
      return AV1B_OK;
    }
  cudaGraph_t graph = nullptr;
  BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
  const cudaError_t le = launch_batch_step(b->d_steps, b->d_hdr, b->tuning, b->n_sm, units_inter,
                                           b->stream, b->side, b->fork, b->join);
  const cudaError_t ce = cudaStreamEndCapture(b->stream, &graph);
  if (le != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return bcuda(b, le, "batched step capture");
  }
  BCK(ce, "graph capture end");
  cudaGraphExec_t exec = nullptr;
  const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  BCK(ie, "graph instantiate");
  b->graphs.push_back({key, exec});
  *out = exec;
  return AV1B_OK;
}

/* One batched step. Decoders are locked in address order for the call. */
int batch_step(av1b_batch* b, int n, av1b_decoder* const* decs, av1b_plan* const* plans,
               const int* slots, int* out_slots, uint8_t* const* nv12, const size_t* pitch,
               const size_t* nv12_len) {
  if (n < 1 || n > AV1B_BATCH_MAX || !decs || !plans)
    return bfail(b, AV1B_ERR_ARG, "1 to 64 streams a step, each with a decoder and a plan");
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) {
    if (!decs[i] || !plans[i]) return bfail(b, AV1B_ERR_ARG, "a null decoder or plan");
    if (decs[i]->device != b->device) return bfail(b, AV1B_ERR_ARG, "a decoder of another device");
    order[i] = i;
  }
  std::sort(order.begin(), order.end(), [&](int x, int y) { return decs[x] < decs[y]; });
  for (int i = 1; i < n; ++i)
    if (decs[order[i]] == decs[order[i - 1]])
      return bfail(b, AV1B_ERR_ARG, "a decoder appears twice in one step");
  BCK(cudaSetDevice(b->device), "device");
  std::vector<std::unique_lock<std::mutex>> locks;
  locks.reserve(n);
  for (int i : order) locks.emplace_back(decs[i]->mu);

  std::vector<StepPrep> sp(n);
  bool units_inter = false;
  size_t n_chains = 0;
  for (int i = 0; i < n; ++i) {
    av1b_decoder* d = decs[i];
    clear_err(d);
    /* the decoder's own stream, when a call queued work there since its last
     * batched step: the step waits for it */
    if (!d->batch_pending) {
      if (!d->ev_batch) BCK(cudaEventCreateWithFlags(&d->ev_batch, cudaEventDisableTiming), "event");
      BCK(cudaEventRecord(d->ev_batch, d->stream), "decoder order");
      BCK(cudaStreamWaitEvent(b->stream, d->ev_batch, 0), "decoder order");
    }
    int rc = prepare_step(d, plans[i], 1, slots ? slots[i] : -1, true, &sp[i], b->stream);
    if (rc) return bfail(b, rc, "stream " + std::to_string(i) + ": " + d->err);
    FilterArgs& f = sp[i].f;
    const Plan& P = plans[i]->P;
    if (nv12 && nv12[i]) {
      const size_t need = nv12_bytes(plans[i]->width, plans[i]->height, plans[i]->ss_x,
                                     plans[i]->ss_y, pitch ? pitch[i] : 0);
      if (!need || !pitch || (nv12_len && nv12_len[i] < need) || pitch[i] > (1u << 30))
        return bfail(b, AV1B_ERR_ARG, "stream " + std::to_string(i) +
                                          ": NV12 needs 4:2:0, an even pitch at least a chroma "
                                          "row wide and room for every row");
      f.nv12 = nv12[i];
      f.nv12_pitch = static_cast<int>(pitch[i]);
      f.nv12_xblocks = static_cast<int>((pitch[i] + 8 * 128 - 1) / (8 * 128));
      f.nv12_rows = d->L.p[0].out_h + (d->L.p[0].out_h + 1) / 2;
      f.fuse_grain = f.grain && b->tuning.fuse_grain_nv12 ? 1 : 0;
      f.nv12_src = f.fuse_grain || !f.grain ? static_cast<const px_t*>(d->cur.p)
                                            : static_cast<const px_t*>(d->disp.p);
      if (f.fuse_grain) d->disp_pending = true;
    }
    units_inter = units_inter || P.units_inter;
    n_chains += P.n_chains;
  }
  if (n_chains > static_cast<size_t>(INT32_MAX)) return bfail(b, AV1B_ERR_SYNTAX, "too many chains");

  /* the descriptors, into a staging buffer of the ring */
  const size_t steps_bytes = sizeof(StreamStep) * n;
  const size_t hdr_off = align_up(steps_bytes, 256);
  const size_t chains_off = align_up(hdr_off + sizeof(BatchHeader), 256);
  const size_t total = chains_off + n_chains * sizeof(int2);
  av1b_batch::Staging& stg = b->ring[b->ring_next];
  b->ring_next = (b->ring_next + 1) % 4;
  if (stg.pending) {
    BCK(cudaEventSynchronize(stg.used), "staging reuse");
    stg.pending = false;
  }
  if (stg.cap < total) {
    if (stg.host) cudaFreeHost(stg.host);
    stg.host = nullptr;
    stg.cap = 0;
    const size_t want = align_up(total + total / 2, 1 << 16);
    BCK(cudaHostAlloc(reinterpret_cast<void**>(&stg.host), want, cudaHostAllocDefault), "staging");
    stg.cap = want;
  }
  StreamStep* hs = reinterpret_cast<StreamStep*>(stg.host);
  BatchHeader* hh = reinterpret_cast<BatchHeader*>(stg.host + hdr_off);
  int2* hc = reinterpret_cast<int2*>(stg.host + chains_off);
  std::memset(hh, 0, sizeof(BatchHeader));
  hh->n = n;
  for (int i = 0; i < n; ++i) {
    hs[i].a = sp[i].a;
    hs[i].f = sp[i].f;
    const FrameArgs& a = sp[i].a;
    const FilterArgs& f = sp[i].f;
    long long items[kBStageCount] = {};
    items[kBInterSimple] = a.n_inter_simple;
    items[kBInterLeanMask] = a.n_inter_lmask;
    items[kBInter] = a.n_inter_tiles - a.n_inter_simple - a.n_inter_lmask - a.n_inter_cmask;
    items[kBInterMask] = a.n_inter_cmask;
    for (int c = 2; c <= 7; ++c) items[kBItx2 + c - 2] = a.n_itx_batches > 0 ? a.itx_class_count[c] : 0;
    items[kBUnits] = a.n_chains;
    items[kBDeblockV] = (f.n_dbv + AV1B_DB_GROUP - 1) / AV1B_DB_GROUP;
    items[kBDeblockH] = (f.n_dbh + AV1B_DB_GROUP - 1) / AV1B_DB_GROUP;
    items[kBCopySnap] = f.copy_items[0];
    items[kBCopyPost] = f.copy_items[1];
    items[kBCopyRef] = f.copy_items[2];
    items[kBCdefSearch] = f.n_cdef > 0 ? (f.cdef_n_grid + f.n_cdef_extra + 127) / 128 : 0;
    items[kBCdef] = (f.n_cdef + 7) / 8;
    items[kBUpscale] = f.up_items[0] + f.up_items[1];
    items[kBLr] = f.lr_tiles ? static_cast<long long>(f.lr_tiles) * f.lr_stripes * 2 : 0;
    items[kBGrainTemplate] = f.grain ? 1 : 0;
    items[kBGrain] = f.grain && !f.fuse_grain ? static_cast<long long>(f.grain_xblocks) * f.grain_rows : 0;
    items[kBNv12] = f.nv12 ? static_cast<long long>(f.nv12_xblocks) * f.nv12_rows : 0;
    for (int k = 0; k < kBStageCount; ++k) {
      const long long nx = static_cast<long long>(hh->pfx[k][i]) + items[k];
      if (nx > INT32_MAX) return bfail(b, AV1B_ERR_SYNTAX, "a step too large for one launch");
      hh->pfx[k][i + 1] = static_cast<int>(nx);
    }
  }
  /* the streams' chains interleaved by the depth of their first block, each
   * stream's in its own order, the streams aligned at their ends: a stream
   * whose dependency path is shorter than the deepest one's starts that many
   * levels later, so the chains on the longest paths (a large key frame's)
   * are claimed first and do not wait behind warps holding chains of short
   * paths that could have run later */
  {
    size_t m = 0;
    size_t levels = 0;
    for (int i = 0; i < n; ++i) levels = std::max(levels, plans[i]->P.depth_first.size());
    for (size_t k = 0; k + 1 < levels; ++k)
      for (int i = 0; i < n; ++i) {
        const std::vector<int>& df = plans[i]->P.depth_first;
        const size_t late = levels - std::max<size_t>(df.size(), 1);   /* >= 0 */
        if (k < late || k - late + 1 >= df.size()) continue;
        const size_t kk = k - late;
        for (int c = df[kk]; c < df[kk + 1]; ++c) hc[m++] = make_int2(i, c);
      }
    if (m != n_chains) return bfail(b, AV1B_ERR_SYNTAX, "chain order of a plan is inconsistent");
  }
  hh->n_chain_order = static_cast<int>(n_chains);
  if (n_chains > b->chains_cap) {
    if (b->d_chains) cudaFree(b->d_chains);
    b->d_chains = nullptr;
    b->chains_cap = 0;
    const size_t want = n_chains + n_chains / 2 + 1024;
    BCK(cudaMalloc(&b->d_chains, want * sizeof(int2)), "chain order");
    b->chains_cap = want;
  }
  hh->chain_order = b->d_chains;

  BCK(cudaMemcpyAsync(b->d_steps, hs, steps_bytes, cudaMemcpyHostToDevice, b->stream), "step upload");
  BCK(cudaMemcpyAsync(b->d_hdr, hh, sizeof(BatchHeader), cudaMemcpyHostToDevice, b->stream), "header upload");
  if (n_chains)
    BCK(cudaMemcpyAsync(b->d_chains, hc, n_chains * sizeof(int2), cudaMemcpyHostToDevice, b->stream),
        "chain upload");
  BCK(cudaEventRecord(stg.used, b->stream), "staging event");
  stg.pending = true;
  if (b->profiling) {
    if (b->prof_free.empty()) {
      std::vector<cudaEvent_t> set(kBStageCount + 2, nullptr);
      for (auto& e : set) BCK(cudaEventCreate(&e), "event");
      b->prof_free.push_back(set);
    }
    std::vector<cudaEvent_t> set = b->prof_free.back();
    b->prof_free.pop_back();
    BCK(launch_batch_step(b->d_steps, b->d_hdr, b->tuning, b->n_sm, units_inter, b->stream, b->side,
                          b->fork, b->join, set.data()), "batched step");
    b->prof_pending.push_back(set);
  } else if (b->use_graph) {
    cudaGraphExec_t exec = nullptr;
    int rc = step_graph(b, units_inter, &exec);
    if (rc) return rc;
    BCK(cudaGraphLaunch(exec, b->stream), "graph launch");
  } else {
    BCK(launch_batch_step(b->d_steps, b->d_hdr, b->tuning, b->n_sm, units_inter, b->stream, b->side,
                          b->fork, b->join), "batched step");
  }
  BCK(cudaEventRecord(b->done, b->stream), "step event");
  b->last.assign(decs, decs + n);
  for (int i = 0; i < n; ++i) {
    int got = -1;
    const int rc = commit_step(decs[i], plans[i], &sp[i], nullptr, &got, false, b->stream);
    if (rc) return bfail(b, rc, "stream " + std::to_string(i) + ": " + decs[i]->err);
    if (out_slots) out_slots[i] = got;
  }
  return AV1B_OK;
}

/* The most CTAs of each stage kernel an SM holds. */
int stage_cap(int stage) { return batch_stage_max_ctas(stage); }

/* Times the step `reps` times (after one untimed step) with the current
 * tuning; the smallest device time in ms. */
int time_step(av1b_batch* b, int n, av1b_decoder* const* decs, av1b_plan* const* plans,
              const int* slots, uint8_t* const* nv12, const size_t* pitch, const size_t* len,
              int reps, double* best) {
  int rc = batch_step(b, n, decs, plans, slots, nullptr, nv12, pitch, len);
  if (rc) return rc;
  *best = 1e30;
  for (int r = 0; r < reps; ++r) {
    BCK(cudaEventRecord(b->t0, b->stream), "event");
    if ((rc = batch_step(b, n, decs, plans, slots, nullptr, nv12, pitch, len))) return rc;
    BCK(cudaEventRecord(b->t1, b->stream), "event");
    BCK(cudaEventSynchronize(b->t1), "event");
    float ms = 0.f;
    BCK(cudaEventElapsedTime(&ms, b->t0, b->t1), "event");
    *best = std::min(*best, static_cast<double>(ms));
  }
  for (av1b_decoder* d : b->last)
    if ((rc = av1b_sync(d))) return bfail(b, rc, "a tuning step failed");
  return AV1B_OK;
}

std::string tune_signature(av1b_batch* b, int n, av1b_plan* const* plans, uint8_t* const* nv12) {
  std::vector<std::string> parts;
  bool ui = false;
  for (int i = 0; i < n; ++i) {
    const av1b_plan* pl = plans[i];
    char buf[96];
    std::snprintf(buf, sizeof(buf), "%dx%d/%d/%db/g%d/l%d/o%d", pl->width, pl->height, pl->coded_width,
                  pl->bit_depth, pl->P.grain ? 1 : 0, pl->P.use_lr ? 1 : 0, nv12 && nv12[i] ? 1 : 0);
    parts.push_back(buf);
    ui = ui || pl->P.units_inter;
  }
  std::sort(parts.begin(), parts.end());
  cudaDeviceProp prop;
  std::string key = cudaGetDeviceProperties(&prop, b->device) == cudaSuccess ? prop.name : "gpu";
  for (char& c : key)
    if (c == ' ') c = '_';
  key += ":" + std::to_string(b->n_sm) + ":" + (ui ? "i" : "n");
  for (const auto& p : parts) key += " " + p;
  return key;
}

std::string tuning_text(const BatchTuning& t) {
  std::string s;
  for (int k = 0; k < kBStageCount; ++k) s += std::to_string(t.ctas_per_sm[k]) + " ";
  return s + std::to_string(t.claim_chunk) + " " + std::to_string(t.fuse_grain_nv12) + " " +
         std::to_string(t.inter_variant);
}

bool parse_tuning(const std::string& s, BatchTuning* t) {
  BatchTuning r{};
  const char* p = s.c_str();
  char* end = nullptr;
  for (int k = 0; k < kBStageCount + 3; ++k) {
    const long v = std::strtol(p, &end, 10);
    if (end == p || v < 0 || v > 64) return false;
    if (k < kBStageCount) r.ctas_per_sm[k] = static_cast<int>(v);
    else if (k == kBStageCount) r.claim_chunk = static_cast<int>(v);
    else if (k == kBStageCount + 1) r.fuse_grain_nv12 = static_cast<int>(v);
    else r.inter_variant = static_cast<int>(v) ? 1 : 0;
    p = end;
  }
  if (r.claim_chunk < 1) return false;
  *t = r;
  return true;
}

/* The cache: one line per signature, "signature<TAB>tuning". */
bool cache_lookup(const char* path, const std::string& key, BatchTuning* t) {
  if (!path || !*path) return false;
  FILE* fp = std::fopen(path, "r");
  if (!fp) return false;
  char line[8192];
  bool found = false;
  while (std::fgets(line, sizeof(line), fp)) {
    std::string l(line);
    while (!l.empty() && (l.back() == '\n' || l.back() == '\r')) l.pop_back();
    const size_t tab = l.find('\t');
    if (tab == std::string::npos || l.compare(0, tab, key) != 0 || tab != key.size()) continue;
    found = parse_tuning(l.substr(tab + 1), t);
  }
  std::fclose(fp);
  return found;
}

void cache_store(const char* path, const std::string& key, const BatchTuning& t) {
  if (!path || !*path) return;
  std::vector<std::string> keep;
  if (FILE* fp = std::fopen(path, "r")) {
    char line[8192];
    while (std::fgets(line, sizeof(line), fp)) {
      std::string l(line);
      while (!l.empty() && (l.back() == '\n' || l.back() == '\r')) l.pop_back();
      const size_t tab = l.find('\t');
      if (tab != std::string::npos && !(tab == key.size() && l.compare(0, tab, key) == 0)) keep.push_back(l);
    }
    std::fclose(fp);
  }
  keep.push_back(key + "\t" + tuning_text(t));
  const std::string tmp = std::string(path) + ".tmp";
  if (FILE* fp = std::fopen(tmp.c_str(), "w")) {
    for (const auto& l : keep) std::fprintf(fp, "%s\n", l.c_str());
    std::fclose(fp);
    std::rename(tmp.c_str(), path);
  }
}

}  // namespace
}  // namespace av1b

/* ---- C ABI of the batched form ------------------------------------------------------------ */
using namespace av1b;

extern "C" {

int av1b_batch_create(int device, av1b_batch** out) {
  if (!out) return AV1B_ERR_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return AV1B_ERR_NO_DEVICE;
  if (device < 0 || device >= n) return AV1B_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return AV1B_ERR_CUDA;
  auto* b = new av1b_batch;
  b->device = device;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) b->n_sm = prop.multiProcessorCount;
  bool ok = set_kernel_attributes() == cudaSuccess && set_batch_kernel_attributes() == cudaSuccess &&
            cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreate(&b->t0) == cudaSuccess && cudaEventCreate(&b->t1) == cudaSuccess &&
            cudaMalloc(&b->d_steps, sizeof(StreamStep) * AV1B_BATCH_MAX) == cudaSuccess &&
            cudaMalloc(&b->d_hdr, sizeof(BatchHeader)) == cudaSuccess;
  for (auto& r : b->ring) ok = ok && cudaEventCreateWithFlags(&r.used, cudaEventDisableTiming) == cudaSuccess;
  if (ok) default_tuning(&b->tuning);   /* after the kernels' attributes: it reads their occupancy */
  if (!ok) {
    av1b_batch_destroy(b);
    return AV1B_ERR_CUDA;
  }
  *out = b;
  return AV1B_OK;
}

int av1b_batch_destroy(av1b_batch* b) {
  if (!b) return AV1B_ERR_ARG;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->side) cudaStreamSynchronize(b->side);
  for (auto& g : b->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  for (auto& r : b->ring) {
    if (r.host) cudaFreeHost(r.host);
    if (r.used) cudaEventDestroy(r.used);
  }
  for (auto* sets : {&b->prof_free, &b->prof_pending})
    for (auto& set : *sets)
      for (cudaEvent_t e : set)
        if (e) cudaEventDestroy(e);
  cudaEvent_t evs[] = {b->fork, b->join, b->done, b->t0, b->t1};
  for (cudaEvent_t e : evs)
    if (e) cudaEventDestroy(e);
  if (b->d_steps) cudaFree(b->d_steps);
  if (b->d_hdr) cudaFree(b->d_hdr);
  if (b->d_chains) cudaFree(b->d_chains);
  if (b->side) cudaStreamDestroy(b->side);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return AV1B_OK;
}

int av1b_batch_decode(av1b_batch* b, int n, av1b_decoder* const* decoders, av1b_plan* const* plans,
                      const int* slots, int* out_slots, uint8_t* const* nv12_device,
                      const size_t* nv12_pitch, const size_t* nv12_len) {
  if (!b) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(b->mu);
  b->err.clear();
  return batch_step(b, n, decoders, plans, slots, out_slots, nv12_device, nv12_pitch, nv12_len);
}

static void collect_batch_profile(av1b_batch* b) {
  for (auto& set : b->prof_pending) {
    if (cudaEventSynchronize(set[kBStageCount]) == cudaSuccess &&
        cudaEventSynchronize(set[kBStageCount + 1]) == cudaSuccess) {
      for (int k = kBInterSimple; k < kBStageCount; ++k) {
        float ms = 0.f;
        /* the stage's own launch to the next stage's (the templates on the
         * side stream from the step's start to their end) */
        if (k == kBGrainTemplate)
          cudaEventElapsedTime(&ms, set[kBInterSimple], set[kBStageCount + 1]);
        else
          cudaEventElapsedTime(&ms, set[k], set[k == kBCopyRef ? kBGrain : (k == kBNv12 ? kBStageCount : k + 1)]);
        b->prof_ms[k] += ms;
      }
      ++b->prof_n;
    }
    b->prof_free.push_back(set);
  }
  b->prof_pending.clear();
}

int av1b_batch_set_profiling(av1b_batch* b, int on) {
  if (!b) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(b->mu);
  collect_batch_profile(b);
  b->profiling = on != 0;
  for (double& v : b->prof_ms) v = 0;
  b->prof_n = 0;
  return AV1B_OK;
}

int av1b_batch_profile(av1b_batch* b, int stage, double* total_ms, long long* steps) {
  if (!b || stage < 0 || stage >= kBStageCount) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(b->mu);
  collect_batch_profile(b);
  if (total_ms) *total_ms = b->prof_ms[stage];
  if (steps) *steps = b->prof_n;
  return AV1B_OK;
}

int av1b_batch_sync(av1b_batch* b) {
  if (!b) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(b->mu);
  int first = AV1B_OK;
  for (size_t i = 0; i < b->last.size(); ++i) {
    const int rc = av1b_sync(b->last[i]);
    if (rc && first == AV1B_OK) {
      first = rc;
      b->err = "stream " + std::to_string(i) + ": " + av1b_last_error(b->last[i]);
    }
  }
  if (b->stream && cudaStreamSynchronize(b->stream) != cudaSuccess && first == AV1B_OK)
    first = bfail(b, AV1B_ERR_CUDA, "batched step failed on the device");
  return first;
}

static void to_config(const av1b_batch* b, av1b_batch_config* c) {
  std::memset(c, 0, sizeof(*c));
  for (int k = 0; k < kBStageCount; ++k) c->ctas_per_sm[k] = b->tuning.ctas_per_sm[k];
  c->claim_chunk = b->tuning.claim_chunk;
  c->fuse_grain_nv12 = b->tuning.fuse_grain_nv12;
  c->use_graph = b->use_graph ? 1 : 0;
  c->inter_variant = b->tuning.inter_variant;
}

int av1b_batch_get_config(av1b_batch* b, av1b_batch_config* out) {
  if (!b || !out) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(b->mu);
  to_config(b, out);
  return AV1B_OK;
}

int av1b_batch_set_config(av1b_batch* b, const av1b_batch_config* c) {
  if (!b || !c) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(b->mu);
  BatchTuning t = b->tuning;
  for (int k = 0; k < kBStageCount; ++k) {
    if (c->ctas_per_sm[k] < 0) return bfail(b, AV1B_ERR_ARG, "negative CTAs per SM");
    if (c->ctas_per_sm[k] > 0) t.ctas_per_sm[k] = std::min(c->ctas_per_sm[k], stage_cap(k));
  }
  if (c->claim_chunk < 0 || c->claim_chunk > 64) return bfail(b, AV1B_ERR_ARG, "claim chunk out of range");
  if (c->claim_chunk > 0) t.claim_chunk = c->claim_chunk;
  t.fuse_grain_nv12 = c->fuse_grain_nv12 ? 1 : 0;
  t.inter_variant = c->inter_variant ? 1 : 0;
  b->tuning = t;
  b->use_graph = c->use_graph != 0;
  return AV1B_OK;
}

int av1b_batch_autotune(av1b_batch* b, int n, av1b_decoder* const* decoders,
                        av1b_plan* const* plans, const int* slots, uint8_t* const* nv12_device,
                        const size_t* nv12_pitch, const size_t* nv12_len, const char* cache_path,
                        int reps, av1b_batch_config* out, double* best_ms) {
  if (!b || n < 1 || !plans) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(b->mu);
  b->err.clear();
  const std::string key = tune_signature(b, n, plans, nv12_device);
  BatchTuning t;
  if (cache_lookup(cache_path, key, &t)) {
    for (int k = 0; k < kBStageCount; ++k) t.ctas_per_sm[k] = std::min(std::max(t.ctas_per_sm[k], 1), stage_cap(k));
    b->tuning = t;
    if (out) to_config(b, out);
    if (best_ms) *best_ms = -1.0;
    return AV1B_OK;
  }
  reps = std::max(1, std::min(reps, 50));
  int rc;
  double best = 0;
  default_tuning(&b->tuning);
  if ((rc = time_step(b, n, decoders, plans, slots, nv12_device, nv12_pitch, nv12_len, reps, &best)))
    return rc;
  /* coordinate descent over groups of stages that share a launch shape,
   * then the claim size, then the grain-in-pack fusion */
  const std::vector<std::vector<int>> groups = {
      {kBInterSimple, kBInterLeanMask, kBInter, kBInterMask},
      {kBItx2, kBItx3, kBItx4, kBItx5, kBItx6, kBItx7},
      {kBUnits},
      {kBDeblockV, kBDeblockH},
      {kBCdefSearch, kBCdef},
      {kBCopySnap, kBCopyPost, kBCopyRef},
      {kBUpscale, kBLr},
      {kBGrainTemplate, kBGrain, kBNv12}};
  const int values[] = {1, 2, 4, 8, 16};
  for (const auto& g : groups) {
    BatchTuning keep = b->tuning;
    for (int v : values) {
      BatchTuning trial = keep;
      bool changed = false;
      for (int st : g) {
        const int c = std::min(v, stage_cap(st));
        changed = changed || c != keep.ctas_per_sm[st];
        trial.ctas_per_sm[st] = c;
      }
      if (!changed) continue;
      b->tuning = trial;
      double ms = 0;
      if ((rc = time_step(b, n, decoders, plans, slots, nv12_device, nv12_pitch, nv12_len, reps, &ms)))
        return rc;
      if (ms < best) {
        best = ms;
        keep = trial;
      }
    }
    b->tuning = keep;
  }
  for (int chunk : {2, 4}) {
    BatchTuning keep = b->tuning;
    b->tuning.claim_chunk = chunk;
    double ms = 0;
    if ((rc = time_step(b, n, decoders, plans, slots, nv12_device, nv12_pitch, nv12_len, reps, &ms)))
      return rc;
    if (ms < best) best = ms;
    else b->tuning = keep;
  }
  {
    BatchTuning keep = b->tuning;
    b->tuning.inter_variant = 1 - keep.inter_variant;
    double ms = 0;
    if ((rc = time_step(b, n, decoders, plans, slots, nv12_device, nv12_pitch, nv12_len, reps, &ms)))
      return rc;
    if (ms < best) best = ms;
    else b->tuning = keep;
  }
  {
    BatchTuning keep = b->tuning;
    b->tuning.fuse_grain_nv12 = 1;
    double ms = 0;
    if ((rc = time_step(b, n, decoders, plans, slots, nv12_device, nv12_pitch, nv12_len, reps, &ms)))
      return rc;
    if (ms < best) best = ms;
    else b->tuning = keep;
  }
  cache_store(cache_path, key, b->tuning);
  if (out) to_config(b, out);
  if (best_ms) *best_ms = best;
  return AV1B_OK;
}

const char* av1b_batch_last_error(av1b_batch* b) { return b ? b->err.c_str() : ""; }

void* av1b_batch_stream(av1b_batch* b) { return b ? b->stream : nullptr; }

}  // extern "C"
