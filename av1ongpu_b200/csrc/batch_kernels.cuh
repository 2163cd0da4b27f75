/*
 * batch_kernels.cuh - the batched form's stage kernels: every stage of one
 * frame of many streams in one persistent launch. Part of kernels.cu's
 * translation unit (included at its end): the kernels call the same stage
 * bodies as the single-stream kernels there, so a stream's samples are the
 * same whether it is decoded alone or in a batch.
 *
 * Each kernel's grid is CTAs-per-SM x SM count. Warp-level stages claim
 * `chunk` items at a time from the stage's counter in the BatchHeader;
 * CTA-level stages stride over their items (blockIdx.x, + gridDim.x, ...) and
 * meet a CTA barrier between items, because their bodies stage tiles in
 * shared memory. Every early return inside a CTA-level body is either uniform
 * over the CTA or after the body's last barrier, so every thread reaches the
 * barrier between items.
 */

/* The stream of item `item` of a stage - the s with pfx[s] <= item <
 * pfx[s + 1] - for items a warp or CTA visits in increasing order (claims
 * from a counter, or strides): the search starts at the stream of the item
 * before, `s`, and moves forward over the streams in between, one comparison
 * for most items. */
__device__ __forceinline__ int batch_stream_next(const int* __restrict__ pfx, int n, int item, int s) {
  while (s + 1 < n && pfx[s + 1] <= item) ++s;
  return s;
}

/* The first of `chunk` consecutive items the warp claims (uniform over it). */
__device__ __forceinline__ int warp_claim(unsigned* ctr, int chunk, int lane) {
  int c = 0;
  if (lane == 0) c = static_cast<int>(atomicAdd(ctr, static_cast<unsigned>(chunk)));
  return __shfl_sync(0xffffffffu, c, 0);
}

/* Five CTAs an SM: the lean tile body plus the loop fit 96 registers
 * without spilling (unbounded, the compiler spilled). */
/* The lean kernel's stages: its unmasked tiles (MASK false, listed first);
 * with the masked build, the wedge and luma difference-weighted tiles listed
 * next (part 0) and, a stage of its own after the luma tiles that write the
 * masks, the chroma tiles that read a luma mask, listed last (part 1). */
template <bool MASK>
__global__ void __launch_bounds__(128, 5) kb_inter_simple(const StreamStep* __restrict__ st,
                                                       BatchHeader* h, int chunk, int part) {
  __shared__ McScratch scr[4];
  __shared__ int pred[4][2][8 * 16];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int stage = !MASK ? kBInterSimple : (part ? kBInterMask : kBInterLeanMask);
  const int* pfx = h->pfx[stage];
  const int n = h->n, total = pfx[n];
  int s = 0;
  for (;;) {
    const int i0 = warp_claim(&h->claim[stage], chunk, lane);
    if (i0 >= total) break;
    const int i1 = mini(i0 + chunk, total);
    for (int i = i0; i < i1; ++i) {
      s = batch_stream_next(pfx, n, i, s);
      const FrameArgs& a = st[s].a;
      const int t0 = !MASK ? 0 : (part ? a.n_inter_tiles - a.n_inter_cmask : a.n_inter_simple);
      inter_simple_tile<MASK>(a, t0 + (i - pfx[s]), scr[wib], pred[wib], lane);
      __syncwarp();
    }
  }
}

/* Two builds, the autotuner's choice (BatchTuning::inter_variant): at
 * three CTAs an SM the tile body gets the registers it needs without
 * spilling, at four it spills a little but more warps are resident and its
 * code is smaller. */
template <int MINB>
__global__ void __launch_bounds__(128, MINB) kb_inter(const StreamStep* __restrict__ st, BatchHeader* h,
                                                      int chunk) {
  __shared__ McScratch scr[4];
  __shared__ int pred[4][2][8 * 16];
  __shared__ int lpred[4][2][4 * 8 * 16];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int stage = kBInter;
  const int* pfx = h->pfx[stage];
  const int n = h->n, total = pfx[n];
  int s = 0;
  for (;;) {
    const int i0 = warp_claim(&h->claim[stage], chunk, lane);
    if (i0 >= total) break;
    const int i1 = mini(i0 + chunk, total);
    for (int i = i0; i < i1; ++i) {
      s = batch_stream_next(pfx, n, i, s);
      const FrameArgs& a = st[s].a;
      inter_full_tile(a, a.n_inter_simple + a.n_inter_lmask + (i - pfx[s]), scr[wib], pred[wib],
                      lpred[wib], lane);
      __syncwarp();
    }
  }
}

template <int CLS>
__global__ void __launch_bounds__(128) kb_itx(const StreamStep* __restrict__ st, BatchHeader* h,
                                              int chunk) {
  extern __shared__ int smem[];
  constexpr int STAGE = kBItx2 + (CLS == 7 ? 5 : CLS - 2);
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* wsm = smem + wib * ItxScratch<CLS>::PER_WARP;
  const int* pfx = h->pfx[STAGE];
  const int n = h->n, total = pfx[n];
  int s = 0;
  for (;;) {
    const int i0 = warp_claim(&h->claim[STAGE], chunk, lane);
    if (i0 >= total) break;
    const int i1 = mini(i0 + chunk, total);
    for (int i = i0; i < i1; ++i) {
      s = batch_stream_next(pfx, n, i, s);
      const FrameArgs& a = st[s].a;
      itx_batch<CLS>(a, a.itx_batches[a.itx_class_first[CLS] + (i - pfx[s])], wsm, lane);
      __syncwarp();
    }
  }
}

/* The dependency-scheduled phase of every stream: warps claim (stream, chain)
 * pairs in the merged order. A stream's chains keep their own claim order
 * in it, so every wait is on a chain of the same stream claimed earlier, and
 * the argument of the single-stream kernel holds: the warp holding the
 * earliest unfinished chain always progresses. */
template <bool INTER>
__global__ void __launch_bounds__(128, AV1B_UNIT_CTAS_PER_SM) kb_units(const StreamStep* __restrict__ st, BatchHeader* h) {
  extern __shared__ int smem[];
  const int wib = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  int* edges = smem + wib * (3 * AV1B_EDGE_LEN + AV1B_UNIT_SCRATCH);
  int* tmp = edges + 3 * AV1B_EDGE_LEN;
  const int total = h->n_chain_order;
  for (;;) {
    const int g = warp_claim(&h->claim[kBUnits], 1, lane);
    if (g >= total) break;
    const int2 sc = h->chain_order[g];
    run_chain<INTER>(st[sc.x].a, sc.y, edges, tmp, lane);
  }
}

/* Deblocking edges, AV1B_DB_GROUP records an item, a warp each: the warps
 * stride over the items (an item is a few cycles of work, so a claim from a
 * counter would cost as much) */
__global__ void __launch_bounds__(256) kb_deblock(const StreamStep* __restrict__ st, BatchHeader* h,
                                                  int vertical) {
  const int lane = threadIdx.x & 31;
  const int stage = vertical ? kBDeblockV : kBDeblockH;
  const int* pfx = h->pfx[stage];
  const int n = h->n, total = pfx[n];
  int s = 0;
  const int warps = static_cast<int>(gridDim.x * (blockDim.x >> 5));
  for (int i = static_cast<int>(blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)); i < total; i += warps) {
    s = batch_stream_next(pfx, n, i, s);
    const FilterArgs& f = st[s].f;
    const int r0 = (i - pfx[s]) * AV1B_DB_GROUP;
    const int nr = vertical ? f.n_dbv : f.n_dbh;
    deblock_group(st[s].a.cur, (vertical ? f.dbv : f.dbh) + r0, mini(AV1B_DB_GROUP, nr - r0), f.sharpness,
                  f.bd, f.maxv, lane);
  }
}

/* A picture copy, AV1B_COPY_ITEM bytes a CTA item, 16 bytes a thread. */
__global__ void __launch_bounds__(256) kb_copy(const StreamStep* __restrict__ st,
                                               const BatchHeader* __restrict__ h, int which) {
  const int stage = which == 0 ? kBCopySnap : (which == 1 ? kBCopyPost : kBCopyRef);
  const int* pfx = h->pfx[stage];
  const int n = h->n, total = pfx[n];
  int s = 0;
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    s = batch_stream_next(pfx, n, item, s);
    const FilterArgs& f = st[s].f;
    const long long off = static_cast<long long>(item - pfx[s]) * AV1B_COPY_ITEM;
    const long long left = f.copy_bytes[which] - off;
    const int vecs = static_cast<int>((left < AV1B_COPY_ITEM ? left : AV1B_COPY_ITEM) >> 4);
    const int4* src = reinterpret_cast<const int4*>(reinterpret_cast<const char*>(f.copy_src[which]) + off);
    int4* dst = reinterpret_cast<int4*>(reinterpret_cast<char*>(f.copy_dst[which]) + off);
    for (int k = threadIdx.x; k < vecs; k += blockDim.x) dst[k] = src[k];
  }
}

/* CDEF direction searches: 128 searches a CTA item. */
__global__ void __launch_bounds__(128) kb_cdef_search(const StreamStep* __restrict__ st,
                                                      const BatchHeader* __restrict__ h) {
  const int* pfx = h->pfx[kBCdefSearch];
  const int n = h->n, total = pfx[n];
  int s = 0;
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    s = batch_stream_next(pfx, n, item, s);
    const FilterArgs& f = st[s].f;
    const int t = (item - pfx[s]) * 128 + static_cast<int>(threadIdx.x);
    if (t < f.cdef_n_grid + f.n_cdef_extra)
      cdef_search_one(f.cdef_src, f.cdef_grid_w, f.cdef_grid_n, f.cdef_n_grid, f.cdef_extra,
                      f.cdef_search, st[s].a.L, t);
  }
}

/* CDEF records: eight a CTA item, a half-warp each. */
__global__ void __launch_bounds__(128) kb_cdef(const StreamStep* __restrict__ st,
                                               const BatchHeader* __restrict__ h) {
  __shared__ int sw[8][12 * 12];
  const int hw = threadIdx.x >> 4, hl = threadIdx.x & 15;
  const unsigned hmask = 0xffffu << (threadIdx.x & 16);
  const int* pfx = h->pfx[kBCdef];
  const int n = h->n, total = pfx[n];
  int s = 0;
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    s = batch_stream_next(pfx, n, item, s);
    const FilterArgs& f = st[s].f;
    const int ri = (item - pfx[s]) * 8 + hw;
    if (ri < f.n_cdef) {
      const CdefRec r = f.cdef[ri];
      cdef_record(f.cdef_src, f.cdef_dst, r, f.cdef_search, st[s].a.L, sw[hw], hl, hmask);
    }
    __syncwarp(hmask);   /* the half-warp's window is reused by its next record */
  }
}

/* Superres: a stream's items are its first pass's CTAs, then its second's. */
__global__ void __launch_bounds__(128) kb_upscale(const StreamStep* __restrict__ st,
                                                 const BatchHeader* __restrict__ h) {
  __shared__ __align__(16) short taps[512];
  __shared__ px_t span[AV1B_UP_SPAN];
  for (int i = threadIdx.x; i < 512; i += blockDim.x) taps[i] = kUpscaleFilter[i];
  __syncthreads();
  const int* pfx = h->pfx[kBUpscale];
  const int n = h->n, total = pfx[n];
  int s = 0;
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    s = batch_stream_next(pfx, n, item, s);
    const FilterArgs& f = st[s].f;
    int local = item - pfx[s];
    const int pass = local < f.up_items[0] ? 0 : 1;
    if (pass) local -= f.up_items[0];
    const int segs = f.up_segs[pass];
    const int yb = local / segs, xb = local - yb * segs;
    upscale_item(f.up_src[pass], f.up_dst[pass], st[s].a.L, f.up, f.maxv, f.up_border[pass],
                 f.up_rows0[pass], xb, yb, taps, span);
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256, 4) kb_lr(const StreamStep* __restrict__ st,
                                             const BatchHeader* __restrict__ h) {
  __shared__ LrSmem sm;
  const int* pfx = h->pfx[kBLr];
  const int n = h->n, total = pfx[n];
  int s = 0;
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    s = batch_stream_next(pfx, n, item, s);
    const FilterArgs& f = st[s].f;
    int local = item - pfx[s];
    const int bx = local % f.lr_tiles;
    local /= f.lr_tiles;
    const int stripe = local % f.lr_stripes, bz = local / f.lr_stripes;
    lr_tile_item(f.lr_cdef, f.lr_curr, f.lr_dst, st[s].a.L, f.lr, f.maxv, f.lr_copy_rest, bx, stripe,
                 bz, sm);
    __syncthreads();
  }
}

/* Grain templates: one stream's a CTA item. */
__global__ void __launch_bounds__(256) kb_grain_template(const StreamStep* __restrict__ st,
                                                         const BatchHeader* __restrict__ h) {
  __shared__ GrainTemplateSmem sm;
  const int* pfx = h->pfx[kBGrainTemplate];
  const int n = h->n, total = pfx[n];
  int s = 0;
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    s = batch_stream_next(pfx, n, item, s);
    const FilterArgs& f = st[s].f;
    /* the frame's grain constants and scaling tables, from its plan */
    {
      constexpr int tail = static_cast<int>(offsetof(GrainState, lut));
      constexpr int words = static_cast<int>((sizeof(GrainState) - tail) / 4);
      int* dst = reinterpret_cast<int*>(reinterpret_cast<char*>(f.gs) + tail);
      for (int k = threadIdx.x; k < words; k += blockDim.x) dst[k] = f.gs_src[k];
    }
    __syncthreads();
    grain_template_body(f.gs, f.gp, f.orbit, f.pos, sm);
    __syncthreads();
  }
}

__global__ void __launch_bounds__(128) kb_grain_blend(const StreamStep* __restrict__ st,
                                                      const BatchHeader* __restrict__ h) {
  const int* pfx = h->pfx[kBGrain];
  const int n = h->n, total = pfx[n];
  int s = 0;
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    s = batch_stream_next(pfx, n, item, s);
    const FilterArgs& f = st[s].f;
    const int local = item - pfx[s];
    const int y = local / f.grain_xblocks, xb = local - y * f.grain_xblocks;
    grain_blend_item(f.grain_src, f.grain_dst, st[s].a.L, f.gs, f.orbit, f.pos,
                     xb * 128 + static_cast<int>(threadIdx.x), y);
  }
}

__global__ void __launch_bounds__(128) kb_nv12(const StreamStep* __restrict__ st,
                                               const BatchHeader* __restrict__ h) {
  const int* pfx = h->pfx[kBNv12];
  const int n = h->n, total = pfx[n];
  int s = 0;
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    s = batch_stream_next(pfx, n, item, s);
    const FilterArgs& f = st[s].f;
    const int local = item - pfx[s];
    const int row = local / f.nv12_xblocks, xb = local - row * f.nv12_xblocks;
    const int x0 = (xb * 128 + static_cast<int>(threadIdx.x)) * 8;
    if (f.fuse_grain)
      nv12_grain_item(f.nv12_src, f.nv12, st[s].a.L, f.nv12_pitch, x0, row, f.gs, f.orbit, f.pos);
    else
      nv12_item(f.nv12_src, f.nv12, st[s].a.L, f.nv12_pitch, x0, row);
  }
}

static inline int batch_grid(const BatchTuning& t, int stage, int n_sm) {
  const int c = t.ctas_per_sm[stage];
  return (c > 0 ? c : 1) * n_sm;
}

template <int CLS>
static void launch_kb_itx(const StreamStep* steps, BatchHeader* hdr, const BatchTuning& t, int n_sm,
                          cudaStream_t s) {
  constexpr int STAGE = kBItx2 + (CLS == 7 ? 5 : CLS - 2);
  kb_itx<CLS><<<batch_grid(t, STAGE, n_sm), 128, 4 * ItxScratch<CLS>::PER_WARP * sizeof(int), s>>>(
      steps, hdr, t.claim_chunk);
}

/* With `prof` (kBStageCount + 2 events), stage k's launch is bracketed by
 * prof[k] and the next stage's event on `s`, prof[kBStageCount] ends the
 * step, and prof[kBStageCount + 1] ends the grain templates on `side` (they
 * start at prof[0]). */
cudaError_t launch_batch_step(const StreamStep* steps, BatchHeader* hdr, const BatchTuning& t,
                              int n_sm, bool units_inter, cudaStream_t s, cudaStream_t side,
                              cudaEvent_t fork, cudaEvent_t join, cudaEvent_t* prof) {
  cudaError_t e;
  const int chunk = t.claim_chunk > 0 ? t.claim_chunk : 1;
  auto mark = [&](int k) {
    if (prof) cudaEventRecord(prof[k], k == kBStageCount + 1 ? side : s);
  };
  /* the claim counters restart every step */
  if ((e = cudaMemsetAsync(hdr->claim, 0, sizeof(hdr->claim), s)) != cudaSuccess) return e;
  /* the grain templates depend only on the parameters: a side branch, joined
   * before the blend */
  if ((e = cudaEventRecord(fork, s)) != cudaSuccess || (e = cudaStreamWaitEvent(side, fork, 0)) != cudaSuccess)
    return e;
  kb_grain_template<<<batch_grid(t, kBGrainTemplate, n_sm), 256, 0, side>>>(steps, hdr);
  mark(kBStageCount + 1);
  if ((e = cudaEventRecord(join, side)) != cudaSuccess) return e;
  mark(kBInterSimple);
  kb_inter_simple<false><<<batch_grid(t, kBInterSimple, n_sm), 128, 0, s>>>(steps, hdr, chunk, 0);
  mark(kBInterLeanMask);
  kb_inter_simple<true><<<batch_grid(t, kBInterLeanMask, n_sm), 128, 0, s>>>(steps, hdr, chunk, 0);
  mark(kBInter);
  if (t.inter_variant) kb_inter<4><<<batch_grid(t, kBInter, n_sm), 128, 0, s>>>(steps, hdr, chunk);
  else kb_inter<3><<<batch_grid(t, kBInter, n_sm), 128, 0, s>>>(steps, hdr, chunk);
  mark(kBInterMask);
  kb_inter_simple<true><<<batch_grid(t, kBInterMask, n_sm), 128, 0, s>>>(steps, hdr, chunk, 1);
  mark(kBItx2);
  launch_kb_itx<2>(steps, hdr, t, n_sm, s);
  mark(kBItx3);
  launch_kb_itx<3>(steps, hdr, t, n_sm, s);
  mark(kBItx4);
  launch_kb_itx<4>(steps, hdr, t, n_sm, s);
  mark(kBItx5);
  launch_kb_itx<5>(steps, hdr, t, n_sm, s);
  mark(kBItx6);
  launch_kb_itx<6>(steps, hdr, t, n_sm, s);
  mark(kBItx7);
  launch_kb_itx<7>(steps, hdr, t, n_sm, s);
  mark(kBUnits);
  {
    const size_t smem = 4 * (3 * AV1B_EDGE_LEN + AV1B_UNIT_SCRATCH) * sizeof(int);
    const int grid = mini(batch_grid(t, kBUnits, n_sm), AV1B_UNIT_CTAS_PER_SM * n_sm);
    if (units_inter) kb_units<true><<<grid, 128, smem, s>>>(steps, hdr);
    else kb_units<false><<<grid, 128, smem, s>>>(steps, hdr);
  }
  mark(kBDeblockV);
  kb_deblock<<<batch_grid(t, kBDeblockV, n_sm), 256, 0, s>>>(steps, hdr, 1);
  mark(kBDeblockH);
  kb_deblock<<<batch_grid(t, kBDeblockH, n_sm), 256, 0, s>>>(steps, hdr, 0);
  mark(kBCopySnap);
  kb_copy<<<batch_grid(t, kBCopySnap, n_sm), 256, 0, s>>>(steps, hdr, 0);
  mark(kBCdefSearch);
  kb_cdef_search<<<batch_grid(t, kBCdefSearch, n_sm), 128, 0, s>>>(steps, hdr);
  mark(kBCdef);
  kb_cdef<<<batch_grid(t, kBCdef, n_sm), 128, 0, s>>>(steps, hdr);
  mark(kBCopyPost);
  kb_copy<<<batch_grid(t, kBCopyPost, n_sm), 256, 0, s>>>(steps, hdr, 1);
  mark(kBUpscale);
  kb_upscale<<<batch_grid(t, kBUpscale, n_sm), 128, 0, s>>>(steps, hdr);
  mark(kBLr);
  kb_lr<<<batch_grid(t, kBLr, n_sm), 256, 0, s>>>(steps, hdr);
  mark(kBCopyRef);
  kb_copy<<<batch_grid(t, kBCopyRef, n_sm), 256, 0, s>>>(steps, hdr, 2);
  if ((e = cudaStreamWaitEvent(s, join, 0)) != cudaSuccess) return e;
  mark(kBGrain);
  kb_grain_blend<<<batch_grid(t, kBGrain, n_sm), 128, 0, s>>>(steps, hdr);
  mark(kBNv12);
  kb_nv12<<<batch_grid(t, kBNv12, n_sm), 128, 0, s>>>(steps, hdr);
  mark(kBStageCount);
  return cudaGetLastError();
}

cudaError_t set_batch_kernel_attributes() {
  const int units_smem = 4 * (3 * AV1B_EDGE_LEN + AV1B_UNIT_SCRATCH) * (int)sizeof(int);
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(kb_units<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, units_smem)) != cudaSuccess ||
      (e = cudaFuncSetAttribute(kb_units<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, units_smem)) != cudaSuccess ||
      (e = cudaFuncSetAttribute(kb_units<true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared)) != cudaSuccess ||
      (e = cudaFuncSetAttribute(kb_units<false>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared)) != cudaSuccess ||
      (e = cudaFuncSetAttribute(kb_itx<6>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                4 * 4096 * (int)sizeof(int))) != cudaSuccess ||
      (e = cudaFuncSetAttribute(kb_itx<7>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                4 * 4096 * (int)sizeof(int))) != cudaSuccess)
    return e;
  /* load every batched kernel now (lazy loading would load one at its first
   * launch, inside a step, waiting for the kernels running) */
  cudaFuncAttributes fa;
  const void* ks[] = {
      reinterpret_cast<const void*>(kb_inter_simple<false>),
      reinterpret_cast<const void*>(kb_inter_simple<true>), reinterpret_cast<const void*>(kb_inter<3>),
      reinterpret_cast<const void*>(kb_inter<4>),
      reinterpret_cast<const void*>(kb_itx<2>), reinterpret_cast<const void*>(kb_itx<3>),
      reinterpret_cast<const void*>(kb_itx<4>), reinterpret_cast<const void*>(kb_itx<5>),
      reinterpret_cast<const void*>(kb_deblock), reinterpret_cast<const void*>(kb_copy),
      reinterpret_cast<const void*>(kb_cdef_search), reinterpret_cast<const void*>(kb_cdef),
      reinterpret_cast<const void*>(kb_upscale), reinterpret_cast<const void*>(kb_lr),
      reinterpret_cast<const void*>(kb_grain_template), reinterpret_cast<const void*>(kb_grain_blend),
      reinterpret_cast<const void*>(kb_nv12)};
  for (const void* k : ks)
    if ((e = cudaFuncGetAttributes(&fa, k)) != cudaSuccess) return e;
  return cudaSuccess;
}

int batch_stage_max_ctas(int stage) {
  const void* k = nullptr;
  int threads = 128;
  size_t smem = 0;
  switch (stage) {
    case kBInterSimple: k = reinterpret_cast<const void*>(kb_inter_simple<false>); break;
    case kBInterLeanMask: case kBInterMask: k = reinterpret_cast<const void*>(kb_inter_simple<true>); break;
    case kBInter: k = reinterpret_cast<const void*>(kb_inter<4>); break;
    case kBItx2: k = reinterpret_cast<const void*>(kb_itx<2>); smem = 4 * ItxScratch<2>::PER_WARP * sizeof(int); break;
    case kBItx3: k = reinterpret_cast<const void*>(kb_itx<3>); smem = 4 * ItxScratch<3>::PER_WARP * sizeof(int); break;
    case kBItx4: k = reinterpret_cast<const void*>(kb_itx<4>); smem = 4 * ItxScratch<4>::PER_WARP * sizeof(int); break;
    case kBItx5: k = reinterpret_cast<const void*>(kb_itx<5>); smem = 4 * ItxScratch<5>::PER_WARP * sizeof(int); break;
    case kBItx6: k = reinterpret_cast<const void*>(kb_itx<6>); smem = 4 * ItxScratch<6>::PER_WARP * sizeof(int); break;
    case kBItx7: k = reinterpret_cast<const void*>(kb_itx<7>); smem = 4 * ItxScratch<7>::PER_WARP * sizeof(int); break;
    case kBUnits: return AV1B_UNIT_CTAS_PER_SM;
    case kBDeblockV: case kBDeblockH: k = reinterpret_cast<const void*>(kb_deblock); threads = 256; break;
    case kBCopySnap: case kBCopyPost: case kBCopyRef: k = reinterpret_cast<const void*>(kb_copy); threads = 256; break;
    case kBCdefSearch: k = reinterpret_cast<const void*>(kb_cdef_search); break;
    case kBCdef: k = reinterpret_cast<const void*>(kb_cdef); break;
    case kBUpscale: k = reinterpret_cast<const void*>(kb_upscale); threads = 128; break;
    case kBLr: k = reinterpret_cast<const void*>(kb_lr); threads = 256; break;
    case kBGrainTemplate: k = reinterpret_cast<const void*>(kb_grain_template); threads = 256; break;
    case kBGrain: k = reinterpret_cast<const void*>(kb_grain_blend); break;
    case kBNv12: k = reinterpret_cast<const void*>(kb_nv12); break;
    default: return 1;
  }
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, threads, smem) != cudaSuccess || n < 1) return 1;
  return n;
}
