/*
 * plan_invariants.cu - host-only check of the planner's dependency schedule
 * (test infrastructure; no GPU needed).
 *
 * The planner source is compiled here with page-locked allocations replaced
 * by plain ones, and build_plan runs on seeded synthetic frames. For every
 * plan it checks what the device's phase B relies on to finish without a
 * cooperative launch:
 *   - the units are the frame's phase B blocks, each exactly once;
 *   - the chains partition the units, and a chain's blocks are in coding order;
 *   - every dependency of a block is an earlier phase B block, listed once,
 *     in ascending order, and lies earlier in the block's own chain or in a
 *     chain claimed before it (so the warp holding the earliest unfinished
 *     chain always progresses);
 * and that the records are the same whatever the number of host threads.
 * Prints one line per frame and "ok" at the end; exits non-zero on a failure.
 */
#include <cuda_runtime.h>
#include <cstdlib>
static cudaError_t plain_host_alloc(void** p, size_t n, unsigned) {
  *p = std::malloc(n ? n : 1);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
static cudaError_t plain_free_host(void* p) {
  std::free(p);
  return cudaSuccess;
}
#define cudaHostAlloc plain_host_alloc
#define cudaFreeHost plain_free_host
#include "decoder.cu"
#include "../../include/av1b_synth.h"
#undef cudaHostAlloc
#undef cudaFreeHost
#include <cstdio>

namespace {

using namespace av1b;

int failures = 0;

#define CHECK(cond, ...)                      \
  do {                                        \
    if (!(cond)) {                            \
      std::printf("FAIL: " __VA_ARGS__);      \
      std::printf("\n");                      \
      ++failures;                             \
      return;                                 \
    }                                         \
  } while (0)

uint64_t fnv(uint64_t h, const void* p, size_t n) {
  const uint8_t* b = static_cast<const uint8_t*>(p);
  for (size_t i = 0; i < n; ++i) {
    h ^= b[i];
    h *= 1099511628211ull;
  }
  return h;
}

template <class V>
uint64_t hash_list(uint64_t h, const V& v) {
  return fnv(h, v.data(), v.size() * sizeof(v[0]));
}

/* Plans one frame on `pool`; returns the hash of its record lists (0 when
 * planning failed). */
uint64_t plan_and_check(av1b_decoder* d, WorkPool* pool, uint8_t* blob, size_t len, int k,
                        const char* name) {
  int32_t refs[8];
  const int n = av1b_blob_get_refs(blob, len, refs, 8);
  int32_t slots[8];
  for (int i = 0; i < n; ++i) slots[i] = ((k - refs[i]) % 4 + 4) % 4;
  av1b_blob_set_refs(blob, len, slots, n);
  av1b_frame_syntax s;
  av1b_syntax_view(blob, len, &s);
  PlanCtx c;
  const int cw = (s.coded_width <= 0 || s.coded_width > s.width) ? s.width : s.coded_width;
  c.L = make_layout(s.width, s.height, cw, s.bit_depth, s.ss_x, s.ss_y);
  for (int i = 0; i < kSlots; ++i) {
    c.slot_used[i] = c.slot_valid[i] = i < 4;
    c.slot_width[i] = s.width;
    c.slot_height[i] = s.height;
  }
  PlanScratch scratch;
  PlanLists lists;
  c.pool = pool;
  c.scratch = &scratch;
  c.levels = s.n_levels > 0;
  c.n_levels = s.n_levels;
  c.n_qm = s.n_qm_pool;
  Plan P;
  P.R = &lists;
  const int rc = build_plan(d, c, s, &P);
  av1b_blob_set_refs(blob, len, refs, n);
  uint64_t h = 0;
  [&] {
    CHECK(rc == 0, "%s frame %d: planning failed (%d) %s", name, k, rc, d->err.c_str());
    const auto& B = lists.blocks;
    const auto& U = lists.units;
    const auto& C = lists.chains;
    const auto& D = lists.deps;
    size_t n_b = 0;
    for (size_t i = 0; i < B.size(); ++i) n_b += B[i].phase_b ? 1 : 0;
    CHECK(U.size() == n_b, "%s frame %d: %zu units for %zu phase B blocks", name, k, U.size(), n_b);
    CHECK(C.size() == P.n_chains + 1 && C[0] == 0 && static_cast<size_t>(C[P.n_chains]) == U.size(),
          "%s frame %d: chain offsets do not cover the units", name, k);
    std::vector<int> chain_of(B.size(), -1), place(B.size(), -1);
    for (size_t ch = 0; ch < P.n_chains; ++ch) {
      CHECK(C[ch] < C[ch + 1], "%s frame %d: chain %zu is empty", name, k, ch);
      for (int i = C[ch]; i < C[ch + 1]; ++i) {
        const int bi = U[i];
        CHECK(bi >= 0 && static_cast<size_t>(bi) < B.size() && B[bi].phase_b,
              "%s frame %d: unit %d is not a phase B block", name, k, bi);
        CHECK(chain_of[bi] < 0, "%s frame %d: block %d listed twice", name, k, bi);
        CHECK(i == C[ch] || U[i - 1] < bi, "%s frame %d: chain %zu out of coding order", name, k, ch);
        chain_of[bi] = static_cast<int>(ch);
        place[bi] = i;
      }
    }
    for (size_t i = 0; i < U.size(); ++i) {
      const int bi = U[i];
      const BlockRec& b = B[bi];
      CHECK(b.dep_first >= 0 && b.dep_count >= 0 &&
                static_cast<size_t>(b.dep_first) + b.dep_count <= D.size(),
            "%s frame %d: block %d's list is outside the dependency array", name, k, bi);
      for (int j = 0; j < b.dep_count; ++j) {
        const int o = D[b.dep_first + j];
        CHECK(o >= 0 && o < bi && B[o].phase_b, "%s frame %d: block %d waits for %d", name, k, bi, o);
        CHECK(j == 0 || D[b.dep_first + j - 1] < o, "%s frame %d: block %d's list is not ascending",
              name, k, bi);
        CHECK(chain_of[o] < chain_of[bi] || (chain_of[o] == chain_of[bi] && place[o] < place[bi]),
              "%s frame %d: block %d (chain %d) waits for %d in chain %d", name, k, bi, chain_of[bi],
              o, chain_of[o]);
      }
    }
    /* the prediction tiles: the lean kernel's unmasked tiles, its masked
     * ones (wedge, luma difference-weighted), the full kernel's (inter-intra,
     * chroma difference-weighted predicting its luma), then the chroma tiles
     * that read their luma block's mask - whose luma block writes it, at the
     * same place of the frame's mask pool */
    const auto& T = lists.inter_tiles;
    const size_t ns = P.n_tiles_simple, nl = P.n_tiles_lmask, nc = P.n_tiles_cmask;
    CHECK(ns + nl + nc <= T.size(), "%s frame %d: tile groups exceed the %zu tiles", name, k, T.size());
    std::vector<size_t> tiles_of(B.size(), 0);
    for (size_t i = 0; i < T.size(); ++i) {
      const int bi = T[i].x;
      CHECK(bi >= 0 && static_cast<size_t>(bi) < B.size() && !B[bi].phase_b && B[bi].is_inter,
            "%s frame %d: tile %zu names block %d, not a parallel inter block", name, k, i, bi);
      ++tiles_of[bi];
      const BlockRec& b = B[bi];
      const bool masked = b.compound && b.mask_kind;
      const bool full = b.interintra || (b.mask_kind == 2 && b.plane > 0 && b.mask_role != 2);
      const int group = i < ns ? 0 : (i < ns + nl ? 1 : (i < T.size() - nc ? 2 : 3));
      const int want = full ? 2 : (b.mask_role == 2 ? 3 : (masked ? 1 : 0));
      CHECK(group == want, "%s frame %d: tile %zu (block %d) in group %d, not %d", name, k, i, bi, group,
            want);
      if (b.mask_role) {
        CHECK(b.mask_off >= 0 && b.mask_w > 0 && static_cast<size_t>(b.mask_off) + static_cast<size_t>(b.mask_w) *
                                                           (b.mask_role == 1 ? b.h : (b.h << c.L.ss_y)) <=
                                                       P.mask_pool,
              "%s frame %d: block %d's mask lies outside the %zu-byte pool", name, k, bi, P.mask_pool);
      }
    }
    for (size_t bi = 0; bi < B.size(); ++bi) {
      const BlockRec& b = B[bi];
      if (b.phase_b || !b.is_inter) continue;
      const size_t want = static_cast<size_t>((b.w + 15) / 16) * ((b.h + 7) / 8);
      CHECK(tiles_of[bi] == want, "%s frame %d: block %zu has %zu tiles, not %zu", name, k, bi, tiles_of[bi],
            want);
    }
    /* the luma masks do not overlap in the pool */
    std::vector<std::pair<int, int>> spans;
    for (const BlockRec& b : B)
      if (b.mask_role == 1) spans.emplace_back(b.mask_off, b.mask_off + b.mask_w * b.h);
    std::sort(spans.begin(), spans.end());
    for (size_t i = 1; i < spans.size(); ++i)
      CHECK(spans[i - 1].second <= spans[i].first, "%s frame %d: two luma masks overlap in the pool", name, k);
    h = 1469598103934665603ull;
    h = hash_list(h, lists.blocks);
    h = hash_list(h, lists.txs);
    h = hash_list(h, lists.units);
    h = hash_list(h, lists.chains);
    h = hash_list(h, lists.deps);
    h = hash_list(h, lists.itx_jobs);
    h = hash_list(h, lists.itx_batches);
    h = hash_list(h, lists.inter_tiles);
    std::printf("%s frame %d: %zu blocks, %zu phase B in %zu chains, depth %d; tiles %zu lean, %zu lean "
                "masked, %zu full, %zu reading a luma mask\n",
                name, k, B.size(), U.size(), P.n_chains, P.unit_depth, ns, nl, T.size() - ns - nl - nc, nc);
  }();
  return h;
}

}  // namespace

int main() {
  av1b_decoder* d = new av1b_decoder;
  WorkPool one(1), several(5);
  struct Case {
    const char* name;
    int w, h, cw, bd, sb, tools, frames, key_interval;
  };
  const int all = (1 << 16) - 1 - (1 << 13);  /* every tool but lossless */
  const Case cases[] = {
      {"720p 8-bit", 1280, 720, 0, 8, 64, (1 << 5) - 1, 3, 30},
      {"1080p 10-bit all tools", 1920, 1080, 0, 10, 64, all, 3, 30},
      {"4K superres 128x128", 3840, 2160, 2880, 10, 128, all, 2, 30},
      {"odd size 12-bit", 998, 514, 750, 12, 128, all, 3, 2},
      {"small, every tool", 240, 136, 0, 10, 64, all | (1 << 11) | (1 << 12) | (1 << 14), 4, 30},
  };
  for (const Case& cs : cases) {
    for (int k = 0; k < cs.frames; ++k) {
      uint8_t* blob = nullptr;
      size_t len = 0;
      if (av1s_synth_frame_ex(cs.w, cs.h, cs.cw, cs.bd, cs.sb, cs.tools, 11, k, cs.key_interval, &blob,
                              &len) != AV1B_OK) {
        std::printf("FAIL: %s frame %d: no synthetic frame\n", cs.name, k);
        return 1;
      }
      const uint64_t h1 = plan_and_check(d, &one, blob, len, k, cs.name);
      const uint64_t h5 = plan_and_check(d, &several, blob, len, k, cs.name);
      if (h1 != h5) {
        std::printf("FAIL: %s frame %d: records differ between 1 and 5 host threads\n", cs.name, k);
        ++failures;
      }
      av1s_blob_free(blob);
    }
  }
  if (failures) {
    std::printf("%d failures\n", failures);
    return 1;
  }
  std::printf("ok\n");
  return 0;
}
