/*
 * server.cpp - the served form: a request loop over many streams.
 *
 * Streams are admitted by the device memory their decoder needs (pictures,
 * reference slots, planned frames; av1b_stream_hbm_estimate), which also
 * becomes that decoder's HBM budget, so an admitted stream can never take
 * more. Frame requests (serialized FrameSyntax, references as frame
 * distances) are planned as they arrive by a pool of host threads, and a
 * scheduler packs the planned frames into batched steps (av1b_batch_*:
 * persistent kernels over all the streams' frames, one CUDA graph replay a
 * step): continuous batching - a step takes every stream whose next frame is
 * planned at the moment it launches, one frame a stream, so frames that
 * arrive while a step runs join the next one, and a stream's frames run in
 * order in successive steps. At most `max_inflight` steps are queued on the
 * GPU at once, which bounds the wait of a frame that just missed a step.
 *
 * A frame's latency runs from its arrival (av1b_server_submit) to the device
 * completion of its step, on the host clock: the completion is the step's
 * CUDA event, placed on the host clock through a reference event recorded
 * when the server started (device time after it = host time of it + the
 * events' elapsed time). All reference pictures and outputs stay on the
 * device; a frame's NV12 pack lands in a ring of eight device buffers per
 * stream.
 *
 * The reference has no served form; its nearest mechanism is the pipelined
 * plan / decode API (include/av1gpu/av1gpu.hpp:656-689) and the one-stream
 * job loop of its DirectShow filter (dsfilter/decode_core.hpp:47-68).
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/av1b.h"

namespace {

using Clock = std::chrono::steady_clock;
constexpr int kOutRing = 8;        /* NV12 buffers a stream cycles through */
constexpr int kMaxRefs = 7;
constexpr int kPlanAhead = 4;      /* frames of a stream planned and not yet complete */
constexpr int kPlansAlive = 8;     /* a decoder's plans: kPlanAhead, or its pool of freed ones */

struct Request {
  int stream = -1;
  uint64_t tag = 0, index = 0;
  const uint8_t* blob = nullptr;   /* the caller's, read until the frame is planned */
  size_t len = 0;
  double arrival_ms = 0, planned_ms = 0;
  av1b_plan* plan = nullptr;
  int plan_rc = AV1B_OK;
  bool planned = false;
};

struct Stream {
  int id = -1;
  bool open = false;
  av1b_stream_desc desc{};
  av1b_decoder* dec = nullptr;
  int ring[kMaxRefs + 1];
  int ring_n = 0;
  size_t hbm = 0;
  uint64_t next_index = 0;       /* given to the next submitted frame */
  uint64_t next_launch = 0;      /* the next frame a step may take */
  std::deque<Request*> pending;  /* submitted, not yet in a step, in order */
  int planning = 0;              /* frames taken by a planner and not yet complete */
  double plan_cost_ms = 0;       /* expected planning time of one of its frames */
  uint8_t* nv12[kOutRing] = {nullptr};
  size_t nv12_bytes = 0;
  int in_steps = 0;              /* frames of the stream in steps not yet complete */
};

struct Step {
  uint64_t id = 0;
  cudaEvent_t ev = nullptr;
  std::vector<Request*> reqs;
  std::vector<int> slots;
  std::vector<int> rcs;          /* each frame's launch */
  int launch_rc = AV1B_OK;
};

}  // namespace

struct av1b_server {
  av1b_server_options opt{};
  av1b_batch* batch = nullptr;
  cudaStream_t bstream = nullptr;
  cudaEvent_t ref_ev = nullptr;
  Clock::time_point t0;
  double ref_ms = 0;             /* host time of ref_ev, ms since t0 */
  std::mutex mu;
  std::condition_variable cv_plan, cv_sched, cv_done, cv_result;
  std::vector<Stream*> streams;
  std::deque<Request*> plan_q;
  std::deque<Step*> done_q;
  std::deque<av1b_server_result> results;
  std::vector<cudaEvent_t> ev_pool;
  size_t hbm_used = 0, hbm_budget = 0;
  int inflight = 0;
  uint64_t submitted = 0, completed = 0, steps = 0, stepped_frames = 0;
  double plan_ms = 0, launch_ms = 0;
  bool stop = false;
  std::vector<std::thread> planners;
  std::thread sched, completer;
  std::string err;
};

namespace {

double now_ms(const av1b_server* s) {
  return std::chrono::duration<double, std::milli>(Clock::now() - s->t0).count();
}

void plan_loop(av1b_server* s) {
  for (;;) {
    Request* r = nullptr;
    Stream* st = nullptr;
    {
      /* the oldest request of a stream with fewer than kPlanAhead frames
       * planned and not complete: a stream whose requests pile up holds a
       * bounded number of plans (and so of device memory) */
      std::unique_lock<std::mutex> lk(s->mu);
      std::deque<Request*>::iterator it;
      /* of the requests whose stream may plan another frame, the one whose
       * plan is expected to finish first (arrival + a cost by frame size):
       * a small frame does not queue behind the plans of 4K frames that
       * arrived just before it, and a large one waits at most its own cost */
      auto pick = [&] {
        double best = 0;
        bool found = false;
        for (auto i = s->plan_q.begin(); i != s->plan_q.end(); ++i) {
          const Stream* q = s->streams[(*i)->stream];
          if (q->planning >= kPlanAhead) continue;
          const double key = (*i)->arrival_ms + q->plan_cost_ms;
          if (!found || key < best) {
            best = key;
            it = i;
            found = true;
          }
        }
        return found;
      };
      s->cv_plan.wait(lk, [&] { return s->stop || pick(); });
      if (s->stop) return;   /* requests left unplanned are freed with the server */
      r = *it;
      s->plan_q.erase(it);
      st = s->streams[r->stream];
      ++st->planning;
    }
    /* a view into the caller's blob, its references (frame distances)
     * mapped to the stream's ring of slots in an array of its own, so the
     * blob is only read (several streams may share one) */
    int rc = AV1B_OK;
    av1b_frame_syntax view;
    int32_t refs[8];
    if (av1b_syntax_view(r->blob, r->len, &view) || view.n_reference_slots > 8) rc = AV1B_ERR_SYNTAX;
    for (size_t i = 0; rc == AV1B_OK && i < view.n_reference_slots; ++i) {
      const int32_t dist = view.reference_slots[i];
      if (dist < 0) {
        refs[i] = -1;   /* an unused entry */
        continue;
      }
      if (dist < 1 || static_cast<uint64_t>(dist) > r->index || dist >= st->ring_n) {
        rc = AV1B_ERR_SYNTAX;
        break;
      }
      refs[i] = st->ring[(r->index - dist) % st->ring_n];
    }
    const double t0 = now_ms(s);
    if (rc == AV1B_OK) {
      view.reference_slots = refs;
      /* returns once the frame's records and coefficients are on the device */
      rc = av1b_plan_frame(st->dec, &view, &r->plan);
    }
    {
      std::lock_guard<std::mutex> lk(s->mu);
      r->planned = true;
      r->plan_rc = rc;
      r->planned_ms = now_ms(s);
      s->plan_ms += r->planned_ms - t0;
    }
    s->cv_sched.notify_one();
  }
}

Stream* st_of(av1b_server* s, const Request* r) { return s->streams[r->stream]; }

cudaEvent_t take_event(av1b_server* s) {
  if (!s->ev_pool.empty()) {
    cudaEvent_t e = s->ev_pool.back();
    s->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

void post_result(av1b_server* s, const Request* r, int status, double done_ms, int slot, int batch,
                 uint64_t step) {
  av1b_server_result res{};
  Stream* st = s->streams[r->stream];
  res.stream_id = r->stream;
  res.status = status;
  res.tag = r->tag;
  res.frame_index = r->index;
  res.arrival_ms = r->arrival_ms;
  res.done_ms = done_ms;
  res.latency_ms = done_ms - r->arrival_ms;
  res.planned_ms = r->planned_ms;
  res.slot = slot;
  res.batch_size = batch;
  res.step = static_cast<int64_t>(step);
  res.nv12_device = st->nv12[0] ? st->nv12[r->index % kOutRing] : nullptr;
  res.nv12_bytes = st->nv12_bytes;
  s->results.push_back(res);
}

void sched_loop(av1b_server* s) {
  cudaSetDevice(s->opt.device);
  for (;;) {
    Step* step = new Step;
    std::vector<Request*> failed;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      auto ready = [&](const Stream* st) {
        return st->open && !st->pending.empty() && st->pending.front()->planned &&
               st->pending.front()->index == st->next_launch;
      };
      auto any_ready = [&] {
        for (const Stream* st : s->streams)
          if (st && ready(st)) return true;
        return false;
      };
      s->cv_sched.wait(lk, [&] { return s->stop || (s->inflight < s->opt.max_inflight && any_ready()); });
      if (s->stop) {
        delete step;
        return;
      }
      /* a batching window: with a step already queued on the GPU, a new one
       * waits (up to batch_wait_us, or until the queued one completes) for a
       * quarter of the open streams to have their next frame ready, so that
       * steps do not shrink to a frame or two while the GPU is busy anyway */
      if (s->inflight > 0 && s->opt.batch_wait_us > 0) {
        auto count = [&] {
          int ready_n = 0, open_n = 0;
          for (const Stream* st : s->streams)
            if (st && st->open) {
              ++open_n;
              ready_n += ready(st);
            }
          return ready_n * 4 >= open_n;
        };
        const int before = s->inflight;
        s->cv_sched.wait_for(lk, std::chrono::microseconds(s->opt.batch_wait_us),
                             [&] { return s->stop || s->inflight < before || count(); });
        if (s->stop) {
          delete step;
          return;
        }
      }
      /* the oldest frames first, one a stream */
      std::vector<Stream*> cand;
      for (Stream* st : s->streams)
        if (st && ready(st)) cand.push_back(st);
      std::sort(cand.begin(), cand.end(), [](const Stream* a, const Stream* b) {
        return a->pending.front()->arrival_ms < b->pending.front()->arrival_ms;
      });
      for (Stream* st : cand) {
        if (static_cast<int>(step->reqs.size()) >= s->opt.max_batch) break;
        Request* r = st->pending.front();
        st->pending.pop_front();
        ++st->next_launch;
        if (r->plan_rc != AV1B_OK) {
          failed.push_back(r);
          continue;
        }
        ++st->in_steps;
        step->reqs.push_back(r);
      }
      for (Request* r : failed) {
        post_result(s, r, r->plan_rc, now_ms(s), -1, 0, 0);
        --st_of(s, r)->planning;
      }
      if (!failed.empty()) s->cv_plan.notify_all();
      s->completed += failed.size();
      if (!failed.empty()) s->cv_result.notify_all();
      if (step->reqs.empty()) {
        delete step;
        for (Request* r : failed) delete r;
        continue;
      }
      ++s->inflight;
      step->ev = take_event(s);
      step->id = s->steps++;
    }
    for (Request* r : failed) delete r;
    const int n = static_cast<int>(step->reqs.size());
    std::vector<av1b_decoder*> decs(n);
    std::vector<av1b_plan*> plans(n);
    std::vector<int> slots(n), out(n, -1);
    std::vector<uint8_t*> nv(n);
    std::vector<size_t> pitch(n), len(n);
    for (int i = 0; i < n; ++i) {
      const Request* r = step->reqs[i];
      const Stream* st = s->streams[r->stream];
      decs[i] = st->dec;
      plans[i] = r->plan;
      slots[i] = st->ring[r->index % st->ring_n];
      nv[i] = st->nv12[0] ? st->nv12[r->index % kOutRing] : nullptr;
      pitch[i] = static_cast<size_t>(st->desc.nv12_pitch);
      len[i] = st->nv12_bytes;
    }
    const double t0 = now_ms(s);
    step->launch_rc = av1b_batch_decode(s->batch, n, decs.data(), plans.data(), slots.data(), out.data(),
                                        nv.data(), pitch.data(), len.data());
    step->rcs.assign(n, step->launch_rc);
    if (step->launch_rc != AV1B_OK && n > 1) {
      /* a frame the step could not take (checked before anything was
       * launched) fails alone: the others run as steps of their own */
      step->launch_rc = AV1B_OK;
      for (int i = 0; i < n; ++i)
        step->rcs[i] = av1b_batch_decode(s->batch, 1, &decs[i], &plans[i], &slots[i], &out[i], &nv[i],
                                         &pitch[i], &len[i]);
    }
    step->slots = out;
    cudaEventRecord(step->ev, s->bstream);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->stepped_frames += n;
      s->launch_ms += now_ms(s) - t0;
      s->done_q.push_back(step);
    }
    s->cv_done.notify_one();
  }
}

void done_loop(av1b_server* s) {
  cudaSetDevice(s->opt.device);
  for (;;) {
    Step* step = nullptr;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_done.wait(lk, [&] { return !s->done_q.empty() || (s->stop && s->done_q.empty()); });
      if (s->done_q.empty()) return;
      step = s->done_q.front();
      s->done_q.pop_front();
    }
    int rc = step->launch_rc;
    const cudaError_t e = cudaEventSynchronize(step->ev);
    if (rc == AV1B_OK && e != cudaSuccess) rc = AV1B_ERR_CUDA;
    float ms = 0.f;
    double done_ms = now_ms(s);
    if (e == cudaSuccess && cudaEventElapsedTime(&ms, s->ref_ev, step->ev) == cudaSuccess)
      done_ms = s->ref_ms + ms;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      const int n = static_cast<int>(step->reqs.size());
      for (int i = 0; i < n; ++i) {
        Request* r = step->reqs[i];
        post_result(s, r, rc != AV1B_OK ? rc : step->rcs[i], done_ms, step->slots[i], n, step->id);
        --s->streams[r->stream]->in_steps;
        --s->streams[r->stream]->planning;
      }
      s->completed += n;
      --s->inflight;
      s->ev_pool.push_back(step->ev);
    }
    for (Request* r : step->reqs) {
      av1b_plan_free(s->streams[r->stream]->dec, r->plan);
      delete r;
    }
    delete step;
    s->cv_sched.notify_one();
    s->cv_plan.notify_all();
    s->cv_result.notify_all();
  }
}

}  // namespace

extern "C" {

int av1b_server_create(const av1b_server_options* options, av1b_server** out) {
  if (!out) return AV1B_ERR_ARG;
  *out = nullptr;
  av1b_server_options o{};
  if (options) o = *options;
  if (o.max_batch <= 0) o.max_batch = AV1B_BATCH_MAX;
  if (o.max_inflight <= 0) o.max_inflight = 2;
  if (o.max_batch > AV1B_BATCH_MAX || o.max_inflight > 8 || o.planner_threads < 0 ||
      o.planner_threads > 64 || o.decoder_threads < 0 || o.decoder_threads > 64)
    return AV1B_ERR_ARG;
  if (o.planner_threads == 0) {
    const unsigned hc = std::thread::hardware_concurrency();
    o.planner_threads = static_cast<int>(std::max(2u, hc / 2));
  }
  if (o.batch_wait_us == 0) o.batch_wait_us = 1000;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return AV1B_ERR_NO_DEVICE;
  if (o.device < 0 || o.device >= ndev) return AV1B_ERR_ARG;
  if (cudaSetDevice(o.device) != cudaSuccess) return AV1B_ERR_CUDA;
  auto* s = new av1b_server;
  s->opt = o;
  s->t0 = Clock::now();
  if (o.hbm_budget == 0) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
      delete s;
      return AV1B_ERR_CUDA;
    }
    s->hbm_budget = free_b / 10 * 9;
  } else {
    s->hbm_budget = o.hbm_budget;
  }
  int rc = av1b_batch_create(o.device, &s->batch);
  if (rc) {
    delete s;
    return rc;
  }
  s->bstream = static_cast<cudaStream_t>(av1b_batch_stream(s->batch));
  if (cudaEventCreate(&s->ref_ev) != cudaSuccess || cudaEventRecord(s->ref_ev, s->bstream) != cudaSuccess ||
      cudaEventSynchronize(s->ref_ev) != cudaSuccess) {
    av1b_batch_destroy(s->batch);
    delete s;
    return AV1B_ERR_CUDA;
  }
  s->ref_ms = now_ms(s);
  for (int i = 0; i < o.planner_threads; ++i) s->planners.emplace_back(plan_loop, s);
  s->sched = std::thread(sched_loop, s);
  s->completer = std::thread(done_loop, s);
  *out = s;
  return AV1B_OK;
}

int av1b_server_destroy(av1b_server* s) {
  if (!s) return AV1B_ERR_ARG;
  av1b_server_drain(s, 60000);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_plan.notify_all();
  s->cv_sched.notify_all();
  s->cv_done.notify_all();
  for (auto& t : s->planners) t.join();
  s->sched.join();
  s->completer.join();
  cudaSetDevice(s->opt.device);
  av1b_batch_sync(s->batch);
  for (Stream* st : s->streams) {
    if (!st) continue;
    for (Request* r : st->pending) {
      if (r->plan) av1b_plan_free(st->dec, r->plan);
      delete r;
    }
    for (auto* p : st->nv12)
      if (p) cudaFree(p);
    if (st->dec) av1b_decoder_destroy(st->dec);
    delete st;
  }
  for (Request* r : s->plan_q) delete r;
  for (cudaEvent_t e : s->ev_pool) cudaEventDestroy(e);
  if (s->ref_ev) cudaEventDestroy(s->ref_ev);
  av1b_batch_destroy(s->batch);
  delete s;
  return AV1B_OK;
}

int av1b_server_open(av1b_server* s, const av1b_stream_desc* desc, int* stream_id, size_t* hbm_bytes) {
  if (!s || !desc || !stream_id) return AV1B_ERR_ARG;
  const av1b_stream_desc& d = *desc;
  if (d.width <= 0 || d.height <= 0 || d.max_refs < 1 || d.max_refs > kMaxRefs || d.nv12_pitch < 0)
    return AV1B_ERR_ARG;
  const int ring_n = d.max_refs + 1;
  const size_t nv12 = d.nv12_pitch ? av1b_nv12_size(d.width, d.height, d.ss_x, d.ss_y, d.nv12_pitch) : 0;
  if (d.nv12_pitch && !nv12) return AV1B_ERR_ARG;
  /* the decoder's pictures, slots and up to kPlansAlive plans, plus the
   * output ring */
  const size_t need = av1b_stream_hbm_estimate(d.width, d.height, d.coded_width, d.bit_depth, d.ss_x,
                                               d.ss_y, ring_n, kPlansAlive) +
                      kOutRing * nv12;
  if (hbm_bytes) *hbm_bytes = need;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->hbm_used + need > s->hbm_budget) return AV1B_ERR_NOMEM;   /* not admitted now */
    s->hbm_used += need;
  }
  auto* st = new Stream;
  st->desc = d;
  st->ring_n = ring_n;
  st->hbm = need;
  /* planner threads by frame size (0: a thread per 0.7 million samples, 1..6) */
  const double px = static_cast<double>(d.width) * d.height;
  const int threads = s->opt.decoder_threads > 0
                          ? s->opt.decoder_threads
                          : std::min(6, std::max(1, static_cast<int>(px / 0.7e6 + 0.5)));
  st->plan_cost_ms = px * 1.6e-6 / std::min(threads, 4);
  av1b_decoder_options dopt{1, threads};
  int rc = av1b_decoder_create_ex(s->opt.device, need - kOutRing * nv12, &dopt, &st->dec);
  for (int i = 0; rc == AV1B_OK && i < ring_n; ++i) rc = av1b_reserve_reference(st->dec, &st->ring[i]);
  if (rc == AV1B_OK && nv12) {
    st->nv12_bytes = nv12;
    for (auto*& p : st->nv12)
      if (cudaMalloc(&p, nv12) != cudaSuccess) rc = AV1B_ERR_NOMEM;
  }
  if (rc) {
    for (auto* p : st->nv12)
      if (p) cudaFree(p);
    if (st->dec) av1b_decoder_destroy(st->dec);
    delete st;
    std::lock_guard<std::mutex> lk(s->mu);
    s->hbm_used -= need;
    return rc;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  int id = -1;
  for (size_t i = 0; i < s->streams.size(); ++i)
    if (!s->streams[i]) {
      id = static_cast<int>(i);
      break;
    }
  if (id < 0) {
    id = static_cast<int>(s->streams.size());
    s->streams.push_back(nullptr);
  }
  st->id = id;
  st->open = true;
  s->streams[id] = st;
  *stream_id = id;
  return AV1B_OK;
}

int av1b_server_close(av1b_server* s, int id) {
  if (!s) return AV1B_ERR_ARG;
  Stream* st = nullptr;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    if (id < 0 || id >= static_cast<int>(s->streams.size()) || !s->streams[id]) return AV1B_ERR_ARG;
    st = s->streams[id];
    /* its frames finish first */
    s->cv_result.wait(lk, [&] { return st->pending.empty() && st->in_steps == 0; });
    st->open = false;
    s->streams[id] = nullptr;
    s->hbm_used -= st->hbm;
  }
  av1b_sync(st->dec);
  for (auto* p : st->nv12)
    if (p) cudaFree(p);
  av1b_decoder_destroy(st->dec);
  delete st;
  return AV1B_OK;
}

int av1b_server_submit(av1b_server* s, int id, const uint8_t* blob, size_t len, uint64_t tag) {
  if (!s || !blob || !len) return AV1B_ERR_ARG;
  auto* r = new Request;
  r->arrival_ms = now_ms(s);
  r->tag = tag;
  r->blob = blob;
  r->len = len;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (id < 0 || id >= static_cast<int>(s->streams.size()) || !s->streams[id] || !s->streams[id]->open) {
      delete r;
      return AV1B_ERR_ARG;
    }
    Stream* st = s->streams[id];
    r->stream = id;
    r->index = st->next_index++;
    st->pending.push_back(r);
    s->plan_q.push_back(r);
    ++s->submitted;
  }
  s->cv_plan.notify_one();
  return AV1B_OK;
}

int av1b_server_poll(av1b_server* s, av1b_server_result* out, int max, int wait_ms, int* n) {
  if (!s || !n || (max > 0 && !out)) return AV1B_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  if (s->results.empty() && wait_ms > 0)
    s->cv_result.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->results.empty(); });
  int k = 0;
  while (k < max && !s->results.empty()) {
    out[k++] = s->results.front();
    s->results.pop_front();
  }
  *n = k;
  return AV1B_OK;
}

int av1b_server_drain(av1b_server* s, int timeout_ms) {
  if (!s) return AV1B_ERR_ARG;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    const bool done = s->cv_result.wait_for(lk, std::chrono::milliseconds(timeout_ms),
                                            [&] { return s->completed == s->submitted; });
    if (!done) return AV1B_ERR_TIMEOUT;
  }
  /* every decoder's device status: a dependency wait that gave up fails here */
  std::vector<av1b_decoder*> decs;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (Stream* st : s->streams)
      if (st) decs.push_back(st->dec);
  }
  int first = AV1B_OK;
  for (av1b_decoder* d : decs) {
    const int rc = av1b_sync(d);
    if (rc && first == AV1B_OK) first = rc;
  }
  return first;
}

int av1b_server_get_stats(av1b_server* s, av1b_server_stats* out) {
  if (!s || !out) return AV1B_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(out, 0, sizeof(*out));
  out->submitted = s->submitted;
  out->completed = s->completed;
  out->steps = s->steps;
  out->stepped_frames = s->stepped_frames;
  out->hbm_used = s->hbm_used;
  out->hbm_budget = s->hbm_budget;
  out->now_ms = now_ms(s);
  out->plan_ms = s->plan_ms;
  out->launch_ms = s->launch_ms;
  for (const Stream* st : s->streams)
    if (st) ++out->streams;
  return AV1B_OK;
}

void* av1b_server_batch(av1b_server* s) { return s ? s->batch : nullptr; }

}  // extern "C"
