// Request server for depth solves of mixed sizes (the serving form of the stage; its admission rule is the one of
// Lux.Library's job queue, Lux.Library/Core/JobQueue.cs:23-28 and Dispatch :474-531).
//
// Requests wait in a queue ordered by priority (lower first), then by arrival. Whenever a worker is free the dispatcher
// walks that order and starts the first request that may start: one whose estimated device memory fits what the running
// requests leave of the HBM budget (or any request when nothing runs). A heavy request (estimate above 1.5 GiB, the
// queue's LightBytes) that does not fit holds back every heavy request behind it, so heavy requests never overtake each
// other, while light ones (previews) may pass it. On the GPU one heavy request runs at a time (a heavy solve fills every
// SM; two side by side only interleave): a heavy request waits while another one runs, as if it did not fit. Requests run on `slots` worker contexts (each its own CUDA stream,
// error word and events, all drawing on the device's memory pool), so requests that arrive while others are on the GPU
// start as soon as a slot and memory are free and their work overlaps on the device with the host-side work (copies,
// planes, schedules) of the others. A request is one layer solved exactly as lux_sgm_layer solves it (prefilter
// included), its depth map read back into the caller's host buffer; the server adds no arithmetic of its own, so every
// result equals the same request run alone.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/lux_sgm.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Pending {
  uint64_t ticket = 0;
  std::vector<lux_img_rgba8> images;
  std::vector<uint8_t> gray;
  std::vector<lux_calib> calibs;
  float near_ = 0.f, far_ = 0.f;
  lux_stereo_params params{};
  int32_t flags = 0;
  float* out_depth = nullptr;
  uint64_t out_bytes = 0;
  uint64_t estimate = 0;
  int32_t priority = 0;
  Clock::time_point submitted, started;
};

constexpr uint64_t kLightBytes = 3ull << 29;  // 1.5 GiB: JobQueue.LightBytes (JobQueue.cs:47)

struct Done {
  lux_result result{};
  bool done = false;
};

}  // namespace

struct lux_server {
  int device = 0;
  uint64_t budget = 0;  // 0: no limit
  std::vector<lux_sgm_ctx*> ctxs;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Pending> queue;
  std::unordered_map<uint64_t, Done> results;
  uint64_t next_ticket = 1;
  uint64_t in_use = 0;  // estimated device bytes of the requests running
  int running = 0;
  int heavy_running = 0;  // requests above kLightBytes on the GPU (at most one)
  bool stop = false;
  std::string last_error;
  uint64_t passed = 0;  // requests started ahead of an earlier-queued request that had to wait
};

namespace {

// Device bytes a request needs, estimated from its sizes: the cost volume and aggregates of its layer (volume = pixels x
// planes, 3 bytes each, plus 2 per kept aggregate set), per-pixel tables and the aggregation scratch (about 100 bytes a
// pixel), the filtered images and half-pixel phase images (40 bytes a pixel per camera), and 64 MiB of slack.
uint64_t estimate_bytes(const Pending& p) {
  const int sc = p.params.scale > 0 ? p.params.scale : 1;
  const uint64_t W = (uint64_t)((p.images[0].w + sc - 1) / sc), H = (uint64_t)((p.images[0].h + sc - 1) / sc);
  std::vector<float> planes(4096 + 64);
  int32_t n = 0;
  if (lux_sgm_planes(p.near_, p.far_, p.calibs.data(), (int32_t)p.calibs.size(), p.params.plane_density, 8, planes.data(), &n) !=
      LUX_OK)
    n = 256;
  const uint64_t vol = W * H * (uint64_t)n;
  uint64_t b = vol * 3 + W * H * 100 + (64ull << 20);
  if (p.flags & LUX_LAYER_KEEP_PASS1) b += vol * 2;
  for (const auto& im : p.images) b += (uint64_t)im.w * im.h * 40;
  return b;
}

// The request a free worker starts (JobQueue.Dispatch, JobQueue.cs:496-521): the queue is kept in (priority, arrival)
// order; the first request whose memory fits starts, a heavy one that does not fit blocks the heavy ones behind it.
// Returns the index in the queue, or -1 when nothing may start now.
long pick(const lux_server* s) {
  const bool anything = s->in_use > 0 || s->running > 0;
  bool heavy_blocked = false;
  for (size_t i = 0; i < s->queue.size(); i++) {
    const Pending& p = s->queue[i];
    const bool heavy = p.estimate > kLightBytes;
    if (heavy && heavy_blocked) continue;
    const bool fits = s->budget == 0 || s->in_use + p.estimate <= s->budget;
    // one heavy request on the GPU at a time: a heavy solve's launches fill every SM, and two of them side by side
    // only interleave their blocks (measured: two 13 MP solves at once took 0.3-1.3 s each instead of 36 ms)
    if ((anything && !fits) || (heavy && s->heavy_running > 0)) {
      if (heavy) heavy_blocked = true;
      continue;
    }
    return (long)i;
  }
  return -1;
}

void worker(lux_server* s, lux_sgm_ctx* ctx) {
  for (;;) {
    Pending p;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      long i = -1;
      s->cv_work.wait(lk, [&] { return (s->stop && s->queue.empty()) || (i = pick(s)) >= 0; });
      if (i < 0) return;  // stop with nothing left
      if (i > 0) s->passed++;
      p = std::move(s->queue[(size_t)i]);
      s->queue.erase(s->queue.begin() + i);
      s->in_use += p.estimate;
      s->running++;
      if (p.estimate > kLightBytes) s->heavy_running++;
    }
    p.started = Clock::now();
    lux_result r{};
    lux_layer* L = nullptr;
    // The aggregation form by size (path-group chains from about 2 MP, the fused wavefront below), unless the request
    // names one: the autotuner's choices are timed on an idle GPU, and beside other requests they need not be the best
    // (measured in the 60/s mixed stream: the lean wavefront for the 520x390 previews, their solo choice, gave a served
    // p99 of 441 ms, the fused wavefront 181 ms).
    int32_t flags = p.flags | LUX_LAYER_PREFILTER;
    if (!(flags & (LUX_LAYER_SGM_FUSED | LUX_LAYER_SGM_SPLIT | LUX_LAYER_SGM_WAVE))) {
      const int sc = p.params.scale > 0 ? p.params.scale : 1;
      const int64_t w = (p.images[0].w + sc - 1) / sc, h = (p.images[0].h + sc - 1) / sc;
      flags |= w * h >= 2000000 ? LUX_LAYER_SGM_SPLIT : LUX_LAYER_SGM_FUSED;
    }
    r.status = lux_sgm_layer(ctx, (int32_t)p.images.size(), p.images.data(), p.gray.data(), p.calibs.data(), p.near_, p.far_,
                             &p.params, 0, 8, nullptr, flags, &L);
    if (r.status == LUX_OK) {
      lux_layer_info info{};
      lux_layer_get_info(L, &info);
      r.w = info.w;
      r.h = info.h;
      r.n_planes = info.n_planes;
      if (p.out_depth) r.status = lux_layer_read(L, LUX_FIELD_DEPTH, p.out_depth, p.out_bytes);
    }
    if (L) lux_layer_destroy(L);
    const auto end = Clock::now();
    r.queue_ms = std::chrono::duration<double, std::milli>(p.started - p.submitted).count();
    r.run_ms = std::chrono::duration<double, std::milli>(end - p.started).count();
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->in_use -= p.estimate;
      s->running--;
      if (p.estimate > kLightBytes) s->heavy_running--;
      Done& d = s->results[p.ticket];
      d.result = r;
      d.done = true;
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
  }
}

}  // namespace

extern "C" {

int lux_server_create(int device, uint64_t hbm_budget_bytes, int32_t slots, lux_server** out) {
  if (!out || slots < 1 || slots > 16) return LUX_ERR_ARG;
  *out = nullptr;
  lux_server* s = new lux_server();
  s->device = device;
  s->budget = hbm_budget_bytes;
  for (int i = 0; i < slots; i++) {
    lux_sgm_ctx* c = nullptr;
    const int rc = lux_sgm_create(device, 0, &c);
    if (rc) {
      for (auto* x : s->ctxs) lux_sgm_destroy(x);
      delete s;
      return rc;
    }
    // Workers do not time the aggregation forms: on a GPU shared with the other workers' requests the timings would
    // measure the contention, not the form (requests pick their form by size, see worker()).
    lux_sgm_set_autotune(c, 0);
    s->ctxs.push_back(c);
  }
  for (auto* c : s->ctxs) s->workers.emplace_back(worker, s, c);
  *out = s;
  return LUX_OK;
}

void lux_server_destroy(lux_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();
  for (auto* c : s->ctxs) lux_sgm_destroy(c);
  delete s;
}

const char* lux_server_last_error(const lux_server* s) { return s ? s->last_error.c_str() : "no server"; }

int lux_server_submit(lux_server* s, const lux_request* req, uint64_t* ticket) {
  if (!s || !req || !ticket || req->n_cams < 2 || req->n_cams > 16 || !req->images || !req->calibs) return LUX_ERR_ARG;
  Pending p;
  p.images.assign(req->images, req->images + req->n_cams);
  p.gray.assign((size_t)req->n_cams, 0);
  if (req->gray) std::memcpy(p.gray.data(), req->gray, (size_t)req->n_cams);
  p.calibs.assign(req->calibs, req->calibs + req->n_cams);
  p.near_ = req->near_;
  p.far_ = req->far_;
  p.params = req->params;
  p.flags = req->flags;
  p.out_depth = req->out_depth;
  p.out_bytes = req->out_bytes;
  p.estimate = estimate_bytes(p);
  p.priority = req->priority;
  p.submitted = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return LUX_ERR_CANCELED;
    p.ticket = s->next_ticket++;
    *ticket = p.ticket;
    s->results[p.ticket] = Done{};
    // insert after every waiting request of the same or a lower priority value (priority, then arrival)
    auto at = s->queue.end();
    while (at != s->queue.begin() && (at - 1)->priority > p.priority) --at;
    s->queue.insert(at, std::move(p));
  }
  s->cv_work.notify_all();
  return LUX_OK;
}

int lux_server_estimate(const lux_request* req, uint64_t* bytes) {
  if (!req || !bytes || req->n_cams < 2 || req->n_cams > 16 || !req->images || !req->calibs) return LUX_ERR_ARG;
  Pending p;
  p.images.assign(req->images, req->images + req->n_cams);
  p.calibs.assign(req->calibs, req->calibs + req->n_cams);
  p.near_ = req->near_;
  p.far_ = req->far_;
  p.params = req->params;
  p.flags = req->flags;
  *bytes = estimate_bytes(p);
  return LUX_OK;
}

uint64_t lux_server_passed(const lux_server* s) {
  if (!s) return 0;
  std::lock_guard<std::mutex> lk(const_cast<lux_server*>(s)->mu);
  return s->passed;
}

int lux_server_cancel(lux_server* s, uint64_t ticket) {
  if (!s) return LUX_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->results.find(ticket);
    if (it == s->results.end()) {
      s->last_error = "unknown ticket";
      return LUX_ERR_ARG;
    }
    size_t i = 0;
    while (i < s->queue.size() && s->queue[i].ticket != ticket) i++;
    if (i == s->queue.size()) {  // running or finished: a started request runs to its end
      s->last_error = "the request has started";
      return LUX_ERR_CANCELED;
    }
    s->queue.erase(s->queue.begin() + (long)i);
    lux_result r{};
    r.status = LUX_ERR_CANCELED;
    it->second.result = r;
    it->second.done = true;
  }
  s->cv_done.notify_all();
  s->cv_work.notify_all();  // a heavy request held back behind it may start now
  return LUX_OK;
}

int lux_server_wait(lux_server* s, uint64_t ticket, uint64_t timeout_ns, lux_result* out) {
  if (!s) return LUX_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->results.find(ticket);
  if (it == s->results.end()) {
    s->last_error = "unknown ticket";
    return LUX_ERR_ARG;
  }
  auto ready = [&] { return s->results[ticket].done; };
  if (timeout_ns == 0) s->cv_done.wait(lk, ready);
  else if (!s->cv_done.wait_for(lk, std::chrono::nanoseconds(timeout_ns), ready)) return LUX_ERR_TIMEOUT;
  if (out) *out = s->results[ticket].result;
  s->results.erase(ticket);
  return LUX_OK;
}

}  // extern "C"
