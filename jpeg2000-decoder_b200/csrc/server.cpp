// server.cpp — continuous-batching decode service (include/j2k_server.h).
//
// Pipeline: a fixed number of slots, each a device context (its own stream and device
// buffer pool); decoded pictures land in pinned host buffers recycled across requests.
// The scheduler thread loops over
//   1. completions: a slot whose end-of-batch event has fired hands every request its
//      status (the output was copied into the request's pinned buffer on the slot's
//      stream) and becomes free;
//   2. admissions: while requests are pending and a slot is free, the oldest pending
//      requests that fit the slot's share of the memory budget form one batch (one Tier-1
//      launch, shared DWT level launches), whose decode and output copies are enqueued
//      on the slot's stream;
// and sleeps on the submit condition only when neither step had work.  Requests that
// arrive while batches run therefore join the next free slot, and up to `pipeline_depth`
// batches overlap on the device (staging and output copies of one with the kernels of
// another; the engine starts a batch whose Tier-1 fills the GPU only after the previous
// decode, see j2k_gpu_batch_run).
#include "../../include/j2k_server.h"
#include "pinned_arena.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/j2k_gpu.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  int64_t id = 0;
  std::vector<uint8_t> cs;
  int fmt = 0, flags = 0;
  j2k_plan *plan = nullptr;
  j2k_image_info info{};
  size_t out_bytes = 0, footprint = 0;
  bool done = false;
  int status = J2K_OK;
  uint8_t *out = nullptr;  // pinned, from the server's pool
  Clock::time_point t_submit, t_done;
};

// Pinned host memory for decoded pictures: pieces of page-locked chunks, recycled between
// requests of any size (pinned_arena.h)
void *page_locked_alloc(size_t n) {
  void *p = nullptr;
  if (cudaMallocHost(&p, n) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}
void page_locked_free(void *p) { cudaFreeHost(p); }
typedef j2k::PinnedArena<void *(*)(size_t), void (*)(void *)> PinnedPool;

struct Slot {
  j2k_gpu_ctx *ctx = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t done_ev = nullptr;  // end of the decode and of the output copies
  std::vector<Request *> reqs;
  bool busy = false;
};

size_t estimate_footprint(const j2k_image_info &I, size_t out_bytes) {
  // the device pool of one batch: coded bytes, block table + order + status, segment
  // lengths, three coefficient buffers, packed output (j2k_gpu_batch_footprint), plus
  // the DWT / output task tables and alignment
  size_t b = I.coded_bytes + (size_t)I.num_cblks * (sizeof(j2k_cblk) + 6) + (size_t)I.num_segs * 4 +
             (size_t)I.coef_elems * 12 + out_bytes;
  return b + b / 32 + (64 << 10);
}

}  // namespace

struct j2k_server {
  j2k_server_config cfg{};
  size_t slot_budget = 0;
  std::vector<Slot> slots;
  PinnedPool pinned{page_locked_alloc, page_locked_free};
  std::mutex mu;
  std::condition_variable cv_submit, cv_done;
  std::deque<Request *> pending;
  std::unordered_map<int64_t, Request *> reqs;
  int64_t next_id = 0;
  uint64_t outstanding = 0;
  bool stop = false;
  std::thread sched;
  // statistics
  std::vector<double> lat_us;
  uint64_t completed = 0, failed = 0, batches = 0, batch_images = 0, pixels = 0, launches = 0;
  double busy_s = 0, gpu_ms = 0, stage_ms = 0, enqueue_ms = 0;
  uint64_t pool_growths = 0, pinned_allocs = 0;
  Clock::time_point busy_since;
  int inflight = 0;

  void run();
  bool complete_ready();
  bool admit();
  int launch(Slot &s, std::vector<Request *> &batch);
};

int j2k_server::launch(Slot &s, std::vector<Request *> &batch) {
  int rc = j2k_gpu_batch_begin(s.ctx);
  for (size_t i = 0; rc == J2K_OK && i < batch.size(); ++i) {
    int slot = -1;
    rc = j2k_gpu_batch_add(s.ctx, batch[i]->plan, batch[i]->fmt, batch[i]->flags, &slot);
  }
  size_t before = 0, after = 0, budget = 0;
  j2k_gpu_mem_usage(s.ctx, &before, &budget);
  const Clock::time_point t0 = Clock::now();
  if (rc == J2K_OK) rc = j2k_gpu_batch_launch(s.ctx, s.stream);
  const double ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
  j2k_gpu_mem_usage(s.ctx, &after, &budget);
  {
    std::lock_guard<std::mutex> lk(mu);
    enqueue_ms += ms;
    if (after > before) pool_growths++;
  }
  if (rc != J2K_OK) return rc;
  int nl = 0;
  if (j2k_gpu_last_launches(s.ctx, &nl) == J2K_OK) {
    std::lock_guard<std::mutex> lk(mu);
    launches += (uint64_t)nl;
  }
  // outputs straight into each request's pinned buffer on the same stream, then the
  // end-of-batch event
  for (size_t i = 0; i < batch.size(); ++i) {
    Request *r = batch[i];
    if (!r->out_bytes) continue;
    if (!r->out) {
      bool fresh = false;
      if (!(r->out = pinned.get(r->out_bytes, &fresh))) return J2K_ERR_NOMEM;
      if (fresh) {
        std::lock_guard<std::mutex> lk(mu);
        pinned_allocs++;
      }
    }
    const void *d = nullptr;
    size_t n = 0;
    if ((rc = j2k_gpu_output_device(s.ctx, (int)i, &d, &n)) != J2K_OK) return rc;
    if (cudaMemcpyAsync(r->out, d, n, cudaMemcpyDeviceToHost, s.stream) != cudaSuccess) return J2K_ERR_CUDA;
  }
  if (cudaEventRecord(s.done_ev, s.stream) != cudaSuccess) return J2K_ERR_CUDA;
  s.reqs = batch;
  s.busy = true;
  return J2K_OK;
}

bool j2k_server::complete_ready() {
  bool any = false;
  for (Slot &s : slots) {
    if (!s.busy) continue;
    const cudaError_t e = cudaEventQuery(s.done_ev);
    if (e == cudaErrorNotReady) continue;
    int rc = e == cudaSuccess ? j2k_gpu_batch_sync(s.ctx, -1) : J2K_ERR_CUDA;
    const Clock::time_point now = Clock::now();
    std::vector<int> st(s.reqs.size(), rc);
    float dev_ms = 0;
    if (rc == J2K_OK) {
      for (size_t i = 0; i < s.reqs.size(); ++i) st[i] = j2k_gpu_image_status(s.ctx, (int)i, nullptr);
      j2k_gpu_last_timing(s.ctx, nullptr, nullptr, nullptr, &dev_ms);
    }
    {
      std::lock_guard<std::mutex> lk(mu);
      gpu_ms += dev_ms;
      for (size_t i = 0; i < s.reqs.size(); ++i) {
        Request *r = s.reqs[i];
        r->status = st[i];
        r->done = true;
        r->t_done = now;
        j2k_plan_destroy(r->plan);
        r->plan = nullptr;
        if (st[i] == J2K_OK) {
          completed++;
          pixels += (uint64_t)r->info.width * r->info.height;
        } else {
          failed++;
        }
        lat_us.push_back(std::chrono::duration<double, std::micro>(r->t_done - r->t_submit).count());
        outstanding--;
      }
      if (--inflight == 0) busy_s += std::chrono::duration<double>(now - busy_since).count();
    }
    cv_done.notify_all();
    s.reqs.clear();
    s.busy = false;
    any = true;
  }
  return any;
}

bool j2k_server::admit() {
  bool any = false;
  for (Slot &s : slots) {
    if (s.busy) continue;
    std::vector<Request *> batch;
    {
      std::lock_guard<std::mutex> lk(mu);
      size_t bytes = 0;
      uint64_t px = 0;
      while (!pending.empty()) {
        Request *r = pending.front();
        const uint64_t rpx = (uint64_t)r->info.width * r->info.height;
        if (!batch.empty() && (bytes + r->footprint > slot_budget || px + rpx > cfg.max_batch_pixels)) break;
        if (cfg.max_batch_images > 0 && (int)batch.size() >= cfg.max_batch_images) break;
        bytes += r->footprint;
        px += rpx;
        batch.push_back(r);
        pending.pop_front();
      }
      if (batch.empty()) return any;
      if (inflight++ == 0) busy_since = Clock::now();
      batches++;
      batch_images += batch.size();
    }
    const Clock::time_point t0 = Clock::now();
    const int rc = launch(s, batch);
    {
      std::lock_guard<std::mutex> lk(mu);
      stage_ms += std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
    }
    if (rc != J2K_OK) {
      // the batch could not be enqueued: fail its requests, keep the slot free
      const Clock::time_point now = Clock::now();
      {
        std::lock_guard<std::mutex> lk(mu);
        for (Request *r : batch) {
          r->status = rc;
          r->done = true;
          r->t_done = now;
          j2k_plan_destroy(r->plan);
          r->plan = nullptr;
          failed++;
          outstanding--;
        }
        if (--inflight == 0) busy_s += std::chrono::duration<double>(now - busy_since).count();
      }
      cv_done.notify_all();
      s.busy = false;
      s.reqs.clear();
    }
    any = true;
  }
  return any;
}

void j2k_server::run() {
  cudaSetDevice(cfg.device);
  for (;;) {
    bool progressed = complete_ready();
    progressed |= admit();
    if (progressed) continue;
    std::unique_lock<std::mutex> lk(mu);
    if (stop && pending.empty() && inflight == 0) break;
    if (inflight > 0) {
      // batches on the device: poll their events again shortly, or sooner on a submit
      cv_submit.wait_for(lk, std::chrono::microseconds(30));
    } else {
      cv_submit.wait(lk, [&] { return stop || !pending.empty(); });
    }
  }
}

extern "C" int j2k_server_create(const j2k_server_config *cfg, j2k_server **out) {
  if (!out) return J2K_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return J2K_ERR_NODEVICE;
  }
  j2k_server *s = new j2k_server();
  if (cfg) s->cfg = *cfg;
  if (s->cfg.pipeline_depth <= 0) s->cfg.pipeline_depth = 2;
  if (s->cfg.max_batch_pixels == 0) s->cfg.max_batch_pixels = 128ull << 20;
  if (cudaSetDevice(s->cfg.device) != cudaSuccess) {
    delete s;
    return J2K_ERR_NODEVICE;
  }
  if (s->cfg.mem_budget == 0) {
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    s->cfg.mem_budget = fr / 10 * 6;
  }
  s->slot_budget = s->cfg.mem_budget / s->cfg.pipeline_depth;
  s->slots.resize(s->cfg.pipeline_depth);
  for (Slot &sl : s->slots) {
    int rc = j2k_gpu_ctx_create(s->cfg.device, s->slot_budget, &sl.ctx);
    if (rc == J2K_OK && cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess) rc = J2K_ERR_CUDA;
    if (rc == J2K_OK && cudaEventCreateWithFlags(&sl.done_ev, cudaEventDisableTiming) != cudaSuccess) rc = J2K_ERR_CUDA;
    if (rc != J2K_OK) {
      j2k_server_destroy(s);
      return rc;
    }
  }
  s->sched = std::thread([s] { s->run(); });
  *out = s;
  return J2K_OK;
}

extern "C" void j2k_server_destroy(j2k_server *s) {
  if (!s) return;
  if (s->sched.joinable()) {
    {
      std::lock_guard<std::mutex> lk(s->mu);
      // requests not yet admitted are failed; batches in flight finish
      for (Request *r : s->pending) {
        r->status = J2K_ERR_STATE;
        r->done = true;
        j2k_plan_destroy(r->plan);
        r->plan = nullptr;
        s->outstanding--;
      }
      s->pending.clear();
      s->stop = true;
    }
    s->cv_submit.notify_all();
    s->sched.join();
  }
  for (Slot &sl : s->slots) {
    if (sl.ctx) j2k_gpu_ctx_destroy(sl.ctx);
    if (sl.stream) cudaStreamDestroy(sl.stream);
    if (sl.done_ev) cudaEventDestroy(sl.done_ev);
  }
  for (auto &kv : s->reqs) {
    if (kv.second->plan) j2k_plan_destroy(kv.second->plan);
    delete kv.second;
  }
  delete s;  // the pinned pool frees its buffers
}

extern "C" int64_t j2k_server_submit(j2k_server *s, const void *cs, size_t len, int fmt, int flags) {
  if (!s || !cs || !len) return J2K_ERR_ARG;
  Request *r = new Request();
  r->t_submit = Clock::now();
  r->cs.assign((const uint8_t *)cs, (const uint8_t *)cs + len);
  r->fmt = fmt;
  r->flags = flags;
  int rc = j2k_plan_create(r->cs.data(), r->cs.size(), 0, 0, 0, &r->plan);
  if (rc == J2K_OK) rc = j2k_plan_info(r->plan, &r->info);
  if (rc != J2K_OK) {
    if (r->plan) j2k_plan_destroy(r->plan);
    delete r;
    return rc;
  }
  r->out_bytes = fmt == J2K_FMT_NONE ? 0 : j2k_output_bytes(&r->info, fmt);
  r->footprint = estimate_footprint(r->info, r->out_bytes);
  if (r->footprint > s->slot_budget) {
    j2k_plan_destroy(r->plan);
    delete r;
    return J2K_ERR_NOMEM;
  }
  int64_t id;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) {
      j2k_plan_destroy(r->plan);
      delete r;
      return J2K_ERR_STATE;
    }
    id = r->id = s->next_id++;
    s->reqs[id] = r;
    s->pending.push_back(r);
    s->outstanding++;
  }
  s->cv_submit.notify_one();
  return id;
}

extern "C" int j2k_server_wait(j2k_server *s, int64_t id, void *dst, size_t cap, size_t *bytes, int timeout_ms) {
  if (!s) return J2K_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return J2K_ERR_ARG;
  Request *r = it->second;
  if (!r->done) {
    if (timeout_ms == 0) return J2K_ERR_TIMEOUT;
    if (timeout_ms < 0) {
      s->cv_done.wait(lk, [&] { return r->done; });
    } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return r->done; })) {
      return J2K_ERR_TIMEOUT;
    }
  }
  if (bytes) *bytes = r->out_bytes;
  if (r->status != J2K_OK) return r->status;
  if (dst && r->out_bytes) {
    if (cap < r->out_bytes) return J2K_ERR_ARG;
    // a finished request is only changed by release(), which must not run concurrently
    // with a wait() on the same id, so the copy runs outside the lock
    const uint8_t *src = r->out;
    const size_t n = r->out_bytes;
    lk.unlock();
    std::memcpy(dst, src, n);
  }
  return J2K_OK;
}

extern "C" int j2k_server_result(j2k_server *s, int64_t id, const void **ptr, size_t *bytes, int timeout_ms) {
  if (!s || !ptr) return J2K_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return J2K_ERR_ARG;
  Request *r = it->second;
  if (!r->done) {
    if (timeout_ms == 0) return J2K_ERR_TIMEOUT;
    if (timeout_ms < 0) {
      s->cv_done.wait(lk, [&] { return r->done; });
    } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return r->done; })) {
      return J2K_ERR_TIMEOUT;
    }
  }
  *ptr = r->out;
  if (bytes) *bytes = r->out_bytes;
  return r->status;
}

extern "C" int j2k_server_latency_us(j2k_server *s, int64_t id, double *us) {
  if (!s || !us) return J2K_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return J2K_ERR_ARG;
  if (!it->second->done) return J2K_ERR_STATE;
  *us = std::chrono::duration<double, std::micro>(it->second->t_done - it->second->t_submit).count();
  return J2K_OK;
}

extern "C" int j2k_server_release(j2k_server *s, int64_t id) {
  if (!s) return J2K_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return J2K_ERR_ARG;
  if (!it->second->done) return J2K_ERR_STATE;
  s->pinned.put(it->second->out);
  delete it->second;
  s->reqs.erase(it);
  return J2K_OK;
}

extern "C" int j2k_server_drain(j2k_server *s) {
  if (!s) return J2K_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  s->cv_done.wait(lk, [&] { return s->outstanding == 0; });
  return J2K_OK;
}

extern "C" int j2k_server_stats_get(j2k_server *s, j2k_server_stats *st) {
  if (!s || !st) return J2K_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(st, 0, sizeof(*st));
  st->completed = s->completed;
  st->failed = s->failed;
  st->batches = s->batches;
  st->mean_batch_images = s->batches ? (double)s->batch_images / s->batches : 0.0;
  st->pixels = s->pixels;
  st->launches = s->launches;
  st->gpu_ms = s->gpu_ms;
  st->stage_ms = s->stage_ms;
  st->enqueue_ms = s->enqueue_ms;
  st->pool_growths = s->pool_growths;
  st->pinned_allocs = s->pinned_allocs;
  st->busy_s = s->busy_s + (s->inflight ? std::chrono::duration<double>(Clock::now() - s->busy_since).count() : 0.0);
  if (!s->lat_us.empty()) {
    std::vector<double> v = s->lat_us;
    std::sort(v.begin(), v.end());
    auto pct = [&](double q) { return v[std::min(v.size() - 1, (size_t)(q * (v.size() - 1) + 0.5))]; };
    st->p50_us = pct(0.50);
    st->p99_us = pct(0.99);
    st->max_us = v.back();
  }
  return J2K_OK;
}

extern "C" int j2k_server_stats_reset(j2k_server *s) {
  if (!s) return J2K_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  s->lat_us.clear();
  s->completed = s->failed = s->batches = s->batch_images = s->pixels = s->launches = 0;
  s->busy_s = 0;
  s->gpu_ms = 0;
  s->stage_ms = s->enqueue_ms = 0;
  s->pool_growths = s->pinned_allocs = 0;
  if (s->inflight) s->busy_since = Clock::now();
  return J2K_OK;
}
