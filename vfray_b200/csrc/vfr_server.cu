// Served form: a request loop over resident meshes with continuous batching.
//
// No counterpart in the reference (its driver renders one view and exits).
// Requests (mesh, camera, resolution) are submitted from any thread.  A
// worker thread admits them in arrival order while their memory footprint
// (their view's scratch and framebuffers; the meshes are resident and
// counted once by the caller's budget) fits the budget left, folds every
// admitted request into the next batch -- meshes and image sizes mixed --
// and launches it on one of two batch slots, each with its own stream.  A
// batch is launched as soon as a slot is free, so requests that arrive while
// another batch is on the GPU start at once on the other slot and the two
// overlap on the device.  When a slot's batch has finished, its images are
// copied to the requests' host buffers, their budget is released and their
// waiters are woken.  Per-request submit / start / done times give the
// latency.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "vfr_internal.h"
#include "vfray.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
  uint64_t ticket = 0;
  vfr_request r{};
  uint64_t footprint = 0;
  Clock::time_point t_submit, t_start, t_done;
  int status = VFR_OK;
  bool done = false;
  uint32_t batch_id = 0, batch_jobs = 0, num_rays = 0;
  uint64_t num_steps = 0;
};

struct Slot {
  vfr::Batch b;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  std::vector<Req*> reqs;
  bool busy = false;
  uint32_t id = 0;
  std::vector<uint8_t> host_rgb8;  // pinned staging would be faster; sizes vary
  uint8_t* pin = nullptr;
  size_t pin_cap = 0;
};

}  // namespace

struct vfr_server {
  vfr_ctx* ctx = nullptr;
  uint64_t budget = 0, used = 0;
  size_t copy_threads = std::max(1u, std::min(8u, std::thread::hardware_concurrency() / 2));
  uint32_t max_batch = 256;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req*> pending;
  std::unordered_map<uint64_t, Req*> all;
  uint64_t next_ticket = 1;
  Slot slots[2];
  std::thread worker;
  bool stop = false;
  uint32_t batches = 0;
  uint64_t rays = 0, steps = 0, completed = 0, rejected = 0;
  Clock::time_point t0 = Clock::now();

  double ms(Clock::time_point t) const {
    return std::chrono::duration<double, std::milli>(t - t0).count();
  }
  uint64_t footprint(const vfr_request& r) {
    vfr::Mesh* m = ctx->impl.mesh(r.mesh_id);
    const uint64_t np = (uint64_t)r.W * r.H;
    uint64_t f = np * (4 + 4 + 3 + 16 + 4);  // winner, rays, rgb8, rgba, steps
    if (r.mode == VFR_MODE_COMPOSITED) f += np * (4 * 3 + 8 * 4);
    if (m) f += (uint64_t)m->nExt * (32 + 4 + 16 + 4) + (r.use_mv ? (uint64_t)m->nV * 16 : 0);
    return f + 4096;
  }
  void loop();
  void retire(Slot& s);
  int launch(Slot& s, std::vector<Req*>& reqs);
};

int vfr_server::launch(Slot& s, std::vector<Req*>& reqs) {
  vfr::Ctx& C = ctx->impl;
  std::vector<vfr::JobSpec> specs(reqs.size());
  size_t pix = 0;
  int mode = reqs[0]->r.mode;
  for (size_t i = 0; i < reqs.size(); ++i) {
    const vfr_request& r = reqs[i]->r;
    specs[i].mesh = r.mesh_id;
    specs[i].W = r.W;
    specs[i].H = r.H;
    specs[i].use_mv = r.use_mv != 0;
    std::memcpy(specs[i].mv, r.mv, sizeof specs[i].mv);
    pix += (size_t)r.W * r.H;
  }
  s.b.ctx = &C;
  s.b.stream = s.stream;
  int rc = s.b.layout(specs, mode, true);
  if (!rc) rc = s.b.upload(true);
  if (!rc) rc = s.b.enqueue_all();
  // the images come back through pinned staging, copied on the slot stream
  if (!rc && s.pin_cap < pix * 3) {
    if (s.pin) cudaFreeHost(s.pin);
    s.pin = nullptr;
    s.pin_cap = 0;
    const size_t want = pix * 3 + pix * 3 / 2;  // headroom: pinning is slow
    if (cudaMallocHost(&s.pin, want) != cudaSuccess) rc = VFR_ERR_NOMEM;
    else s.pin_cap = want;
  }
  if (!rc)
    rc = C.cuda(cudaMemcpyAsync(s.pin, s.b.out_rgb8.p, pix * 3, cudaMemcpyDeviceToHost, s.stream),
                "served image read");
  if (!rc) rc = C.cuda(cudaEventRecord(s.done, s.stream), "served event");
  const Clock::time_point now = Clock::now();
  s.id = ++batches;
  for (Req* q : reqs) {
    q->t_start = now;
    q->batch_id = s.id;
    q->batch_jobs = (uint32_t)reqs.size();
    if (rc) q->status = rc;
  }
  s.reqs = reqs;
  s.busy = true;
  return rc;
}

void vfr_server::retire(Slot& s) {
  vfr::Ctx& C = ctx->impl;
  cudaEventSynchronize(s.done);
  std::vector<vfr::ViewCounters> k;
  int rc = s.b.counters(k);
  // images from the pinned staging into the requests' buffers, split over
  // a few threads when there is much to copy (the callers' buffers are often
  // fresh memory whose first touch costs more than the copy)
  {
    std::vector<std::pair<size_t, size_t>> span(s.reqs.size());  // (pixel offset, pixels)
    size_t off = 0, total = 0;
    for (size_t i = 0; i < s.reqs.size(); ++i) {
      const size_t np = (size_t)s.reqs[i]->r.W * s.reqs[i]->r.H;
      span[i] = {off, np};
      off += np;
      if (!rc && s.reqs[i]->status == VFR_OK && s.reqs[i]->r.rgb8_host) total += np * 3;
    }
    auto copy = [&](size_t lo, size_t hi) {
      for (size_t i = lo; i < hi; ++i) {
        Req* q = s.reqs[i];
        if (!rc && q->status == VFR_OK && q->r.rgb8_host)
          std::memcpy(q->r.rgb8_host, s.pin + 3 * span[i].first, span[i].second * 3);
      }
    };
    const size_t nthreads = std::min<size_t>(copy_threads, std::max<size_t>(1, total >> 23));
    if (nthreads <= 1) {
      copy(0, s.reqs.size());
    } else {  // split by bytes
      std::vector<std::thread> th;
      size_t lo = 0, acc = 0, next = 1;
      for (size_t i = 0; i < s.reqs.size(); ++i) {
        acc += span[i].second * 3;
        if (acc >= total * next / nthreads && next < nthreads) {
          th.emplace_back(copy, lo, i + 1);
          lo = i + 1;
          ++next;
        }
      }
      copy(lo, s.reqs.size());
      for (auto& t : th) t.join();
    }
  }
  const Clock::time_point now = Clock::now();
  std::lock_guard<std::mutex> g(mu);
  for (size_t i = 0; i < s.reqs.size(); ++i) {
    Req* q = s.reqs[i];
    if (q->status == VFR_OK && !rc) {
      q->num_rays = k[i].nrays;
      q->num_steps = k[i].steps;
      if (k[i].status) q->status = C.check_status(k[i].status, 0);
    } else if (q->status == VFR_OK) {
      q->status = rc;
    }
    q->t_done = now;
    q->done = true;
    used -= q->footprint;
    rays += q->num_rays;
    steps += q->num_steps;
    ++completed;
  }
  s.reqs.clear();
  s.busy = false;
  cv_done.notify_all();
  cv_work.notify_all();
}

void vfr_server::loop() {
  cudaSetDevice(ctx->impl.device);
  for (;;) {
    // retire finished slots
    for (Slot& s : slots)
      if (s.busy && cudaEventQuery(s.done) != cudaErrorNotReady) retire(s);
    std::vector<Req*> take;
    Slot* free_slot = nullptr;
    {
      std::unique_lock<std::mutex> lk(mu);
      if (stop && pending.empty() && !slots[0].busy && !slots[1].busy) break;
      for (Slot& s : slots)
        if (!s.busy) {
          free_slot = &s;
          break;
        }
      if (free_slot && !pending.empty()) {
        const int mode = pending.front()->r.mode;
        while (!pending.empty() && take.size() < max_batch) {
          Req* q = pending.front();
          if (q->r.mode != mode) break;
          if (used + q->footprint > budget) break;  // wait for memory to free up
          used += q->footprint;
          take.push_back(q);
          pending.pop_front();
        }
      }
      if (take.empty()) {
        const bool any_busy = slots[0].busy || slots[1].busy;
        if (!any_busy) {
          cv_work.wait_for(lk, std::chrono::milliseconds(5));
        } else {
          lk.unlock();
          // a batch is on the GPU: poll its completion briefly
          std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
        continue;
      }
    }
    launch(*free_slot, take);
  }
}

extern "C" {

int vfr_server_create(vfr_ctx* ctx, uint64_t budget_bytes, uint32_t max_batch, vfr_server** out) {
  if (!ctx || !out || budget_bytes == 0) return VFR_ERR_INVALID;
  cudaSetDevice(ctx->impl.device);
  if (!ctx->impl.d_tf) return ctx->impl.fail(VFR_ERR_STATE, "tables not uploaded");
  vfr_server* s = new vfr_server;
  s->ctx = ctx;
  s->budget = budget_bytes;
  s->max_batch = max_batch ? max_batch : 256;
  for (Slot& sl : s->slots) {
    sl.b.ctx = &ctx->impl;
    if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess) {
      delete s;
      return VFR_ERR_CUDA;
    }
    sl.b.stream = sl.stream;
  }
  s->worker = std::thread([s] { s->loop(); });
  *out = s;
  return VFR_OK;
}

int vfr_server_submit(vfr_server* s, const vfr_request* r, uint64_t* ticket) {
  if (!s || !r || !ticket) return VFR_ERR_INVALID;
  if (!s->ctx->impl.mesh(r->mesh_id)) return VFR_ERR_STATE;
  if (r->W < 2 || r->H < 2 || (uint64_t)r->W * r->H > (1ull << 28)) return VFR_ERR_INVALID;
  if (r->mode != VFR_MODE_REF && r->mode != VFR_MODE_COMPOSITED) return VFR_ERR_INVALID;
  Req* q = new Req;
  q->r = *r;
  q->footprint = s->footprint(*r);
  q->t_submit = Clock::now();
  std::lock_guard<std::mutex> g(s->mu);
  if (q->footprint > s->budget) {  // can never fit: refuse now
    ++s->rejected;
    delete q;
    return VFR_ERR_BUDGET;
  }
  q->ticket = s->next_ticket++;
  s->all[q->ticket] = q;
  s->pending.push_back(q);
  *ticket = q->ticket;
  s->cv_work.notify_one();
  return VFR_OK;
}

int vfr_server_wait(vfr_server* s, uint64_t ticket, int timeout_ms, vfr_request_info* info) {
  if (!s) return VFR_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(ticket);
  if (it == s->all.end()) return VFR_ERR_STATE;
  Req* q = it->second;
  const auto deadline = Clock::now() + std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms);
  while (!q->done) {
    if (timeout_ms < 0) {
      s->cv_done.wait(lk);
    } else if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && !q->done) {
      return VFR_ERR_TIMEOUT;
    }
  }
  if (info) {
    info->status = q->status;
    info->t_submit_ms = s->ms(q->t_submit);
    info->t_start_ms = s->ms(q->t_start);
    info->t_done_ms = s->ms(q->t_done);
    info->batch_id = q->batch_id;
    info->batch_jobs = q->batch_jobs;
    info->num_rays = q->num_rays;
    info->num_steps = q->num_steps;
  }
  const int st = q->status;
  s->all.erase(it);
  delete q;
  return st;
}

int vfr_server_stats(vfr_server* s, vfr_server_counters* out) {
  if (!s || !out) return VFR_ERR_INVALID;
  std::lock_guard<std::mutex> g(s->mu);
  out->batches = s->batches;
  out->completed = s->completed;
  out->rejected = s->rejected;
  out->pending = (uint32_t)s->pending.size();
  out->budget_used = s->used;
  out->rays = s->rays;
  out->steps = s->steps;
  return VFR_OK;
}

void vfr_server_destroy(vfr_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop = true;
    s->cv_work.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();
  cudaSetDevice(s->ctx->impl.device);
  for (Slot& sl : s->slots) {
    if (sl.stream) cudaStreamSynchronize(sl.stream);
    if (sl.pin) cudaFreeHost(sl.pin);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.stream) cudaStreamDestroy(sl.stream);
    sl.b.ctx = &s->ctx->impl;
  }
  for (auto& kv : s->all) delete kv.second;
  delete s;
}

}  // extern "C"
