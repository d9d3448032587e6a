// Served form: a request loop with continuous batching over resident meshes.
//
// No counterpart in the reference (its driver renders one view and exits).
// Requests (mesh, camera, resolution, mode) are submitted from any thread.
// A worker thread owns all GPU work of the server:
//
//  * One long-lived persistent traversal launch (serve_kernel, the drain)
//    runs on its own stream and takes rays from a table of segments.  It
//    leaves a few CTA slots of the GPU free.
//  * The worker admits pending requests in arrival order while their memory
//    footprint fits the budget, lays each admitted group out as a segment in
//    the server's arena, runs the segment's stages (a) and (b) on a second
//    stream -- in the CTA slots the drain leaves free, while the drain runs --
//    and publishes it into the segment table.  The running drain folds the
//    new rays in: requests that arrive while others are on the GPU start as
//    soon as their preparation ends, whatever the size of the frames in
//    flight.
//  * The drain sets a per-job completion flag in mapped host memory when a
//    job's last ray ends; the worker then copies that job's image out on a
//    third stream, hands it to the request and releases its footprint.
//
// Memory: the budget covers the resident meshes of the context (counted
// once) and, per request in flight, its job-table entry, view vertices,
// planes, visible list, boxes, winner map or entry lists, ray list and RGB8
// image.  Those live in one arena allocated when the server starts, so
// serving allocates and frees no device memory.  Inside one drain launch
// the arena and the segment table are only ever appended to (the launch's
// caches never see reused memory); the worker starts a new epoch -- arena
// and table from the start -- between launches: when the server has been
// idle for a while, or when the arena or the table is used up (then it
// stops admitting, lets the work in flight finish, and stops the launch).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "vfr_internal.h"
#include "vfray.h"

namespace {

using Clock = std::chrono::steady_clock;
using vfr::Batch;
using vfr::JobSpec;

constexpr uint32_t kMaxSegs = 8192;        // segment-table entries per epoch
constexpr uint32_t kMaxFlags = 1u << 20;   // completion flags per epoch
constexpr int kReserveDivisor = 2;        // traversal CTAs left out for the preparation: SMs / this
constexpr uint32_t kIdleLimit = 400000;    // default: microseconds an idle drain waits for work
constexpr double kLingerMs = 50.0;         // default: idle time before the worker stops the drain

struct Seg;

enum class St { Pending, InFlight, Copying, Done };

struct Req {
  uint64_t ticket = 0;
  vfr_request r{};
  uint64_t footprint = 0;
  Clock::time_point t_submit, t_start, t_ready, t_done;
  int status = VFR_OK;
  St state = St::Pending;
  bool claimed = false;  // a waiter holds it (a second waiter is refused)
  Seg* seg = nullptr;
  uint32_t job = 0, flag = 0;  // index in the segment, completion flag index
  uint32_t batch_id = 0, batch_jobs = 0, num_rays = 0, dev_status = 0;
  uint64_t num_steps = 0;
  char* stage = nullptr;  // pinned: the image (unless copied directly), then the job's counters
  size_t stage_bytes = 0, img_off = 0;
  cudaEvent_t copied = nullptr;
};

// Pinned host memory allocated once when the server starts and handed out
// by first fit in 256-byte units: allocating pinned memory waits for all
// work on the device, the running drain included, so nothing is pinned
// while the server serves.
struct PinPool {
  char* base = nullptr;
  size_t cap = 0;
  std::map<size_t, size_t> free_;  // offset -> bytes
  static size_t round(size_t n) { return (n + 255) & ~(size_t)255; }
  void init(char* b, size_t c) {
    base = b;
    cap = c;
    free_.clear();
    if (c) free_[0] = c;
  }
  char* alloc(size_t n) {
    n = round(n);
    for (auto it = free_.begin(); it != free_.end(); ++it)
      if (it->second >= n) {
        const size_t off = it->first, left = it->second - n;
        free_.erase(it);
        if (left) free_[off + n] = left;
        return base + off;
      }
    return nullptr;
  }
  void release(char* p, size_t n) {
    if (!p) return;
    n = round(n);
    size_t off = (size_t)(p - base);
    auto next = free_.lower_bound(off);
    if (next != free_.end() && off + n == next->first) {  // merge with the block after
      n += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {  // and with the block before
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        prev->second += n;
        return;
      }
    }
    free_[off] = n;
  }
};

// One admitted group of requests: a batch laid out in the arena.
struct Seg {
  uint32_t seq = 0;     // entry of the segment table (in this epoch)
  uint32_t id = 0;      // over the server's life
  std::unique_ptr<Batch> b;
  std::vector<Req*> reqs;
  uint32_t remaining = 0;
  char* up = nullptr;  // pinned staging of its job-table upload
  size_t up_bytes = 0;
  cudaEvent_t prep0 = nullptr, prep1 = nullptr;  // its preparation on the device
};

}  // namespace

struct vfr_server {
  vfr_ctx* ctx = nullptr;
  vfr::Ctx* C = nullptr;
  uint64_t budget = 0, mesh_bytes = 0, used = 0;  // used: footprints in flight
  uint32_t max_batch = 256;

  // device side
  vfr::Arena arena;
  vfr::SegDev* segs = nullptr;  // kMaxSegs entries
  vfr::ServeCtl* ctl = nullptr;
  uint32_t* flags = nullptr;    // mapped host memory, kMaxFlags completion flags
  uint32_t* stop = nullptr;     // pinned: [0] the stop word copied to the drain, [16] its status back
  cudaStream_t prep = nullptr, drain = nullptr, copy = nullptr;
  cudaEvent_t drain_done = nullptr;
  int drain_grid = 0;
  bool drain_running = false;
  bool stopping = false;        // epoch end requested: admit nothing until it is done
  uint32_t seq = 0, flags_used = 0;  // this epoch's table entries and flags
  uint32_t launches = 0, epochs = 0, queue_timeouts = 0;
  uint32_t dev_status = 0;
  double prep_ms = 0;  // device time of the retired segments' preparation
  std::atomic<uint32_t> idle_limit{kIdleLimit};
  std::atomic<double> linger_ms{kLingerMs};
  Clock::time_point last_busy = Clock::now();

  // host side
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req*> pending;
  std::unordered_map<uint64_t, Req*> all;
  std::deque<Seg*> inflight;
  std::vector<std::unique_ptr<Batch>> spare;  // host-side batch objects to reuse
  PinPool pool;                               // pinned staging of uploads and image copies
  uint64_t next_ticket = 1;
  std::thread worker;
  bool stop_req = false;
  uint32_t segments = 0;
  uint64_t rays = 0, steps = 0, completed = 0, rejected = 0;
  int fatal = VFR_OK;  // a CUDA failure of the worker: every request fails with it
  Clock::time_point t0 = Clock::now();

  double ms(Clock::time_point t) const {
    return std::chrono::duration<double, std::milli>(t - t0).count();
  }
  uint64_t footprint(const vfr_request& r) const;
  void loop();
  int start(uint64_t budget_bytes);
  void release_device();
  bool poll_completions();
  bool admit();
  int launch_drain();
  void epoch_reset();
  void send_stop();
  bool stop_sent = false;
  cudaEvent_t stop_copied = nullptr;  // the stop copy, ordered before the next launch's reset
  void fail_all(int rc);

};

// Arena bytes of the request's job laid out alone: an upper bound of what
// it adds to any segment (a segment shares the 256-byte rounding of its
// buffers between its jobs).
uint64_t vfr_server::footprint(const vfr_request& r) const {
  JobSpec q;
  q.mesh = r.mesh_id;
  q.W = r.W;
  q.H = r.H;
  q.use_mv = r.use_mv != 0;
  return Batch::arena_bytes(*C, {q}, r.mode, 256, true);
}

int vfr_server::start(uint64_t budget_bytes) {
  vfr::Range nvtx("vfr_server start");
  vfr::Ctx& X = *C;
  budget = budget_bytes;
  int rc = X.cuda(cudaStreamCreateWithFlags(&prep, cudaStreamNonBlocking), "server streams");
  if (!rc) rc = X.cuda(cudaStreamCreateWithFlags(&drain, cudaStreamNonBlocking), "server streams");
  if (!rc) rc = X.cuda(cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking), "server streams");
  if (!rc) rc = X.cuda(cudaEventCreateWithFlags(&drain_done, cudaEventDisableTiming), "server event");
  if (!rc) rc = X.cuda(cudaEventCreateWithFlags(&stop_copied, cudaEventDisableTiming), "server event");
  // every resident mesh gets its distinct edges now (allocations and waits
  // are not allowed once the drain runs); their bytes count against the budget
  for (auto& m : X.meshes)
    if (m && !rc) {
      rc = X.mesh_edges(m.get(), prep);
      mesh_bytes += m->bytes;
    }
  if (rc) return rc;
  if (budget <= mesh_bytes + (16u << 20))
    return X.fail(VFR_ERR_BUDGET, "the budget does not cover the resident meshes");
  size_t free_b = 0, total_b = 0;
  rc = X.cuda(cudaMemGetInfo(&free_b, &total_b), "memory info");
  if (rc) return rc;
  const size_t margin = 512u << 20;
  size_t cap = (size_t)std::min<uint64_t>(budget - mesh_bytes, free_b > margin ? free_b - margin : 0);
  cap &= ~(size_t)255;
  if (cap < (16u << 20)) return X.fail(VFR_ERR_NOMEM, "no device memory for the server's arena");
  rc = X.cuda(cudaMalloc((void**)&arena.base, cap), "server arena");
  if (rc) return rc;
  arena.cap = cap;
  rc = X.cuda(cudaMalloc((void**)&segs, sizeof(vfr::SegDev) * kMaxSegs), "segment table");
  if (!rc) rc = X.cuda(cudaMalloc((void**)&ctl, sizeof(vfr::ServeCtl)), "server control");
  if (!rc)
    rc = X.cuda(cudaHostAlloc((void**)&flags, sizeof(uint32_t) * kMaxFlags, cudaHostAllocMapped),
                "completion flags");
  if (!rc) rc = X.cuda(cudaHostAlloc((void**)&stop, 256, cudaHostAllocDefault), "stop word");
  // pinned staging for every upload and image copy of the server's life:
  // a sixteenth of the budget, between 64 MB and 1 GB
  const size_t pool_cap =
      std::min<size_t>(1ull << 30, std::max<size_t>(64ull << 20, (size_t)(budget / 16))) & ~(size_t)255;
  char* pool_base = nullptr;
  if (!rc) rc = X.cuda(cudaHostAlloc((void**)&pool_base, pool_cap, cudaHostAllocDefault), "pinned staging");
  if (rc) return rc;
  pool.init(pool_base, pool_cap);
  std::memset(flags, 0, sizeof(uint32_t) * kMaxFlags);
  *(volatile uint32_t*)stop = 0;
  int occ = 0;
  if (vfr::serve_blocks_per_sm(&occ) != VFR_OK) return X.fail(VFR_ERR_CUDA, "drain occupancy");
  drain_grid = std::max(X.num_sms, occ * X.num_sms - X.num_sms / kReserveDivisor);
  rc = X.cuda(cudaMemsetAsync(ctl, 0, sizeof(vfr::ServeCtl), prep), "server control");
  if (!rc) rc = X.cuda(cudaStreamSynchronize(prep), "server start");
  return rc;
}

void vfr_server::release_device() {
  for (cudaStream_t s : {prep, drain, copy})
    if (s) cudaStreamSynchronize(s);
  for (Seg* g : inflight) {
    if (g->prep0) cudaEventDestroy(g->prep0);
    if (g->prep1) cudaEventDestroy(g->prep1);
    delete g;
  }
  inflight.clear();
  spare.clear();
  if (pool.base) cudaFreeHost(pool.base);
  pool.init(nullptr, 0);
  if (arena.base) cudaFree(arena.base);
  if (segs) cudaFree(segs);
  if (ctl) cudaFree(ctl);
  if (flags) cudaFreeHost(flags);
  if (stop) cudaFreeHost(stop);
  if (drain_done) cudaEventDestroy(drain_done);
  if (stop_copied) cudaEventDestroy(stop_copied);
  for (cudaStream_t s : {prep, drain, copy})
    if (s) cudaStreamDestroy(s);
}


// (Re)starts the drain from the oldest segment with work left.  Rays a
// previous launch took were all finished before its warps left (a warp
// leaves only when its lanes are idle), so the heads stand as they are.
int vfr_server::launch_drain() {
  vfr::Range nvtx("vfr_server drain launch");
  vfr::Ctx& X = *C;
  vfr::ServeParams SP;
  std::memset(&SP, 0, sizeof SP);
  SP.T.tf = X.d_tf;
  SP.T.psi = X.d_psi;
  SP.T.e2tab = reinterpret_cast<const double*>(X.d_tf + 256);
  SP.T.step_cap = X.step_cap;
  SP.T.refill = X.tune.refill;
  SP.segs = segs;
  SP.ctl = ctl;
  SP.idle_limit = idle_limit.load();
  SP.first = inflight.empty() ? seq : inflight.front()->seq;
  if (stop_sent && cudaStreamWaitEvent(drain, stop_copied, 0) != cudaSuccess) return VFR_ERR_CUDA;
  stop_sent = false;
  if (cudaMemsetAsync(&ctl->stop, 0, sizeof(uint32_t), drain) != cudaSuccess) return VFR_ERR_CUDA;
  if (vfr::launch_serve(SP, drain_grid, drain) != cudaSuccess) return VFR_ERR_CUDA;
  // the control word's status comes back with the launch's end
  if (cudaMemcpyAsync(stop + 16, &ctl->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, drain) !=
          cudaSuccess ||
      cudaEventRecord(drain_done, drain) != cudaSuccess)
    return VFR_ERR_CUDA;
  drain_running = true;
  ++launches;
  return VFR_OK;
}

// Asks the drain's idle warps to leave: the stop word goes to device memory
// by a copy on the copy stream (the drain polls device memory only).
void vfr_server::send_stop() {
  if (stop_sent) return;
  *(volatile uint32_t*)stop = 1u;
  if (cudaMemcpyAsync(&ctl->stop, stop, sizeof(uint32_t), cudaMemcpyHostToDevice, copy) != cudaSuccess ||
      cudaEventRecord(stop_copied, copy) != cudaSuccess)
    cudaGetLastError();
  stop_sent = true;
}

// A new epoch: the drain has left and nothing is in flight, so the arena,
// the segment table and the flags start again from the beginning.
void vfr_server::epoch_reset() {
  vfr::Range nvtx("vfr_server epoch reset");
  arena.off = 0;
  seq = 0;
  std::memset(flags, 0, sizeof(uint32_t) * flags_used);
  flags_used = 0;
  if (cudaMemsetAsync(ctl, 0, sizeof(vfr::ServeCtl), prep) != cudaSuccess ||
      cudaStreamSynchronize(prep) != cudaSuccess)
    fail_all(VFR_ERR_CUDA);
  ++epochs;
}

// A CUDA failure of the worker: every request not yet done fails with it.
void vfr_server::fail_all(int rc) {
  cudaGetLastError();
  std::lock_guard<std::mutex> g(mu);
  fatal = rc;
  const Clock::time_point now = Clock::now();
  auto finish = [&](Req* q) {
    if (q->state == St::Done) return;
    if (q->state != St::Pending) used -= q->footprint;  // admitted: it held its footprint
    q->status = rc;
    q->state = St::Done;
    q->t_done = now;
    ++completed;
  };
  for (Req* q : pending) finish(q);
  pending.clear();
  for (Seg* s : inflight)
    for (Req* q : s->reqs) finish(q);
  cv_done.notify_all();
}

// Jobs whose completion flag the drain has set get their image and counters
// copied out (copy stream, pinned staging); copies that have landed hand
// the image to the request, which is then done.  Returns whether anything
// moved.
bool vfr_server::poll_completions() {
  vfr::Range nvtx("vfr_server completions");
  bool progress = false;
  const volatile uint32_t* f = flags;
  for (Seg* g : inflight)
    for (Req* q : g->reqs) {
      if (q->state == St::InFlight && f[q->flag]) {
        const JobSpec& sp = g->b->specs[q->job];
        const size_t img = 3 * (size_t)sp.W * sp.H;
        const bool staged = q->r.rgb8_host && img + 256 <= pool.cap / 4;
        q->img_off = staged ? PinPool::round(img) : 0;
        q->stage_bytes = q->img_off + sizeof(vfr::ViewCounters);
        q->stage = pool.alloc(q->stage_bytes);
        if (!q->stage) continue;  // staging in use: copies in flight free it
        if (!q->copied && cudaEventCreateWithFlags(&q->copied, cudaEventDisableTiming) != cudaSuccess) {
          fail_all(VFR_ERR_CUDA);
          return true;
        }
        cudaError_t e = cudaSuccess;
        if (q->r.rgb8_host)  // an image too large for the staging is copied directly
          e = cudaMemcpyAsync(staged ? (void*)q->stage : q->r.rgb8_host, sp.rgb8, img,
                              cudaMemcpyDeviceToHost, copy);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(q->stage + q->img_off, g->b->jobs[q->job].ctr, sizeof(vfr::ViewCounters),
                              cudaMemcpyDeviceToHost, copy);
        if (e == cudaSuccess) e = cudaEventRecord(q->copied, copy);
        if (e != cudaSuccess) {
          fail_all(VFR_ERR_CUDA);
          return true;
        }
        q->t_ready = Clock::now();
        q->state = St::Copying;
        progress = true;
      }
      if (q->state == St::Copying && cudaEventQuery(q->copied) != cudaErrorNotReady) {
        const JobSpec& sp = g->b->specs[q->job];
        const size_t img = 3 * (size_t)sp.W * sp.H;
        vfr::ViewCounters k;
        std::memcpy(&k, q->stage + q->img_off, sizeof k);
        if (q->r.rgb8_host && q->img_off) std::memcpy(q->r.rgb8_host, q->stage, img);
        pool.release(q->stage, q->stage_bytes);
        q->stage = nullptr;
        cudaEventDestroy(q->copied);
        q->copied = nullptr;
        std::lock_guard<std::mutex> lk(mu);
        q->num_rays = k.nrays;
        q->num_steps = k.steps;
        if (k.status & (VFR_DEV_CYCLE | VFR_DEV_RANGE | VFR_DEV_STEP_CAP | VFR_DEV_OVERFLOW))
          q->status = VFR_ERR_DEVICE;
        q->dev_status = k.status;
        q->t_done = Clock::now();
        q->state = St::Done;
        used -= q->footprint;
        rays += k.nrays;
        steps += k.steps;
        ++completed;
        --g->remaining;
        cv_done.notify_all();
        progress = true;
      }
    }
  // segments are retired in order; their arena memory returns with the epoch
  while (!inflight.empty() && inflight.front()->remaining == 0) {
    Seg* g = inflight.front();
    inflight.pop_front();
    float ms = 0;
    if (g->prep0 && cudaEventElapsedTime(&ms, g->prep0, g->prep1) == cudaSuccess) prep_ms += ms;
    cudaGetLastError();
    if (g->prep0) cudaEventDestroy(g->prep0);
    if (g->prep1) cudaEventDestroy(g->prep1);
    pool.release(g->up, g->up_bytes);
    g->b->arena = nullptr;
    g->b->ext_stage = nullptr;
    spare.push_back(std::move(g->b));
    delete g;
  }
  return progress;
}

// Admits pending requests of one mode, in arrival order, while their
// footprints fit the budget (with the resident meshes) and this epoch's
// arena, table and flags; lays them out as a segment, prepares it on the
// preparation stream and publishes it to the drain.  Returns whether a
// segment was formed.
bool vfr_server::admit() {
  vfr::Range nvtx("vfr_server admit");
  if (stopping || fatal) return false;
  std::vector<Req*> take;
  uint64_t bytes = 0;
  bool epoch_full = false;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (pending.empty()) return false;
    const int mode = pending.front()->r.mode;
    while (!pending.empty() && take.size() < max_batch) {
      Req* q = pending.front();
      if (q->r.mode != mode) break;
      if (used + q->footprint > budget - mesh_bytes) break;  // wait for memory to free up
      if (arena.off + bytes + q->footprint > arena.cap || seq >= kMaxSegs ||
          flags_used + take.size() + 1 > kMaxFlags) {
        epoch_full = true;  // this epoch's space is used up: start a new one
        break;
      }
      used += q->footprint;
      bytes += q->footprint;
      take.push_back(q);
      pending.pop_front();
    }
  }
  if (take.empty()) {
    if (epoch_full) stopping = true;
    return false;
  }
  // pinned staging of the segment's job table and prefixes
  const size_t up_bytes = sizeof(vfr::JobDev) * take.size() + sizeof(uint32_t) * 5 * (take.size() + 1);
  char* up = pool.alloc(up_bytes);
  if (!up) {  // staging in use: put the requests back and try again later
    std::lock_guard<std::mutex> lk(mu);
    for (auto it = take.rbegin(); it != take.rend(); ++it) {
      used -= (*it)->footprint;
      pending.push_front(*it);
    }
    return false;
  }
  Seg* g = new Seg;
  g->up = up;
  g->up_bytes = up_bytes;
  g->seq = seq;
  g->id = ++segments;
  g->reqs = take;
  g->remaining = (uint32_t)take.size();
  if (spare.empty()) {
    g->b.reset(new Batch);
  } else {
    g->b = std::move(spare.back());
    spare.pop_back();
  }
  Batch& B = *g->b;
  B.ctx = C;
  B.stream = prep;
  B.arena = &arena;
  B.rgb8_only = true;
  B.fb = 256;
  B.ent_cap = 0;
  B.bin_cap = 0;
  B.ext_stage = up;
  B.ext_stage_cap = up_bytes;
  std::vector<JobSpec> specs(take.size());
  for (size_t i = 0; i < take.size(); ++i) {
    const vfr_request& r = take[i]->r;
    specs[i].mesh = r.mesh_id;
    specs[i].W = r.W;
    specs[i].H = r.H;
    specs[i].use_mv = r.use_mv != 0;
    std::memcpy(specs[i].mv, r.mv, sizeof specs[i].mv);
  }
  uint32_t* flags_dev = nullptr;
  int rc = B.layout(specs, take[0]->r.mode, true);
  if (!rc) rc = B.upload(true);
  if (!rc && (cudaEventCreate(&g->prep0) != cudaSuccess || cudaEventCreate(&g->prep1) != cudaSuccess ||
              cudaEventRecord(g->prep0, prep) != cudaSuccess))
    rc = VFR_ERR_CUDA;
  if (!rc) rc = B.enqueue_a();
  if (!rc) rc = B.enqueue_b();
  if (!rc && cudaHostGetDevicePointer((void**)&flags_dev, flags, 0) != cudaSuccess) rc = VFR_ERR_CUDA;
  if (!rc) {
    if (vfr::launch_publish(segs, ctl, seq, B.d_jobs.as<vfr::JobDev>(), B.ray_pref(),
                            flags_dev + flags_used, B.njobs, prep) != cudaSuccess ||
        cudaEventRecord(g->prep1, prep) != cudaSuccess)
      rc = VFR_ERR_CUDA;
  }
  const Clock::time_point now = Clock::now();
  {
    std::lock_guard<std::mutex> lk(mu);
    for (size_t i = 0; i < take.size(); ++i) {
      Req* q = take[i];
      q->seg = g;
      q->job = (uint32_t)i;
      q->flag = flags_used + (uint32_t)i;
      q->state = St::InFlight;
      q->t_start = now;
      q->batch_id = g->id;
      q->batch_jobs = (uint32_t)take.size();
    }
  }
  flags_used += (uint32_t)take.size();
  ++seq;
  inflight.push_back(g);
  if (rc) {
    fail_all(rc);
    return true;
  }
  if (!drain_running && launch_drain() != VFR_OK) fail_all(VFR_ERR_CUDA);
  return true;
}

void vfr_server::loop() {
  cudaSetDevice(C->device);
  for (;;) {
    if (fatal) {  // every request has failed: stop the drain and leave
      if (drain_running) send_stop();
      if (!drain_running || cudaEventQuery(drain_done) != cudaErrorNotReady) break;
      std::this_thread::sleep_for(std::chrono::microseconds(50));
      continue;
    }
    bool progress = poll_completions();
    if (drain_running && cudaEventQuery(drain_done) != cudaErrorNotReady) {
      drain_running = false;  // its warps left: stopped, or the bounded idle wait gave up
      const uint32_t st = *(volatile uint32_t*)(stop + 16);
      dev_status |= st;
      if (st & VFR_DEV_QUEUE) ++queue_timeouts;
      progress = true;
    }
    const bool busy = !inflight.empty();
    if (!drain_running) {
      if (busy) {
        if (launch_drain() != VFR_OK) fail_all(VFR_ERR_CUDA);  // work left: run it
      } else if (stopping) {
        epoch_reset();
        stopping = false;
        progress = true;
      }
    }
    if (admit()) progress = true;
    bool idle, quit;
    {
      std::lock_guard<std::mutex> lk(mu);
      idle = pending.empty() && inflight.empty();
      quit = stop_req && pending.empty() && inflight.empty() && !drain_running;
    }
    if (quit) break;
    const Clock::time_point now = Clock::now();
    if (!idle) {
      last_busy = now;
    } else if (drain_running &&
               (stop_req ||
                std::chrono::duration<double, std::milli>(now - last_busy).count() > linger_ms.load())) {
      stopping = true;  // idle for a while (or shutting down): let the drain go
    }
    if (stopping && inflight.empty() && drain_running) send_stop();
    if (!progress) {
      if (busy || drain_running) {
        std::this_thread::sleep_for(std::chrono::microseconds(20));
      } else {
        std::unique_lock<std::mutex> lk(mu);
        if (pending.empty() && !stop_req) cv_work.wait_for(lk, std::chrono::milliseconds(2));
      }
    }
  }
  drain_running = false;
}

extern "C" {

int vfr_server_create(vfr_ctx* ctx, uint64_t budget_bytes, uint32_t max_batch, vfr_server** out) {
  if (!ctx || !out || budget_bytes == 0) return VFR_ERR_INVALID;
  *out = nullptr;
  vfr::Ctx& X = ctx->impl;
  cudaSetDevice(X.device);
  if (!X.d_tf) return X.fail(VFR_ERR_STATE, "tables not uploaded");
  std::unique_ptr<vfr_server> s(new vfr_server);
  s->ctx = ctx;
  s->C = &X;
  s->max_batch = max_batch ? max_batch : 256;
  const int rc = s->start(budget_bytes);
  if (rc) {
    s->release_device();
    return rc;
  }
  vfr_server* p = s.release();
  p->worker = std::thread([p] { p->loop(); });
  *out = p;
  return VFR_OK;
}

int vfr_server_submit(vfr_server* s, const vfr_request* r, uint64_t* ticket) {
  if (!s || !r || !ticket) return VFR_ERR_INVALID;
  if (!s->C->mesh(r->mesh_id)) return VFR_ERR_STATE;
  if (r->W < 2 || r->H < 2 || (uint64_t)r->W * r->H > (1ull << 28)) return VFR_ERR_INVALID;
  if (r->mode != VFR_MODE_REF && r->mode != VFR_MODE_COMPOSITED) return VFR_ERR_INVALID;
  Req* q = new Req;
  q->r = *r;
  q->footprint = s->footprint(*r);
  q->t_submit = Clock::now();
  std::lock_guard<std::mutex> g(s->mu);
  if (s->fatal || s->stop_req) {
    delete q;
    return s->fatal ? s->fatal : VFR_ERR_STATE;
  }
  if (q->footprint > std::min<uint64_t>(s->budget - s->mesh_bytes, s->arena.cap)) {
    ++s->rejected;  // can never fit: refuse now
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
  if (q->claimed) return VFR_ERR_STATE;  // another thread waits for it
  q->claimed = true;
  const auto deadline = Clock::now() + std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms);
  while (q->state != St::Done) {
    if (timeout_ms < 0) {
      s->cv_done.wait(lk);
    } else if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout &&
               q->state != St::Done) {
      q->claimed = false;  // the ticket stays valid: wait again later
      return VFR_ERR_TIMEOUT;
    }
  }
  if (info) {
    info->status = q->status;
    info->t_submit_ms = s->ms(q->t_submit);
    info->t_start_ms = q->t_start == Clock::time_point() ? info->t_submit_ms : s->ms(q->t_start);
    info->t_done_ms = s->ms(q->t_done);
    info->t_ready_ms = q->t_ready == Clock::time_point() ? info->t_done_ms : s->ms(q->t_ready);
    info->batch_id = q->batch_id;
    info->batch_jobs = q->batch_jobs;
    info->num_rays = q->num_rays;
    info->num_steps = q->num_steps;
    info->device_status = q->dev_status;
  }
  const int st = q->status;
  s->all.erase(it);
  delete q;
  return st;
}

int vfr_server_set_idle(vfr_server* s, uint32_t drain_idle_us, uint32_t linger_ms) {
  if (!s || drain_idle_us == 0) return VFR_ERR_INVALID;
  s->idle_limit = drain_idle_us;
  s->linger_ms = (double)linger_ms;
  return VFR_OK;
}

int vfr_server_stats(vfr_server* s, vfr_server_counters* out) {
  if (!s || !out) return VFR_ERR_INVALID;
  std::lock_guard<std::mutex> g(s->mu);
  out->batches = s->segments;
  out->completed = s->completed;
  out->rejected = s->rejected;
  out->pending = (uint32_t)s->pending.size();
  out->budget_used = s->used + s->mesh_bytes;
  out->rays = s->rays;
  out->steps = s->steps;
  out->launches = s->launches;
  out->epochs = s->epochs;
  out->queue_timeouts = s->queue_timeouts;
  out->mesh_bytes = s->mesh_bytes;
  out->arena_bytes = s->arena.cap;
  out->prep_ms = s->prep_ms;
  return VFR_OK;
}

void vfr_server_destroy(vfr_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop_req = true;
    s->cv_work.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();
  cudaSetDevice(s->C->device);
  s->release_device();
  for (auto& kv : s->all) {
    if (kv.second->copied) cudaEventDestroy(kv.second->copied);
    delete kv.second;
  }
  delete s;
}

}  // extern "C"
