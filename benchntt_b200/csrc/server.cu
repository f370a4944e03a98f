// server.cu -- the serving loop: admission by an HBM budget, continuous
// batching over several in-flight launches, latency accounting.
//
// Submitted requests wait in a FIFO.  A worker thread, whenever one of its
// `slots` is free, admits requests from the head of the FIFO while the output
// arena (the budget) has room, builds one schedule for the admitted NTTs and
// launches the persistent kernel on the slot's stream, launches the admitted
// vvmul / axpy requests on the same stream, and records an event.  It polls
// the events of busy slots and turns finished requests into completions.
// Nothing waits for the previous launch to end before the next one starts, so
// later arrivals overlap earlier work on the device.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <thread>

#include "batch_host.h"

namespace bntt {

enum : int { OP_MUL_ = 2, OP_AXPY_ = 3 };  // launch_blas op codes

// First-fit allocator over one device region (256-byte granules).
class Arena {
 public:
  void init(char* base, size_t bytes) {
    base_ = base;
    free_.clear();
    free_[0] = bytes;
    used_ = 0;
  }
  void* alloc(size_t bytes) {
    bytes = (bytes + 255) & ~(size_t)255;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      const size_t off = it->first, rest = it->second - bytes;
      free_.erase(it);
      if (rest) free_[off + bytes] = rest;
      live_[off] = bytes;
      used_ += bytes;
      peak_ = std::max(peak_, used_);
      return base_ + off;
    }
    return nullptr;
  }
  bool release(void* p) {
    const size_t off = static_cast<char*>(p) - base_;
    auto it = live_.find(off);
    if (it == live_.end()) return false;
    size_t bytes = it->second, start = off;
    live_.erase(it);
    used_ -= bytes;
    auto nx = free_.lower_bound(start);
    if (nx != free_.end() && nx->first == start + bytes) {  // merge with next
      bytes += nx->second;
      free_.erase(nx);
    }
    auto pv = free_.lower_bound(start);
    if (pv != free_.begin()) {
      --pv;
      if (pv->first + pv->second == start) {  // merge with previous
        start = pv->first;
        bytes += pv->second;
        free_.erase(pv);
      }
    }
    free_[start] = bytes;
    return true;
  }
  size_t peak() const { return peak_; }

 private:
  char* base_ = nullptr;
  std::map<size_t, size_t> free_, live_;
  size_t used_ = 0, peak_ = 0;
};

struct PendingReq {
  bntt_request r;
  void* y = nullptr;
  size_t bytes = 0;
  double t_admit = 0;
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  bool busy = false;
  Schedule sched;
  void* dev = nullptr;  // schedule arrays on the device
  size_t dev_cap = 0;
  void* pinned = nullptr;  // the same, staged in pinned host memory
  size_t pinned_cap = 0;
  // outgrown staging buffers, freed when the server is destroyed: cudaFree and
  // cudaFreeHost wait for the whole device, which would stall the worker
  // behind every launch in flight
  std::vector<void*> old_dev, old_pinned;
  std::vector<PendingReq> reqs;
};

// Output bytes admitted into one launch (a single larger request is admitted
// alone).  Bounds the work a request can wait behind in its own launch and
// the size of a launch's schedule, so the staging buffers are sized once.
constexpr size_t kLaunchBytes = (size_t)256 << 20;

// Staging bytes of the schedule of a launch with at most `jobs` NTTs holding
// at most `elems` elements: every pass of a transform of 2^11 or more
// elements has 2^n / 1024 tiles, and a small-size tile holds one job or more.
inline size_t schedule_bytes_bound(size_t jobs, size_t elems) {
  auto r256 = [](size_t v) { return (v + 255) & ~(size_t)255; };
  const size_t large = std::min(jobs, elems >> 11);
  const size_t items = jobs + kMaxPasses * (elems >> 10);
  return r256((kCtlHeader + large * kMaxPasses) * 4) + r256(large * kMaxPasses * 4) +
         r256(items * sizeof(WorkItem)) + r256(jobs * 4) + r256(jobs * sizeof(DevJob));
}

}  // namespace bntt

using namespace bntt;

struct bntt_server {
  bntt_ctx* ctx = nullptr;
  bntt_batch* engine = nullptr;  // plans, shapes, modulus of the NTTs
  ModParams blas_mp{};
  bool blas_fast = false;
  bntt_server_config cfg{};
  void* arena_mem = nullptr;
  Arena arena;  // guarded by mu
  std::chrono::steady_clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<PendingReq> pending;
  std::vector<bntt_completion> done;
  std::vector<Slot> slots;
  std::thread worker;
  std::atomic<bool> stop{false};
  std::atomic<uint64_t> submitted{0}, completed{0}, launches{0}, admission_waits{0};
  int worker_error = BNTT_OK;
  int batch_bps = 0;  // resident batch-kernel CTAs per SM

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace bntt {

static size_t request_bytes(const bntt_server* s, const bntt_request& r) {
  if (r.kind == BNTT_REQ_NTT) return (size_t)16 << s->engine->plans[r.plan]->log2n;
  return (size_t)r.len * 16;
}

// Launches the requests in slot.reqs on the slot's stream.
static int launch_slot(bntt_server* s, Slot& slot) {
  bntt_ctx* c = s->ctx;
  std::vector<bntt_job> jobs;
  for (const PendingReq& p : slot.reqs)
    if (p.r.kind == BNTT_REQ_NTT) jobs.push_back(bntt_job{p.r.x, p.y, p.r.plan, 0});
  if (!jobs.empty()) {
    Schedule& sc = slot.sched;
    if (int rc = build_schedule(s->engine, sc, jobs.data(), jobs.size())) return rc;
    const size_t cb = (kCtlHeader + sc.nslots * kMaxPasses) * 4, pb = sc.pass_tiles.size() * 4,
                 ib = sc.items.size() * sizeof(WorkItem), ob = sc.order.size() * 4,
                 jb = sc.djobs.size() * sizeof(DevJob);
    auto r256 = [](size_t v) { return (v + 255) & ~(size_t)255; };
    const size_t o_pt = r256(cb), o_it = r256(o_pt + pb), o_or = r256(o_it + ib),
                 o_jb = r256(o_or + ob), need = r256(o_jb + jb);
    if (slot.pinned_cap < need || slot.dev_cap < need) {  // not reached within kLaunchBytes
      void *h = nullptr, *d = nullptr;
      BNTT_CK(cudaMallocHost(&h, need * 2));
      if (int rc = ctx_alloc(c, &d, need * 2)) {
        cudaFreeHost(h);
        return rc;
      }
      if (slot.pinned) slot.old_pinned.push_back(slot.pinned);
      if (slot.dev) slot.old_dev.push_back(slot.dev);
      slot.pinned = h;
      slot.dev = d;
      slot.pinned_cap = slot.dev_cap = need * 2;
    }
    char* h = static_cast<char*>(slot.pinned);
    memset(h, 0, cb);  // control words start at zero
    memcpy(h + o_pt, sc.pass_tiles.data(), pb);
    memcpy(h + o_it, sc.items.data(), ib);
    memcpy(h + o_or, sc.order.data(), ob);
    memcpy(h + o_jb, sc.djobs.data(), jb);
    char* d = static_cast<char*>(slot.dev);
    BNTT_CK(cudaMemcpyAsync(d, h, need, cudaMemcpyHostToDevice, slot.stream));
    const void* fn = batch_kernel(s->engine->fast, s->engine->layout);
    size_t smem = 0;
    for (const WorkItem& w : sc.items) smem = std::max(smem, shape_smem(w.shape));
    // occupancy queried once at creation
    const unsigned grid =
        (unsigned)std::max<size_t>(1, std::min<size_t>((size_t)s->batch_bps * c->sms, sc.items.size()));
    BatchArgs ba;
    ba.items = reinterpret_cast<const WorkItem*>(d + o_it);
    ba.nitems = (uint32_t)sc.items.size();
    ba.jobs = reinterpret_cast<const DevJob*>(d + o_jb);
    ba.order = reinterpret_cast<const uint32_t*>(d + o_or);
    ba.ctl = reinterpret_cast<uint32_t*>(d);
    ba.pass_tiles = reinterpret_cast<const uint32_t*>(d + o_pt);
    ba.wait_polls = kWaitPolls;
    ModParams mp = s->engine->mp;
    int layout = s->engine->layout;
    void* args[] = {&ba, &mp, &layout};
    BNTT_CK(cudaLaunchKernel(fn, dim3(grid), dim3(kBatchThreads), args, smem, slot.stream));
    c->launches++;
  }
  for (const PendingReq& p : slot.reqs) {
    if (p.r.kind == BNTT_REQ_NTT) continue;
    const int op = p.r.kind == BNTT_REQ_VVMUL ? OP_MUL_ : OP_AXPY_;
    if (int rc = launch_blas(c, op, p.y, p.r.x, p.r.b, to_limbs(to_u128(p.r.scalar)), (size_t)p.r.len,
                             s->blas_mp, s->blas_fast, s->engine->layout, slot.stream))
      return rc;
  }
  BNTT_CK(cudaEventRecord(slot.done, slot.stream));
  s->launches++;
  return BNTT_OK;
}

static void worker_main(bntt_server* s) {
  cudaSetDevice(s->ctx->device);
  while (!s->stop.load()) {
    bool progress = false;
    // finished launches -> completions
    for (Slot& slot : s->slots) {
      if (!slot.busy) continue;
      cudaError_t q = cudaEventQuery(slot.done);
      if (q == cudaErrorNotReady) continue;
      const double t = s->now();
      const int st = q == cudaSuccess ? BNTT_OK : cuda_error(q, "server launch");
      std::lock_guard<std::mutex> g(s->mu);
      for (const PendingReq& p : slot.reqs)
        s->done.push_back(bntt_completion{p.r.tag, p.y, p.bytes, p.r.t_arrive, p.t_admit, t, st});
      s->completed += slot.reqs.size();
      slot.reqs.clear();
      slot.busy = false;
      progress = true;
      s->cv.notify_all();
    }
    // a free slot takes the admissible head of the queue
    Slot* free_slot = nullptr;
    for (Slot& slot : s->slots)
      if (!slot.busy) {
        free_slot = &slot;
        break;
      }
    if (free_slot) {
      {
        std::lock_guard<std::mutex> g(s->mu);
        const double t = s->now();
        size_t launch_bytes = 0;
        while (!s->pending.empty() && free_slot->reqs.size() < s->cfg.max_batch) {
          PendingReq& head = s->pending.front();
          if (!free_slot->reqs.empty() && launch_bytes + head.bytes > kLaunchBytes) break;
          void* y = s->arena.alloc(head.bytes);
          if (!y) {  // wait for memory: keep arrival order
            s->admission_waits++;
            break;
          }
          head.y = y;
          head.t_admit = t;
          launch_bytes += head.bytes;
          free_slot->reqs.push_back(head);
          s->pending.pop_front();
        }
      }
      if (!free_slot->reqs.empty()) {
        int rc = launch_slot(s, *free_slot);
        if (rc) {
          s->worker_error = rc;
          // complete the requests with the error so waiters do not hang
          std::lock_guard<std::mutex> g(s->mu);
          const double t = s->now();
          for (const PendingReq& p : free_slot->reqs)
            s->done.push_back(bntt_completion{p.r.tag, p.y, p.bytes, p.r.t_arrive, p.t_admit, t, rc});
          s->completed += free_slot->reqs.size();
          free_slot->reqs.clear();
          s->cv.notify_all();
        } else {
          free_slot->busy = true;
        }
        progress = true;
      }
    }
    if (!progress) {
      bool idle;
      {
        std::lock_guard<std::mutex> g(s->mu);
        idle = s->pending.empty();
      }
      bool busy = false;
      for (Slot& slot : s->slots) busy |= slot.busy;
      if (idle && !busy) {
        std::unique_lock<std::mutex> g(s->mu);
        s->cv.wait_for(g, std::chrono::microseconds(200),
                       [&] { return !s->pending.empty() || s->stop.load(); });
      } else {
        std::this_thread::yield();
      }
    }
  }
}

}  // namespace bntt

extern "C" {

int bntt_server_create(bntt_ctx* c, bntt_server** out, bntt_plan* const* plans, size_t nplans,
                       const bntt_modulus* blas_modulus, const bntt_server_config* cfg) {
  BNTT_REQUIRE(c && out && plans && nplans && blas_modulus, "NULL argument");
  *out = nullptr;
  if (int rc = ctx_use_device(c)) return rc;
  auto* s = new bntt_server();
  s->ctx = c;
  if (cfg) s->cfg = *cfg;
  if (!s->cfg.hbm_budget) s->cfg.hbm_budget = (size_t)32 << 30;
  if (!s->cfg.slots) s->cfg.slots = 4;
  if (!s->cfg.max_batch) s->cfg.max_batch = 4096;
  int rc = bntt_batch_create(c, &s->engine, plans, nplans);
  if (!rc) rc = ctx_alloc(c, &s->arena_mem, s->cfg.hbm_budget);
  if (rc) {
    if (s->engine) bntt_batch_destroy(s->engine);
    delete s;
    return rc;
  }
  s->arena.init(static_cast<char*>(s->arena_mem), s->cfg.hbm_budget);
  if ((rc = batch_kernel_bps(batch_kernel(s->engine->fast, s->engine->layout), &s->batch_bps))) {
    ctx_free(c, s->arena_mem);
    bntt_batch_destroy(s->engine);
    delete s;
    return rc;
  }
  bool fast = false;
  s->blas_mp = make_params(*blas_modulus, &fast);
  s->blas_fast = arith_fast(c, fast);
  // staging for the largest schedule one launch can have: kLaunchBytes of
  // outputs, or one transform of the largest plan
  unsigned max_log = 0;
  for (const bntt_plan* p : s->engine->plans) max_log = std::max(max_log, p->log2n);
  const size_t stage = schedule_bytes_bound(s->cfg.max_batch, std::max(kLaunchBytes / 16, (size_t)1 << max_log));
  s->slots.resize(s->cfg.slots);
  for (Slot& slot : s->slots) {
    cudaStreamCreateWithFlags(&slot.stream, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&slot.done, cudaEventDisableTiming);
    if (!rc && cudaMallocHost(&slot.pinned, stage) == cudaSuccess) slot.pinned_cap = stage;
    else if (!rc) rc = cuda_error(cudaErrorMemoryAllocation, "cudaMallocHost of the launch staging");
    if (!rc) rc = ctx_alloc(c, &slot.dev, stage);
    if (!rc) slot.dev_cap = stage;
  }
  if (rc) {
    for (Slot& slot : s->slots) {
      if (slot.dev) ctx_free(c, slot.dev);
      if (slot.pinned) cudaFreeHost(slot.pinned);
      cudaStreamDestroy(slot.stream);
      cudaEventDestroy(slot.done);
    }
    ctx_free(c, s->arena_mem);
    bntt_batch_destroy(s->engine);
    delete s;
    return rc;
  }
  s->t0 = std::chrono::steady_clock::now();
  s->worker = std::thread(worker_main, s);
  *out = s;
  return BNTT_OK;
}

int bntt_server_destroy(bntt_server* s) {
  if (!s) return BNTT_OK;
  bntt_server_drain(s);
  s->stop = true;
  s->cv.notify_all();
  s->worker.join();
  cudaSetDevice(s->ctx->device);
  for (Slot& slot : s->slots) {
    cudaStreamSynchronize(slot.stream);
    free_schedule(s->ctx, slot.sched);
    if (slot.dev) ctx_free(s->ctx, slot.dev);
    if (slot.pinned) cudaFreeHost(slot.pinned);
    for (void* p : slot.old_dev) ctx_free(s->ctx, p);
    for (void* p : slot.old_pinned) cudaFreeHost(p);
    cudaStreamDestroy(slot.stream);
    cudaEventDestroy(slot.done);
  }
  ctx_free(s->ctx, s->arena_mem);
  bntt_batch_destroy(s->engine);
  delete s;
  return BNTT_OK;
}

double bntt_server_clock(bntt_server* s) { return s ? s->now() : 0.0; }

int bntt_server_submit(bntt_server* s, const bntt_request* r) {
  BNTT_REQUIRE(s && r, "NULL argument");
  BNTT_REQUIRE(r->kind <= BNTT_REQ_AXPY, "unknown request kind %u", r->kind);
  if (r->kind == BNTT_REQ_NTT) {
    BNTT_REQUIRE(r->plan < s->engine->plans.size(), "plan index %u out of range", r->plan);
    BNTT_REQUIRE(r->x && ((uintptr_t)r->x & 15) == 0, "NTT input must be a 16-byte aligned device pointer");
  } else {
    BNTT_REQUIRE(r->len > 0 && r->x && r->b && (((uintptr_t)r->x | (uintptr_t)r->b) & 15) == 0,
                 "BLAS operands must be 16-byte aligned device pointers");
  }
  PendingReq p;
  p.r = *r;
  p.bytes = request_bytes(s, *r);
  if (p.bytes > s->cfg.hbm_budget)
    return set_error(BNTT_EBUDGET, "request needs %zu bytes, the budget is %zu", p.bytes, s->cfg.hbm_budget);
  if (p.r.t_arrive <= 0) p.r.t_arrive = s->now();
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->pending.push_back(p);
  }
  s->submitted++;
  s->cv.notify_all();
  return BNTT_OK;
}

int bntt_server_poll(bntt_server* s, bntt_completion* out, size_t cap, size_t* n) {
  BNTT_REQUIRE(s && n && (out || cap == 0), "NULL argument");
  std::lock_guard<std::mutex> g(s->mu);
  const size_t k = std::min(cap, s->done.size());
  std::copy(s->done.begin(), s->done.begin() + k, out);
  s->done.erase(s->done.begin(), s->done.begin() + k);
  *n = k;
  return BNTT_OK;
}

int bntt_server_release(bntt_server* s, void* y) {
  BNTT_REQUIRE(s && y, "NULL argument");
  bool ok;
  {
    std::lock_guard<std::mutex> g(s->mu);
    ok = s->arena.release(y);
  }
  s->cv.notify_all();
  BNTT_REQUIRE(ok, "%p is not a live server output", y);
  return BNTT_OK;
}

int bntt_server_drain(bntt_server* s) {
  BNTT_REQUIRE(s, "NULL argument");
  std::unique_lock<std::mutex> g(s->mu);
  s->cv.wait(g, [&] { return s->completed.load() >= s->submitted.load(); });
  return s->worker_error;
}

int bntt_server_get_stats(bntt_server* s, bntt_server_stats* st) {
  BNTT_REQUIRE(s && st, "NULL argument");
  std::lock_guard<std::mutex> g(s->mu);
  st->submitted = s->submitted;
  st->completed = s->completed;
  st->launches = s->launches;
  st->admission_waits = s->admission_waits;
  st->peak_bytes = s->arena.peak();
  return BNTT_OK;
}

int bntt_server_replay(bntt_server* s, const bntt_request* reqs, size_t n, int serial,
                       double* latency_s, double* wall_s) {
  return bntt_server_replay_ex(s, reqs, n, serial, latency_s, nullptr, wall_s);
}

int bntt_server_replay_ex(bntt_server* s, const bntt_request* reqs, size_t n, int serial,
                          double* latency_s, double* service_s, double* wall_s) {
  BNTT_REQUIRE(s && (reqs || n == 0) && latency_s && wall_s, "NULL argument");
  if (n == 0) {
    *wall_s = 0;
    return BNTT_OK;
  }
  for (size_t i = 1; i < n; ++i)
    BNTT_REQUIRE(reqs[i].t_arrive >= reqs[i - 1].t_arrive, "requests must be in arrival order");
  if (int rc = ctx_use_device(s->ctx)) return rc;
  const double base = s->now() + 1e-3;
  double last_done = base;
  if (serial) {
    // one call at a time: each request alone on the context stream, waited for
    size_t out_bytes = 0;
    for (size_t i = 0; i < n; ++i) out_bytes = std::max(out_bytes, request_bytes(s, reqs[i]));
    void* y = nullptr;
    {
      std::lock_guard<std::mutex> g(s->mu);
      y = s->arena.alloc(out_bytes);
    }
    if (!y) return set_error(BNTT_EBUDGET, "arena cannot hold the largest request");
    int rc = BNTT_OK;
    for (size_t i = 0; i < n && !rc; ++i) {
      const bntt_request& r = reqs[i];
      const double t_arr = base + r.t_arrive;
      while (s->now() < t_arr) {
      }
      const double t_start = s->now();  // the call begins: its admission
      if (r.kind == BNTT_REQ_NTT) {
        rc = ntt_forward_on(s->engine->plans[r.plan], y, r.x, 1, s->ctx->stream);
      } else {
        rc = launch_blas(s->ctx, r.kind == BNTT_REQ_VVMUL ? OP_MUL_ : OP_AXPY_, y, r.x, r.b,
                         to_limbs(to_u128(r.scalar)), (size_t)r.len, s->blas_mp, s->blas_fast,
                         s->engine->layout, s->ctx->stream);
      }
      if (!rc) {
        cudaError_t e = cudaStreamSynchronize(s->ctx->stream);
        if (e != cudaSuccess) rc = cuda_error(e, "serial replay");
      }
      last_done = s->now();
      latency_s[i] = last_done - t_arr;
      if (service_s) service_s[i] = last_done - t_start;
    }
    {
      std::lock_guard<std::mutex> g(s->mu);
      s->arena.release(y);
    }
    *wall_s = last_done - base;
    return rc;
  }
  // continuous batching: submit at arrival times, collect as they finish
  std::vector<bntt_completion> got(1024);
  size_t received = 0;
  int rc = BNTT_OK;
  auto collect = [&]() {
    size_t k = 0;
    bntt_server_poll(s, got.data(), got.size(), &k);
    for (size_t j = 0; j < k; ++j) {
      const bntt_completion& cpl = got[j];
      if (cpl.tag < n) {
        latency_s[cpl.tag] = cpl.t_done - cpl.t_arrive;
        if (service_s) service_s[cpl.tag] = cpl.t_done - cpl.t_admit;
      }
      if (cpl.status && !rc) rc = cpl.status;
      last_done = std::max(last_done, cpl.t_done);
      bntt_server_release(s, cpl.y);
    }
    received += k;
  };
  for (size_t i = 0; i < n && !rc; ++i) {
    bntt_request r = reqs[i];
    r.t_arrive = base + reqs[i].t_arrive;
    r.tag = i;
    while (s->now() < r.t_arrive) collect();
    if (int e = bntt_server_submit(s, &r)) return e;
  }
  while (received < n && !rc) {
    collect();
    if (received < n) std::this_thread::yield();
  }
  *wall_s = last_done - base;
  return rc;
}

}  // extern "C"
