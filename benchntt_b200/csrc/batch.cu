// batch.cu -- host side of the batch engine (schedules, uploads, CUDA graphs)
// and the bntt_batch_* entry points.  Device code: batch_dev.cuh,
// instantiated in batch_kfast.cu / batch_kref.cu.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>

#include "batch_host.h"

namespace bntt {

const void* batch_kernel_fast_minb(int minb, int layout);
const void* batch_kernel_ref();

// Resident CTAs per SM the fast batch kernel is compiled for (2 to 5,
// default 4), read once at start-up from BNTT_BATCH_MINB.
static const int g_batch_minb = [] {
  const char* e = getenv("BNTT_BATCH_MINB");
  const int v = e ? atoi(e) : 4;
  return v == 2 || v == 3 || v == 5 ? v : 4;
}();

size_t shape_smem(int s) {
  const BatchShape& b = kShapes[s];
  const int npass = (b.m + b.logr - 1) / b.logr;
  if (npass <= 1) return 0;
  if (b.m <= 2) return (size_t)b.tpc * ((size_t)1 << b.m) * 16;  // one-thread tiles
  return NttEngine<kBatchLogR, ArithFast>::smem_slots(b.m, b.map, kBatchThreads) * 16;
}

// Resident CTAs per SM of a batch kernel (forward or inverse) at the largest
// tile's shared memory, per device.  Every tile fits the default 48 KB of
// dynamic shared memory, so no launch raises the kernel's limit: a limit set
// for one job list (and lowered for the next) would fail launches of others
// that share the kernel, such as the serving loop's.
int batch_kernel_bps(const void* fn, int* bps) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, int> cache;
  int dev = 0;
  BNTT_CK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  auto it = cache.find({fn, dev});
  if (it != cache.end()) {
    *bps = it->second;
    return BNTT_OK;
  }
  size_t smem = 0;
  for (int k = 0; k < kNumShapes; ++k) smem = std::max(smem, shape_smem(k));
  BNTT_REQUIRE(smem <= 48 * 1024, "batch tile needs %zu bytes of shared memory", smem);
  int b = 0;
  BNTT_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, kBatchThreads, smem));
  if (b < 1) return set_error(BNTT_ECUDA, "batch kernel does not fit on an SM (smem %zu)", smem);
  cache[{fn, dev}] = b;
  *bps = b;
  return BNTT_OK;
}

// First shape for (m, map) with the preferred radix (0 = any).
int batch_shape_for(int m, int map, int logr_pref) {
  for (int s = 0; s < kNumShapes; ++s)
    if (kShapes[s].m == m && kShapes[s].map == map && (logr_pref ? kShapes[s].logr == logr_pref : true))
      return s;
  return -1;
}

}  // namespace bntt

using namespace bntt;

namespace bntt {

int grow(bntt_ctx* c, void** p, size_t* cap, size_t bytes, bool headroom) {
  if (*cap >= bytes && *p) return BNTT_OK;
  if (*p) ctx_free(c, *p);  // waits for the device: rare with headroom
  *p = nullptr;
  *cap = 0;
  const size_t want = std::max<size_t>(headroom ? bytes + bytes / 4 : bytes, 256);
  if (int rc = ctx_alloc(c, p, want)) return rc;
  *cap = want;
  return BNTT_OK;
}

void free_schedule(bntt_ctx* c, Schedule& s) {
  if (s.exec) cudaGraphExecDestroy(s.exec);
  s.exec = nullptr;
  for (cudaGraphExec_t e : s.retired) cudaGraphExecDestroy(e);
  s.retired.clear();
  for (int i = 0; i < 2; ++i) {
    if (s.stage_done[i]) cudaEventSynchronize(s.stage_done[i]);
    if (s.set_free[i]) cudaEventSynchronize(s.set_free[i]);
    if (s.stage[i]) cudaFreeHost(s.stage[i]);
    s.staged_raw = nullptr;
    s.staged_count = 0;
    if (s.stage_done[i]) cudaEventDestroy(s.stage_done[i]);
    if (s.set_free[i]) cudaEventDestroy(s.set_free[i]);
    if (s.d_sched[i]) ctx_free(c, s.d_sched[i]);
    s.stage[i] = s.d_sched[i] = nullptr;
    s.stage_done[i] = s.set_free[i] = nullptr;
    s.stage_cap[i] = s.d_sched_cap[i] = 0;
    s.set_used[i] = false;
  }
  if (s.set_ready) cudaEventDestroy(s.set_ready);
  s.set_ready = nullptr;
  if (s.d_ctl) ctx_free(c, s.d_ctl);
  s.d_ctl = nullptr;
  s.d_ctl_cap = 0;
}

const void* batch_kernel(bool fast, int layout) {
  return fast ? batch_kernel_fast_minb(g_batch_minb, layout) : batch_kernel_ref();
}

constexpr int kMaxLog2n = 24;  // plans hold 2^1..2^24 points

// HBM passes of a large batch job: the fewest passes, then the fewest
// engine passes (a pass of m stages is ceil(m / 2) of them).  A strided pass
// (all but the last) has 5..7 stages, so its tile of 2^(10 - m) adjacent
// columns covers at least 128 bytes of each row, and needs that many columns
// (2^(10 - m) <= 2^l); the last, contiguous pass has 3..10 stages.
static std::vector<int> batch_split(int n) {
  std::vector<int> best, cur;
  int best_passes = 1 << 30, best_cost = 1 << 30;
  std::function<void(int, int, int)> rec = [&](int s0, int cost, int depth) {
    const int left = n - s0;
    if (left >= 3 && left <= 10) {  // finish with a contiguous pass
      cur.push_back(left);
      const int passes = (int)cur.size(), c = cost + (left + 1) / 2;
      if (passes < best_passes || (passes == best_passes && c < best_cost)) {
        best_passes = passes;
        best_cost = c;
        best = cur;
      }
      cur.pop_back();
    }
    if (depth + 1 >= kMaxPasses) return;
    for (int m = 7; m >= 5; --m) {
      const int l = n - s0 - m;
      if (l < 3 || 10 - m > l) continue;
      cur.push_back(m);
      rec(s0 + m, cost + (m + 1) / 2, depth + 1);
      cur.pop_back();
    }
  };
  rec(0, 0, 0);
  return best;
}

// batch_split for every size a batch job can have, computed once.
static const std::vector<int>& split_of(int n) {
  static const std::vector<std::vector<int>> table = [] {
    std::vector<std::vector<int>> t(kMaxLog2n + 1);
    for (int m = 11; m <= kMaxLog2n; ++m) t[m] = batch_split(m);
    return t;
  }();
  return table[n];
}

std::vector<int> tile_split(int n) { return n >= 11 && n <= kMaxLog2n ? split_of(n) : std::vector<int>{}; }

// The plans' fields, looked up once instead of per job.
static void plan_fields(const bntt_batch* b, Schedule& sc, bool inverse) {
  const size_t np = b->plans.size();
  sc.plan_tw.resize(np);
  sc.plan_log2n.resize(np);
  for (size_t k = 0; k < np; ++k) {
    sc.plan_tw[k] = static_cast<const uint4*>(inverse ? b->plans[k]->tw_inv : b->plans[k]->tw);
    sc.plan_log2n[k] = (uint8_t)b->plans[k]->log2n;
  }
}

// First position of each small size in the size-sorted order, largest size
// first; returns the number of small jobs.
static uint32_t size_offsets(const uint32_t per_size[11], uint32_t first[11]) {
  uint32_t small = 0;
  first[0] = 0;
  for (int n = 10; n >= 1; --n) {
    first[n] = small;
    small += per_size[n];
  }
  return small;
}

// The work items of a job list from its per-size counts and its large jobs
// (sc.large / sc.large_n, slot = position there): passes that run first,
// small tiles from the largest size down, the other passes in run order.
static int make_items(const bntt_batch* b, Schedule& sc, const uint32_t per_size[11],
                      const uint32_t first[11], bool inverse) {
  sc.items.clear();
  for (auto& l : sc.later) l.clear();
  sc.nslots = sc.large.size();
  sc.pass_tiles.assign(sc.nslots * kMaxPasses, 0);
  for (size_t slot = 0; slot < sc.large.size(); ++slot) {
    const uint32_t ji = sc.large[slot];
    const int n = sc.large_n[slot];
    const std::vector<int>& passes = split_of(n);
    BNTT_REQUIRE(!passes.empty() && passes.size() <= (size_t)kMaxPasses, "log2n %d needs too many passes", n);
    int s0 = 0;
    for (size_t p = 0; p < passes.size(); ++p) {
      const int m = passes[p];
      const int l = n - s0 - m;
      const int shape = l > 0 ? b->shapes.pass_il[m] : b->shapes.pass_contig[m];
      BNTT_REQUIRE(shape >= 0, "no batch shape for pass m=%d", m);
      const uint32_t tpc = (uint32_t)kShapes[shape].tpc;
      const uint64_t nsub = 1ull << (n - m);
      const uint32_t tiles = (uint32_t)((nsub + tpc - 1) / tpc);
      sc.pass_tiles[slot * kMaxPasses + p] = tiles;
      // position in the run order: forward pass p runs p-th, the inverse runs
      // the passes last to first
      const size_t run = inverse ? passes.size() - 1 - p : p;
      std::vector<WorkItem>& q = sc.later[run];
      WorkItem w{};
      w.shape = (uint16_t)shape;
      w.kind = ITEM_PASS;
      w.a = ji;
      w.pass = (uint16_t)p;
      w.wait = (uint16_t)((run > 0 ? 1 : 0) | (run == 0 ? 2 : 0) | (s0 << 8));
      for (uint32_t t = 0; t < tiles; ++t) {
        w.b = t * tpc;
        q.push_back(w);
      }
      s0 += m;
    }
  }
  std::vector<WorkItem>& small = sc.small_items;
  small.clear();
  for (int n = 10; n >= 1; --n) {
    const uint32_t cnt = per_size[n];
    if (cnt == 0) continue;
    const int shape = b->shapes.small[n];
    BNTT_REQUIRE(shape >= 0, "no batch shape for size 2^%d", n);
    const uint32_t tpc = (uint32_t)kShapes[shape].tpc;
    WorkItem w{};
    w.shape = (uint16_t)shape;
    w.kind = ITEM_SMALL;
    for (uint32_t s = 0; s < cnt; s += tpc) {
      w.a = first[n] + s;
      w.b = std::min<uint32_t>(tpc, cnt - s);
      small.push_back(w);
    }
  }
  // first passes, then the small tiles cut into one segment before each
  // later pass group, so a later pass is queued well after the pass it
  // waits for
  int groups = 0;
  for (int p = 1; p < kMaxPasses; ++p) groups += sc.later[p].empty() ? 0 : 1;
  sc.items.insert(sc.items.end(), sc.later[0].begin(), sc.later[0].end());
  size_t from = 0;
  int seg = 0;
  for (int p = 1; p < kMaxPasses; ++p) {
    if (sc.later[p].empty()) continue;
    const size_t to = small.size() * (size_t)(++seg) / (size_t)(groups + 1);
    sc.items.insert(sc.items.end(), small.begin() + from, small.begin() + to);
    from = to;
    sc.items.insert(sc.items.end(), sc.later[p].begin(), sc.later[p].end());
  }
  sc.items.insert(sc.items.end(), small.begin() + from, small.end());
  return BNTT_OK;
}

// One validating pass over the jobs: sizes counted per small size, large
// jobs listed.  `fill` also writes the jobs' device descriptors.
static int scan_jobs(const bntt_batch* b, Schedule& sc, const bntt_job* jobs, size_t count,
                     uint32_t per_size[11], bool fill) {
  const size_t np = b->plans.size();
  const uint4* const* tw = sc.plan_tw.data();
  const uint8_t* plog = sc.plan_log2n.data();
  sc.large.clear();
  sc.large_n.clear();
  if (fill) {
    sc.djobs.resize(count);
    sc.job_log2n.resize(count);
  }
  for (size_t i = 0; i < count; ++i) {
    const bntt_job& jb = jobs[i];
    BNTT_REQUIRE(jb.plan < np, "job %zu: plan index %u out of range", i, jb.plan);
    BNTT_REQUIRE(jb.x && jb.y, "job %zu: NULL buffer", i);
    BNTT_REQUIRE((((uintptr_t)jb.x | (uintptr_t)jb.y) & 15) == 0, "job %zu: buffers must be 16-byte aligned", i);
    const uint32_t n = plog[jb.plan];
    if (n <= 10) {
      ++per_size[n];
    } else {
      sc.large.push_back((uint32_t)i);
      sc.large_n.push_back((uint8_t)n);
    }
    if (fill) {
      DevJob& d = sc.djobs[i];
      d.x = static_cast<const uint4*>(jb.x);
      d.y = static_cast<uint4*>(jb.y);
      d.tw = tw[jb.plan];
      d.log2n = n;
      d.slot = n <= 10 ? 0u : (uint32_t)(sc.large.size() - 1);
      sc.job_log2n[i] = (uint8_t)n;
    }
  }
  return BNTT_OK;
}

int build_schedule(const bntt_batch* b, Schedule& sc, const bntt_job* jobs, size_t count,
                   bool inverse) {
  sc.dev_build = false;
  plan_fields(b, sc, inverse);
  uint32_t per_size[11] = {}, first[11], fill[11];
  if (int rc = scan_jobs(b, sc, jobs, count, per_size, true)) return rc;
  // small jobs in size order, largest size first (a counting sort over the
  // compact size array)
  const uint32_t small = size_offsets(per_size, first);
  std::copy(first, first + 11, fill);
  sc.order.resize(small);
  const uint8_t* sizes = sc.job_log2n.data();
  for (size_t i = 0; i < count; ++i) {
    const uint32_t n = sizes[i];
    if (n <= 10) sc.order[fill[n]++] = (uint32_t)i;
  }
  return make_items(b, sc, per_size, first, inverse);
}

// The host half of a schedule whose job descriptors and size order the
// device builds (k_build_jobs): validation, sizes, work items, the table of
// large jobs and the plans' table.  The caller's job array is read again by
// the upload that follows.
int build_schedule_dev(const bntt_batch* b, Schedule& sc, const bntt_job* jobs, size_t count,
                       bool inverse) {
  sc.dev_build = true;
  plan_fields(b, sc, inverse);
  uint32_t per_size[11] = {};
  if (int rc = scan_jobs(b, sc, jobs, count, per_size, false)) return rc;
  sc.small = size_offsets(per_size, sc.first);
  sc.count = count;
  sc.raw = jobs;
  sc.djobs.clear();
  sc.order.clear();
  sc.plan_ref.resize(b->plans.size());
  for (size_t k = 0; k < b->plans.size(); ++k) sc.plan_ref[k] = PlanRef{sc.plan_tw[k], sc.plan_log2n[k], 0u};
  sc.large_ref.resize(sc.large.size());
  for (size_t k = 0; k < sc.large.size(); ++k) sc.large_ref[k] = LargeRef{sc.large[k], (uint32_t)k};
  return make_items(b, sc, per_size, sc.first, inverse);
}

// Graphs of earlier job lists; the caller has synchronized `sc.stream`.
static void destroy_retired(Schedule& sc) {
  for (cudaGraphExec_t e : sc.retired) cudaGraphExecDestroy(e);
  sc.retired.clear();
}

// Copies the schedule to the device and sizes its launch on `stream`.  The
// copy goes through pinned staging into the device buffer that the previous
// job list's launches do not read; with `copy_stream` it runs there, waiting
// only for the last launch that read that buffer, so it overlaps the launches
// in flight, and `stream` waits for it.  Without, it is queued on `stream`.
// The previous list's graph is retired, not destroyed, since a replay of it
// may still be running.  sticky_err: launches leave the error word alone (it
// is cleared here and by whoever reads it), so errors of several launches
// accumulate until they are read.
static int upload(bntt_batch* b, Schedule& sc, cudaStream_t stream, bool inverse = false,
                  bool sticky_err = false, cudaStream_t copy_stream = nullptr) {
  bntt_ctx* c = b->ctx;
  const size_t ib = sc.items.size() * sizeof(WorkItem), cb = (kCtlHeader + sc.nslots * kMaxPasses) * 4,
               pb = sc.pass_tiles.size() * 4;
  auto r256 = [](size_t v) { return (v + 255) & ~(size_t)255; };
  // Host-built: [djobs][order][items][pass tiles], all copied.  Device-built:
  // [the caller's jobs][plans][large jobs][items][pass tiles] copied, then
  // [djobs][order][fill counters] written on the device by k_build_jobs.
  size_t o_jb = 0, o_ob = 0, o_ib = 0, o_pb = 0, staged = 0, total = 0;
  size_t o_raw = 0, o_plan = 0, o_large = 0, o_fill = 0;
  if (!sc.dev_build) {
    const size_t jb = sc.djobs.size() * sizeof(DevJob), ob = sc.order.size() * 4;
    o_ob = r256(jb);
    o_ib = o_ob + r256(ob);
    o_pb = o_ib + r256(ib);
    staged = total = o_pb + r256(pb);
  } else {
    const size_t rb = sc.count * sizeof(bntt_job), plb = sc.plan_ref.size() * sizeof(PlanRef),
                 lb = sc.large_ref.size() * sizeof(LargeRef);
    o_plan = r256(rb);
    o_large = o_plan + r256(plb);
    o_ib = o_large + r256(lb);
    o_pb = o_ib + r256(ib);
    staged = o_pb + r256(pb);
    o_jb = staged;
    o_ob = o_jb + r256(sc.count * sizeof(DevJob));
    o_fill = o_ob + r256((size_t)sc.small * 4);
    total = o_fill + 256;
  }
  if (sc.exec) {
    sc.retired.push_back(sc.exec);
    sc.exec = nullptr;
  }
  if (sc.retired.size() > 8) {  // bound the graphs kept alive
    BNTT_CK(cudaStreamSynchronize(sc.stream ? sc.stream : stream));
    destroy_retired(sc);
  }
  const int set = sc.cur ^ 1;
  cudaStream_t cs = copy_stream ? copy_stream : stream;
  if (int rc = grow(c, &sc.d_sched[set], &sc.d_sched_cap[set], total, true)) return rc;
  if (int rc = grow(c, &sc.d_ctl, &sc.d_ctl_cap, cb, true)) return rc;
  if (sc.set_used[set] && cs != stream) BNTT_CK(cudaStreamWaitEvent(cs, sc.set_free[set], 0));
  const int si = sc.stage_next;
  sc.stage_next ^= 1;
  if (sc.stage_done[si]) BNTT_CK(cudaEventSynchronize(sc.stage_done[si]));
  else BNTT_CK(cudaEventCreateWithFlags(&sc.stage_done[si], cudaEventDisableTiming));
  if (sc.stage_cap[si] < staged) {
    if (sc.stage[si]) cudaFreeHost(sc.stage[si]);
    sc.stage[si] = nullptr;
    sc.stage_cap[si] = 0;
    BNTT_CK(cudaMallocHost(&sc.stage[si], staged + staged / 2));
    sc.stage_cap[si] = staged + staged / 2;
  }
  char* h = static_cast<char*>(sc.stage[si]);
  if (!sc.dev_build) {
    if (!sc.djobs.empty()) memcpy(h + o_jb, sc.djobs.data(), sc.djobs.size() * sizeof(DevJob));
    if (!sc.order.empty()) memcpy(h + o_ob, sc.order.data(), sc.order.size() * 4);
  } else {
    if (sc.count) memcpy(h + o_raw, sc.raw, sc.count * sizeof(bntt_job));
    sc.staged_raw = reinterpret_cast<const bntt_job*>(h + o_raw);
    sc.staged_count = sc.count;
    memcpy(h + o_plan, sc.plan_ref.data(), sc.plan_ref.size() * sizeof(PlanRef));
    if (!sc.large_ref.empty()) memcpy(h + o_large, sc.large_ref.data(), sc.large_ref.size() * sizeof(LargeRef));
    sc.raw = nullptr;  // the caller's array is not read after this point
  }
  if (ib) memcpy(h + o_ib, sc.items.data(), ib);
  if (pb) {
    uint32_t* t = reinterpret_cast<uint32_t*>(h + o_pb);
    memcpy(t, sc.pass_tiles.data(), pb);
    if (b->inject_polls)  // injected fault: every wait needs one tile more than exists
      for (size_t i = 0; i < sc.pass_tiles.size(); ++i) t[i] += 1;
  }
  char* d = static_cast<char*>(sc.d_sched[set]);
  BNTT_CK(cudaMemcpyAsync(d, h, staged, cudaMemcpyHostToDevice, cs));
  BNTT_CK(cudaEventRecord(sc.stage_done[si], cs));
  // descriptors and size order, built on the device after the copy, on the
  // copy's stream: the build runs while earlier launches finish (it writes
  // only the buffer they do not read), off the path between two launches
  if (sc.dev_build && sc.count) {
    BNTT_CK(cudaMemsetAsync(d + o_fill, 0, 256, cs));
    if (int rc = launch_build_jobs(reinterpret_cast<const bntt_job*>(d + o_raw), sc.count,
                                   reinterpret_cast<const PlanRef*>(d + o_plan),
                                   reinterpret_cast<const LargeRef*>(d + o_large),
                                   (uint32_t)sc.large_ref.size(), sc.first, reinterpret_cast<uint32_t*>(d + o_fill),
                                   reinterpret_cast<DevJob*>(d + o_jb), reinterpret_cast<uint32_t*>(d + o_ob), cs))
      return rc;
    c->launches++;
    b->last_launches++;
  }
  if (cs != stream) {
    if (!sc.set_ready) BNTT_CK(cudaEventCreateWithFlags(&sc.set_ready, cudaEventDisableTiming));
    BNTT_CK(cudaEventRecord(sc.set_ready, cs));
    BNTT_CK(cudaStreamWaitEvent(stream, sc.set_ready, 0));
  }
  sc.cur = set;
  if (sticky_err) BNTT_CK(cudaMemsetAsync(sc.d_ctl, 0, cb, stream));
  sc.stream = stream;
  sc.inverse = inverse;
  sc.sticky_err = sticky_err;
  sc.grid = 0;
  if (sc.items.empty()) return BNTT_OK;
  const void* fn = inverse ? batch_kernel_inverse(b->layout) : batch_kernel(b->fast, b->layout);
  size_t smem = 0;
  bool used[kNumShapes] = {};
  for (const WorkItem& w : sc.items) used[w.shape] = true;
  for (int s = 0; s < kNumShapes; ++s)
    if (used[s]) smem = std::max(smem, shape_smem(s));
  int bps = 0;
  if (int rc = batch_kernel_bps(fn, &bps)) return rc;
  sc.grid = (int)std::min<size_t>((size_t)bps * c->sms, sc.items.size());
  sc.smem = smem;
  BatchArgs& ba = sc.args;
  ba.items = reinterpret_cast<const WorkItem*>(d + o_ib);
  ba.nitems = (uint32_t)sc.items.size();
  ba.jobs = reinterpret_cast<const DevJob*>(d + o_jb);
  ba.order = reinterpret_cast<const uint32_t*>(d + o_ob);
  ba.ctl = static_cast<uint32_t*>(sc.d_ctl);
  ba.pass_tiles = reinterpret_cast<const uint32_t*>(d + o_pb);
  ba.wait_polls = b->inject_polls ? b->inject_polls : kWaitPolls;
  return BNTT_OK;
}

// [clear the control words, kernel] of an uploaded schedule on `stream`.
static cudaError_t enqueue_run(bntt_batch* b, Schedule& sc, cudaStream_t stream) {
  const size_t cb = (kCtlHeader + sc.nslots * kMaxPasses) * 4;
  cudaError_t e;
  if (!sc.sticky_err) {
    e = cudaMemsetAsync(sc.d_ctl, 0, cb, stream);
  } else {  // ctl[0] (queue head) and ctl[2..] (pass counters), not ctl[1]
    e = cudaMemsetAsync(sc.d_ctl, 0, 4, stream);
    if (e == cudaSuccess && cb > 8) e = cudaMemsetAsync(static_cast<char*>(sc.d_ctl) + 8, 0, cb - 8, stream);
  }
  if (e != cudaSuccess) return e;
  const void* fn = sc.inverse ? batch_kernel_inverse(b->layout) : batch_kernel(b->fast, b->layout);
  BatchArgs ba = sc.args;
  ModParams mp = b->mp;
  int layout = b->layout;
  void* args[] = {&ba, &mp, &layout};
  return cudaLaunchKernel(fn, dim3(sc.grid), dim3(kBatchThreads), args, sc.smem, stream);
}

// Captures the schedule's launch into a graph for later replays.
static int capture(bntt_batch* b, Schedule& sc) {
  if (sc.exec || sc.grid == 0) return BNTT_OK;
  cudaGraph_t graph = nullptr;
  BNTT_CK(cudaStreamBeginCapture(sc.stream, cudaStreamCaptureModeThreadLocal));
  const cudaError_t e1 = enqueue_run(b, sc, sc.stream);
  const cudaError_t e2 = cudaStreamEndCapture(sc.stream, &graph);
  if (e1 != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return cuda_error(e1, "batch launch (capture)");
  }
  if (e2 != cudaSuccess) return cuda_error(e2, "cudaStreamEndCapture");
  const cudaError_t e3 = cudaGraphInstantiate(&sc.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e3 != cudaSuccess) {
    sc.exec = nullptr;
    return cuda_error(e3, "cudaGraphInstantiate");
  }
  return BNTT_OK;
}

// A replay of the captured graph, or the launch itself when there is none.
static int launch_schedule(bntt_batch* b, Schedule& sc, cudaStream_t stream) {
  if (sc.grid == 0) return BNTT_OK;
  if (sc.exec) {
    BNTT_CK(cudaGraphLaunch(sc.exec, stream));
  } else {
    const cudaError_t e = enqueue_run(b, sc, stream);
    if (e != cudaSuccess) return cuda_error(e, "batch launch");
  }
  if (!sc.set_free[sc.cur]) BNTT_CK(cudaEventCreateWithFlags(&sc.set_free[sc.cur], cudaEventDisableTiming));
  BNTT_CK(cudaEventRecord(sc.set_free[sc.cur], stream));
  sc.set_used[sc.cur] = true;
  b->ctx->launches++;
  b->last_launches++;
  return BNTT_OK;
}

static int schedule_status(Schedule& sc) {
  if (!sc.d_ctl) return BNTT_OK;
  uint32_t err = 0;
  BNTT_CK(cudaMemcpy(&err, static_cast<uint32_t*>(sc.d_ctl) + 1, 4, cudaMemcpyDeviceToHost));
  if (err) return set_error(BNTT_ETIMEOUT, "a pass of a large transform waited too long for its predecessor");
  return BNTT_OK;
}

}  // namespace bntt

extern "C" {

int bntt_batch_create(bntt_ctx* c, bntt_batch** out, bntt_plan* const* plans, size_t nplans) {
  BNTT_REQUIRE(c && out && plans && nplans > 0, "NULL argument");
  *out = nullptr;
  for (size_t i = 0; i < nplans; ++i) {
    BNTT_REQUIRE(plans[i] && plans[i]->ctx == c, "plan %zu is NULL or from another context", i);
    BNTT_REQUIRE(memcmp(&plans[i]->mod, &plans[0]->mod, sizeof(bntt_modulus)) == 0 &&
                     plans[i]->layout == plans[0]->layout,
                 "all plans of a batch must share modulus and layout");
  }
  if (int rc = ctx_use_device(c)) return rc;
  auto* b = new bntt_batch();
  b->ctx = c;
  b->plans.assign(plans, plans + nplans);
  b->mp = plans[0]->mp;
  b->fast = arith_fast(c, plans[0]->fast);
  b->layout = plans[0]->layout;
  for (int m = 0; m <= 10; ++m) {
    const int tuned = tuned_batch_small_shape(m);
    b->shapes.small[m] = tuned >= 0 ? tuned : batch_shape_for(m, MAP_CONTIG, 0);
    b->shapes.pass_il[m] = batch_shape_for(m, MAP_INTERLEAVED, 0);
    b->shapes.pass_contig[m] = batch_shape_for(m, MAP_CONTIG, 4);
    if (b->shapes.pass_contig[m] < 0) b->shapes.pass_contig[m] = batch_shape_for(m, MAP_CONTIG, 0);
  }
  if (cudaError_t e = cudaStreamCreateWithFlags(&b->upload_stream, cudaStreamNonBlocking)) {
    delete b;
    return cuda_error(e, "cudaStreamCreateWithFlags");
  }
  *out = b;
  return BNTT_OK;
}

int bntt_batch_destroy(bntt_batch* b) {
  if (!b) return BNTT_OK;
  bntt_ctx* c = b->ctx;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (int s = 0; s < 2; ++s) cudaStreamSynchronize(c->copy_stream[s]);
  if (b->upload_stream) cudaStreamSynchronize(b->upload_stream);
  free_schedule(c, b->main);
  free_schedule(c, b->inv);
  for (Schedule& s : b->groups) free_schedule(c, s);
  if (b->region) ctx_free(c, b->region);
  if (b->group_err) cudaFreeHost(b->group_err);
  for (cudaEvent_t e : b->group_out) cudaEventDestroy(e);
  if (b->upload_stream) cudaStreamDestroy(b->upload_stream);
  delete b;
  return BNTT_OK;
}

// The job list `sc` was last uploaded with (its staged copy), on `stream`.
static bool same_list(const Schedule& sc, const bntt_job* jobs, size_t count, cudaStream_t stream) {
  return sc.staged_raw && sc.staged_count == count && sc.stream == stream &&
         memcmp(sc.staged_raw, jobs, count * sizeof(bntt_job)) == 0;
}

int bntt_batch_run_dev(bntt_batch* b, const bntt_job* jobs, size_t count) {
  BNTT_REQUIRE(b && (jobs || count == 0), "NULL argument");
  if (int rc = ctx_use_device(b->ctx)) return rc;
  b->last_launches = 0;
  b->noalloc_err = nullptr;
  if (count == 0) return BNTT_OK;
  const bool inject = b->inject_polls != 0;
  const bool same = !inject && same_list(b->main, jobs, count, b->ctx->stream);
  if (!same) {  // a new list is launched directly; a graph is captured if it comes again
    b->main.staged_raw = nullptr;
    if (int rc = build_schedule_dev(b, b->main, jobs, count, false)) return rc;
    if (int rc = upload(b, b->main, b->ctx->stream, false, false, b->upload_stream)) return rc;
    if (inject) b->main.staged_raw = nullptr;  // the next run rebuilds without the injected fault
  } else if (int rc = capture(b, b->main)) {
    return rc;
  }
  b->inject_polls = 0;  // an injected fault lasts one run
  return launch_schedule(b, b->main, b->ctx->stream);
}

// Inverse transforms of a job list: same schedule machinery, the inverse
// kernel, the plans' inverse tables (built on first use).
int bntt_batch_run_inverse_dev(bntt_batch* b, const bntt_job* jobs, size_t count) {
  BNTT_REQUIRE(b && (jobs || count == 0), "NULL argument");
  if (int rc = ctx_use_device(b->ctx)) return rc;
  b->last_launches = 0;
  b->noalloc_err = nullptr;
  if (count == 0) return BNTT_OK;
  BNTT_REQUIRE(b->fast, "the inverse transform needs q = 2^124 - k (k < 2^28), mu = floor(2^251/q) "
               "and the default arithmetic");
  for (bntt_plan* p : b->plans)
    if (int rc = plan_ensure_inverse(p)) return rc;
  const bool same = same_list(b->inv, jobs, count, b->ctx->stream);
  if (!same) {
    b->inv.staged_raw = nullptr;
    if (int rc = build_schedule_dev(b, b->inv, jobs, count, true)) return rc;
    if (int rc = upload(b, b->inv, b->ctx->stream, true, false, b->upload_stream)) return rc;
  } else if (int rc = capture(b, b->inv)) {
    return rc;
  }
  return launch_schedule(b, b->inv, b->ctx->stream);
}

int bntt_batch_status(bntt_batch* b) {
  BNTT_REQUIRE(b, "NULL batch");
  if (int rc = ctx_use_device(b->ctx)) return rc;
  BNTT_CK(cudaStreamSynchronize(b->ctx->stream));
  destroy_retired(b->main);
  destroy_retired(b->inv);
  if (b->noalloc_err) {  // the latest run used the shared no-allocation array
    uint32_t err = 0;
    BNTT_CK(cudaMemcpy(&err, b->noalloc_err, 4, cudaMemcpyDeviceToHost));
    if (err) return set_error(BNTT_ETIMEOUT, "a pass of a large transform waited too long for its predecessor");
    return BNTT_OK;
  }
  if (int rc = schedule_status(b->main)) return rc;
  if (int rc = schedule_status(b->inv)) return rc;
  for (Schedule& s : b->groups)
    if (int rc = schedule_status(s)) return rc;
  return BNTT_OK;
}

size_t bntt_batch_last_launches(bntt_batch* b) { return b ? b->last_launches : 0; }

// Reads and clears the host groups' error words (the host pipeline's graphs
// leave them sticky); every host-run stream must be idle.
static int host_groups_status(bntt_batch* b) {
  bntt_ctx* c = b->ctx;
  cudaStream_t s = c->copy_stream[1];
  const size_t ng = b->groups.size();
  for (size_t g = 0; g < ng; ++g) {
    b->group_err[g] = 0;
    if (!b->groups[g].d_ctl) continue;
    uint32_t* w = static_cast<uint32_t*>(b->groups[g].d_ctl) + 1;
    BNTT_CK(cudaMemcpyAsync(&b->group_err[g], w, 4, cudaMemcpyDeviceToHost, s));
    BNTT_CK(cudaMemsetAsync(w, 0, 4, s));
  }
  BNTT_CK(cudaStreamSynchronize(s));
  bool err = b->host_err_pending;
  b->host_err_pending = false;
  for (size_t g = 0; g < ng; ++g) err |= b->group_err[g] != 0;
  if (err) return set_error(BNTT_ETIMEOUT, "a pass of a large transform waited too long for its predecessor");
  return BNTT_OK;
}

// Host buffers: jobs are packed into one device region (in place), split into
// groups of about 1/16 of the bytes each.  Group g's inputs go up on one copy
// stream, its graph runs on the context stream, its outputs come back on the
// other copy stream, so transfers of neighbouring groups overlap each other
// and the kernels.  Host copies of jobs adjacent in host memory are merged.
// Schedules and graphs are cached while the job list stays the same.  A run
// returns once it is queued: the next run's input copy of group g waits only
// for this run's output copy of group g, so back-to-back runs keep both copy
// directions busy across the boundary between runs.
int bntt_batch_run_host_async(bntt_batch* b, const bntt_job* jobs, size_t count) {
  BNTT_REQUIRE(b && (jobs || count == 0), "NULL argument");
  bntt_ctx* c = b->ctx;
  if (int rc = ctx_use_device(c)) return rc;
  b->last_launches = 0;
  b->noalloc_err = nullptr;
  if (count == 0) return BNTT_OK;
  cudaStream_t s_in = c->copy_stream[0], s_out = c->copy_stream[1], s_run = c->stream;
  const bool inject = b->inject_polls != 0;
  const bool same = !inject && b->host_last_jobs.size() == count &&
                    memcmp(b->host_last_jobs.data(), jobs, count * sizeof(bntt_job)) == 0;
  for (size_t i = 0; i < count && !same; ++i) {
    BNTT_REQUIRE(jobs[i].plan < b->plans.size(), "job %zu: plan index out of range", i);
    BNTT_REQUIRE(jobs[i].x && jobs[i].y, "job %zu: NULL buffer", i);
  }
  auto bytes_of = [&](size_t i) { return (size_t)16 << b->plans[jobs[i].plan]->log2n; };
  if (!same) {
    // earlier runs may still use the region and the groups' schedules: let
    // them finish and keep their status for the next bntt_batch_sync
    BNTT_CK(cudaStreamSynchronize(s_in));
    BNTT_CK(cudaStreamSynchronize(s_run));
    BNTT_CK(cudaStreamSynchronize(s_out));
    if (b->host_inflight) {
      const int rc = host_groups_status(b);
      b->host_err_pending = rc == BNTT_ETIMEOUT;
      if (rc && rc != BNTT_ETIMEOUT) return rc;
      b->host_inflight = false;
    }
    b->host_last_jobs.clear();
    size_t total = 0;
    b->dev_off.assign(count, 0);
    for (size_t i = 0; i < count; ++i) {
      b->dev_off[i] = total;
      total += bytes_of(i);
    }
    if (int rc = grow(c, &b->region, &b->region_cap, total)) return rc;
    // 16 groups: copies in, kernels and copies out of neighbouring groups
    // overlap; fewer groups leave longer pipeline fill and drain, more add
    // launch and event overhead (measured on B200 over PCIe Gen5 x16).
    const size_t target = std::max<size_t>(total / 16, 8u << 20);
    b->group_first.clear();
    b->group_first.push_back(0);
    size_t acc = 0;
    for (size_t i = 0; i < count; ++i) {
      acc += bytes_of(i);
      if (acc >= target && i + 1 < count) {
        b->group_first.push_back(i + 1);
        acc = 0;
      }
    }
    b->group_first.push_back(count);
    const size_t ng = b->group_first.size() - 1;
    for (size_t g = ng; g < b->groups.size(); ++g) free_schedule(c, b->groups[g]);
    b->groups.resize(ng);
    std::vector<bntt_job> dj(jobs, jobs + count);
    for (size_t i = 0; i < count; ++i) {
      void* p = static_cast<char*>(b->region) + b->dev_off[i];
      dj[i].x = p;
      dj[i].y = p;
    }
    for (size_t g = 0; g < ng; ++g) {
      const size_t f = b->group_first[g], e = b->group_first[g + 1];
      if (int rc = build_schedule(b, b->groups[g], dj.data() + f, e - f)) return rc;
      if (int rc = upload(b, b->groups[g], s_run, false, true)) return rc;
      if (int rc = capture(b, b->groups[g])) return rc;
    }
    if (b->group_err_cap < ng) {
      if (b->group_err) cudaFreeHost(b->group_err);
      b->group_err = nullptr;
      b->group_err_cap = 0;
      BNTT_CK(cudaMallocHost(&b->group_err, ng * sizeof(uint32_t)));
      b->group_err_cap = ng;
    }
    // a fresh event per group: "group g's output copy of the latest run"
    for (cudaEvent_t e : b->group_out) cudaEventDestroy(e);
    b->group_out.assign(ng, nullptr);
    for (cudaEvent_t& e : b->group_out) BNTT_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->group_out_recorded = false;
    if (!inject) b->host_last_jobs.assign(jobs, jobs + count);
  }
  b->inject_polls = 0;  // an injected fault lasts one run
  // work queued earlier on the context stream comes first
  BNTT_CK(cudaEventRecord(c->ev[0], s_run));
  BNTT_CK(cudaStreamWaitEvent(s_in, c->ev[0], 0));
  BNTT_CK(cudaStreamWaitEvent(s_out, c->ev[0], 0));
  char* region = static_cast<char*>(b->region);
  const size_t ng = b->groups.size();
  for (size_t g = 0; g < ng; ++g) {
    const size_t f = b->group_first[g], e = b->group_first[g + 1];
    // the previous run's output copy of this group has left the region
    if (b->group_out_recorded) BNTT_CK(cudaStreamWaitEvent(s_in, b->group_out[g], 0));
    for (size_t i = f; i < e;) {  // merged input copies
      size_t j = i + 1, run = bytes_of(i);
      while (j < e && static_cast<const char*>(jobs[j].x) == static_cast<const char*>(jobs[i].x) + run) {
        run += bytes_of(j);
        ++j;
      }
      BNTT_CK(cudaMemcpyAsync(region + b->dev_off[i], jobs[i].x, run, cudaMemcpyHostToDevice, s_in));
      i = j;
    }
    cudaEvent_t in_done = c->ev[1 + (g % 3)], run_done = c->ev[4 + (g % 3)];
    BNTT_CK(cudaEventRecord(in_done, s_in));
    BNTT_CK(cudaStreamWaitEvent(s_run, in_done, 0));
    if (int rc = launch_schedule(b, b->groups[g], s_run)) return rc;
    BNTT_CK(cudaEventRecord(run_done, s_run));
    BNTT_CK(cudaStreamWaitEvent(s_out, run_done, 0));
    for (size_t i = f; i < e;) {  // merged output copies
      size_t j = i + 1, run = bytes_of(i);
      while (j < e && static_cast<char*>(jobs[j].y) == static_cast<char*>(jobs[i].y) + run) {
        run += bytes_of(j);
        ++j;
      }
      BNTT_CK(cudaMemcpyAsync(jobs[i].y, region + b->dev_off[i], run, cudaMemcpyDeviceToHost, s_out));
      i = j;
    }
    BNTT_CK(cudaEventRecord(b->group_out[g], s_out));
  }
  b->group_out_recorded = true;
  b->host_inflight = true;
  return BNTT_OK;
}

int bntt_batch_sync(bntt_batch* b) {
  BNTT_REQUIRE(b, "NULL batch");
  bntt_ctx* c = b->ctx;
  if (int rc = ctx_use_device(c)) return rc;
  BNTT_CK(cudaStreamSynchronize(c->copy_stream[0]));
  BNTT_CK(cudaStreamSynchronize(c->stream));
  BNTT_CK(cudaStreamSynchronize(c->copy_stream[1]));
  for (Schedule& s : b->groups) destroy_retired(s);
  if (!b->host_inflight && !b->host_err_pending) return BNTT_OK;
  b->host_inflight = false;
  return host_groups_status(b);
}

int bntt_batch_run_host(bntt_batch* b, const bntt_job* jobs, size_t count) {
  if (int rc = bntt_batch_run_host_async(b, jobs, count)) return rc;
  return bntt_batch_sync(b);
}

}  // extern "C"

namespace bntt {

int batch_shape_count() { return kNumShapes; }

int batch_shape_info(int s, int* m, int* logr, int* tpc, int* map) {
  *m = kShapes[s].m;
  *logr = kShapes[s].logr;
  *tpc = kShapes[s].tpc;
  *map = kShapes[s].map;
  return BNTT_OK;
}

// Median time of the persistent kernel over `count` contiguous transforms of
// one plan with small-tile shape `shape` (autotuner measurement).
int batch_time_uniform(bntt_ctx* c, bntt_plan* plan, int shape, size_t count, void* x, void* y,
                       float* ms) {
  bntt_batch* b = nullptr;
  if (int rc = bntt_batch_create(c, &b, &plan, 1)) return rc;
  b->shapes.small[plan->log2n] = shape;
  count = std::min<size_t>(count, 65536);
  const size_t bytes = (size_t)16 << plan->log2n;
  std::vector<bntt_job> jobs(count);
  for (size_t i = 0; i < count; ++i) {
    jobs[i].x = static_cast<char*>(x) + i * bytes;
    jobs[i].y = static_cast<char*>(y) + i * bytes;
    jobs[i].plan = 0;
    jobs[i].reserved = 0;
  }
  int rc = bntt_batch_run_dev(b, jobs.data(), count);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  std::vector<float> t;
  if (!rc) {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int r = 0; r < 5 && !rc; ++r) {
      cudaEventRecord(e0, c->stream);
      rc = bntt_batch_run_dev(b, jobs.data(), count);
      cudaEventRecord(e1, c->stream);
      cudaError_t e = cudaEventSynchronize(e1);
      if (!rc && e != cudaSuccess) rc = cuda_error(e, "autotune batch timing");
      float v = 0;
      cudaEventElapsedTime(&v, e0, e1);
      t.push_back(v);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  bntt_batch_destroy(b);
  if (rc) return rc;
  std::sort(t.begin(), t.end());
  *ms = t[t.size() / 2];
  return BNTT_OK;
}

}  // namespace bntt

// The plain per-call path over the same job list: every job is its own
// forward transform, launched separately (one launch per transform of at most
// 1024 points, one per HBM pass above).  This is the comparison point of the
// persistent kernel, issued from C so that only launch cost is measured.
extern "C" int bntt_batch_run_percall_dev(bntt_batch* b, const bntt_job* jobs, size_t count) {
  BNTT_REQUIRE(b && (jobs || count == 0), "NULL argument");
  if (int rc = ctx_use_device(b->ctx)) return rc;
  b->last_launches = 0;
  b->noalloc_err = nullptr;
  const uint64_t before = b->ctx->launches;
  for (size_t i = 0; i < count; ++i) {
    BNTT_REQUIRE(jobs[i].plan < b->plans.size(), "job %zu: plan index out of range", i);
    BNTT_REQUIRE(jobs[i].x && jobs[i].y && (((uintptr_t)jobs[i].x | (uintptr_t)jobs[i].y) & 15) == 0,
                 "job %zu: NULL or misaligned buffer", i);
    if (int rc = ntt_forward_on(b->plans[jobs[i].plan], jobs[i].y, jobs[i].x, 1, b->ctx->stream)) return rc;
  }
  b->last_launches = (size_t)(b->ctx->launches - before);
  return BNTT_OK;
}

// ------------------------------------------------ run without allocating
// Some callers cannot allocate device memory when they submit work: their
// device memory is already reserved by another allocator (a framework's
// caching pool that holds nearly all of HBM), or they sit on a latency
// critical path where cudaMalloc / cudaFree would stall the device, or they
// must not meet an out-of-memory error after initialisation.  For them the
// batch run below keeps its scratch -- the work items, job descriptors, size
// order and control words the persistent kernel reads and updates -- in one
// fixed array compiled into the library instead of buffers from cudaMalloc.
namespace bntt {

constexpr size_t kNoAllocScratchBytes = 4u << 20;  // 4 MiB on every GPU that loads the library
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static size_t round256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace bntt

extern "C" int bntt_batch_run_dev_noalloc(bntt_batch* b, const bntt_job* jobs, size_t count) {
  BNTT_REQUIRE(b && (jobs || count == 0), "NULL argument");
  bntt_ctx* c = b->ctx;
  if (int rc = ctx_use_device(c)) return rc;
  b->last_launches = 0;
  b->noalloc_err = nullptr;
  // The schedule is copied from host vectors that are freed when this call
  // returns; captured into a graph, those copies would read freed memory at
  // every replay.  Checked before any other CUDA call, so a refused call
  // leaves the capture intact.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  BNTT_CK(cudaStreamIsCapturing(c->stream, &cap));
  BNTT_REQUIRE(cap == cudaStreamCaptureStatusNone,
               "bntt_batch_run_dev_noalloc cannot run while its stream is being captured");
  if (count == 0) return BNTT_OK;
  // Once per context, with its device current: the device address of the
  // array (its name is only a host-side stand-in in host code).
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> g(c->mu);
    if (!c->noalloc_base) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(no-alloc scratch)");
      c->noalloc_base = p;
    }
    base = c->noalloc_base;
  }
  Schedule sc;  // host-side vectors only
  if (int rc = build_schedule(b, sc, jobs, count)) return rc;
  const size_t cb = (kCtlHeader + sc.nslots * kMaxPasses) * 4, pb = sc.pass_tiles.size() * 4,
               ib = sc.items.size() * sizeof(WorkItem), ob = sc.order.size() * 4,
               jb = sc.djobs.size() * sizeof(DevJob);
  const size_t o_ctl = 0, o_pt = round256(o_ctl + cb), o_it = round256(o_pt + pb),
               o_or = round256(o_it + ib), o_jb = round256(o_or + ob), need = round256(o_jb + jb);
  if (need > kNoAllocScratchBytes)
    return set_error(BNTT_EINVAL,
                     "this job list needs %zu bytes of scratch; the no-allocation entry point "
                     "holds at most %zu (about 70,000 transforms; split the list)",
                     need, kNoAllocScratchBytes);
  char* s = static_cast<char*>(base);
  cudaStream_t st = c->stream;
  // the array keeps the previous call's contents: the control words (queue
  // head, error word, pass counters) must start at zero
  BNTT_CK(cudaMemsetAsync(s + o_ctl, 0, cb, st));
  b->noalloc_err = reinterpret_cast<const uint32_t*>(s + o_ctl) + 1;
  if (pb) BNTT_CK(cudaMemcpyAsync(s + o_pt, sc.pass_tiles.data(), pb, cudaMemcpyHostToDevice, st));
  if (ib) BNTT_CK(cudaMemcpyAsync(s + o_it, sc.items.data(), ib, cudaMemcpyHostToDevice, st));
  if (ob) BNTT_CK(cudaMemcpyAsync(s + o_or, sc.order.data(), ob, cudaMemcpyHostToDevice, st));
  if (jb) BNTT_CK(cudaMemcpyAsync(s + o_jb, sc.djobs.data(), jb, cudaMemcpyHostToDevice, st));
  if (sc.items.empty()) return BNTT_OK;
  const void* fn = batch_kernel(b->fast, b->layout);
  size_t smem = 0;
  bool used[kNumShapes] = {};
  for (const WorkItem& w : sc.items) used[w.shape] = true;
  for (int k = 0; k < kNumShapes; ++k)
    if (used[k]) smem = std::max(smem, shape_smem(k));
  int bps = 0;
  if (int rc = batch_kernel_bps(fn, &bps)) return rc;
  const unsigned grid = (unsigned)std::min<size_t>((size_t)bps * c->sms, sc.items.size());
  BatchArgs ba;
  ba.items = reinterpret_cast<const WorkItem*>(s + o_it);
  ba.nitems = (uint32_t)sc.items.size();
  ba.jobs = reinterpret_cast<const DevJob*>(s + o_jb);
  ba.order = reinterpret_cast<const uint32_t*>(s + o_or);
  ba.ctl = reinterpret_cast<uint32_t*>(s + o_ctl);
  ba.pass_tiles = reinterpret_cast<const uint32_t*>(s + o_pt);
  ba.wait_polls = kWaitPolls;
  ModParams mp = b->mp;
  int layout = b->layout;
  void* args[] = {&ba, &mp, &layout};
  BNTT_CK(cudaLaunchKernel(fn, dim3(grid), dim3(kBatchThreads), args, smem, st));
  c->launches++;
  b->last_launches = 1;
  return BNTT_OK;
}

// Fault injection for tests of the failure path: the next bntt_batch_run_dev
// makes every wait of a later HBM pass require one tile more than the earlier
// pass has, and gives up after `poll_limit` polls (about 100 ns each).  The
// kernel ends normally, the affected transforms are left incomplete, and
// bntt_batch_status() reports BNTT_ETIMEOUT.  No GPU fault is involved.
extern "C" int bntt_batch_inject_wait_timeout(bntt_batch* b, uint32_t poll_limit) {
  BNTT_REQUIRE(b && poll_limit > 0, "NULL batch or zero poll limit");
  b->inject_polls = poll_limit;
  return BNTT_OK;
}
