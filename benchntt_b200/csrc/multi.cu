// multi.cu -- one job list over several GPUs (bntt_multi_*, bntt_split_by_cost).
//
// The transforms of a job list are independent, so several devices share one
// list without exchanging data: the list is split by cost, each device runs
// its part on its own batch (own context, own copy of every plan's table),
// and nothing crosses between GPUs -- no peer access, no collective.  The
// split is the longest-processing-time greedy: jobs in decreasing cost
// (N/2 * log2 N butterflies), ties by job index, each to the device with the
// least work so far (ties to the lower index), so every caller that splits
// the same list gets the same owners.
#include <algorithm>
#include <numeric>
#include <vector>

#include "batch_host.h"

struct bntt_multi {
  std::vector<bntt_batch*> batches;
  std::vector<std::vector<bntt_job>> parts;  // per device, reused between runs
};

namespace bntt {

static uint64_t job_cost(unsigned log2n) { return ((uint64_t)1 << log2n) / 2 * log2n; }

static void split_by_cost(const uint32_t* log2n, size_t count, uint32_t parts, uint32_t* owner) {
  std::vector<uint32_t> order(count);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return job_cost(log2n[a]) > job_cost(log2n[b]); });
  std::vector<uint64_t> load(parts, 0);
  for (uint32_t i : order) {
    uint32_t best = 0;
    for (uint32_t r = 1; r < parts; ++r)
      if (load[r] < load[best]) best = r;
    owner[i] = best;
    load[best] += job_cost(log2n[i]);
  }
}

}  // namespace bntt

using namespace bntt;

extern "C" {

int bntt_split_by_cost(const uint32_t* log2n, size_t count, uint32_t parts, uint32_t* owner) {
  BNTT_REQUIRE((log2n && owner) || count == 0, "NULL argument");
  BNTT_REQUIRE(parts >= 1, "parts must be at least 1");
  for (size_t i = 0; i < count; ++i)
    BNTT_REQUIRE(log2n[i] >= 1 && log2n[i] <= 24, "job %zu: log2n %u outside [1, 24]", i, log2n[i]);
  split_by_cost(log2n, count, parts, owner);
  return BNTT_OK;
}

int bntt_multi_create(bntt_multi** out, bntt_batch* const* batches, size_t n) {
  BNTT_REQUIRE(out && batches && n > 0, "NULL argument or no batches");
  *out = nullptr;
  for (size_t i = 0; i < n; ++i) {
    BNTT_REQUIRE(batches[i], "batch %zu is NULL", i);
    const bntt_batch* b0 = batches[0];
    const bntt_batch* bi = batches[i];
    BNTT_REQUIRE(bi->plans.size() == b0->plans.size(), "batch %zu holds %zu plans, batch 0 holds %zu", i,
                 bi->plans.size(), b0->plans.size());
    for (size_t k = 0; k < b0->plans.size(); ++k)
      BNTT_REQUIRE(bi->plans[k]->log2n == b0->plans[k]->log2n,
                   "batch %zu: plan %zu has log2n %u, batch 0's has %u", i, k, bi->plans[k]->log2n,
                   b0->plans[k]->log2n);
    for (size_t j = 0; j < i; ++j) BNTT_REQUIRE(batches[j] != bi, "batch %zu repeats batch %zu", i, j);
  }
  auto* m = new bntt_multi();
  m->batches.assign(batches, batches + n);
  m->parts.resize(n);
  *out = m;
  return BNTT_OK;
}

int bntt_multi_destroy(bntt_multi* m) {
  delete m;
  return BNTT_OK;
}

int bntt_multi_split(bntt_multi* m, const bntt_job* jobs, size_t count, uint32_t* owner) {
  BNTT_REQUIRE(m && ((jobs && owner) || count == 0), "NULL argument");
  const bntt_batch* b0 = m->batches[0];
  std::vector<uint32_t> log2n(count);
  for (size_t i = 0; i < count; ++i) {
    BNTT_REQUIRE(jobs[i].plan < b0->plans.size(), "job %zu: plan index %u out of range", i, jobs[i].plan);
    log2n[i] = b0->plans[jobs[i].plan]->log2n;
  }
  split_by_cost(log2n.data(), count, (uint32_t)m->batches.size(), owner);
  return BNTT_OK;
}

int bntt_multi_run_host(bntt_multi* m, const bntt_job* jobs, size_t count) {
  BNTT_REQUIRE(m && (jobs || count == 0), "NULL argument");
  const size_t nd = m->batches.size();
  std::vector<uint32_t> owner(count);
  if (int rc = bntt_multi_split(m, jobs, count, owner.data())) return rc;
  for (auto& p : m->parts) p.clear();
  for (size_t i = 0; i < count; ++i) m->parts[owner[i]].push_back(jobs[i]);
  // queue every device's part, then wait for all of them
  int first_err = BNTT_OK;
  size_t queued = 0;
  for (size_t d = 0; d < nd; ++d) {
    if (m->parts[d].empty()) continue;
    const int rc = bntt_batch_run_host_async(m->batches[d], m->parts[d].data(), m->parts[d].size());
    if (rc) {
      first_err = rc;
      break;
    }
    queued = d + 1;
  }
  for (size_t d = 0; d < queued; ++d) {
    if (m->parts[d].empty()) continue;
    const int rc = bntt_batch_sync(m->batches[d]);
    if (rc && !first_err) first_err = rc;
  }
  return first_err;
}

}  // extern "C"
