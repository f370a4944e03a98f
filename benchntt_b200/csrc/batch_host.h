// batch_host.h -- host-side structures of the batch engine, shared by
// batch.cu (bntt_batch_*) and server.cu (the serving loop).
#pragma once
#include "batch_dev.cuh"

namespace bntt {

// Shape choice per size: small tiles, interleaved passes, contiguous passes.
struct ShapeChoice {
  int small[11];
  int pass_il[11];
  int pass_contig[11];
};

// One job list turned into work items, with its device copies and graph.
struct Schedule {
  std::vector<DevJob> djobs;
  std::vector<uint32_t> order;
  std::vector<WorkItem> items;
  std::vector<WorkItem> small_items;  // make_items' scratch: the small tiles before interleaving
  std::vector<uint32_t> pass_tiles;
  std::vector<WorkItem> later[kMaxPasses];  // build scratch: pass items by run position
  std::vector<uint8_t> job_log2n;           // build scratch: each job's size
  std::vector<uint32_t> large;              // build scratch: jobs above 2^10 points
  std::vector<uint8_t> large_n;             // build scratch: their sizes
  std::vector<const uint4*> plan_tw;        // build scratch: the plans' tables
  std::vector<uint8_t> plan_log2n;
  size_t nslots = 0;
  // device-built schedules (bntt_batch_run_dev / run_inverse_dev): djobs and
  // order are left empty on the host; k_build_jobs writes them on the device
  // from a copy of the caller's job array, the plans' table and the large
  // jobs' slots
  bool dev_build = false;
  size_t count = 0;                         // jobs in the list
  uint32_t small = 0;                       // jobs of at most 2^10 points
  uint32_t first[11] = {};                  // first position of each small size
  const bntt_job* raw = nullptr;            // the caller's jobs (valid during the upload)
  // the latest device-built list as copied into pinned staging: a later call
  // with the same jobs is recognised by comparing with it (the staging buffer
  // is rewritten only by the upload after next)
  const bntt_job* staged_raw = nullptr;
  size_t staged_count = 0;
  std::vector<PlanRef> plan_ref;
  std::vector<LargeRef> large_ref;
  // device copies of djobs, order, items and pass_tiles in one buffer, two
  // buffers used in turn: a new job list is copied into the one the running
  // launches do not read, so the copy overlaps them
  void* d_sched[2] = {nullptr, nullptr};
  size_t d_sched_cap[2] = {0, 0};
  cudaEvent_t set_free[2] = {nullptr, nullptr};  // after the last launch reading d_sched[i]
  bool set_used[2] = {false, false};
  int cur = 1;                        // buffer of the current job list
  cudaEvent_t set_ready = nullptr;    // the current list's copy has landed
  void* d_ctl = nullptr;              // control words (queue head, error word, pass counters)
  size_t d_ctl_cap = 0;
  cudaGraphExec_t exec = nullptr;     // captured when the same job list runs again
  std::vector<cudaGraphExec_t> retired;  // graphs of earlier job lists, destroyed once idle
  // pinned staging of the uploads, two buffers used in turn: an upload waits
  // only for the copy that read the same buffer two uploads before
  void* stage[2] = {nullptr, nullptr};
  size_t stage_cap[2] = {0, 0};
  cudaEvent_t stage_done[2] = {nullptr, nullptr};
  int stage_next = 0;
  cudaStream_t stream = nullptr;      // stream the schedule was uploaded for
  bool inverse = false;               // k_batch_inv instead of k_batch
  bool sticky_err = false;            // launches leave the error word alone
  BatchArgs args{};
  int grid = 0;
  size_t smem = 0;
};

}  // namespace bntt

struct bntt_batch {
  bntt_ctx* ctx = nullptr;
  std::vector<bntt_plan*> plans;
  bntt::ModParams mp{};
  bool fast = false;
  int layout = 0;
  bntt::ShapeChoice shapes{};
  // device-pointer runs
  bntt::Schedule main;
  // host-pointer runs: packed device region, job groups with own schedules
  std::vector<bntt_job> host_last_jobs;
  std::vector<bntt::Schedule> groups;
  std::vector<size_t> group_first;   // first job of each group (+ end)
  std::vector<size_t> dev_off;       // byte offset of each job in the region
  void* region = nullptr;
  size_t region_cap = 0;
  uint32_t* group_err = nullptr;     // pinned copies of the groups' error words
  size_t group_err_cap = 0;
  std::vector<cudaEvent_t> group_out;  // per group: its output copy of the latest run
  bool group_out_recorded = false;
  bool host_inflight = false;        // host runs not yet passed to bntt_batch_sync
  bool host_err_pending = false;     // an error of runs finished before a rebuild
  size_t last_launches = 0;
  // the latest run was bntt_batch_run_dev_noalloc: bntt_batch_status reads
  // the error word it left in the shared no-allocation array
  const uint32_t* noalloc_err = nullptr;
  // fault injection for tests of the failure path (bntt_batch_inject_wait_timeout)
  uint32_t inject_polls = 0;
  // inverse runs (bntt_batch_run_inverse_dev)
  bntt::Schedule inv;
  cudaStream_t upload_stream = nullptr;  // schedule copies of device-pointer runs
};


namespace bntt {
// device buffer of at least `bytes` (headroom: a quarter more when it grows)
int grow(bntt_ctx* c, void** p, size_t* cap, size_t bytes, bool headroom = false);
void free_schedule(bntt_ctx* c, Schedule& s);
const void* batch_kernel(bool fast, int layout);
const void* batch_kernel_inverse(int layout);
// resident CTAs per SM of a batch kernel (cached per device)
int batch_kernel_bps(const void* fn, int* bps);
size_t shape_smem(int s);
// inverse = true: the jobs' inverse transforms (plans' inverse tables, the
// passes of a large job queued last to first)
int build_schedule(const bntt_batch* b, Schedule& sc, const bntt_job* jobs, size_t count,
                   bool inverse = false);
// The host half of a schedule whose descriptors and size order k_build_jobs
// writes on the device; the job array must stay valid until the upload.
int build_schedule_dev(const bntt_batch* b, Schedule& sc, const bntt_job* jobs, size_t count,
                       bool inverse = false);
// k_build_jobs (batch_build.cu): descriptors of `count` jobs and the order of
// the small ones, from device copies of the job array, the plans' table and
// the large jobs' slots; fill[11] must be zero.
int launch_build_jobs(const bntt_job* raw, size_t count, const PlanRef* plans, const LargeRef* large,
                      uint32_t nlarge, const uint32_t first[11], uint32_t* fill, DevJob* djobs,
                      uint32_t* order, cudaStream_t stream);
}  // namespace bntt
