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
  std::vector<uint32_t> pass_tiles;
  size_t nslots = 0;
  void* d_jobs = nullptr;
  size_t d_jobs_cap = 0;
  void* d_order = nullptr;
  size_t d_order_cap = 0;
  void* d_items = nullptr;
  size_t d_items_cap = 0;
  void* d_ctl = nullptr;
  size_t d_ctl_cap = 0;
  void* d_pass_tiles = nullptr;
  size_t d_pass_tiles_cap = 0;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t exec_stream = nullptr;  // stream the graph was captured on
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
  std::vector<bntt_job> last_jobs;
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
  // fault injection for tests of the failure path (bntt_batch_inject_wait_timeout)
  uint32_t inject_polls = 0;
  // inverse runs (bntt_batch_run_inverse_dev)
  std::vector<bntt_job> inv_last_jobs;
  bntt::Schedule inv;
};


namespace bntt {
int grow(bntt_ctx* c, void** p, size_t* cap, size_t bytes);
void free_schedule(bntt_ctx* c, Schedule& s);
const void* batch_kernel(bool fast);
const void* batch_kernel_inverse();
size_t shape_smem(int s);
// inverse = true: the jobs' inverse transforms (plans' inverse tables, the
// passes of a large job queued last to first)
int build_schedule(const bntt_batch* b, Schedule& sc, const bntt_job* jobs, size_t count,
                   bool inverse = false);
}  // namespace bntt
