// batch_build.cu -- the device half of a new job list's schedule.
//
// bntt_batch_run_dev and bntt_batch_run_inverse_dev meet a new job list
// whenever the caller's list changes (serving traffic: every step).  The host
// validates the jobs, counts them per size and writes the work items; the
// per-job part -- a 32-byte descriptor per job and the size-sorted order of
// the small jobs -- is written here, from a copy of the caller's job array,
// so the host does not write (and copy) it for every new list.
//
// Small jobs land in their size's segment of the order by warp-aggregated
// atomics, so their order within a segment depends on timing; every job is
// still in exactly one tile of its size, and results do not depend on which.
#include "batch_host.h"

namespace bntt {

constexpr uint32_t kNotSmall = 31;

__global__ void __launch_bounds__(256) k_build_jobs(const bntt_job* raw, uint32_t count,
                                                    const PlanRef* plans, const LargeRef* large,
                                                    uint32_t nlarge, SizeFirst first, uint32_t* fill,
                                                    DevJob* djobs, uint32_t* order) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  // large jobs: their descriptors carry the counter slot the host assigned
  if (i < nlarge) {
    const LargeRef L = large[i];
    const bntt_job j = raw[L.job];
    const PlanRef p = plans[j.plan];
    djobs[L.job] = DevJob{static_cast<const uint4*>(j.x), static_cast<uint4*>(j.y), p.tw, p.log2n, L.slot};
  }
  uint32_t n = kNotSmall;
  if (i < count) {
    const bntt_job j = raw[i];
    const PlanRef p = plans[j.plan];
    if (p.log2n <= 10) {
      n = p.log2n;
      djobs[i] = DevJob{static_cast<const uint4*>(j.x), static_cast<uint4*>(j.y), p.tw, p.log2n, 0u};
    }
  }
  // one atomic per size present in the warp (every launch is whole warps)
  const unsigned peers = __match_any_sync(0xffffffffu, n);
  if (n != kNotSmall) {
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&fill[n], (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    order[first.first[n] + base + (uint32_t)__popc(peers & ((1u << lane) - 1u))] = i;
  }
}

int launch_build_jobs(const bntt_job* raw, size_t count, const PlanRef* plans, const LargeRef* large,
                      uint32_t nlarge, const uint32_t first[11], uint32_t* fill, DevJob* djobs,
                      uint32_t* order, cudaStream_t stream) {
  if (count == 0) return BNTT_OK;
  SizeFirst f;
  for (int k = 0; k < 11; ++k) f.first[k] = first[k];
  const unsigned grid = (unsigned)((count + 255) / 256);
  k_build_jobs<<<grid, 256, 0, stream>>>(raw, (uint32_t)count, plans, large, nlarge, f, fill, djobs, order);
  BNTT_CK(cudaGetLastError());
  return BNTT_OK;
}

}  // namespace bntt
