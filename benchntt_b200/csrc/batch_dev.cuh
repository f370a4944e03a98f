// batch_dev.cuh -- device side of the batch engine: many independent transforms of uneven sizes in one persistent,
// graph-launched work-queue kernel.
//
// Work items (16 bytes each) are tiles of 256 threads:
//   SMALL   TPC transforms of one size 2^n <= 1024, taken from a list of
//           jobs sorted by size (one sub-transform per job)
//   PASS p  TPC sub-transforms of HBM pass p of one large transform
//           (n > 10, passes from engine_split: at most kBatchMaxPass stages
//           so strided passes keep >= 8 adjacent columns, and the fewest
//           engine passes: 2^16 = 8 + 8, 2^20 = 8 + 6 + 6)
// A CTA takes the next item with an atomic counter.  Queue order is: all
// first passes of large jobs, then small tiles from the largest size down,
// then later passes.  Pass p > 0 of a job reads what pass p-1 wrote, so its
// tiles first wait until the job's pass p-1 counter reaches that pass's tile
// count.  The wait cannot deadlock: every pass p-1 tile was handed out
// before any pass p tile and its CTA finishes it without waiting.  The wait is
// still bounded; when it gives up it raises the error word, the tile is
// skipped, and bntt_batch_status() reports BNTT_ETIMEOUT.
//
// The control words (queue head, error word, per-job pass counters) live in a
// device workspace owned by the batch and are cleared by a memset node of the
// same CUDA graph before each launch.
#pragma once
#include "internal.h"
#include "ntt_core.cuh"
#include "ntt_engine.cuh"

namespace bntt {

constexpr int kBatchThreads = 256;
// Largest HBM pass of a large transform (engine_split): a strided pass of
// 2^m points has 256 >> (m - 3) adjacent columns per tile, and at least 8
// (128 contiguous bytes per row) keep its loads coalesced.
constexpr int kBatchMaxPass = 8;

struct DevJob {
  const uint4* x;
  uint4* y;
  const uint4* tw;
  uint32_t log2n;
  uint32_t slot;  // counter slot for large jobs
};

// Device build of a new job list's descriptors (k_build_jobs): a plan's table
// and size, and a large job's counter slot.
struct PlanRef {
  const uint4* tw;
  uint32_t log2n;
  uint32_t pad;
};
struct LargeRef {
  uint32_t job;
  uint32_t slot;
};
// first position of each small size in the size-sorted order
struct SizeFirst {
  uint32_t first[11];
};

enum : uint32_t { ITEM_SMALL = 0, ITEM_PASS = 1 };

struct WorkItem {
  uint16_t shape;   // index into the shape table below
  uint16_t kind;    // ITEM_SMALL or ITEM_PASS
  uint32_t a;       // SMALL: first position in the size-sorted order; PASS: job index
  uint32_t b;       // SMALL: number of jobs in the tile; PASS: first sub-transform id
  uint16_t pass;    // PASS: pass index
  uint16_t wait;    // PASS: bit 0 the tile waits for the pass run before it,
                    // bit 1 the pass reads the job's input, bits 8.. its first stage
};
static_assert(sizeof(WorkItem) == 16, "work item layout");

// Tile shapes of the persistent kernel (all 256 threads).  Sizes 2^1 and
// 2^2 use unrolled one-thread tiles; every other size and both mappings run
// on NttEngine<kBatchLogR> (4 elements per thread), whose code is shared by
// all of them.  TPC = 256 / (threads per sub-transform).  Interleaved
// (strided) tiles keep at least 8 adjacent columns (128 bytes of each row).
constexpr int kBatchLogR = 2;
#define BNTT_BATCH_SHAPES(X)               \
  X(0, 1, 1, 256, MAP_CONTIG)              \
  X(1, 2, 2, 256, MAP_CONTIG)              \
  X(2, 3, 2, 128, MAP_CONTIG)              \
  X(3, 4, 2, 64, MAP_CONTIG)               \
  X(4, 5, 2, 32, MAP_CONTIG)               \
  X(5, 6, 2, 16, MAP_CONTIG)               \
  X(6, 7, 2, 8, MAP_CONTIG)                \
  X(7, 8, 2, 4, MAP_CONTIG)                \
  X(8, 9, 2, 2, MAP_CONTIG)                \
  X(9, 10, 2, 1, MAP_CONTIG)               \
  X(10, 5, 2, 32, MAP_INTERLEAVED)         \
  X(11, 6, 2, 16, MAP_INTERLEAVED)         \
  X(12, 7, 2, 8, MAP_INTERLEAVED)

struct BatchShape {
  int m, logr, tpc, map;
};
inline constexpr BatchShape kShapes[] = {
#define BNTT_SHAPE_ROW(id, M, LOGR, TPC, MAP) {M, LOGR, TPC, MAP},
    BNTT_BATCH_SHAPES(BNTT_SHAPE_ROW)
#undef BNTT_SHAPE_ROW
};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

// the same table for device code: size and mapping of a shape id
__device__ __forceinline__ void shape_of(int id, int* m, int* map) {
  switch (id) {
#define BNTT_SHAPE_DEV(sid, M, LOGR, TPC, MAP) \
  case sid:                                    \
    *m = M;                                    \
    *map = MAP;                                \
    break;
    BNTT_BATCH_SHAPES(BNTT_SHAPE_DEV)
#undef BNTT_SHAPE_DEV
    default:
      *m = 3;
      *map = MAP_CONTIG;
  }
}

// control words: [0] queue head, [1] error word, [2 + 4*slot + p] pass counters
constexpr int kCtlHeader = 2;
constexpr int kMaxPasses = 4;
// bounded wait: default poll limit (polls x ~100 ns sleeps, a few seconds)
constexpr uint32_t kWaitPolls = 1u << 25;

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

struct BatchArgs {
  const WorkItem* items;
  uint32_t nitems;
  const DevJob* jobs;
  const uint32_t* order;   // job indices sorted by size (SMALL tiles)
  uint32_t* ctl;
  const uint32_t* pass_tiles;  // [slot * kMaxPasses + p] tile count of pass p
  uint32_t wait_polls;         // give up a dependency wait after this many polls
};

// The sub-transform a work item hands to thread `sub` of the tile: a whole
// small job, or one sub-transform of an HBM pass of a large job.  Returns
// false when the item is a later pass whose wait for its predecessor gave up
// (the error word is set; the tile is skipped).  INV: the passes of a large
// job run last to first (inverse transform), so a pass waits for the pass
// after it and the last pass is the one that reads the job's input.
template <bool INV = false>
__device__ __forceinline__ bool item_subref(const WorkItem& it, const BatchArgs& ba, int m, int sub,
                                            int* s_flag, SubRef* out) {
  if (it.kind == ITEM_SMALL) {
    SubRef sr;
    sr.valid = (uint32_t)sub < it.b;
    const DevJob& j = ba.jobs[ba.order[it.a + (sr.valid ? (uint32_t)sub : 0u)]];
    sr.x = j.x;
    sr.y = j.y;
    sr.tw = j.tw;
    sr.trow = 1;
    sr.lshift = 0;
    *out = sr;
    return true;
  }
  const DevJob& j = ba.jobs[it.a];
  const int n = (int)j.log2n;
  const int s0 = it.wait >> 8;  // first stage of this pass (engine_split on the host)
  if (it.wait & 1) {
    uint32_t* counters = ba.ctl + kCtlHeader + j.slot * kMaxPasses;
    const int pred = INV ? (int)it.pass + 1 : (int)it.pass - 1;
    if (threadIdx.x == 0) {
      const uint32_t want = ba.pass_tiles[j.slot * kMaxPasses + pred];
      uint32_t polls = 0;
      int ok = 1;
      while (ld_acquire(&counters[pred]) < want) {
        if (++polls > ba.wait_polls) {
          atomicOr(&ba.ctl[1], 1u);
          ok = 0;
          break;
        }
        __nanosleep(100);
      }
      *s_flag = ok;
    }
    __syncthreads();
    if (!*s_flag) return false;
  }
  SubGeom g;
  g.x = (it.wait & 2) ? j.x : j.y;
  g.y = j.y;
  g.tw = j.tw;
  g.n = (uint32_t)n;
  g.s0 = (uint32_t)s0;
  g.m = (uint32_t)m;
  g.l = (uint32_t)(n - s0 - m);
  g.nsub = 1ull << (n - m);
  *out = make_subref(g, (uint64_t)it.b + (uint64_t)sub);
  return true;
}

// A pass tile publishes its completion: every thread's stores, then one
// release increment of the job's pass counter.
__device__ __forceinline__ void item_publish(const WorkItem& it, const BatchArgs& ba) {
  if (it.kind != ITEM_PASS) return;
  __syncthreads();
  if (threadIdx.x == 0) {
    const DevJob& j = ba.jobs[it.a];
    __threadfence();
    atomicAdd(&ba.ctl[kCtlHeader + j.slot * kMaxPasses + it.pass], 1u);
  }
}

// The item functions are templates on the kernel's MINB as well: a
// non-inlined function is compiled once for all its callers, at the smallest
// register budget among them, so a kernel variant with more resident CTAs
// would otherwise make every variant's items spill.

// Sizes 2^1, 2^2: one thread per transform, fully unrolled.
template <int M, class Arith, int MINB, int LY>
__device__ __noinline__ void run_item_tiny(const WorkItem& it, const BatchArgs& ba, uint4* smem,
                                           const ModParams& mp, int layout_arg, int* s_flag) {
  const int layout = LY >= 0 ? LY : layout_arg;
  using T = NttTile<M, M, kBatchThreads, MAP_CONTIG, Arith>;
  const int sub = threadIdx.x;
  SubRef sr;
  if (!item_subref(it, ba, M, sub, s_flag, &sr)) return;
  T::template run<LD_NC>(sr, sub, 0, smem, mp, layout);
  item_publish(it, ba);
}

// Every other shape: the runtime-size engine.
template <class Arith, int MINB, int LY>
__device__ __noinline__ void run_item_engine(const WorkItem& it, const BatchArgs& ba, uint4* smem,
                                             const ModParams& mp, int layout_arg, int* s_flag) {
  const int layout = LY >= 0 ? LY : layout_arg;
  using E = NttEngine<kBatchLogR, Arith>;
  int m, map;
  shape_of(it.shape, &m, &map);
  int sub, lane;
  E::place(threadIdx.x, m, map, kBatchThreads, &sub, &lane);
  SubRef sr;
  if (!item_subref(it, ba, m, sub, s_flag, &sr)) return;
  // One load policy for every item: L2-coherent loads (a later pass reads what
  // other CTAs wrote in this launch).  A second instantiation for first
  // passes would double the engine's code, and instruction fetch is one of
  // the kernel's main stalls.
  E::template run<LD_CG>(m, map, kBatchThreads, sr, sub, lane, smem, mp, layout);
  item_publish(it, ba);
}

// Items of the shapes that carry most work run on the compile-time tile of the
// plan kernels (NttTile: strides and pass widths are constants) instead of the
// runtime-size engine: contiguous 2^7..2^10 (small jobs, the last passes of
// 2^16 and 2^20 jobs) and the interleaved 2^6 passes of 2^16 and 2^20 jobs.
// Measured on the uneven batch: 159 -> 168 G butterflies/s (2^10 items +6 %,
// 2^9 +7 %, 2^8 +7 %, 2^20 jobs +9 %).  Specialising the smaller and the other
// interleaved shapes as well made the kernel 5 % slower overall (a larger
// kernel), so they stay on the engine.
template <int M, int TPC, int MAP, class Arith, int MINB, int LY>
__device__ __noinline__ void run_item_tile(const WorkItem& it, const BatchArgs& ba, uint4* smem,
                                           const ModParams& mp, int layout_arg, int* s_flag) {
  const int layout = LY >= 0 ? LY : layout_arg;
  using T = NttTile<M, kBatchLogR, TPC, MAP, Arith>;
  static_assert(T::THREADS == kBatchThreads, "tile shape");
  const int sub = T::sub_of(threadIdx.x), lane = T::lane_of(threadIdx.x);
  SubRef sr;
  if (!item_subref(it, ba, M, sub, s_flag, &sr)) return;
  T::template run<LD_CG>(sr, sub, lane, smem, mp, layout);
  item_publish(it, ba);
}

// MINB: resident CTAs per SM requested from the compiler (register budget).
// LY: the element layout as a constant (LAYOUT_HILO or LAYOUT_U128), or -1
// for the `layout` argument.  A constant layout removes the runtime word
// select of every HBM load and store (measured +0.9 % on the uneven batch).
template <class Arith, int MINB, int LY = -1>
__global__ void __launch_bounds__(kBatchThreads, MINB) k_batch(BatchArgs ba, ModParams mp, int layout) {
  extern __shared__ uint4 smem[];
  __shared__ uint32_t s_item;
  __shared__ int s_flag;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(&ba.ctl[0], 1u);
    __syncthreads();
    const uint32_t i = s_item;
    if (i >= ba.nitems) break;
    const WorkItem it = ba.items[i];
    if (it.shape == 0) run_item_tiny<1, Arith, MINB, LY>(it, ba, smem, mp, layout, &s_flag);
    else if (it.shape == 1) run_item_tiny<2, Arith, MINB, LY>(it, ba, smem, mp, layout, &s_flag);
    else if (it.shape == 9) run_item_tile<10, 1, MAP_CONTIG, Arith, MINB, LY>(it, ba, smem, mp, layout, &s_flag);
    else if (it.shape == 8) run_item_tile<9, 2, MAP_CONTIG, Arith, MINB, LY>(it, ba, smem, mp, layout, &s_flag);
    else if (it.shape == 7) run_item_tile<8, 4, MAP_CONTIG, Arith, MINB, LY>(it, ba, smem, mp, layout, &s_flag);
    else if (it.shape == 6) run_item_tile<7, 8, MAP_CONTIG, Arith, MINB, LY>(it, ba, smem, mp, layout, &s_flag);
    else if (it.shape == 11) run_item_tile<6, 16, MAP_INTERLEAVED, Arith, MINB, LY>(it, ba, smem, mp, layout, &s_flag);
    else run_item_engine<Arith, MINB, LY>(it, ba, smem, mp, layout, &s_flag);
    __syncthreads();  // smem and s_item are reused by the next item
  }
}

}  // namespace bntt
