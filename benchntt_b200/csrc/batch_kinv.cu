// batch_kinv.cu -- the persistent batch kernel for inverse transforms
// (bntt_batch_run_inverse_dev).  Same work queue and items as k_batch; each
// item runs the inverse network (the compile-time tile's run_inv for the
// shapes k_batch runs on tiles, else ntt_engine.cuh in inverse mode; stages
// last to first with the plans' inverse tables), the passes of a large job run
// from the last to the first, and whatever finishes a transform -- a small
// tile, or pass 0 of a large job -- multiplies by N^-1 as it stores, read
// from entry 0 of the job's inverse table (no stage uses that entry).
// Fast moduli only, like the plans' inverse.
#include "batch_dev.cuh"

namespace bntt {

namespace {

// 2^1, 2^2: one thread per transform.
template <int M, int LY>
__device__ __noinline__ void run_item_tiny_inv(const WorkItem& it, const BatchArgs& ba,
                                               const ModParams& mp, int layout_arg, int* s_flag) {
  const int layout = LY >= 0 ? LY : layout_arg;
  SubRef sr;
  if (!item_subref<true>(it, ba, M, threadIdx.x, s_flag, &sr)) return;
  if (!sr.valid) return;
  constexpr int N = 1 << M;
  U128 v[N];
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] = from_mem(__ldcg(sr.x + i), layout);
#pragma unroll
  for (int s = M - 1; s >= 0; --s) {
    const int half = N >> (s + 1);
#pragma unroll
    for (int i = 0; i < N; ++i) {
      if (i & half) continue;
      const uint4 tv = __ldg(sr.tw + (1 << s) + (i >> (M - s)));
      gs_butterfly<ArithFast>(v[i], v[i + half], U128{{tv.x, tv.y, tv.z, tv.w}}, mp);
    }
  }
  const uint4 f = __ldg(sr.tw);  // N^-1
  const U128 ninv = U128{{f.x, f.y, f.z, f.w}};
#pragma unroll
  for (int i = 0; i < N; ++i)  // the second half carries N^-1 through table entry 1
    sr.y[i] = to_mem(i < N / 2 ? ArithFast::mul(v[i], ninv, mp) : v[i], layout);
}

template <int LY>
__device__ __noinline__ void run_item_engine_inv(const WorkItem& it, const BatchArgs& ba, uint4* smem,
                                                 const ModParams& mp, int layout_arg, int* s_flag) {
  const int layout = LY >= 0 ? LY : layout_arg;
  using E = NttEngine<kBatchLogR, ArithFast>;
  int m, map;
  shape_of(it.shape, &m, &map);
  int sub, lane;
  E::place(threadIdx.x, m, map, kBatchThreads, &sub, &lane);
  SubRef sr;
  if (!item_subref<true>(it, ba, m, sub, s_flag, &sr)) return;
  // the store that finishes a transform applies N^-1
  const bool finishes = it.kind == ITEM_SMALL || it.pass == 0;
  Epilogue ep;
  ep.scale_at = it.kind == ITEM_SMALL ? sr.tw : ba.jobs[it.a].tw;  // N^-1
  E::template run<LD_CG, true, EPI_SCALE_AT>(m, map, kBatchThreads, sr, sub, lane, smem, mp, layout,
                                        finishes ? &ep : nullptr);
  item_publish(it, ba);
}

// The shapes that carry most work on the compile-time tile, as in k_batch:
// contiguous 2^7..2^10 and the interleaved 2^6 passes of large jobs.
template <int M, int TPC, int MAP, int LY>
__device__ __noinline__ void run_item_tile_inv(const WorkItem& it, const BatchArgs& ba, uint4* smem,
                                               const ModParams& mp, int layout_arg, int* s_flag) {
  const int layout = LY >= 0 ? LY : layout_arg;
  using T = NttTile<M, kBatchLogR, TPC, MAP, ArithFast>;
  static_assert(T::THREADS == kBatchThreads, "tile shape");
  const int sub = T::sub_of(threadIdx.x), lane = T::lane_of(threadIdx.x);
  SubRef sr;
  if (!item_subref<true>(it, ba, M, sub, s_flag, &sr)) return;
  const bool finishes = it.kind == ITEM_SMALL || it.pass == 0;
  const uint4* scale_at = !finishes ? nullptr : it.kind == ITEM_SMALL ? sr.tw : ba.jobs[it.a].tw;
  T::template run_inv<LD_CG>(sr, sub, lane, smem, mp, layout, scale_at);
  item_publish(it, ba);
}

// LY: the element layout as a constant, as in k_batch.
template <int MINB, int LY>
__global__ void __launch_bounds__(kBatchThreads, MINB)
    k_batch_inv(BatchArgs ba, ModParams mp, int layout) {
  extern __shared__ uint4 smem[];
  __shared__ uint32_t s_item;
  __shared__ int s_flag;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(&ba.ctl[0], 1u);
    __syncthreads();
    const uint32_t i = s_item;
    if (i >= ba.nitems) break;
    const WorkItem it = ba.items[i];
    if (it.shape == 0) run_item_tiny_inv<1, LY>(it, ba, mp, layout, &s_flag);
    else if (it.shape == 1) run_item_tiny_inv<2, LY>(it, ba, mp, layout, &s_flag);
    else if (it.shape == 9) run_item_tile_inv<10, 1, MAP_CONTIG, LY>(it, ba, smem, mp, layout, &s_flag);
    else if (it.shape == 8) run_item_tile_inv<9, 2, MAP_CONTIG, LY>(it, ba, smem, mp, layout, &s_flag);
    else if (it.shape == 7) run_item_tile_inv<8, 4, MAP_CONTIG, LY>(it, ba, smem, mp, layout, &s_flag);
    else if (it.shape == 6) run_item_tile_inv<7, 8, MAP_CONTIG, LY>(it, ba, smem, mp, layout, &s_flag);
    else if (it.shape == 11) run_item_tile_inv<6, 16, MAP_INTERLEAVED, LY>(it, ba, smem, mp, layout, &s_flag);
    else run_item_engine_inv<LY>(it, ba, smem, mp, layout, &s_flag);
    __syncthreads();  // smem and s_item are reused by the next item
  }
}

}  // namespace

const void* batch_kernel_inverse(int layout) {
  return layout == LAYOUT_HILO ? (const void*)&k_batch_inv<4, LAYOUT_HILO>
                               : (const void*)&k_batch_inv<4, LAYOUT_U128>;
}

}  // namespace bntt
