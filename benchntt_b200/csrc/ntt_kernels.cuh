// ntt_kernels.cuh -- kernel template over NttTile and its registry entries.
#pragma once
#include "internal.h"
#include "ntt_core.cuh"

namespace bntt {

// Persistent launch over the tiles of a geometry: tile t holds sub-transforms
// [t*TPC, t*TPC + TPC); each CTA walks tiles blockIdx.x, +gridDim.x, ...
// MINB > 0 asks for at least MINB resident CTAs per SM (fewer registers per
// thread, more warps to hide the latency of the carry chains).
template <int M, int LOGR, int TPC, int MAP, class Arith, int MINB>
__global__ void __launch_bounds__(NttTile<M, LOGR, TPC, MAP, Arith>::THREADS, MINB)
    k_ntt_sub(SubGeom g, ModParams mp, int layout) {
  using T = NttTile<M, LOGR, TPC, MAP, Arith>;
  extern __shared__ uint4 smem[];
  const int tid = threadIdx.x;
  const int sub = T::sub_of(tid), lane = T::lane_of(tid);
  const uint64_t ntiles = (g.nsub + TPC - 1) / TPC;
  for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const SubRef sr = make_subref(g, tile * TPC + (uint64_t)sub);
    // the element layout as a constant in each branch: no word select per
    // HBM load and store
    if (layout == LAYOUT_HILO) T::template run<LD_NC>(sr, sub, lane, smem, mp, LAYOUT_HILO, MulB{g.b, g.y, g.bmask});
    else T::template run<LD_NC>(sr, sub, lane, smem, mp, LAYOUT_U128, MulB{g.b, g.y, g.bmask});
    if constexpr (T::NPASS > 1) T::sync();  // smem is reused by the next tile
  }
}

// The same over contiguous sub-transforms (L = 0: tile t is the 16-byte
// elements [t*TPC*2^M, (t+1)*TPC*2^M) of g.x), with every tile's input copied
// into shared memory by cp.async one tile ahead: while a CTA transforms tile
// t, the copy of its next tile is in flight, so the load latency that bounds
// small transforms (little work per element, a few tiles per CTA) overlaps
// the arithmetic.  The copy lands in the tile's exchange slots, the first pass
// gathers from there and every pass exchanges in place (a thread writes back
// only the slots it read).  Two tile buffers per CTA.  With TW_SHARED the
// CTA first copies the table's 2^M entries into shared memory (only for
// whole transforms, S0 = 0, where a tile reads entries below 2^M).
template <int M, int LOGR, int TPC, class Arith, int MINB, int SRC>
__global__ void __launch_bounds__(NttTile<M, LOGR, TPC, MAP_CONTIG, Arith>::THREADS, MINB)
    k_ntt_sub_staged(SubGeom g, ModParams mp, int layout) {
  using T = NttTile<M, LOGR, TPC, MAP_CONTIG, Arith>;
  constexpr int N = 1 << M;
  constexpr int TILE = TPC * N;  // elements per tile
  static_assert(T::THREADS * T::R == TILE, "tile shape");
  extern __shared__ uint4 smem[];
  const int tid = threadIdx.x;
  const int sub = T::sub_of(tid), lane = T::lane_of(tid);
  const uint64_t ntiles = (g.nsub + TPC - 1) / TPC;
  // tile t's valid elements, copied into `dst` in slot order
  auto stage = [&](uint64_t t, uint4* dst) {
    const uint64_t first = t * TPC;
    const uint64_t left = g.nsub - first;
    const uint32_t elems = (uint32_t)(left < (uint64_t)TPC ? left : (uint64_t)TPC) << M;
    const uint4* src = g.x + (first << M);
#pragma unroll
    for (int k = 0; k < T::R; ++k) {
      const uint32_t e = (uint32_t)tid + (uint32_t)k * T::THREADS;
      if (e < elems) cp_async16(&dst[T::slot((int)(e >> M), (int)(e & (N - 1)))], src + e);
    }
  };
  const uint4* tw = g.tw;
  if constexpr ((SRC & TW_SHARED) != 0) {
    uint4* const tws = smem + 2 * TILE;
    for (int e = tid; e < N; e += T::THREADS) tws[e] = __ldg(g.tw + e);
    tw = tws;  // made visible by the barrier before the first tile
  }
  uint64_t tile = blockIdx.x;
  if (tile < ntiles) stage(tile, smem);
  cp_async_commit();
  for (int b = 0; tile < ntiles; tile += gridDim.x, b ^= 1) {
    const uint64_t next = tile + gridDim.x;
    if (next < ntiles) stage(next, smem + (b ^ 1) * TILE);
    cp_async_commit();
    cp_async_wait<1>();  // every group but the newest: this tile's copies
    __syncthreads();
    SubRef sr = make_subref(g, tile * TPC + (uint64_t)sub);
    sr.tw = tw;
    if (layout == LAYOUT_HILO)
      T::template run<LD_NC, SRC | SRC_STAGED>(sr, sub, lane, smem + b * TILE, mp, LAYOUT_HILO,
                                               MulB{g.b, g.y, g.bmask});
    else
      T::template run<LD_NC, SRC | SRC_STAGED>(sr, sub, lane, smem + b * TILE, mp, LAYOUT_U128,
                                               MulB{g.b, g.y, g.bmask});
    __syncthreads();  // this buffer is refilled by the next iteration's copy
  }
  cp_async_wait<0>();
}

}  // namespace bntt

#define BNTT_SUBK_B(M, LOGR, TPC, MAP, ARITH, MINB)                                       \
  ::bntt::SubKernel {                                                                     \
    M, LOGR, TPC, MAP, ARITH::kFast ? 1 : 0, ::bntt::NttTile<M, LOGR, TPC, MAP, ARITH>::THREADS, \
        (size_t)::bntt::NttTile<M, LOGR, TPC, MAP, ARITH>::SMEM_SLOTS * 16u,              \
        (const void*)&::bntt::k_ntt_sub<M, LOGR, TPC, MAP, ARITH, MINB>, 0, MINB          \
  }
#define BNTT_SUBK(M, LOGR, TPC, MAP, ARITH) BNTT_SUBK_B(M, LOGR, TPC, MAP, ARITH, 1)
// staged contiguous kernels: two tile buffers (+ the table with TW_SHARED)
#define BNTT_SUBK_STAGED(M, LOGR, TPC, ARITH, MINB, SRC)                                       \
  ::bntt::SubKernel {                                                                         \
    M, LOGR, TPC, ::bntt::MAP_CONTIG, ARITH::kFast ? 1 : 0,                                   \
        ::bntt::NttTile<M, LOGR, TPC, ::bntt::MAP_CONTIG, ARITH>::THREADS,                    \
        (size_t)(2 * (TPC << M) + (((SRC) & ::bntt::TW_SHARED) ? (1 << M) : 0)) * 16u,        \
        (const void*)&::bntt::k_ntt_sub_staged<M, LOGR, TPC, ARITH, MINB, SRC>, 0, MINB, SRC  \
  }
