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
    T::template run<LD_NC>(sr, sub, lane, smem, mp, layout, MulB{g.b, g.y, g.bmask});
    if constexpr (T::NPASS > 1) T::sync();  // smem is reused by the next tile
  }
}

}  // namespace bntt

#define BNTT_SUBK_B(M, LOGR, TPC, MAP, ARITH, MINB)                                       \
  ::bntt::SubKernel {                                                                     \
    M, LOGR, TPC, MAP, ARITH::kFast ? 1 : 0, ::bntt::NttTile<M, LOGR, TPC, MAP, ARITH>::THREADS, \
        (size_t)::bntt::NttTile<M, LOGR, TPC, MAP, ARITH>::SMEM_SLOTS * 16u,              \
        (const void*)&::bntt::k_ntt_sub<M, LOGR, TPC, MAP, ARITH, MINB>, 0, MINB          \
  }
#define BNTT_SUBK(M, LOGR, TPC, MAP, ARITH) BNTT_SUBK_B(M, LOGR, TPC, MAP, ARITH, 1)
