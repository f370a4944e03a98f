// Instantiations: ArithFast, contiguous, 4 elements per thread capped at 48
// registers (5 resident CTAs of 256 threads per SM), plain and staged, and 8
// elements per thread at 64 registers for 2^4: autotuner candidates for small
// transforms, where a batch of 65,536 needs more threads than fit on the GPU
// at once and more resident warps shorten the second round.
#include "ntt_kernels.cuh"

namespace bntt {
void append_fast_occ5(std::vector<SubKernel>& v) {
  using A = ArithFast;
#define BNTT_OCC5(M, TPC)                                                 \
  v.push_back(BNTT_SUBK_B(M, 2, TPC, MAP_CONTIG, A, 5));                 \
  v.push_back(BNTT_SUBK_STAGED(M, 2, TPC, A, 5, SRC_STAGED));            \
  v.push_back(BNTT_SUBK_STAGED(M, 2, TPC, A, 5, SRC_STAGED | TW_SHARED))
  BNTT_OCC5(3, 128);
  BNTT_OCC5(4, 64);
  BNTT_OCC5(5, 32);
  BNTT_OCC5(6, 16);
  BNTT_OCC5(7, 8);
  BNTT_OCC5(8, 4);
#undef BNTT_OCC5
  v.push_back(BNTT_SUBK_B(4, 3, 128, MAP_CONTIG, A, 4));
}
}  // namespace bntt
