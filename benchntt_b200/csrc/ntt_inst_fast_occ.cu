// Instantiations: ArithFast, contiguous and interleaved shapes compiled for
// three resident CTAs per SM (at most 85 registers per thread): autotuner
// candidates that trade registers for warps.
#include "ntt_kernels.cuh"

namespace bntt {
void append_fast_occ(std::vector<SubKernel>& v) {
  using A = ArithFast;
  v.push_back(BNTT_SUBK_B(5, 3, 64, MAP_CONTIG, A, 3));
  v.push_back(BNTT_SUBK_B(6, 3, 32, MAP_CONTIG, A, 3));
  v.push_back(BNTT_SUBK_B(7, 3, 16, MAP_CONTIG, A, 3));
  v.push_back(BNTT_SUBK_B(8, 3, 8, MAP_CONTIG, A, 3));
  v.push_back(BNTT_SUBK_B(9, 3, 4, MAP_CONTIG, A, 3));
  v.push_back(BNTT_SUBK_B(10, 3, 2, MAP_CONTIG, A, 3));
  v.push_back(BNTT_SUBK_B(4, 4, 128, MAP_CONTIG, A, 3));
  v.push_back(BNTT_SUBK_B(9, 4, 4, MAP_INTERLEAVED, A, 3));
  // (10, 4, 4, interleaved) at three CTAs per SM holds 64 data registers in a
  // budget of 80 and spills 832 bytes per thread: not a candidate
}
}  // namespace bntt
