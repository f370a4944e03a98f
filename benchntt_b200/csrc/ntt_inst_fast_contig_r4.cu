// Instantiations: ArithFast, contiguous, 16 elements per thread (autotuner
// candidates).
#include "ntt_kernels.cuh"

namespace bntt {
void append_fast_contig_r4(std::vector<SubKernel>& v) {
  using A = ArithFast;
  v.push_back(BNTT_SUBK(5, 4, 128, MAP_CONTIG, A));
  v.push_back(BNTT_SUBK(6, 4, 64, MAP_CONTIG, A));
  v.push_back(BNTT_SUBK(7, 4, 32, MAP_CONTIG, A));
  v.push_back(BNTT_SUBK(8, 4, 16, MAP_CONTIG, A));
  v.push_back(BNTT_SUBK(9, 4, 8, MAP_CONTIG, A));
  v.push_back(BNTT_SUBK(10, 4, 4, MAP_CONTIG, A));
}
}  // namespace bntt
