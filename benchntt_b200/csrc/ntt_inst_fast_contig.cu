// Instantiations: ArithFast, contiguous sub-transforms (small transforms and
// the last HBM pass of large ones).
#include "ntt_kernels.cuh"

namespace bntt {
void append_fast_contig(std::vector<SubKernel>& v) {
  using A = ArithFast;
  v.push_back(BNTT_SUBK(1, 1, 256, MAP_CONTIG, A));
  v.push_back(BNTT_SUBK(2, 2, 256, MAP_CONTIG, A));
  v.push_back(BNTT_SUBK(3, 3, 256, MAP_CONTIG, A));
  v.push_back(BNTT_SUBK(4, 4, 128, MAP_CONTIG, A));
  v.push_back(BNTT_SUBK(5, 3, 64, MAP_CONTIG, A));
  v.push_back(BNTT_SUBK(6, 3, 32, MAP_CONTIG, A));
  v.push_back(BNTT_SUBK(7, 3, 16, MAP_CONTIG, A));
  v.push_back(BNTT_SUBK(8, 3, 8, MAP_CONTIG, A));
  v.push_back(BNTT_SUBK(9, 3, 4, MAP_CONTIG, A));
  v.push_back(BNTT_SUBK(10, 3, 2, MAP_CONTIG, A));
}
}  // namespace bntt
