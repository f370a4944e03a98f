// Instantiations: ArithFast, interleaved sub-transforms (HBM passes whose
// elements are strided; TPC adjacent columns per CTA keep loads coalesced).
#include "ntt_kernels.cuh"

namespace bntt {
void append_fast_il(std::vector<SubKernel>& v) {
  using A = ArithFast;
  v.push_back(BNTT_SUBK(5, 4, 8, MAP_INTERLEAVED, A));
  v.push_back(BNTT_SUBK(6, 4, 8, MAP_INTERLEAVED, A));
  v.push_back(BNTT_SUBK(7, 4, 8, MAP_INTERLEAVED, A));
  v.push_back(BNTT_SUBK(8, 4, 8, MAP_INTERLEAVED, A));
  v.push_back(BNTT_SUBK(9, 4, 4, MAP_INTERLEAVED, A));
  v.push_back(BNTT_SUBK(10, 4, 4, MAP_INTERLEAVED, A));
  v.push_back(BNTT_SUBK(9, 4, 8, MAP_INTERLEAVED, A));
  v.push_back(BNTT_SUBK(10, 4, 8, MAP_INTERLEAVED, A));
}
}  // namespace bntt
