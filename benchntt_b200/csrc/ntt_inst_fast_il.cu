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
  // the persistent kernel's strided-pass tiles (4 elements per thread, 4
  // resident CTAs per SM, 2^(10 - M) adjacent columns): plans above 2^10
  // points run their HBM passes on these and the matching contiguous tiles
  v.push_back(BNTT_SUBK_B(5, 2, 32, MAP_INTERLEAVED, A, 4));
  v.push_back(BNTT_SUBK_B(6, 2, 16, MAP_INTERLEAVED, A, 4));
  v.push_back(BNTT_SUBK_B(7, 2, 8, MAP_INTERLEAVED, A, 4));
}
}  // namespace bntt
