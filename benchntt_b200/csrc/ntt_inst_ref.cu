// Instantiations: ArithRef (word-for-word replica of the reference multiply),
// one shape per size and mapping.
#include "ntt_kernels.cuh"

namespace bntt {
void append_ref(std::vector<SubKernel>& v) {
  using A = ArithRef;
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
  v.push_back(BNTT_SUBK(5, 4, 8, MAP_INTERLEAVED, A));
  v.push_back(BNTT_SUBK(6, 4, 8, MAP_INTERLEAVED, A));
  v.push_back(BNTT_SUBK(7, 4, 8, MAP_INTERLEAVED, A));
  v.push_back(BNTT_SUBK(8, 4, 8, MAP_INTERLEAVED, A));
  v.push_back(BNTT_SUBK(9, 4, 4, MAP_INTERLEAVED, A));
  v.push_back(BNTT_SUBK(10, 4, 4, MAP_INTERLEAVED, A));
}
}  // namespace bntt
