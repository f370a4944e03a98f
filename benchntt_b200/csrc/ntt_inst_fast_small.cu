// Instantiations: ArithFast, contiguous shapes with 4 (or 8) elements per
// thread, so a transform spreads over more threads (an N = 16 transform on 4
// threads instead of 1, an N = 1024 transform on 256 instead of 128):
// autotuner candidates and the untuned defaults for 2^3..2^10.  At 2^9 and
// 2^10 they also cut the latency of a lone transform (one CTA: fewer
// dependent butterflies per thread).
#include "ntt_kernels.cuh"

namespace bntt {
void append_fast_small(std::vector<SubKernel>& v) {
  using A = ArithFast;
  v.push_back(BNTT_SUBK_B(3, 2, 128, MAP_CONTIG, A, 4));
  v.push_back(BNTT_SUBK_B(4, 2, 64, MAP_CONTIG, A, 4));
  v.push_back(BNTT_SUBK_B(4, 3, 128, MAP_CONTIG, A, 3));
  v.push_back(BNTT_SUBK_B(5, 2, 32, MAP_CONTIG, A, 4));
  v.push_back(BNTT_SUBK_B(6, 2, 16, MAP_CONTIG, A, 4));
  v.push_back(BNTT_SUBK_B(7, 2, 8, MAP_CONTIG, A, 4));
  v.push_back(BNTT_SUBK_B(8, 2, 4, MAP_CONTIG, A, 4));
  v.push_back(BNTT_SUBK_B(9, 2, 2, MAP_CONTIG, A, 4));
  v.push_back(BNTT_SUBK_B(10, 2, 1, MAP_CONTIG, A, 4));
}
}  // namespace bntt
