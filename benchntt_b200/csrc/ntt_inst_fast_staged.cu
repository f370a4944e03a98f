// Instantiations: ArithFast, contiguous, 4 elements per thread, inputs staged
// into shared memory one tile ahead (k_ntt_sub_staged), with the table read
// through L1 or copied into shared memory first: autotuner candidates for
// 2^3..2^10 (their inputs' load latency and the table's placement are what
// the tuner measures here).
#include "ntt_kernels.cuh"

namespace bntt {
void append_fast_staged(std::vector<SubKernel>& v) {
  using A = ArithFast;
#define BNTT_STAGED_PAIR(M, TPC)                                         \
  v.push_back(BNTT_SUBK_STAGED(M, 2, TPC, A, 4, SRC_STAGED));           \
  v.push_back(BNTT_SUBK_STAGED(M, 2, TPC, A, 4, SRC_STAGED | TW_SHARED))
  BNTT_STAGED_PAIR(3, 128);
  BNTT_STAGED_PAIR(4, 64);
  BNTT_STAGED_PAIR(5, 32);
  BNTT_STAGED_PAIR(6, 16);
  BNTT_STAGED_PAIR(7, 8);
  BNTT_STAGED_PAIR(8, 4);
  BNTT_STAGED_PAIR(9, 2);
  BNTT_STAGED_PAIR(10, 1);
#undef BNTT_STAGED_PAIR
}
}  // namespace bntt
