// batch_kfast.cu -- the persistent batch kernel with ArithFast, compiled for
// two to five resident CTAs per SM (register budget 128, 85, 64 or 48 per
// thread; four is the default).
#include "batch_dev.cuh"

namespace bntt {
const void* batch_kernel_fast_minb(int minb) {
  return minb == 2   ? (const void*)&k_batch<ArithFast, 2>
         : minb == 3 ? (const void*)&k_batch<ArithFast, 3>
         : minb == 5 ? (const void*)&k_batch<ArithFast, 5>
                     : (const void*)&k_batch<ArithFast, 4>;
}
}  // namespace bntt
