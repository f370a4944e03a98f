// batch_kfast.cu -- the persistent batch kernel with ArithFast, compiled for
// two, three or four resident CTAs per SM (register budget 128, 85 or 64 per
// thread; four is the default).
#include "batch_dev.cuh"

namespace bntt {
const void* batch_kernel_fast_minb(int minb) {
  return minb == 2   ? (const void*)&k_batch<ArithFast, 2>
         : minb == 3 ? (const void*)&k_batch<ArithFast, 3>
                     : (const void*)&k_batch<ArithFast, 4>;
}
}  // namespace bntt
