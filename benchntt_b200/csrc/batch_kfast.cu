// batch_kfast.cu -- the persistent batch kernel with ArithFast, compiled for
// two to five resident CTAs per SM (register budget 128, 85, 64 or 48 per
// thread; four is the default).
#include "batch_dev.cuh"

namespace bntt {
// The default four-CTA kernel is compiled once per element layout; the
// other variants read the layout at run time.
const void* batch_kernel_fast_minb(int minb, int layout) {
  return minb == 2   ? (const void*)&k_batch<ArithFast, 2>
         : minb == 3 ? (const void*)&k_batch<ArithFast, 3>
         : minb == 5 ? (const void*)&k_batch<ArithFast, 5>
         : layout == LAYOUT_HILO ? (const void*)&k_batch<ArithFast, 4, LAYOUT_HILO>
                                 : (const void*)&k_batch<ArithFast, 4, LAYOUT_U128>;
}
}  // namespace bntt
