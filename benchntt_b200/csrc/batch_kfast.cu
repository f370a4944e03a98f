// batch_kfast.cu -- the persistent batch kernel with ArithFast.
#include "batch_dev.cuh"

namespace bntt {
const void* batch_kernel_fast() { return (const void*)&k_batch<ArithFast>; }
}  // namespace bntt
