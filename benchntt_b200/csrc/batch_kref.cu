// batch_kref.cu -- the persistent batch kernel with ArithRef.
#include "batch_dev.cuh"

namespace bntt {
const void* batch_kernel_ref() { return (const void*)&k_batch<ArithRef, 2>; }
}  // namespace bntt
