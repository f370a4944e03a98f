// blas.cu -- element-wise mod-q vector operations of benchNTT
// (src/blas_scalar.c:578-608) as HBM streams.
//
// Each element is 16 bytes; a thread moves U elements per iteration with
// 128-bit loads marked evict-first (every byte is touched once), so the
// kernels are bound by HBM bandwidth: 48 bytes per element (two reads, one
// write).  No shared memory; the grid is up to 8 waves of resident blocks
// and walks the vector with a grid-stride loop.
#include <algorithm>
#include <atomic>

#include "internal.h"

namespace bntt {

enum : int { OP_ADD = 0, OP_SUB = 1, OP_MUL = 2, OP_AXPY = 3 };

template <int OP, class Arith, int U>
__global__ void __launch_bounds__(256) k_blas(uint4* c, const uint4* a, const uint4* b, size_t n,
                                              ModParams mp, U128 x, int layout) {
  const size_t step = (size_t)blockDim.x * U;
  for (size_t base = (size_t)blockIdx.x * step + threadIdx.x; base < n;
       base += (size_t)gridDim.x * step) {
    uint4 va[U], vb[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const size_t i = base + (size_t)u * blockDim.x;
      if (i < n) {
        va[u] = __ldcs(a + i);
        vb[u] = __ldcs(b + i);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const size_t i = base + (size_t)u * blockDim.x;
      if (i < n) {
        const U128 ea = from_mem(va[u], layout), eb = from_mem(vb[u], layout);
        U128 r;
        if constexpr (OP == OP_ADD) r = addmod_ref(ea, eb, mp.q);
        else if constexpr (OP == OP_SUB) r = submod_ref(ea, eb, mp.q);
        else if constexpr (OP == OP_MUL) r = Arith::mul(ea, eb, mp);
        else r = addmod_ref(ea, Arith::mul(x, eb, mp), mp.q);
        __stcs(c + i, to_mem(r, layout));
      }
    }
  }
}

constexpr int kBlasUnroll = 4;
constexpr int kBlasThreads = 256;

template <int OP, class Arith>
static const void* blas_fn() {
  return (const void*)&k_blas<OP, Arith, kBlasUnroll>;
}

int launch_blas(bntt_ctx* ctx, int op, void* c, const void* a, const void* b, U128 x, size_t len,
                const ModParams& mp, bool fast, int layout, cudaStream_t stream) {
  if (len == 0) return BNTT_OK;
  const void* fn = nullptr;
  switch (op) {
    case OP_ADD: fn = blas_fn<OP_ADD, ArithFast>(); break;  // add/sub take no multiply
    case OP_SUB: fn = blas_fn<OP_SUB, ArithFast>(); break;
    case OP_MUL: fn = fast ? blas_fn<OP_MUL, ArithFast>() : blas_fn<OP_MUL, ArithRef>(); break;
    case OP_AXPY: fn = fast ? blas_fn<OP_AXPY, ArithFast>() : blas_fn<OP_AXPY, ArithRef>(); break;
    default: return set_error(BNTT_EINVAL, "unknown BLAS op %d", op);
  }
  // resident blocks per SM of each kernel (the same on every B200); relaxed
  // atomics because several host threads may launch at once
  static std::atomic<int> bps_cache[8];
  const int slot = op * 2 + (fast ? 1 : 0);
  if (bps_cache[slot].load(std::memory_order_relaxed) == 0) {
    int b = 0;
    BNTT_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, kBlasThreads, 0));
    bps_cache[slot].store(std::max(1, b), std::memory_order_relaxed);
  }
  const size_t per_block = (size_t)kBlasThreads * kBlasUnroll;
  const size_t blocks_needed = (len + per_block - 1) / per_block;
  // up to 8 waves of resident blocks: at 2^24 elements (805 MB per op) a
  // sweep of unroll x waves on B200 put 8 waves at 103-104 % of the measured
  // copy bandwidth for vvadd, vvmul and axpy, against 91-99 % at 2 waves
  const size_t cap = (size_t)bps_cache[slot].load(std::memory_order_relaxed) * (size_t)ctx->sms * 8;
  const unsigned grid = (unsigned)std::min(blocks_needed, cap);
  uint4* cc = static_cast<uint4*>(c);
  const uint4* aa = static_cast<const uint4*>(a);
  const uint4* bb = static_cast<const uint4*>(b);
  size_t n = len;
  ModParams m = mp;
  U128 xx = x;
  int lay = layout;
  void* args[] = {&cc, &aa, &bb, &n, &m, &xx, &lay};
  BNTT_CK(cudaLaunchKernel(fn, dim3(grid), dim3(kBlasThreads), args, 0, stream));
  ctx->launches++;
  return BNTT_OK;
}

}  // namespace bntt
