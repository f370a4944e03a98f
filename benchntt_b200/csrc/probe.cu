// probe.cu -- measured peak of the 32-bit integer multiply-add pipe, the
// roofline of the NTT kernels (exact integer arithmetic: no tensor cores).
//
// Each thread runs 8 independent chains a = a * m + c (one mad.lo.u32 each),
// so the loop is issue-bound on IMAD; the grid fills every SM.
#include <algorithm>

#include "internal.h"

namespace bntt {

__global__ void __launch_bounds__(256) k_imad_probe(uint32_t* out, uint32_t iters, uint32_t m) {
  uint32_t a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = threadIdx.x * 2654435761u + k + blockIdx.x;
  for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
#pragma unroll
      for (int k = 0; k < 8; ++k) a[k] = a[k] * m + (uint32_t)(k + u);
    }
  }
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s ^= a[k];
  if (s == 0x9E3779B9u) out[0] = s;  // keeps the chains live
}

}  // namespace bntt

extern "C" int bntt_probe_imad_peak(bntt_ctx* c, double* ops_per_second) {
  using namespace bntt;
  BNTT_REQUIRE(c && ops_per_second, "NULL argument");
  if (int rc = ctx_use_device(c)) return rc;
  void* out = nullptr;
  if (int rc = ctx_alloc(c, &out, 16)) return rc;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const uint32_t iters = 4096;
  const unsigned grid = (unsigned)c->sms * 8;
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(e0, c->stream);
    k_imad_probe<<<grid, 256, 0, c->stream>>>(static_cast<uint32_t*>(out), iters, 0x5bd1e995u);
    cudaEventRecord(e1, c->stream);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) {
      ctx_free(c, out);
      return cuda_error(e, "imad probe");
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0) best = std::min(best, ms);  // first launch warms up
  }
  c->launches += 4;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ctx_free(c, out);
  const double ops = (double)grid * 256.0 * iters * 16.0 * 8.0;
  *ops_per_second = ops / (best * 1e-3);
  return BNTT_OK;
}

// Butterfly ceiling: the kernels' own butterfly (pseudo-Mersenne multiply,
// the reference's addmod / submod) on register-resident data, in radix-4
// groups of 4 butterflies (the persistent kernel's 4 elements per thread), at
// the persistent kernel's occupancy (4 CTAs of 256 threads per SM).  No
// memory traffic, no index arithmetic: the rate any NTT kernel of this
// arithmetic can approach.
namespace bntt {

constexpr int kProbeCtasPerSm = 4;
constexpr int kProbeButterfliesPerIter = 4;

__global__ void __launch_bounds__(256, kProbeCtasPerSm) k_butterfly_probe(uint4* out, uint32_t iters,
                                                                         ModParams mp) {
  U128 v[4], w[3];
  uint32_t h = (blockIdx.x * 256u + threadIdx.x) * 2654435761u + 1u;
#pragma unroll
  for (int e = 0; e < 7; ++e) {
    U128 t;
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      h ^= h << 13; h ^= h >> 17; h ^= h << 5;
      t.w[l] = h;
    }
    t.w[3] &= 0x07FFFFFFu;  // < 2^123 < q
    if (e < 4) v[e] = t;
    else w[e - 4] = t;
  }
  for (uint32_t it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 2; ++k) butterfly<ArithFast>(v[k], v[k + 2], w[0], mp);
    butterfly<ArithFast>(v[0], v[1], w[1], mp);
    butterfly<ArithFast>(v[2], v[3], w[2], mp);
  }
  uint32_t s = 0;
#pragma unroll
  for (int e = 0; e < 4; ++e) s ^= v[e].w[0] ^ v[e].w[1] ^ v[e].w[2] ^ v[e].w[3];
  if (s == 0x9E3779B9u) out[0] = make_uint4(s, 0u, 0u, 0u);  // keeps the results live
}

}  // namespace bntt

extern "C" int bntt_probe_butterfly_peak(bntt_ctx* c, double* butterflies_per_second) {
  using namespace bntt;
  BNTT_REQUIRE(c && butterflies_per_second, "NULL argument");
  if (int rc = ctx_use_device(c)) return rc;
  void* out = nullptr;
  if (int rc = ctx_alloc(c, &out, 16)) return rc;
  bool fast = false;
  const ModParams mp = make_params(bntt_modulus_ntt_reference(), &fast);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const uint32_t iters = 1536;
  const unsigned grid = (unsigned)c->sms * kProbeCtasPerSm;
  float best = 1e30f;
  for (int rep = 0; rep < 3; ++rep) {
    cudaEventRecord(e0, c->stream);
    k_butterfly_probe<<<grid, 256, 0, c->stream>>>(static_cast<uint4*>(out), iters, mp);
    cudaEventRecord(e1, c->stream);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) {
      ctx_free(c, out);
      return cuda_error(e, "butterfly probe");
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0) best = std::min(best, ms);  // first launch warms up
  }
  c->launches += 3;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ctx_free(c, out);
  const double bfly = (double)grid * 256.0 * iters * kProbeButterfliesPerIter;
  *butterflies_per_second = bfly / (best * 1e-3);
  return BNTT_OK;
}
