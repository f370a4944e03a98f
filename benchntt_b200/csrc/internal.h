// internal.h -- host-side structures shared by the libbntt translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstddef>
#include <cstdint>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/bntt.h"
#include "u128.cuh"

namespace bntt {

// ------------------------------------------------------------------ errors
int set_error(int status, const char* fmt, ...);
int cuda_error(cudaError_t e, const char* what);

#define BNTT_CK(call)                                         \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return ::bntt::cuda_error(e_, #call); \
  } while (0)

#define BNTT_REQUIRE(cond, ...)                                        \
  do {                                                                 \
    if (!(cond)) return ::bntt::set_error(BNTT_EINVAL, __VA_ARGS__);   \
  } while (0)

// ----------------------------------------------------------------- modulus
typedef unsigned __int128 u128;

inline u128 to_u128(bntt_u128 v) { return ((u128)v.hi << 64) | v.lo; }
inline bntt_u128 from_u128(u128 v) { return bntt_u128{(uint64_t)(v >> 64), (uint64_t)v}; }
inline U128 to_limbs(u128 v) {
  U128 r;
  for (int i = 0; i < 4; ++i) r.w[i] = (uint32_t)(v >> (32 * i));
  return r;
}

// floor(2^251 / q) for 2^123 < q < 2^128 (binary long division).
u128 barrett_mu(u128 q);
// True when the pseudo-Mersenne multiply is bit-identical to the reference.
bool modulus_fast(u128 q, u128 mu, uint32_t* k_out);
ModParams make_params(const bntt_modulus& m, bool* fast_out);
// Exact host arithmetic for 2^123 < q < 2^124, mu = floor(2^251 / q); a, b < q.
u128 host_mulmod(u128 a, u128 b, u128 q, u128 mu);
u128 host_powmod(u128 a, u128 e, u128 q, u128 mu);

// ----------------------------------------------------------------- kernels
struct SubGeom;  // ntt_core.cuh

// One compiled sub-transform kernel shape.
struct SubKernel {
  int m;        // log2 of the sub-transform
  int logr;     // log2 elements per thread
  int tpc;      // sub-transforms per CTA
  int map;      // MAP_CONTIG / MAP_INTERLEAVED
  int fast;     // ArithFast (1) or ArithRef (0)
  int threads;  // CTA size
  size_t smem;  // dynamic shared memory bytes
  const void* fn;
  int max_blocks_per_sm;  // filled lazily
  int minb;               // __launch_bounds__ minimum resident CTAs
  int src = 0;            // SRC_STAGED / TW_SHARED (k_ntt_sub_staged), else 0
};

const std::vector<SubKernel>& sub_kernels();
// Default shape for (m, map, fast); nullptr if none compiled.
const SubKernel* pick_sub_kernel(int m, int map, int fast, int logr_pref = 0, int tpc_pref = 0);
// Launch over a geometry; returns BNTT status.
int launch_sub(bntt_ctx* ctx, const SubKernel* k, const void* geom, const ModParams& mp,
               int layout, cudaStream_t stream, int grid_cap = 0);
int blocks_per_sm(const SubKernel* k);

// Autotuner choices (nullptr / -1 when not tuned).
const SubKernel* tuned_sub_kernel(int m, int map, int fast, int l);
int tuned_batch_small_shape(int m);

// Pass decomposition of a 2^n transform: sizes of HBM passes (each <= max_m).
// Plans use max_m = 10; the persistent kernel uses kBatchMaxPass.
std::vector<int> split_passes(int n, int max_m = 10);
// HBM passes of a 2^n transform (n > 10) on the tile engine (batch kernel,
// engine plans): fewest passes of <= 8 stages, then fewest engine passes.
std::vector<int> engine_split(int n);
// HBM passes of a 2^n transform (11 <= n <= 24) on 4-element tiles, as the
// persistent kernel splits its large jobs: strided passes of 5..7 stages
// (2^(10 - m) adjacent columns per tile), then a contiguous pass of up to 10;
// the fewest passes, then the fewest tile passes.  Empty outside that range.
std::vector<int> tile_split(int n);

int launch_blas(bntt_ctx* ctx, int op, void* c, const void* a, const void* b, U128 x, size_t len,
                const ModParams& mp, bool fast, int layout, cudaStream_t stream);
int launch_fill(bntt_ctx* ctx, void* buf, size_t count, uint64_t seed, uint64_t offset, u128 q,
                int layout, cudaStream_t stream);

}  // namespace bntt

// --------------------------------------------------------------- handles
struct bntt_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int arith = BNTT_ARITH_AUTO;
  size_t budget = 0;
  size_t in_use = 0;
  std::unordered_map<void*, size_t> allocs;
  int sms = 0;
  uint64_t launches = 0;
  // pinned staging and extra streams for host-pointer entry points
  void* pinned = nullptr;
  size_t pinned_bytes = 0;
  void* stage = nullptr;       // device staging of host-pointer calls
  size_t stage_bytes = 0;
  cudaStream_t copy_stream[2] = {nullptr, nullptr};
  cudaEvent_t ev[8] = {};
  // device address of the no-allocation scratch array, looked up by the
  // context's first bntt_batch_run_dev_noalloc call (a context created after
  // a device reset looks it up again)
  void* noalloc_base = nullptr;
  std::mutex mu;
};

struct bntt_plan {
  bntt_ctx* ctx = nullptr;
  unsigned log2n = 0;
  bntt_modulus mod{};
  bntt::ModParams mp{};
  bool fast = false;
  int layout = 0;
  void* tw = nullptr;
  bool own_tw = false;
  // inverse transform: table of inverse twiddles (limb order) and N^-1 mod q,
  // built on the first inverse call
  void* tw_inv = nullptr;
  bntt::U128 ninv{};
  // kernel per HBM pass
  std::vector<int> passes;
  std::vector<const bntt::SubKernel*> kernels;
};

namespace bntt {
int ctx_alloc(bntt_ctx* ctx, void** p, size_t bytes);
int ctx_free(bntt_ctx* ctx, void* p);
int ctx_use_device(bntt_ctx* ctx);
bool arith_fast(bntt_ctx* ctx, bool modulus_fast);
int plan_choose_kernels(bntt_plan* p);
// Builds the plan's inverse table and N^-1 on first use (fast moduli only).
int plan_ensure_inverse(bntt_plan* p);
int plan_create_common(bntt_ctx* c, bntt_plan** out, unsigned log2n, const bntt_modulus* m,
                       int layout);
// b != nullptr fuses y = y * b into the last pass (MulB in ntt_core.cuh).
int ntt_forward_on(bntt_plan* plan, void* y, const void* x, size_t batch, cudaStream_t s,
                   const void* b = nullptr, uint64_t bmask = 0);
// The same on the runtime-size tile engine (fast multiply, log2n >= 3);
// ntt_forward_on uses it above 2^10 points.
int engine_forward_on(bntt_plan* plan, void* y, const void* x, size_t batch, cudaStream_t s,
                      const void* b, uint64_t bmask);
}  // namespace bntt
