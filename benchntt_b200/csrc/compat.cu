// compat.cu -- entry points with the reference's call shapes
// (include/bntt_compat.h, include/bntt_compat_simd.h) and its text data
// format (src/config.c).
//
// The compat calls run on a process-wide default context (device from the
// BNTT_DEVICE environment variable, else 0), created on first use.  Plans are
// cached per (size, modulus, layout) and keep a host copy of their twiddle
// table: a call with a table whose contents differ re-uploads it, so callers
// may reuse or rewrite their arrays freely, as with the reference functions.
#include <cerrno>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <tuple>

#include "internal.h"

using bntt::u128;

namespace {

struct CachedPlan {
  bntt_plan* plan = nullptr;
  std::vector<unsigned char> table;  // host copy of the uploaded table
};

std::mutex g_mu;
bntt_ctx* g_ctx = nullptr;
std::map<std::tuple<unsigned, u128, u128, int>, CachedPlan> g_plans;

int default_ctx(bntt_ctx** out) {
  if (!g_ctx) {
    const char* d = getenv("BNTT_DEVICE");
    if (int rc = bntt_ctx_create(&g_ctx, d ? atoi(d) : 0, nullptr)) return rc;
  }
  *out = g_ctx;
  return BNTT_OK;
}

int cached_plan(unsigned log2n, u128 q, u128 mu, const void* table, int layout, bntt_plan** out) {
  bntt_ctx* c = nullptr;
  if (int rc = default_ctx(&c)) return rc;
  const size_t bytes = (size_t)16 << log2n;
  CachedPlan& cp = g_plans[std::make_tuple(log2n, q, mu, layout)];
  const bool same = cp.plan && cp.table.size() == bytes && memcmp(cp.table.data(), table, bytes) == 0;
  if (!same) {
    if (cp.plan) bntt_plan_destroy(cp.plan);
    cp.plan = nullptr;
    bntt_modulus m{bntt::from_u128(q), bntt::from_u128(mu)};
    if (int rc = bntt_plan_create(c, &cp.plan, log2n, &m, table, layout)) return rc;
    cp.table.assign(static_cast<const unsigned char*>(table), static_cast<const unsigned char*>(table) + bytes);
  }
  *out = cp.plan;
  return BNTT_OK;
}

// state of the SIMD-shaped sequence ntt_pre -> ntt -> ntt_post
struct SimdState {
  const uint64_t* x = nullptr;
  bntt_plan* plan = nullptr;
  unsigned log2n = 0;
} g_simd;

}  // namespace

extern "C" {

// ntt(Y, X, modulus, mu, twiddles, as0, as1) of src/ntt_scalar.c:582 on
// native uint128_t arrays, N = 2^stages.  Returns when Y holds the result.
int bntt_compat_ntt_u128(unsigned __int128* Y, const unsigned __int128* X, unsigned __int128 modulus,
                         unsigned __int128 mu, const unsigned __int128* twiddles, unsigned stages) {
  BNTT_REQUIRE(Y && X && twiddles, "NULL argument");
  std::lock_guard<std::mutex> g(g_mu);
  bntt_plan* p = nullptr;
  if (int rc = cached_plan(stages, modulus, mu, twiddles, BNTT_LAYOUT_U128, &p)) return rc;
  return bntt_ntt_forward_host(p, Y, X, 1);
}

// Same transform on hi-first u64 pairs (the layout of the SIMD drivers and
// of the data files).
int bntt_compat_ntt_pairs(uint64_t* Y, const uint64_t* X, unsigned __int128 modulus,
                          unsigned __int128 mu, const uint64_t* twiddles, unsigned stages) {
  BNTT_REQUIRE(Y && X && twiddles, "NULL argument");
  std::lock_guard<std::mutex> g(g_mu);
  bntt_plan* p = nullptr;
  if (int rc = cached_plan(stages, modulus, mu, twiddles, BNTT_LAYOUT_HILO, &p)) return rc;
  return bntt_ntt_forward_host(p, Y, X, 1);
}

// vector_add / vector_sub / vector_mul / axpy of src/blas_scalar.c:578-608
// on native uint128_t arrays; op 0..3, len elements (the reference: 1024).
int bntt_compat_blas_u128(int op, unsigned __int128* c, const unsigned __int128* a,
                          const unsigned __int128* b, unsigned __int128 x, unsigned __int128 m,
                          unsigned __int128 mu, size_t len) {
  std::lock_guard<std::mutex> g(g_mu);
  bntt_ctx* ctx = nullptr;
  if (int rc = default_ctx(&ctx)) return rc;
  bntt_modulus mm{bntt::from_u128(m), bntt::from_u128(mu)};
  switch (op) {
    case 0: return bntt_vvadd_host(ctx, c, a, b, len, &mm, BNTT_LAYOUT_U128);
    case 1: return bntt_vvsub_host(ctx, c, a, b, len, &mm, BNTT_LAYOUT_U128);
    case 2: return bntt_vvmul_host(ctx, c, a, b, len, &mm, BNTT_LAYOUT_U128);
    case 3: return bntt_axpy_host(ctx, c, a, b, bntt::from_u128(x), len, &mm, BNTT_LAYOUT_U128);
    default: return bntt::set_error(BNTT_EINVAL, "unknown BLAS op %d", op);
  }
}

// Same on hi-first u64 pairs (the layout the SIMD BLAS drivers pass as
// __m256i / __m512i arrays, src/blas_avx512.c:401-476).
int bntt_compat_blas_pairs(int op, uint64_t* c, const uint64_t* a, const uint64_t* b,
                           unsigned __int128 x, unsigned __int128 m, unsigned __int128 mu, size_t len) {
  std::lock_guard<std::mutex> g(g_mu);
  bntt_ctx* ctx = nullptr;
  if (int rc = default_ctx(&ctx)) return rc;
  bntt_modulus mm{bntt::from_u128(m), bntt::from_u128(mu)};
  switch (op) {
    case 0: return bntt_vvadd_host(ctx, c, a, b, len, &mm, BNTT_LAYOUT_HILO);
    case 1: return bntt_vvsub_host(ctx, c, a, b, len, &mm, BNTT_LAYOUT_HILO);
    case 2: return bntt_vvmul_host(ctx, c, a, b, len, &mm, BNTT_LAYOUT_HILO);
    case 3: return bntt_axpy_host(ctx, c, a, b, bntt::from_u128(x), len, &mm, BNTT_LAYOUT_HILO);
    default: return bntt::set_error(BNTT_EINVAL, "unknown BLAS op %d", op);
  }
}

// The SIMD drivers' three-step shape (src/ntt_avx512.c:386-528): ntt_pre
// prepares (here: makes the table device-resident and remembers X), ntt
// computes and leaves the output where ntt_post reads it (`as`, 2N u64 in
// hi-first pair order), ntt_post stores it to Y.
int bntt_compat_simd_pre(const uint64_t* X, const uint64_t* twiddles, unsigned __int128 modulus,
                         unsigned __int128 mu, unsigned stages) {
  BNTT_REQUIRE(X && twiddles, "NULL argument");
  std::lock_guard<std::mutex> g(g_mu);
  bntt_plan* p = nullptr;
  if (int rc = cached_plan(stages, modulus, mu, twiddles, BNTT_LAYOUT_HILO, &p)) return rc;
  g_simd.x = X;
  g_simd.plan = p;
  g_simd.log2n = stages;
  return BNTT_OK;
}

int bntt_compat_simd_run(void* as_out) {
  BNTT_REQUIRE(as_out, "NULL argument");
  std::lock_guard<std::mutex> g(g_mu);
  BNTT_REQUIRE(g_simd.plan && g_simd.x, "ntt called before ntt_pre");
  return bntt_ntt_forward_host(g_simd.plan, as_out, g_simd.x, 1);
}

int bntt_compat_simd_post(uint64_t* Y, const void* as_in) {
  BNTT_REQUIRE(Y && as_in, "NULL argument");
  std::lock_guard<std::mutex> g(g_mu);
  BNTT_REQUIRE(g_simd.plan, "ntt_post called before ntt_pre");
  memcpy(Y, as_in, (size_t)16 << g_simd.log2n);
  return BNTT_OK;
}

// Text format of the reference data files (src/config.c:17-31): one decimal
// u64 per line, high word then low word per element.  Reads `n` elements
// into hi-first pairs.  Errors are returned, never exit().
int bntt_load_pairs_text(const char* path, uint64_t* pairs, size_t n) {
  BNTT_REQUIRE(path && (pairs || n == 0), "NULL argument");
  FILE* f = fopen(path, "r");
  if (!f) return bntt::set_error(BNTT_EINVAL, "cannot open %s: %s", path, strerror(errno));
  for (size_t i = 0; i < 2 * n; ++i) {
    if (fscanf(f, "%" SCNu64, &pairs[i]) != 1) {
      fclose(f);
      return bntt::set_error(BNTT_EINVAL, "%s: expected %zu values, read %zu", path, 2 * n, i);
    }
  }
  fclose(f);
  return BNTT_OK;
}

int bntt_save_pairs_text(const char* path, const uint64_t* pairs, size_t n) {
  BNTT_REQUIRE(path && (pairs || n == 0), "NULL argument");
  FILE* f = fopen(path, "w");
  if (!f) return bntt::set_error(BNTT_EINVAL, "cannot create %s: %s", path, strerror(errno));
  for (size_t i = 0; i < 2 * n; ++i) fprintf(f, "%" PRIu64 "\n", pairs[i]);
  if (fclose(f) != 0) return bntt::set_error(BNTT_EINVAL, "write error on %s", path);
  return BNTT_OK;
}

// load_twiddles / load_test_inputs of src/config.c:6-141: reads
// <dir>/<kind>_<N>.txt; for N > 1024 the 1024-entry file is repeated
// (element k = element k mod 1024), as the reference loader does.
int bntt_load_reference_data(const char* dir, const char* kind, uint64_t* pairs, size_t n) {
  BNTT_REQUIRE(dir && kind && pairs && n > 0, "NULL argument");
  char path[4096];
  const size_t file_n = n <= 1024 ? n : 1024;
  snprintf(path, sizeof(path), "%s/%s_%zu.txt", dir, kind, file_n);
  if (int rc = bntt_load_pairs_text(path, pairs, file_n)) return rc;
  for (size_t i = file_n; i < n; ++i) {
    pairs[2 * i] = pairs[2 * (i % 1024)];
    pairs[2 * i + 1] = pairs[2 * (i % 1024) + 1];
  }
  return BNTT_OK;
}

// Releases the default context and cached plans of the compat calls.
int bntt_compat_shutdown(void) {
  std::lock_guard<std::mutex> g(g_mu);
  for (auto& kv : g_plans)
    if (kv.second.plan) bntt_plan_destroy(kv.second.plan);
  g_plans.clear();
  g_simd = SimdState{};
  if (g_ctx) bntt_ctx_destroy(g_ctx);
  g_ctx = nullptr;
  return BNTT_OK;
}

}  // extern "C"
