// roots.cu -- NTT-friendly prime mode: prime search, roots of unity and
// root-power twiddle tables for the reference network.
//
// The reference's NTT modulus 2^124 - 719 has q - 1 = 2^4 * odd, so it has no
// 2-power root of unity of order above 16; the reference fills its tables
// with data-file values (load_twiddles, src/config.c:6-60) and ntt()
// (src/ntt_scalar.c:582)
// treats them as arbitrary constants.  ntt() takes the modulus, mu and the
// table as run-time arguments, so the same network computes a true transform
// when q = 2^124 - k has 2^t | q - 1 and the table holds root powers:
//
//   T[k] = psi^brv_n(k)   (k = 1 .. N-1; brv_n reverses n = log2 N bits)
//
// with psi a primitive 2N-th root of unity.  Stage s of the network uses
// T[2^s + b] for block b (the in-place form of src/ntt_scalar.c:584-626), and
// the output is the negacyclic transform in bit-reversed order:
//
//   Y[i] = sum_j X[j] * psi^((2*brv_n(i) + 1) * j)   (mod q)
//
// i.e. the evaluations of X(x) at the roots of x^N + 1.
//
// Host arithmetic here is exact for every q in (2^123, 2^124): a 256-bit
// product and a Barrett quotient that is at most one short, then a
// correction.  Device tables use the pseudo-Mersenne multiply, which is exact
// for the moduli this mode produces (k < 2^28).
#include <algorithm>
#include <vector>

#include "internal.h"

namespace bntt {

namespace {
struct U256 {
  u128 hi, lo;
};

U256 mul_full(u128 a, u128 b) {
  const uint64_t a0 = (uint64_t)a, a1 = (uint64_t)(a >> 64);
  const uint64_t b0 = (uint64_t)b, b1 = (uint64_t)(b >> 64);
  const u128 p00 = (u128)a0 * b0, p01 = (u128)a0 * b1;
  const u128 p10 = (u128)a1 * b0, p11 = (u128)a1 * b1;
  const u128 mid = (p00 >> 64) + (uint64_t)p01 + (uint64_t)p10;  // < 3 * 2^64
  U256 r;
  r.lo = (mid << 64) | (uint64_t)p00;
  r.hi = p11 + (p01 >> 64) + (p10 >> 64) + (mid >> 64);
  return r;
}
}  // namespace

// a * b mod q for a, b < q, 2^123 < q < 2^124, mu = floor(2^251 / q).
// P < 2^248; qq = floor(floor(P / 2^122) * mu / 2^129) is floor(P/q) or one
// less (the truncations lose < 2^122/q + P/2^251 < 5/8), and P - qq*q < 2q
// fits 128 bits, so it is formed mod 2^128.
u128 host_mulmod(u128 a, u128 b, u128 q, u128 mu) {
  const U256 P = mul_full(a, b);
  const u128 ql = (P.hi << 6) | (P.lo >> 122);
  const U256 t = mul_full(ql, mu);
  const u128 qq = t.hi >> 1;
  u128 r = P.lo - qq * q;
  while (r >= q) r -= q;
  return r;
}

u128 host_powmod(u128 a, u128 e, u128 q, u128 mu) {
  u128 r = 1, b = a % q;
  while (e) {
    if (e & 1) r = host_mulmod(r, b, q, mu);
    b = host_mulmod(b, b, q, mu);
    e >>= 1;
  }
  return r;
}

namespace {

// Strong probable-prime test to the first 24 prime bases.  A composite passes
// one base with probability at most 1/4, so all 24 with at most 2^-48 in the
// worst case (far less for the numbers searched here).
bool miller_rabin(u128 n, u128 mu) {
  static const uint32_t kBases[24] = {2,  3,  5,  7,  11, 13, 17, 19, 23, 29, 31, 37,
                                      41, 43, 47, 53, 59, 61, 67, 71, 73, 79, 83, 89};
  for (uint32_t p : kBases)
    if (n % p == 0) return n == p;
  u128 d = n - 1;
  int s = 0;
  while ((d & 1) == 0) {
    d >>= 1;
    ++s;
  }
  for (uint32_t a : kBases) {
    u128 x = host_powmod(a, d, n, mu);
    if (x == 1 || x == n - 1) continue;
    bool witness = true;
    for (int i = 1; i < s && witness; ++i) {
      x = host_mulmod(x, x, n, mu);
      if (x == n - 1) witness = false;
    }
    if (witness) return false;
  }
  return true;
}

uint32_t bit_reverse(uint32_t k, unsigned n) {
  uint32_t r = 0;
  for (unsigned i = 0; i < n; ++i) r |= ((k >> i) & 1u) << (n - 1 - i);
  return r;
}

__device__ __forceinline__ uint32_t bit_reverse_dev(uint32_t k, unsigned n) {
  return __brev(k) >> (32 - n);  // n >= 1
}

bool modulus_in_range(u128 q, u128 mu) {
  const u128 lo = (u128)1 << 123, hi = (u128)1 << 124;
  return q > lo && q < hi && mu == barrett_mu(q);
}

// psi^(2^i) for i < n: the factors a device thread multiplies for exponent e.
struct PowTable {
  uint4 p[24];
};

__global__ void k_negacyclic_table(uint4* __restrict__ t, unsigned n, PowTable pw, ModParams mp) {
  const uint32_t count = 1u << n;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
    const uint32_t e = bit_reverse_dev(k, n);
    U128 acc = U128{{1u, 0u, 0u, 0u}};
    for (unsigned i = 0; i < n; ++i) {
      if ((e >> i) & 1u) {
        const uint4 f = pw.p[i];
        acc = ArithFast::mul(acc, U128{{f.x, f.y, f.z, f.w}}, mp);
      }
    }
    t[k] = make_uint4(acc.w[0], acc.w[1], acc.w[2], acc.w[3]);
  }
}

}  // namespace
}  // namespace bntt

using namespace bntt;

extern "C" {

int bntt_ntt_prime(unsigned log2_order, bntt_modulus* m) {
  BNTT_REQUIRE(m, "NULL argument");
  BNTT_REQUIRE(log2_order >= 1 && log2_order <= 30, "log2_order %u outside [1, 30]", log2_order);
  const u128 top = (u128)1 << 124;
  for (uint64_t c = 1;; ++c) {
    const u128 k = ((u128)c << log2_order) - 1;
    if (k >= ((u128)1 << 28)) break;
    const u128 q = top - k;
    const u128 mu = barrett_mu(q);
    if (miller_rabin(q, mu)) {
      m->q = from_u128(q);
      m->mu = from_u128(mu);
      return BNTT_OK;
    }
  }
  return set_error(BNTT_EINVAL, "no prime 2^124 - (c*2^%u - 1) with c*2^%u - 1 < 2^28", log2_order,
                   log2_order);
}

int bntt_powmod(const bntt_modulus* m, bntt_u128 a, bntt_u128 e, bntt_u128* out) {
  BNTT_REQUIRE(m && out, "NULL argument");
  const u128 q = to_u128(m->q), mu = to_u128(m->mu);
  BNTT_REQUIRE(modulus_in_range(q, mu), "modulus must satisfy 2^123 < q < 2^124, mu = floor(2^251/q)");
  *out = from_u128(host_powmod(to_u128(a), to_u128(e), q, mu));
  return BNTT_OK;
}

int bntt_root_of_unity(const bntt_modulus* m, unsigned log2_order, bntt_u128* root) {
  BNTT_REQUIRE(m && root, "NULL argument");
  const u128 q = to_u128(m->q), mu = to_u128(m->mu);
  BNTT_REQUIRE(modulus_in_range(q, mu), "modulus must satisfy 2^123 < q < 2^124, mu = floor(2^251/q)");
  BNTT_REQUIRE(log2_order >= 1 && log2_order <= 120, "log2_order %u outside [1, 120]", log2_order);
  BNTT_REQUIRE((((q - 1) >> log2_order) << log2_order) == q - 1, "2^%u does not divide q - 1",
               log2_order);
  const u128 cofactor = (q - 1) >> log2_order;
  // w = g^((q-1)/2^t) has order dividing 2^t; it is exactly 2^t when
  // w^(2^(t-1)) = -1.  For prime q half of all g give such a w.
  for (uint32_t g = 2; g < 4096; ++g) {
    const u128 w = host_powmod(g, cofactor, q, mu);
    const u128 h = host_powmod(w, (u128)1 << (log2_order - 1), q, mu);
    if (h == q - 1) {
      *root = from_u128(w);
      return BNTT_OK;
    }
  }
  return set_error(BNTT_EINVAL, "no root of unity of order 2^%u found (is q prime?)", log2_order);
}

int bntt_twiddles_negacyclic(const bntt_modulus* m, unsigned log2n, bntt_u128 psi, void* table,
                             int layout) {
  BNTT_REQUIRE(m && table, "NULL argument");
  BNTT_REQUIRE(log2n >= 1 && log2n <= 24, "log2n %u outside [1, 24]", log2n);
  BNTT_REQUIRE(layout == BNTT_LAYOUT_HILO || layout == BNTT_LAYOUT_U128, "bad layout %d", layout);
  const u128 q = to_u128(m->q), mu = to_u128(m->mu), p = to_u128(psi);
  BNTT_REQUIRE(modulus_in_range(q, mu), "modulus must satisfy 2^123 < q < 2^124, mu = floor(2^251/q)");
  BNTT_REQUIRE(p < q && host_powmod(p, (u128)1 << log2n, q, mu) == q - 1,
               "psi is not a primitive 2^%u-th root of unity (psi^N != -1)", log2n + 1);
  const uint32_t n = 1u << log2n;
  std::vector<u128> pw(n);
  pw[0] = 1;
  for (uint32_t j = 1; j < n; ++j) pw[j] = host_mulmod(pw[j - 1], p, q, mu);
  uint64_t* out = static_cast<uint64_t*>(table);
  for (uint32_t k = 0; k < n; ++k) {
    const u128 v = pw[bit_reverse(k, log2n)];
    const uint64_t hi = (uint64_t)(v >> 64), lo = (uint64_t)v;
    out[2 * k] = layout == BNTT_LAYOUT_HILO ? hi : lo;
    out[2 * k + 1] = layout == BNTT_LAYOUT_HILO ? lo : hi;
  }
  return BNTT_OK;
}

int bntt_plan_create_negacyclic(bntt_ctx* c, bntt_plan** out, unsigned log2n, const bntt_modulus* m,
                                bntt_u128 psi, int layout) {
  BNTT_REQUIRE(m, "NULL argument");
  const u128 q = to_u128(m->q), mu = to_u128(m->mu), p = to_u128(psi);
  BNTT_REQUIRE(modulus_fast(q, mu, nullptr),
               "root-power tables are built on the device for q = 2^124 - k (k < 2^28), "
               "mu = floor(2^251/q); build others with bntt_twiddles_negacyclic");
  BNTT_REQUIRE(log2n >= 1 && log2n <= 24, "log2n %u outside [1, 24]", log2n);
  BNTT_REQUIRE(p < q && host_powmod(p, (u128)1 << log2n, q, mu) == q - 1,
               "psi is not a primitive 2^%u-th root of unity (psi^N != -1)", log2n + 1);
  int rc = plan_create_common(c, out, log2n, m, layout);
  if (rc) return rc;
  bntt_plan* pl = *out;
  const size_t n = (size_t)1 << log2n;
  if ((rc = ctx_alloc(c, &pl->tw, n * 16)) != 0) {
    delete pl;
    *out = nullptr;
    return rc;
  }
  pl->own_tw = true;
  PowTable pw{};
  u128 f = p;
  for (unsigned i = 0; i < log2n; ++i) {
    const U128 l = to_limbs(f);
    pw.p[i] = make_uint4(l.w[0], l.w[1], l.w[2], l.w[3]);
    f = host_mulmod(f, f, q, mu);
  }
  const unsigned grid = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)c->sms * 8);
  k_negacyclic_table<<<grid, 256, 0, c->stream>>>(static_cast<uint4*>(pl->tw), log2n, pw, pl->mp);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) rc = cuda_error(e, "k_negacyclic_table");
  else {
    c->launches++;
    rc = plan_choose_kernels(pl);
  }
  if (rc) {
    ctx_free(c, pl->tw);
    delete pl;
    *out = nullptr;
  }
  return rc;
}

}  // extern "C"
