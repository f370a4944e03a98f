// u128.cuh -- 128-bit modular arithmetic on sm_100a for the benchNTT hot path.
//
// A residue is four little-endian 32-bit limbs (w[0] least significant).
// In HBM an element is 16 bytes in one of two layouts:
//   HILO : the reference's u64 pair, high word first (src/config.c:29-30);
//          as u32 words: [hi.lo32, hi.hi32, lo.lo32, lo.hi32]
//   U128 : a native little-endian unsigned __int128 (the scalar API's
//          uint128_t arrays, src/ntt_scalar.c:582)
//
// Two multiply policies produce results bit-identical to the reference
// mulmod128 (src/ntt_scalar.c:173-199):
//   ArithFast -- q = 2^124 - k with k < 2^28 and mu = floor(2^251 / q) (both
//     reference primes and the NTT-friendly primes of roots.cu).  For such (q, mu) and operands below 2^124 the
//     reference's Barrett quotient is within one of the true quotient, so its
//     single conditional subtraction always lands in [0, q): the reference
//     returns exactly a*b mod q.  ArithFast computes that value with a
//     pseudo-Mersenne fold (2^128 == 16k, 2^124 == k mod q): four 64-bit
//     products for a*b, 4 limb products for the first fold, 1 for the second,
//     one conditional subtraction.  Its operands must be below 2^124.
//   ArithRef  -- every other (q, mu): a replica of the reference's 64-bit word
//     data flow, including the points where it drops carries, so it matches
//     for arbitrary 128-bit inputs.
// add and sub are the reference's exact semantics in both policies,
// including addmod's two corner behaviours (see addmod_ref).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace bntt {

struct U128 {
  uint32_t w[4];
};

// Parameters of one modulus as the kernels see them.
struct ModParams {
  U128 q;        // modulus
  U128 mu;       // Barrett constant of the reference (used by ArithRef)
  uint32_t k;    // q = 2^124 - k (used by ArithFast)
  uint32_t pad[3];
};

enum Layout : int { LAYOUT_HILO = 0, LAYOUT_U128 = 1 };

__device__ __forceinline__ U128 from_mem(uint4 v, int layout) {
  U128 r;
  if (layout == LAYOUT_HILO) {
    r.w[0] = v.z; r.w[1] = v.w; r.w[2] = v.x; r.w[3] = v.y;
  } else {
    r.w[0] = v.x; r.w[1] = v.y; r.w[2] = v.z; r.w[3] = v.w;
  }
  return r;
}

__device__ __forceinline__ uint4 to_mem(const U128& a, int layout) {
  if (layout == LAYOUT_HILO) return make_uint4(a.w[2], a.w[3], a.w[0], a.w[1]);
  return make_uint4(a.w[0], a.w[1], a.w[2], a.w[3]);
}

// ---------------------------------------------------------------- add / sub

// Reference addmod128 (src/ntt_scalar.c:49-79).  s = a + b mod 2^128 and
// e = q - s mod 2^128; the borrow out of e is "s > q" (a strict test, so
// s == q is returned as q).  The reference assembles s - q from e's 64-bit
// words as (~e.hi, -e.lo): equal to s - q except when lo64(s) == lo64(q),
// where its high word comes out one lower.  This routine reproduces exactly
// that.
__device__ __forceinline__ U128 addmod_ref(const U128& a, const U128& b, const U128& q) {
  uint32_t s0, s1, s2, s3, e0, e1, e2, e3, gt;
  asm("add.cc.u32  %0, %9, %13;\n\t"
      "addc.cc.u32 %1, %10, %14;\n\t"
      "addc.cc.u32 %2, %11, %15;\n\t"
      "addc.u32    %3, %12, %16;\n\t"
      "sub.cc.u32  %4, %17, %0;\n\t"
      "subc.cc.u32 %5, %18, %1;\n\t"
      "subc.cc.u32 %6, %19, %2;\n\t"
      "subc.cc.u32 %7, %20, %3;\n\t"
      "subc.u32    %8, 0, 0;\n\t"
      : "=&r"(s0), "=&r"(s1), "=&r"(s2), "=&r"(s3), "=&r"(e0), "=&r"(e1), "=&r"(e2),
        "=&r"(e3), "=r"(gt)
      : "r"(a.w[0]), "r"(a.w[1]), "r"(a.w[2]), "r"(a.w[3]), "r"(b.w[0]), "r"(b.w[1]),
        "r"(b.w[2]), "r"(b.w[3]), "r"(q.w[0]), "r"(q.w[1]), "r"(q.w[2]), "r"(q.w[3]));
  uint32_t n0, n1;
  asm("sub.cc.u32 %0, 0, %2;\n\t"
      "subc.u32   %1, 0, %3;\n\t"
      : "=r"(n0), "=r"(n1)
      : "r"(e0), "r"(e1));
  U128 r;
  const bool sub = gt != 0u;
  r.w[0] = sub ? n0 : s0;
  r.w[1] = sub ? n1 : s1;
  r.w[2] = sub ? ~e2 : s2;
  r.w[3] = sub ? ~e3 : s3;
  return r;
}

// Reference submod128 (src/ntt_scalar.c:81-104): d = a - b, plus q on borrow.
__device__ __forceinline__ U128 submod_ref(const U128& a, const U128& b, const U128& q) {
  uint32_t d0, d1, d2, d3, bw;
  asm("sub.cc.u32  %0, %5, %9;\n\t"
      "subc.cc.u32 %1, %6, %10;\n\t"
      "subc.cc.u32 %2, %7, %11;\n\t"
      "subc.cc.u32 %3, %8, %12;\n\t"
      "subc.u32    %4, 0, 0;\n\t"
      : "=&r"(d0), "=&r"(d1), "=&r"(d2), "=&r"(d3), "=r"(bw)
      : "r"(a.w[0]), "r"(a.w[1]), "r"(a.w[2]), "r"(a.w[3]), "r"(b.w[0]), "r"(b.w[1]),
        "r"(b.w[2]), "r"(b.w[3]));
  // add (q & borrow-mask): one chain, no select
  uint32_t m0 = q.w[0] & bw, m1 = q.w[1] & bw, m2 = q.w[2] & bw, m3 = q.w[3] & bw;
  U128 r;
  asm("add.cc.u32  %0, %4, %8;\n\t"
      "addc.cc.u32 %1, %5, %9;\n\t"
      "addc.cc.u32 %2, %6, %10;\n\t"
      "addc.u32    %3, %7, %11;\n\t"
      : "=r"(r.w[0]), "=r"(r.w[1]), "=r"(r.w[2]), "=r"(r.w[3])
      : "r"(d0), "r"(d1), "r"(d2), "r"(d3), "r"(m0), "r"(m1), "r"(m2), "r"(m3));
  return r;
}

// The same two operations for q = 2^124 - k with k < 2^31, whose limbs are
// (2^32 - k, 0xFFFFFFFF, 0xFFFFFFFF, 0x0FFFFFFF): three of them become
// immediates, which frees registers in the butterfly loops.
__device__ __forceinline__ U128 addmod_pm(const U128& a, const U128& b, uint32_t q0) {
  uint32_t s0, s1, s2, s3, e0, e1, e2, e3, gt;
  asm("add.cc.u32  %0, %9, %13;\n\t"
      "addc.cc.u32 %1, %10, %14;\n\t"
      "addc.cc.u32 %2, %11, %15;\n\t"
      "addc.u32    %3, %12, %16;\n\t"
      "sub.cc.u32  %4, %17, %0;\n\t"
      "subc.cc.u32 %5, 0xFFFFFFFF, %1;\n\t"
      "subc.cc.u32 %6, 0xFFFFFFFF, %2;\n\t"
      "subc.cc.u32 %7, 0x0FFFFFFF, %3;\n\t"
      "subc.u32    %8, 0, 0;\n\t"
      : "=&r"(s0), "=&r"(s1), "=&r"(s2), "=&r"(s3), "=&r"(e0), "=&r"(e1), "=&r"(e2),
        "=&r"(e3), "=r"(gt)
      : "r"(a.w[0]), "r"(a.w[1]), "r"(a.w[2]), "r"(a.w[3]), "r"(b.w[0]), "r"(b.w[1]),
        "r"(b.w[2]), "r"(b.w[3]), "r"(q0));
  uint32_t n0, n1;
  asm("sub.cc.u32 %0, 0, %2;\n\t"
      "subc.u32   %1, 0, %3;\n\t"
      : "=r"(n0), "=r"(n1)
      : "r"(e0), "r"(e1));
  U128 r;
  const bool sub = gt != 0u;
  r.w[0] = sub ? n0 : s0;
  r.w[1] = sub ? n1 : s1;
  r.w[2] = sub ? ~e2 : s2;
  r.w[3] = sub ? ~e3 : s3;
  return r;
}

__device__ __forceinline__ U128 submod_pm(const U128& a, const U128& b, uint32_t q0) {
  uint32_t d0, d1, d2, d3, bw;
  asm("sub.cc.u32  %0, %5, %9;\n\t"
      "subc.cc.u32 %1, %6, %10;\n\t"
      "subc.cc.u32 %2, %7, %11;\n\t"
      "subc.cc.u32 %3, %8, %12;\n\t"
      "subc.u32    %4, 0, 0;\n\t"
      : "=&r"(d0), "=&r"(d1), "=&r"(d2), "=&r"(d3), "=r"(bw)
      : "r"(a.w[0]), "r"(a.w[1]), "r"(a.w[2]), "r"(a.w[3]), "r"(b.w[0]), "r"(b.w[1]),
        "r"(b.w[2]), "r"(b.w[3]));
  U128 r;
  asm("add.cc.u32  %0, %4, %8;\n\t"
      "addc.cc.u32 %1, %5, %9;\n\t"
      "addc.cc.u32 %2, %6, %9;\n\t"
      "addc.u32    %3, %7, %10;\n\t"
      : "=r"(r.w[0]), "=r"(r.w[1]), "=r"(r.w[2]), "=r"(r.w[3])
      : "r"(d0), "r"(d1), "r"(d2), "r"(d3), "r"(q0 & bw), "r"(bw), "r"(bw & 0x0FFFFFFFu));
  return r;
}

// ------------------------------------------------------------------ ArithFast

// p = a * b for a, b < 2^124 (every residue of an ArithFast modulus), as
// four 64 x 64 -> 128-bit products of the 64-bit halves: the middle sum
// a0*b1 + a1*b0 stays below 2^125 because the high halves are below 2^60.
// Written on 64-bit halves so that the compiler picks the instructions for
// the 32-bit partial products and their carries: the register-only butterfly
// probe runs at 233 G butterflies/s this way, against 209 G/s with a
// hand-written PTX carry chain per row of 32-bit limbs (mad.lo.cc/madc.hi.cc)
// and 212 G/s when the middle sum's carry is kept for full 128-bit operands.
__device__ __forceinline__ void mul_128x128(const U128& a, const U128& b, uint32_t p[8]) {
  typedef unsigned __int128 u128x;
  typedef unsigned long long u64x;
  const u64x a0 = ((u64x)a.w[1] << 32) | a.w[0], a1 = ((u64x)a.w[3] << 32) | a.w[2];
  const u64x b0 = ((u64x)b.w[1] << 32) | b.w[0], b1 = ((u64x)b.w[3] << 32) | b.w[2];
  const u128x p00 = (u128x)a0 * b0, p11 = (u128x)a1 * b1;
  const u128x mid = (u128x)a0 * b1 + (u128x)a1 * b0;
  const u128x lo = p00 + (mid << 64);
  const u128x hi = p11 + (mid >> 64) + (lo < p00 ? 1u : 0u);
  p[0] = (uint32_t)lo;
  p[1] = (uint32_t)(lo >> 32);
  p[2] = (uint32_t)(lo >> 64);
  p[3] = (uint32_t)(lo >> 96);
  p[4] = (uint32_t)hi;
  p[5] = (uint32_t)(hi >> 32);
  p[6] = (uint32_t)(hi >> 64);
  p[7] = (uint32_t)(hi >> 96);
}

// r = P mod q for q = 2^124 - k, P < 2^248, k < 2^28, folding first at the
// limb boundary 2^128 (2^128 = 16 * 2^124 == 16k mod q), which needs no
// shifts of P:
//   P = H*2^128 + L      ->  t = L + H*16k          (< 2^128 + 2^152: 5 limbs)
//   t = h*2^124 + l      ->  r = l + h*k            (h < 2^29; r < 2^124 + 2^57 < 2q)
//   r >= q ? r - q : r, tested as bit 124 of r + k; r >= q needs r's top
//   limb at least 0x0FFFFFFF, about one case in 2^28 for spread residues, so
//   the exact test and the subtraction sit behind a branch.
// Folding at 2^124 twice instead costs six more ALU instructions (funnel
// shifts of P, the second fold's product added outside the multiply-add
// chain): 204 against 209 G butterflies/s in the register-only probe.  Both reference
// moduli and every prime bntt_ntt_prime returns have k < 2^28.
__device__ __forceinline__ U128 reduce_pm124(const uint32_t p[8], uint32_t k) {
  const uint32_t c = k << 4;
  uint32_t t0, t1, t2, t3, t4;
  asm("mad.lo.cc.u32  %0, %5, %9, %10;\n\t"
      "madc.lo.cc.u32 %1, %6, %9, %11;\n\t"
      "madc.lo.cc.u32 %2, %7, %9, %12;\n\t"
      "madc.lo.cc.u32 %3, %8, %9, %13;\n\t"
      "madc.hi.u32    %4, %8, %9, 0;\n\t"
      "mad.hi.cc.u32  %1, %5, %9, %1;\n\t"
      "madc.hi.cc.u32 %2, %6, %9, %2;\n\t"
      "madc.hi.cc.u32 %3, %7, %9, %3;\n\t"
      "addc.u32       %4, %4, 0;\n\t"
      : "=&r"(t0), "=&r"(t1), "=&r"(t2), "=&r"(t3), "=&r"(t4)
      : "r"(p[4]), "r"(p[5]), "r"(p[6]), "r"(p[7]), "r"(c), "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]));
  const uint32_t h = __funnelshift_r(t3, t4, 28);  // t >> 124
  U128 r;
  asm("mad.lo.cc.u32  %0, %4, %5, %6;\n\t"
      "madc.hi.cc.u32 %1, %4, %5, %7;\n\t"
      "addc.cc.u32    %2, %8, 0;\n\t"
      "addc.u32       %3, %9, 0;\n\t"
      : "=r"(r.w[0]), "=r"(r.w[1]), "=r"(r.w[2]), "=r"(r.w[3])
      : "r"(h), "r"(k), "r"(t0), "r"(t1), "r"(t2), "r"(t3 & 0x0FFFFFFFu));
  if (__builtin_expect(r.w[3] >= 0x0FFFFFFFu, 0)) {  // r >= q is possible only here
    uint32_t s0, s1, s2, s3;
    asm("add.cc.u32  %0, %4, %8;\n\t"
        "addc.cc.u32 %1, %5, 0;\n\t"
        "addc.cc.u32 %2, %6, 0;\n\t"
        "addc.u32    %3, %7, 0;\n\t"
        : "=r"(s0), "=r"(s1), "=r"(s2), "=r"(s3)
        : "r"(r.w[0]), "r"(r.w[1]), "r"(r.w[2]), "r"(r.w[3]), "r"(k));
    if (s3 >> 28) {  // r + k >= 2^124, i.e. r >= q
      r.w[0] = s0; r.w[1] = s1; r.w[2] = s2; r.w[3] = s3 & 0x0FFFFFFFu;
    }
  }
  return r;
}

struct ArithFast {
  static constexpr bool kFast = true;
  __device__ __forceinline__ static U128 mul(const U128& a, const U128& b, const ModParams& m) {
    uint32_t p[8];
    mul_128x128(a, b, p);
    return reduce_pm124(p, m.k);
  }
};

// ------------------------------------------------------------------- ArithRef

struct W128 {
  uint64_t hi, lo;
};

__device__ __forceinline__ W128 w_add(W128 a, W128 b) {  // mod 2^128
  W128 r;
  r.lo = a.lo + b.lo;
  r.hi = a.hi + b.hi + (r.lo < a.lo ? 1ull : 0ull);
  return r;
}
__device__ __forceinline__ W128 w_mul64(uint64_t a, uint64_t b) {
  return W128{__umul64hi(a, b), a * b};
}
__device__ __forceinline__ W128 to_w(const U128& a) {
  return W128{((uint64_t)a.w[3] << 32) | a.w[2], ((uint64_t)a.w[1] << 32) | a.w[0]};
}
__device__ __forceinline__ U128 from_w(W128 a) {
  U128 r;
  r.w[0] = (uint32_t)a.lo; r.w[1] = (uint32_t)(a.lo >> 32);
  r.w[2] = (uint32_t)a.hi; r.w[3] = (uint32_t)(a.hi >> 32);
  return r;
}

// Reference mulmod128 with MBITS = 124, word for word: the 128x128 product
// keeps its middle sum to 128 bits (src/ntt_scalar.c:106-128), the high
// product of the quotient estimate likewise (:151-171), the low product keeps
// its cross terms to 64 bits (:130-149), and one conditional subtraction ends
// it (:194-196).
struct ArithRef {
  static constexpr bool kFast = false;
  __device__ __forceinline__ static U128 mul(const U128& ua, const U128& ub, const ModParams& m) {
    const W128 a = to_w(ua), b = to_w(ub), q = to_w(m.q), mu = to_w(m.mu);
    // product
    W128 p00 = w_mul64(a.lo, b.lo), p01 = w_mul64(a.lo, b.hi);
    W128 p10 = w_mul64(a.hi, b.lo), p11 = w_mul64(a.hi, b.hi);
    W128 mid = w_add(w_add(p01, p10), W128{0, p00.hi});
    W128 ph = w_add(p11, W128{0, mid.hi});
    W128 pl = W128{mid.lo, p00.lo};
    // quotient estimate from bits 122.. of the product
    // t = (P >> 122) mod 2^128 = (ph << 6) | (pl >> 122)
    W128 t = W128{(ph.hi << 6) | (ph.lo >> 58), (ph.lo << 6) | (pl.hi >> 58)};
    uint64_t top = ph.hi >> 58;
    W128 m01 = w_mul64(t.lo, mu.hi), m10 = w_mul64(t.hi, mu.lo), m11 = w_mul64(t.hi, mu.hi);
    W128 mm = w_add(w_add(m01, m10), W128{0, __umul64hi(t.lo, mu.lo)});
    W128 qm = w_add(w_add(m11, W128{0, mm.hi}), W128{0, top * mu.lo});
    W128 qq = W128{qm.hi >> 1, (qm.lo >> 1) | (qm.hi << 63)};
    // low product qq*q
    W128 l00 = w_mul64(qq.lo, q.lo);
    uint64_t cross = qq.lo * q.hi + qq.hi * q.lo + l00.hi;
    W128 qql = W128{cross, l00.lo};
    // r = pl - qql mod 2^128
    W128 r;
    r.lo = pl.lo - qql.lo;
    r.hi = pl.hi - qql.hi - (pl.lo < qql.lo ? 1ull : 0ull);
    const bool lt = (r.hi < q.hi) || (r.hi == q.hi && r.lo < q.lo);
    if (!lt) {
      uint64_t lo2 = r.lo - q.lo;
      r.hi = r.hi - q.hi - (r.lo < q.lo ? 1ull : 0ull);
      r.lo = lo2;
    }
    return from_w(r);
  }
};

// One butterfly of the network: (x, y) <- (x + w*y, x - w*y) with the
// reference's addmod / submod (src/ntt_scalar.c:586-588).
template <class Arith>
__device__ __forceinline__ void butterfly(U128& x, U128& y, const U128& w, const ModParams& m) {
  const U128 p = Arith::mul(w, y, m);
  if constexpr (Arith::kFast) {  // q = 2^124 - k: limbs 1..3 are constants
    const U128 s = addmod_pm(x, p, m.q.w[0]);
    y = submod_pm(x, p, m.q.w[0]);
    x = s;
  } else {
    const U128 s = addmod_ref(x, p, m.q);
    y = submod_ref(x, p, m.q);
    x = s;
  }
}

// Exact a + b mod q for q = 2^124 - k (a, b <= q): the sum less q when it
// is at least q.  Used by the inverse transform, which has no reference
// counterpart and computes canonical residues.
__device__ __forceinline__ U128 addmod_exact_pm(const U128& a, const U128& b, uint32_t q0) {
  uint32_t s0, s1, s2, s3, t0, t1, t2, t3, bw;
  asm("add.cc.u32  %0, %9, %13;\n\t"
      "addc.cc.u32 %1, %10, %14;\n\t"
      "addc.cc.u32 %2, %11, %15;\n\t"
      "addc.u32    %3, %12, %16;\n\t"
      "sub.cc.u32  %4, %0, %17;\n\t"
      "subc.cc.u32 %5, %1, 0xFFFFFFFF;\n\t"
      "subc.cc.u32 %6, %2, 0xFFFFFFFF;\n\t"
      "subc.cc.u32 %7, %3, 0x0FFFFFFF;\n\t"
      "subc.u32    %8, 0, 0;\n\t"
      : "=&r"(s0), "=&r"(s1), "=&r"(s2), "=&r"(s3), "=&r"(t0), "=&r"(t1), "=&r"(t2),
        "=&r"(t3), "=r"(bw)
      : "r"(a.w[0]), "r"(a.w[1]), "r"(a.w[2]), "r"(a.w[3]), "r"(b.w[0]), "r"(b.w[1]),
        "r"(b.w[2]), "r"(b.w[3]), "r"(q0));
  const bool keep = bw != 0u;  // s < q
  return U128{{keep ? s0 : t0, keep ? s1 : t1, keep ? s2 : t2, keep ? s3 : t3}};
}

// Inverse (Gentleman-Sande) butterfly: (x, y) <- (x + y, (x - y) * w) with
// exact sums.  With w the inverse of the forward twiddle it undoes
// butterfly() up to a factor 2 on both outputs.  Fast moduli only.
template <class Arith>
__device__ __forceinline__ void gs_butterfly(U128& x, U128& y, const U128& w, const ModParams& m) {
  static_assert(Arith::kFast, "the inverse transform uses the pseudo-Mersenne arithmetic");
  const U128 d = submod_pm(x, y, m.q.w[0]);
  x = addmod_exact_pm(x, y, m.q.w[0]);
  y = Arith::mul(w, d, m);
}

}  // namespace bntt
