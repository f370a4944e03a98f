// ntt_core.cuh -- the forward network of benchNTT on sm_100a.
//
// The reference transform (src/ntt_scalar.c:582-627) is a radix-2 network:
// with n = log2 N, stage s (0 <= s < n) pairs indices that differ in bit
// n-1-s and multiplies by the table entry T[2^s + (index >> (n - s))].  The
// reference evaluates it in constant-geometry order with ping-pong buffers;
// here it is evaluated in place, in natural order, which yields the same
// outputs (tests check both against the reference).
//
// Sub-transforms.  Stages [S0, S0 + M) of an n-point transform touch index
// bits [L, L + M) with L = n - S0 - M; every assignment of the other bits --
// the top S0 bits H and the low L bits c -- selects an independent 2^M-point
// sub-network on the elements
//     idx(j) = (H << (n - S0)) | (j << L) | c,     j in [0, 2^M)
// whose stage S0 + s multiplies by
//     T[((2^S0 + H) << s) + (j >> (M - s))].
// A small transform is one sub-transform (S0 = L = 0).  Large transforms run
// as passes over HBM: for 2^20, pass A has S0 = 0, M = 10, L = 10 (columns)
// and pass B has S0 = 10, M = 10, L = 0 (rows).  This holds for any table T
// because it only regroups the network's data flow.
//
// Inside a sub-transform each thread holds R = 2^LOGR elements in registers.
// The M stages are cut into passes of at most LOGR stages; in a pass a thread
// owns R / 2^r groups of 2^r elements that differ only in that pass's bits
// and runs the r stages on them without communication.  Passes exchange data
// through shared memory (XOR-swizzled 16-byte slots), the first pass reads
// HBM and the last writes HBM.
#pragma once
#include "u128.cuh"

namespace bntt {

enum : int { MAP_CONTIG = 0, MAP_INTERLEAVED = 1 };

// Where one sub-transform's elements and twiddles live, as a thread sees it.
struct SubRef {
  const uint4* x;    // element j at x[j << L]
  uint4* y;          // element j at y[j << L]
  const uint4* tw;   // table of the whole transform, limb order (LAYOUT_U128)
  uint32_t trow;     // 2^S0 + H
  uint32_t lshift;   // L
  bool valid;
};

// Load policy for the first pass's HBM reads: the read-only path, or L2 only
// (coherent with writes made earlier in the same kernel by other CTAs).
enum : int { LD_NC = 0, LD_CG = 1 };

template <int LDP>
__device__ __forceinline__ uint4 ld_data(const uint4* p) {
  if constexpr (LDP == LD_CG) return __ldcg(p);
  else return __ldg(p);
}

// Optional pointwise product fused into the store of a transform's last
// pass: element e of y becomes y[e] * b[e'] mod q (vector_mul,
// src/blas_scalar.c:594), e' = (e's offset from ybase) & bmask.  bmask = N - 1
// applies one vector to every transform of the batch; all ones pairs
// transform t with b's t-th vector.  b == nullptr: plain store.
struct MulB {
  const uint4* b = nullptr;
  const uint4* ybase = nullptr;
  uint64_t bmask = 0;
};

// What the last store of an engine kernel applies (ntt_engine.cuh): an
// optional scalar multiply (the inverse transform's N^-1, held here or read
// at the store from device memory), then an optional pointwise product
// (MulB).
struct Epilogue {
  U128 scale{};
  int has_scale = 0;
  const uint4* scale_at = nullptr;  // EPI_SCALE_AT: the scalar, limb order
  MulB mul;
};

// Where a tile's first pass finds its inputs and every pass its twiddles.
//   SRC_STAGED  the inputs were copied into the tile's shared-memory slots
//               beforehand (cp.async, k_ntt_sub_staged); the first pass
//               gathers from there like the later passes
//   TW_SHARED   sr.tw points at a copy of the table in shared memory
enum : int { SRC_GLOBAL = 0, SRC_STAGED = 1, TW_SHARED = 2 };

// 16-byte asynchronous copy global -> shared (cp.async, L2 only), and the
// group commit / wait that order them.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory");
}
__device__ __forceinline__ uint4 lds128(const uint4* p) {
  uint4 v;
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
  asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
  return v;
}

template <int M, int LOGR, int TPC, int MAP, class Arith>
struct NttTile {
  static constexpr int R = 1 << LOGR;
  static constexpr int N = 1 << M;
  static constexpr int TPT = N / R;             // threads per sub-transform
  static constexpr int THREADS = TPC * TPT;
  static constexpr int NPASS = (M + LOGR - 1) / LOGR;
  static constexpr int PBASE = M / NPASS, PEXTRA = M % NPASS;
  static constexpr int SMEM_SLOTS = NPASS > 1 ? TPC * N : 0;
  // a sub-transform's threads sit in one warp
  static constexpr bool WARP_LOCAL = (MAP == MAP_CONTIG) && (TPT <= 32);
  static_assert(M >= 1 && LOGR >= 1 && LOGR <= M, "bad shape");

  __host__ __device__ static constexpr int bits(int p) { return PBASE + (p < PEXTRA ? 1 : 0); }
  __host__ __device__ static constexpr int start(int p) {
    return p * PBASE + (p < PEXTRA ? p : PEXTRA);
  }

  __device__ __forceinline__ static int sub_of(int tid) {
    return MAP == MAP_INTERLEAVED ? tid % TPC : tid / TPT;
  }
  __device__ __forceinline__ static int lane_of(int tid) {
    return MAP == MAP_INTERLEAVED ? tid / TPC : tid % TPT;
  }

  // shared-memory slot of element j of sub-transform `sub`
  __device__ __forceinline__ static int slot(int sub, int j) {
    if constexpr (MAP == MAP_INTERLEAVED) {
      return j * TPC + sub;
    } else {
      const int sw = (M >= 3) ? (j ^ ((j >> 3) & 7)) : j;
      return (sub << M) | sw;
    }
  }

  __device__ __forceinline__ static void sync() {
    if constexpr (WARP_LOCAL) __syncwarp();
    else __syncthreads();
  }

  // slot(sub, base | c) from sb = slot(sub, base) when base and c share no
  // bit and c is a constant (c = j << lo in a pass): the swizzle
  // x ^ ((x >> 3) & 7) is linear over XOR, so a contiguous tile's slot is
  // sb ^ swizzle(c); without swizzle, and for interleaved tiles, the parts
  // add.  One operation per element, with the constant folded.
  __host__ __device__ static constexpr int swz(int c) { return (M >= 3) ? (c ^ ((c >> 3) & 7)) : c; }
  __device__ __forceinline__ static int slot_at(int sb, int c) {
    if constexpr (MAP == MAP_INTERLEAVED) return sb + c * TPC;
    else if constexpr (M >= 3) return sb ^ swz(c);
    else return sb + c;
  }

  // Lowest local bit pass p touches.
  __host__ __device__ static constexpr int low(int p) { return M - start(p) - bits(p); }
  // Passes a and b exchange within each warp when both hold one group per
  // thread (r = LOGR) of a contiguous tile and both start at local bit 5 or
  // below: a warp's 32 consecutive groups then cover the indices whose bits
  // from 5 + LOGR up equal the warp's number, in both passes, so each warp
  // reads back only slots it wrote itself (the slot swizzle keeps indices in
  // their 8-aligned block).
  __host__ __device__ static constexpr bool warp_exchange(int a, int b) {
    return WARP_LOCAL || (MAP == MAP_CONTIG && bits(a) == LOGR && bits(b) == LOGR && low(a) <= 5 &&
                          low(b) <= 5);
  }
  template <int A, int B>
  __device__ __forceinline__ static void sync_between() {
    if constexpr (warp_exchange(A, B)) __syncwarp();
    else __syncthreads();
  }

  // Runs the whole sub-transform.  Every thread of the tile must call it
  // (it synchronises); threads whose sub-transform is not valid compute on
  // zeros and store nothing.
  template <int LDP, int SRC = SRC_GLOBAL>
  __device__ __forceinline__ static void run(const SubRef& sr, int sub, int lane, uint4* smem,
                                             const ModParams& mp, int layout,
                                             const MulB& mb = MulB{}) {
    U128 v[R];
    pass<0, LDP, SRC>(v, sr, sub, lane, smem, mp, layout, mb);
  }

  template <int P, int LDP, int SRC = SRC_GLOBAL>
  __device__ __forceinline__ static void pass(U128 (&v)[R], const SubRef& sr, int sub, int lane,
                                              uint4* smem, const ModParams& mp, int layout,
                                              const MulB& mb) {
    constexpr int r = bits(P);
    constexpr int s0 = start(P);
    constexpr int lo = M - s0 - r;        // lowest local bit this pass touches
    constexpr int G = 1 << r;             // elements per group
    constexpr int GPT = R / G;            // groups per thread
    static_assert(GPT >= 1, "pass wider than the register tile");
    // element j of a group in HBM: the group's first element plus j * gstep
    const size_t gstep = (size_t)1 << (lo + sr.lshift);

    // ---- gather
#pragma unroll
    for (int i = 0; i < GPT; ++i) {
      const int g = lane + i * TPT;
      const int base = (g & ((1 << lo) - 1)) | ((g >> lo) << (lo + r));
      const int sb = slot(sub, base);
#pragma unroll
      for (int j = 0; j < G; ++j) {
        if constexpr (P == 0 && (SRC & SRC_STAGED) != 0) {
          v[i * G + j] = from_mem(smem[slot_at(sb, j << lo)], layout);  // staged in memory order
        } else if constexpr (P == 0) {
          if (sr.valid) {
            v[i * G + j] = from_mem(ld_data<LDP>(sr.x + ((size_t)base << sr.lshift) + (size_t)j * gstep), layout);
          } else {
#pragma unroll
            for (int w = 0; w < 4; ++w) v[i * G + j].w[w] = 0u;
          }
        } else {
          const uint4 t = smem[slot_at(sb, j << lo)];
          v[i * G + j] = U128{{t.x, t.y, t.z, t.w}};
        }
      }
    }

    // ---- r stages on each group
#pragma unroll
    for (int i = 0; i < GPT; ++i) {
      const int g = lane + i * TPT;
      const uint32_t gt = (sr.trow << s0) + (uint32_t)(g >> lo);
#pragma unroll
      for (int t = 0; t < r; ++t) {
        const int half = 1 << (r - 1 - t);
#pragma unroll
        for (int u = 0; u < (1 << t); ++u) {
          // tables are stored in limb order (LAYOUT_U128) by the plan
          const uint4* twt = sr.tw + (gt << t);  // u as an immediate offset
          const uint4 tv = (SRC & TW_SHARED) != 0 ? lds128(twt + u) : __ldg(twt + u);
          const U128 w = U128{{tv.x, tv.y, tv.z, tv.w}};
#pragma unroll
          for (int k = 0; k < half; ++k) {
            const int j = (u << (r - t)) | k;
            butterfly<Arith>(v[i * G + j], v[i * G + j + half], w, mp);
          }
        }
      }
    }

    // ---- scatter
#pragma unroll
    for (int i = 0; i < GPT; ++i) {
      const int g = lane + i * TPT;
      const int base = (g & ((1 << lo) - 1)) | ((g >> lo) << (lo + r));
      const int sb = slot(sub, base);
#pragma unroll
      for (int j = 0; j < G; ++j) {
        if constexpr (P == NPASS - 1) {
          if (sr.valid) {
            uint4* yp = sr.y + ((size_t)base << sr.lshift) + (size_t)j * gstep;
            U128 o = v[i * G + j];
            if (mb.b) {
              const uint4 bv = __ldg(mb.b + ((uint64_t)(yp - mb.ybase) & mb.bmask));
              o = Arith::mul(o, from_mem(bv, layout), mp);
            }
            *yp = to_mem(o, layout);
          }
        } else {
          const U128& e = v[i * G + j];
          smem[slot_at(sb, j << lo)] = make_uint4(e.w[0], e.w[1], e.w[2], e.w[3]);
        }
      }
    }
    if constexpr (P + 1 < NPASS) {
      sync_between<P, P + 1>();
      pass<P + 1, LDP, SRC>(v, sr, sub, lane, smem, mp, layout, mb);
    }
  }

  // The inverse network of the same passes: the last pass first, each pass's
  // stages in reverse order as Gentleman-Sande butterflies on the inverse
  // table (gs_butterfly).  The store that finishes the transform (pass 0)
  // multiplies the lower half of each group -- the x outputs of stage 0 --
  // by *scale_at (N^-1) when scale_at is not null; the upper half gets N^-1
  // through the inverse table's entry 1.  Fast moduli only.
  template <int LDP>
  __device__ __forceinline__ static void run_inv(const SubRef& sr, int sub, int lane, uint4* smem,
                                                 const ModParams& mp, int layout,
                                                 const uint4* scale_at) {
    U128 v[R];
    pass_inv<NPASS - 1, LDP>(v, sr, sub, lane, smem, mp, layout, scale_at);
  }

  // stage t of a group of 2^r registers from e0, inverse butterflies
  template <int r, int t>
  __device__ __forceinline__ static void stage_inv(U128 (&v)[R], int e0, uint32_t gt,
                                                   const uint4* tw, const ModParams& mp) {
    constexpr int half = 1 << (r - 1 - t);
#pragma unroll
    for (int u = 0; u < (1 << t); ++u) {
      const uint4 tv = __ldg(tw + (gt << t) + u);
      const U128 w = U128{{tv.x, tv.y, tv.z, tv.w}};
#pragma unroll
      for (int k = 0; k < half; ++k) {
        const int j = e0 + ((u << (r - t)) | k);
        gs_butterfly<Arith>(v[j], v[j + half], w, mp);
      }
    }
  }

  template <int P, int LDP>
  __device__ __forceinline__ static void pass_inv(U128 (&v)[R], const SubRef& sr, int sub, int lane,
                                                  uint4* smem, const ModParams& mp, int layout,
                                                  const uint4* scale_at) {
    constexpr int r = bits(P);
    constexpr int s0 = start(P);
    constexpr int lo = M - s0 - r;
    constexpr int G = 1 << r;
    constexpr int GPT = R / G;
    static_assert(GPT >= 1 && r <= 4, "pass shape");
    const size_t gstep = (size_t)1 << (lo + sr.lshift);  // HBM distance of j and j + 1

    // ---- gather: the inverse reads its input in the last pass's order
#pragma unroll
    for (int i = 0; i < GPT; ++i) {
      const int g = lane + i * TPT;
      const int base = (g & ((1 << lo) - 1)) | ((g >> lo) << (lo + r));
      const int sb = slot(sub, base);
#pragma unroll
      for (int j = 0; j < G; ++j) {
        if constexpr (P == NPASS - 1) {
          if (sr.valid) {
            v[i * G + j] = from_mem(ld_data<LDP>(sr.x + ((size_t)base << sr.lshift) + (size_t)j * gstep), layout);
          } else {
#pragma unroll
            for (int w = 0; w < 4; ++w) v[i * G + j].w[w] = 0u;
          }
        } else {
          const uint4 t = smem[slot_at(sb, j << lo)];
          v[i * G + j] = U128{{t.x, t.y, t.z, t.w}};
        }
      }
    }

    // ---- r stages on each group, the last first
#pragma unroll
    for (int i = 0; i < GPT; ++i) {
      const int g = lane + i * TPT;
      const uint32_t gt = (sr.trow << s0) + (uint32_t)(g >> lo);
      if constexpr (r > 3) stage_inv<r, 3>(v, i * G, gt, sr.tw, mp);
      if constexpr (r > 2) stage_inv<r, 2>(v, i * G, gt, sr.tw, mp);
      if constexpr (r > 1) stage_inv<r, 1>(v, i * G, gt, sr.tw, mp);
      stage_inv<r, 0>(v, i * G, gt, sr.tw, mp);
    }

    // ---- N^-1 on the finishing store
    if constexpr (P == 0) {
      if (scale_at && sr.valid) {
        const uint4 f = __ldg(scale_at);
        const U128 fs = U128{{f.x, f.y, f.z, f.w}};
#pragma unroll
        for (int i = 0; i < GPT; ++i)
#pragma unroll
          for (int j = 0; j < G / 2; ++j) v[i * G + j] = Arith::mul(v[i * G + j], fs, mp);
      }
    }

    // ---- scatter
#pragma unroll
    for (int i = 0; i < GPT; ++i) {
      const int g = lane + i * TPT;
      const int base = (g & ((1 << lo) - 1)) | ((g >> lo) << (lo + r));
      const int sb = slot(sub, base);
#pragma unroll
      for (int j = 0; j < G; ++j) {
        if constexpr (P == 0) {
          if (sr.valid) sr.y[((size_t)base << sr.lshift) + (size_t)j * gstep] = to_mem(v[i * G + j], layout);
        } else {
          const U128& e = v[i * G + j];
          smem[slot_at(sb, j << lo)] = make_uint4(e.w[0], e.w[1], e.w[2], e.w[3]);
        }
      }
    }
    if constexpr (P > 0) {
      sync_between<P, P - 1>();
      pass_inv<P - 1, LDP>(v, sr, sub, lane, smem, mp, layout, scale_at);
    }
  }
};

// Geometry of one launch over sub-transforms (see the header comment).
struct SubGeom {
  const uint4* x;
  uint4* y;
  const uint4* tw;
  uint32_t n;       // log2 of the whole transform
  uint32_t s0;      // first stage of this pass
  uint32_t m;       // stages in this pass
  uint32_t l;       // low bits below the pass bits
  uint64_t nsub;    // number of sub-transforms (all transforms of the batch)
  const uint4* b = nullptr;  // last pass only: fused pointwise product (MulB)
  uint64_t bmask = 0;
};

// Sub-transform `sid` of a geometry: sid = (transform << (S0 + L)) | (H << L) | c.
__device__ __forceinline__ SubRef make_subref(const SubGeom& g, uint64_t sid) {
  SubRef r;
  r.valid = sid < g.nsub;
  const uint64_t s = r.valid ? sid : 0;
  const uint64_t big = s >> (g.s0 + g.l);
  const uint64_t hbits = (s >> g.l) & ((1ull << g.s0) - 1);
  const uint64_t c = s & ((1ull << g.l) - 1);
  const uint64_t off = (big << g.n) + (hbits << (g.n - g.s0)) + c;
  r.x = g.x + off;
  r.y = g.y + off;
  r.tw = g.tw;
  r.trow = (1u << g.s0) + (uint32_t)hbits;
  r.lshift = g.l;
  return r;
}

}  // namespace bntt
