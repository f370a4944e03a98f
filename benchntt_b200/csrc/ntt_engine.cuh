// ntt_engine.cuh -- the tile engine of ntt_core.cuh with the sub-transform
// size as a runtime value.
//
// NttTile (ntt_core.cuh) unrolls every pass of one fixed size; a persistent
// kernel that must handle every size then holds one unrolled copy per size
// and spends its time fetching instructions.  NttEngine keeps the same data
// flow -- each thread holds R = 2^LOGR elements, the M stages run as passes of
// at most LOGR stages, passes exchange through XOR-swizzled shared memory --
// but only the butterfly body of a pass is specialised, on the pass width r.
// Index arithmetic (which elements a thread owns, where they live) is runtime
// integer work done once per element per pass, and the register tile is
// still indexed statically.  One engine covers every size 2^LOGR..2^10 and
// both thread mappings; its shared memory is threads * R * 16 bytes for all
// of them.
#pragma once
#include "ntt_core.cuh"

namespace bntt {

template <int LOGR, class Arith>
struct NttEngine {
  static constexpr int R = 1 << LOGR;

  // The pass schedule of a 2^M sub-transform: balanced passes of <= LOGR.
  struct Passes {
    int n, base, extra;
    __device__ __forceinline__ explicit Passes(int M) {
      n = (M + LOGR - 1) / LOGR;
      base = M / n;
      extra = M - base * n;
    }
    __device__ __forceinline__ int bits(int p) const { return base + (p < extra ? 1 : 0); }
    __device__ __forceinline__ int start(int p) const { return p * base + (p < extra ? p : extra); }
  };

  // Thread -> (sub-transform in the tile, lane within it).
  __device__ __forceinline__ static void place(int tid, int M, int map, int threads, int* sub,
                                               int* lane) {
    const int tpt_log = M - LOGR;
    if (map == MAP_INTERLEAVED) {
      const int tpc = threads >> tpt_log;
      *sub = tid % tpc;
      *lane = tid / tpc;
    } else {
      *sub = tid >> tpt_log;
      *lane = tid & ((1 << tpt_log) - 1);
    }
  }

  __device__ __forceinline__ static int slot(int M, int map, int tpc, int sub, int idx) {
    if (map == MAP_INTERLEAVED) return idx * tpc + sub;
    return (sub << M) | (idx ^ ((idx >> 3) & 7));
  }

  // r stages on the groups of one pass; register indices are static.
  template <int r>
  __device__ __forceinline__ static void body(U128 (&v)[R], const SubRef& sr, int s0, int lo,
                                              int lane, int tpt, const ModParams& mp) {
    constexpr int G = 1 << r, GPT = R / G;
#pragma unroll
    for (int i = 0; i < GPT; ++i) {
      const int g = lane + i * tpt;
      const uint32_t gt = (sr.trow << s0) + (uint32_t)(g >> lo);
#pragma unroll
      for (int t = 0; t < r; ++t) {
        const int half = 1 << (r - 1 - t);
#pragma unroll
        for (int u = 0; u < (1 << t); ++u) {
          const uint4 tv = __ldg(sr.tw + ((gt << t) + (uint32_t)u));
          const U128 w = U128{{tv.x, tv.y, tv.z, tv.w}};
#pragma unroll
          for (int k = 0; k < half; ++k) {
            const int j = (u << (r - t)) | k;
            butterfly<Arith>(v[i * G + j], v[i * G + j + half], w, mp);
          }
        }
      }
    }
  }

  // Index of element e of the thread's register tile in pass (r, lo).
  __device__ __forceinline__ static int elem_index(int e, int r, int lo, int lane, int tpt) {
    const int i = e >> r, j = e & ((1 << r) - 1);
    const int g = lane + i * tpt;
    const int base = (g & ((1 << lo) - 1)) | ((g >> lo) << (lo + r));
    return base | (j << lo);
  }

  // One tile: `threads` threads, sub-transforms of 2^M points (LOGR <= M <= 10).
  // Every thread of the CTA calls it; threads of invalid sub-transforms
  // compute on zeros and store nothing.
  template <int LDP>
  __device__ __forceinline__ static void run(int M, int map, int threads, const SubRef& sr,
                                             int sub, int lane, uint4* smem, const ModParams& mp,
                                             int layout) {
    const Passes ps(M);
    const int tpt = 1 << (M - LOGR);
    const int tpc = threads >> (M - LOGR);
    const bool warp_local = map == MAP_CONTIG && tpt <= 32;
    U128 v[R];
    for (int p = 0; p < ps.n; ++p) {
      const int r = ps.bits(p), s0 = ps.start(p), lo = M - s0 - r;
      // gather
#pragma unroll
      for (int e = 0; e < R; ++e) {
        const int idx = elem_index(e, r, lo, lane, tpt);
        if (p == 0) {
          if (sr.valid) {
            v[e] = from_mem(ld_data<LDP>(sr.x + ((size_t)idx << sr.lshift)), layout);
          } else {
#pragma unroll
            for (int w = 0; w < 4; ++w) v[e].w[w] = 0u;
          }
        } else {
          const uint4 t = smem[slot(M, map, tpc, sub, idx)];
          v[e] = U128{{t.x, t.y, t.z, t.w}};
        }
      }
      // stages (pass widths run from 2 to LOGR for sizes >= 2^(LOGR+1))
      if constexpr (LOGR >= 4) {
        if (r == 4) body<(LOGR >= 4 ? 4 : 1)>(v, sr, s0, lo, lane, tpt, mp);
      }
      if (r == 3) body<3>(v, sr, s0, lo, lane, tpt, mp);
      else if (r == 2) body<2>(v, sr, s0, lo, lane, tpt, mp);
      else if (r == 1) body<1>(v, sr, s0, lo, lane, tpt, mp);
      // scatter
      const bool last = p == ps.n - 1;
#pragma unroll
      for (int e = 0; e < R; ++e) {
        const int idx = elem_index(e, r, lo, lane, tpt);
        if (last) {
          if (sr.valid) sr.y[(size_t)idx << sr.lshift] = to_mem(v[e], layout);
        } else {
          smem[slot(M, map, tpc, sub, idx)] = make_uint4(v[e].w[0], v[e].w[1], v[e].w[2], v[e].w[3]);
        }
      }
      if (!last) {
        if (warp_local) __syncwarp();
        else __syncthreads();
      }
    }
  }
};

}  // namespace bntt
