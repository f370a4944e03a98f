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
// integer work (a group base per pass, then one add per element), and the
// register tile is still indexed statically.  One engine covers every size
// 2^LOGR..2^10 and both thread mappings; its shared memory is smem_slots()
// 16-byte slots.
#pragma once
#include "ntt_core.cuh"

namespace bntt {

enum : int { EPI_SCALE = 1, EPI_MUL = 2, EPI_SCALE_AT = 4 };

template <int LOGR, class Arith>
struct NttEngine {
  static constexpr int R = 1 << LOGR;

  // The pass schedule of a 2^M sub-transform: balanced passes of <= LOGR.
  struct Passes {
    int n, base, extra;
    __device__ __forceinline__ explicit Passes(int M) {
      n = (M + LOGR - 1) / LOGR;
      // M / n without a division instruction: n <= 4 and M <= 31, or n = 5
      // and M <= 10 (the 4-element engine's 2^9 and 2^10)
      base = n == 1 ? M : n == 2 ? M >> 1 : n == 3 ? (M * 11) >> 5 : n == 4 ? M >> 2 : (M * 13) >> 6;
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

  // Shared-memory slots (16 bytes each) of a tile.  Element idx of
  // sub-transform `sub` has the linear index
  //   contiguous tiles:  L = (sub << M) + idx
  //   interleaved tiles: L = idx * TPC + sub
  // and lives in slot L + (L >> 3): one pad slot per 8 spreads the strided
  // accesses of every pass over the banks.  Within a pass, element j of a
  // group is L(base) + j * (lmul << lo), so each element costs one
  // multiply-add and one shifted add.
  __host__ __device__ static constexpr size_t smem_slots(int M, int map, int threads) {
    (void)M;
    (void)map;
    return (size_t)threads * R + ((size_t)threads * R >> 3);
  }

  struct Layout {
    int lbase, lmul;  // linear index L(idx) = lbase + idx * lmul
  };
  __device__ __forceinline__ static int pad(int l) { return l + (l >> 3); }

  // Stage t of a group of 2^r elements starting at register e0: butterflies
  // of distance 2^(r-1-t), twiddle T[(gt << t) + u] for the u-th block.
  template <int r, int t, bool INV>
  __device__ __forceinline__ static void stage(U128 (&v)[R], int e0, uint32_t gt, const uint4* tw,
                                               const ModParams& mp) {
    constexpr int half = 1 << (r - 1 - t);
#pragma unroll
    for (int u = 0; u < (1 << t); ++u) {
      const uint4 tv = __ldg(tw + (gt << t) + u);
      const U128 w = U128{{tv.x, tv.y, tv.z, tv.w}};
#pragma unroll
      for (int k = 0; k < half; ++k) {
        const int j = e0 + ((u << (r - t)) | k);
        if constexpr (INV) gs_butterfly<Arith>(v[j], v[j + half], w, mp);
        else butterfly<Arith>(v[j], v[j + half], w, mp);
      }
    }
  }

  // One pass of width r (1 <= r <= LOGR) over the thread's GPT = R / 2^r
  // groups: gather (global on the first pass, else shared), r butterfly
  // stages with static register indices, scatter (global on the last pass).
  //
  // INV runs the inverse of the same r stages: the stages in reverse order,
  // each an inverse (Gentleman-Sande) butterfly with the table holding the
  // inverse twiddles.  EPI applies *ep (when not null) on the last store:
  // bit EPI_SCALE its scalar multiply, EPI_SCALE_AT the multiply by the
  // scalar at ep->scale_at, bit EPI_MUL its pointwise product.
  template <int r, int LDP, bool INV = false, int EPI = 0>
  __device__ __forceinline__ static void pass(U128 (&v)[R], const SubRef& sr, int s0, int lo,
                                              int lane, int tpt, bool first, bool last,
                                              const Layout& lay, uint4* smem, const ModParams& mp,
                                              int layout, const Epilogue* ep = nullptr) {
    constexpr int G = 1 << r, GPT = R / G;
    const int hi_mask = ~((1 << lo) - 1);
    const int step = lay.lmul << lo;  // linear-index distance of j and j + 1
    // Slot of element j of a group: pad(lb + j*step).  With 4 elements per
    // thread it is pad(lb) plus an offset that does not depend on lb, so each
    // element costs one add: step a multiple of 8 (interleaved tiles, whose
    // lmul is a multiple of 8, and contiguous passes with lo >= 3) adds step
    // plus its pad slots; contiguous passes with lo <= 2 start a group at a
    // linear index whose position in its 8-slot block leaves room for the
    // group up to one pad slot, crossed between elements 1 and 2 when the
    // step is 4 (the group base is (g mod 2^lo) + (g >> lo) * G * 2^lo on top
    // of a multiple of 8).
    const int s9 = step >= 8 ? step + (step >> 3) : step;
    const int c2 = step == 4 ? 1 : 0;
    auto slot_of = [&](int lb, int j) {
      if constexpr (LOGR == 2) return pad(lb) + j * s9 + (j >> 1) * c2;
      else return pad(lb + j * step);
    };
    const uint32_t gstep = 1u << (lo + sr.lshift);  // the same in global memory
    // group i's local index base: (g & lomask) | ((g >> lo) << (lo + r))
    auto base = [&](int i) {
      const int g = lane + i * tpt;
      return g + (g & hi_mask) * (G - 1);
    };
    // gather
#pragma unroll
    for (int i = 0; i < GPT; ++i) {
      if (first) {
        const uint4* gp = sr.x + ((size_t)base(i) << sr.lshift);
#pragma unroll
        for (int j = 0; j < G; ++j) {
          if (sr.valid) {
            v[i * G + j] = from_mem(ld_data<LDP>(gp + (size_t)(j * gstep)), layout);
          } else {
#pragma unroll
            for (int w = 0; w < 4; ++w) v[i * G + j].w[w] = 0u;
          }
        }
      } else {
        const int lb = lay.lbase + base(i) * lay.lmul;
#pragma unroll
        for (int j = 0; j < G; ++j) {
          const uint4 t = smem[slot_of(lb, j)];
          v[i * G + j] = U128{{t.x, t.y, t.z, t.w}};
        }
      }
    }
    // r stages per group; stage t of the group reads T[(gt << t) + u],
    // u < 2^t.  The inverse runs them in reverse order; with 3 or 4 stages
    // each of its stages is a separate instantiation (stage()), since the
    // compiler otherwise keeps v in local memory for the reversed loop.
#pragma unroll
    for (int i = 0; i < GPT; ++i) {
      const int g = lane + i * tpt;
      const uint32_t gt = (sr.trow << s0) + (uint32_t)(g >> lo);
      if constexpr (INV && r > 2) {
        if constexpr (r > 3) stage<r, 3, true>(v, i * G, gt, sr.tw, mp);
        stage<r, 2, true>(v, i * G, gt, sr.tw, mp);
        stage<r, 1, true>(v, i * G, gt, sr.tw, mp);
        stage<r, 0, true>(v, i * G, gt, sr.tw, mp);
      } else {
#pragma unroll
        for (int tt = 0; tt < r; ++tt) {
          const int t = INV ? r - 1 - tt : tt;
          const int half = 1 << (r - 1 - t);
#pragma unroll
          for (int u = 0; u < (1 << t); ++u) {
            const uint4 tv = __ldg(sr.tw + (gt << t) + u);
            const U128 w = U128{{tv.x, tv.y, tv.z, tv.w}};
#pragma unroll
            for (int k = 0; k < half; ++k) {
              const int j = (u << (r - t)) | k;
              if constexpr (INV) gs_butterfly<Arith>(v[i * G + j], v[i * G + j + half], w, mp);
              else butterfly<Arith>(v[i * G + j], v[i * G + j + half], w, mp);
            }
          }
        }
      }
    }
    // the inverse's N^-1 (EPI_SCALE_AT): the upper half of each group holds
    // y outputs of the last stage, whose table entry carries it already
    if constexpr ((EPI & EPI_SCALE_AT) != 0) {
      if (last && ep && sr.valid) {
        const uint4 f = __ldg(ep->scale_at);
        const U128 fs = U128{{f.x, f.y, f.z, f.w}};
#pragma unroll
        for (int i = 0; i < GPT; ++i)
#pragma unroll
          for (int j = 0; j < (INV ? G / 2 : G); ++j) v[i * G + j] = Arith::mul(v[i * G + j], fs, mp);
      }
    }
    // scatter
#pragma unroll
    for (int i = 0; i < GPT; ++i) {
      if (last) {
        uint4* const gq = sr.y + ((size_t)base(i) << sr.lshift);
#pragma unroll
        for (int j = 0; j < G; ++j) {
          if (sr.valid) {
            uint4* yp = gq + (size_t)(j * gstep);
            if constexpr (EPI != 0) {
              if (ep) {
                // the inverse's N^-1: the upper half of the group holds y
                // outputs of the last stage, whose table entry carries it
                const bool scaled = !INV || j < G / 2;
                if constexpr ((EPI & EPI_SCALE) != 0) {
                  if (ep->has_scale && scaled) v[i * G + j] = Arith::mul(v[i * G + j], ep->scale, mp);
                }
                if ((EPI & EPI_MUL) != 0 && ep->mul.b) {
                  const uint4 bv = __ldg(ep->mul.b + ((uint64_t)(yp - ep->mul.ybase) & ep->mul.bmask));
                  v[i * G + j] = Arith::mul(v[i * G + j], from_mem(bv, layout), mp);
                }
              }
            }
            *yp = to_mem(v[i * G + j], layout);
          }
        }
      } else {
        const int lb = lay.lbase + base(i) * lay.lmul;
#pragma unroll
        for (int j = 0; j < G; ++j) {
          const U128& e = v[i * G + j];
          smem[slot_of(lb, j)] =
              make_uint4(e.w[0], e.w[1], e.w[2], e.w[3]);
        }
      }
    }
  }

  // One tile: `threads` threads, sub-transforms of 2^M points (LOGR <= M <= 10).
  // Every thread of the CTA calls it; threads of invalid sub-transforms
  // compute on zeros and store nothing.
  //
  // INV = true runs the inverse network of the same passes (last pass
  // first); EPI (EPI_SCALE | EPI_MUL bits) applies *ep (when not null) to the
  // stored results.
  template <int LDP, bool INV = false, int EPI = 0>
  __device__ __forceinline__ static void run(int M, int map, int threads, const SubRef& sr,
                                             int sub, int lane, uint4* smem, const ModParams& mp,
                                             int layout, const Epilogue* ep = nullptr) {
    const Passes ps(M);
    const int tpt = 1 << (M - LOGR);
    const bool contig = map == MAP_CONTIG;
    const bool warp_local = contig && tpt <= 32;
    Layout lay;
    lay.lbase = contig ? sub << M : sub;
    lay.lmul = contig ? 1 : threads >> (M - LOGR);
    U128 v[R];
    for (int pp = 0; pp < ps.n; ++pp) {
      const int p = INV ? ps.n - 1 - pp : pp;
      const int r = ps.bits(p), s0 = ps.start(p), lo = M - s0 - r;
      const bool first = pp == 0, last = pp == ps.n - 1;
      if constexpr (LOGR >= 4) {
        if (r == 4)
          pass<(LOGR >= 4 ? 4 : 1), LDP, INV, EPI>(v, sr, s0, lo, lane, tpt, first, last, lay, smem, mp,
                                              layout, ep);
      }
      // with LOGR = 3 the balanced passes of 2^3..2^10 points have 2 or 3
      // stages, so width 1 needs no code there
      if (LOGR >= 3 && r == 3)
        pass<(LOGR >= 3 ? 3 : 1), LDP, INV, EPI>(v, sr, s0, lo, lane, tpt, first, last, lay, smem, mp,
                                                 layout, ep);
      else if (r == 2)
        pass<2, LDP, INV, EPI>(v, sr, s0, lo, lane, tpt, first, last, lay, smem, mp, layout, ep);
      else if (LOGR != 3)
        pass<1, LDP, INV, EPI>(v, sr, s0, lo, lane, tpt, first, last, lay, smem, mp, layout, ep);
      if (!last) {
        // the next pass exchanges within each warp when both hold one group
        // per thread of a contiguous tile and start at local bit 5 or below
        // (NttTile::warp_exchange); M and the mapping are the same for the
        // whole CTA, so every thread takes the same branch
        const int pn = INV ? p - 1 : p + 1;
        const int rn = ps.bits(pn), lon = M - ps.start(pn) - rn;
        if (warp_local || (contig && r == LOGR && rn == LOGR && lo <= 5 && lon <= 5)) __syncwarp();
        else __syncthreads();
      }
    }
  }
};

}  // namespace bntt
