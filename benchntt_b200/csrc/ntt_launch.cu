// ntt_launch.cu -- registry of compiled sub-transform kernels, the HBM pass
// split, and the stream-ordered forward transform.
#include <algorithm>
#include <functional>
#include <mutex>

#include "internal.h"
#include "ntt_core.cuh"

namespace bntt {

void append_fast_contig(std::vector<SubKernel>& v);
void append_fast_contig_r4(std::vector<SubKernel>& v);
void append_fast_il(std::vector<SubKernel>& v);
void append_ref(std::vector<SubKernel>& v);
void append_fast_occ(std::vector<SubKernel>& v);
void append_fast_small(std::vector<SubKernel>& v);
void append_fast_staged(std::vector<SubKernel>& v);
void append_fast_occ5(std::vector<SubKernel>& v);

const std::vector<SubKernel>& sub_kernels() {
  static std::vector<SubKernel> v = [] {
    std::vector<SubKernel> r;
    append_fast_contig(r);
    append_fast_contig_r4(r);
    append_fast_il(r);
    append_ref(r);
    append_fast_occ(r);
    append_fast_small(r);
    append_fast_staged(r);
    append_fast_occ5(r);
    return r;
  }();
  return v;
}

const SubKernel* pick_sub_kernel(int m, int map, int fast, int logr_pref, int tpc_pref) {
  const SubKernel* best = nullptr;
  for (const SubKernel& k : sub_kernels()) {
    if (k.m != m || k.map != map || k.fast != fast) continue;
    if (logr_pref && k.logr != logr_pref) continue;
    if (tpc_pref && k.tpc != tpc_pref) continue;
    if (!best) best = &k;  // the first registered shape is the default
  }
  return best;
}

int blocks_per_sm(const SubKernel* k) {
  static std::mutex mu;
  std::lock_guard<std::mutex> g(mu);
  SubKernel* mk = const_cast<SubKernel*>(k);
  if (mk->max_blocks_per_sm > 0) return mk->max_blocks_per_sm;
  if (k->smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k->fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)k->smem);
    if (e != cudaSuccess) return -cuda_error(e, "cudaFuncSetAttribute(smem)");
  }
  int b = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k->fn, k->threads, k->smem);
  if (e != cudaSuccess) return -cuda_error(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (b < 1) return -set_error(BNTT_ECUDA, "kernel m=%d logr=%d tpc=%d does not fit on an SM", k->m,
                               k->logr, k->tpc);
  mk->max_blocks_per_sm = b;
  return b;
}

int launch_sub(bntt_ctx* ctx, const SubKernel* k, const void* geom, const ModParams& mp,
               int layout, cudaStream_t stream, int grid_cap) {
  const SubGeom& g = *static_cast<const SubGeom*>(geom);
  const uint64_t ntiles = (g.nsub + (uint64_t)k->tpc - 1) / (uint64_t)k->tpc;
  if (ntiles == 0) return BNTT_OK;
  const int bps = blocks_per_sm(k);
  if (bps < 0) return -bps;
  uint64_t grid = std::min<uint64_t>(ntiles, (uint64_t)bps * (uint64_t)ctx->sms);
  if (grid_cap > 0) grid = std::min<uint64_t>(grid, (uint64_t)grid_cap);
  SubGeom gg = g;
  ModParams mm = mp;
  int lay = layout;
  void* args[] = {&gg, &mm, &lay};
  BNTT_CK(cudaLaunchKernel(k->fn, dim3((unsigned)grid), dim3(k->threads), args, k->smem, stream));
  ctx->launches++;
  return BNTT_OK;
}

// Balanced split of n stages into HBM passes of at most `max_m` stages each
// (a 2^10-point sub-transform is the largest that lives in one CTA).
std::vector<int> split_passes(int n, int max_m) {
  std::vector<int> p;
  const int k = (n + max_m - 1) / max_m;
  for (int i = 0; i < k; ++i) p.push_back(n / k + (i < n % k ? 1 : 0));
  return p;
}

// Split of a 2^n transform (n > 10) for the tile engine: the fewest HBM
// passes of at most 8 stages, and among those the split with the fewest
// engine passes (each engine pass covers at most 3 stages, so a pass of 6
// stages costs 2 and one of 7 costs 3), then the widest first pass.  For
// 2^20 that is 8 + 6 + 6 (7 engine passes) instead of 7 + 7 + 6 (8).
std::vector<int> engine_split(int n) {
  const int k = (n + 7) / 8;
  std::vector<int> best, cur(k, 0);
  int best_cost = 1 << 30;
  // enumerate compositions of n into k parts in [1, 8], first part largest first
  std::vector<int> stack;
  std::function<void(int, int)> rec = [&](int i, int left) {
    if (i == k - 1) {
      if (left < 1 || left > 8) return;
      cur[i] = left;
      int cost = 0, s0 = 0;
      for (int j = 0; j < k; ++j) {
        const int m = cur[j], l = n - s0 - m;
        if (m < 3) return;  // the engine needs >= 2^3 points
        // a strided pass: at least 2^5 points (the interleaved tile shapes),
        // and its 256 >> (m - 3) columns per tile must exist (<= 2^l)
        if (l > 0 && (m < 5 || 11 - m > l)) return;
        cost += (m + 2) / 3;
        s0 += m;
      }
      if (cost < best_cost) {
        best_cost = cost;
        best = cur;
      }
      return;
    }
    for (int m = 8; m >= 1; --m) {
      if (left - m < (k - 1 - i) || left - m > 8 * (k - 1 - i)) continue;
      cur[i] = m;
      rec(i + 1, left - m);
    }
  };
  rec(0, n);
  return best;
}

int plan_choose_kernels(bntt_plan* p) {
  const int n = (int)p->log2n;
  p->passes = split_passes(n);
  p->kernels.clear();
  const bool fast = arith_fast(p->ctx, p->fast);
  int s0 = 0;
  for (size_t i = 0; i < p->passes.size(); ++i) {
    const int m = p->passes[i];
    const int l = n - s0 - m;
    const int map = l > 0 ? MAP_INTERLEAVED : MAP_CONTIG;
    // the tuned shape if the autotuner ran, else the first registered shape
    // that fits (interleaved tiles need TPC adjacent columns, so TPC <= 2^l)
    const SubKernel* k = tuned_sub_kernel(m, map, fast ? 1 : 0, l);
    // a table copied into shared memory holds entries below 2^m only: whole
    // transforms (s0 = 0)
    if (k && (k->src & TW_SHARED) && s0 != 0) k = nullptr;
    // untuned contiguous passes with the fast multiply: the 4-element shape
    // capped at 4 resident CTAs per SM (2^3..2^10), else the shape capped at
    // 3 -- measured on B200; without a cap the compiler spends up to 214
    // registers and one CTA fills the SM
    for (int want_minb : {4, 3}) {
      for (const SubKernel& c : sub_kernels()) {
        if (k || map != MAP_CONTIG || !fast) break;
        if (c.m == m && c.map == map && c.fast == 1 && c.minb == want_minb && c.src == 0) k = &c;
      }
    }
    for (const SubKernel& c : sub_kernels()) {
      if (k) break;
      if (c.m != m || c.map != map || c.fast != (fast ? 1 : 0) || c.src != 0) continue;
      if (map == MAP_INTERLEAVED && (1 << l) < c.tpc) continue;
      k = &c;
    }
    if (!k) return set_error(BNTT_EINVAL, "no kernel compiled for pass m=%d map=%d", m, map);
    p->kernels.push_back(k);
    s0 += m;
  }
  return BNTT_OK;
}

int ntt_forward_on(bntt_plan* plan, void* y, const void* x, size_t batch, cudaStream_t s,
                   const void* b, uint64_t bmask) {
  if (batch == 0) return BNTT_OK;
  const int n = (int)plan->log2n;
  // above 2^10 points: the persistent kernel's split on 4-element tiles
  // (strided passes of 5..7 stages over 2^(10-m) adjacent columns, 256 B or
  // more per row, then a contiguous pass), else the runtime-size engine with
  // passes of at most 8 stages.  Measured at 2^16: 0.83 against 0.73 of the
  // IMAD roofline for the engine; compiled tiles with 10-stage passes, whose
  // strided passes touch 2 or 4 columns per row, were 1.5x slower than that.
  if (n > 10 && arith_fast(plan->ctx, plan->fast)) {
    const std::vector<int> split = tile_split(n);
    std::vector<const SubKernel*> ks;
    int s0 = 0;
    for (int m : split) {
      const int map = n - s0 - m > 0 ? MAP_INTERLEAVED : MAP_CONTIG;
      const SubKernel* found = nullptr;
      for (const SubKernel& k : sub_kernels())
        if (k.m == m && k.map == map && k.fast == 1 && k.logr == 2 && k.tpc == (256 >> (m - 2)) &&
            k.minb == 4 && k.src == 0)
          found = &k;
      if (!found) break;
      ks.push_back(found);
      s0 += m;
    }
    if (split.empty() || ks.size() != split.size()) return engine_forward_on(plan, y, x, batch, s, b, bmask);
    s0 = 0;
    for (size_t i = 0; i < split.size(); ++i) {
      const int m = split[i];
      SubGeom g;
      g.x = static_cast<const uint4*>(i == 0 ? x : y);
      g.y = static_cast<uint4*>(y);
      g.tw = static_cast<const uint4*>(plan->tw);
      g.n = (uint32_t)n;
      g.s0 = (uint32_t)s0;
      g.m = (uint32_t)m;
      g.l = (uint32_t)(n - s0 - m);
      g.nsub = (uint64_t)batch << (n - m);
      if (i + 1 == split.size()) {
        g.b = static_cast<const uint4*>(b);
        g.bmask = bmask;
      }
      if (int rc = launch_sub(plan->ctx, ks[i], &g, plan->mp, plan->layout, s)) return rc;
      s0 += m;
    }
    return BNTT_OK;
  }
  int s0 = 0;
  for (size_t i = 0; i < plan->passes.size(); ++i) {
    const int m = plan->passes[i];
    SubGeom g;
    g.x = static_cast<const uint4*>(i == 0 ? x : y);
    g.y = static_cast<uint4*>(y);
    g.tw = static_cast<const uint4*>(plan->tw);
    g.n = (uint32_t)n;
    g.s0 = (uint32_t)s0;
    g.m = (uint32_t)m;
    g.l = (uint32_t)(n - s0 - m);
    g.nsub = (uint64_t)batch << (n - m);
    if (i + 1 == plan->passes.size()) {
      g.b = static_cast<const uint4*>(b);
      g.bmask = bmask;
    }
    int rc = launch_sub(plan->ctx, plan->kernels[i], &g, plan->mp, plan->layout, s);
    if (rc) return rc;
    s0 += m;
  }
  return BNTT_OK;
}

}  // namespace bntt
