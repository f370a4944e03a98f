// ntt_engine_plan.cu -- plan transforms on the runtime-size tile engine:
// the inverse transform, and the forward transform above 2^10 points.
//
// The reference has no inverse transform.  The forward network
// (src/ntt_scalar.c:582-627, in its in-place form: stage s pairs indices
// that differ in bit n-1-s with twiddle T[2^s + (index >> (n-s))]) is a
// product of butterflies (x, y) -> (x + w y, x - w y); each is invertible
// when w is, with inverse (u, v) -> ((u + v) / 2, (u - v) / (2 w)).  So
// running the stages from the last to the first with Gentleman-Sande
// butterflies (x, y) -> (x + y, (x - y) w^-1) and multiplying by N^-1 at the
// end returns the input, for every table whose entries are invertible mod a
// prime q.  With the root-power tables of roots.cu it is the inverse
// negacyclic NTT, and ntt^-1(ntt(a) o ntt(b)) = a * b mod (x^N + 1).
//
// Sums here are exact mod q (no reference quirk applies: the reference has
// no such code); results are canonical residues in [0, q).  The fast
// pseudo-Mersenne multiply is required (q = 2^124 - k, k < 2^28).
//
// Kernels: the compile-time tile in inverse mode (k_ntt_tile_inv), one
// launch for N = 2^3..2^10 and above that one launch per HBM pass of the
// persistent kernel's split (tile_split), in reverse pass order (the pass
// over the low index bits first); a one-thread-per-transform kernel for N = 2
// and 4.  The runtime-size tile engine (ntt_engine.cuh) in inverse mode
// remains for splits without a tile kernel, and in forward mode for the
// forward transforms above 2^10 points (engine_forward_on) likewise: passes
// of at most 8 stages keep the strided passes coalesced.
#include <algorithm>
#include <atomic>
#include <vector>

#include "internal.h"
#include "ntt_core.cuh"
#include "ntt_engine.cuh"

namespace bntt {
namespace {

// Tiles of 256 threads; the HBM passes of a large transform come from
// engine_split (at most 8 stages each, so a strided tile covers at least 8
// adjacent columns: 128 contiguous bytes per row).
constexpr int kEngThreads = 256;

using PlanEngine = NttEngine<3, ArithFast>;

// One HBM pass of a plan transform on the tile engine: tiles of 256 threads,
// persistent over the pass's tiles.  INV selects the inverse network; `ep`
// is applied by the last store when use_ep is set.
template <bool INV>
__global__ void __launch_bounds__(kEngThreads, 3)
    k_ntt_engine(SubGeom g, ModParams mp, int layout, int m, int map, Epilogue ep, int use_ep) {
  extern __shared__ uint4 smem[];
  int sub, lane;
  PlanEngine::place(threadIdx.x, m, map, kEngThreads, &sub, &lane);
  const int tpc = kEngThreads >> (m - 3);
  const uint64_t ntiles = (g.nsub + (uint64_t)tpc - 1) / (uint64_t)tpc;
  for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const SubRef sr = make_subref(g, tile * (uint64_t)tpc + (uint64_t)sub);
    PlanEngine::run<LD_CG, INV, INV ? EPI_SCALE : EPI_MUL>(m, map, kEngThreads, sr, sub, lane, smem, mp, layout,
                                      use_ep ? &ep : nullptr);
    __syncthreads();  // shared memory is reused by the next tile
  }
}

// N = 2 or 4: one thread per transform, stages in reverse order, then N^-1.
__global__ void __launch_bounds__(256)
    k_ntt_inv_tiny(uint4* x, const uint4* y, const uint4* tw, uint64_t count, int n, ModParams mp,
                   int layout, U128 scale) {
  const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (t >= count) return;
  const int N = 1 << n;
  U128 v[4];
  for (int i = 0; i < N; ++i) v[i] = from_mem(__ldcg(y + t * N + i), layout);
  for (int s = n - 1; s >= 0; --s) {
    const int half = N >> (s + 1);
    for (int i = 0; i < N; ++i) {
      if (i & half) continue;
      const uint4 tv = __ldg(tw + (1 << s) + (i >> (n - s)));
      gs_butterfly<ArithFast>(v[i], v[i + half], U128{{tv.x, tv.y, tv.z, tv.w}}, mp);
    }
  }
  // the second half already carries N^-1 through table entry 1
  for (int i = 0; i < N; ++i) x[t * N + i] = to_mem(i < N / 2 ? ArithFast::mul(v[i], scale, mp) : v[i], layout);
}

// One HBM pass of the inverse on the compile-time tile (NttTile::run_inv, 4
// elements per thread, 256-thread CTAs of 256 / 2^(M-2) sub-transforms, 4
// resident per SM), persistent over the tiles like the forward k_ntt_sub:
// whole transforms of 2^3..2^10 points (contiguous), or one pass of a larger
// transform (interleaved for the strided passes).  `finishing` marks the
// pass that ends the transform (stage 0 inside it), which applies N^-1 from
// entry 0 of the inverse table.
template <int M, int MAP>
__global__ void __launch_bounds__(256, 4)
    k_ntt_tile_inv(SubGeom g, ModParams mp, int layout, int finishing) {
  constexpr int TPC = 256 >> (M - 2);
  using T = NttTile<M, 2, TPC, MAP, ArithFast>;
  static_assert(T::THREADS == 256, "tile shape");
  extern __shared__ uint4 smem[];
  const int sub = T::sub_of(threadIdx.x), lane = T::lane_of(threadIdx.x);
  const uint64_t ntiles = (g.nsub + TPC - 1) / TPC;
  const uint4* scale_at = finishing ? g.tw : nullptr;
  for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const SubRef sr = make_subref(g, tile * TPC + (uint64_t)sub);
    if (layout == LAYOUT_HILO) T::template run_inv<LD_NC>(sr, sub, lane, smem, mp, LAYOUT_HILO, scale_at);
    else T::template run_inv<LD_NC>(sr, sub, lane, smem, mp, LAYOUT_U128, scale_at);
    T::sync();  // smem is reused by the next tile
  }
}

template <int M, int MAP>
int launch_tile_inv(bntt_plan* p, const SubGeom& g, int finishing, cudaStream_t s) {
  constexpr int TPC = 256 >> (M - 2);
  using T = NttTile<M, 2, TPC, MAP, ArithFast>;
  constexpr size_t smem = (size_t)T::SMEM_SLOTS * 16;
  static std::atomic<int> cached{0};  // resident CTAs per SM; relaxed: same value from any thread
  int bps = cached.load(std::memory_order_relaxed);
  if (!bps) {
    BNTT_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, (const void*)k_ntt_tile_inv<M, MAP>, 256, smem));
    bps = std::max(1, bps);
    cached.store(bps, std::memory_order_relaxed);
  }
  const uint64_t ntiles = (g.nsub + TPC - 1) / TPC;
  const unsigned grid = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)bps * p->ctx->sms);
  k_ntt_tile_inv<M, MAP><<<grid, 256, smem, s>>>(g, p->mp, p->layout, finishing);
  BNTT_CK(cudaGetLastError());
  p->ctx->launches++;
  return BNTT_OK;
}

// One pass of m stages (a whole transform of 2^3..2^10 points, a strided
// pass of 5..7 or a contiguous last pass of a larger one); EINVAL for a shape
// without a tile kernel.
int tile_inv_pass(bntt_plan* p, const SubGeom& g, int finishing, cudaStream_t s) {
  if (g.l > 0) {
    switch (g.m) {
      case 5: return launch_tile_inv<5, MAP_INTERLEAVED>(p, g, finishing, s);
      case 6: return launch_tile_inv<6, MAP_INTERLEAVED>(p, g, finishing, s);
      case 7: return launch_tile_inv<7, MAP_INTERLEAVED>(p, g, finishing, s);
      default: break;
    }
  } else {
    switch (g.m) {
      case 3: return launch_tile_inv<3, MAP_CONTIG>(p, g, finishing, s);
      case 4: return launch_tile_inv<4, MAP_CONTIG>(p, g, finishing, s);
      case 5: return launch_tile_inv<5, MAP_CONTIG>(p, g, finishing, s);
      case 6: return launch_tile_inv<6, MAP_CONTIG>(p, g, finishing, s);
      case 7: return launch_tile_inv<7, MAP_CONTIG>(p, g, finishing, s);
      case 8: return launch_tile_inv<8, MAP_CONTIG>(p, g, finishing, s);
      case 9: return launch_tile_inv<9, MAP_CONTIG>(p, g, finishing, s);
      case 10: return launch_tile_inv<10, MAP_CONTIG>(p, g, finishing, s);
      default: break;
    }
  }
  return set_error(BNTT_EINVAL, "no inverse tile for a pass of %u stages", g.m);
}

template <bool INV>
int engine_blocks_per_sm(size_t smem) {
  static std::atomic<int> cached[2];  // per smem class; relaxed: same value from any thread
  const int slot = smem > 0 ? 1 : 0;
  if (const int c = cached[slot].load(std::memory_order_relaxed)) return c;
  int b = 0;
  const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &b, (const void*)k_ntt_engine<INV>, kEngThreads, smem);
  if (e != cudaSuccess) return -cuda_error(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  cached[slot].store(std::max(1, b), std::memory_order_relaxed);
  return std::max(1, b);
}

// The HBM passes of a 2^n transform (n >= 3) on the engine: forward in pass
// order, inverse in reverse order.  The first pass run reads `in`, every
// pass writes `out` (in place after the first), and the last pass run
// applies `ep` when use_ep is set.
template <bool INV>
int engine_passes(bntt_plan* p, void* out, const void* in, size_t batch, const void* tw,
                  const Epilogue& ep, int use_ep, cudaStream_t s) {
  const int n = (int)p->log2n;
  const std::vector<int> passes = n <= 10 ? std::vector<int>{n} : engine_split(n);
  const int np = (int)passes.size();
  std::vector<int> starts(np, 0);
  for (int i = 1; i < np; ++i) starts[i] = starts[i - 1] + passes[i - 1];
  for (int k = 0; k < np; ++k) {
    const int i = INV ? np - 1 - k : k;
    const int m = passes[i];
    SubGeom g;
    g.x = static_cast<const uint4*>(k == 0 ? in : out);
    g.y = static_cast<uint4*>(out);
    g.tw = static_cast<const uint4*>(tw);
    g.n = (uint32_t)n;
    g.s0 = (uint32_t)starts[i];
    g.m = (uint32_t)m;
    g.l = (uint32_t)(n - starts[i] - m);
    g.nsub = (uint64_t)batch << (n - m);
    const int map = g.l > 0 ? MAP_INTERLEAVED : MAP_CONTIG;
    const size_t smem = PlanEngine::smem_slots(m, map, kEngThreads) * 16;
    const int bps = engine_blocks_per_sm<INV>(smem);
    if (bps < 0) return -bps;
    const int tpc = kEngThreads >> (m - 3);
    const uint64_t ntiles = (g.nsub + (uint64_t)tpc - 1) / (uint64_t)tpc;
    const unsigned grid = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)bps * p->ctx->sms);
    k_ntt_engine<INV><<<grid, kEngThreads, smem, s>>>(g, p->mp, p->layout, m, map, ep,
                                                      (k == np - 1 && use_ep) ? 1 : 0);
    BNTT_CK(cudaGetLastError());
    p->ctx->launches++;
  }
  return BNTT_OK;
}

// Inverse table (T[k]^-1, limb order) and N^-1, built once per plan: the
// forward table comes back from the device and is inverted on the host with
// one modular exponentiation and three multiplies per entry (batch
// inversion).  Entry 0, which no network stage reads, holds N^-1 (the
// inverse batch kernel takes each job's scale from its own table), and
// entry 1 holds T[1]^-1 * N^-1: every inverse kernel then scales only the
// first half of its outputs (the x outputs of the last stage).
static u128 entry_of(const std::vector<uint32_t>& t, size_t k) {
  u128 v = 0;
  for (int l = 3; l >= 0; --l) v = (v << 32) | t[4 * k + l];
  return v;
}

int ensure_inverse(bntt_plan* p) {
  if (p->tw_inv) return BNTT_OK;
  const u128 q = to_u128(p->mod.q), mu = to_u128(p->mod.mu);
  const size_t n = (size_t)1 << p->log2n;
  std::vector<uint32_t> t(4 * n);
  // copies on the context's stream (ordered after any work that wrote the
  // table, and finished before the first inverse launch reads the result)
  BNTT_CK(cudaMemcpyAsync(t.data(), p->tw, n * 16, cudaMemcpyDeviceToHost, p->ctx->stream));
  BNTT_CK(cudaStreamSynchronize(p->ctx->stream));
  auto entry = [&](size_t k) {
    u128 v = 0;
    for (int l = 3; l >= 0; --l) v = (v << 32) | t[4 * k + l];
    return v;
  };
  // prefix products, one inverse, then walk back
  std::vector<u128> pre(n, 1);
  u128 acc = 1;
  for (size_t k = 1; k < n; ++k) {
    const u128 e = entry(k);
    BNTT_REQUIRE(e != 0 && e < q, "twiddle %zu is 0 mod q (or not a residue): no inverse", k);
    pre[k] = acc;
    acc = host_mulmod(acc, e, q, mu);
  }
  u128 inv = host_powmod(acc, q - 2, q, mu);
  BNTT_REQUIRE(host_mulmod(inv, acc, q, mu) == 1,
               "the product of the twiddles has no inverse mod q (q is not prime)");
  std::vector<uint32_t> ti(4 * n, 0);
  for (size_t k = n - 1; k >= 1; --k) {
    const u128 ik = host_mulmod(inv, pre[k], q, mu);  // = T[k]^-1
    inv = host_mulmod(inv, entry(k), q, mu);
    for (int l = 0; l < 4; ++l) ti[4 * k + l] = (uint32_t)(ik >> (32 * l));
  }
  const u128 ninv = host_powmod((u128)n % q, q - 2, q, mu);
  BNTT_REQUIRE(host_mulmod(ninv, (u128)n % q, q, mu) == 1, "N has no inverse mod q");
  for (int l = 0; l < 4; ++l) ti[l] = (uint32_t)(ninv >> (32 * l));
  // entry 1 (the last inverse stage, which ends in y = (x - y) * T[1]^-1)
  // carries N^-1 too, so the final scaling multiplies the x half only
  const u128 t1 = host_mulmod(entry_of(ti, 1), ninv, q, mu);
  for (int l = 0; l < 4; ++l) ti[4 + l] = (uint32_t)(t1 >> (32 * l));
  void* d = nullptr;
  if (int rc = ctx_alloc(p->ctx, &d, n * 16)) return rc;
  cudaError_t e = cudaMemcpyAsync(d, ti.data(), n * 16, cudaMemcpyHostToDevice, p->ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(p->ctx->stream);
  if (e != cudaSuccess) {
    ctx_free(p->ctx, d);
    return cuda_error(e, "copy of the inverse twiddles");
  }
  p->tw_inv = d;
  p->ninv = to_limbs(ninv);
  return BNTT_OK;
}

int inverse_on(bntt_plan* p, void* x, const void* y, size_t batch, cudaStream_t s) {
  const int n = (int)p->log2n;
  if (n <= 2) {
    const unsigned grid = (unsigned)((batch + 255) / 256);
    k_ntt_inv_tiny<<<grid, 256, 0, s>>>(static_cast<uint4*>(x), static_cast<const uint4*>(y),
                                        static_cast<const uint4*>(p->tw_inv), (uint64_t)batch, n,
                                        p->mp, p->layout, p->ninv);
    BNTT_CK(cudaGetLastError());
    p->ctx->launches++;
    return BNTT_OK;
  }
  // up to 2^10 points one tile pass; above, the persistent kernel's split
  // (strided passes of 5..7 stages, then a contiguous one), run last pass
  // first, the first run reading y and every run writing x
  const std::vector<int> split = n <= 10 ? std::vector<int>{n} : tile_split(n);
  if (!split.empty()) {
    const int np = (int)split.size();
    std::vector<int> starts(np, 0);
    for (int i = 1; i < np; ++i) starts[i] = starts[i - 1] + split[i - 1];
    for (int k = 0; k < np; ++k) {
      const int i = np - 1 - k;
      SubGeom g;
      g.x = static_cast<const uint4*>(k == 0 ? y : x);
      g.y = static_cast<uint4*>(x);
      g.tw = static_cast<const uint4*>(p->tw_inv);
      g.n = (uint32_t)n;
      g.s0 = (uint32_t)starts[i];
      g.m = (uint32_t)split[i];
      g.l = (uint32_t)(n - starts[i] - split[i]);
      g.nsub = (uint64_t)batch << (n - split[i]);
      if (int rc = tile_inv_pass(p, g, i == 0 ? 1 : 0, s)) return rc;
    }
    return BNTT_OK;
  }
  Epilogue ep;
  ep.scale = p->ninv;
  ep.has_scale = 1;
  return engine_passes<true>(p, x, y, batch, p->tw_inv, ep, 1, s);
}

}  // namespace

int plan_ensure_inverse(bntt_plan* p) {
  if (!p->fast) return set_error(BNTT_EINVAL, "the inverse transform needs q = 2^124 - k (k < 2^28), mu = floor(2^251/q)");
  return ensure_inverse(p);
}

// Forward transform of a plan on the engine (fast multiply, n >= 3), with
// the optional fused pointwise product of MulB on the last pass.
int engine_forward_on(bntt_plan* p, void* y, const void* x, size_t batch, cudaStream_t s,
                      const void* b, uint64_t bmask) {
  Epilogue ep;
  ep.mul.b = static_cast<const uint4*>(b);
  ep.mul.ybase = static_cast<const uint4*>(y);
  ep.mul.bmask = bmask;
  return engine_passes<false>(p, y, x, batch, p->tw, ep, b ? 1 : 0, s);
}

}  // namespace bntt

using namespace bntt;

extern "C" int bntt_ntt_inverse_dev(bntt_plan* p, void* x, const void* y, size_t batch) {
  BNTT_REQUIRE(p, "plan is NULL");
  if (batch == 0) return BNTT_OK;
  BNTT_REQUIRE(x && y, "NULL buffer");
  BNTT_REQUIRE(((uintptr_t)x & 15) == 0 && ((uintptr_t)y & 15) == 0,
               "device buffers must be 16-byte aligned");
  BNTT_REQUIRE(p->fast, "the inverse transform needs q = 2^124 - k (k < 2^28), mu = floor(2^251/q)");
  if (int rc = ctx_use_device(p->ctx)) return rc;
  if (int rc = ensure_inverse(p)) return rc;
  return inverse_on(p, x, y, batch, p->ctx->stream);
}
