// runtime.cu -- context, allocator, modulus analysis, plans and the NTT / BLAS
// entry points of the C ABI (include/bntt.h).
#include <algorithm>
#include <cstdio>
#include <cstring>

#include "internal.h"

using bntt::u128;

namespace bntt {

// ------------------------------------------------------------------ errors
static thread_local char g_last_error[512] = "";

int set_error(int status, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return status;
}

int cuda_error(cudaError_t e, const char* what) {
  cudaGetLastError();  // clear a sticky launch error so the context stays usable
  if (e == cudaErrorMemoryAllocation)
    return set_error(BNTT_ENOMEM, "%s: %s", what, cudaGetErrorString(e));
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
    return set_error(BNTT_ENODEV, "%s: %s", what, cudaGetErrorString(e));
  return set_error(BNTT_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

// ----------------------------------------------------------------- modulus
u128 barrett_mu(u128 q) {
  // floor(2^251 / q): shift 2^251 in bit by bit; q > 2^123 keeps the
  // remainder below 2^124 and the quotient below 2^128.
  u128 r = 0, quo = 0;
  for (int bit = 251; bit >= 0; --bit) {
    r = (r << 1) | (bit == 251 ? 1 : 0);
    quo <<= 1;
    if (r >= q) {
      r -= q;
      quo |= 1;
    }
  }
  return quo;
}

// The pseudo-Mersenne multiply equals the reference mulmod128 when
//   2^123 < q = 2^124 - k,  1 <= k < 2^28,  mu = floor(2^251 / q):
// for operands below 2^124 the reference's intermediate sums cannot wrap
// (mu = 2^127 + d with d < 2^35, so its mulhi128 cross terms stay below
// 2^128), and its quotient estimate is floor(P/q) or one less (the two
// truncations lose less than 2^122/q + P/2^251 < 1/2 + 1/8), so one
// conditional subtraction returns P mod q.  (The reference's exactness holds
// up to k < 2^31; the device multiply folds at 2^128 with the factor 16k,
// which must fit in 32 bits.)
bool modulus_fast(u128 q, u128 mu, uint32_t* k_out) {
  const u128 top = (u128)1 << 124;
  if (q >= top || q <= ((u128)1 << 123)) return false;
  const u128 k = top - q;
  if (k >= ((u128)1 << 28)) return false;
  if (mu != barrett_mu(q)) return false;
  if (k_out) *k_out = (uint32_t)k;
  return true;
}

ModParams make_params(const bntt_modulus& m, bool* fast_out) {
  ModParams p{};
  const u128 q = to_u128(m.q), mu = to_u128(m.mu);
  p.q = to_limbs(q);
  p.mu = to_limbs(mu);
  uint32_t k = 0;
  const bool f = modulus_fast(q, mu, &k);
  p.k = k;
  if (fast_out) *fast_out = f;
  return p;
}

// --------------------------------------------------------------- context
int ctx_use_device(bntt_ctx* ctx) {
  BNTT_CK(cudaSetDevice(ctx->device));
  return BNTT_OK;
}

bool arith_fast(bntt_ctx* ctx, bool modulus_is_fast) {
  return modulus_is_fast && ctx->arith == BNTT_ARITH_AUTO;
}

int ctx_alloc(bntt_ctx* ctx, void** p, size_t bytes) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (ctx->budget && ctx->in_use + bytes > ctx->budget)
    return set_error(BNTT_EBUDGET, "allocation of %zu bytes exceeds the HBM budget (%zu of %zu in use)",
                     bytes, ctx->in_use, ctx->budget);
  void* d = nullptr;
  cudaError_t e = cudaMalloc(&d, bytes ? bytes : 16);
  if (e != cudaSuccess) return cuda_error(e, "cudaMalloc");
  ctx->allocs[d] = bytes;
  ctx->in_use += bytes;
  *p = d;
  return BNTT_OK;
}

int ctx_free(bntt_ctx* ctx, void* p) {
  if (!p) return BNTT_OK;
  std::lock_guard<std::mutex> g(ctx->mu);
  auto it = ctx->allocs.find(p);
  if (it == ctx->allocs.end()) return set_error(BNTT_EINVAL, "pointer %p was not allocated by this context", p);
  ctx->in_use -= it->second;
  ctx->allocs.erase(it);
  BNTT_CK(cudaFree(p));
  return BNTT_OK;
}

}  // namespace bntt

using namespace bntt;

// =================================================================== C ABI
extern "C" {

const char* bntt_version(void) { return "bntt 0.1 (sm_100a)"; }
const char* bntt_last_error(void) { return g_last_error; }

const char* bntt_status_string(int s) {
  switch (s) {
    case BNTT_OK: return "ok";
    case BNTT_EINVAL: return "invalid argument";
    case BNTT_ENOMEM: return "out of memory";
    case BNTT_EBUDGET: return "HBM budget exceeded";
    case BNTT_ECUDA: return "CUDA error";
    case BNTT_ETIMEOUT: return "device wait timed out";
    case BNTT_ENODEV: return "no CUDA device";
    case BNTT_EBUSY: return "busy";
    default: return "unknown status";
  }
}

int bntt_modulus_is_fast(const bntt_modulus* m) {
  if (!m) return 0;
  return modulus_fast(to_u128(m->q), to_u128(m->mu), nullptr) ? 1 : 0;
}

bntt_modulus bntt_modulus_ntt_reference(void) {
  // src/ntt_scalar.c:632-633
  return bntt_modulus{{1152921504606846975ull, 18446744073709550897ull},
                      {9223372036854775808ull, 5752ull}};
}

bntt_modulus bntt_modulus_blas_reference(void) {
  // src/blas_scalar.c:23-30
  return bntt_modulus{{0x0FFFFFFFFFFFFFFFull, 0xFFFFFFFFFFFFFFC5ull},
                      {0x8000000000000000ull, 0x1D8ull}};
}

int bntt_ctx_create(bntt_ctx** out, int device, void* stream) {
  BNTT_REQUIRE(out, "ctx output pointer is NULL");
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(BNTT_ENODEV, "no CUDA device (%s)", cudaGetErrorString(e));
  }
  BNTT_REQUIRE(device >= 0 && device < ndev, "device %d out of range (%d devices)", device, ndev);
  BNTT_CK(cudaSetDevice(device));
  cudaDeviceProp prop;
  BNTT_CK(cudaGetDeviceProperties(&prop, device));
  auto* c = new bntt_ctx();
  c->device = device;
  c->sms = prop.multiProcessorCount;
  if (stream) {
    c->stream = static_cast<cudaStream_t>(stream);
  } else {
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      delete c;
      return cuda_error(e, "cudaStreamCreate");
    }
    c->own_stream = true;
  }
  for (auto& s : c->copy_stream) cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  for (auto& ev : c->ev) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  *out = c;
  return BNTT_OK;
}

int bntt_ctx_destroy(bntt_ctx* c) {
  if (!c) return BNTT_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (auto& kv : c->allocs) cudaFree(kv.first);
  for (auto& s : c->copy_stream)
    if (s) cudaStreamDestroy(s);
  for (auto& ev : c->ev)
    if (ev) cudaEventDestroy(ev);
  if (c->pinned) cudaFreeHost(c->pinned);
  if (c->own_stream) cudaStreamDestroy(c->stream);
  delete c;
  return BNTT_OK;
}

int bntt_ctx_synchronize(bntt_ctx* c) {
  BNTT_REQUIRE(c, "ctx is NULL");
  if (int rc = ctx_use_device(c)) return rc;
  BNTT_CK(cudaStreamSynchronize(c->stream));
  return BNTT_OK;
}

void* bntt_ctx_stream(bntt_ctx* c) { return c ? (void*)c->stream : nullptr; }

int bntt_ctx_set_arith(bntt_ctx* c, int arith) {
  BNTT_REQUIRE(c, "ctx is NULL");
  BNTT_REQUIRE(arith == BNTT_ARITH_AUTO || arith == BNTT_ARITH_REFERENCE, "unknown arith %d", arith);
  c->arith = arith;
  return BNTT_OK;
}

int bntt_ctx_set_hbm_budget(bntt_ctx* c, size_t bytes) {
  BNTT_REQUIRE(c, "ctx is NULL");
  c->budget = bytes;
  return BNTT_OK;
}

size_t bntt_ctx_hbm_in_use(bntt_ctx* c) { return c ? c->in_use : 0; }
int bntt_ctx_sm_count(bntt_ctx* c) { return c ? c->sms : 0; }
uint64_t bntt_ctx_launch_count(bntt_ctx* c) { return c ? c->launches : 0; }

int bntt_dev_alloc(bntt_ctx* c, void** p, size_t bytes) {
  BNTT_REQUIRE(c && p, "NULL argument");
  if (int rc = ctx_use_device(c)) return rc;
  return ctx_alloc(c, p, bytes);
}

int bntt_dev_free(bntt_ctx* c, void* p) {
  BNTT_REQUIRE(c, "ctx is NULL");
  if (int rc = ctx_use_device(c)) return rc;
  return ctx_free(c, p);
}

int bntt_copy_h2d(bntt_ctx* c, void* dst, const void* src, size_t bytes) {
  BNTT_REQUIRE(c && (bytes == 0 || (dst && src)), "NULL argument");
  if (int rc = ctx_use_device(c)) return rc;
  BNTT_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
  BNTT_CK(cudaStreamSynchronize(c->stream));
  return BNTT_OK;
}

int bntt_copy_d2h(bntt_ctx* c, void* dst, const void* src, size_t bytes) {
  BNTT_REQUIRE(c && (bytes == 0 || (dst && src)), "NULL argument");
  if (int rc = ctx_use_device(c)) return rc;
  BNTT_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
  BNTT_CK(cudaStreamSynchronize(c->stream));
  return BNTT_OK;
}

}  // extern "C"

// ------------------------------------------------------------- generator
namespace bntt {

__host__ __device__ __forceinline__ uint64_t splitmix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Element i: high word from counter 2i+1, low word from 2i+2 (0x9E37...
// increments), masked to bitlen(q) bits, q subtracted once if still >= q.
__host__ __device__ __forceinline__ void uniform_at(uint64_t seed, uint64_t idx, uint64_t qh,
                                                    uint64_t ql, int qbits, uint64_t* h,
                                                    uint64_t* l) {
  const uint64_t G = 0x9E3779B97F4A7C15ull;
  uint64_t hh = splitmix(seed + (2 * idx + 1) * G);
  uint64_t ll = splitmix(seed + (2 * idx + 2) * G);
  if (qbits <= 64) {
    hh = 0;
    if (qbits < 64) ll &= (1ull << qbits) - 1;
  } else if (qbits < 128) {
    hh &= (1ull << (qbits - 64)) - 1;
  }
  if (hh > qh || (hh == qh && ll >= ql)) {
    const uint64_t b = ll < ql ? 1 : 0;
    ll -= ql;
    hh = hh - qh - b;
  }
  *h = hh;
  *l = ll;
}

static int bitlen(u128 q) {
  int b = 0;
  while (q) {
    ++b;
    q >>= 1;
  }
  return b;
}

__global__ void k_fill_uniform(uint64_t* buf, size_t count, uint64_t seed, uint64_t offset,
                               uint64_t qh, uint64_t ql, int qbits, int layout) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count;
       i += (size_t)gridDim.x * blockDim.x) {
    uint64_t h, l;
    uniform_at(seed, offset + i, qh, ql, qbits, &h, &l);
    if (layout == LAYOUT_HILO) {
      buf[2 * i] = h;
      buf[2 * i + 1] = l;
    } else {
      buf[2 * i] = l;
      buf[2 * i + 1] = h;
    }
  }
}

int launch_fill(bntt_ctx* ctx, void* buf, size_t count, uint64_t seed, uint64_t offset, u128 q,
                int layout, cudaStream_t stream) {
  if (!count) return BNTT_OK;
  const unsigned grid = (unsigned)std::min<size_t>((count + 255) / 256, (size_t)ctx->sms * 16);
  k_fill_uniform<<<grid, 256, 0, stream>>>(static_cast<uint64_t*>(buf), count, seed, offset,
                                          (uint64_t)(q >> 64), (uint64_t)q, bitlen(q), layout);
  BNTT_CK(cudaGetLastError());
  ctx->launches++;
  return BNTT_OK;
}

// Fields shared by every plan constructor; the table is set by the caller.
int plan_create_common(bntt_ctx* c, bntt_plan** out, unsigned log2n, const bntt_modulus* m,
                       int layout) {
  BNTT_REQUIRE(c && out && m, "NULL argument");
  *out = nullptr;
  BNTT_REQUIRE(log2n >= 1 && log2n <= 24, "log2n %u outside [1, 24]", log2n);
  BNTT_REQUIRE(layout == BNTT_LAYOUT_HILO || layout == BNTT_LAYOUT_U128, "bad layout %d", layout);
  if (int rc = ctx_use_device(c)) return rc;
  auto* p = new bntt_plan();
  p->ctx = c;
  p->log2n = log2n;
  p->mod = *m;
  p->layout = layout;
  p->mp = make_params(*m, &p->fast);
  *out = p;
  return BNTT_OK;
}

}  // namespace bntt

extern "C" {

int bntt_fill_uniform_host(void* buf, size_t count, uint64_t seed, uint64_t offset,
                           const bntt_modulus* m, int layout) {
  BNTT_REQUIRE(m && (buf || count == 0), "NULL argument");
  BNTT_REQUIRE(layout == BNTT_LAYOUT_HILO || layout == BNTT_LAYOUT_U128, "bad layout %d", layout);
  const u128 q = to_u128(m->q);
  BNTT_REQUIRE(q >= 2, "modulus must be >= 2");
  const int qb = bitlen(q);
  uint64_t* p = static_cast<uint64_t*>(buf);
  for (size_t i = 0; i < count; ++i) {
    uint64_t h, l;
    uniform_at(seed, offset + i, m->q.hi, m->q.lo, qb, &h, &l);
    p[2 * i] = layout == BNTT_LAYOUT_HILO ? h : l;
    p[2 * i + 1] = layout == BNTT_LAYOUT_HILO ? l : h;
  }
  return BNTT_OK;
}

int bntt_fill_uniform_dev(bntt_ctx* c, void* buf, size_t count, uint64_t seed, uint64_t offset,
                          const bntt_modulus* m, int layout) {
  BNTT_REQUIRE(c && m && (buf || count == 0), "NULL argument");
  BNTT_REQUIRE(layout == BNTT_LAYOUT_HILO || layout == BNTT_LAYOUT_U128, "bad layout %d", layout);
  BNTT_REQUIRE(to_u128(m->q) >= 2, "modulus must be >= 2");
  if (int rc = ctx_use_device(c)) return rc;
  return launch_fill(c, buf, count, seed, offset, to_u128(m->q), layout, c->stream);
}

// -------------------------------------------------------------------- NTT

// Plans keep their table in limb order (LAYOUT_U128: the kernels' register
// order), whatever the caller's layout, so no kernel reorders twiddle words.
int bntt_plan_create(bntt_ctx* c, bntt_plan** out, unsigned log2n, const bntt_modulus* m,
                     const void* twiddles, int layout) {
  BNTT_REQUIRE(twiddles, "twiddles is NULL");
  int rc = bntt::plan_create_common(c, out, log2n, m, layout);
  if (rc) return rc;
  bntt_plan* p = *out;
  const size_t n = (size_t)1 << log2n, bytes = n * 16;
  if ((rc = ctx_alloc(c, &p->tw, bytes)) != 0) {
    delete p;
    *out = nullptr;
    return rc;
  }
  p->own_tw = true;
  cudaError_t e;
  if (layout == BNTT_LAYOUT_HILO) {
    std::vector<uint64_t> t(2 * n);
    const uint64_t* src = static_cast<const uint64_t*>(twiddles);
    for (size_t i = 0; i < n; ++i) {
      t[2 * i] = src[2 * i + 1];
      t[2 * i + 1] = src[2 * i];
    }
    e = cudaMemcpyAsync(p->tw, t.data(), bytes, cudaMemcpyHostToDevice, c->stream);
  } else {
    e = cudaMemcpyAsync(p->tw, twiddles, bytes, cudaMemcpyHostToDevice, c->stream);
  }
  // on the context's (non-blocking) stream and complete before the plan is
  // used: a plain cudaMemcpy from pageable memory may return before its DMA
  // lands, and the default stream does not order it with that stream
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) rc = plan_choose_kernels(p);
  else rc = cuda_error(e, "copy of the twiddle table");
  if (rc) {
    ctx_free(c, p->tw);
    delete p;
    *out = nullptr;
  }
  return rc;
}

// With a device table in U128 layout the plan uses it in place; a HILO table
// is copied once into a plan-owned buffer with its two words swapped.
int bntt_plan_create_dev(bntt_ctx* c, bntt_plan** out, unsigned log2n, const bntt_modulus* m,
                         const void* twiddles_dev, int layout) {
  BNTT_REQUIRE(twiddles_dev && ((uintptr_t)twiddles_dev & 15) == 0,
               "twiddles_dev must be a 16-byte aligned device pointer");
  int rc = bntt::plan_create_common(c, out, log2n, m, layout);
  if (rc) return rc;
  bntt_plan* p = *out;
  if (layout == BNTT_LAYOUT_U128) {
    p->tw = const_cast<void*>(twiddles_dev);
  } else {
    const size_t n = (size_t)1 << log2n;
    if ((rc = ctx_alloc(c, &p->tw, n * 16)) != 0) {
      delete p;
      *out = nullptr;
      return rc;
    }
    p->own_tw = true;
    char* d = static_cast<char*>(p->tw);
    const char* s = static_cast<const char*>(twiddles_dev);
    // on the context's stream, finished before the plan is used
    cudaError_t e = cudaMemcpy2DAsync(d, 16, s + 8, 16, 8, n, cudaMemcpyDeviceToDevice, c->stream);
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync(d + 8, 16, s, 16, 8, n, cudaMemcpyDeviceToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
      rc = cuda_error(e, "copy of the twiddle table");
      ctx_free(c, p->tw);
      delete p;
      *out = nullptr;
      return rc;
    }
  }
  if ((rc = plan_choose_kernels(p)) != 0) {
    if (p->own_tw) ctx_free(c, p->tw);
    delete p;
    *out = nullptr;
  }
  return rc;
}

int bntt_plan_destroy(bntt_plan* p) {
  if (!p) return BNTT_OK;
  if (p->own_tw && p->tw) {
    ctx_use_device(p->ctx);
    ctx_free(p->ctx, p->tw);
  }
  if (p->tw_inv) {
    ctx_use_device(p->ctx);
    ctx_free(p->ctx, p->tw_inv);
  }
  delete p;
  return BNTT_OK;
}

unsigned bntt_plan_log2n(const bntt_plan* p) { return p ? p->log2n : 0; }

static bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

int bntt_ntt_forward_dev(bntt_plan* p, void* y, const void* x, size_t batch) {
  BNTT_REQUIRE(p, "plan is NULL");
  if (batch == 0) return BNTT_OK;
  BNTT_REQUIRE(x && y, "NULL buffer");
  BNTT_REQUIRE(aligned16(x) && aligned16(y), "device buffers must be 16-byte aligned");
  if (int rc = ctx_use_device(p->ctx)) return rc;
  return ntt_forward_on(p, y, x, batch, p->ctx->stream);
}

int bntt_ntt_forward_mul_dev(bntt_plan* p, void* y, const void* x, const void* b,
                             int b_per_transform, size_t batch) {
  BNTT_REQUIRE(p, "plan is NULL");
  if (batch == 0) return BNTT_OK;
  BNTT_REQUIRE(x && y && b, "NULL buffer");
  BNTT_REQUIRE(aligned16(x) && aligned16(y) && aligned16(b),
               "device buffers must be 16-byte aligned");
  BNTT_REQUIRE(b_per_transform == 0 || b_per_transform == 1, "b_per_transform must be 0 or 1");
  const size_t n = (size_t)1 << p->log2n;
  const uintptr_t y0 = (uintptr_t)y, y1 = y0 + batch * n * 16;
  const uintptr_t b0 = (uintptr_t)b, b1 = b0 + (b_per_transform ? batch : 1) * n * 16;
  BNTT_REQUIRE(b1 <= y0 || b0 >= y1, "b must not overlap y");
  if (int rc = ctx_use_device(p->ctx)) return rc;
  return ntt_forward_on(p, y, x, batch, p->ctx->stream, b,
                        b_per_transform ? ~0ull : (uint64_t)(n - 1));
}

}  // extern "C"

// ------------------------------------------------- host-pointer pipelines
namespace bntt {

// Device staging for host-pointer calls: kSlots slots, each big enough for
// one chunk of every operand, charged to the budget and kept for reuse.
static constexpr int kSlots = 3;
static constexpr size_t kChunkBytes = 32ull << 20;

static int staging(bntt_ctx* c, size_t bytes, void** out) {
  if (c->stage_bytes < bytes) {
    if (c->stage) ctx_free(c, c->stage);
    c->stage = nullptr;
    c->stage_bytes = 0;
    if (int rc = ctx_alloc(c, &c->stage, bytes)) return rc;
    c->stage_bytes = bytes;
  }
  *out = c->stage;
  return BNTT_OK;
}

// Runs `chunks` pieces through kSlots streams: copy in, compute, copy out.
// Piece i uses slot i % kSlots; consecutive pieces overlap their transfers
// with each other's compute.
template <class In, class Run, class Out>
static int pipeline(bntt_ctx* c, size_t chunks, In in, Run run, Out out) {
  cudaStream_t st[kSlots] = {c->stream, c->copy_stream[0], c->copy_stream[1]};
  // all slots start after work already queued on the context stream
  BNTT_CK(cudaEventRecord(c->ev[0], c->stream));
  for (int s = 1; s < kSlots; ++s) BNTT_CK(cudaStreamWaitEvent(st[s], c->ev[0], 0));
  for (size_t i = 0; i < chunks; ++i) {
    cudaStream_t s = st[i % kSlots];
    int rc;
    if ((rc = in(i, (int)(i % kSlots), s)) != 0) return rc;
    if ((rc = run(i, (int)(i % kSlots), s)) != 0) return rc;
    if ((rc = out(i, (int)(i % kSlots), s)) != 0) return rc;
  }
  for (int s = 0; s < kSlots; ++s) BNTT_CK(cudaStreamSynchronize(st[s]));
  return BNTT_OK;
}

}  // namespace bntt

extern "C" int bntt_ntt_forward_host(bntt_plan* p, void* y, const void* x, size_t batch) {
  BNTT_REQUIRE(p, "plan is NULL");
  if (batch == 0) return BNTT_OK;
  BNTT_REQUIRE(x && y, "NULL buffer");
  bntt_ctx* c = p->ctx;
  if (int rc = ctx_use_device(c)) return rc;
  const size_t tbytes = (size_t)16 << p->log2n;
  const size_t per = std::max<size_t>(1, kChunkBytes / tbytes);
  const size_t chunks = (batch + per - 1) / per;
  void* stage = nullptr;
  const size_t slot_bytes = std::min(per, batch) * tbytes;
  if (int rc = staging(c, slot_bytes * kSlots, &stage)) return rc;
  auto slot_ptr = [&](int s) { return static_cast<char*>(stage) + (size_t)s * slot_bytes; };
  auto count = [&](size_t i) { return std::min(per, batch - i * per); };
  return pipeline(
      c, chunks,
      [&](size_t i, int s, cudaStream_t st) -> int {
        BNTT_CK(cudaMemcpyAsync(slot_ptr(s), static_cast<const char*>(x) + i * per * tbytes,
                                count(i) * tbytes, cudaMemcpyHostToDevice, st));
        return BNTT_OK;
      },
      [&](size_t i, int s, cudaStream_t st) -> int {
        return ntt_forward_on(p, slot_ptr(s), slot_ptr(s), count(i), st);
      },
      [&](size_t i, int s, cudaStream_t st) -> int {
        BNTT_CK(cudaMemcpyAsync(static_cast<char*>(y) + i * per * tbytes, slot_ptr(s),
                                count(i) * tbytes, cudaMemcpyDeviceToHost, st));
        return BNTT_OK;
      });
}

// ------------------------------------------------------------------- BLAS
namespace bntt {

static int blas_dev(bntt_ctx* c, int op, void* cc, const void* a, const void* b, bntt_u128 x,
                    size_t len, const bntt_modulus* m, int layout) {
  BNTT_REQUIRE(c && m, "NULL argument");
  if (len == 0) return BNTT_OK;
  BNTT_REQUIRE(cc && a && b, "NULL buffer");
  BNTT_REQUIRE(((uintptr_t)cc | (uintptr_t)a | (uintptr_t)b) % 16 == 0,
               "device buffers must be 16-byte aligned");
  BNTT_REQUIRE(layout == BNTT_LAYOUT_HILO || layout == BNTT_LAYOUT_U128, "bad layout %d", layout);
  if (int rc = ctx_use_device(c)) return rc;
  bool fast = false;
  const ModParams mp = make_params(*m, &fast);
  return launch_blas(c, op, cc, a, b, to_limbs(to_u128(x)), len, mp, arith_fast(c, fast), layout,
                     c->stream);
}

static int blas_host(bntt_ctx* c, int op, void* cc, const void* a, const void* b, bntt_u128 x,
                     size_t len, const bntt_modulus* m, int layout) {
  BNTT_REQUIRE(c && m, "NULL argument");
  if (len == 0) return BNTT_OK;
  BNTT_REQUIRE(cc && a && b, "NULL buffer");
  BNTT_REQUIRE(layout == BNTT_LAYOUT_HILO || layout == BNTT_LAYOUT_U128, "bad layout %d", layout);
  if (int rc = ctx_use_device(c)) return rc;
  bool fast = false;
  const ModParams mp = make_params(*m, &fast);
  const U128 xl = to_limbs(to_u128(x));
  const bool f = arith_fast(c, fast);
  const size_t per = kChunkBytes / 16;
  const size_t chunks = (len + per - 1) / per;
  const size_t slot_elems = std::min(per, len);
  void* stage = nullptr;
  if (int rc = staging(c, slot_elems * 16 * 2 * kSlots, &stage)) return rc;
  auto A = [&](int s) { return static_cast<char*>(stage) + (size_t)s * 2 * slot_elems * 16; };
  auto B = [&](int s) { return A(s) + slot_elems * 16; };
  auto count = [&](size_t i) { return std::min(per, len - i * per); };
  return pipeline(
      c, chunks,
      [&](size_t i, int s, cudaStream_t st) -> int {
        BNTT_CK(cudaMemcpyAsync(A(s), static_cast<const char*>(a) + i * per * 16, count(i) * 16,
                                cudaMemcpyHostToDevice, st));
        BNTT_CK(cudaMemcpyAsync(B(s), static_cast<const char*>(b) + i * per * 16, count(i) * 16,
                                cudaMemcpyHostToDevice, st));
        return BNTT_OK;
      },
      [&](size_t i, int s, cudaStream_t st) -> int {
        return launch_blas(c, op, A(s), A(s), B(s), xl, count(i), mp, f, layout, st);
      },
      [&](size_t i, int s, cudaStream_t st) -> int {
        BNTT_CK(cudaMemcpyAsync(static_cast<char*>(cc) + i * per * 16, A(s), count(i) * 16,
                                cudaMemcpyDeviceToHost, st));
        return BNTT_OK;
      });
}

}  // namespace bntt

extern "C" {

int bntt_vvadd_dev(bntt_ctx* c, void* cc, const void* a, const void* b, size_t len,
                   const bntt_modulus* m, int layout) {
  return blas_dev(c, 0, cc, a, b, bntt_u128{0, 0}, len, m, layout);
}
int bntt_vvsub_dev(bntt_ctx* c, void* cc, const void* a, const void* b, size_t len,
                   const bntt_modulus* m, int layout) {
  return blas_dev(c, 1, cc, a, b, bntt_u128{0, 0}, len, m, layout);
}
int bntt_vvmul_dev(bntt_ctx* c, void* cc, const void* a, const void* b, size_t len,
                   const bntt_modulus* m, int layout) {
  return blas_dev(c, 2, cc, a, b, bntt_u128{0, 0}, len, m, layout);
}
int bntt_axpy_dev(bntt_ctx* c, void* cc, const void* a, const void* b, bntt_u128 x, size_t len,
                  const bntt_modulus* m, int layout) {
  return blas_dev(c, 3, cc, a, b, x, len, m, layout);
}
int bntt_vvadd_host(bntt_ctx* c, void* cc, const void* a, const void* b, size_t len,
                    const bntt_modulus* m, int layout) {
  return blas_host(c, 0, cc, a, b, bntt_u128{0, 0}, len, m, layout);
}
int bntt_vvsub_host(bntt_ctx* c, void* cc, const void* a, const void* b, size_t len,
                    const bntt_modulus* m, int layout) {
  return blas_host(c, 1, cc, a, b, bntt_u128{0, 0}, len, m, layout);
}
int bntt_vvmul_host(bntt_ctx* c, void* cc, const void* a, const void* b, size_t len,
                    const bntt_modulus* m, int layout) {
  return blas_host(c, 2, cc, a, b, bntt_u128{0, 0}, len, m, layout);
}
int bntt_axpy_host(bntt_ctx* c, void* cc, const void* a, const void* b, bntt_u128 x, size_t len,
                   const bntt_modulus* m, int layout) {
  return blas_host(c, 3, cc, a, b, x, len, m, layout);
}

}  // extern "C"
