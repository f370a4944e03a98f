// autotune.cu -- measured choice of kernel shapes per transform size.
//
// For every size the library has several compiled shapes: elements per thread
// (radix 8 or 16 register tiles, which also sets the number of shared-memory
// passes), transforms per CTA (CTA shape), register budgets (two or three
// resident CTAs per SM), inputs read from HBM by the first pass or staged
// into shared memory a tile ahead, and the twiddle table read through L1 or
// copied into shared memory per CTA (twiddle placement).  The tuner times each candidate on this device with
// seeded data larger than L2 and makes the fastest the default for plans and
// batches created afterwards in the process.  Choices can be written to and
// read from a small text file (keyed by device name and SM count).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "internal.h"
#include "ntt_core.cuh"

namespace bntt {

// choice tables: [m][map][fast] -> kernel; batch shapes per size
static std::mutex g_tune_mu;
static const SubKernel* g_sub_choice[11][2][2] = {};
static int g_batch_small_choice[11];
static bool g_batch_small_set[11] = {};

const SubKernel* tuned_sub_kernel(int m, int map, int fast, int l) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  if (m < 1 || m > 10) return nullptr;
  const SubKernel* k = g_sub_choice[m][map][fast];
  if (k && map == MAP_INTERLEAVED && (1 << l) < k->tpc) return nullptr;
  return k;
}

int tuned_batch_small_shape(int m) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  return (m >= 1 && m <= 10 && g_batch_small_set[m]) ? g_batch_small_choice[m] : -1;
}

int batch_shape_count();
int batch_shape_info(int s, int* m, int* logr, int* tpc, int* map);
int batch_time_uniform(bntt_ctx* c, bntt_plan* plan, int shape, size_t count, void* x, void* y,
                       float* ms);

static std::string device_key(bntt_ctx* c) {
  cudaDeviceProp p;
  cudaGetDeviceProperties(&p, c->device);
  char buf[320];
  snprintf(buf, sizeof(buf), "%s|sms=%d", p.name, p.multiProcessorCount);
  for (char* q = buf; *q; ++q)
    if (*q == ' ') *q = '_';
  return buf;
}

// time one kernel over a geometry: median of `reps` launches; with `flush`
// (a buffer larger than L2) the L2 is overwritten before each timed launch,
// so inputs that would fit in it come from HBM as in a first use
static int time_sub(bntt_ctx* c, const SubKernel* k, const SubGeom& g, const ModParams& mp, int reps,
                    float* out_ms, void* flush = nullptr, size_t flush_bytes = 0) {
  cudaEvent_t e0, e1;
  BNTT_CK(cudaEventCreate(&e0));
  BNTT_CK(cudaEventCreate(&e1));
  std::vector<float> t;
  int rc = BNTT_OK;
  for (int r = 0; r < reps + 1 && !rc; ++r) {
    if (flush) cudaMemsetAsync(flush, r & 0xff, flush_bytes, c->stream);
    cudaEventRecord(e0, c->stream);
    rc = launch_sub(c, k, &g, mp, BNTT_LAYOUT_HILO, c->stream);
    cudaEventRecord(e1, c->stream);
    if (!rc) {
      cudaError_t e = cudaEventSynchronize(e1);
      if (e != cudaSuccess) rc = cuda_error(e, "autotune timing");
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0) t.push_back(ms);  // first launch warms up
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  std::sort(t.begin(), t.end());
  *out_ms = t[t.size() / 2];
  return BNTT_OK;
}

}  // namespace bntt

using namespace bntt;

extern "C" {

// Measures every compiled shape for transform sizes 2^1..2^10 (contiguous
// tiles and, for 2^5..2^10, the strided first HBM pass of large transforms),
// and the persistent kernel's tile shape per size; installs the fastest as
// defaults.  If `path` is non-NULL the choices are also written there.
// Contiguous shapes are timed on batches of 65,536 transforms (at most 2^24
// elements) with the L2 flushed before each launch: the size of a uniform
// batch, whose small transforms fit in L2 only when reused.
// Takes a few seconds and about 1 GiB of device memory.
int bntt_autotune(bntt_ctx* c, const char* path) {
  BNTT_REQUIRE(c, "ctx is NULL");
  if (int rc = ctx_use_device(c)) return rc;
  const size_t elems = (size_t)1 << 24;  // 256 MiB per buffer: larger than L2
  void *x = nullptr, *y = nullptr, *tw = nullptr, *flush = nullptr;
  int rc;
  if ((rc = ctx_alloc(c, &x, elems * 16)) || (rc = ctx_alloc(c, &y, elems * 16)) ||
      (rc = ctx_alloc(c, &tw, elems * 16)) || (rc = ctx_alloc(c, &flush, elems * 16))) {
    ctx_free(c, x);
    ctx_free(c, y);
    ctx_free(c, tw);
    return rc;
  }
  const bntt_modulus mod = bntt_modulus_ntt_reference();
  bool fast_mod = false;
  const ModParams mp = make_params(mod, &fast_mod);
  launch_fill(c, x, elems, 11, 0, to_u128(mod.q), BNTT_LAYOUT_HILO, c->stream);
  launch_fill(c, tw, elems, 12, 0, to_u128(mod.q), BNTT_LAYOUT_U128, c->stream);
  std::string report = "bntt-autotune 1 " + device_key(c) + "\n";
  for (int m = 1; m <= 10 && !rc; ++m) {
    for (int map = 0; map < 2 && !rc; ++map) {
      if (map == MAP_INTERLEAVED && m < 5) continue;
      for (int fast = 0; fast < 2 && !rc; ++fast) {
        const SubKernel* best = nullptr;
        float best_ms = 1e30f;
        for (const SubKernel& k : sub_kernels()) {
          if (k.m != m || k.map != map || k.fast != fast) continue;
          SubGeom g;
          g.x = static_cast<const uint4*>(x);
          g.y = static_cast<uint4*>(y);
          g.tw = static_cast<const uint4*>(tw);
          if (map == MAP_CONTIG) {
            g.n = (uint32_t)m;
            g.s0 = 0;
            g.l = 0;
          } else {  // first pass of a 2^(2m) transform: columns of stride 2^m
            g.n = (uint32_t)(2 * m);
            g.s0 = 0;
            g.l = (uint32_t)m;
          }
          g.m = (uint32_t)m;
          g.nsub = elems >> m;
          float ms = 0;
          if (map == MAP_CONTIG) {
            g.nsub = std::min<uint64_t>(g.nsub, 65536);
            rc = time_sub(c, &k, g, mp, 5, &ms, flush, elems * 16);
          } else {
            rc = time_sub(c, &k, g, mp, 5, &ms);
          }
          if (rc) break;
          char line[160];
          snprintf(line, sizeof(line), "# sub m=%d map=%d fast=%d logr=%d tpc=%d minb=%d src=%d %.4f ms\n",
                   m, map, fast, k.logr, k.tpc, k.minb, k.src, ms);
          report += line;
          if (ms < best_ms) {
            best_ms = ms;
            best = &k;
          }
        }
        if (best) {
          std::lock_guard<std::mutex> g(g_tune_mu);
          g_sub_choice[m][map][fast] = best;
          char line[128];
          snprintf(line, sizeof(line), "sub %d %d %d %d %d %d %d\n", m, map, fast, best->logr, best->tpc,
                   best->minb, best->src);
          report += line;
        }
      }
    }
  }
  // persistent kernel: tile shape per small size (fast arithmetic)
  if (!rc) {
    for (int m = 1; m <= 10 && !rc; ++m) {
      bntt_plan* plan = nullptr;
      if ((rc = bntt_plan_create_dev(c, &plan, (unsigned)m, &mod, tw, BNTT_LAYOUT_U128)) != 0) break;
      int best = -1;
      float best_ms = 1e30f;
      for (int s = 0; s < batch_shape_count() && !rc; ++s) {
        int sm, slogr, stpc, smap;
        batch_shape_info(s, &sm, &slogr, &stpc, &smap);
        if (sm != m || smap != MAP_CONTIG) continue;
        float ms = 0;
        if ((rc = batch_time_uniform(c, plan, s, elems >> m, x, y, &ms)) != 0) break;
        char line[128];
        snprintf(line, sizeof(line), "# batch m=%d shape=%d logr=%d tpc=%d %.4f ms\n", m, s, slogr, stpc, ms);
        report += line;
        if (ms < best_ms) {
          best_ms = ms;
          best = s;
        }
      }
      bntt_plan_destroy(plan);
      if (best >= 0) {
        std::lock_guard<std::mutex> g(g_tune_mu);
        g_batch_small_choice[m] = best;
        g_batch_small_set[m] = true;
        int sm, slogr, stpc, smap;
        batch_shape_info(best, &sm, &slogr, &stpc, &smap);
        char line[96];
        snprintf(line, sizeof(line), "batch %d %d %d\n", m, slogr, stpc);
        report += line;
      }
    }
  }
  ctx_free(c, x);
  ctx_free(c, y);
  ctx_free(c, tw);
  ctx_free(c, flush);
  if (rc) return rc;
  if (path) {
    FILE* f = fopen(path, "w");
    if (!f) return set_error(BNTT_EINVAL, "cannot write %s", path);
    fputs(report.c_str(), f);
    fclose(f);
  }
  return BNTT_OK;
}

// Installs choices saved by bntt_autotune.  A file tuned on a different
// device (name or SM count) is refused with BNTT_EINVAL.
int bntt_autotune_load(bntt_ctx* c, const char* path) {
  BNTT_REQUIRE(c && path, "NULL argument");
  FILE* f = fopen(path, "r");
  if (!f) return set_error(BNTT_EINVAL, "cannot open %s", path);
  char line[512];
  int rc = BNTT_OK;
  if (!fgets(line, sizeof(line), f)) rc = set_error(BNTT_EINVAL, "%s is empty", path);
  if (!rc) {
    std::string head = line;
    while (!head.empty() && (head.back() == '\n' || head.back() == '\r')) head.pop_back();
    if (head != "bntt-autotune 1 " + device_key(c))
      rc = set_error(BNTT_EINVAL, "%s was tuned for another device (%s)", path, head.c_str());
  }
  while (!rc && fgets(line, sizeof(line), f)) {
    int m, map, fast, logr, tpc, minb, src = 0;
    const int got = sscanf(line, "sub %d %d %d %d %d %d %d", &m, &map, &fast, &logr, &tpc, &minb, &src);
    if (got == 6 || got == 7) {  // files without the last field name an unstaged shape
      bool found = false;
      for (const SubKernel& k : sub_kernels())
        if (k.m == m && k.map == map && k.fast == fast && k.logr == logr && k.tpc == tpc && k.minb == minb &&
            k.src == src) {
          std::lock_guard<std::mutex> g(g_tune_mu);
          g_sub_choice[m][map][fast] = &k;
          found = true;
        }
      if (!found)
        rc = set_error(BNTT_EINVAL, "%s names a kernel shape this library does not have: %s", path, line);
    } else if (sscanf(line, "batch %d %d %d", &m, &logr, &tpc) == 3) {
      for (int s = 0; s < batch_shape_count(); ++s) {
        int sm, slogr, stpc, smap;
        batch_shape_info(s, &sm, &slogr, &stpc, &smap);
        if (sm == m && slogr == logr && stpc == tpc && smap == MAP_CONTIG && m >= 1 && m <= 10) {
          std::lock_guard<std::mutex> g(g_tune_mu);
          g_batch_small_choice[m] = s;
          g_batch_small_set[m] = true;
        }
      }
    }
  }
  fclose(f);
  return rc;
}

// Forgets all tuned choices (the compiled defaults apply again).
int bntt_autotune_reset(void) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  memset(g_sub_choice, 0, sizeof(g_sub_choice));
  memset(g_batch_small_set, 0, sizeof(g_batch_small_set));
  return BNTT_OK;
}

}  // extern "C"
