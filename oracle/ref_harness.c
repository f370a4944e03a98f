/*
 * ref_harness.c -- a thin C driver around the benchNTT reference functions,
 * compiled from the reference's own sources by oracle/Makefile into
 * oracle/_ref/ (never committed).  TEST INFRASTRUCTURE ONLY: it is the parity
 * pin for the oracle and the timed CPU baseline, never part of the product.
 *
 * One shared object is built per (implementation, stages) because the
 * reference fixes N at compile time (src/ntt_scalar.c:21-22).  The reference
 * translation unit is compiled with -Dmain=bntt_ref_main so that its
 * benchmark driver is not an entry point; everything else is unmodified.
 *
 * Build macros: REF_KIND_NTT or REF_KIND_BLAS; REF_IMPL_SCALAR, REF_IMPL_AVX2
 * or REF_IMPL_AVX512; REF_STAGES (NTT only).
 *
 * Buffers are hi-first u64 pairs (src/config.c:29-30).  Batch calls split the
 * work over `threads` POSIX threads, each with private scratch; the reference
 * globals (SIMD constants one/negone/t) are read-only after ref_init().  Batch
 * calls return the wall time of the work itself (after scratch allocation).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <immintrin.h>

typedef __uint128_t uint128_t;
#define MK(h, l) (((uint128_t)(uint64_t)(h) << 64) | (uint128_t)(uint64_t)(l))

/* ------------------------------------------------------------ declarations */
#if defined(REF_IMPL_SCALAR)
uint128_t addmod128(uint128_t a, uint128_t b, uint128_t m);   /* ntt_scalar.c:49 */
uint128_t submod128(uint128_t a, uint128_t b, uint128_t m);   /* ntt_scalar.c:81 */
uint128_t mulmod128(uint128_t a, uint128_t b, uint128_t m, uint128_t mu); /* :173 */
#endif

#if defined(REF_KIND_NTT)
#define REF_N (1 << REF_STAGES)
#if defined(REF_IMPL_SCALAR)
void ntt(uint128_t *Y, uint128_t *X, uint128_t modulus, uint128_t mu, uint128_t *twiddles,
         uint128_t *as0, uint128_t *as1);                      /* ntt_scalar.c:582 */
#elif defined(REF_IMPL_AVX2)
typedef __m256i vec;
#define LANES 4
extern vec one, negone, t;                                      /* ntt_avx2.c:48 */
void ntt_pre(uint64_t *X, uint64_t *twiddles, uint128_t modulus, uint128_t mu, vec *tempx,
             vec *twdh, vec *twdl, vec *mh, vec *ml, vec *muh, vec *mul);   /* :507 */
void ntt(vec *tempx, vec *twdh, vec *twdl, vec mh, vec ml, vec muh, vec mul, vec *xh, vec *xl,
         vec *ash, vec *asl, vec *th, vec *tl, vec *as);                     /* :566 */
void ntt_post(uint64_t *Y, vec *as);                                         /* :651 */
#elif defined(REF_IMPL_AVX512)
typedef __m512i vec;
#define LANES 8
extern vec one, negone;                                         /* ntt_avx512.c:50 */
void ntt_pre(uint64_t *X, uint64_t *twiddles, uint128_t modulus, uint128_t mu, vec *tempx,
             vec *twdh, vec *twdl, vec *mh, vec *ml, vec *muh, vec *mul, vec *permutehi,
             vec *permutelo);                                                /* :386 */
void ntt(vec *tempx, vec *twdh, vec *twdl, vec mh, vec ml, vec muh, vec mul, vec permutehi,
         vec permutelo, vec *xh, vec *xl, vec *ash, vec *asl, vec *th, vec *tl, vec *as); /* :461 */
void ntt_post(uint64_t *Y, vec *as);                                         /* :524 */
#endif
#endif /* REF_KIND_NTT */

#if defined(REF_KIND_BLAS)
#if defined(REF_IMPL_SCALAR)
void vector_add(uint128_t *c, uint128_t *a, uint128_t *b, uint128_t m);     /* blas_scalar.c:578 */
void vector_sub(uint128_t *c, uint128_t *a, uint128_t *b, uint128_t m);     /* :586 */
void vector_mul(uint128_t *c, uint128_t *a, uint128_t *b, uint128_t m, uint128_t mu); /* :594 */
void axpy(uint128_t *c, uint128_t *a, uint128_t *b, uint128_t x, uint128_t m, uint128_t mu); /* :602 */
#else
#if defined(REF_IMPL_AVX2)
typedef __m256i vec;
#define LANES 4
extern vec one, negone, t;                                      /* blas_avx2.c:42 */
#define SET1(x) _mm256_set1_epi64x((long long)(x))
#else
typedef __m512i vec;
#define LANES 8
extern vec one, negone;                                         /* blas_avx512.c:42 */
#define SET1(x) _mm512_set1_epi64((long long)(x))
#endif
void vector_add(vec *c, vec *a, vec *b, vec mh, vec ml);
void vector_sub(vec *c, vec *a, vec *b, vec mh, vec ml);
void vector_mul(vec *c, vec *a, vec *b, vec mh, vec ml, vec muh, vec mul);
void axpy(vec *c, vec *a, vec *b, vec xh, vec xl, vec mh, vec ml, vec muh, vec mul);
#endif
#endif /* REF_KIND_BLAS */

/* --------------------------------------------------------------- utilities */
static void ref_init(void)
{
#if defined(REF_IMPL_AVX2)
    /* values the reference's main() assigns (ntt_avx2.c:658-660, blas_avx2.c) */
    negone = _mm256_set1_epi64x(-1);
    one = _mm256_set1_epi64x(1);
    t = _mm256_set1_epi64x((long long)0x8000000000000000ULL);
#elif defined(REF_IMPL_AVX512)
    negone = _mm512_set1_epi64(-1);                             /* ntt_avx512.c:531-532 */
    one = _mm512_abs_epi64(negone);
#endif
}

static void *xalloc(size_t bytes)
{
    void *p = aligned_alloc(64, (bytes + 63) & ~(size_t)63);
    if (p) memset(p, 0, (bytes + 63) & ~(size_t)63);
    return p;
}

#include <time.h>

typedef void (*range_fn)(void *ctx, size_t begin, size_t end);
struct par { range_fn fn; void *ctx; size_t n; int threads; int id; };

/* Timing: every thread allocates its scratch, then waits at this barrier;
 * the clock runs from the barrier to the last thread's end, as the reference
 * drivers allocate before their timing loops (src/ntt_scalar.c:635-638). */
static pthread_barrier_t g_barrier;
static int g_barrier_on = 0;
static double g_t0;
static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static void start_gate(void)
{
    if (!g_barrier_on) return;
    if (pthread_barrier_wait(&g_barrier) == PTHREAD_BARRIER_SERIAL_THREAD) g_t0 = now_s();
}

static void *par_body(void *arg)
{
    struct par *p = arg;
    size_t per = (p->n + (size_t)p->threads - 1) / (size_t)p->threads;
    size_t b = per * (size_t)p->id, e = b + per;
    if (e > p->n) e = p->n;
    if (b < e) p->fn(p->ctx, b, e);
    else start_gate();
    return NULL;
}

/* Runs fn over [0, n) on `threads` threads; returns the seconds from the
 * start gate to the end of the last thread. */
static double parallel_for(range_fn fn, void *ctx, size_t n, int threads)
{
    ref_init();
    if (threads < 1) threads = 1;
    if ((size_t)threads > n) threads = n ? (int)n : 1;
    pthread_barrier_init(&g_barrier, NULL, (unsigned)threads);
    g_barrier_on = 1;
    g_t0 = now_s();
    pthread_t *th = malloc(sizeof(pthread_t) * (size_t)threads);
    struct par *ps = malloc(sizeof(struct par) * (size_t)threads);
    for (int i = 0; i < threads; ++i) {
        ps[i] = (struct par){fn, ctx, n, threads, i};
        pthread_create(&th[i], NULL, par_body, &ps[i]);
    }
    for (int i = 0; i < threads; ++i) pthread_join(th[i], NULL);
    double t = now_s() - g_t0;
    g_barrier_on = 0;
    pthread_barrier_destroy(&g_barrier);
    free(th); free(ps);
    return t;
}

/* --------------------------------------------------------------- scalar KAT */
#if defined(REF_IMPL_SCALAR) && defined(REF_KIND_NTT)
void bntt_ref_addmod(uint64_t *out, uint64_t ah, uint64_t al, uint64_t bh, uint64_t bl,
                     uint64_t mh, uint64_t ml)
{
    uint128_t r = addmod128(MK(ah, al), MK(bh, bl), MK(mh, ml));
    out[0] = (uint64_t)(r >> 64); out[1] = (uint64_t)r;
}
void bntt_ref_submod(uint64_t *out, uint64_t ah, uint64_t al, uint64_t bh, uint64_t bl,
                     uint64_t mh, uint64_t ml)
{
    uint128_t r = submod128(MK(ah, al), MK(bh, bl), MK(mh, ml));
    out[0] = (uint64_t)(r >> 64); out[1] = (uint64_t)r;
}
void bntt_ref_mulmod(uint64_t *out, uint64_t ah, uint64_t al, uint64_t bh, uint64_t bl,
                     uint64_t mh, uint64_t ml, uint64_t muh, uint64_t mul)
{
    uint128_t r = mulmod128(MK(ah, al), MK(bh, bl), MK(mh, ml), MK(muh, mul));
    out[0] = (uint64_t)(r >> 64); out[1] = (uint64_t)r;
}
/* element-wise arrays of pairs, for fuzzing */
void bntt_ref_arith_many(int op, uint64_t *out, const uint64_t *a, const uint64_t *b, size_t n,
                         uint64_t mh, uint64_t ml, uint64_t muh, uint64_t mul)
{
    uint128_t m = MK(mh, ml), mu = MK(muh, mul);
    for (size_t i = 0; i < n; ++i) {
        uint128_t x = MK(a[2 * i], a[2 * i + 1]), y = MK(b[2 * i], b[2 * i + 1]), r;
        if (op == 0) r = addmod128(x, y, m);
        else if (op == 1) r = submod128(x, y, m);
        else r = mulmod128(x, y, m, mu);
        out[2 * i] = (uint64_t)(r >> 64); out[2 * i + 1] = (uint64_t)r;
    }
}
#endif

/* ---------------------------------------------------------------------- NTT */
#if defined(REF_KIND_NTT)
int bntt_ref_stages(void) { return REF_STAGES; }

struct ntt_ctx {
    uint64_t *Y; const uint64_t *X; const uint64_t *T;
    uint128_t m, mu;
};

static void ntt_range(void *vctx, size_t b, size_t e)
{
    struct ntt_ctx *c = vctx;
    const size_t n = REF_N;
#if defined(REF_IMPL_SCALAR)
    uint128_t *x = xalloc(n * 16), *y = xalloc(n * 16), *tw = xalloc(n * 16);
    uint128_t *as0 = xalloc(n * 16), *as1 = xalloc(n * 16);
    for (size_t i = 0; i < n; ++i) tw[i] = MK(c->T[2 * i], c->T[2 * i + 1]);
    start_gate();
    for (size_t j = b; j < e; ++j) {
        const uint64_t *xs = c->X + 2 * n * j;
        uint64_t *ys = c->Y + 2 * n * j;
        for (size_t i = 0; i < n; ++i) x[i] = MK(xs[2 * i], xs[2 * i + 1]);
        ntt(y, x, c->m, c->mu, tw, as0, as1);
        for (size_t i = 0; i < n; ++i) { ys[2 * i] = (uint64_t)(y[i] >> 64); ys[2 * i + 1] = (uint64_t)y[i]; }
    }
    free(x); free(y); free(tw); free(as0); free(as1);
#else
    /* scratch sizes follow the reference drivers (ntt_avx2.c:663-677,
     * ntt_avx512.c:535-551) */
    const size_t ops = n / (2 * LANES), v = n / LANES;
    vec *twdh = xalloc(sizeof(vec) * REF_STAGES * ops), *twdl = xalloc(sizeof(vec) * REF_STAGES * ops);
    vec *tempx = xalloc(sizeof(vec) * (2 * n / LANES)), *as = xalloc(sizeof(vec) * (2 * n / LANES));
    vec *xh = xalloc(sizeof(vec) * v), *xl = xalloc(sizeof(vec) * v);
    vec *ash = xalloc(sizeof(vec) * v), *asl = xalloc(sizeof(vec) * v);
    vec *th = xalloc(sizeof(vec) * v), *tl = xalloc(sizeof(vec) * v);
    vec mh, ml, muh, mul;
    start_gate();
    for (size_t j = b; j < e; ++j) {
        uint64_t *xs = (uint64_t *)(c->X + 2 * n * j);
        uint64_t *ys = c->Y + 2 * n * j;
#if defined(REF_IMPL_AVX2)
        ntt_pre(xs, (uint64_t *)c->T, c->m, c->mu, tempx, twdh, twdl, &mh, &ml, &muh, &mul);
        ntt(tempx, twdh, twdl, mh, ml, muh, mul, xh, xl, ash, asl, th, tl, as);
#else
        vec ph, pl;
        ntt_pre(xs, (uint64_t *)c->T, c->m, c->mu, tempx, twdh, twdl, &mh, &ml, &muh, &mul, &ph, &pl);
        ntt(tempx, twdh, twdl, mh, ml, muh, mul, ph, pl, xh, xl, ash, asl, th, tl, as);
#endif
        ntt_post(ys, as);
    }
    free(twdh); free(twdl); free(tempx); free(as); free(xh); free(xl);
    free(ash); free(asl); free(th); free(tl);
#endif
}

/* Per-transform entry points for a whole mixed-size batch run by
 * oracle/ref_batch.c, one shared object per size:
 *   bntt_ref_prep(T, q, mu)      the size's table in the form ntt() reads,
 *                                built once per size (the table expansion
 *                                ntt_pre performs, src/ntt_avx512.c:386-441,
 *                                src/ntt_avx2.c:507-552), before any timing
 *   bntt_ref_scratch_new/free    one thread's working arrays for ntt()
 *   bntt_ref_ntt_only(prep, scratch, x, y)
 *                                ntt() alone: the reference drivers' timed
 *                                region (src/ntt_avx512.c:585-590,
 *                                src/ntt_avx2.c:713-718, src/ntt_scalar.c:
 *                                670-676).  SIMD: x is the packed input
 *                                ntt_pre leaves in tempx, which is the pair
 *                                array itself, and y receives `as`, which is
 *                                the output pair array ntt_post stores
 *                                (both 64-byte aligned).  Scalar: x and y are
 *                                native uint128_t arrays.
 *   bntt_ref_ntt_full(T, q, mu, scratch, x, y)
 *                                the whole per-call sequence on hi-first
 *                                pairs: ntt_pre + ntt + ntt_post (SIMD), or
 *                                the pair conversions around ntt() (scalar). */
struct ref_prep {
#if defined(REF_IMPL_SCALAR)
    uint128_t *tw;
#else
    vec *twdh, *twdl;
    vec mh, ml, muh, mul, ph, pl;
#endif
    uint128_t m, mu;
};

struct ref_scratch {
#if defined(REF_IMPL_SCALAR)
    uint128_t *x, *y, *tw, *as0, *as1;
#else
    vec *twdh, *twdl, *tempx, *as, *xh, *xl, *ash, *asl, *th, *tl;
#endif
};

/* Sets the SIMD constants the reference's main() sets; call once per shared
 * object before any thread uses it. */
void bntt_ref_init(void) { ref_init(); }

void *bntt_ref_scratch_new(void)
{
    const size_t n = REF_N;
    struct ref_scratch *s = calloc(1, sizeof *s);
#if defined(REF_IMPL_SCALAR)
    s->x = xalloc(n * 16); s->y = xalloc(n * 16); s->tw = xalloc(n * 16);
    s->as0 = xalloc(n * 16); s->as1 = xalloc(n * 16);
#else
    const size_t ops = n / (2 * LANES), v = n / LANES;
    s->twdh = xalloc(sizeof(vec) * REF_STAGES * ops); s->twdl = xalloc(sizeof(vec) * REF_STAGES * ops);
    s->tempx = xalloc(sizeof(vec) * (2 * n / LANES)); s->as = xalloc(sizeof(vec) * (2 * n / LANES));
    s->xh = xalloc(sizeof(vec) * v); s->xl = xalloc(sizeof(vec) * v);
    s->ash = xalloc(sizeof(vec) * v); s->asl = xalloc(sizeof(vec) * v);
    s->th = xalloc(sizeof(vec) * v); s->tl = xalloc(sizeof(vec) * v);
#endif
    return s;
}

void bntt_ref_scratch_free(void *p)
{
    struct ref_scratch *s = p;
    if (!s) return;
#if defined(REF_IMPL_SCALAR)
    free(s->x); free(s->y); free(s->tw); free(s->as0); free(s->as1);
#else
    free(s->twdh); free(s->twdl); free(s->tempx); free(s->as); free(s->xh); free(s->xl);
    free(s->ash); free(s->asl); free(s->th); free(s->tl);
#endif
    free(s);
}

void *bntt_ref_prep(const uint64_t *T, uint64_t mh, uint64_t ml, uint64_t muh, uint64_t mul)
{
    const size_t n = REF_N;
    struct ref_prep *p = xalloc(sizeof *p);  /* holds vectors: 64-byte aligned */
    p->m = MK(mh, ml);
    p->mu = MK(muh, mul);
#if defined(REF_IMPL_SCALAR)
    p->tw = xalloc(n * 16);
    for (size_t i = 0; i < n; ++i) p->tw[i] = MK(T[2 * i], T[2 * i + 1]);
#else
    ref_init();
    const size_t ops = n / (2 * LANES);
    p->twdh = xalloc(sizeof(vec) * REF_STAGES * ops);
    p->twdl = xalloc(sizeof(vec) * REF_STAGES * ops);
    vec *tempx = xalloc(sizeof(vec) * (2 * n / LANES));
    uint64_t *x0 = xalloc(n * 16);
#if defined(REF_IMPL_AVX2)
    ntt_pre(x0, (uint64_t *)T, p->m, p->mu, tempx, p->twdh, p->twdl, &p->mh, &p->ml, &p->muh, &p->mul);
#else
    ntt_pre(x0, (uint64_t *)T, p->m, p->mu, tempx, p->twdh, p->twdl, &p->mh, &p->ml, &p->muh, &p->mul,
            &p->ph, &p->pl);
#endif
    free(tempx);
    free(x0);
#endif
    return p;
}

void bntt_ref_prep_free(void *vp)
{
    struct ref_prep *p = vp;
    if (!p) return;
#if defined(REF_IMPL_SCALAR)
    free(p->tw);
#else
    free(p->twdh); free(p->twdl);
#endif
    free(p);
}

void bntt_ref_ntt_only(void *vp, void *vs, const uint64_t *x, uint64_t *y)
{
    struct ref_prep *p = vp;
    struct ref_scratch *s = vs;
#if defined(REF_IMPL_SCALAR)
    ntt((uint128_t *)y, (uint128_t *)x, p->m, p->mu, p->tw, s->as0, s->as1);
#elif defined(REF_IMPL_AVX2)
    ntt((vec *)x, p->twdh, p->twdl, p->mh, p->ml, p->muh, p->mul, s->xh, s->xl, s->ash, s->asl, s->th,
        s->tl, (vec *)y);
#else
    ntt((vec *)x, p->twdh, p->twdl, p->mh, p->ml, p->muh, p->mul, p->ph, p->pl, s->xh, s->xl, s->ash,
        s->asl, s->th, s->tl, (vec *)y);
#endif
}

void bntt_ref_ntt_full(const uint64_t *T, uint64_t mh, uint64_t ml, uint64_t muh, uint64_t mul,
                       void *vs, const uint64_t *xs, uint64_t *ys)
{
    struct ref_scratch *s = vs;
    const size_t n = REF_N;
    const uint128_t m = MK(mh, ml), mu = MK(muh, mul);
#if defined(REF_IMPL_SCALAR)
    for (size_t i = 0; i < n; ++i) s->tw[i] = MK(T[2 * i], T[2 * i + 1]);
    for (size_t i = 0; i < n; ++i) s->x[i] = MK(xs[2 * i], xs[2 * i + 1]);
    ntt(s->y, s->x, m, mu, s->tw, s->as0, s->as1);
    for (size_t i = 0; i < n; ++i) { ys[2 * i] = (uint64_t)(s->y[i] >> 64); ys[2 * i + 1] = (uint64_t)s->y[i]; }
#else
    vec vmh, vml, vmuh, vmul;
#if defined(REF_IMPL_AVX2)
    ntt_pre((uint64_t *)xs, (uint64_t *)T, m, mu, s->tempx, s->twdh, s->twdl, &vmh, &vml, &vmuh, &vmul);
    ntt(s->tempx, s->twdh, s->twdl, vmh, vml, vmuh, vmul, s->xh, s->xl, s->ash, s->asl, s->th, s->tl, s->as);
#else
    vec ph, pl;
    ntt_pre((uint64_t *)xs, (uint64_t *)T, m, mu, s->tempx, s->twdh, s->twdl, &vmh, &vml, &vmuh, &vmul,
            &ph, &pl);
    ntt(s->tempx, s->twdh, s->twdl, vmh, vml, vmuh, vmul, ph, pl, s->xh, s->xl, s->ash, s->asl, s->th,
        s->tl, s->as);
#endif
    ntt_post(ys, s->as);
#endif
}

/* `batch` contiguous transforms of N = 2^REF_STAGES hi-first pairs sharing
 * table T; each transform is the reference's full per-call sequence
 * (scalar: ntt(); SIMD: ntt_pre + ntt + ntt_post). */
double bntt_ref_ntt_batch(uint64_t *Y, const uint64_t *X, const uint64_t *T, size_t batch,
                          uint64_t mh, uint64_t ml, uint64_t muh, uint64_t mul, int threads)
{
    struct ntt_ctx c = {Y, X, T, MK(mh, ml), MK(muh, mul)};
    return parallel_for(ntt_range, &c, batch, threads);
}
#endif /* REF_KIND_NTT */

/* --------------------------------------------------------------------- BLAS */
#if defined(REF_KIND_BLAS)
struct blas_ctx {
    int op; uint64_t *C; const uint64_t *A, *B;
    uint128_t x, m, mu;
};

static void blas_range(void *vctx, size_t b, size_t e)
{
    struct blas_ctx *c = vctx;
#if defined(REF_IMPL_SCALAR)
    uint128_t *a = xalloc(1024 * 16), *bb = xalloc(1024 * 16), *cc = xalloc(1024 * 16);
    start_gate();
    for (size_t k = b; k < e; ++k) {
        const uint64_t *as = c->A + 2048 * k, *bs = c->B + 2048 * k;
        uint64_t *cs = c->C + 2048 * k;
        for (int i = 0; i < 1024; ++i) { a[i] = MK(as[2 * i], as[2 * i + 1]); bb[i] = MK(bs[2 * i], bs[2 * i + 1]); }
        switch (c->op) {
        case 0: vector_add(cc, a, bb, c->m); break;
        case 1: vector_sub(cc, a, bb, c->m); break;
        case 2: vector_mul(cc, a, bb, c->m, c->mu); break;
        default: axpy(cc, a, bb, c->x, c->m, c->mu); break;
        }
        for (int i = 0; i < 1024; ++i) { cs[2 * i] = (uint64_t)(cc[i] >> 64); cs[2 * i + 1] = (uint64_t)cc[i]; }
    }
    free(a); free(bb); free(cc);
#else
    vec mh = SET1(c->m >> 64), ml = SET1((uint64_t)c->m);
    vec muh = SET1(c->mu >> 64), mul = SET1((uint64_t)c->mu);
    vec xh = SET1(c->x >> 64), xl = SET1((uint64_t)c->x);
    vec *sa = xalloc(1024 * 16), *sb = xalloc(1024 * 16), *sc = xalloc(1024 * 16);
    start_gate();
    for (size_t k = b; k < e; ++k) {
        /* the SIMD kernels index vec arrays, so operands must be 64-byte
         * aligned; unaligned chunks are staged through aligned scratch */
        vec *a = (vec *)(c->A + 2048 * k), *bb = (vec *)(c->B + 2048 * k), *cc = (vec *)(c->C + 2048 * k);
        int al = (((uintptr_t)a | (uintptr_t)bb | (uintptr_t)cc) & 63) == 0;
        if (!al) { memcpy(sa, a, 16384); memcpy(sb, bb, 16384); a = sa; bb = sb; cc = sc; }
        switch (c->op) {
        case 0: vector_add(cc, a, bb, mh, ml); break;
        case 1: vector_sub(cc, a, bb, mh, ml); break;
        case 2: vector_mul(cc, a, bb, mh, ml, muh, mul); break;
        default: axpy(cc, a, bb, xh, xl, mh, ml, muh, mul); break;
        }
        if (!al) memcpy(c->C + 2048 * k, sc, 16384);
    }
    free(sa); free(sb); free(sc);
#endif
}

/* op: 0 vvadd, 1 vvsub, 2 vvmul, 3 axpy (c = a + x*b).  len must be a
 * multiple of 1024, the reference's fixed vector length
 * (src/blas_scalar.c:580); each 1024-element chunk is one reference call. */
double bntt_ref_blas(int op, uint64_t *C, const uint64_t *A, const uint64_t *B, uint64_t xh,
                     uint64_t xl, size_t len, uint64_t mh, uint64_t ml, uint64_t muh, uint64_t mul,
                     int threads)
{
    if (len % 1024) return -1.0;
    struct blas_ctx c = {op, C, A, B, MK(xh, xl), MK(mh, ml), MK(muh, mul)};
    return parallel_for(blas_range, &c, len / 1024, threads);
}
#endif /* REF_KIND_BLAS */
