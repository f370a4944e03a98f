/*
 * bntt_oracle.c -- CPU restatement of benchNTT's scalar path (the parity oracle).
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load this library, and only as the checker.
 * The product (benchntt_b200/libbntt.so) never links, loads or calls it.
 *
 * What it restates (paths relative to the benchNTT repository):
 *   addmod128   src/ntt_scalar.c:49-79   (identical copy src/blas_scalar.c:44-74)
 *   submod128   src/ntt_scalar.c:81-104
 *   mul128      src/ntt_scalar.c:106-128
 *   mullo128    src/ntt_scalar.c:130-149
 *   mulhi128    src/ntt_scalar.c:151-171
 *   mulmod128   src/ntt_scalar.c:173-199  (Barrett, MBITS = 124)
 *   ntt         src/ntt_scalar.c:582-627  (constant-geometry radix-2 network)
 *   vector_add / vector_sub / vector_mul / axpy   src/blas_scalar.c:578-608
 * and, with no reference counterpart, the inverse of the network
 * (orc_ntt_inverse_batch), the checker of libbntt's inverse transform.
 *
 * Every 64-bit word operation keeps the reference's truncation points, so the
 * results equal the reference's for ANY 128-bit inputs, including the two
 * corner behaviours the reference has:
 *   - addmod returns s (not s - q) when s == q (strict '>' test), and
 *   - when s > q and lo64(s) == lo64(q) the reference borrows one from the
 *     high word that exact arithmetic would not (the borrow of the low word is
 *     taken as "lo64(q) >= lo64(s)" instead of "lo64(q) > lo64(s)").
 * Parity pin: tests/test_oracle.py checks this file against the reference's
 * golden vectors (data/ver_N.txt, data/{vvadd,vvsub,vvmul,axpy}_1024.txt,
 * committed as tests/golden/ref_data.npz) and against the reference compiled
 * from its own sources (oracle/_ref, built by `make -C oracle ref`).
 *
 * Buffers at the C ABI are "hi-first u64 pairs": element i is buf[2i] (high
 * 64 bits) and buf[2i+1] (low 64 bits), the layout of the reference's data
 * files and SIMD paths (src/config.c:29-30).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

typedef unsigned __int128 u128;

#define HI(x) ((uint64_t)((x) >> 64))
#define LO(x) ((uint64_t)(x))
#define MK(h, l) (((u128)(uint64_t)(h) << 64) | (u128)(uint64_t)(l))

static inline u128 get_pair(const uint64_t *p, size_t i) { return MK(p[2 * i], p[2 * i + 1]); }
static inline void put_pair(uint64_t *p, size_t i, u128 v) { p[2 * i] = HI(v); p[2 * i + 1] = LO(v); }

/* ---------------------------------------------------------------- arithmetic */

/* src/ntt_scalar.c:49-79.  s = a + b (mod 2^128); e = m - s (mod 2^128); the
 * "is s > m" flag is the borrow out of e.  The reference forms s - m from e's
 * words as (hi: s_hi - m_hi - [m_lo >= s_lo], lo: s_lo - m_lo), which is
 * (~e_hi, -e_lo). */
u128 orc_addmod(u128 a, u128 b, u128 m)
{
    uint64_t s_lo = LO(a) + LO(b);
    uint64_t c = s_lo < LO(a);
    uint64_t s_hi = HI(a) + HI(b) + c;            /* carry out of 128 bits dropped */
    uint64_t m_lo = LO(m), m_hi = HI(m);
    uint64_t lo_borrow = m_lo < s_lo;              /* borrow of m_lo - s_lo */
    /* borrow of (m_hi - s_hi - lo_borrow) as a 65-bit subtraction */
    int gt = ((u128)m_hi < (u128)s_hi + lo_borrow);
    if (!gt) return MK(s_hi, s_lo);
    uint64_t r_lo = s_lo - m_lo;
    uint64_t r_hi = s_hi - m_hi - (uint64_t)(!lo_borrow);
    return MK(r_hi, r_lo);
}

/* src/ntt_scalar.c:81-104.  d = a - b (mod 2^128); add m back on borrow. */
u128 orc_submod(u128 a, u128 b, u128 m)
{
    uint64_t d_lo = LO(a) - LO(b);
    uint64_t bl = LO(a) < LO(b);
    uint64_t d_hi = HI(a) - HI(b) - bl;
    int borrow = ((u128)HI(a) < (u128)HI(b) + bl);
    u128 d = MK(d_hi, d_lo);
    return borrow ? d + m : d;
}

/* src/ntt_scalar.c:106-128: 128x128 -> 256 from four 64x64 products; the two
 * middle sums are kept to 128 bits as in the reference. */
static void orc_mul128(u128 *hi, u128 *lo, u128 a, u128 b)
{
    u128 p00 = (u128)LO(a) * LO(b), p01 = (u128)LO(a) * HI(b);
    u128 p10 = (u128)HI(a) * LO(b), p11 = (u128)HI(a) * HI(b);
    u128 mid = p01 + p10;
    u128 mid2 = mid + (p00 >> 64);
    *hi = p11 + (mid2 >> 64);
    *lo = MK(LO(mid2), LO(p00));
}

/* src/ntt_scalar.c:130-149: low 128 bits, cross terms kept to 64 bits. */
static u128 orc_mullo128(u128 a, u128 b)
{
    u128 p00 = (u128)LO(a) * LO(b);
    uint64_t cross = LO(a) * HI(b) + HI(a) * LO(b);
    uint64_t top = cross + HI(p00);
    return MK(top, LO(p00));
}

/* src/ntt_scalar.c:151-171: high 128 bits, middle sums kept to 128 bits. */
static u128 orc_mulhi128(u128 a, u128 b)
{
    u128 p00h = ((u128)LO(a) * LO(b)) >> 64;
    u128 p01 = (u128)LO(a) * HI(b), p10 = (u128)HI(a) * LO(b);
    u128 p11 = (u128)HI(a) * HI(b);
    u128 mid = p01 + p10;
    u128 mid2 = mid + p00h;
    return p11 + (mid2 >> 64);
}

#define ORC_MBITS 124

/* src/ntt_scalar.c:173-199: Barrett with MBITS = 124 and one conditional
 * subtraction. */
u128 orc_mulmod(u128 a, u128 b, u128 m, u128 mu)
{
    u128 ph, pl;
    orc_mul128(&ph, &pl, a, b);
    u128 t = (pl >> (ORC_MBITS - 2)) | (ph << (128 - (ORC_MBITS - 2)));
    uint64_t top = (uint64_t)(ph >> (ORC_MBITS - 2));
    u128 qm = orc_mulhi128(t, mu) + (u128)(uint64_t)(top * LO(mu));
    u128 qq = qm >> 1;
    u128 r = pl - orc_mullo128(qq, m);
    return (r < m) ? r : r - m;
}

/* Exact a*b mod m by shift-and-subtract over the full 256-bit product.
 * Independent of the reference; used by tests to confirm that the Barrett
 * path above is exact for the reference moduli on in-range inputs. */
u128 orc_mulmod_exact(u128 a, u128 b, u128 m)
{
    u128 ph, pl;
    /* exact 256-bit product (no truncation) */
    u128 p00 = (u128)LO(a) * LO(b), p01 = (u128)LO(a) * HI(b);
    u128 p10 = (u128)HI(a) * LO(b), p11 = (u128)HI(a) * HI(b);
    u128 mid = (p00 >> 64) + LO(p01) + LO(p10);
    pl = MK(LO(mid), LO(p00));
    ph = p11 + HI(p01) + HI(p10) + (mid >> 64);
    u128 r = 0;
    for (int i = 255; i >= 0; --i) {
        int bit = i >= 128 ? (int)((ph >> (i - 128)) & 1) : (int)((pl >> i) & 1);
        int top = (int)(r >> 127);
        r = (r << 1) | (u128)bit;
        if (top || r >= m) r -= m;
    }
    return r;
}

/* hi-first-pair wrappers for ctypes */
#define DEF_BIN(name, expr)                                                          \
    void name##_pairs(uint64_t *out, uint64_t ah, uint64_t al, uint64_t bh, uint64_t bl, \
                      uint64_t mh, uint64_t ml, uint64_t muh, uint64_t mul)          \
    {                                                                                \
        u128 a = MK(ah, al), b = MK(bh, bl), m = MK(mh, ml), mu = MK(muh, mul);      \
        (void)mu;                                                                    \
        u128 r = (expr);                                                             \
        out[0] = HI(r); out[1] = LO(r);                                              \
    }
DEF_BIN(orc_addmod, orc_addmod(a, b, m))
DEF_BIN(orc_submod, orc_submod(a, b, m))
DEF_BIN(orc_mulmod, orc_mulmod(a, b, m, mu))
DEF_BIN(orc_mulmod_exact, orc_mulmod_exact(a, b, m))

/* ---------------------------------------------------------------------- NTT */

/* src/ntt_scalar.c:582-627, constant-geometry form.  Stage 0 reads X, stage s
 * (1 <= s < n) uses twiddle T[2^s + (j mod 2^s)] for output pair j, and
 * writes positions 2j / 2j+1; the reference ping-pongs between two scratch
 * arrays and lets the last stage write Y.  Works for any n >= 1; for n = 1 the
 * single stage uses T[1] and writes Y directly. */
static void ntt_cg_one(u128 *y, const u128 *x, int logn, u128 m, u128 mu, const u128 *T,
                       u128 *buf0, u128 *buf1)
{
    size_t n = (size_t)1 << logn, half = n >> 1;
    const u128 *src = x;
    for (int s = 0; s < logn; ++s) {
        u128 *dst = (s == logn - 1) ? y : ((s & 1) ? buf1 : buf0);
        size_t tw_base = (size_t)1 << s;
        for (size_t j = 0; j < half; ++j) {
            u128 w = T[tw_base + (j & (tw_base - 1))];
            u128 p = orc_mulmod(w, src[j + half], m, mu);
            u128 a = src[j];
            dst[2 * j] = orc_addmod(a, p, m);
            dst[2 * j + 1] = orc_submod(a, p, m);
        }
        src = dst;
    }
}

/* The same network written in place in natural order: stage s pairs indices
 * that differ in bit (logn-1-s) and multiplies by T[2^s + (index >> (logn-s))].
 * Used by tests to confirm the equivalence the GPU kernels rely on. */
static void ntt_inplace_one(u128 *v, int logn, u128 m, u128 mu, const u128 *T)
{
    size_t n = (size_t)1 << logn;
    for (int s = 0; s < logn; ++s) {
        size_t half = n >> (s + 1);
        for (size_t blk = 0; blk < ((size_t)1 << s); ++blk) {
            u128 w = T[((size_t)1 << s) + blk];
            size_t base = blk * 2 * half;
            for (size_t k = base; k < base + half; ++k) {
                u128 p = orc_mulmod(w, v[k + half], m, mu);
                u128 a = v[k];
                v[k] = orc_addmod(a, p, m);
                v[k + half] = orc_submod(a, p, m);
            }
        }
    }
}

struct ntt_job {
    uint64_t *y;
    const uint64_t *x;
    const uint64_t *t;
    int logn;
};

struct ntt_work {
    const struct ntt_job *jobs;
    size_t njobs;
    u128 m, mu;
    int form;              /* 0 = constant geometry, 1 = in place */
    size_t next;           /* shared cursor */
    pthread_mutex_t lock;
};

static void run_job(const struct ntt_job *jb, u128 m, u128 mu, int form)
{
    size_t n = (size_t)1 << jb->logn;
    u128 *x = malloc(n * sizeof(u128)), *t = malloc(n * sizeof(u128));
    u128 *y = malloc(n * sizeof(u128));
    u128 *b0 = malloc(n * sizeof(u128)), *b1 = malloc(n * sizeof(u128));
    for (size_t i = 0; i < n; ++i) { x[i] = get_pair(jb->x, i); t[i] = get_pair(jb->t, i); }
    if (form == 0) {
        ntt_cg_one(y, x, jb->logn, m, mu, t, b0, b1);
    } else {
        memcpy(y, x, n * sizeof(u128));
        ntt_inplace_one(y, jb->logn, m, mu, t);
    }
    for (size_t i = 0; i < n; ++i) put_pair(jb->y, i, y[i]);
    free(x); free(t); free(y); free(b0); free(b1);
}

static void *worker(void *arg)
{
    struct ntt_work *w = arg;
    for (;;) {
        pthread_mutex_lock(&w->lock);
        size_t i = w->next++;
        pthread_mutex_unlock(&w->lock);
        if (i >= w->njobs) break;
        run_job(&w->jobs[i], w->m, w->mu, w->form);
    }
    return NULL;
}

/* Forward transforms of `count` independent inputs.  Job i reads
 * xs[i] (2^logns[i] hi-first pairs), twiddle table ts[i] (same length) and
 * writes ys[i].  `threads` <= 1 runs serially. */
void orc_ntt_jobs(uint64_t **ys, const uint64_t **xs, const uint64_t **ts, const int *logns,
                  size_t count, uint64_t mh, uint64_t ml, uint64_t muh, uint64_t mul, int form,
                  int threads)
{
    struct ntt_job *jobs = malloc(count * sizeof(*jobs));
    for (size_t i = 0; i < count; ++i) {
        jobs[i].y = ys[i]; jobs[i].x = xs[i]; jobs[i].t = ts[i]; jobs[i].logn = logns[i];
    }
    struct ntt_work w = {jobs, count, MK(mh, ml), MK(muh, mul), form, 0};
    pthread_mutex_init(&w.lock, NULL);
    if (threads <= 1) {
        worker(&w);
    } else {
        pthread_t *th = malloc((size_t)threads * sizeof(pthread_t));
        for (int i = 0; i < threads; ++i) pthread_create(&th[i], NULL, worker, &w);
        for (int i = 0; i < threads; ++i) pthread_join(th[i], NULL);
        free(th);
    }
    pthread_mutex_destroy(&w.lock);
    free(jobs);
}

/* Uniform batch: `batch` contiguous transforms of size 2^logn sharing T. */
void orc_ntt_batch(uint64_t *Y, const uint64_t *X, const uint64_t *T, int logn, size_t batch,
                   uint64_t mh, uint64_t ml, uint64_t muh, uint64_t mul, int form, int threads)
{
    size_t n = (size_t)1 << logn;
    uint64_t **ys = malloc(batch * sizeof(*ys));
    const uint64_t **xs = malloc(batch * sizeof(*xs));
    const uint64_t **ts = malloc(batch * sizeof(*ts));
    int *ls = malloc(batch * sizeof(int));
    for (size_t b = 0; b < batch; ++b) {
        ys[b] = Y + 2 * n * b; xs[b] = X + 2 * n * b; ts[b] = T; ls[b] = logn;
    }
    orc_ntt_jobs(ys, xs, ts, ls, batch, mh, ml, muh, mul, form, threads);
    free(ys); free(xs); free(ts); free(ls);
}

/* ------------------------------------------------------------ inverse NTT */

/* Not in the reference (it has no inverse transform): the inverse of the
 * in-place network above, which libbntt's bntt_ntt_inverse_dev computes.
 * Stages run from logn-1 down to 0; stage s pairs indices that differ in bit
 * logn-1-s, block b uses Tinv[2^s + b] = T[2^s + b]^-1, and each pair
 * (x, y) becomes (x + y, (x - y) * w) with exact sums: x + y less q when it
 * is at least q, x - y plus q on borrow.  Finally every element is
 * multiplied by N^-1.  Products use orc_mulmod, exact for q = 2^124 - k with
 * k < 2^31 and mu = floor(2^251/q) (checked by tests/test_oracle.py). */
static u128 orc_powmod(u128 a, u128 e, u128 m, u128 mu)
{
    u128 r = 1;
    while (e) {
        if (e & 1) r = orc_mulmod(r, a, m, mu);
        a = orc_mulmod(a, a, m, mu);
        e >>= 1;
    }
    return r;
}

static void ntt_inverse_one(u128 *v, int logn, u128 m, u128 mu, const u128 *Tinv, u128 ninv)
{
    size_t n = (size_t)1 << logn;
    for (int s = logn - 1; s >= 0; --s) {
        size_t half = n >> (s + 1);
        for (size_t blk = 0; blk < ((size_t)1 << s); ++blk) {
            u128 w = Tinv[((size_t)1 << s) + blk];
            size_t base = blk * 2 * half;
            for (size_t k = base; k < base + half; ++k) {
                u128 a = v[k], b = v[k + half];
                u128 sum = a + b;
                v[k] = sum >= m ? sum - m : sum;
                v[k + half] = orc_mulmod(w, orc_submod(a, b, m), m, mu);
            }
        }
    }
    for (size_t i = 0; i < n; ++i) v[i] = orc_mulmod(v[i], ninv, m, mu);
}

/* `batch` contiguous inverse transforms of size 2^logn; T is the FORWARD
 * table (2^logn hi-first pairs), inverted here entry by entry (Fermat).
 * Returns 0, or -1 when an entry or N has no inverse. */
int orc_ntt_inverse_batch(uint64_t *X, const uint64_t *Y, const uint64_t *T, int logn, size_t batch,
                          uint64_t mh, uint64_t ml, uint64_t muh, uint64_t mul)
{
    u128 m = MK(mh, ml), mu = MK(muh, mul);
    size_t n = (size_t)1 << logn;
    u128 *tinv = malloc(n * sizeof(u128)), *v = malloc(n * sizeof(u128));
    int rc = 0;
    tinv[0] = 1;
    for (size_t k = 1; k < n && !rc; ++k) {
        u128 t = get_pair(T, k);
        tinv[k] = orc_powmod(t, m - 2, m, mu);
        if (orc_mulmod(tinv[k], t, m, mu) != 1) rc = -1;
    }
    u128 ninv = orc_powmod((u128)n % m, m - 2, m, mu);
    if (orc_mulmod(ninv, (u128)n % m, m, mu) != 1) rc = -1;
    for (size_t b = 0; b < batch && !rc; ++b) {
        for (size_t i = 0; i < n; ++i) v[i] = get_pair(Y, b * n + i);
        ntt_inverse_one(v, logn, m, mu, tinv, ninv);
        for (size_t i = 0; i < n; ++i) put_pair(X, b * n + i, v[i]);
    }
    free(tinv);
    free(v);
    return rc;
}

/* --------------------------------------------------------------------- BLAS */

/* src/blas_scalar.c:578-608, for any length (the reference fixes 1024). */
void orc_vvadd(uint64_t *c, const uint64_t *a, const uint64_t *b, size_t len, uint64_t mh,
               uint64_t ml)
{
    u128 m = MK(mh, ml);
    for (size_t i = 0; i < len; ++i) put_pair(c, i, orc_addmod(get_pair(a, i), get_pair(b, i), m));
}

void orc_vvsub(uint64_t *c, const uint64_t *a, const uint64_t *b, size_t len, uint64_t mh,
               uint64_t ml)
{
    u128 m = MK(mh, ml);
    for (size_t i = 0; i < len; ++i) put_pair(c, i, orc_submod(get_pair(a, i), get_pair(b, i), m));
}

void orc_vvmul(uint64_t *c, const uint64_t *a, const uint64_t *b, size_t len, uint64_t mh,
               uint64_t ml, uint64_t muh, uint64_t mul)
{
    u128 m = MK(mh, ml), mu = MK(muh, mul);
    for (size_t i = 0; i < len; ++i)
        put_pair(c, i, orc_mulmod(get_pair(a, i), get_pair(b, i), m, mu));
}

/* c[i] = addmod(a[i], mulmod(x, b[i])) -- blas_scalar.c:602-606 */
void orc_axpy(uint64_t *c, const uint64_t *a, const uint64_t *b, uint64_t xh, uint64_t xl,
              size_t len, uint64_t mh, uint64_t ml, uint64_t muh, uint64_t mul)
{
    u128 m = MK(mh, ml), mu = MK(muh, mul), x = MK(xh, xl);
    for (size_t i = 0; i < len; ++i)
        put_pair(c, i, orc_addmod(get_pair(a, i), orc_mulmod(x, get_pair(b, i), m, mu), m));
}
