/* Negacyclic polynomial products through the native C ABI (include/bntt.h):
 * the three-call pipeline of the NTT-friendly prime mode -- forward(b),
 * forward(a) fused with the pointwise product, inverse -- checked against a
 * schoolbook product mod (x^N + 1) computed here on the host.
 * Usage: polymul_driver <log2n> <batch>; prints "<N> fail: <count>". */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bntt.h"

typedef unsigned __int128 u128;

static u128 to128(bntt_u128 v) { return ((u128)v.hi << 64) | v.lo; }

/* a * b mod q by double-and-add (a, b < q < 2^124: no intermediate overflow) */
static u128 mulmod(u128 a, u128 b, u128 q)
{
    u128 r = 0;
    for (int i = 123; i >= 0; --i) {
        r <<= 1;
        if (r >= q) r -= q;
        if ((b >> i) & 1) {
            r += a;
            if (r >= q) r -= q;
        }
    }
    return r;
}

#define CHECK(call)                                                              \
    do {                                                                         \
        int rc_ = (call);                                                        \
        if (rc_) {                                                               \
            fprintf(stderr, "%s: %d %s\n", #call, rc_, bntt_last_error());       \
            return 1;                                                            \
        }                                                                        \
    } while (0)

int main(int argc, char **argv)
{
    unsigned logn = argc > 1 ? (unsigned)atoi(argv[1]) : 6;
    size_t batch = argc > 2 ? (size_t)atoi(argv[2]) : 2;
    size_t n = (size_t)1 << logn, total = n * batch;

    bntt_modulus m;
    bntt_u128 w, psi, e;
    CHECK(bntt_ntt_prime(21, &m));
    CHECK(bntt_root_of_unity(&m, 21, &w));
    e.hi = 0;
    e.lo = (uint64_t)1 << (20 - logn);                /* psi = w^(2^(20 - log2n)): order 2N */
    CHECK(bntt_powmod(&m, w, e, &psi));

    bntt_ctx *ctx;
    bntt_plan *plan;
    CHECK(bntt_ctx_create(&ctx, 0, NULL));
    CHECK(bntt_plan_create_negacyclic(ctx, &plan, logn, &m, psi, BNTT_LAYOUT_HILO));

    uint64_t *a = malloc(total * 16), *b = malloc(total * 16), *c = malloc(total * 16);
    CHECK(bntt_fill_uniform_host(a, total, 101, 0, &m, BNTT_LAYOUT_HILO));
    CHECK(bntt_fill_uniform_host(b, total, 202, 0, &m, BNTT_LAYOUT_HILO));

    void *da, *db, *dbh, *dc;
    CHECK(bntt_dev_alloc(ctx, &da, total * 16));
    CHECK(bntt_dev_alloc(ctx, &db, total * 16));
    CHECK(bntt_dev_alloc(ctx, &dbh, total * 16));
    CHECK(bntt_dev_alloc(ctx, &dc, total * 16));
    CHECK(bntt_copy_h2d(ctx, da, a, total * 16));
    CHECK(bntt_copy_h2d(ctx, db, b, total * 16));
    CHECK(bntt_ntt_forward_dev(plan, dbh, db, batch));              /* b^ = ntt(b)        */
    CHECK(bntt_ntt_forward_mul_dev(plan, dc, da, dbh, 1, batch));   /* c = ntt(a) o b^    */
    CHECK(bntt_ntt_inverse_dev(plan, dc, dc, batch));               /* c = a * b mod x^N+1 */
    CHECK(bntt_ctx_synchronize(ctx));
    CHECK(bntt_copy_d2h(ctx, c, dc, total * 16));

    u128 q = to128(m.q);
    size_t fail = 0;
    u128 *want = calloc(n, sizeof(u128));
    for (size_t t = 0; t < batch; ++t) {
        const uint64_t *ap = a + 2 * n * t, *bp = b + 2 * n * t, *cp = c + 2 * n * t;
        memset(want, 0, n * sizeof(u128));
        for (size_t i = 0; i < n; ++i) {
            u128 ai = ((u128)ap[2 * i] << 64) | ap[2 * i + 1];
            for (size_t j = 0; j < n; ++j) {
                u128 bj = ((u128)bp[2 * j] << 64) | bp[2 * j + 1];
                u128 p = mulmod(ai, bj, q);
                size_t k = i + j;
                if (k < n) {
                    want[k] += p;
                    if (want[k] >= q) want[k] -= q;
                } else {
                    k -= n;
                    want[k] = want[k] >= p ? want[k] - p : want[k] + q - p;
                }
            }
        }
        for (size_t k = 0; k < n; ++k) {
            u128 got = ((u128)cp[2 * k] << 64) | cp[2 * k + 1];
            if (got != want[k]) ++fail;
        }
    }
    printf("%zu fail: %zu\n", n, fail);

    free(want);
    free(a);
    free(b);
    free(c);
    bntt_dev_free(ctx, da);
    bntt_dev_free(ctx, db);
    bntt_dev_free(ctx, dbh);
    bntt_dev_free(ctx, dc);
    bntt_plan_destroy(plan);
    bntt_ctx_destroy(ctx);
    return fail != 0;
}
