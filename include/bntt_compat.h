/*
 * bntt_compat.h -- the benchNTT reference's scalar call shapes on libbntt.
 *
 * A C program written against the reference's scalar functions
 *   ntt(Y, X, modulus, mu, twiddles, as0, as1)     src/ntt_scalar.c:582
 *   vector_add(c, a, b, m)                         src/blas_scalar.c:578
 *   vector_sub(c, a, b, m)                         src/blas_scalar.c:586
 *   vector_mul(c, a, b, m, mu)                     src/blas_scalar.c:594
 *   axpy(c, a, b, x, m, mu)                        src/blas_scalar.c:602
 * includes this header instead of defining them, and links -lbntt.  As in the
 * reference, N comes from the program's `stages` macro (src/ntt_scalar.c:21)
 * at each call site and the BLAS length is 1024 (src/blas_scalar.c:580; set
 * BNTT_COMPAT_BLAS_LEN before including to change it).  The scratch arrays
 * as0/as1 are accepted and not used.  Arrays are native uint128_t (lo word
 * first in memory), host memory; each call returns with the result in place.
 * The reference functions return void; here a failure prints the library's
 * message and aborts (define BNTT_COMPAT_ON_ERROR to handle it otherwise).
 *
 * The data-file loaders of src/config.c have counterparts that return a
 * status instead of calling exit(): bntt_load_reference_data (load_twiddles /
 * load_test_inputs / load_test_outputs, with their 1024-entry tiling for
 * N > 1024), bntt_load_pairs_text and bntt_save_pairs_text.
 * Define BNTT_COMPAT_NO_MACROS to get the functions without the name macros.
 */
#ifndef BNTT_COMPAT_H
#define BNTT_COMPAT_H

#include <stdio.h>
#include <stdlib.h>

#include "bntt.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef __uint128_t bntt_uint128;

int bntt_compat_ntt_u128(bntt_uint128 *Y, const bntt_uint128 *X, bntt_uint128 modulus,
                         bntt_uint128 mu, const bntt_uint128 *twiddles, unsigned log2n);
int bntt_compat_ntt_pairs(uint64_t *Y, const uint64_t *X, bntt_uint128 modulus, bntt_uint128 mu,
                          const uint64_t *twiddles, unsigned log2n);
int bntt_compat_blas_u128(int op, bntt_uint128 *c, const bntt_uint128 *a, const bntt_uint128 *b,
                          bntt_uint128 x, bntt_uint128 m, bntt_uint128 mu, size_t len);
int bntt_compat_blas_pairs(int op, uint64_t *c, const uint64_t *a, const uint64_t *b,
                           bntt_uint128 x, bntt_uint128 m, bntt_uint128 mu, size_t len);
int bntt_compat_simd_pre(const uint64_t *X, const uint64_t *twiddles, bntt_uint128 modulus,
                         bntt_uint128 mu, unsigned log2n);
int bntt_compat_simd_run(void *as_out);
int bntt_compat_simd_post(uint64_t *Y, const void *as_in);
int bntt_compat_shutdown(void);

int bntt_load_pairs_text(const char *path, uint64_t *pairs, size_t n);
int bntt_save_pairs_text(const char *path, const uint64_t *pairs, size_t n);
/* <dir>/<kind>_<N>.txt with kind "twd", "x" or "ver" (src/config.c:10,78,146) */
int bntt_load_reference_data(const char *dir, const char *kind, uint64_t *pairs, size_t n);

#ifdef __cplusplus
}
#endif

#ifndef BNTT_COMPAT_ON_ERROR
static inline int bntt_compat_check_(int status, const char *what)
{
    if (status != BNTT_OK) {
        fprintf(stderr, "%s: %s (%s)\n", what, bntt_status_string(status), bntt_last_error());
        abort();
    }
    return status;
}
#define BNTT_COMPAT_ON_ERROR(status, what) bntt_compat_check_((status), (what))
#endif

#ifndef BNTT_COMPAT_BLAS_LEN
#define BNTT_COMPAT_BLAS_LEN 1024
#endif

#ifndef BNTT_COMPAT_NO_MACROS
/* the scratch arguments are named in an unevaluated sizeof only */
#define ntt(Y, X, modulus, mu, twiddles, as0, as1)                                                \
    ((void)sizeof((as0) == (as1)),                                                              \
     BNTT_COMPAT_ON_ERROR(bntt_compat_ntt_u128((Y), (X), (modulus), (mu), (twiddles), (stages)), \
                          "ntt"))
#define vector_add(c, a, b, m) \
    BNTT_COMPAT_ON_ERROR(bntt_compat_blas_u128(0, (c), (a), (b), 0, (m), 0, BNTT_COMPAT_BLAS_LEN), "vector_add")
#define vector_sub(c, a, b, m) \
    BNTT_COMPAT_ON_ERROR(bntt_compat_blas_u128(1, (c), (a), (b), 0, (m), 0, BNTT_COMPAT_BLAS_LEN), "vector_sub")
#define vector_mul(c, a, b, m, mu) \
    BNTT_COMPAT_ON_ERROR(bntt_compat_blas_u128(2, (c), (a), (b), 0, (m), (mu), BNTT_COMPAT_BLAS_LEN), "vector_mul")
#define axpy(c, a, b, x, m, mu) \
    BNTT_COMPAT_ON_ERROR(bntt_compat_blas_u128(3, (c), (a), (b), (x), (m), (mu), BNTT_COMPAT_BLAS_LEN), "axpy")
#endif

#endif /* BNTT_COMPAT_H */
