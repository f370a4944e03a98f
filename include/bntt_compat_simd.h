/*
 * bntt_compat_simd.h -- the benchNTT reference's AVX2 / AVX-512 call shapes
 * on libbntt.
 *
 * The SIMD drivers run a transform in three calls (src/ntt_avx512.c:386-528,
 * src/ntt_avx2.c:507-655):
 *   ntt_pre(X, twiddles, modulus, mu, tempx, twdh, twdl, ...)   prepare
 *   ntt(tempx, twdh, twdl, ..., as)                             compute
 *   ntt_post(Y, as)                                             store
 * and run the BLAS ops on __m256i / __m512i arrays holding hi-first u64 pairs
 * (src/blas_avx512.c:401-476).  Including this header instead of defining
 * those functions maps them onto the GPU: ntt_pre makes the table
 * device-resident and records X, ntt runs the transform and writes the output
 * into `as` (2N u64, hi-first pairs: the same bytes ntt_post stores), ntt_post
 * copies `as` to Y.  The vector-register arguments (tempx, twdh, mh_512, the
 * permutation vectors, ...) are accepted and ignored.  N = 2^stages from the
 * program's `stages` macro.  Works for both the 4-lane and 8-lane drivers.
 * The BLAS macros take the driver's vector arrays as hi-first pairs, length
 * 1024, with the modulus / mu / scalar given as the split vectors the driver
 * passes: their first lane carries the value.
 */
#ifndef BNTT_COMPAT_SIMD_H
#define BNTT_COMPAT_SIMD_H

#include <string.h>

#define BNTT_COMPAT_NO_MACROS
#include "bntt_compat.h"
#undef BNTT_COMPAT_NO_MACROS

/* the last of the arguments (ntt's output vector array), 14 or 16 of them */
#define BNTT_ARG16_(a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11, a12, a13, a14, a15, a16, ...) a16
#define BNTT_ARG14_(a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11, a12, a13, a14, ...) a14
#define BNTT_NARGS_(...) BNTT_NARGS_I_(__VA_ARGS__, 16, 15, 14, 13, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2, 1)
#define BNTT_NARGS_I_(a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11, a12, a13, a14, a15, a16, n, ...) n
#define BNTT_CAT_(a, b) BNTT_CAT_I_(a, b)
#define BNTT_CAT_I_(a, b) a##b
#define BNTT_LAST_14_(...) BNTT_ARG14_(__VA_ARGS__, 0)
#define BNTT_LAST_16_(...) BNTT_ARG16_(__VA_ARGS__, 0)
#define BNTT_LAST_(...) BNTT_CAT_(BNTT_LAST_, BNTT_CAT_(BNTT_NARGS_(__VA_ARGS__), _))(__VA_ARGS__)

/* first 64-bit lane of a vector value, as an unsigned integer (copied out
 * with memcpy: reading a vector object through a uint64_t pointer would break
 * the aliasing rules) */
static inline uint64_t bntt_compat_lane0_(const void *p)
{
    uint64_t r;
    memcpy(&r, p, sizeof r);
    return r;
}
#define BNTT_LANE0_(v) (__extension__({ __typeof__(v) bntt_v_ = (v); bntt_compat_lane0_(&bntt_v_); }))
#define BNTT_U128_(hi, lo) (((bntt_uint128)BNTT_LANE0_(hi) << 64) | (bntt_uint128)BNTT_LANE0_(lo))

/* arguments that are not used are named in an unevaluated sizeof only */
#define BNTT_UNUSED_(...) ((void)sizeof(bntt_compat_touch_(0, __VA_ARGS__)))
static inline int bntt_compat_touch_(int first, ...) { return first; }
#define ntt_pre(X, twiddles, modulus, mu, ...)                                                    \
    (BNTT_UNUSED_(__VA_ARGS__),                                                                 \
     BNTT_COMPAT_ON_ERROR(bntt_compat_simd_pre((X), (twiddles), (modulus), (mu), (stages)), "ntt_pre"))
#define ntt(...) \
    (BNTT_UNUSED_(__VA_ARGS__), BNTT_COMPAT_ON_ERROR(bntt_compat_simd_run((void *)(BNTT_LAST_(__VA_ARGS__))), "ntt"))
#define ntt_post(Y, as) BNTT_COMPAT_ON_ERROR(bntt_compat_simd_post((Y), (const void *)(as)), "ntt_post")

#define vector_add(c, a, b, mh, ml)                                                               \
    BNTT_COMPAT_ON_ERROR(bntt_compat_blas_pairs(0, (uint64_t *)(c), (const uint64_t *)(a),      \
                                                (const uint64_t *)(b), 0, BNTT_U128_(mh, ml), 0,  \
                                                1024), "vector_add")
#define vector_sub(c, a, b, mh, ml)                                                               \
    BNTT_COMPAT_ON_ERROR(bntt_compat_blas_pairs(1, (uint64_t *)(c), (const uint64_t *)(a),      \
                                                (const uint64_t *)(b), 0, BNTT_U128_(mh, ml), 0,  \
                                                1024), "vector_sub")
#define vector_mul(c, a, b, mh, ml, muh, mul)                                                     \
    BNTT_COMPAT_ON_ERROR(bntt_compat_blas_pairs(2, (uint64_t *)(c), (const uint64_t *)(a),      \
                                                (const uint64_t *)(b), 0, BNTT_U128_(mh, ml),     \
                                                BNTT_U128_(muh, mul), 1024), "vector_mul")
#define axpy(c, a, b, xh, xl, mh, ml, muh, mul)                                                   \
    BNTT_COMPAT_ON_ERROR(bntt_compat_blas_pairs(3, (uint64_t *)(c), (const uint64_t *)(a),      \
                                                (const uint64_t *)(b), BNTT_U128_(xh, xl),        \
                                                BNTT_U128_(mh, ml), BNTT_U128_(muh, mul), 1024), "axpy")

#endif /* BNTT_COMPAT_SIMD_H */
