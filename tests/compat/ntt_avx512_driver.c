/* A driver in the shape of the reference's AVX-512 NTT program
 * (src/ntt_avx512.c:530-635): ntt_pre with the permutation vectors, the
 * 16-argument ntt and ntt_post on the driver's __m512i scratch arrays, through
 * bntt_compat_simd.h.  Prints "N fail: K". */
#include <immintrin.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "bntt_compat_simd.h"

typedef __uint128_t uint128_t;
#ifndef stages
#define stages 10
#endif
#define N (1 << stages)
#define operations (N / 16)
#define v (N / 8)
#define INT128(hi, lo) (((uint128_t)(hi) << 64) | (uint128_t)(lo))

int main(int argc, char **argv)
{
    if (argc < 2) return 2;
    __m512i *twdh = aligned_alloc(64, sizeof(__m512i) * (stages * operations + 1));
    __m512i *twdl = aligned_alloc(64, sizeof(__m512i) * (stages * operations + 1));
    __m512i *tempx = aligned_alloc(64, sizeof(__m512i) * ((N * 2) / 8));
    __m512i mh_512, ml_512, muh_512, mul_512;
    __m512i permutehi, permutelo;
    __m512i *xh = aligned_alloc(64, sizeof(__m512i) * v), *xl = aligned_alloc(64, sizeof(__m512i) * v);
    __m512i *ash = aligned_alloc(64, sizeof(__m512i) * v), *asl = aligned_alloc(64, sizeof(__m512i) * v);
    __m512i *th = aligned_alloc(64, sizeof(__m512i) * v), *tl = aligned_alloc(64, sizeof(__m512i) * v);
    __m512i *as = aligned_alloc(64, sizeof(__m512i) * ((N * 2) / 8));
    uint64_t *y = malloc(sizeof(uint64_t) * N * 2);
    uint128_t mu = INT128(9223372036854775808ULL, 5752ULL);
    uint128_t modulus = INT128(1152921504606846975ULL, 18446744073709550897ULL);
    uint64_t *twd_s = malloc(sizeof(uint64_t) * N * 2), *x_s = malloc(sizeof(uint64_t) * N * 2),
             *ver_s = malloc(sizeof(uint64_t) * N * 2);
    if (bntt_load_reference_data(argv[1], "twd", twd_s, N) || bntt_load_reference_data(argv[1], "x", x_s, N) ||
        bntt_load_reference_data(argv[1], "ver", ver_s, N)) {
        printf("load error: %s\n", bntt_last_error());
        return 1;
    }
    for (int j = 0; j < 3; j++) {
        ntt_pre(x_s, twd_s, modulus, mu, tempx, twdh, twdl, &mh_512, &ml_512, &muh_512, &mul_512,
                &permutehi, &permutelo);
        ntt(tempx, twdh, twdl, mh_512, ml_512, muh_512, mul_512, permutehi, permutelo, xh, xl, ash, asl, th,
            tl, as);
        ntt_post(y, as);
    }
    int fail = 0;
    for (int i = 0; i < N * 2; i++)
        if (y[i] != ver_s[i]) fail++;
    printf("%d fail: %d\n", N, fail);
    bntt_compat_shutdown();
    return fail != 0;
}
