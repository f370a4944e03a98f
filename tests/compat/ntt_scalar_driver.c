/* A driver in the shape of the reference's scalar NTT program
 * (src/ntt_scalar.c:630-719) that includes bntt_compat.h instead of
 * defining ntt(): loads data/<kind>_N.txt, calls ntt() 3 times, compares with
 * ver_N and prints "fail: K" as the reference does (:685-701).
 * Build: gcc -Dstages=S -I include ntt_scalar_driver.c -L... -lbntt */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "bntt_compat.h"

typedef __uint128_t uint128_t;
#ifndef stages
#define stages 10
#endif
#define N (1 << stages)
#define INT128(hi, lo) (((uint128_t)(hi) << 64) | (uint128_t)(lo))

int main(int argc, char **argv)
{
    if (argc < 2) return 2;
    uint128_t mu = INT128(9223372036854775808ULL, 5752ULL);
    uint128_t modulus = INT128(1152921504606846975ULL, 18446744073709550897ULL);
    uint64_t *twd_s = malloc(sizeof(uint64_t) * 2 * N), *x_s = malloc(sizeof(uint64_t) * 2 * N),
             *ver_s = malloc(sizeof(uint64_t) * 2 * N);
    uint128_t *twd = malloc(sizeof(uint128_t) * N), *x = malloc(sizeof(uint128_t) * N),
              *y = malloc(sizeof(uint128_t) * N), *as0 = malloc(sizeof(uint128_t) * N),
              *as1 = malloc(sizeof(uint128_t) * N);
    if (bntt_load_reference_data(argv[1], "twd", twd_s, N) || bntt_load_reference_data(argv[1], "x", x_s, N) ||
        bntt_load_reference_data(argv[1], "ver", ver_s, N)) {
        printf("load error: %s\n", bntt_last_error());
        return 1;
    }
    for (int i = 0; i < N; i++) {
        twd[i] = INT128(twd_s[2 * i], twd_s[2 * i + 1]);
        x[i] = INT128(x_s[2 * i], x_s[2 * i + 1]);
    }
    for (int j = 0; j < 3; j++) ntt(y, x, modulus, mu, twd, as0, as1);
    int fail = 0;
    for (int i = 0; i < N; i++)
        if (y[i] != INT128(ver_s[2 * i], ver_s[2 * i + 1])) fail++;
    printf("%d fail: %d\n", N, fail);
    bntt_compat_shutdown();
    return fail != 0;
}
