/* A driver in the shape of the reference's scalar BLAS program
 * (src/blas_scalar.c:610-780) through bntt_compat.h: a = twd_1024,
 * b = x_1024, the 4 ops, compared with the golden files; prints one line per
 * op with its mismatch count. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "bntt_compat.h"

typedef __uint128_t uint128_t;
#define INT128(hi, lo) (((uint128_t)(hi) << 64) | (uint128_t)(lo))
#define MODULUS INT128(0xFFFFFFFFFFFFFFFULL, 0xFFFFFFFFFFFFFFC5ULL)
#define MU INT128(0x8000000000000000ULL, 0x1D8ULL)

static int compare(const char *dir, const char *name, const uint128_t *c)
{
    uint64_t ver[2048];
    char path[4096];
    snprintf(path, sizeof(path), "%s/%s_1024.txt", dir, name);
    if (bntt_load_pairs_text(path, ver, 1024)) return -1;
    int fail = 0;
    for (int i = 0; i < 1024; i++)
        if (c[i] != INT128(ver[2 * i], ver[2 * i + 1])) fail++;
    return fail;
}

int main(int argc, char **argv)
{
    if (argc < 2) return 2;
    uint128_t m = MODULUS, mu = MU, scalar = INT128(208488538572646751ULL, 12808410693871070164ULL);
    uint64_t a_s[2048], b_s[2048];
    if (bntt_load_reference_data(argv[1], "twd", a_s, 1024) || bntt_load_reference_data(argv[1], "x", b_s, 1024))
        return 1;
    static uint128_t a[1024], b[1024], add[1024], sub[1024], mul[1024], ax[1024];
    for (int i = 0; i < 1024; i++) {
        a[i] = INT128(a_s[2 * i], a_s[2 * i + 1]);
        b[i] = INT128(b_s[2 * i], b_s[2 * i + 1]);
    }
    vector_add(add, a, b, m);
    vector_sub(sub, a, b, m);
    vector_mul(mul, a, b, m, mu);
    axpy(ax, a, b, scalar, m, mu);
    int f0 = compare(argv[1], "vvadd", add), f1 = compare(argv[1], "vvsub", sub);
    int f2 = compare(argv[1], "vvmul", mul), f3 = compare(argv[1], "axpy", ax);
    printf("vvadd fail: %d\nvvsub fail: %d\nvvmul fail: %d\naxpy fail: %d\n", f0, f1, f2, f3);
    bntt_compat_shutdown();
    return (f0 || f1 || f2 || f3) != 0;
}
