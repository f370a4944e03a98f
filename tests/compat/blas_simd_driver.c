/* A driver in the shape of the reference's SIMD BLAS programs
 * (src/blas_avx512.c:478-681, src/blas_avx2.c:525-730) through
 * bntt_compat_simd.h: a = twd_1024 and b = x_1024 packed into vector arrays,
 * the modulus, mu and axpy scalar broadcast into split vectors, the four ops
 * called as vector_add(c, a, b, mh, ml) ... axpy(c, a, b, xh, xl, mh, ml,
 * muh, mul), the results compared with the golden files.  Built with
 * -DBNTT_DRIVER_AVX512 (__m512i, 8 lanes) or without (__m256i, 4 lanes).
 * Prints one line per op with its mismatch count. */
#include <immintrin.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "bntt_compat_simd.h"

typedef __uint128_t uint128_t;
#define INT128(hi, lo) (((uint128_t)(hi) << 64) | (uint128_t)(lo))
#define HI64(x) ((uint64_t)((x) >> 64))
#define LO64(x) ((uint64_t)(x))
#define MODULUS INT128(0xFFFFFFFFFFFFFFFULL, 0xFFFFFFFFFFFFFFC5ULL)
#define MU INT128(0x8000000000000000ULL, 0x1D8ULL)

#ifdef BNTT_DRIVER_AVX512
typedef __m512i vec;
#define LANES 8
#define SET1(x) _mm512_set1_epi64((long long)(x))
#else
typedef __m256i vec;
#define LANES 4
#define SET1(x) _mm256_set1_epi64x((long long)(x))
#endif

static int compare(const char *dir, const char *name, const vec *c)
{
    uint64_t ver[2048];
    char path[4096];
    snprintf(path, sizeof(path), "%s/%s_1024.txt", dir, name);
    if (bntt_load_pairs_text(path, ver, 1024)) return -1;
    const uint64_t *got = (const uint64_t *)c;
    int fail = 0;
    for (int i = 0; i < 2048; i++)
        if (got[i] != ver[i]) fail++;
    return fail;
}

int main(int argc, char **argv)
{
    if (argc < 2) return 2;
    uint128_t m = MODULUS, mu = MU, scalar = INT128(208488538572646751ULL, 12808410693871070164ULL);
    vec mh = SET1(HI64(m)), ml = SET1(LO64(m)), muh = SET1(HI64(mu)), mul = SET1(LO64(mu));
    vec sh = SET1(HI64(scalar)), sl = SET1(LO64(scalar));
    uint64_t *twd_s = malloc(sizeof(uint64_t) * 2048), *x_s = malloc(sizeof(uint64_t) * 2048);
    if (bntt_load_reference_data(argv[1], "twd", twd_s, 1024) || bntt_load_reference_data(argv[1], "x", x_s, 1024))
        return 1;
    /* the driver's packing: lane i of vector j holds word i + j * LANES */
    vec *tempa = aligned_alloc(64, sizeof(vec) * (2048 / LANES));
    vec *tempb = aligned_alloc(64, sizeof(vec) * (2048 / LANES));
    for (int j = 0; j < 2048 / LANES; j++)
        for (int i = 0; i < LANES; i++) {
            ((uint64_t *)&tempa[j])[i] = twd_s[i + j * LANES];
            ((uint64_t *)&tempb[j])[i] = x_s[i + j * LANES];
        }
    vec *add = aligned_alloc(64, sizeof(vec) * (2048 / LANES));
    vec *sub = aligned_alloc(64, sizeof(vec) * (2048 / LANES));
    vec *mlt = aligned_alloc(64, sizeof(vec) * (2048 / LANES));
    vec *ax = aligned_alloc(64, sizeof(vec) * (2048 / LANES));
    vector_add(add, tempa, tempb, mh, ml);
    vector_sub(sub, tempa, tempb, mh, ml);
    vector_mul(mlt, tempa, tempb, mh, ml, muh, mul);
    axpy(ax, tempa, tempb, sh, sl, mh, ml, muh, mul);
    int f0 = compare(argv[1], "vvadd", add), f1 = compare(argv[1], "vvsub", sub);
    int f2 = compare(argv[1], "vvmul", mlt), f3 = compare(argv[1], "axpy", ax);
    printf("vvadd fail: %d\nvvsub fail: %d\nvvmul fail: %d\naxpy fail: %d\n", f0, f1, f2, f3);
    bntt_compat_shutdown();
    return (f0 || f1 || f2 || f3) != 0;
}
