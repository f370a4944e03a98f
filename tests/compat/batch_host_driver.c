/* Mixed-size batches from host memory through the native C ABI
 * (include/bntt.h): several bntt_batch_run_host_async calls queued back to
 * back on different input and output buffers, one bntt_batch_sync, then
 * every job compared with the plan's own single-transform host call
 * (bntt_ntt_forward_host, one transform per call).
 * Usage: batch_host_driver <runs> <jobs per run>; prints "fail: <count>". */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bntt.h"

#define CHECK(call)                                                              \
    do {                                                                         \
        int rc_ = (call);                                                        \
        if (rc_) {                                                               \
            fprintf(stderr, "%s: %d %s\n", #call, rc_, bntt_last_error());       \
            return 1;                                                            \
        }                                                                        \
    } while (0)

#define NSIZES 5
static const unsigned kLog2n[NSIZES] = {4, 7, 10, 12, 16};

int main(int argc, char **argv)
{
    int runs = argc > 1 ? atoi(argv[1]) : 3;
    int per_run = argc > 2 ? atoi(argv[2]) : 40;
    bntt_modulus m = bntt_modulus_ntt_reference();
    bntt_ctx *ctx;
    CHECK(bntt_ctx_create(&ctx, 0, NULL));

    bntt_plan *plans[NSIZES];
    for (int s = 0; s < NSIZES; ++s) {
        size_t n = (size_t)1 << kLog2n[s];
        uint64_t *t = malloc(n * 16);
        CHECK(bntt_fill_uniform_host(t, n, 900 + s, 0, &m, BNTT_LAYOUT_HILO));
        CHECK(bntt_plan_create(ctx, &plans[s], kLog2n[s], &m, t, BNTT_LAYOUT_HILO));
        free(t);
    }
    bntt_batch *batch;
    CHECK(bntt_batch_create(ctx, &batch, plans, NSIZES));

    /* every run: the same job list shape, its own inputs and outputs */
    size_t total = 0;
    unsigned *which = malloc(per_run * sizeof(unsigned));
    size_t *off = malloc(per_run * sizeof(size_t));
    for (int j = 0; j < per_run; ++j) {
        which[j] = (unsigned)((j * 7 + 3) % NSIZES);
        off[j] = total;
        total += (size_t)1 << kLog2n[which[j]];
    }
    uint64_t **x = malloc(runs * sizeof(uint64_t *)), **y = malloc(runs * sizeof(uint64_t *));
    bntt_job **jobs = malloc(runs * sizeof(bntt_job *));
    for (int r = 0; r < runs; ++r) {
        x[r] = malloc(total * 16);
        y[r] = calloc(total, 16);
        CHECK(bntt_fill_uniform_host(x[r], total, 1000 + r, 0, &m, BNTT_LAYOUT_HILO));
        jobs[r] = malloc(per_run * sizeof(bntt_job));
        for (int j = 0; j < per_run; ++j) {
            jobs[r][j].x = x[r] + 2 * off[j];
            jobs[r][j].y = y[r] + 2 * off[j];
            jobs[r][j].plan = which[j];
            jobs[r][j].reserved = 0;
        }
    }
    for (int r = 0; r < runs; ++r) CHECK(bntt_batch_run_host_async(batch, jobs[r], per_run));
    CHECK(bntt_batch_sync(batch));

    size_t fail = 0;
    uint64_t *want = malloc(((size_t)1 << 16) * 16);
    for (int r = 0; r < runs; ++r)
        for (int j = 0; j < per_run; ++j) {
            size_t n = (size_t)1 << kLog2n[which[j]];
            CHECK(bntt_ntt_forward_host(plans[which[j]], want, x[r] + 2 * off[j], 1));
            if (memcmp(want, y[r] + 2 * off[j], n * 16) != 0) ++fail;
        }
    printf("fail: %zu\n", fail);

    free(want);
    for (int r = 0; r < runs; ++r) {
        free(x[r]);
        free(y[r]);
        free(jobs[r]);
    }
    free(x);
    free(y);
    free(jobs);
    free(which);
    free(off);
    bntt_batch_destroy(batch);
    for (int s = 0; s < NSIZES; ++s) bntt_plan_destroy(plans[s]);
    bntt_ctx_destroy(ctx);
    return fail != 0;
}
