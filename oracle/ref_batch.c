/*
 * ref_batch.c -- runs a whole mixed-size list of transforms through the
 * benchNTT reference functions on a pool of POSIX threads.  TEST
 * INFRASTRUCTURE ONLY: it times the CPU baseline of bench.py and is never
 * part of the product.  It holds no reference code: the per-size functions
 * come from the shared objects oracle/Makefile builds from the reference's
 * sources (ref_harness.c: bntt_ref_scratch_new/free, bntt_ref_prep,
 * bntt_ref_ntt_only, bntt_ref_ntt_full), passed in by address.
 *
 * The list is cut into tasks (a run of same-size transforms contiguous in
 * memory); threads take the next task from an atomic counter, so a list
 * ordered largest first packs the threads evenly.  Every thread allocates
 * its working arrays for every size before the start gate; the clock runs
 * from the gate to the end of the last thread, as the reference drivers
 * allocate before their timing loops (src/ntt_avx512.c:535-551).
 *
 * mode 0: ntt() alone per transform, with each size's table expanded once
 *         beforehand -- the reference drivers' timed region
 *         (src/ntt_avx512.c:583-590).
 * mode 1: the whole per-call sequence per transform (ntt_pre, ntt, ntt_post
 *         for the SIMD builds).
 */
#include <pthread.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdlib.h>
#include <time.h>

#define REF_MAX_LOG2N 24

typedef void *(*scratch_new_fn)(void);
typedef void (*scratch_free_fn)(void *);
typedef void (*ntt_only_fn)(void *prep, void *scratch, const uint64_t *x, uint64_t *y);
typedef void (*ntt_full_fn)(const uint64_t *T, uint64_t mh, uint64_t ml, uint64_t muh, uint64_t mul,
                            void *scratch, const uint64_t *x, uint64_t *y);

/* One size's entry points; unused sizes have scratch_new == NULL. */
struct ref_size {
    scratch_new_fn scratch_new;
    scratch_free_fn scratch_free;
    ntt_only_fn ntt_only;
    ntt_full_fn ntt_full;
    void *prep;            /* mode 0: bntt_ref_prep of this size's table */
    const uint64_t *T;     /* mode 1: the table, hi-first pairs */
};

/* `count` transforms of 2^log2n elements, back to back from x and y. */
struct ref_task {
    uint32_t log2n;
    uint32_t count;
    const uint64_t *x;
    uint64_t *y;
};

struct run {
    const struct ref_size *sizes;
    const struct ref_task *tasks;
    size_t ntasks;
    int mode;
    uint64_t mh, ml, muh, mul;
    atomic_size_t next;
    pthread_barrier_t gate;
    double t0;
};

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void *worker(void *arg)
{
    struct run *r = arg;
    void *scratch[REF_MAX_LOG2N + 1] = {0};
    for (int n = 0; n <= REF_MAX_LOG2N; ++n)
        if (r->sizes[n].scratch_new) scratch[n] = r->sizes[n].scratch_new();
    if (pthread_barrier_wait(&r->gate) == PTHREAD_BARRIER_SERIAL_THREAD) r->t0 = now_s();
    for (;;) {
        const size_t i = atomic_fetch_add(&r->next, 1);
        if (i >= r->ntasks) break;
        const struct ref_task *t = &r->tasks[i];
        const struct ref_size *s = &r->sizes[t->log2n];
        const size_t words = (size_t)2 << t->log2n;
        for (uint32_t j = 0; j < t->count; ++j) {
            const uint64_t *x = t->x + words * j;
            uint64_t *y = t->y + words * j;
            if (r->mode == 0) s->ntt_only(s->prep, scratch[t->log2n], x, y);
            else s->ntt_full(s->T, r->mh, r->ml, r->muh, r->mul, scratch[t->log2n], x, y);
        }
    }
    for (int n = 0; n <= REF_MAX_LOG2N; ++n)
        if (scratch[n]) r->sizes[n].scratch_free(scratch[n]);
    return NULL;
}

/* Runs every task on `threads` threads; returns the seconds from the start
 * gate to the end of the last thread, or a negative value on bad input. */
double bntt_ref_run_tasks(const struct ref_size *sizes, const struct ref_task *tasks, size_t ntasks,
                          int mode, uint64_t mh, uint64_t ml, uint64_t muh, uint64_t mul, int threads)
{
    if (threads < 1 || (mode != 0 && mode != 1)) return -1.0;
    for (size_t i = 0; i < ntasks; ++i) {
        const struct ref_task *t = &tasks[i];
        if (t->log2n > REF_MAX_LOG2N || !sizes[t->log2n].scratch_new) return -1.0;
        if (mode == 0 && (!sizes[t->log2n].ntt_only || !sizes[t->log2n].prep)) return -1.0;
        if (mode == 1 && (!sizes[t->log2n].ntt_full || !sizes[t->log2n].T)) return -1.0;
    }
    struct run r = {sizes, tasks, ntasks, mode, mh, ml, muh, mul};
    atomic_init(&r.next, 0);
    pthread_barrier_init(&r.gate, NULL, (unsigned)threads);
    pthread_t *th = malloc(sizeof(pthread_t) * (size_t)threads);
    for (int i = 0; i < threads; ++i) pthread_create(&th[i], NULL, worker, &r);
    for (int i = 0; i < threads; ++i) pthread_join(th[i], NULL);
    const double t = now_s() - r.t0;
    pthread_barrier_destroy(&r.gate);
    free(th);
    return t;
}
