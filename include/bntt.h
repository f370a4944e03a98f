/*
 * bntt.h -- C ABI of libbntt, a B200 (sm_100a) implementation of benchNTT's
 * 128-bit modular NTT and BLAS-style vector operations.
 *
 * Results are bit-identical to the reference scalar path
 * (src/ntt_scalar.c, src/blas_scalar.c of benchNTT) on the same inputs.
 *
 * Conventions
 *   - Every function returns an int status (bntt_status).  On failure
 *     bntt_last_error() gives a message for the calling thread.  Nothing
 *     calls exit() (the reference loader does, src/config.c:11-14).
 *   - 128-bit scalars cross the ABI as bntt_u128 {hi, lo}.
 *   - Element buffers hold 16-byte residues in one of two layouts:
 *       BNTT_LAYOUT_HILO  u64 pairs, high word first: the layout of the
 *                         reference's data files and SIMD entry points
 *                         (src/config.c:29-30, src/ntt_avx512.c:386)
 *       BNTT_LAYOUT_U128  native little-endian unsigned __int128: the
 *                         reference scalar API's uint128_t arrays
 *                         (src/ntt_scalar.c:582)
 *   - "_dev" functions take device pointers and are asynchronous on the
 *     context's stream; "_host" functions take host pointers and return when
 *     the result is in host memory.  Device pointers must be 16-byte aligned.
 *   - Inputs are residues in [0, q] as in the reference (its data are in
 *     [0, q); intermediate values may equal q).  With the default arithmetic
 *     the results equal the reference's for every such input; with
 *     BNTT_ARITH_REFERENCE they equal it for any 128-bit input.
 *   - A context is used by one host thread at a time.
 */
#ifndef BNTT_H
#define BNTT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BNTT_VERSION_MAJOR 0
#define BNTT_VERSION_MINOR 1

typedef enum bntt_status {
    BNTT_OK = 0,
    BNTT_EINVAL = 1,     /* bad argument: null pointer, size, log2n, alignment, layout */
    BNTT_ENOMEM = 2,     /* device or pinned-host allocation failed */
    BNTT_EBUDGET = 3,    /* request does not fit the context's HBM budget */
    BNTT_ECUDA = 4,      /* CUDA runtime error; text in bntt_last_error() */
    BNTT_ETIMEOUT = 5,   /* a bounded device-side wait gave up */
    BNTT_ENODEV = 6,     /* no usable CUDA device */
    BNTT_EBUSY = 7       /* object is in use (e.g. server running) */
} bntt_status;

typedef struct bntt_u128 {
    uint64_t hi;
    uint64_t lo;
} bntt_u128;

/* Modulus and Barrett constant with the reference's MBITS = 124
 * (src/ntt_scalar.c:28-29): mu = floor(2^251 / q). */
typedef struct bntt_modulus {
    bntt_u128 q;
    bntt_u128 mu;
} bntt_modulus;

#define BNTT_LAYOUT_HILO 0
#define BNTT_LAYOUT_U128 1

/* Arithmetic selection.
 * AUTO: a pseudo-Mersenne multiply when q = 2^124 - k (k < 2^28) and
 *       mu = floor(2^251/q) -- both reference moduli and the NTT-friendly
 *       primes of bntt_ntt_prime -- for which the
 *       reference's Barrett reduction provably returns a*b mod q exactly
 *       for operands below 2^124 (every residue); otherwise the replica
 *       below.  Inputs at or above 2^124 need REFERENCE.
 * REFERENCE: a word-for-word replica of mulmod128 (src/ntt_scalar.c:173-199),
 *       identical to the reference for any 128-bit operands. */
#define BNTT_ARITH_AUTO 0
#define BNTT_ARITH_REFERENCE 1

typedef struct bntt_ctx bntt_ctx;
typedef struct bntt_plan bntt_plan;
typedef struct bntt_batch bntt_batch;

/* ------------------------------------------------------------------ basics */
const char *bntt_version(void);
const char *bntt_last_error(void);
const char *bntt_status_string(int status);

/* 1 if `m` takes the fast multiply under BNTT_ARITH_AUTO, else 0. */
int bntt_modulus_is_fast(const bntt_modulus *m);

/* The moduli the reference programs use: the NTT drivers' q = 2^124 - 719
 * (src/ntt_scalar.c:632-633) and the BLAS drivers' q = 2^124 - 59
 * (src/blas_scalar.c:23-30). */
bntt_modulus bntt_modulus_ntt_reference(void);
bntt_modulus bntt_modulus_blas_reference(void);

/* Context: device, stream, allocator accounting and HBM budget.
 * `stream` is a cudaStream_t to run on, or NULL for a new non-blocking one. */
int bntt_ctx_create(bntt_ctx **ctx, int device, void *stream);
int bntt_ctx_destroy(bntt_ctx *ctx);
int bntt_ctx_synchronize(bntt_ctx *ctx);
void *bntt_ctx_stream(bntt_ctx *ctx);
int bntt_ctx_set_arith(bntt_ctx *ctx, int arith);
/* Cap on device bytes the context may hold (0 = no cap). */
int bntt_ctx_set_hbm_budget(bntt_ctx *ctx, size_t bytes);
size_t bntt_ctx_hbm_in_use(bntt_ctx *ctx);
int bntt_ctx_sm_count(bntt_ctx *ctx);

/* Device buffers charged to the context's budget. */
int bntt_dev_alloc(bntt_ctx *ctx, void **ptr, size_t bytes);
int bntt_dev_free(bntt_ctx *ctx, void *ptr);
int bntt_copy_h2d(bntt_ctx *ctx, void *dst_dev, const void *src_host, size_t bytes);
int bntt_copy_d2h(bntt_ctx *ctx, void *dst_host, const void *src_dev, size_t bytes);

/* Seeded uniform residues in [0, q) (counter-based SplitMix64; element i
 * depends only on seed and offset + i).  Host and device fills agree. */
int bntt_fill_uniform_host(void *buf, size_t count, uint64_t seed, uint64_t offset,
                           const bntt_modulus *m, int layout);
int bntt_fill_uniform_dev(bntt_ctx *ctx, void *buf_dev, size_t count, uint64_t seed,
                          uint64_t offset, const bntt_modulus *m, int layout);

/* -------------------------------------------------------------------- NTT */
/* A plan holds one transform size, modulus and twiddle table, uploaded once
 * and kept in HBM (what ntt_pre prepares per call in the SIMD drivers,
 * src/ntt_avx512.c:386-460).  `twiddles` is a host array of 2^log2n
 * elements; entry 0 is never read (src/ntt_scalar.c:586-622).
 * 1 <= log2n <= 24. */
int bntt_plan_create(bntt_ctx *ctx, bntt_plan **plan, unsigned log2n, const bntt_modulus *m,
                     const void *twiddles, int layout);
/* Same, with the table already in device memory.  A BNTT_LAYOUT_U128 table
 * is used in place (not copied; it must outlive the plan); a HILO table is
 * copied once into plan-owned memory in limb order. */
int bntt_plan_create_dev(bntt_ctx *ctx, bntt_plan **plan, unsigned log2n,
                         const bntt_modulus *m, const void *twiddles_dev, int layout);
int bntt_plan_destroy(bntt_plan *plan);
unsigned bntt_plan_log2n(const bntt_plan *plan);

/* NTT-friendly prime mode.  The reference's tables are arbitrary constants
 * (data/twd_N.txt; 2^124 - 719 has 2-power roots of unity only up to order
 * 16), but ntt()
 * takes modulus, mu and table at run time (src/ntt_scalar.c:582), so the same
 * network computes the negacyclic transform
 *     Y[i] = sum_j X[j] * psi^((2*brv(i) + 1) * j)  mod q
 * (outputs in bit-reversed order; brv reverses log2 N bits) when q has
 * 2N | q - 1, psi is a primitive 2N-th root of unity and
 *     T[k] = psi^brv(k)  (k = 1..N-1;  T[0] = 1, never read).
 *
 * bntt_ntt_prime: q = 2^124 - (c*2^log2_order - 1) for the smallest c >= 1
 *   that passes a Miller-Rabin test to the first 24 prime bases, with
 *   mu = floor(2^251/q); k = 2^124 - q < 2^28, so the default fast multiply
 *   applies.  EINVAL if no such prime exists.
 * bntt_root_of_unity: a primitive 2^log2_order-th root of unity mod q
 *   (g^((q-1)/2^log2_order) for the smallest g >= 2 of that exact order).
 * bntt_powmod: a^e mod q (host, exact) for 2^123 < q < 2^124.
 * bntt_twiddles_negacyclic: the table above on the host (2^log2n elements).
 * bntt_plan_create_negacyclic: a plan whose table is generated on the device
 *   from psi (no host table, no upload); q must take the fast multiply. */
int bntt_ntt_prime(unsigned log2_order, bntt_modulus *m);
int bntt_root_of_unity(const bntt_modulus *m, unsigned log2_order, bntt_u128 *root);
int bntt_powmod(const bntt_modulus *m, bntt_u128 a, bntt_u128 e, bntt_u128 *out);
int bntt_twiddles_negacyclic(const bntt_modulus *m, unsigned log2n, bntt_u128 psi, void *table,
                             int layout);
int bntt_plan_create_negacyclic(bntt_ctx *ctx, bntt_plan **plan, unsigned log2n,
                                const bntt_modulus *m, bntt_u128 psi, int layout);

/* Forward transform of `batch` contiguous inputs (replaces ntt(),
 * src/ntt_scalar.c:582).  y may equal x.  One launch for 2^log2n <= 1024,
 * one launch per HBM pass above. */
int bntt_ntt_forward_dev(bntt_plan *plan, void *y, const void *x, size_t batch);
/* Host-pointer form: copies in, transforms, copies out (the reference's
 * call shape; pipelined over chunks of the batch). */
int bntt_ntt_forward_host(bntt_plan *plan, void *y, const void *x, size_t batch);
/* Inverse of the plan's forward transform: x = ntt^-1(y) for `batch`
 * contiguous vectors (x may equal y).  The reference has no inverse; this
 * one runs the forward network's stages in reverse order with inverse
 * (Gentleman-Sande) butterflies and the inverted table, then multiplies by
 * N^-1, so ntt^-1(ntt(x)) = x for every table whose entries are invertible
 * mod a prime q.  With a negacyclic plan it is the inverse negacyclic NTT.
 * Results are canonical residues in [0, q).  Needs the fast multiply
 * (q = 2^124 - k, k < 2^28, mu = floor(2^251/q)); the inverse table is
 * built on the first call (EINVAL if a twiddle is 0 mod q or q is not
 * prime). */
int bntt_ntt_inverse_dev(bntt_plan *plan, void *x, const void *y, size_t batch);

/* Transform fused with the pointwise product that follows it in a
 * polynomial-multiply pipeline:  y_t = vector_mul(ntt(x_t), b_t)
 * (src/ntt_scalar.c:582 then src/blas_scalar.c:594) under the plan's
 * modulus, with the product applied as the last pass stores, so the
 * transform's output never makes a second trip through HBM.
 * b_per_transform = 1: b holds `batch` vectors of 2^log2n elements, one per
 * transform; 0: one vector applied to every transform.  y may equal x; b may
 * equal x but must not overlap y.  Same layout for x, y and b. */
int bntt_ntt_forward_mul_dev(bntt_plan *plan, void *y, const void *x, const void *b,
                             int b_per_transform, size_t batch);

/* ------------------------------------------------------- mixed-size batch */
/* One transform of a mixed batch: x and y are device pointers (or host
 * pointers for bntt_batch_run_host) to 2^log2n elements of plans[plan]. */
typedef struct bntt_job {
    const void *x;
    void *y;
    uint32_t plan;
    uint32_t reserved;
} bntt_job;

/* A batch object runs many independent transforms of uneven sizes in one
 * persistent work-queue kernel.  `plans` must all use the same modulus and
 * layout and outlive the batch. */
int bntt_batch_create(bntt_ctx *ctx, bntt_batch **batch, bntt_plan *const *plans,
                      size_t nplans);
int bntt_batch_destroy(bntt_batch *batch);
/* Device pointers, asynchronous.  The schedule (work items, their order and
 * the per-size kernel shapes) is rebuilt only when the job list changes: a
 * new list is built on the host and copied while earlier launches run, then
 * launched; a list run again is replayed from a CUDA graph.  Only a list
 * larger than any before (its buffers grow) waits for the device. */
int bntt_batch_run_dev(bntt_batch *batch, const bntt_job *jobs, size_t count);
/* Host pointers: inputs copied in, batch run, outputs copied back. */
int bntt_batch_run_host(bntt_batch *batch, const bntt_job *jobs, size_t count);
/* The same, returning once the copies and launches are queued.  The host
 * buffers must stay valid, the inputs unchanged and the outputs unread until
 * bntt_batch_sync.  Back-to-back calls overlap: one call's output copies run
 * under the next call's input copies.  No counterpart in the reference (its
 * functions are synchronous, src/ntt_scalar.c:582). */
int bntt_batch_run_host_async(bntt_batch *batch, const bntt_job *jobs, size_t count);
/* Waits for every bntt_batch_run_host_async call so far; BNTT_ETIMEOUT if a
 * device-side wait of any of them gave up. */
int bntt_batch_sync(bntt_batch *batch);
/* The same jobs, each launched on its own (one launch per transform of at
 * most 1024 points, one per HBM pass above): the per-call path the
 * persistent kernel is compared with.  Device pointers, asynchronous. */
int bntt_batch_run_percall_dev(bntt_batch *batch, const bntt_job *jobs, size_t count);
/* Inverse transforms of a job list (the inverse of bntt_batch_run_dev for
 * each job: x = ntt^-1(y) with job.x the input and job.y the output), in one
 * persistent launch like the forward batch.  The inverse of the reference's
 * network has no counterpart in the reference; see bntt_ntt_inverse_dev for
 * its definition.  Needs the fast multiply and the default arithmetic; the
 * plans' inverse tables are built on the first call. */
int bntt_batch_run_inverse_dev(bntt_batch *batch, const bntt_job *jobs, size_t count);

/* Same as bntt_batch_run_dev, but allocates no device memory: for callers
 * that cannot call cudaMalloc when they submit work (device memory owned by
 * another allocator's pool, latency-critical paths where an allocation would
 * stall the device, services that must not hit out-of-memory after start-up).
 * No counterpart in the reference, which runs on the CPU only.
 * Its scratch (work items, job descriptors, control words) lives in one
 * 4 MiB array inside the library, present on every GPU that loads it until
 * the process exits; a job list whose schedule needs more (roughly 70,000
 * transforms) is rejected with BNTT_EINVAL.  The first call through a context
 * looks up that array's device address (again for a context created after a
 * device reset).  The schedule is copied from host memory that is released
 * when the call returns, so the call is refused with BNTT_EINVAL while the
 * context's stream is being captured into a CUDA graph.  Every call reuses
 * the same array: the control words are cleared on each call, and calls whose
 * work overlaps on the GPU (several streams, contexts or threads on one
 * device) race -- serialise them.  Asynchronous on the context's stream. */
int bntt_batch_run_dev_noalloc(bntt_batch *batch, const bntt_job *jobs, size_t count);
/* Status of the batch's latest run: BNTT_OK, or BNTT_ETIMEOUT if a
 * device-side wait gave up (synchronises the stream).  After
 * bntt_batch_run_dev_noalloc it reads the error word that run left in the
 * shared array, so read it before another no-allocation call on the same
 * device reuses the array. */
int bntt_batch_status(bntt_batch *batch);
/* Fault injection for tests of the failure path: the next
 * bntt_batch_run_dev makes the waits of later HBM passes unreachable and gives
 * up after `poll_limit` polls (about 100 ns each); the kernel still ends, and
 * bntt_batch_status() then reports BNTT_ETIMEOUT.  One run only. */
int bntt_batch_inject_wait_timeout(bntt_batch *batch, uint32_t poll_limit);
/* Kernel launches the last run issued (graph replays count their kernels). */
size_t bntt_batch_last_launches(bntt_batch *batch);

/* ------------------------------------------------------------------- BLAS */
/* Element-wise mod-q operations over `len` elements (the reference fixes
 * len = 1024, src/blas_scalar.c:580):
 *   vvadd  c[i] = addmod(a[i], b[i])            src/blas_scalar.c:578
 *   vvsub  c[i] = submod(a[i], b[i])            src/blas_scalar.c:586
 *   vvmul  c[i] = mulmod(a[i], b[i])            src/blas_scalar.c:594
 *   axpy   c[i] = addmod(a[i], mulmod(x, b[i])) src/blas_scalar.c:602
 * c may alias a or b. */
int bntt_vvadd_dev(bntt_ctx *ctx, void *c, const void *a, const void *b, size_t len,
                   const bntt_modulus *m, int layout);
int bntt_vvsub_dev(bntt_ctx *ctx, void *c, const void *a, const void *b, size_t len,
                   const bntt_modulus *m, int layout);
int bntt_vvmul_dev(bntt_ctx *ctx, void *c, const void *a, const void *b, size_t len,
                   const bntt_modulus *m, int layout);
int bntt_axpy_dev(bntt_ctx *ctx, void *c, const void *a, const void *b, bntt_u128 x, size_t len,
                  const bntt_modulus *m, int layout);

int bntt_vvadd_host(bntt_ctx *ctx, void *c, const void *a, const void *b, size_t len,
                    const bntt_modulus *m, int layout);
int bntt_vvsub_host(bntt_ctx *ctx, void *c, const void *a, const void *b, size_t len,
                    const bntt_modulus *m, int layout);
int bntt_vvmul_host(bntt_ctx *ctx, void *c, const void *a, const void *b, size_t len,
                    const bntt_modulus *m, int layout);
int bntt_axpy_host(bntt_ctx *ctx, void *c, const void *a, const void *b, bntt_u128 x,
                   size_t len, const bntt_modulus *m, int layout);

/* Kernel launches issued by this context since creation (all entry points). */
uint64_t bntt_ctx_launch_count(bntt_ctx *ctx);

/* ------------------------------------------------------------ several GPUs */
/* The transforms of a job list are independent, so several devices share one
 * list with no data exchange: the list is split by cost and each device runs
 * its part on its own batch.  The reference has no multi-device path (one
 * transform per call on one CPU core, src/ntt_scalar.c:582).
 *
 * bntt_split_by_cost: owner[i] in [0, parts) for each job of size 2^log2n[i]:
 *   jobs in decreasing cost (N/2 * log2 N butterflies, ties by index), each to
 *   the part with the least work so far (ties to the lower part).  Needs no
 *   GPU; every caller splitting the same sizes gets the same owners.
 * bntt_multi_create: one batch per device, each created on its own context
 *   with its own plans (every device holds its own copy of the tables; no
 *   device reads another's memory).  The batches must list plans of the same
 *   sizes in the same order; a job's `plan` indexes that list.
 * bntt_multi_split: bntt_split_by_cost over the job list's plan sizes.
 * bntt_multi_run_host: splits the list, queues each part from host buffers on
 *   its device (bntt_batch_run_host_async), then waits for all of them; the
 *   outputs are in host memory when it returns.  BNTT_ETIMEOUT if a
 *   device-side wait of any part gave up. */
typedef struct bntt_multi bntt_multi;
int bntt_split_by_cost(const uint32_t *log2n, size_t count, uint32_t parts, uint32_t *owner);
int bntt_multi_create(bntt_multi **multi, bntt_batch *const *batches, size_t n);
int bntt_multi_destroy(bntt_multi *multi);
int bntt_multi_split(bntt_multi *multi, const bntt_job *jobs, size_t count, uint32_t *owner);
int bntt_multi_run_host(bntt_multi *multi, const bntt_job *jobs, size_t count);

/* ---------------------------------------------------------------- serving */
/* A request loop with continuous batching.  Requests (forward NTTs of any
 * plan size, vvmul, axpy) name device-resident operands; the server admits
 * them in arrival order while its output arena (the HBM budget) has room,
 * packs the admitted NTTs of each launch into one persistent-kernel run and
 * the BLAS ops next to it, and keeps up to `slots` launches in flight on
 * separate streams, so requests that arrive while others run are admitted as
 * slots and memory free up and their work overlaps on the device.  Each
 * completion carries its output (in the arena, until released) and the
 * arrival / admission / completion times.  The reference has no serving
 * path (one call per process, src/ntt_scalar.c:630). */
typedef struct bntt_server bntt_server;

typedef struct bntt_server_config {
    size_t hbm_budget;   /* bytes of the output arena; 0 = 32 GiB */
    uint32_t slots;      /* launches in flight at once; 0 = 4 */
    uint32_t max_batch;  /* most requests per launch; 0 = 4096 */
} bntt_server_config;

#define BNTT_REQ_NTT 0
#define BNTT_REQ_VVMUL 1
#define BNTT_REQ_AXPY 2

typedef struct bntt_request {
    uint32_t kind;      /* BNTT_REQ_* */
    uint32_t plan;      /* NTT: index into the server's plans */
    uint64_t len;       /* vvmul / axpy: number of elements */
    const void *x;      /* NTT input, or BLAS operand a (device) */
    const void *b;      /* BLAS operand b (device) */
    bntt_u128 scalar;   /* axpy: c = a + scalar * b */
    uint64_t tag;       /* returned in the completion */
    double t_arrive;    /* server clock (s); <= 0 means "now" at submit */
} bntt_request;

typedef struct bntt_completion {
    uint64_t tag;
    void *y;            /* output in the arena (device); bntt_server_release it */
    size_t bytes;
    double t_arrive;    /* server clock, seconds */
    double t_admit;
    double t_done;
    int status;
} bntt_completion;

typedef struct bntt_server_stats {
    uint64_t submitted;
    uint64_t completed;
    uint64_t launches;        /* batch launches (each: one kernel + BLAS kernels) */
    uint64_t admission_waits; /* times the head request waited for arena space */
    size_t peak_bytes;        /* most arena bytes in use at once */
} bntt_server_stats;

/* `plans` (NTT sizes) share one modulus; BLAS requests use `blas_modulus`. */
int bntt_server_create(bntt_ctx *ctx, bntt_server **srv, bntt_plan *const *plans, size_t nplans,
                       const bntt_modulus *blas_modulus, const bntt_server_config *cfg);
int bntt_server_destroy(bntt_server *srv);
double bntt_server_clock(bntt_server *srv);
/* Thread-safe.  A request larger than the whole arena is refused (EBUDGET). */
int bntt_server_submit(bntt_server *srv, const bntt_request *req);
/* Moves up to `cap` completions to `out`; *n gets the count. */
int bntt_server_poll(bntt_server *srv, bntt_completion *out, size_t cap, size_t *n);
int bntt_server_release(bntt_server *srv, void *y);
/* Waits until every submitted request has completed. */
int bntt_server_drain(bntt_server *srv);
int bntt_server_get_stats(bntt_server *srv, bntt_server_stats *stats);
/* Replays `n` requests at their t_arrive offsets (seconds from the start of
 * the replay) and returns each one's latency (completion - arrival) and the
 * wall time from the first arrival to the last completion.  serial = 0: the
 * server's continuous batching; serial = 1: one call at a time in arrival
 * order (each request alone, synchronised, the per-call path).  Outputs are
 * released as they complete. */
int bntt_server_replay(bntt_server *srv, const bntt_request *reqs, size_t n, int serial,
                       double *latency_s, double *wall_s);
/* The same, also returning each request's service time in `service_s` (may
 * be NULL): completion less admission, i.e. the latency without the time
 * spent queued before it was admitted (serial: before its call began). */
int bntt_server_replay_ex(bntt_server *srv, const bntt_request *reqs, size_t n, int serial,
                          double *latency_s, double *service_s, double *wall_s);

/* ------------------------------------------------------------- autotuner */
/* Times every compiled kernel shape for transform sizes 2^1..2^10 (register
 * tile of 4, 8 or 16 elements per thread = radix and number of shared-memory
 * passes, transforms per CTA, two to four resident CTAs per SM, inputs read
 * by the first pass or staged into shared memory a tile ahead, twiddles read
 * through L1 or from a copy of the table in shared memory), the strided
 * first pass of large transforms, and the persistent kernel's tile shape per
 * size, on this device; the fastest become the defaults of plans and batches
 * created afterwards in this process.  Writes the choices to `path` if it is
 * not NULL.  Contiguous shapes are timed on 65,536 transforms (at most 2^24
 * elements) with the L2 flushed before each launch.  A few seconds; about
 * 1 GiB of device memory while it runs.
 * The reference fixes one scalar / SIMD code path per size at compile time
 * (src/ntt_scalar.c:21, benchmark/run_ntt.sh); no counterpart there. */
int bntt_autotune(bntt_ctx *ctx, const char *path);
/* Installs choices saved by bntt_autotune (refused for another device, or
 * when a line names a kernel shape this build does not have). */
int bntt_autotune_load(bntt_ctx *ctx, const char *path);
/* Drops tuned choices; compiled defaults apply to new plans and batches. */
int bntt_autotune_reset(void);

/* ------------------------------------------------------------ diagnostics */
/* Measured throughput of the 32-bit integer multiply-add pipe on this device
 * (independent mad.lo.u32 chains on every SM), in operations per second: the
 * roofline the NTT kernels are reported against.  No reference counterpart
 * (the reference times CPU code only, src/ntt_scalar.c:670-683). */
int bntt_probe_imad_peak(bntt_ctx *ctx, double *ops_per_second);
/* Butterflies per second of the kernels' own butterfly (fast multiply,
 * reference add/sub) on register-resident data at the persistent kernel's
 * occupancy: the compute ceiling of the NTT kernels, with no memory traffic
 * or index arithmetic. */
int bntt_probe_butterfly_peak(bntt_ctx *ctx, double *butterflies_per_second);

#ifdef __cplusplus
}
#endif

#endif /* BNTT_H */
