/*
 * CPU timing harness — TEST/BENCHMARK INFRASTRUCTURE, NOT PART OF THE PRODUCT.
 *
 * Times OneFFT's CPU implementation of the transform on the host cores, the way the reference
 * library is meant to be parallelised by its callers: one shared, read-only plan per size and
 * N pthreads that each pull transform indices from an atomic counter and call the thread-safe
 * plan_forward / plan_inverse (OneFFT include/onefft.h:102-106, tests/test_onefft.c:207-259).
 * Each sample is wall-clock (CLOCK_MONOTONIC), the reported figure is the minimum over samples,
 * as OneFFT bench/bench.c:151-166 does.
 *
 * Built twice by oracle/Makefile:
 *   - with the reference library's own sources (oracle/_ref/libonefft_ref.so, kind "reference");
 *   - with the plain-C restatement in oracle.c (oracle/liboracle.so, kind "port"), selected by
 *     -DCPU_BENCH_PORT.
 */
#define _POSIX_C_SOURCE 200809L
#include <pthread.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <time.h>
#include <unistd.h>

#define BENCH_EXPORT __attribute__((visibility("default")))

#ifdef CPU_BENCH_PORT
typedef struct oracle_plan oracle_plan;
oracle_plan *oracle_plan_create(size_t n);
void oracle_plan_destroy(oracle_plan *p);
void oracle_plan_forward(const oracle_plan *p, const float *in, float *out);
void oracle_plan_inverse(const oracle_plan *p, const float *in, float *out);
typedef oracle_plan bench_plan;
#define PLAN_CREATE oracle_plan_create
#define PLAN_DESTROY oracle_plan_destroy
#define PLAN_FORWARD oracle_plan_forward
#define PLAN_INVERSE oracle_plan_inverse
static const char *impl_name(void) { return "port"; }
#else
#include "onefft.h"
typedef onefft_plan bench_plan;
#define PLAN_CREATE onefft_plan_create
#define PLAN_DESTROY onefft_plan_destroy
#define PLAN_FORWARD onefft_plan_forward
#define PLAN_INVERSE onefft_plan_inverse
static const char *impl_name(void) { return onefft_implementation(); }
#endif

BENCH_EXPORT const char *cpu_bench_impl(void) { return impl_name(); }
BENCH_EXPORT int cpu_bench_ncores(void) { return (int)sysconf(_SC_NPROCESSORS_ONLN); }

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* One unit of work: transform `index` of the job. */
typedef struct {
    size_t count;            /* transforms in one pass */
    const bench_plan **plan; /* per transform (uniform batches repeat one plan) */
    const int64_t *offset;   /* per transform, in complex values; NULL = index * n */
    const int32_t *inverse;  /* per transform; NULL = `direction` */
    int direction;
    size_t n; /* uniform batches */
    const float *in;
    float *out;
    size_t next; /* atomic work counter */
} bench_job;

static void *worker(void *arg) {
    bench_job *job = (bench_job *)arg;
    for (;;) {
        size_t i = __atomic_fetch_add(&job->next, 1, __ATOMIC_RELAXED);
        if (i >= job->count) break;
        const bench_plan *p = job->plan[job->offset ? i : 0];
        size_t off = job->offset ? (size_t)job->offset[i] : i * job->n;
        int inv = job->inverse ? job->inverse[i] : job->direction;
        if (inv) PLAN_INVERSE(p, job->in + 2 * off, job->out + 2 * off);
        else PLAN_FORWARD(p, job->in + 2 * off, job->out + 2 * off);
    }
    return NULL;
}

static double run_pass(bench_job *job, int threads) {
    pthread_t tid[512];
    if (threads < 1) threads = 1;
    if (threads > 512) threads = 512;
    job->next = 0;
    double t0 = now_s();
    for (int t = 1; t < threads; t++) pthread_create(&tid[t], NULL, worker, job);
    worker(job);
    for (int t = 1; t < threads; t++) pthread_join(tid[t], NULL);
    return now_s() - t0;
}

/* Batch of `batch` transforms of size n at in + 2*n*i. Runs `samples` timed passes after one
 * untimed pass; returns the minimum seconds per pass (negative on an invalid size). */
BENCH_EXPORT double cpu_bench_batched(size_t n, size_t batch, int threads, int inverse, const float *in, float *out,
                                      int samples) {
    bench_plan *plan = PLAN_CREATE(n);
    if (!plan) return -1.0;
    const bench_plan *plans[1] = {plan};
    bench_job job = {batch, plans, NULL, NULL, inverse, n, in, out, 0};
    run_pass(&job, threads);
    double best = 1e300;
    for (int s = 0; s < samples; s++) {
        double t = run_pass(&job, threads);
        if (t < best) best = t;
    }
    PLAN_DESTROY(plan);
    return best;
}

/* Uneven batch: transform i has size 2^log2n[i], starts at complex offset[i] and runs in
 * direction inverse[i]. Plans for all sizes are created before timing. */
BENCH_EXPORT double cpu_bench_uneven(const int32_t *log2n, const int64_t *offset, const int32_t *inverse, size_t count,
                                     int threads, const float *in, float *out, int samples) {
    bench_plan *by_size[31] = {0};
    const bench_plan **plan = (const bench_plan **)malloc((count ? count : 1) * sizeof(*plan));
    if (!plan) return -1.0;
    double result = -1.0;
    for (size_t i = 0; i < count; i++) {
        int l = log2n[i];
        if (l < 0 || l > 30) goto done;
        if (!by_size[l] && !(by_size[l] = PLAN_CREATE((size_t)1 << l))) goto done;
        plan[i] = by_size[l];
    }
    {
        bench_job job = {count, plan, offset, inverse, 0, 0, in, out, 0};
        run_pass(&job, threads);
        double best = 1e300;
        for (int s = 0; s < samples; s++) {
            double t = run_pass(&job, threads);
            if (t < best) best = t;
        }
        result = best;
    }
done:
    for (int l = 0; l <= 30; l++) PLAN_DESTROY(by_size[l]);
    free(plan);
    return result;
}
