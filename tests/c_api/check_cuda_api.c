/*
 * A C99 caller of include/onefft_cuda.h: device-pointer batched transforms and the column
 * transform of the distributed four-step, on device buffers the program allocates itself with the
 * CUDA runtime (the header needs no CUDA include; streams travel as void *). Results are checked
 * against a direct FP64 DFT with integer-reduced angles. Built and run by tests/test_c_api.py:
 *   cc -std=c99 -I include -I <cuda>/include check_cuda_api.c -L onefft_b200 -lonefft_cuda
 *      -L <cuda>/lib64 -lcudart -lm
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "onefft_cuda.h"

static int failures = 0;

static void check(int ok, const char *what) {
    if (!ok) {
        printf("FAILED: %s (%s)\n", what, onefft_last_error());
        ++failures;
    }
}

/* exp(-2 pi i t / n) for t reduced modulo n in integers */
static void root(unsigned long long t, unsigned long long n, double *re, double *im) {
    const double a = -2.0 * 3.14159265358979323846 * (double)(t % n) / (double)n;
    *re = cos(a);
    *im = sin(a);
}

/* relative RMS of got (float pairs) against want (double pairs), count complex values */
static double rel_rms(const float *got, const double *want, size_t count) {
    double num = 0.0, den = 0.0;
    for (size_t i = 0; i < 2 * count; ++i) {
        const double d = (double)got[i] - want[i];
        num += d * d;
        den += want[i] * want[i];
    }
    return sqrt(num / den);
}

static float *device_copy(const float *host, size_t floats) {
    void *d = NULL;
    if (cudaMalloc(&d, floats * sizeof(float)) != cudaSuccess) return NULL;
    if (cudaMemcpy(d, host, floats * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) return NULL;
    return (float *)d;
}

static unsigned long long lcg = 12345u;
static float uniform(void) {
    lcg = lcg * 6364136223846793005ull + 1442695040888963407ull;
    return (float)((double)(lcg >> 11) / 9007199254740992.0 * 2.0 - 1.0);
}

/* eight forward transforms of 1024 values through onefft_dev_forward_batched on a stream */
static void batched_on_device(void) {
    const size_t n = 1024, batch = 8, floats = 2 * n * batch;
    float *x = malloc(floats * sizeof(float)), *y = malloc(floats * sizeof(float));
    double *want = malloc(2 * n * sizeof(double));
    for (size_t i = 0; i < floats; ++i) x[i] = uniform();
    onefft_plan *plan = onefft_plan_create(n);
    float *dx = device_copy(x, floats), *dy = NULL;
    cudaStream_t s = NULL;
    check(plan && dx && cudaMalloc((void **)&dy, floats * sizeof(float)) == cudaSuccess &&
              cudaStreamCreate(&s) == cudaSuccess, "setup of the batched case");
    check(onefft_dev_forward_batched(plan, dx, dy, batch, (void *)s) == 0, "onefft_dev_forward_batched");
    check(cudaStreamSynchronize(s) == cudaSuccess && onefft_plan_status(plan) == 0, "batched kernels");
    check(cudaMemcpy(y, dy, floats * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess, "copy back");
    for (size_t b = 0; b < batch; ++b) {
        const float *xb = x + 2 * n * b;
        for (size_t k = 0; k < n; ++k) {
            double re = 0.0, im = 0.0;
            for (size_t j = 0; j < n; ++j) {
                double wr, wi;
                root((unsigned long long)j * k, n, &wr, &wi);
                re += xb[2 * j] * wr - xb[2 * j + 1] * wi;
                im += xb[2 * j] * wi + xb[2 * j + 1] * wr;
            }
            want[2 * k] = re;
            want[2 * k + 1] = im;
        }
        check(rel_rms(y + 2 * n * b, want, n) < 1.4e-6, "batched transform against the FP64 DFT");
    }
    /* misuse is reported, not run */
    check(onefft_dev_forward_batched(NULL, dx, dy, batch, NULL) == ONEFFT_ERR_ARG, "NULL plan rejected");
    check(onefft_dev_forward_batched(plan, dx, dx, batch, NULL) == ONEFFT_ERR_ARG, "overlap rejected");
    cudaStreamDestroy(s);
    cudaFree(dx);
    cudaFree(dy);
    onefft_plan_destroy(plan);
    free(x);
    free(y);
    free(want);
}

/* one rank's first local step of a 2^14-point transform over 4 ranks: 256-point columns of a
 * 256 x 16 block (columns 32 .. 47 of the whole), the 2^14-point twiddle, the 4-block send layout */
static void column_transform(void) {
    const size_t n = 256, cols = 16, blocks = 4, r = n / blocks, count = n * cols;
    const unsigned long long big_n = 1u << 14, col0 = 32;
    float *x = malloc(2 * count * sizeof(float)), *y = malloc(2 * count * sizeof(float));
    double *want = malloc(2 * count * sizeof(double));
    for (size_t i = 0; i < 2 * count; ++i) x[i] = uniform();
    onefft_columns *c = onefft_columns_create(n, cols, blocks, big_n, col0);
    float *dx = device_copy(x, 2 * count), *dy = NULL;
    check(c && dx && cudaMalloc((void **)&dy, 2 * count * sizeof(float)) == cudaSuccess, "setup of the column case");
    check(onefft_columns_execute(c, dx, dy, 0, NULL) == 0, "onefft_columns_execute");
    check(cudaDeviceSynchronize() == cudaSuccess && onefft_columns_status(c) == 0, "column kernels");
    check(cudaMemcpy(y, dy, 2 * count * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess, "copy back");
    for (size_t b = 0; b < cols; ++b) {
        for (size_t k = 0; k < n; ++k) {
            double re = 0.0, im = 0.0, tr, ti;
            for (size_t j = 0; j < n; ++j) {
                double wr, wi;
                root((unsigned long long)j * k, n, &wr, &wi);
                const double xr = x[2 * (j * cols + b)], xi = x[2 * (j * cols + b) + 1];
                re += xr * wr - xi * wi;
                im += xr * wi + xi * wr;
            }
            root((col0 + b) * (unsigned long long)k, big_n, &tr, &ti);
            const size_t at = ((k / r) * cols + b) * r + k % r;
            want[2 * at] = re * tr - im * ti;
            want[2 * at + 1] = re * ti + im * tr;
        }
    }
    check(rel_rms(y, want, count) < 1.4e-6, "column transform against the FP64 DFT");
    check(onefft_columns_execute(c, dx, dy, 4, NULL) == ONEFFT_ERR_ARG, "unknown flag rejected");
    check(onefft_columns_create(n, 8, 1, 0, 0) == NULL, "too few columns rejected");
    check(onefft_columns_create(n, cols, 1, big_n, big_n) == NULL, "column offset past big_n / n rejected");
    onefft_columns_destroy(c);
    onefft_columns_destroy(NULL);
    cudaFree(dx);
    cudaFree(dy);
    free(x);
    free(y);
    free(want);
}

int main(void) {
    printf("implementation: %s\n", onefft_implementation());
    batched_on_device();
    column_transform();
    if (failures) {
        printf("%d check(s) failed\n", failures);
        return 1;
    }
    printf("all checks passed\n");
    return 0;
}
