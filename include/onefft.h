/*
 * onefft_b200 — drop-in C API of OneFFT, served by hand-written CUDA kernels on an NVIDIA B200.
 *
 * Every declaration below keeps the name, signature and meaning of OneFFT's public header
 * (OneFFT include/onefft.h:76-116, version 0.1.0), so code written against OneFFT compiles and
 * links against libonefft_cuda.so unchanged:
 *
 *   complex-to-complex, single precision, out of place, power-of-two n from 1 to 2^30;
 *   interleaved data: n complex values are 2n floats re, im, re, im, ...;
 *   forward  out[k] = sum_j in[j] exp(-2 pi i j k / n),
 *   inverse  out[k] = sum_j in[j] exp(+2 pi i j k / n), neither normalised.
 *
 * Buffers may be host memory (pageable or pinned) or device memory of the current CUDA device;
 * no alignment is required. Host buffers are copied to the device and back inside the call.
 * Every function is safe to call from any number of threads at once (each thread gets its own
 * CUDA stream and staging buffers), except onefft_cache_clear() as documented below.
 *
 * Device-pointer batched entry points, the uneven-batch launch and error reporting are declared
 * beside this header in onefft_cuda.h.
 */
#ifndef ONEFFT_H
#define ONEFFT_H

#include <stddef.h>

#define ONEFFT_VERSION_MAJOR 0
#define ONEFFT_VERSION_MINOR 1
#define ONEFFT_VERSION_PATCH 0

/* Symbols exported by libonefft_cuda.so (built with hidden default visibility). */
#if defined(__GNUC__)
#define ONEFFT_API __attribute__((visibility("default")))
#else
#define ONEFFT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces OneFFT include/onefft.h:76-77 (src/onefft.c:1169-1181).
 * Transform n complex values from `in` to `out` (non-overlapping). The first call for a size, in
 * either direction, builds that size's device tables (FP64 on the device, rounded to FP32) and
 * keeps them until onefft_cache_clear(); later calls find them with one atomic load.
 * Returns 0 on success, -1 with `out` untouched if n is not a power of two in [1, 2^30], if the
 * tables or buffers cannot be allocated, or if the device reports an error. */
ONEFFT_API int onefft_forward(const float *in, float *out, size_t n);
ONEFFT_API int onefft_inverse(const float *in, float *out, size_t n);

/* Replaces OneFFT include/onefft.h:82 (src/onefft.c:1183). Builds the tables for size n now.
 * Returns 0 on success, -1 for an invalid n or on allocation failure. */
ONEFFT_API int onefft_cache_prepare(size_t n);

/* Replaces OneFFT include/onefft.h:86 (src/onefft.c:1185-1189). Frees every cached plan. Must not
 * be called while another thread is inside onefft_forward/onefft_inverse or is using a cached
 * plan; the cache refills on demand. */
ONEFFT_API void onefft_cache_clear(void);

typedef struct onefft_plan onefft_plan;

/* Replaces OneFFT include/onefft.h:97 (src/onefft.c:1111-1130). Creates a plan for size n on the
 * current CUDA device: one device allocation holding the twiddle tables. Returns NULL if n is not
 * a power of two in [1, 2^30] or if the allocation or table build fails. */
ONEFFT_API onefft_plan *onefft_plan_create(size_t n);

/* Replaces OneFFT include/onefft.h:100 (src/onefft.c:1132-1136). NULL is allowed. */
ONEFFT_API void onefft_plan_destroy(onefft_plan *plan);

/* Replaces OneFFT include/onefft.h:105-106 (src/onefft.c:1138-1140). Transform with a plan; the
 * plan is never modified, so one plan serves any number of threads in both directions. These
 * calls return nothing, as in OneFFT; on a device error `out` is left untouched and the reason is
 * available from onefft_last_error() (onefft_cuda.h). */
ONEFFT_API void onefft_plan_forward(const onefft_plan *plan, const float *in, float *out);
ONEFFT_API void onefft_plan_inverse(const onefft_plan *plan, const float *in, float *out);

/* Replaces OneFFT include/onefft.h:109 (src/onefft.c:1142). */
ONEFFT_API size_t onefft_plan_size(const onefft_plan *plan);

/* Replaces OneFFT include/onefft.h:116 (src/onefft.c:1080-1092): "cuda sm_100a". */
ONEFFT_API const char *onefft_implementation(void);

#ifdef __cplusplus
} /* extern "C" */

#include <complex>

/* C++ convenience layer: OneFFT's own (include/onefft.h:123-169), kept with the same names,
 * signatures and behaviour so C++ callers compile unchanged; get() is added.
 * OneFFT's C++ layer: Copyright (c) 2026 Torben Thaysen, MIT License. */
namespace onefft {

inline bool forward(const std::complex<float> *in, std::complex<float> *out, std::size_t n) {
    return onefft_forward(reinterpret_cast<const float *>(in), reinterpret_cast<float *>(out), n) == 0;
}
inline bool inverse(const std::complex<float> *in, std::complex<float> *out, std::size_t n) {
    return onefft_inverse(reinterpret_cast<const float *>(in), reinterpret_cast<float *>(out), n) == 0;
}

/* Owns a plan; move-only. */
class Plan {
public:
    explicit Plan(std::size_t n) : plan_(onefft_plan_create(n)) {}
    ~Plan() { onefft_plan_destroy(plan_); }
    Plan(Plan &&other) noexcept : plan_(other.plan_) { other.plan_ = nullptr; }
    Plan &operator=(Plan &&other) noexcept {
        if (this != &other) {
            onefft_plan_destroy(plan_);
            plan_ = other.plan_;
            other.plan_ = nullptr;
        }
        return *this;
    }
    Plan(const Plan &) = delete;
    Plan &operator=(const Plan &) = delete;

    explicit operator bool() const { return plan_ != nullptr; }
    std::size_t size() const { return onefft_plan_size(plan_); }
    const onefft_plan *get() const { return plan_; }

    void forward(const std::complex<float> *in, std::complex<float> *out) const {
        onefft_plan_forward(plan_, reinterpret_cast<const float *>(in), reinterpret_cast<float *>(out));
    }
    void inverse(const std::complex<float> *in, std::complex<float> *out) const {
        onefft_plan_inverse(plan_, reinterpret_cast<const float *>(in), reinterpret_cast<float *>(out));
    }
    void forward(const float *in, float *out) const { onefft_plan_forward(plan_, in, out); }
    void inverse(const float *in, float *out) const { onefft_plan_inverse(plan_, in, out); }

private:
    onefft_plan *plan_;
};

} /* namespace onefft */
#endif /* __cplusplus */

#endif /* ONEFFT_H */
