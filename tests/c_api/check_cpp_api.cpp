// A C++ caller of the drop-in API, compiled as C++11 against include/onefft.h and linked to
// libonefft_cuda.so (tests/test_c_api.py builds and runs it). It makes the checks of OneFFT's
// C++ interface test (tests/test_cpp.cpp:10-36) through the header's C++ layer, with its own
// inputs and a few additions:
//   - onefft::Plan creation and size(), forward then inverse: inverse(forward(x)) / n = x;
//   - moving a plan (construction and assignment) leaves the source empty and the target
//     producing the same results bit for bit;
//   - onefft::forward / onefft::inverse (the cached path) equal the plan's results bit for bit;
//   - the float-pointer overloads equal the complex ones;
//   - an invalid size is refused by onefft::forward and by onefft::Plan;
//   - a multi-pass size (2^20) round trip through the same layer.
// Prints one line per failed check and "c++ api: all checks passed"; exit status 0 only then.
#include "onefft.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <utility>
#include <vector>

namespace {

int failures = 0;

void check(bool ok, const char *what) {
    if (!ok) {
        ++failures;
        std::printf("FAILED: %s\n", what);
    }
}

typedef std::vector<std::complex<float> > Signal;

Signal make_signal(std::size_t n, std::uint32_t seed) {
    Signal s(n);
    std::uint32_t x = seed;
    for (std::size_t i = 0; i < n; ++i) {
        float v[2];
        for (int k = 0; k < 2; ++k) {  // xorshift32, uniform in [-1, 1)
            x ^= x << 13;
            x ^= x >> 17;
            x ^= x << 5;
            v[k] = float(x >> 8) * (2.0f / 16777216.0f) - 1.0f;
        }
        s[i] = std::complex<float>(v[0], v[1]);
    }
    return s;
}

// max |back / n - in| over max |in|
double round_trip_error(const Signal &in, const Signal &back) {
    const double n = double(in.size());
    double worst = 0, scale = 0;
    for (std::size_t i = 0; i < in.size(); ++i) {
        const std::complex<double> d = std::complex<double>(back[i]) / n - std::complex<double>(in[i]);
        worst = std::max(worst, std::abs(d));
        scale = std::max(scale, double(std::abs(in[i])));
    }
    return worst / scale;
}

bool same_bits(const Signal &a, const Signal &b) { return a == b; }

}  // namespace

int main() {
    const std::size_t n = 512;
    const Signal in = make_signal(n, 0x2545F491u);
    Signal spectrum(n), back(n), again(n);

    onefft::Plan plan(n);
    check(bool(plan) && plan.size() == n, "plan creation and size");
    plan.forward(in.data(), spectrum.data());
    plan.inverse(spectrum.data(), back.data());
    check(round_trip_error(in, back) < 1e-5, "round trip through the plan");

    onefft::Plan moved(std::move(plan));
    check(!plan && bool(moved), "move construction");
    moved.forward(in.data(), again.data());
    check(same_bits(again, spectrum), "moved plan forward equals the original");
    moved.inverse(reinterpret_cast<const float *>(spectrum.data()), reinterpret_cast<float *>(again.data()));
    check(same_bits(again, back), "float-pointer inverse equals the complex one");

    onefft::Plan assigned(64);
    assigned = std::move(moved);
    check(!moved && bool(assigned) && assigned.size() == n, "move assignment");
    assigned.forward(reinterpret_cast<const float *>(in.data()), reinterpret_cast<float *>(again.data()));
    check(same_bits(again, spectrum), "assigned plan forward equals the original");

    check(onefft::forward(in.data(), again.data(), n) && same_bits(again, spectrum), "cached forward");
    check(onefft::inverse(spectrum.data(), again.data(), n) && same_bits(again, back), "cached inverse");

    Signal untouched(100, std::complex<float>(7.0f, 7.0f)), small_in(100);
    check(!onefft::forward(small_in.data(), untouched.data(), 100), "invalid size accepted by onefft::forward");
    check(untouched[0] == std::complex<float>(7.0f, 7.0f) && untouched[99] == untouched[0],
          "output written for an invalid size");
    check(!onefft::Plan(100), "invalid plan size accepted");

    const std::size_t big = std::size_t(1) << 20;
    const Signal big_in = make_signal(big, 0x9E3779B9u);
    Signal big_out(big), big_back(big);
    onefft::Plan big_plan(big);
    check(bool(big_plan), "multi-pass plan creation");
    big_plan.forward(big_in.data(), big_out.data());
    big_plan.inverse(big_out.data(), big_back.data());
    check(round_trip_error(big_in, big_back) < 1e-5, "multi-pass round trip");

    onefft_cache_clear();
    if (failures == 0) std::puts("c++ api: all checks passed");
    return failures == 0 ? 0 : 1;
}
