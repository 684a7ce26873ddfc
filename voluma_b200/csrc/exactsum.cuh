// Exact, order-independent summation of doubles on the device: the superaccumulator of
// par::ExactSum (src/fvm/parallel/Comm.h:42-93, Comm.cpp:107-164).  Device functions only (no
// kernels), so several translation units can include it.
#pragma once

#include <cuda_runtime.h>

namespace vlm {

// The superaccumulator of par::ExactSum (src/fvm/parallel/Comm.h:42-93, Comm.cpp:107-164):
// a double M*2^E is split over three 32-bit-aligned int64 bins; integer addition is
// associative, so the total does not depend on the summation order, and the final
// conversion reproduces the reference's value bit for bit.
constexpr int kExactBins = 72;
constexpr int kExactStride = kExactBins + 1;  // bins + non-finite flags per partial

__device__ __forceinline__ void exact_add(long long* bins, int* flags, double v) {
    const unsigned long long bits = (unsigned long long)__double_as_longlong(v);
    const int ex = (int)((bits >> 52) & 0x7ff);
    if (ex == 0x7ff) {  // Inf / NaN: remembered as flags (their sum is order independent)
        if ((bits & ((1ull << 52) - 1)) != 0)
            atomicOr(flags, 1);
        else
            atomicOr(flags, (bits >> 63) ? 4 : 2);
        return;
    }
    long long M = (long long)(bits & ((1ull << 52) - 1));
    if (ex != 0) M |= 1ll << 52;
    if (M == 0) return;
    const int p = (ex == 0 ? 1 : ex) - 1;
    const int i = p >> 5, sh = p & 31;
    const long long sgn = -(long long)(bits >> 63);
    long long lo = (M & ((1ll << (32 - sh)) - 1)) << sh;
    const long long r = M >> (32 - sh);
    long long mid = r & 0xFFFFFFFFll;
    long long hi = r >> 32;
    lo = (lo ^ sgn) - sgn;
    mid = (mid ^ sgn) - sgn;
    hi = (hi ^ sgn) - sgn;
    atomicAdd((unsigned long long*)&bins[i], (unsigned long long)lo);
    atomicAdd((unsigned long long*)&bins[i + 1], (unsigned long long)mid);
    atomicAdd((unsigned long long*)&bins[i + 2], (unsigned long long)hi);
}

__device__ __forceinline__ void exact_normalize(long long* b) {
    for (int k = 0; k < kExactBins - 1; ++k) {
        const long long carry = b[k] >> 32;
        b[k] -= carry * (1ll << 32);
        b[k + 1] += carry;
    }
}

// binsToDouble (Comm.cpp:135-156)
__device__ inline double exact_value(long long* b, int flags) {
    if (flags & 1) return __longlong_as_double(0x7ff8000000000000ll);
    if ((flags & 6) == 6) return __longlong_as_double(0x7ff8000000000000ll);
    if (flags & 2) return __longlong_as_double(0x7ff0000000000000ll);
    if (flags & 4) return __longlong_as_double((long long)0xfff0000000000000ull);
    exact_normalize(b);
    double sign = 1.0;
    if (b[kExactBins - 1] < 0) {
        sign = -1.0;
        for (int k = 0; k < kExactBins; ++k) b[k] = -b[k];
        exact_normalize(b);
    }
    double r = 0.0;
    for (int k = kExactBins - 1; k >= 0; --k)
        if (b[k] != 0) r += ldexp((double)b[k], 32 * k - 1074);
    return sign * r;
}

}  // namespace vlm
