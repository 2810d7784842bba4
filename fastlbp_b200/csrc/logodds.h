// Log-odds of a folded constant, log(p / (1 - p)), the same bits on the host
// and on the GPU.
//
// A singleton factor (1-p, p) (causal_bp_parall.cu:110-112) and an AND/OR
// factor reduced to its head (:115-117, :154-156) become a finite prior
// constant +-log(p / (1 - p)) of their variable. The host layout build, the
// device layout build and the probability setters all compute it, and the
// engines they make must agree bit for bit, but a platform's log and the
// GPU's may differ in the last place. So the logarithm is written out here
// from correctly rounded IEEE double operations only (+, -, *, /; on the
// device through the _rn intrinsics, which the compiler never fuses):
//
//   x = 2^k m, m in [sqrt(1/2), sqrt(2));  s = (m - 1) / (m + 1), |s| <= 0.1716;
//   log m = 2 atanh(s) = 2 s (1 + s^2/3 + s^4/5 + ... + s^20/21)  (the rest < 2^-60);
//   log x = k log 2 + log m, log 2 in two parts (the first of 40 bits, so
//   that k times it is exact).
//
// Error: at most 2 units in the last place of log x; the log-odds within
// 3e-16 of the exact value (relative to max(1, |log-odds|)), checked against
// a 60-digit reference for 2e5 arguments over the whole double range.

#pragma once

#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define FLBP_LOGODDS_HD __host__ __device__ __forceinline__
#else
#define FLBP_LOGODDS_HD inline
#endif

#if !defined(__CUDA_ARCH__) && (defined(__FMA__) || defined(__FP_FAST_FMA))
// The host compiler could fuse the multiply-adds below into FMAs and round
// them differently from the device: build the host code without FMA.
#error "logodds.h needs host code built without FMA contraction"
#endif

namespace flbp {
namespace logodds_detail {

FLBP_LOGODDS_HD double mul(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
FLBP_LOGODDS_HD double add(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
FLBP_LOGODDS_HD double sub(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
FLBP_LOGODDS_HD double div(double a, double b) {
#ifdef __CUDA_ARCH__
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}
FLBP_LOGODDS_HD uint64_t bits(double x) {
#ifdef __CUDA_ARCH__
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t b;
    std::memcpy(&b, &x, 8);
    return b;
#endif
}
FLBP_LOGODDS_HD double from_bits(uint64_t b) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    double x;
    std::memcpy(&x, &b, 8);
    return x;
#endif
}

}  // namespace logodds_detail

// Natural logarithm: log(0) = -inf, log(+inf) = +inf, NaN for NaN and x < 0.
FLBP_LOGODDS_HD double det_log(double x) {
    using namespace logodds_detail;
    const double inf = from_bits(0x7ff0000000000000ull);
    if (!(x >= 0.0)) return from_bits(0x7ff8000000000000ull);  // NaN, x < 0
    if (x == 0.0) return -inf;
    if (x == inf) return inf;
    int k = 0;
    if (x < 2.2250738585072014e-308) {  // subnormal: scale by 2^54 (exact)
        x = mul(x, 18014398509481984.0);
        k = -54;
    }
    const uint64_t b = bits(x);
    k += (int)((b >> 52) & 0x7ff) - 1023;
    double m = from_bits((b & 0x000fffffffffffffull) | 0x3ff0000000000000ull);  // [1, 2)
    if (m > 1.4142135623730951) {  // sqrt(2) rounded
        m = mul(m, 0.5);
        k += 1;
    }
    const double s = div(sub(m, 1.0), add(m, 1.0));  // m - 1 is exact
    const double t = add(s, s), z = mul(s, s);
    // 1/(2n+1), n = 1..10, each correctly rounded
    double P = 0.047619047619047616;
    P = add(mul(P, z), 0.05263157894736842);
    P = add(mul(P, z), 0.058823529411764705);
    P = add(mul(P, z), 0.06666666666666667);
    P = add(mul(P, z), 0.07692307692307693);
    P = add(mul(P, z), 0.09090909090909091);
    P = add(mul(P, z), 0.1111111111111111);
    P = add(mul(P, z), 0.14285714285714285);
    P = add(mul(P, z), 0.2);
    P = add(mul(P, z), 0.3333333333333333);
    const double lm = add(t, mul(t, mul(z, P)));
    const double kd = (double)k;
    const double ln2_hi = 0.6931471805592082;   // log 2 to 40 bits
    const double ln2_lo = 7.371002565167799e-13;  // log 2 - ln2_hi
    return add(mul(kd, ln2_hi), add(mul(kd, ln2_lo), lm));
}

// log(p / (1 - p)) for p in [0, 1]: -inf at 0, +inf at 1, NaN for NaN or p
// outside [0, 1].
FLBP_LOGODDS_HD double det_logit(double p) {
    using namespace logodds_detail;
    if (p == 1.0) return from_bits(0x7ff0000000000000ull);
    return det_log(div(p, sub(1.0, p)));
}

}  // namespace flbp
