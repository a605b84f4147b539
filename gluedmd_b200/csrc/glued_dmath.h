// Deterministic double-precision exp / log / log1p / pow.
//
// The OPES deposit takes integer decisions (merge into kernel k, or append) from
// FP64 quantities that pass through exp/log/pow (Silverman bandwidth, heights).
// CUDA's and glibc's transcendental functions can differ in the last bit, which
// can flip a near-tie decision. These functions use only IEEE-754 correctly
// rounded +, -, *, / with no fused multiply-add, so they return the same bits on
// the host and on the device; the deposit kernel and the CPU oracle both call
// them and their decisions can be compared exactly.
//
// Methods (textbook, written for this file):
//   exp : Cody-Waite argument reduction x = k*ln2 + r with ln2 split into a
//         high part with trailing zero bits and a low correction, |r| <= ln2/2,
//         then the Taylor series of e^r to degree 17 in Horner form.
//   log : x = m * 2^e with m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(f),
//         f = (m-1)/(m+1), odd series to f^27.
//   log1p: Goldberg's correction log1p(x) = log(u) * x / (u - 1), u = 1 + x.
//   pow : exp(b * log(a)) for a > 0.
// Accuracy is a few ulp; what matters here is identical bits on both sides.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define GD_FN __host__ __device__ __forceinline__
#else
#define GD_FN static inline
#endif

namespace glued_dmath {

#if defined(__CUDA_ARCH__)
GD_FN double gd_mul(double a, double b) { return __dmul_rn(a, b); }
GD_FN double gd_add(double a, double b) { return __dadd_rn(a, b); }
GD_FN double gd_sub(double a, double b) { return __dsub_rn(a, b); }
GD_FN double gd_div(double a, double b) { return __ddiv_rn(a, b); }
GD_FN int64_t gd_bits(double x) { return __double_as_longlong(x); }
GD_FN double gd_from_bits(int64_t b) { return __longlong_as_double(b); }
GD_FN double gd_rint(double x) { return rint(x); }
#else
GD_FN double gd_mul(double a, double b) { volatile double r = a * b; return r; }
GD_FN double gd_add(double a, double b) { volatile double r = a + b; return r; }
GD_FN double gd_sub(double a, double b) { volatile double r = a - b; return r; }
GD_FN double gd_div(double a, double b) { volatile double r = a / b; return r; }
GD_FN int64_t gd_bits(double x) { int64_t b; __builtin_memcpy(&b, &x, 8); return b; }
GD_FN double gd_from_bits(int64_t b) { double x; __builtin_memcpy(&x, &b, 8); return x; }
GD_FN double gd_rint(double x) { return __builtin_rint(x); }
#endif

// 2^k for k in the normal exponent range [-1022, 1023].
GD_FN double gd_pow2(int k) { return gd_from_bits((int64_t)(k + 1023) << 52); }

GD_FN double gd_exp(double x) {
    if (x != x) return x;
    if (x > 709.782712893384) return gd_from_bits(0x7ff0000000000000LL);  // +inf
    if (x < -745.1332191019412) return 0.0;
    const double LN2_HI = 6.93147180369123816490e-01;  // ln2 with 32 trailing zero bits
    const double LN2_LO = 1.90821492927058770002e-10;  // ln2 - LN2_HI
    const double INV_LN2 = 1.44269504088896338700e+00;
    double kd = gd_rint(gd_mul(x, INV_LN2));
    int k = (int)kd;
    double r = gd_sub(gd_sub(x, gd_mul(kd, LN2_HI)), gd_mul(kd, LN2_LO));
    // Taylor series of e^r, degree 17, Horner form: sum r^n / n!
    double p = 1.0 / 355687428096000.0;            // 1/17!
    p = gd_add(gd_mul(p, r), 1.0 / 20922789888000.0);   // 1/16!
    p = gd_add(gd_mul(p, r), 1.0 / 1307674368000.0);    // 1/15!
    p = gd_add(gd_mul(p, r), 1.0 / 87178291200.0);      // 1/14!
    p = gd_add(gd_mul(p, r), 1.0 / 6227020800.0);       // 1/13!
    p = gd_add(gd_mul(p, r), 1.0 / 479001600.0);        // 1/12!
    p = gd_add(gd_mul(p, r), 1.0 / 39916800.0);         // 1/11!
    p = gd_add(gd_mul(p, r), 1.0 / 3628800.0);          // 1/10!
    p = gd_add(gd_mul(p, r), 1.0 / 362880.0);           // 1/9!
    p = gd_add(gd_mul(p, r), 1.0 / 40320.0);            // 1/8!
    p = gd_add(gd_mul(p, r), 1.0 / 5040.0);             // 1/7!
    p = gd_add(gd_mul(p, r), 1.0 / 720.0);              // 1/6!
    p = gd_add(gd_mul(p, r), 1.0 / 120.0);              // 1/5!
    p = gd_add(gd_mul(p, r), 1.0 / 24.0);               // 1/4!
    p = gd_add(gd_mul(p, r), 1.0 / 6.0);                // 1/3!
    p = gd_add(gd_mul(p, r), 0.5);                      // 1/2!
    p = gd_add(gd_mul(p, r), 1.0);
    p = gd_add(gd_mul(p, r), 1.0);
    if (k >= -1021) {
        if (k > 1023) return gd_mul(gd_mul(p, gd_pow2(1023)), gd_pow2(k - 1023));
        return gd_mul(p, gd_pow2(k));
    }
    // Subnormal result: scale in two exact steps.
    return gd_mul(gd_mul(p, gd_pow2(k + 600)), gd_pow2(-600));
}

GD_FN double gd_log(double x) {
    if (x != x || x < 0.0) return gd_from_bits(0x7ff8000000000000LL);  // NaN
    if (x == 0.0) return gd_from_bits((int64_t)0xfff0000000000000ULL);  // -inf
    if (gd_bits(x) >= 0x7ff0000000000000LL) return x;                 // +inf
    int e = 0;
    if (x < 2.2250738585072014e-308) { x = gd_mul(x, gd_pow2(600)); e = -600; }
    int64_t b = gd_bits(x);
    e += (int)((b >> 52) & 0x7ff) - 1023;
    double m = gd_from_bits((b & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);  // [1, 2)
    if (m > 1.4142135623730951) { m = gd_mul(m, 0.5); e += 1; }
    double f = gd_div(gd_sub(m, 1.0), gd_add(m, 1.0));
    double f2 = gd_mul(f, f);
    double s = 1.0 / 27.0;
    s = gd_add(gd_mul(s, f2), 1.0 / 25.0);
    s = gd_add(gd_mul(s, f2), 1.0 / 23.0);
    s = gd_add(gd_mul(s, f2), 1.0 / 21.0);
    s = gd_add(gd_mul(s, f2), 1.0 / 19.0);
    s = gd_add(gd_mul(s, f2), 1.0 / 17.0);
    s = gd_add(gd_mul(s, f2), 1.0 / 15.0);
    s = gd_add(gd_mul(s, f2), 1.0 / 13.0);
    s = gd_add(gd_mul(s, f2), 1.0 / 11.0);
    s = gd_add(gd_mul(s, f2), 1.0 / 9.0);
    s = gd_add(gd_mul(s, f2), 1.0 / 7.0);
    s = gd_add(gd_mul(s, f2), 1.0 / 5.0);
    s = gd_add(gd_mul(s, f2), 1.0 / 3.0);
    s = gd_add(gd_mul(s, f2), 1.0);
    double lm = gd_mul(gd_mul(2.0, f), s);
    const double LN2_HI = 6.93147180369123816490e-01;
    const double LN2_LO = 1.90821492927058770002e-10;
    double ed = (double)e;
    return gd_add(gd_mul(ed, LN2_HI), gd_add(gd_mul(ed, LN2_LO), lm));
}

GD_FN double gd_log1p(double x) {
    double u = gd_add(1.0, x);
    if (u == 1.0) return x;
    return gd_div(gd_mul(gd_log(u), x), gd_sub(u, 1.0));
}

GD_FN double gd_pow(double a, double b) { return gd_exp(gd_mul(b, gd_log(a))); }

}  // namespace glued_dmath
