// ccc_libm.h — elementary functions used by the continuous-collision root solver.
//
// The cubic solver follows the reference's closed-form (Cardano / trigonometric) method
// (collisions_continuous.cu:511-613), which calls cbrt, acos, cos and sin.  CUDA's device
// library and the host C library give different last-bit results for those calls, which
// would make the GPU path and the CPU oracle disagree by an ulp on times of impact.  To
// make the two bit-identical, both include this header and evaluate the functions with
// the same sequence of IEEE-754 double operations (+, -, *, /, sqrt and explicit fused
// multiply-adds through ccc_fma; nothing is contracted implicitly: the device side is
// compiled with -fmad=false, the host side with -ffp-contract=off).
//
// Methods (all from elementary analysis, not from any vendor library):
//   ccc_cbrt : exponent split a = m * 2^(3q+r); the inverse cube root of m' = m 2^r from a
//              chord on [1,2) scaled by 2^(-r/3), three division-free Newton steps
//              r <- r + r (1 - m' r^3) / 3, then y = m' r^2 and one Newton step
//              y <- y - (y^3 - m') / (3 y^2) with an fma residual.  Error <= 1 ulp.
//   ccc_sin / ccc_cos : Maclaurin series in fma Horner form, terms 1/(2n+1)! and 1/(2n)!
//              (exact rationals rounded once to double), valid and accurate for |x| <= 1.1,
//              which covers the solver's only use, k/3 with k = acos(.) in [0, pi].  Larger
//              arguments are halved and recombined with the double-angle identities.
//   ccc_acos : acos(x) = pi/2 - asin(x) for |x| < 1/2, 2 asin(sqrt((1-x)/2)) for x >= 1/2,
//              pi - 2 asin(sqrt((1+x)/2)) for x <= -1/2; asin on [0, 1/2] by its Maclaurin
//              series sum (2n)!/(4^n (n!)^2 (2n+1)) x^(2n+1), 30 terms, evaluated as even and
//              odd halves in x^4 (two independent fma chains).
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define CCC_HD __host__ __device__ __forceinline__
// larger helpers are kept out of line on the device: the solver calls each several times
// and warps in different branches would otherwise thrash the instruction cache
#define CCC_HD_CALL static __host__ __device__ __noinline__
#else
#define CCC_HD static inline
#define CCC_HD_CALL static
#include <math.h>
#include <string.h>
#endif

// correctly rounded fused multiply-add on both sides (the solver's own arithmetic never
// contracts; these helpers use fma explicitly, identically on host and device)
CCC_HD double ccc_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return fma(a, b, c);
#endif
}

// Rounded product, sum and difference that a compiler never fuses with a neighbouring
// operation, even in a translation unit built with multiply-add contraction on (the
// continuous narrow phase is; the host side is built with -ffp-contract=off).  Every
// product in this header that feeds a sum is one of these or an operand of ccc_fma.
CCC_HD double ccc_mul(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
CCC_HD double ccc_add(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
CCC_HD double ccc_sub(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}

CCC_HD uint64_t ccc_dbits(double x) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t u;
    memcpy(&u, &x, sizeof(u));
    return u;
#endif
}

CCC_HD double ccc_dfrombits(uint64_t u) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)u);
#else
    double x;
    memcpy(&x, &u, sizeof(x));
    return x;
#endif
}

CCC_HD double ccc_sqrt(double x) {
#if defined(__CUDA_ARCH__)
    return __dsqrt_rn(x);
#else
    return sqrt(x);
#endif
}

// 2^n as a double for n in [-1022, 1023] (built from the exponent field; exact).
CCC_HD double ccc_pow2i(int n) {
    return ccc_dfrombits((uint64_t)(n + 1023) << 52);
}

// Exact x * 2^n (single rounding when the result is subnormal), for |n| <= 2000.
CCC_HD double ccc_ldexp(double x, int n) {
    // split into at most three in-range power-of-two factors; each intermediate stays
    // normal except possibly the last multiply, so only one rounding can occur
    while (n > 1023) {
        x = ccc_mul(x, ccc_pow2i(1023));
        n -= 1023;
    }
    if (n < -1022) {
        // keep an intermediate in range before the final (possibly rounding) multiply
        if (n < -1022 - 1022) {
            x = ccc_mul(x, ccc_pow2i(-1022));
            n += 1022;
        }
        x = ccc_mul(x, ccc_pow2i(n + 60));
        return ccc_mul(x, ccc_pow2i(-60));
    }
    return ccc_mul(x, ccc_pow2i(n));
}

// Exponent e of frexp: x = m * 2^e with |m| in [0.5, 1); 0 for x == 0 (and for inf/NaN).
CCC_HD int ccc_frexp_exp(double x) {
    uint64_t u = ccc_dbits(x);
    int be = (int)((u >> 52) & 0x7ff);
    if (be == 0x7ff) return 0;
    if (be == 0) {
        if ((u << 1) == 0) return 0;
        // subnormal: scale up by 2^64 (exact) and re-read
        double y = ccc_mul(x, ccc_pow2i(64));
        uint64_t v = ccc_dbits(y);
        return (int)((v >> 52) & 0x7ff) - 1022 - 64;
    }
    return be - 1022;
}

CCC_HD_CALL double ccc_cbrt(double x) {
    if (x == 0.0 || x != x) return x + x;          // +-0 kept, NaN propagated
    uint64_t u = ccc_dbits(x);
    uint64_t sign = u & 0x8000000000000000ull;
    uint64_t mag = u & 0x7fffffffffffffffull;
    if ((mag >> 52) == 0x7ff) return x;             // +-inf
    double a = ccc_dfrombits(mag);
    int ebias = 0;
    if ((mag >> 52) == 0) {                         // subnormal: scale into normal range
        a = a * ccc_pow2i(54);
        ebias = -54;
    }
    uint64_t ua = ccc_dbits(a);
    int e = (int)((ua >> 52) & 0x7ff) - 1023 + ebias;     // a = m * 2^e, m in [1,2)
    double m = ccc_dfrombits((ua & 0x000fffffffffffffull) | 0x3ff0000000000000ull);
    int q = (e >= 0) ? e / 3 : -((-e + 2) / 3);          // floor(e/3)
    int r = e - 3 * q;                                    // 0, 1, 2
    double mr = m;
    double scale = 1.0;
    if (r == 1) { mr = m * 2.0; scale = 0x1.965fea53d6e3dp-1; }   // 2^(-1/3)
    if (r == 2) { mr = m * 4.0; scale = 0x1.428a2f98d728bp-1; }   // 2^(-2/3)
    // m^(-1/3) on [1,2): chord through the end points, within 2.7 %
    double ri = ccc_fma(-0x1.a68056b0a470cp-3, m - 1.0, 1.0) * scale;
    const double third = 0x1.5555555555555p-2;
    for (int it = 0; it < 3; ++it) {
        double r3 = ri * ri * ri;
        double err = ccc_fma(-mr, r3, 1.0);
        ri = ccc_fma(ri * err, third, ri);
    }
    double y = (mr * ri) * ri;
    double t = y * y;
    double res = ccc_fma(t, y, -mr);
    y = y - res / (3.0 * t);
    y = ccc_ldexp(y, q);
    return sign ? -y : y;
}

// cube root of a float argument, returned in float (the solver's triple-root branch casts
// its argument to float before taking the root)
CCC_HD float ccc_cbrtf(float x) {
    return (float)ccc_cbrt((double)x);
}

CCC_HD double ccc_sin_series(double x) {
    double z = x * x;
    double p = 0x1.3f3ccdd165fa9p-84;                     //  1/25!
    p = ccc_fma(p, z, -0x1.761b41316381ap-75);            // -1/23!
    p = ccc_fma(p, z, 0x1.71b8ef6dcf572p-66);             //  1/21!
    p = ccc_fma(p, z, -0x1.2f49b46814157p-57);            // -1/19!
    p = ccc_fma(p, z, 0x1.952c77030ad4ap-49);             //  1/17!
    p = ccc_fma(p, z, -0x1.ae7f3e733b81fp-41);            // -1/15!
    p = ccc_fma(p, z, 0x1.6124613a86d09p-33);             //  1/13!
    p = ccc_fma(p, z, -0x1.ae64567f544e4p-26);            // -1/11!
    p = ccc_fma(p, z, 0x1.71de3a556c734p-19);             //  1/9!
    p = ccc_fma(p, z, -0x1.a01a01a01a01ap-13);            // -1/7!
    p = ccc_fma(p, z, 0x1.1111111111111p-7);              //  1/5!
    p = ccc_fma(p, z, -0x1.5555555555555p-3);             // -1/3!
    return ccc_fma(x * z, p, x);
}

CCC_HD double ccc_cos_series(double x) {
    double z = x * x;
    double p = 0x1.f2cf01972f578p-80;                     //  1/24!
    p = ccc_fma(p, z, -0x1.0ce396db7f853p-70);            // -1/22!
    p = ccc_fma(p, z, 0x1.e542ba4020225p-62);             //  1/20!
    p = ccc_fma(p, z, -0x1.6827863b97d97p-53);            // -1/18!
    p = ccc_fma(p, z, 0x1.ae7f3e733b81fp-45);             //  1/16!
    p = ccc_fma(p, z, -0x1.93974a8c07c9dp-37);            // -1/14!
    p = ccc_fma(p, z, 0x1.1eed8eff8d898p-29);             //  1/12!
    p = ccc_fma(p, z, -0x1.27e4fb7789f5cp-22);            // -1/10!
    p = ccc_fma(p, z, 0x1.a01a01a01a01ap-16);             //  1/8!
    p = ccc_fma(p, z, -0x1.6c16c16c16c17p-10);            // -1/6!
    p = ccc_fma(p, z, 0x1.5555555555555p-5);              //  1/4!
    p = ccc_fma(p, z, -0x1.0000000000000p-1);             // -1/2!
    return ccc_fma(z, p, 1.0);
}

CCC_HD_CALL double ccc_sin(double x) {
    if (x != x) return x + x;
    double ax = x < 0 ? -x : x;
    if (ax <= 1.1) return ccc_sin_series(x);
    // halve until in range, then s(2a) = 2 s(a) c(a), c(2a) = 1 - 2 s(a)^2
    int k = 0;
    double h = x;
    while ((h < 0 ? -h : h) > 1.1 && k < 64) { h = h * 0.5; ++k; }
    double s = ccc_sin_series(h), c = ccc_cos_series(h);
    for (int i = 0; i < k; ++i) {
        double s2 = 2.0 * s * c;
        double c2 = ccc_sub(1.0, ccc_mul(2.0 * s, s));
        s = s2;
        c = c2;
    }
    return s;
}

CCC_HD_CALL double ccc_cos(double x) {
    if (x != x) return x + x;
    double ax = x < 0 ? -x : x;
    if (ax <= 1.1) return ccc_cos_series(x);
    int k = 0;
    double h = x;
    while ((h < 0 ? -h : h) > 1.1 && k < 64) { h = h * 0.5; ++k; }
    double s = ccc_sin_series(h), c = ccc_cos_series(h);
    for (int i = 0; i < k; ++i) {
        double s2 = 2.0 * s * c;
        double c2 = ccc_sub(1.0, ccc_mul(2.0 * s, s));
        s = s2;
        c = c2;
    }
    return c;
}

// asin on [0, 1/2]: x + x z P(z), z = x^2, with P(z) = E(w) + z O(w), w = z^2 (the even and
// odd coefficient halves run as two independent fma chains)
CCC_HD double ccc_asin_small(double x) {
    double z = x * x;
    double w = z * z;
    double pe = 0x1.cf7dea5b6e830p-10;
    pe = ccc_fma(pe, w, 0x1.018f963c229bfp-9);
    pe = ccc_fma(pe, w, 0x1.208d3570ae5a6p-9);
    pe = ccc_fma(pe, w, 0x1.464c0950f7d47p-9);
    pe = ccc_fma(pe, w, 0x1.750de64d7d05fp-9);
    pe = ccc_fma(pe, w, 0x1.b026f57b13b14p-9);
    pe = ccc_fma(pe, w, 0x1.fcaf8fb6db6dbp-9);
    pe = ccc_fma(pe, w, 0x1.31683bdef7bdfp-8);
    pe = ccc_fma(pe, w, 0x1.782dda12f684cp-8);
    pe = ccc_fma(pe, w, 0x1.df3bd37a6f4dfp-8);
    pe = ccc_fma(pe, w, 0x1.3fde50d79435ep-7);
    pe = ccc_fma(pe, w, 0x1.c99999999999ap-7);
    pe = ccc_fma(pe, w, 0x1.6e8ba2e8ba2e9p-6);
    pe = ccc_fma(pe, w, 0x1.6db6db6db6db7p-5);
    pe = ccc_fma(pe, w, 0x1.5555555555555p-3);
    double po = 0x1.e82be60d9127ep-10;
    po = ccc_fma(po, w, 0x1.1052bc5fa960ap-9);
    po = ccc_fma(po, w, 0x1.3275586c5f2f0p-9);
    po = ccc_fma(po, w, 0x1.5c5f56efaaaabp-9);
    po = ccc_fma(po, w, 0x1.90cb77f60c7cep-9);
    po = ccc_fma(po, w, 0x1.d3d2a8e0dd67dp-9);
    po = ccc_fma(po, w, 0x1.15ee9d45d1746p-8);
    po = ccc_fma(po, w, 0x1.51ba308d3dcb1p-8);
    po = ccc_fma(po, w, 0x1.a6863d70a3d71p-8);
    po = ccc_fma(po, w, 0x1.12ef3cf3cf3cfp-7);
    po = ccc_fma(po, w, 0x1.7a87878787878p-7);
    po = ccc_fma(po, w, 0x1.1c4ec4ec4ec4fp-6);
    po = ccc_fma(po, w, 0x1.f1c71c71c71c7p-6);
    po = ccc_fma(po, w, 0x1.3333333333333p-4);
    double p = ccc_fma(z, po, pe);
    return ccc_fma(x * z, p, x);
}

CCC_HD_CALL double ccc_acos(double x) {
    const double PI = 0x1.921fb54442d18p+1;
    const double PI_2 = 0x1.921fb54442d18p+0;
    if (x != x) return x + x;
    if (x > 1.0 || x < -1.0) return (x - x) / (x - x);   // NaN outside the domain
    if (x >= 0.5) return 2.0 * ccc_asin_small(ccc_sqrt((1.0 - x) * 0.5));
    if (x <= -0.5) return ccc_sub(PI, 2.0 * ccc_asin_small(ccc_sqrt((1.0 + x) * 0.5)));
    return PI_2 - ccc_asin_small(x);
}
