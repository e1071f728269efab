// ccc_ddmul.h — certified double-double products used by the cubic solver.
//
// The reference computes b^3, a^2, a^3 and f^3 inside its Cardano solver with the CAMPARY
// library's certifiedMul<1,1,2> and certifiedMul<2,1,2> (include/campari/multiplication.h:
// 132-184, errorFreeTransf.h:38-81, renorm.h:138-149) and keeps only the leading term.
// The leading term is not always the correctly rounded product, so the solver's branch
// decisions depend on the exact algorithm.  This header restates that published algorithm
// (Joldes, Muller, Popescu et al., "Arithmetic algorithms for extended precision using
// floating-point expansions", IEEE TC 2016: fixed-point bins of 45 bits, biased by 1.5 ulp
// constants, followed by VecSumErrBranch renormalisation) for the two shapes the solver
// needs: an expansion of K in {1,2} terms times one double, rounded to R = 2 terms.
//
// Every operation is a single IEEE-754 double add / multiply / fma, so host and device
// produce identical bits.
#pragma once

#include "ccc_libm.h"

CCC_HD double ccc_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return fma(a, b, c);
#endif
}

// s = fl(a + b) and the exact error b - (s - a); valid when |a| >= |b|
CCC_HD double ccc_fast_two_sum(double a, double b, double* err) {
    double s = a + b;
    double z = s - a;
    *err = b - z;
    return s;
}

// r[0..1] = expansion (x[0] (+ x[1] when k == 2)) * y, bins of 45 bits, 4 live bins.
CCC_HD void ccc_certmul_r2(const double* x, int k, double y, double* r) {
    const int BIN = 45;
    const int NB = 4;                      // 2*53/45 + 2
    double bins[NB + 2], bias[NB + 2];
    int ex0 = ccc_frexp_exp(x[0]);
    int ex1 = (k > 1) ? ccc_frexp_exp(x[1]) : 0;
    int ey = ccc_frexp_exp(y);
    int e0 = ex0 + ey;
    bias[0] = ccc_ldexp(1.5, e0 - BIN + 52);
    bins[0] = bias[0];
    const double step = ccc_pow2i(-BIN);
    for (int i = 1; i < NB + 2; ++i) {
        bias[i] = bias[i - 1] * step;
        bins[i] = bias[i];
    }
    for (int i = 0; i < k; ++i) {
        double xi = x[i];
        // a zero partial product leaves every bin unchanged
        if (xi == 0.0 || y == 0.0) continue;
        int l = e0 - ((i == 0 ? ex0 : ex1) + ey);
        int sh = l / BIN;
        l = l - sh * BIN;
        if (sh < 0 || sh >= NB - 1) continue;
        double p = xi * y;
        double e = ccc_fma(xi, y, -p);
        if (l < 30) {
            bins[sh] = ccc_fast_two_sum(bins[sh], p, &p);
            bins[sh + 1] = bins[sh + 1] + p;
            bins[sh + 1] = ccc_fast_two_sum(bins[sh + 1], e, &e);
            bins[sh + 2] = bins[sh + 2] + e;
        } else if (l < 37) {
            bins[sh] = ccc_fast_two_sum(bins[sh], p, &p);
            bins[sh + 1] = bins[sh + 1] + p;
            bins[sh + 1] = ccc_fast_two_sum(bins[sh + 1], e, &e);
            bins[sh + 2] = ccc_fast_two_sum(bins[sh + 2], e, &e);
            bins[sh + 3] = bins[sh + 3] + e;
        } else {
            bins[sh] = ccc_fast_two_sum(bins[sh], p, &p);
            bins[sh + 1] = ccc_fast_two_sum(bins[sh + 1], p, &p);
            bins[sh + 2] = bins[sh + 2] + p;
            bins[sh + 2] = ccc_fast_two_sum(bins[sh + 2], e, &e);
            bins[sh + 3] = bins[sh + 3] + e;
        }
    }
    for (int i = 0; i < NB; ++i) bins[i] = bins[i] + (-bias[i]);
    // VecSumErrBranch: carry a running sum, emit a term whenever its error is non-zero
    int out = 0;
    double carry = bins[0];
    for (int i = 1; i < NB && out < 2; ++i) {
        double err;
        double s = ccc_fast_two_sum(carry, bins[i], &err);
        r[out] = s;
        carry = err;
        if (carry == 0.0) carry = s;
        else ++out;
    }
    if (out < 2 && carry != 0.0) r[out++] = carry;
    for (int i = out; i < 2; ++i) r[i] = 0.0;
}

// Leading terms the solver uses: x^2 (as a 2-term expansion) and x^3 = (x^2) * x.
CCC_HD void ccc_sq_dd(double x, double* r2) {
    ccc_certmul_r2(&x, 1, x, r2);
}
CCC_HD double ccc_cube_hi(double x) {
    double s[2], c[2];
    ccc_certmul_r2(&x, 1, x, s);
    ccc_certmul_r2(s, 2, x, c);
    return c[0];
}
