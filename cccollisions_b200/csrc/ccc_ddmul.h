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
// produce identical bits; every product is a ccc_mul, so the results stay the same in a
// translation unit compiled with multiply-add contraction.
#pragma once

#include "ccc_libm.h"

// Values are passed and returned by value (no pointers into locals), which keeps the
// device code straightforward.
struct ccc_dd {
    double hi, lo;
};

// s = fl(a + b) and the exact error b - (s - a); valid when |a| >= |b|
CCC_HD ccc_dd ccc_fast_two_sum(double a, double b) {
    ccc_dd r;
    r.hi = a + b;
    double z = r.hi - a;
    r.lo = b - z;
    return r;
}

// (x0 (+ x1 when K == 2)) * y rounded to a 2-term expansion: bins of 45 bits, 4 live bins.
// K is a template parameter so that the solver's six products a call compile to straight
// code (the first partial product always lands at bin offset 0).
template <int K> CCC_HD ccc_dd ccc_certmul_k(double x0, double x1, double y) {
    const int k = K;
    const int BIN = 45;
    double b0, b1, b2, b3, b4, b5;           // bins (6 slots, the last two spill targets)
    double s0, s1, s2, s3;                   // biases of the live bins
    int ex0 = ccc_frexp_exp(x0);
    int ex1 = (k > 1) ? ccc_frexp_exp(x1) : 0;
    int ey = ccc_frexp_exp(y);
    int e0 = ex0 + ey;
    const double step = ccc_pow2i(-BIN);
    s0 = ccc_ldexp(1.5, e0 - BIN + 52);
    s1 = ccc_mul(s0, step);
    s2 = ccc_mul(s1, step);
    s3 = ccc_mul(s2, step);
    double s4 = ccc_mul(s3, step);
    double s5 = ccc_mul(s4, step);
    b0 = s0; b1 = s1; b2 = s2; b3 = s3; b4 = s4; b5 = s5;
    for (int i = 0; i < k; ++i) {
        double xi = i == 0 ? x0 : x1;
        // a zero partial product leaves every bin unchanged
        if (xi == 0.0 || y == 0.0) continue;
        int l = e0 - ((i == 0 ? ex0 : ex1) + ey);
        int sh = l / BIN;
        l = l - sh * BIN;
        if (sh < 0 || sh >= 3) continue;
        double p = ccc_mul(xi, y);
        double e = ccc_fma(xi, y, -p);
        // the bins touched are sh .. sh+3; work on a window w0..w3 and write it back
        double w0 = sh == 0 ? b0 : (sh == 1 ? b1 : b2);
        double w1 = sh == 0 ? b1 : (sh == 1 ? b2 : b3);
        double w2 = sh == 0 ? b2 : (sh == 1 ? b3 : b4);
        double w3 = sh == 0 ? b3 : (sh == 1 ? b4 : b5);
        ccc_dd t;
        if (l < 30) {
            t = ccc_fast_two_sum(w0, p); w0 = t.hi; p = t.lo;
            w1 = w1 + p;
            t = ccc_fast_two_sum(w1, e); w1 = t.hi; e = t.lo;
            w2 = w2 + e;
        } else if (l < 37) {
            t = ccc_fast_two_sum(w0, p); w0 = t.hi; p = t.lo;
            w1 = w1 + p;
            t = ccc_fast_two_sum(w1, e); w1 = t.hi; e = t.lo;
            t = ccc_fast_two_sum(w2, e); w2 = t.hi; e = t.lo;
            w3 = w3 + e;
        } else {
            t = ccc_fast_two_sum(w0, p); w0 = t.hi; p = t.lo;
            t = ccc_fast_two_sum(w1, p); w1 = t.hi; p = t.lo;
            w2 = w2 + p;
            t = ccc_fast_two_sum(w2, e); w2 = t.hi; e = t.lo;
            w3 = w3 + e;
        }
        if (sh == 0) { b0 = w0; b1 = w1; b2 = w2; b3 = w3; }
        else if (sh == 1) { b1 = w0; b2 = w1; b3 = w2; b4 = w3; }
        else { b2 = w0; b3 = w1; b4 = w2; b5 = w3; }
    }
    b0 = b0 + (-s0);
    b1 = b1 + (-s1);
    b2 = b2 + (-s2);
    b3 = b3 + (-s3);
    // VecSumErrBranch: carry a running sum, emit a term whenever its error is non-zero
    double r0 = 0.0, r1 = 0.0;
    int out = 0;
    double carry = b0;
    for (int i = 1; i < 4 && out < 2; ++i) {
        double bi = i == 1 ? b1 : (i == 2 ? b2 : b3);
        ccc_dd t = ccc_fast_two_sum(carry, bi);
        if (out == 0) r0 = t.hi;
        else r1 = t.hi;
        carry = t.lo;
        if (carry == 0.0) carry = t.hi;
        else ++out;
    }
    if (out < 2 && carry != 0.0) {
        if (out == 0) r0 = carry;
        else r1 = carry;
        ++out;
    }
    if (out < 1) r0 = 0.0;
    if (out < 2) r1 = 0.0;
    ccc_dd r;
    r.hi = r0;
    r.lo = r1;
    return r;
}


// the same with the number of terms K in {1, 2} given at run time (kept out of line: the
// short paths below call it only for their rare fallback cases)
CCC_HD_CALL ccc_dd ccc_certmul(double x0, double x1, int k, double y) {
    return k > 1 ? ccc_certmul_k<2>(x0, x1, y) : ccc_certmul_k<1>(x0, x1, y);
}

// ---- Short paths with the same results --------------------------------------------------
//
// With x, y finite and non-zero, e0 = exponent(x) + exponent(y) (frexp exponents), the bins
// of ccc_certmul_k hold, after the un-biasing, b0 = the partial products rounded to the grid
// 2^(e0-45), b1 = the rest rounded to the grid 2^(e0-90), b2, b3 = the remainder; each bin
// is exact for these magnitudes as long as the bias constants are normal numbers.  Then:
//
//  * K = 1 (x * y = p + e exactly, p = RN(x y), e = fma(x, y, -p)): b0 + b1 = p + E with E = e
//    rounded to the grid 2^(e0-90), so |E| <= ulp(p) / 2, and the renormalisation returns
//    (p, e) unless |E| = ulp(p) / 2 exactly, where RN(p + E) may tie away from p.  That
//    needs |e| within 2^(e0-91) of ulp(p) / 2.
//  * K = 2, leading term only (V = (x0 + x1) y exactly, |x1| <= ulp(x0) / 2): b0 + b1
//    differs from V by less than 2^(e0-88), and the leading term is RN(b0 + b1) (or, when
//    that sum is exact, the rounded sum with the next bins), so it is RN(V) whenever V is
//    farther than 2^(e0-88) from the midpoint of two neighbouring doubles.
//
// The short paths compute (p, e) and RN(V) with TwoProd and a compensated sum (error far
// below 2^(e0-100)) and use them when the distance to the critical point exceeds 2^(e0-80)
// and the operands are in the range where every bias constant is normal; anything else
// (zeros, ties and near-ties, powers of two, extreme exponents, non-finite values) takes
// the bin algorithm itself.  The CPU test suite checks both paths against each other on
// random, short-mantissa (exact and tied products) and special operands.
CCC_HD int ccc_bexp(double x) { return (int)((ccc_dbits(x) >> 52) & 0x7ff); }
CCC_HD bool ccc_pow2_or_special(double x) {
    uint64_t u = ccc_dbits(x);
    int be = (int)((u >> 52) & 0x7ff);
    return (u & 0x000fffffffffffffull) == 0 || be == 0 || be == 0x7ff;
}

// certifiedMul<1,1,2>(x, y)
CCC_HD ccc_dd ccc_certmul1(double x, double y) {
    const int bx = ccc_bexp(x), by = ccc_bexp(y);
    const int e0 = (bx - 1022) + (by - 1022);
    const double p = ccc_mul(x, y);
    const double e = ccc_fma(x, y, -p);
    bool easy = x != 0.0 && y != 0.0 && bx != 0 && bx != 0x7ff && by != 0 && by != 0x7ff && e0 >= -700 &&
                e0 <= 1000 && !ccc_pow2_or_special(p);
    if (easy) {
        const double half_ulp = ccc_pow2i(ccc_bexp(p) - 1023 - 53);
        easy = half_ulp - fabs(e) > ccc_pow2i(e0 - 80);
    }
    if (easy) {
        ccc_dd r;
        r.hi = p;
        r.lo = e;
        return r;
    }
    return ccc_certmul(x, 0.0, 1, y);
}

// certifiedMul<2,1,2>((x0, x1), y), leading term
CCC_HD double ccc_certmul2_hi(double x0, double x1, double y) {
    const int b0 = ccc_bexp(x0), by = ccc_bexp(y);
    const int e0 = (b0 - 1022) + (by - 1022);
    const double p0 = ccc_mul(x0, y);
    const double er = ccc_fma(x0, y, -p0);
    const double rest = er + ccc_mul(x1, y);
    const double c = p0 + rest;
    bool easy = x0 != 0.0 && y != 0.0 && b0 != 0 && b0 != 0x7ff && by != 0 && by != 0x7ff && e0 >= -700 &&
                e0 <= 1000 && !ccc_pow2_or_special(c) && ccc_bexp(x1) != 0x7ff &&
                fabs(x1) <= ccc_pow2i(b0 - 1023 - 53);
    if (easy) {
        const double res = (p0 - c) + rest;
        const double half_ulp = ccc_pow2i(ccc_bexp(c) - 1023 - 53);
        easy = fabs(fabs(res) - half_ulp) > ccc_pow2i(e0 - 80);
    }
    if (easy) return c;
    return ccc_certmul(x0, x1, 2, y).hi;
}

// Leading terms the solver uses: x^2 (as a 2-term expansion) and x^3 = (x^2) * x.
CCC_HD ccc_dd ccc_sq_dd(double x) { return ccc_certmul1(x, x); }
CCC_HD double ccc_cube_hi(double x) {
    ccc_dd s = ccc_sq_dd(x);
    return ccc_certmul2_hi(s.hi, s.lo, x);
}
