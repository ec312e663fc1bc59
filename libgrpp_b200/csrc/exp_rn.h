// exp(x) rounded to nearest, for the values that must reproduce libgrpp's to the last bit.
//
// libgrpp's radial integrands multiply and sum exponentials of the C library, whose exp is
// correctly rounded except in rare hard cases; the device's exp is within one unit in the last
// place of it. Contracted Gaussians with coefficients of both signs cancel in the integrand,
// which turns those last-bit differences into tens of units in the last place of the radial
// integrals and flips their absolute 1e-16 stop tests. This function evaluates exp in
// double-double arithmetic and rounds once, so its results equal the correctly rounded ones
// except where the exact value lies within about 2^-100 relative of a rounding boundary:
//   x = k ln2 + r, k = rint(x / ln2), |r| <= ln2 / 2, with ln2 as a double-double (Cody and
//   Waite's reduction; k ln2_hi split exactly by a fused multiply-add);
//   exp(r) = sum_n r^n / n!, the terms up to r^7 by Horner's rule in double-double arithmetic,
//   the tail r^8 / 8! ... r^24 / 24! in double (below 2^-60 of the result);
//   the double-double sum rounded to double and scaled by 2^k.
// Below the smallest subnormal the result is 0; in the subnormal range the scaling rounds a
// second time (those values are below 2.3e-308). Written for host and device: the fused
// multiply-adds are explicit, and the error-free transformations contain no product that a
// compiler could contract.
#pragma once

#include <cmath>

#ifndef GRPP_HD
#ifdef __CUDACC__
#define GRPP_HD __host__ __device__
#else
#define GRPP_HD
#endif
#endif

namespace grpp {

GRPP_HD inline void exp_rn_dd_mul_add(double &ah, double &al, double rh, double rl, double ch, double cl)
{
    // (ah, al) = (ah, al) * (rh, rl) + (ch, cl)
    const double p = ah * rh;
    double pe = fma(ah, rh, -p);
    pe = fma(ah, rl, pe);
    pe = fma(al, rh, pe);
    // p + pe, then + c by a two-sum on the leading parts
    const double s = p + ch;
    const double bb = s - p;
    const double e = (p - (s - bb)) + (ch - bb);
    const double lo = e + pe + cl;
    ah = s + lo;
    al = lo - (ah - s);
}

GRPP_HD inline double exp_rn(double x)
{
    if (x != x) return x;
    if (x < -745.2) return 0.0;
    if (x > 709.78) return HUGE_VAL;
    const double ln2_hi = 0x1.62e42fefa39efp-1, ln2_lo = 0x1.abc9e3b39803fp-56;
    const double k = rint(x * 0x1.71547652b82fep+0);
    const double p = k * ln2_hi;
    const double pe = fma(k, ln2_hi, -p);  // k ln2_hi = p + pe exactly
    const double s = x - p;                // exact: x and p are within a factor of 2 (or k = 0)
    // r = s - pe - k ln2_lo as a double-double
    double rh = s - pe;
    double rl = (s - rh) - pe;
    rl = fma(-k, ln2_lo, rl);
    const double t = rh + rl;
    rl = rl - (t - rh);
    rh = t;
    // tail: sum_{n=8}^{24} r^(n-8) / n! by Horner's rule in double
    double tail = 1.0 / 620448401733239439360000.0;
    tail = fma(tail, rh, 1.0 / 25852016738884976640000.0);
    tail = fma(tail, rh, 1.0 / 1124000727777607680000.0);
    tail = fma(tail, rh, 1.0 / 51090942171709440000.0);
    tail = fma(tail, rh, 1.0 / 2432902008176640000.0);
    tail = fma(tail, rh, 1.0 / 121645100408832000.0);
    tail = fma(tail, rh, 1.0 / 6402373705728000.0);
    tail = fma(tail, rh, 1.0 / 355687428096000.0);
    tail = fma(tail, rh, 1.0 / 20922789888000.0);
    tail = fma(tail, rh, 1.0 / 1307674368000.0);
    tail = fma(tail, rh, 1.0 / 87178291200.0);
    tail = fma(tail, rh, 1.0 / 6227020800.0);
    tail = fma(tail, rh, 1.0 / 479001600.0);
    tail = fma(tail, rh, 1.0 / 39916800.0);
    tail = fma(tail, rh, 1.0 / 3628800.0);
    tail = fma(tail, rh, 1.0 / 362880.0);
    tail = fma(tail, rh, 1.0 / 40320.0);
    // n = 7 .. 0 in double-double, 1/n! as (high, low) parts
    double ah = tail, al = 0.0;
    exp_rn_dd_mul_add(ah, al, rh, rl, 0x1.a01a01a01a01ap-13, 0x1.a01a01a01a01ap-73);
    exp_rn_dd_mul_add(ah, al, rh, rl, 0x1.6c16c16c16c17p-10, -0x1.f49f49f49f49fp-65);
    exp_rn_dd_mul_add(ah, al, rh, rl, 0x1.1111111111111p-7, 0x1.1111111111111p-63);
    exp_rn_dd_mul_add(ah, al, rh, rl, 0x1.5555555555555p-5, 0x1.5555555555555p-59);
    exp_rn_dd_mul_add(ah, al, rh, rl, 0x1.5555555555555p-3, 0x1.5555555555555p-57);
    exp_rn_dd_mul_add(ah, al, rh, rl, 0x1.0p-1, 0.0);
    exp_rn_dd_mul_add(ah, al, rh, rl, 1.0, 0.0);
    exp_rn_dd_mul_add(ah, al, rh, rl, 1.0, 0.0);
    // one rounding of the double-double, then the exact (or, subnormal, once rounded) scaling
    return ldexp(ah + al, (int)k);
}

}  // namespace grpp
