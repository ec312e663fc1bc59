// Device special functions of the GRPP engine (FP64).
//
//   bessel_scaled      M_l(x) = exp(-x) i_l(x), the scheme of
//                      libgrpp/specfunc_scaled_mod_sph_bessel.c:72-122: x <= 1e-7 series,
//                      x <= 16 4th-order Taylor about the nearest 0.01 point, asymptotic above
//   bessel_scaled_row  the same for all orders 0..lmax at one x (one table row)
//   boys               F_n(x), 6th-order Taylor on a 0.1 grid below 30, asymptotic above
//                      (libgrpp/specfunc_boys.c:21-47)
//   gfun_values        G_n(x) = int_0^1 t^(2n) exp(-x(1-t^2)) dt: series + downward
//                      recursion for x <= 12, Dawson + upward recursion above
//                      (libgrpp/specfunc_gfun.c:40-93)
//   dawson             Daw(y) for y >= 3: Taylor about a 1/32 grid with derivatives from
//                      Daw' = 1 - 2 y Daw; asymptotic series for large y
#pragma once

#include "grpp_common.cuh"

namespace grpp {

// device table addresses; defined once, in the single CUDA translation unit that includes this header
__constant__ DeviceTables c_tab;

__device__ __forceinline__ double bessel_small(int n, double x)
{
    switch (n) {
    case 0: return 1.0 - x;
    case 1: return (1.0 - x) * x * (1.0 / 3.0);
    case 2: return (1.0 - x) * x * x * (1.0 / 15.0);
    default: return 0.0;
    }
}

__device__ __forceinline__ double bessel_asym(int n, double x)
{
    const double *c = c_tab.rfun + n * kRfunL;
    double inv = 1.0 / (-x), den = 1.0, sum = 0.0;
    for (int k = 0; k <= n; k++) {
        sum += __ldg(c + k) * den;
        den *= inv;
    }
    return sum / (2.0 * x);
}

__device__ __forceinline__ double taylor4(const double *d, double dx)
{
    double dx2 = dx * dx, dx3 = dx2 * dx, dx4 = dx3 * dx;
    return __ldg(d) + __ldg(d + 1) * dx + __ldg(d + 2) * dx2 * 0.5 + __ldg(d + 3) * dx3 * (1.0 / 6.0) +
           __ldg(d + 4) * dx4 * (1.0 / 24.0);
}

__device__ __forceinline__ double bessel_scaled(int n, double x)
{
    if (x <= 1e-7) return bessel_small(n, x);
    if (x <= 16.0) {
        int i0 = (int)(round(x * 100) + 1e-5);
        double dx = x - i0 * 0.01;
        return taylor4(c_tab.bessel + ((size_t)i0 * kBesL + n) * 5, dx);
    }
    return bessel_asym(n, x);
}

// M_l(x) for l = 0..lmax (lmax < kBesL); out has lmax+1 entries.
template <int LMAX_STATIC>
__device__ __forceinline__ void bessel_scaled_row(int lmax, double x, double *out)
{
    if (x <= 1e-7) {
#pragma unroll
        for (int l = 0; l <= LMAX_STATIC; l++)
            if (l <= lmax) out[l] = bessel_small(l, x);
    } else if (x <= 16.0) {
        int i0 = (int)(round(x * 100) + 1e-5);
        double dx = x - i0 * 0.01;
        double dx2 = dx * dx, dx3 = dx2 * dx, dx4 = dx3 * dx;
        double h2 = dx2 * 0.5, h3 = dx3 * (1.0 / 6.0), h4 = dx4 * (1.0 / 24.0);
        const double *d = c_tab.bessel + (size_t)i0 * kBesL * 5;
#pragma unroll
        for (int l = 0; l <= LMAX_STATIC; l++)
            if (l <= lmax) {
                const double *e = d + 5 * l;
                // same association as the scalar form: d0 + d1 dx + d2 dx2 0.5 + ...
                out[l] = __ldg(e) + __ldg(e + 1) * dx + __ldg(e + 2) * dx2 * 0.5 + __ldg(e + 3) * dx3 * (1.0 / 6.0) +
                         __ldg(e + 4) * dx4 * (1.0 / 24.0);
                (void)h2;
                (void)h3;
                (void)h4;
            }
    } else {
#pragma unroll
        for (int l = 0; l <= LMAX_STATIC; l++)
            if (l <= lmax) out[l] = bessel_asym(l, x);
    }
}

__device__ __forceinline__ double dfact(int n) { return __ldg(c_tab.dfact + n + 1); }

__device__ __forceinline__ double boys(int n, double x)
{
    if (x <= 30.0) {
        int idx = (int)(round(x / 0.1) + 1e-6);
        double dx = x - idx * 0.1;
        double dx2 = dx * dx, dx3 = dx * dx2, dx4 = dx * dx3, dx5 = dx * dx4, dx6 = dx * dx5;
        const double *b = c_tab.boys + idx * kBoysNN + n;
        return +__ldg(b) - __ldg(b + 1) * dx + __ldg(b + 2) * dx2 / 2.0 - __ldg(b + 3) * dx3 / 6.0 +
               __ldg(b + 4) * dx4 / 24.0 - __ldg(b + 5) * dx5 / 120.0 + __ldg(b + 6) * dx6 / 720.0;
    }
    return dfact(2 * n - 1) / pow(2.0, n + 1) * sqrt(kPi / pow(x, 2 * n + 1));
}

__device__ inline double dawson(double y)
{
    if (y < kDawY0) {
        // exp(-y^2) sum_k y^(2k+1)/(k!(2k+1)), all terms positive
        double y2 = y * y, p = y, s = y;
        for (int k = 1; k < 200; k++) {
            p *= y2 / k;
            double t = p / (2.0 * k + 1.0);
            s += t;
            if (t < 1e-18 * s) break;
        }
        return exp(-y2) * s;
    }
    int j = (int)round((y - kDawY0) / kDawH);
    if (j < kDawNY) {
        double y0 = kDawY0 + j * kDawH, h = y - y0;
        double f0 = __ldg(c_tab.dawson + j), f1 = 1.0 - 2.0 * y0 * f0;
        double sum = f0 + f1 * h, hk = h, fkm1 = f0, fk = f1;
        for (int k = 1; k < 18; k++) {
            double fk1 = -2.0 * y0 * fk - 2.0 * k * fkm1;
            hk *= h / (k + 1);
            sum += fk1 * hk;
            fkm1 = fk;
            fk = fk1;
        }
        return sum;
    }
    // 1/(2y) sum_k (2k-1)!! / (2y^2)^k while the terms decrease
    double x2 = 2.0 * y * y, term = 1.0, s = 1.0;
    for (int k = 1; k < 200; k++) {
        double nt = term * (2.0 * k - 1.0) / x2;
        if (nt >= term) break;
        term = nt;
        s += term;
        if (term < 1e-18 * s) break;
    }
    return s / (2.0 * y);
}

// g[0..nmax]
__device__ inline void gfun_values(double x, int nmax, double *g)
{
    if (x <= 12.0) {
        double ex = exp(-x), sum = 0.0, xk = 1.0, fk = 1.0;
        for (int k = 0; k < 100; k++) {
            if (k > 0) {
                xk *= x;
                fk *= k;
            }
            double c = ex * xk / fk / (2.0 * nmax + 2.0 * k + 1.0);
            sum += c;
            if (fabs(c) < 1e-15) break;
        }
        g[nmax] = sum;
        for (int n = nmax; n > 0; n--) g[n - 1] = (1.0 - 2.0 * x * g[n]) / (2.0 * n - 1.0);
    } else {
        double sx = sqrt(x);
        g[0] = dawson(sx) / sx;
        for (int n = 0; n < nmax; n++) g[n + 1] = (1.0 - (2 * n + 1) * g[n]) / (2.0 * x);
    }
}

// gfun_values by one warp (all 32 lanes call it; g[] is written by lane 0). For x <= 12
// lane k forms the series term k with the same product chains as the serial loop
// (x^k and k! by repeated multiplication from 1), and lane 0 adds the terms in order up
// to the first one below 1e-15, as the serial loop does; the recursions stay on lane 0.
__device__ inline void gfun_values_warp(double x, int nmax, double *g, int lane)
{
    if (x <= 12.0) {
        const double ex = exp(-x);
        double sum = 0.0;
        for (int k0 = 0; k0 < 100; k0 += 32) {
            const int k = k0 + lane;
            double xk = 1.0, fk = 1.0;
            for (int i = 1; i <= k; i++) {
                xk *= x;
                fk *= i;
            }
            const double c = ex * xk / fk / (2.0 * nmax + 2.0 * k + 1.0);
            const unsigned stop = __ballot_sync(0xffffffffu, k >= 99 || fabs(c) < 1e-15);
            const int last = stop ? __ffs(stop) - 1 : 31;  // last term added in this block
            for (int j = 0; j <= last; j++) {
                const double cj = __shfl_sync(0xffffffffu, c, j);
                if (lane == 0) sum += cj;
            }
            if (stop) break;
        }
        if (lane == 0) {
            g[nmax] = sum;
            for (int n = nmax; n > 0; n--) g[n - 1] = (1.0 - 2.0 * x * g[n]) / (2.0 * n - 1.0);
        }
    } else if (lane == 0) {
        gfun_values(x, nmax, g);
    }
}

// (2a/pi)^(3/4) (4a)^(L/2)  (libgrpp/norm_gaussian.c:16-23)
__device__ __forceinline__ double gaussian_norm(int L, double a)
{
    return pow(2 * a / kPi, 0.75) * pow(4 * a, 0.5 * L);
}

}  // namespace grpp
