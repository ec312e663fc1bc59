// Radial integrals of the semilocal (type 2) and spin-orbit GRPP terms.
//
// Reference algorithm: libgrpp/radial_type2_integral.c:101-489 and
// libgrpp/screening.c:193-378. For one task (shells A, B, centre C) and each
// semilocal potential p of the centre, the table
//   Q_p[l1][l2][N] = int_0^inf U_p(r) F^A_l1(r) F^B_l2(r) r^N dr,
//   F_l(r) = sum_i c_i N_i exp(-a_i (r-CA)^2) M_l(2 a_i CA r),
// with l1 <= L_p + la, l2 <= L_p + lb, N <= la + lb, is computed by
//   * the one-centre analytic formula when CA = CB = 0;
//   * otherwise, per entry, the Shaw-Hill screening estimate (entries below
//     1e-16 return the estimate) and the nested Log3 quadrature
//     r_i = -5 ln(1 - x_i^3), levels of 31, 63, ..., 8191 points, stopping when
//     |S_L - S_{L-1}| <= 1e-16 unless |S|/|estimate| < 1e-3, capped at 8191 points.
//
// GPU mapping, two kernels:
//  * radial_screen_flat_kernel: one thread per (task, entry) over the entries of the
//    whole batch. A thread walks the primitive triples (i, j, k) of its entry in
//    libgrpp's order and stops at the first failing one, exactly as libgrpp does,
//    so the estimate and the gate decision are those of the reference, and no
//    work is spent on triples libgrpp never evaluates. One-centre tasks get their
//    analytic table here and need no grid walk.
//  * radial_walk_kernel: one CTA per task that has entries left. The grid is
//    walked level by level in chunks of one point per thread; a point's
//    integrand values
//      w U_p(r) for every potential, F^A_l, F^B_l for every order, r^N,
//    are evaluated once and shared by all potentials and entries; every thread
//    then advances the running sums of the entries it owns, point by point in
//    the reference's order and association ((((w U) F1) F2) r^N).
#pragma once

#include "grpp_common.cuh"
#include "specfunc.cuh"
#include "exp_rn.h"

namespace grpp {

constexpr int kRadThreads = 128;
#ifndef GRPP_SCR_MINB
#define GRPP_SCR_MINB 5  // resident 128-thread blocks per SM asked of the flat screening kernel
#endif
constexpr int kRadMaxPrims = 64;     // primitives per shell on the radial path
constexpr int kRadMaxPots = 24;      // semilocal potentials per centre
constexpr int kRadMaxTerms = 256;    // potential terms per centre (all semilocal potentials)
constexpr int kRadMaxLam = 24;       // lambda <= L + l
constexpr int kRadMaxN = 24;         // N <= la + lb
constexpr int kRadMaxLevel = 8;      // 8191 points
constexpr int kRadMaxEntries = 16384;

// entry flag bits
constexpr uint8_t kEntActive = 1, kEntScrOk = 2;

// A run of used entries of one semilocal potential of one task, screened by one block of
// radial_screen_unit_kernel (or, for short runs, by the flat kernel): item, potential index,
// offset of the potential's (l1, l2, N) box within the item's table, offset of the run in ulist,
// number of entries.
struct ScrUnit {
    int item, pot, pe, uo, ne;
};

struct RadialArgs {
    int n_items;
    int64_t n_entries;          // total entries of all items (flat screening)
    const int *item_task;
    const int *task_a, *task_b, *task_c;
    const int *shell_L;
    const double *shell_origin;
    // shrunk (|c| > 1e-14) primitives with the normalisation folded in (radial_type2_integral.c:164-172)
    const int *rp_off, *rp_n;
    const double *rp_coef, *rp_alpha;
    // unshrunk primitives (one-centre branch, radial_type2_integral.c:126-155)
    const int *shell_nprim, *shell_prim_off;
    const double *prim_coef, *prim_alpha;
    const double *centre_origin;
    const int *centre_grpp;
    const int *grpp_sl_off, *grpp_sl_n, *sl_pot;
    const int *pot_L, *pot_nprim, *pot_prim_off, *pot_powers;
    const double *pot_coef, *pot_alpha;
    const int64_t *q_off;       // per item
    // walk: two lists of active entry indices (uint16) of up to list_max entries each, after
    // chunk_doubles doubles of point arrays in dynamic shared memory; list_max = 0: no lists
    int list_max, chunk_doubles;
    // w U_p(r) at every grid point per GRPP and semilocal potential slot, at
    // wu[(grpp * wu_npot + slot) * kRadGridPts + point] (wu_table_kernel); null: the walk
    // evaluates the potential terms itself
    const double *wu;
    int wu_npot;
    // F_l(r) = sum_i c_i N_i exp(-a_i (r-CS)^2) M_l(2 a_i CS r), l = 0..fp_lmax[k], at every grid
    // point for each (shell, centre) pair k of the batch (ftab_kernel), at
    // ftab[fp_off[k] + l * kRadGridPts + point]; item_fa / item_fb: the pairs (A, C) and (B, C)
    // of an item. ftab null: the walk evaluates F itself
    const double *ftab;
    const int64_t *fp_off;
    const int *fp_shell, *fp_centre, *fp_lmax, *item_fa, *item_fb;
    int n_fpairs;
    // entries the angular sums read, per item: u_off[item] = first used index; per class
    // (L, la, lb) ucls = {offset into ulist, count}; ulist = entry offsets within a potential's block
    const int64_t *u_off;
    int64_t n_used;
    const int2 *ucls;
    const uint16_t *ulist;
    // screening split: runs of at least kScrUnitMin entries go to radial_screen_unit_kernel
    // (scr_units), the others to the flat kernel through su, with prefix entry offsets su_off
    // (su_off null: the flat kernel covers every used entry of every item through u_off);
    // scr_lw: orders 0..scr_lw-1 of the unit kernel's Bessel tables
    const ScrUnit *scr_units;
    int n_scr_units, scr_lw;
    const ScrUnit *su;
    const int64_t *su_off;
    int n_su;
    int64_t n_su_entries;
    double *Q;                  // table values (running sums during the walk)
    double *S_prev, *scr;       // per entry scratch, same indexing as Q
    uint8_t *eflag;             // per entry: kEntActive | kEntScrOk
    uint8_t *walk;              // per item: 1 if the grid walk has work
    int8_t *stop_level;         // per item: deepest level walked (learning labels), may be null
    const int8_t *pred_level;   // per item: predicted level (learned mode), may be null
    int *fallback_count;        // learned mode: items that needed more than predicted+1
    // learned mode: the walk pops items from this order (deepest predicted level first)
    const int *order;           // may be null: static round-robin over all items
    const int *n_order;
    int *queue;
    int *status;
    // operation counters (accumulated per CTA, one atomic add per item), see kRadCnt*
    unsigned long long *counters;
};

// counter slots: the FLOP model of the radial path is built from these counts
enum RadialCounter {
    kRadCntScreenCycles = 0,   // SM clock cycles spent in screening (sum over CTAs)
    kRadCntQuadCycles,         // SM clock cycles spent in the grid walk
    kRadCntItems,              // tasks through the grid walk
    kRadCntPoints,             // integrand points evaluated
    kRadCntBessel,             // M_l(x) evaluations of the integrand (points x prims x orders)
    kRadCntPrimPts,            // primitive Gaussians evaluated (points x prims)
    kRadCntTermPts,            // potential terms evaluated (points x terms)
    kRadCntPowPts,             // r^N evaluations (points x (la+lb+1))
    kRadCntAccum,              // entry x point accumulations
    kRadCntScrCombos,          // primitive screening estimates started
    kRadCntScrIters,           // fixed-point iterations of the screening
    kRadCntScrFinal,           // screening envelopes evaluated
    kRadCntLevels,             // grid levels walked (sum over tasks)
    kRadCntMmdTriples,         // type 1 / overlap primitive triples evaluated (mmd_kernel)
    kRadCntMmdFlops,           // their FP64 operations by the model of mmd_kernel's counting
    kRadCntNum
};

struct RadialShared {
    double CA, CB;
    int la, lb, np_a, np_b, npot, nterm_tot, d_n;
    int l1max_all, l2max_all;
    int one_centre;
    int grpp;
    int64_t fa_off, fb_off;  // F tables of (A, C) and (B, C), when tabulated
    int n_entries;
    int any_active;
    double ca[kRadMaxPrims], xa[kRadMaxPrims], ka[kRadMaxPrims];
    double cb[kRadMaxPrims], xb[kRadMaxPrims], kb[kRadMaxPrims];
    int pL[kRadMaxPots], pn[kRadMaxPots], poff[kRadMaxPots], pent[kRadMaxPots + 1];
    int tpow[kRadMaxTerms];
    double tcoef[kRadMaxTerms], talpha[kRadMaxTerms];
};

// ---- screening (screening.c:243-362) ------------------------------------------

// M_a(x) / M_b(x) for the adjacent orders (a, b) = (1, 0) if l = 0, else (l-1, l), both
// from one table row (screening.c:332-346 evaluates them as two separate calls)
__device__ __noinline__ double scr_ratio(int l, double x)
{
    const int na = l == 0 ? 1 : l - 1, nb = l == 0 ? 0 : l;
    if (x <= 1e-7) return bessel_small(na, x) / bessel_small(nb, x);
    if (x <= 16.0) {
        const int i0 = (int)(round(x * 100) + 1e-5);
        const double dx = x - i0 * 0.01;
        const double *row = c_tab.bessel + (size_t)i0 * kBesL * 5;
        return taylor4(row + 5 * na, dx) / taylor4(row + 5 * nb, dx);
    }
    return bessel_asym(na, x) / bessel_asym(nb, x);
}

__device__ __noinline__ double bessel_scaled_nl(int n, double x) { return bessel_scaled(n, x); }

// returns true on failure; *val is the primitive estimate
__device__ inline bool scr_prim(int l1, int l2, int n, double CA2, double CB2, double aA, double aB, double k1,
                                double k2, double eta, double *val, int *iters)
{
    *val = 0.0;
    *iters = 0;
    if (l1 >= 1 && fabs(k1) <= kZeroThresh) return false;
    if (l2 >= 1 && fabs(k2) <= kZeroThresh) return false;
    const double p = aA + aB + eta, CA = sqrt(CA2), CB = sqrt(CB2);
    if (l1 == 0 && l2 == 0 && fabs(k1) <= kZeroThresh && fabs(k2) <= kZeroThresh) {
        double gi;
        if (n % 2 == 0) {
            int k = n / 2;
            gi = dfact(2 * k - 1) / (pow(2.0, k + 1) * pow(p, k)) * sqrt(kPi / p);
        } else {
            int k = (n - 1) / 2;
            double f = 1.0;
            for (int q = 2; q <= k; q++) f *= q;
            gi = f / (2.0 * pow(p, k + 1));
        }
        *val = exp(-aA * CA * CA - aB * CB * CB) * gi;
        return false;
    }
    double r0 = (aA * CA + aB * CB) / p, r0p;
    int steps = 0;
    do {
        steps++;
        if (steps == 5) {
            *val = 0.0;
            return true;
        }
        r0p = r0;
        const double x1 = k1 * r0, x2 = k2 * r0;
        double a = scr_ratio(l1, x1) * x1 + scr_ratio(l2, x2) * x2 + n;
        if (l1 > 0) a = a - l1 - 1;
        if (l2 > 0) a = a - l2 - 1;
        r0 = sqrt(a / (2.0 * p));
        *iters = steps;
    } while (fabs(r0 - r0p) > 1e-2);
    *val = sqrt(kPi / p) * pow(r0, n) * bessel_scaled_nl(l1, k1 * r0) * bessel_scaled_nl(l2, k2 * r0) *
           exp(-eta * r0 * r0 - aA * (r0 - CA) * (r0 - CA) - aB * (r0 - CB) * (r0 - CB)) * 0.5 * (1 + erf(sqrt(p) * r0));
    *iters = -*iters - 1;  // negative: the envelope was evaluated
    return false;
}

// x^n for a small non-negative integer n by binary powering (libgrpp calls pow(r0, n);
// the estimate only feeds threshold tests, and the two agree to a few ulps)
__device__ __forceinline__ double ipow(double x, int n)
{
    double r = 1.0, b = x;
    while (n) {
        if (n & 1) r *= b;
        b *= b;
        n >>= 1;
    }
    return r;
}

// M_a(x) and M_b(x) with (a, b) = (1, 0) if l = 0, else (l-1, l) (screening.c:329-346), up to
// a common factor: the numerator and denominator of the ratio the fixed-point step uses.
// Above x = 16 both are the asymptotic series sum_k c_k (-1/x)^k / (2x); the 1/(2x) factor
// cancels in the ratio and is left out, so one reciprocal of x serves both.
__device__ __forceinline__ void scr_ratio_parts(int l, double x, double &num, double &den)
{
    const int na = l == 0 ? 1 : l - 1, nb = l == 0 ? 0 : l;
    if (x <= 1e-7) {
        num = bessel_small(na, x);
        den = bessel_small(nb, x);
    } else if (x <= 16.0) {
        const int i0 = (int)(round(x * 100) + 1e-5);
        const double dx = x - i0 * 0.01;
        const double *row = c_tab.bessel + (size_t)i0 * kBesL * 5;
        num = taylor4(row + 5 * na, dx);
        den = taylor4(row + 5 * nb, dx);
    } else {
        const double ninv = -1.0 / x;
        const double *ca = c_tab.rfun + na * kRfunL, *cb = c_tab.rfun + nb * kRfunL;
        double pw = 1.0, sa = 0.0, sb = 0.0;
        const int kmax = na > nb ? na : nb;
        for (int k = 0; k <= kmax; k++) {
            if (k <= na) sa += __ldg(ca + k) * pw;
            if (k <= nb) sb += __ldg(cb + k) * pw;
            pw *= ninv;
        }
        num = sa;
        den = sb;
    }
}

// M_l(x) with one reciprocal of x in the asymptotic range (bessel_scaled divides twice there)
__device__ __forceinline__ double bessel_scaled_1r(int n, double x)
{
    if (x <= 16.0) return bessel_scaled(n, x);
    const double inv = 1.0 / x, ninv = -inv;
    const double *c = c_tab.rfun + n * kRfunL;
    double pw = 1.0, sum = 0.0;
    for (int k = 0; k <= n; k++) {
        sum += __ldg(c + k) * pw;
        pw *= ninv;
    }
    return sum * (0.5 * inv);
}

// Gaussian integral int_0^inf r^n exp(-p r^2) dr (screening.c:255-265): the
// screening estimate of two s functions on the centre and the one-centre analytic table
__device__ __forceinline__ double scr_gaussian_integral(int n, double p)
{
    if (n % 2 == 0) {
        const int k = n / 2;
        return dfact(2 * k - 1) / (pow(2.0, k + 1) * pow(p, k)) * sqrt(kPi / p);
    }
    const int k = (n - 1) / 2;
    double f = 1.0;
    for (int q = 2; q <= k; q++) f *= q;
    return f / (2.0 * pow(p, k + 1));
}

// The envelope of screening.c:308-318 at the fixed point r0, with sqpi = sqrt(pi / p) and
// sqp = sqrt(p). Every factor is finite and non-negative: a Gaussian factor that underflowed to
// exactly 0 makes the product exactly 0, so the other factors are not needed; and 1 + erf(z) is
// exactly 2 once erfc(z) < 2^-54 (z > 5.9), taken here as p r0^2 > 49 (z > 7). The product keeps
// libgrpp's order (screening.c:333-338).
__device__ __forceinline__ double scr_envelope(int l1, int l2, int n, double CA, double CB, double aA, double aB,
                                               double eta, double p, double k1, double k2, double r0, double sqpi,
                                               double sqp)
{
    const double e1 = r0 - CA, e2 = r0 - CB;
    const double ex = exp(-eta * r0 * r0 - aA * e1 * e1 - aB * e2 * e2);
    if (ex == 0.0) return 0.0;
    const double z2 = p * r0 * r0;
    const double erf_part = z2 > 49.0 ? 2.0 : 1 + erf(sqp * r0);
    return sqpi * ipow(r0, n) * bessel_scaled_1r(l1, k1 * r0) * bessel_scaled_1r(l2, k2 * r0) * ex * 0.5 * erf_part;
}

// The fixed-point update of screening.c:329-362 from the Bessel ratio parts (n1/d1 = M_a/M_b of
// side A at x1, n2/d2 of side B at x2): r0' = sqrt(s / (2p)),
// s = M_a1/M_b1 x1 + M_a2/M_b2 x2 + n - (l1 + 1 if l1 > 0) - (l2 + 1 if l2 > 0),
// the two ratios over one common denominator
__device__ __forceinline__ double scr_update(int l1, int l2, int n, double n1, double d1, double n2, double d2,
                                             double x1, double x2, double inv2p)
{
    double s = (n1 * x1 * d2 + n2 * x2 * d1) / (d1 * d2) + n;
    if (l1 > 0) s = s - l1 - 1;
    if (l2 > 0) s = s - l2 - 1;
    return sqrt(s * inv2p);
}

// One fixed-point step from r0
__device__ __forceinline__ double scr_step(int l1, int l2, int n, double k1, double k2, double inv2p, double r0)
{
    const double x1 = k1 * r0, x2 = k2 * r0;
    double n1, d1, n2, d2;
    scr_ratio_parts(l1, x1, n1, d1);
    scr_ratio_parts(l2, x2, n2, d2);
    return scr_update(l1, l2, n, n1, d1, n2, d2, x1, x2, inv2p);
}

// Primitive screening estimate (screening.c:243-318) with CA, CB as distances.
// Returns true on failure (no fixed point in 4 steps). *iters: steps taken, negative
// (-(steps)-1) when the envelope was evaluated.
__device__ __forceinline__ bool scr_prim_flat(int l1, int l2, int n, double CA, double CB, double aA, double aB,
                                              double k1, double k2, double eta, double *val, int *iters)
{
    *val = 0.0;
    *iters = 0;
    if (l1 >= 1 && fabs(k1) <= kZeroThresh) return false;
    if (l2 >= 1 && fabs(k2) <= kZeroThresh) return false;
    const double p = aA + aB + eta;
    if (l1 == 0 && l2 == 0 && fabs(k1) <= kZeroThresh && fabs(k2) <= kZeroThresh) {
        *val = exp(-aA * CA * CA - aB * CB * CB) * scr_gaussian_integral(n, p);
        return false;
    }
    // one reciprocal of p serves the start point, the fixed-point step and the envelope
    // (libgrpp divides by p three times; the estimate only feeds threshold tests)
    const double inv_p = 1.0 / p, inv2p = 0.5 * inv_p;
    double r0 = (aA * CA + aB * CB) * inv_p, r0p;
    int steps = 0;
    do {
        steps++;
        if (steps == 5) {
            *iters = steps - 1;
            return true;
        }
        r0p = r0;
        r0 = scr_step(l1, l2, n, k1, k2, inv2p, r0);
    } while (fabs(r0 - r0p) > 1e-2);
    *iters = -steps - 1;
    *val = scr_envelope(l1, l2, n, CA, CB, aA, aB, eta, p, k1, k2, r0, sqrt(kPi * inv_p), sqrt(p));
    return false;
}

// One-centre entry (CA = CB = 0): libgrpp's analytic table (radial_type2_integral.c:126-155),
// only l1 = l2 = 0 non-zero
__device__ double scr_one_centre_entry(const RadialArgs &a, int sa, int sb, int la, int lb, int l1, int l2, int N,
                                       int nk, int po)
{
    if (l1 != 0 || l2 != 0) return 0.0;
    const int na = __ldg(a.shell_nprim + sa), nb = __ldg(a.shell_nprim + sb);
    const double *pca = a.prim_coef + __ldg(a.shell_prim_off + sa), *pxa = a.prim_alpha + __ldg(a.shell_prim_off + sa);
    const double *pcb = a.prim_coef + __ldg(a.shell_prim_off + sb), *pxb = a.prim_alpha + __ldg(a.shell_prim_off + sb);
    double v = 0.0;
    for (int i = 0; i < na; i++) {
        const double ci = __ldg(pca + i) * gaussian_norm(la, __ldg(pxa + i));
        for (int j = 0; j < nb; j++) {
            const double cj = __ldg(pcb + j) * gaussian_norm(lb, __ldg(pxb + j));
            for (int k = 0; k < nk; k++) {
                const double pp = __ldg(pxa + i) + __ldg(pxb + j) + __ldg(a.pot_alpha + po + k);
                const double f = ci * cj * __ldg(a.pot_coef + po + k);
                v += f * scr_gaussian_integral(__ldg(a.pot_powers + po + k) + N, pp);
            }
        }
    }
    return v;
}

// libgrpp's decision for a screened entry (radial_type2_integral.c:264-279): an estimate below
// 1e-16 is the entry's value; otherwise the entry is walked, with forced refinement only when
// the estimate is valid
__device__ __forceinline__ void scr_store(const RadialArgs &a, int item, int64_t g, double sum, bool fail)
{
    a.scr[g] = sum;
    if (!fail && fabs(sum) < 1e-16) {
        a.Q[g] = sum;
        a.eflag[g] = kEntScrOk;
    } else {
        a.Q[g] = 0.0;
        a.eflag[g] = kEntActive | (fail ? 0 : kEntScrOk);
        a.walk[item] = 1;
    }
}

#ifndef GRPP_RADIAL_TABLES_ONLY
// Screening of (task, entry) pairs, one thread per entry over a flattened entry space (entries
// of one task are consecutive, tasks in item order): no per-task barrier and no ragged last
// round. With a.su_off the space is the short runs of a.su (the long ones go to
// radial_screen_unit_kernel); without it, every used entry of every item. A thread follows
// screening.c:193-220 for its entry: primitive triples (i, j, k) in libgrpp's order, stopping at
// the first failure. The outcome per entry is written to Q (value if screened out), scr
// (estimate) and eflag; walk[item] is set to 1 when any entry of the item needs the grid (walk[]
// is zeroed by the host before the launch). One-centre tasks get their analytic table.
__global__ void __launch_bounds__(kRadThreads, GRPP_SCR_MINB) radial_screen_flat_kernel(RadialArgs a)
{
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const long long t0 = clock64();
    unsigned long long c_combo = 0, c_iter = 0, c_final = 0;
    const int64_t n_flat = a.su_off ? a.n_su_entries : a.n_used;
    for (int64_t gu = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gu < n_flat; gu += stride) {
        int item, pot, e;
        int64_t pe = 0;
        if (a.su_off) {
            int lo = 0, hi = a.n_su - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (__ldg(a.su_off + mid) <= gu) lo = mid;
                else hi = mid - 1;
            }
            const ScrUnit &U = a.su[lo];
            item = U.item;
            pot = U.pot;
            pe = U.pe;
            e = a.ulist[U.uo + (int)(gu - __ldg(a.su_off + lo))];
        } else {
            int lo = 0, hi = a.n_items - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (__ldg(a.u_off + mid) <= gu) lo = mid;
                else hi = mid - 1;
            }
            item = lo;
            int ku = (int)(gu - __ldg(a.u_off + item));
            const int t = __ldg(a.item_task + item);
            const int sa = __ldg(a.task_a + t), sb = __ldg(a.task_b + t), c = __ldg(a.task_c + t);
            const int la = __ldg(a.shell_L + sa), lb = __ldg(a.shell_L + sb), dn = la + lb + 1;
            const int gr = __ldg(a.centre_grpp + c), npot = __ldg(a.grpp_sl_n + gr), slo = __ldg(a.grpp_sl_off + gr);
            // libgrpp tabulates the whole (l1, l2, N) box of every potential, but its angular sums
            // read only the entries with N = n1 + n2 (n1 <= la, n2 <= lb), l1 in [max(L-n1,0), L+n1]
            // of the parity of L+n1, l2 likewise (type2_integrals.c:169-184,
            // spin_orbit_integrals.c:189-204). Only those are screened and walked: the others cannot
            // change an output, and every entry's walk and stop level are its own
            // (radial_type2_integral.c:242-318). The host lists them per class (L, la, lb).
            pot = -1;
            e = 0;
            for (int p = 0; p < npot; p++) {
                pot = __ldg(a.sl_pot + slo + p);
                const int Lp = __ldg(a.pot_L + pot);
                const int2 cls = a.ucls[(Lp * (kMaxL + 1) + la) * (kMaxL + 1) + lb];
                if (ku < cls.y) {
                    e = a.ulist[cls.x + ku];
                    break;
                }
                ku -= cls.y;
                pe += (Lp + la + 1) * (Lp + lb + 1) * dn;
            }
        }
        const int t = __ldg(a.item_task + item);
        const int sa = __ldg(a.task_a + t), sb = __ldg(a.task_b + t), c = __ldg(a.task_c + t);
        const double *Ao = a.shell_origin + 3 * sa, *Bo = a.shell_origin + 3 * sb, *Co = a.centre_origin + 3 * c;
        double CA2 = 0.0, CB2 = 0.0;
        for (int d = 0; d < 3; d++) {
            const double u = __ldg(Co + d) - __ldg(Ao + d), v = __ldg(Co + d) - __ldg(Bo + d);
            CA2 += u * u;
            CB2 += v * v;
        }
        const int la = __ldg(a.shell_L + sa), lb = __ldg(a.shell_L + sb), dn = la + lb + 1;
        const int Lp = __ldg(a.pot_L + pot);
        const int64_t g = __ldg(a.q_off + item) + pe + e;
        const int d2 = Lp + lb + 1;
        const int l1 = e / (d2 * dn), rem = e - l1 * d2 * dn, l2 = rem / dn, N = rem - l2 * dn;
        const int nk = __ldg(a.pot_nprim + pot), po = __ldg(a.pot_prim_off + pot);
        if (CA2 < 1e-14 && CB2 < 1e-14) {
            a.Q[g] = scr_one_centre_entry(a, sa, sb, la, lb, l1, l2, N, nk, po);
            a.eflag[g] = 0;
            continue;
        }
        const double CA = sqrt(CA2), CB = sqrt(CB2);
        const int na = __ldg(a.rp_n + sa), nb = __ldg(a.rp_n + sb);
        const double *ca = a.rp_coef + __ldg(a.rp_off + sa), *xa = a.rp_alpha + __ldg(a.rp_off + sa);
        const double *cb = a.rp_coef + __ldg(a.rp_off + sb), *xb = a.rp_alpha + __ldg(a.rp_off + sb);
        // screening.c:193-220: triples in (bra, ket, potential term) order, stop at the first failure
        double sum = 0.0;
        bool fail = false;
        for (int i = 0; i < na && !fail; i++) {
            const double aA = __ldg(xa + i), ci = __ldg(ca + i), k1 = 2 * aA * CA;
            for (int j = 0; j < nb && !fail; j++) {
                const double aB = __ldg(xb + j), cij = ci * __ldg(cb + j), k2 = 2 * aB * CB;
                for (int k = 0; k < nk; k++) {
                    double v;
                    int it;
                    const bool f = scr_prim_flat(l1, l2, N + __ldg(a.pot_powers + po + k), CA, CB, aA, aB, k1, k2,
                                                 __ldg(a.pot_alpha + po + k), &v, &it);
                    c_combo++;
                    if (it < 0) {
                        c_final++;
                        it = -it - 1;
                    }
                    c_iter += it;
                    if (f) {
                        fail = true;
                        break;
                    }
                    sum += cij * __ldg(a.pot_coef + po + k) * v;
                }
            }
        }
        scr_store(a, item, g, sum, fail);
    }
    if (a.counters) {
        unsigned long long v[3] = {c_combo, c_iter, c_final};
        for (int k = 0; k < 3; k++)
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
        if (lane == 0) {
            atomicAdd(a.counters + kRadCntScrCombos, v[0]);
            atomicAdd(a.counters + kRadCntScrIters, v[1]);
            atomicAdd(a.counters + kRadCntScrFinal, v[2]);
            atomicAdd(a.counters + kRadCntScreenCycles, (unsigned long long)(clock64() - t0));
        }
    }
}

// ---- screening of long runs: radial_screen_unit_kernel ----------------------------------------
//
// A block screens one run of entries of one (task, semilocal potential) (ScrUnit), a thread per
// entry. Everything of a primitive triple (i, j, k) that does not depend on the entry
// (l1, l2, N) is formed once per block, a triple per thread, kScrChunk triples at a time, into
// shared memory: p = a_A + a_B + eta, 1/p, sqrt(pi/p), sqrt(p), k = 2 a C, the fixed point's start
// r0 = (a_A CA + a_B CB)/p and its arguments x = k r0, and the Bessel parts of the first step for
// every order 0..lw-1 of both sides (the first step's arguments do not depend on the entry).
// Every entry then runs libgrpp's per-triple estimate (screening.c:193-220, 243-362) over the
// staged triples in libgrpp's order, reading its first step from the tables: the same
// expressions, operands and order as the flat kernel, so the estimates and gate decisions are
// the same.
constexpr int kScrUnitThreads = 64;  // threads per block = entries per run at most
constexpr int kScrUnitMin = 32;      // runs with fewer entries stay in the flat kernel
constexpr int kScrChunk = 64;        // primitive triples staged per round (one per thread)
static_assert(kScrChunk == kScrUnitThreads, "one staged triple per thread");

// Bessel parts of orders 0..n-1 at x, as scr_ratio_parts forms them: the value (x <= 16) or, above
// x = 16, the asymptotic sum without its 1/(2x) factor (it cancels in the ratio of two orders)
__device__ __forceinline__ void scr_parts_row(int n, double x, double *out)
{
    if (x <= 1e-7) {
        for (int l = 0; l < n; l++) out[l] = bessel_small(l, x);
    } else if (x <= 16.0) {
        const int i0 = (int)(round(x * 100) + 1e-5);
        const double dx = x - i0 * 0.01;
        const double *row = c_tab.bessel + (size_t)i0 * kBesL * 5;
        for (int l = 0; l < n; l++) out[l] = taylor4(row + 5 * l, dx);
    } else {
        const double ninv = -1.0 / x;
        for (int l = 0; l < n; l++) {
            const double *cl = c_tab.rfun + l * kRfunL;
            double pw = 1.0, sum = 0.0;
            for (int k = 0; k <= l; k++) {
                sum += __ldg(cl + k) * pw;
                pw *= ninv;
            }
            out[l] = sum;
        }
    }
}

__global__ void __launch_bounds__(kScrUnitThreads, 10) radial_screen_unit_kernel(RadialArgs a)
{
    extern __shared__ double ptab[];  // [kScrChunk][2][scr_lw]: Bessel parts, sides A and B
    __shared__ double t_aA[kScrChunk], t_aB[kScrChunk], t_eta[kScrChunk], t_p[kScrChunk], t_ip[kScrChunk],
        t_sqpi[kScrChunk], t_sqp[kScrChunk], t_k1[kScrChunk], t_k2[kScrChunk], t_r0[kScrChunk], t_x1[kScrChunk],
        t_x2[kScrChunk], t_c[kScrChunk];
    __shared__ int t_pw[kScrChunk];
    const int tid = threadIdx.x, lane = tid & 31, lw = a.scr_lw;
    const long long t0 = clock64();
    unsigned long long c_combo = 0, c_iter = 0, c_final = 0;
    for (int u = blockIdx.x; u < a.n_scr_units; u += gridDim.x) {
        const int item = a.scr_units[u].item, pot = a.scr_units[u].pot, ne = a.scr_units[u].ne;
        const int t = __ldg(a.item_task + item);
        const int sa = __ldg(a.task_a + t), sb = __ldg(a.task_b + t), c = __ldg(a.task_c + t);
        const double *Ao = a.shell_origin + 3 * sa, *Bo = a.shell_origin + 3 * sb, *Co = a.centre_origin + 3 * c;
        double CA2 = 0.0, CB2 = 0.0;
        for (int d = 0; d < 3; d++) {
            const double uu = __ldg(Co + d) - __ldg(Ao + d), vv = __ldg(Co + d) - __ldg(Bo + d);
            CA2 += uu * uu;
            CB2 += vv * vv;
        }
        const int la = __ldg(a.shell_L + sa), lb = __ldg(a.shell_L + sb), dn = la + lb + 1;
        const int Lp = __ldg(a.pot_L + pot), d2 = Lp + lb + 1;
        const int nk = __ldg(a.pot_nprim + pot), po = __ldg(a.pot_prim_off + pot);
        const bool have = tid < ne;
        int l1 = 0, l2 = 0, N = 0;
        int64_t g = 0;
        if (have) {
            const int e = a.ulist[a.scr_units[u].uo + tid];
            g = __ldg(a.q_off + item) + a.scr_units[u].pe + e;
            l1 = e / (d2 * dn);
            const int rem = e - l1 * d2 * dn;
            l2 = rem / dn;
            N = rem - l2 * dn;
        }
        if (CA2 < 1e-14 && CB2 < 1e-14) {  // one-centre tasks are the flat kernel's; kept for safety
            if (have) {
                a.Q[g] = scr_one_centre_entry(a, sa, sb, la, lb, l1, l2, N, nk, po);
                a.eflag[g] = 0;
            }
            continue;
        }
        const double CA = sqrt(CA2), CB = sqrt(CB2);
        const int na = __ldg(a.rp_n + sa), nb = __ldg(a.rp_n + sb);
        const double *ca = a.rp_coef + __ldg(a.rp_off + sa), *xa = a.rp_alpha + __ldg(a.rp_off + sa);
        const double *cb = a.rp_coef + __ldg(a.rp_off + sb), *xb = a.rp_alpha + __ldg(a.rp_off + sb);
        // orders of the first step's ratios (screening.c:329-346): (1, 0) for l = 0, else (l-1, l)
        const int oa1 = l1 == 0 ? 1 : l1 - 1, ob1 = l1 == 0 ? 0 : l1, oa2 = l2 == 0 ? 1 : l2 - 1, ob2 = l2 == 0 ? 0 : l2;
        const int nA = max(2, Lp + la + 1), nB = max(2, Lp + lb + 1);  // orders the run's entries can use
        double sum = 0.0;
        bool fail = !have;
        const int T = na * nb * nk;
        for (int c0 = 0; c0 < T; c0 += kScrChunk) {
            const int nc = min(kScrChunk, T - c0);
            __syncthreads();  // the previous round's tables are consumed
            if (tid < nc) {
                const int q = c0 + tid, i = q / (nb * nk), j = (q / nk) % nb, k = q % nk;
                const double aA = __ldg(xa + i), aB = __ldg(xb + j), eta = __ldg(a.pot_alpha + po + k);
                const double k1 = 2 * aA * CA, k2 = 2 * aB * CB;
                const double p = aA + aB + eta, inv_p = 1.0 / p;
                const double r0 = (aA * CA + aB * CB) * inv_p;
                const double cij = __ldg(ca + i) * __ldg(cb + j);
                t_aA[tid] = aA;
                t_aB[tid] = aB;
                t_eta[tid] = eta;
                t_p[tid] = p;
                t_ip[tid] = inv_p;
                t_sqpi[tid] = sqrt(kPi * inv_p);
                t_sqp[tid] = sqrt(p);
                t_k1[tid] = k1;
                t_k2[tid] = k2;
                t_r0[tid] = r0;
                t_x1[tid] = k1 * r0;
                t_x2[tid] = k2 * r0;
                t_c[tid] = cij * __ldg(a.pot_coef + po + k);
                t_pw[tid] = __ldg(a.pot_powers + po + k);
                scr_parts_row(nA, k1 * r0, ptab + (size_t)(2 * tid) * lw);
                scr_parts_row(nB, k2 * r0, ptab + (size_t)(2 * tid + 1) * lw);
            }
            __syncthreads();
            if (fail) continue;
            for (int q = 0; q < nc; q++) {
                const double k1 = t_k1[q], k2 = t_k2[q];
                double v = 0.0;
                int it = 0;
                bool f = false;
                if (!(l1 >= 1 && fabs(k1) <= kZeroThresh) && !(l2 >= 1 && fabs(k2) <= kZeroThresh)) {
                    const int n = N + t_pw[q];
                    const double p = t_p[q];
                    if (l1 == 0 && l2 == 0 && fabs(k1) <= kZeroThresh && fabs(k2) <= kZeroThresh) {
                        v = exp(-t_aA[q] * CA * CA - t_aB[q] * CB * CB) * scr_gaussian_integral(n, p);
                    } else {
                        const double inv2p = 0.5 * t_ip[q];
                        const double *PA = ptab + (size_t)(2 * q) * lw, *PB = PA + lw;
                        double r0p = t_r0[q];
                        double r0 = scr_update(l1, l2, n, PA[oa1], PA[ob1], PB[oa2], PB[ob2], t_x1[q], t_x2[q], inv2p);
                        int steps = 1;
                        while (fabs(r0 - r0p) > 1e-2) {
                            steps++;
                            if (steps == 5) {
                                f = true;
                                break;
                            }
                            r0p = r0;
                            r0 = scr_step(l1, l2, n, k1, k2, inv2p, r0);
                        }
                        if (f) {
                            it = steps - 1;
                        } else {
                            it = steps;
                            c_final++;
                            v = scr_envelope(l1, l2, n, CA, CB, t_aA[q], t_aB[q], t_eta[q], p, k1, k2, r0, t_sqpi[q],
                                             t_sqp[q]);
                        }
                    }
                }
                c_combo++;
                c_iter += it;
                if (f) {
                    fail = true;
                    break;
                }
                sum += t_c[q] * v;
            }
        }
        if (have) scr_store(a, item, g, sum, fail);
    }
    if (a.counters) {
        unsigned long long v[3] = {c_combo, c_iter, c_final};
        for (int k = 0; k < 3; k++)
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
        if (lane == 0) {
            atomicAdd(a.counters + kRadCntScrCombos, v[0]);
            atomicAdd(a.counters + kRadCntScrIters, v[1]);
            atomicAdd(a.counters + kRadCntScrFinal, v[2]);
            atomicAdd(a.counters + kRadCntScreenCycles, (unsigned long long)(clock64() - t0));
        }
    }
}

#endif  // GRPP_RADIAL_TABLES_ONLY

// decode entry index within an item -> (potential, l1, l2, N)
__device__ __forceinline__ void decode_entry(const RadialShared &sh, int e, int &p, int &l1, int &l2, int &N)
{
    p = 0;
    while (e >= sh.pent[p + 1]) p++;
    int r = e - sh.pent[p];
    const int d2 = sh.pL[p] + sh.lb + 1, dn = sh.d_n;
    l1 = r / (d2 * dn);
    r -= l1 * d2 * dn;
    l2 = r / dn;
    N = r - l2 * dn;
}

// Log3 point i of a grid of nr points (radial_type2_integral.c:357-365)
__device__ __forceinline__ void log3_point(int i, int nr, double &r, double &w)
{
    const double R = 5.0, R3 = R * R * R;
    const double xi = i / (nr + 1.0), xi3 = xi * xi * xi, ln = log(1 - xi3);
    w = 3 * R3 * xi * xi * ln * ln / ((1 - xi3) * (nr + 1.0));
    r = -R * ln;
}

// r and w of walk-order point f (point i of the level's nr-point grid): libgrpp's values from
// the host-built grid table (grpp_common.cuh) when present, else computed here
__device__ __forceinline__ void grid_point(int f, int i, int nr, double &r, double &w)
{
    if (c_tab.grid) {
        r = __ldg(c_tab.grid + (size_t)kGridRowR * kGridPts + f);
        w = __ldg(c_tab.grid + (size_t)kGridRowW * kGridPts + f);
    } else {
        log3_point(i, nr, r, w);
    }
}

// r^(n-2) of a potential term (n = 0, 1, 2) at walk-order point f: pow(r, n-2) from the grid
// table when present (potential.c:70-81), else 1/r^2, 1/r from the given reciprocals
__device__ __forceinline__ double grid_rpow_m2(int f, int pw, double ir, double ir2)
{
    if (pw == 2) return 1.0;
    if (c_tab.grid) return __ldg(c_tab.grid + (size_t)(pw == 1 ? kGridRowRinv : kGridRowRinv2) * kGridPts + f);
    return pw == 1 ? ir : ir2;
}


// task geometry, primitives and potential terms into shared memory
__device__ void load_task(const RadialArgs &a, int item, RadialShared &sh, int tid, int nthr)
{
    const int t = a.item_task[item];
    const int sa = a.task_a[t], sb = a.task_b[t], c = a.task_c[t];
    if (tid == 0) {
        const double *Ao = a.shell_origin + 3 * sa, *Bo = a.shell_origin + 3 * sb, *Co = a.centre_origin + 3 * c;
        double CAv[3], CBv[3];
        for (int d = 0; d < 3; d++) {
            CAv[d] = Co[d] - Ao[d];
            CBv[d] = Co[d] - Bo[d];
        }
        const double CA2 = CAv[0] * CAv[0] + CAv[1] * CAv[1] + CAv[2] * CAv[2];
        const double CB2 = CBv[0] * CBv[0] + CBv[1] * CBv[1] + CBv[2] * CBv[2];
        sh.one_centre = CA2 < 1e-14 && CB2 < 1e-14;
        sh.CA = sqrt(CA2);
        sh.CB = sqrt(CB2);
        sh.la = a.shell_L[sa];
        sh.lb = a.shell_L[sb];
        sh.d_n = sh.la + sh.lb + 1;
        const int g = a.centre_grpp[c];
        sh.grpp = g;
        sh.npot = a.grpp_sl_n[g];
        int e = 0, nt = 0, l1m = 0, l2m = 0;
        for (int p = 0; p < sh.npot; p++) {
            const int pot = a.sl_pot[a.grpp_sl_off[g] + p];
            sh.pL[p] = a.pot_L[pot];
            sh.pn[p] = a.pot_nprim[pot];
            sh.poff[p] = nt;
            for (int k = 0; k < sh.pn[p]; k++) {
                const int o = a.pot_prim_off[pot] + k;
                sh.tpow[nt] = a.pot_powers[o];
                sh.tcoef[nt] = a.pot_coef[o];
                sh.talpha[nt] = a.pot_alpha[o];
                nt++;
            }
            sh.pent[p] = e;
            e += (sh.pL[p] + sh.la + 1) * (sh.pL[p] + sh.lb + 1) * sh.d_n;
            l1m = max(l1m, sh.pL[p] + sh.la);
            l2m = max(l2m, sh.pL[p] + sh.lb);
        }
        sh.pent[sh.npot] = e;
        sh.n_entries = e;
        sh.nterm_tot = nt;
        sh.l1max_all = l1m;
        sh.l2max_all = l2m;
        sh.np_a = a.rp_n[sa];
        sh.np_b = a.rp_n[sb];
        if (a.ftab) {
            sh.fa_off = a.fp_off[a.item_fa[item]];
            sh.fb_off = a.fp_off[a.item_fb[item]];
        }
    }
    __syncthreads();
    for (int i = tid; i < sh.np_a; i += nthr) {
        sh.ca[i] = a.rp_coef[a.rp_off[sa] + i];
        sh.xa[i] = a.rp_alpha[a.rp_off[sa] + i];
        sh.ka[i] = 2.0 * sh.xa[i] * sh.CA;
    }
    for (int i = tid; i < sh.np_b; i += nthr) {
        sh.cb[i] = a.rp_coef[a.rp_off[sb] + i];
        sh.xb[i] = a.rp_alpha[a.rp_off[sb] + i];
        sh.kb[i] = 2.0 * sh.xb[i] * sh.CB;
    }
    __syncthreads();
}

// analytic one-centre entry (radial_type2_integral.c:126-155): only l1 = l2 = 0 is non-zero
__device__ double one_centre_entry(const RadialArgs &a, const RadialShared &sh, int sa, int sb, int p, int l1, int l2, int N)
{
    double v = 0.0;
    if (l1 != 0 || l2 != 0) return 0.0;
    const int na = a.shell_nprim[sa], nb = a.shell_nprim[sb];
    const double *pca = a.prim_coef + a.shell_prim_off[sa], *pxa = a.prim_alpha + a.shell_prim_off[sa];
    const double *pcb = a.prim_coef + a.shell_prim_off[sb], *pxb = a.prim_alpha + a.shell_prim_off[sb];
    for (int i = 0; i < na; i++) {
        const double ci = pca[i] * gaussian_norm(sh.la, pxa[i]);
        for (int j = 0; j < nb; j++) {
            const double cj = pcb[j] * gaussian_norm(sh.lb, pxb[j]);
            for (int k = 0; k < sh.pn[p]; k++) {
                const int tk = sh.poff[p] + k;
                const double pp = pxa[i] + pxb[j] + sh.talpha[tk];
                const double f = ci * cj * sh.tcoef[tk];
                const int n = sh.tpow[tk] + N;
                double gi;
                if (n % 2 == 0) {
                    const int kk = n / 2;
                    gi = dfact(2 * kk - 1) / (pow(2.0, kk + 1) * pow(pp, kk)) * sqrt(kPi / pp);
                } else {
                    const int kk = (n - 1) / 2;
                    double fct = 1.0;
                    for (int q = 2; q <= kk; q++) fct *= q;
                    gi = fct / (2.0 * pow(pp, kk + 1));
                }
                v += f * gi;
            }
        }
    }
    return v;
}

#ifndef GRPP_RADIAL_TABLES_ONLY
__global__ void __launch_bounds__(kRadThreads) radial_screen_kernel(RadialArgs a)
{
    __shared__ RadialShared sh;
    const int tid = threadIdx.x, lane = tid & 31;
    for (int item = blockIdx.x; item < a.n_items; item += gridDim.x) {
        __syncthreads();
        load_task(a, item, sh, tid, kRadThreads);
        const int t = a.item_task[item];
        const int sa = a.task_a[t], sb = a.task_b[t];
        const int64_t qo = a.q_off[item];
        double *Q = a.Q + qo, *SC = a.scr + qo;
        uint8_t *EF = a.eflag + qo;
        const int nE = sh.n_entries, np_a = sh.np_a, np_b = sh.np_b;
        const long long t0 = clock64();
        unsigned long long c_combo = 0, c_iter = 0, c_final = 0;
        int active = 0;
        if (sh.one_centre) {
            for (int e = tid; e < nE; e += kRadThreads) {
                int p, l1, l2, N;
                decode_entry(sh, e, p, l1, l2, N);
                Q[e] = one_centre_entry(a, sh, sa, sb, p, l1, l2, N);
                EF[e] = 0;
            }
        } else {
            const double CA2 = sh.CA * sh.CA, CB2 = sh.CB * sh.CB;
            for (int e = tid; e < nE; e += kRadThreads) {
                int p, l1, l2, N;
                decode_entry(sh, e, p, l1, l2, N);
                // screening.c:193-220: triples in (bra, ket, potential term) order, stop at the first failure
                double sum = 0.0;
                bool fail = false;
                const int nk = sh.pn[p];
                for (int i = 0; i < np_a && !fail; i++)
                    for (int j = 0; j < np_b && !fail; j++)
                        for (int k = 0; k < nk; k++) {
                            const int tk = sh.poff[p] + k;
                            double v;
                            int it;
                            const bool f = scr_prim(l1, l2, N + sh.tpow[tk], CA2, CB2, sh.xa[i], sh.xb[j], sh.ka[i],
                                                    sh.kb[j], sh.talpha[tk], &v, &it);
                            c_combo++;
                            if (it < 0) {
                                c_final++;
                                it = -it - 1;
                            }
                            c_iter += it;
                            if (f) {
                                fail = true;
                                break;
                            }
                            sum += sh.ca[i] * sh.cb[j] * sh.tcoef[tk] * v;
                        }
                SC[e] = sum;
                if (!fail && fabs(sum) < 1e-16) {
                    Q[e] = sum;
                    EF[e] = kEntScrOk;
                } else {
                    Q[e] = 0.0;
                    EF[e] = kEntActive | (fail ? 0 : kEntScrOk);
                    active = 1;
                }
            }
        }
        const int any = __syncthreads_or(active);
        if (tid == 0) {
            a.walk[item] = (uint8_t)any;
            if (a.stop_level) a.stop_level[item] = 0;
        }
        if (a.counters) {
            unsigned long long v[3] = {c_combo, c_iter, c_final};
            for (int k = 0; k < 3; k++)
                for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
            if (lane == 0) {
                atomicAdd(a.counters + kRadCntScrCombos, v[0]);
                atomicAdd(a.counters + kRadCntScrIters, v[1]);
                atomicAdd(a.counters + kRadCntScrFinal, v[2]);
            }
            if (tid == 0) atomicAdd(a.counters + kRadCntScreenCycles, (unsigned long long)(clock64() - t0));
        }
    }
}
#endif  // GRPP_RADIAL_TABLES_ONLY

// dst[l * stride] += e * M_l(x) for l = 0..lmax, one table row (specfunc_scaled_mod_sph_bessel.c:72-122)
__device__ __forceinline__ void bessel_row_acc(int lmax, double x, double e, double *dst, int stride)
{
    if (x <= 1e-7) {
#pragma unroll 1
        for (int l = 0; l <= lmax; l++) dst[l * stride] += e * bessel_small(l, x);
    } else if (x <= 16.0) {
        const int i0 = (int)(round(x * 100) + 1e-5);
        const double dx = x - i0 * 0.01;
        const double dx2 = dx * dx, dx3 = dx2 * dx, dx4 = dx3 * dx;
        // orders l, l+1 from one 80-byte block of the pair layout: five 16-byte loads
        const double2 *d = reinterpret_cast<const double2 *>(c_tab.bessel_p) + (size_t)i0 * kBesL * 5 / 2;
#pragma unroll 1
        for (int l = 0; l <= lmax; l += 2) {
            const double2 *q = d + 5 * (l / 2);
            const double2 c0 = __ldg(q), c1 = __ldg(q + 1), c2 = __ldg(q + 2), c3 = __ldg(q + 3), c4 = __ldg(q + 4);
            const double m0 = c0.x + c1.x * dx + c2.x * dx2 * 0.5 + c3.x * dx3 * (1.0 / 6.0) + c4.x * dx4 * (1.0 / 24.0);
            dst[l * stride] += e * m0;
            if (l < lmax) {
                const double m1 = c0.y + c1.y * dx + c2.y * dx2 * 0.5 + c3.y * dx3 * (1.0 / 6.0) + c4.y * dx4 * (1.0 / 24.0);
                dst[(l + 1) * stride] += e * m1;
            }
        }
    } else {
#pragma unroll 1
        for (int l = 0; l <= lmax; l++) dst[l * stride] += e * bessel_asym(l, x);
    }
}

constexpr int kRadRow = kRadThreads + 1;  // padded row stride of the chunk arrays (no bank conflicts)
constexpr int kRadGridPts = kGridPts;     // points of levels 0..8 together

// Level of point f of the nested grid in walk order (level 0: f = 0..30; level L >= 1:
// f = 2^(L+4)-1 .. 2^(L+5)-2), and the point's index i on that level's grid of nr points.
__device__ __forceinline__ void walk_point(int f, int &level, int &i, int &nr)
{
    const int lg = 31 - __clz(f + 1);  // floor(log2(f + 1))
    level = lg > 4 ? lg - 4 : 0;
    if (level == 0) {
        i = f + 1;
        nr = 31;
    } else {
        i = 2 * (f - ((1 << (level + 4)) - 1)) + 1;
        nr = (1 << (level + 5)) - 1;
    }
}

// last walk-order point of level L
__device__ __forceinline__ int level_last_point(int L) { return (1 << (L + 5)) - 2; }

// The nested Log3 grid of every task with entries left, one CTA per task.
// Points are taken in walk order (level 0, then the new points of level 1, 2, ...)
// in chunks of kRadThreads. Per chunk, thread t evaluates point f0 + t once for all
// potentials and orders still needed (w U_p, F^A_l, F^B_l, r^N into shared memory);
// then every thread advances the entries it owns over the chunk's points, in the
// reference's order and association, applying libgrpp's per-level rules
// (radial_type2_integral.c:285-315) when an entry passes the last point of a level:
//   level 0: continue; forced refinement while |S|/|estimate| < 1e-3 (estimate valid);
//   converged when |S_L - S_{L-1}| <= 1e-16; otherwise S_prev = S_L, S = S_L / 2.
// An entry therefore ends with exactly the sum the level-by-level walk gives it.
// The walk of a task stops at the first chunk boundary after which no entry is active;
// points evaluated past that are never added. The orders, powers and potentials
// evaluated per point shrink with the set of active entries.
#ifndef GRPP_NO_RADIAL_TABLE_KERNELS
// F_l(r) of every (shell, centre) pair of the batch at every point of the nested grid, one
// CTA per pair and chunk of 128 points: the same point, distance CS (as load_task forms it),
// primitives, exact-zero skips and Bessel rows as the walk's own evaluation, so every order
// l holds the walk's value. Dynamic shared memory: (max fp_lmax + 1) x kRadRow doubles.
__global__ void __launch_bounds__(kRadThreads) ftab_kernel(RadialArgs a, double *ftab)
{
    extern __shared__ double cf[];
    const int tid = threadIdx.x;
    const int nchunk = (kRadGridPts + kRadThreads - 1) / kRadThreads;
    for (int64_t blk = blockIdx.x; blk < (int64_t)a.n_fpairs * nchunk; blk += gridDim.x) {
        const int pr = (int)(blk / nchunk), f = (int)(blk % nchunk) * kRadThreads + tid;
        if (f >= kRadGridPts) continue;
        const int s = a.fp_shell[pr], c = a.fp_centre[pr], lmax = a.fp_lmax[pr];
        const double *So = a.shell_origin + 3 * s, *Co = a.centre_origin + 3 * c;
        double CSv[3];
        for (int d = 0; d < 3; d++) CSv[d] = Co[d] - So[d];
        const double CS2 = CSv[0] * CSv[0] + CSv[1] * CSv[1] + CSv[2] * CSv[2];
        const double CS = sqrt(CS2);
        int lev, i, nr;
        walk_point(f, lev, i, nr);
        double r, w;
        grid_point(f, i, nr, r, w);
        for (int l = 0; l <= lmax; l++) cf[l * kRadRow + tid] = 0.0;
        const double d2 = (r - CS) * (r - CS);
        const int np = a.rp_n[s], off = a.rp_off[s];
#pragma unroll 1
        for (int q = 0; q < np; q++) {
            const double x = a.rp_alpha[off + q];
            const double e = a.rp_coef[off + q] * exp_rn(-x * d2);
            if (e != 0.0) bessel_row_acc(lmax, (2.0 * x * CS) * r, e, cf + tid, kRadRow);
        }
        double *dst = ftab + a.fp_off[pr] + f;
        for (int l = 0; l <= lmax; l++) dst[(int64_t)l * kRadGridPts] = cf[l * kRadRow + tid];
    }
}

// w U_p(r) = w sum_k c_k r^(n_k-2) exp(-zeta_k r^2) at every point of the nested grid, for
// every semilocal potential slot of every GRPP: the grid does not depend on the task, so
// the walk reads these values instead of evaluating the terms for each task. Same point,
// weight, terms, order and exact-zero skips as the walk's own evaluation.
__global__ void wu_table_kernel(RadialArgs a, int n_grpps, double *wu)
{
    const int64_t total = (int64_t)n_grpps * a.wu_npot * kRadGridPts;
    for (int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; id < total; id += (int64_t)gridDim.x * blockDim.x) {
        const int f = (int)(id % kRadGridPts);
        const int64_t gp = id / kRadGridPts;
        const int pp = (int)(gp % a.wu_npot), g = (int)(gp / a.wu_npot);
        if (pp >= a.grpp_sl_n[g]) {
            wu[id] = 0.0;
            continue;
        }
        const int pot = a.sl_pot[a.grpp_sl_off[g] + pp];
        int lev, i, nr;
        walk_point(f, lev, i, nr);
        double r, w;
        grid_point(f, i, nr, r, w);
        const double r2 = r * r, ir = 1.0 / r, ir2 = 1.0 / r2;
        double u = 0.0;
        for (int k = 0; k < a.pot_nprim[pot]; k++) {
            const int o = a.pot_prim_off[pot] + k;
            const double ex = exp_rn(-a.pot_alpha[o] * r2);
            if (ex == 0.0) continue;  // the term adds an exact zero
            const double rp = grid_rpow_m2(f, a.pot_powers[o], ir, ir2);  // r^(n-2)
            u += a.pot_coef[o] * rp * ex;
        }
        wu[id] = w * u;
    }
}
#endif  // GRPP_NO_RADIAL_TABLE_KERNELS

#ifndef GRPP_RADIAL_TABLES_ONLY
__global__ void __launch_bounds__(kRadThreads, 5) radial_walk_kernel(RadialArgs a)
{
    __shared__ RadialShared sh;
    __shared__ int s_need[2][4];  // per buffer: max l1, max l2, max N of active entries, potential mask
    __shared__ int s_lvl;         // deepest level at which an entry converged
    extern __shared__ double chunk[];  // [npot + l1max+1 + l2max+1 + dn][kRadRow]
    __shared__ int s_item;
    __shared__ int s_cnt[2];      // lengths of the two active-entry lists
    const int tid = threadIdx.x, lane = tid & 31;
    const bool use_list = a.list_max > 0;
    uint16_t *lists[2] = {reinterpret_cast<uint16_t *>(chunk + a.chunk_doubles),
                          reinterpret_cast<uint16_t *>(chunk + a.chunk_doubles) + a.list_max};
    int next_static = blockIdx.x;
    for (;;) {
        int item;
        if (a.order) {
            // work queue: one pop per CTA (every loop iteration below ends with a barrier)
            __syncthreads();
            if (tid == 0) {
                const int k = atomicAdd(a.queue, 1);
                s_item = k < *a.n_order ? a.order[k] : -1;
            }
            __syncthreads();
            item = s_item;
            if (item < 0) break;
        } else {
            item = next_static;
            next_static += gridDim.x;
            if (item >= a.n_items) break;
            if (!a.walk[item]) continue;
        }
        __syncthreads();
        if (tid < 8) s_need[tid >> 2][tid & 3] = tid == 3 || tid == 7 ? 0 : -1;
        if (tid == 0) {
            s_lvl = 0;
            s_cnt[0] = 0;
        }
        load_task(a, item, sh, tid, kRadThreads);
        const int64_t qo = a.q_off[item];
        double *Q = a.Q + qo, *Sp = a.S_prev + qo;
        const double *SC = a.scr + qo;
        uint8_t *EF = a.eflag + qo;
        const int nE = sh.n_entries, np_a = sh.np_a, np_b = sh.np_b;
        const int npot = sh.npot, l1m = sh.l1max_all, l2m = sh.l2max_all, dn = sh.d_n;
        double *cwu = chunk;                       // [npot][kRadRow]
        double *cf1 = cwu + npot * kRadRow;        // [l1m+1][kRadRow]
        double *cf2 = cf1 + (l1m + 1) * kRadRow;   // [l2m+1][kRadRow]
        double *crn = cf2 + (l2m + 1) * kRadRow;   // [dn][kRadRow]
        const long long t0 = clock64();
        unsigned long long c_acc = 0;
        // what the entries active after screening need from each point
        {
            int n1 = -1, n2 = -1, nN = -1, mask = 0;
            for (int e = tid; e < nE; e += kRadThreads)
                if (EF[e] & kEntActive) {
                    int p, l1, l2, N;
                    decode_entry(sh, e, p, l1, l2, N);
                    n1 = max(n1, l1);
                    n2 = max(n2, l2);
                    nN = max(nN, N);
                    mask |= 1 << p;
                    if (use_list) lists[0][atomicAdd(&s_cnt[0], 1)] = (uint16_t)e;
                }
            atomicMax(&s_need[1][0], n1);
            atomicMax(&s_need[1][1], n2);
            atomicMax(&s_need[1][2], nN);
            atomicOr(&s_need[1][3], mask);
        }
        int any = 1, chunk_no = 0;
        for (int f0 = 0; f0 < kRadGridPts; f0 += kRadThreads, chunk_no++) {
            const int np = min(kRadThreads, kRadGridPts - f0);
            any = __syncthreads_or(any);
            if (!any) break;
            const int nb = (chunk_no + 1) & 1;  // buffer written by the previous chunk (the scan for chunk 0)
            const int u1 = s_need[nb][0], u2 = s_need[nb][1], uN = s_need[nb][2], umask = s_need[nb][3];
            // this chunk's buffer: nobody reads or writes it between the two barriers
            if (tid < 4) s_need[chunk_no & 1][tid] = tid == 3 ? 0 : -1;
            // the list this chunk writes (read last by the chunk before the previous one)
            if (tid == 0) s_cnt[(chunk_no + 1) & 1] = 0;
            if (tid < np) {
                int lev, i, nr;
                walk_point(f0 + tid, lev, i, nr);
                double r, w;
                grid_point(f0 + tid, i, nr, r, w);
                const double r2 = r * r, ir = 1.0 / r, ir2 = 1.0 / r2;
                const double *wug = a.wu ? a.wu + (int64_t)sh.grpp * a.wu_npot * kRadGridPts + f0 + tid : nullptr;
                for (int pp = 0; pp < npot; pp++) {
                    if (!((umask >> pp) & 1)) continue;
                    if (wug) {
                        cwu[pp * kRadRow + tid] = __ldg(wug + (int64_t)pp * kRadGridPts);
                        continue;
                    }
                    double u = 0.0;
                    for (int k = 0; k < sh.pn[pp]; k++) {
                        const int tk = sh.poff[pp] + k;
                        const double ex = exp_rn(-sh.talpha[tk] * r2);
                        if (ex == 0.0) continue;  // the term adds an exact zero
                        const double rp = grid_rpow_m2(f0 + tid, sh.tpow[tk], ir, ir2);  // r^(n-2)
                        u += sh.tcoef[tk] * rp * ex;
                    }
                    cwu[pp * kRadRow + tid] = w * u;
                }
                if (a.ftab) {
                    // F^A_l, F^B_l of this point from the (shell, centre) tables
                    const double *FA = a.ftab + sh.fa_off + f0 + tid, *FB = a.ftab + sh.fb_off + f0 + tid;
                    for (int l = 0; l <= u1; l++) cf1[l * kRadRow + tid] = __ldg(FA + (int64_t)l * kRadGridPts);
                    for (int l = 0; l <= u2; l++) cf2[l * kRadRow + tid] = __ldg(FB + (int64_t)l * kRadGridPts);
                } else {
                    for (int l = 0; l <= u1; l++) cf1[l * kRadRow + tid] = 0.0;
                    for (int l = 0; l <= u2; l++) cf2[l * kRadRow + tid] = 0.0;
                }
                const double dA2 = (r - sh.CA) * (r - sh.CA), dB2 = (r - sh.CB) * (r - sh.CB);
                if (!a.ftab && u1 >= 0) {
#pragma unroll 1
                    for (int q = 0; q < np_a; q++) {
                        const double e = sh.ca[q] * exp_rn(-sh.xa[q] * dA2);
                        if (e != 0.0) bessel_row_acc(u1, sh.ka[q] * r, e, cf1 + tid, kRadRow);
                    }
                }
                if (!a.ftab && u2 >= 0) {
#pragma unroll 1
                    for (int q = 0; q < np_b; q++) {
                        const double e = sh.cb[q] * exp_rn(-sh.xb[q] * dB2);
                        if (e != 0.0) bessel_row_acc(u2, sh.kb[q] * r, e, cf2 + tid, kRadRow);
                    }
                }
                if (c_tab.grid) {
                    // r^N = pow(r, N) as libgrpp tabulates it (radial_type2_integral.c:440-441)
                    const double *gp = c_tab.grid + (size_t)kGridRowPow0 * kGridPts + f0 + tid;
                    for (int n = 0; n <= uN; n++) crn[n * kRadRow + tid] = __ldg(gp + (size_t)n * kGridPts);
                } else {
                    double rn = 1.0;
                    for (int n = 0; n <= uN; n++) {
                        crn[n * kRadRow + tid] = rn;
                        rn *= r;
                    }
                }
            }
            __syncthreads();
            int lev0, i0, nr0;
            walk_point(f0, lev0, i0, nr0);
            int my_active = 0, n1 = -1, n2 = -1, nN = -1, mask = 0, my_lvl = 0;
            // active entries: from the compacted list (an even share per thread), else all entries
            const int ncur = use_list ? s_cnt[chunk_no & 1] : nE;
            const uint16_t *lcur = lists[chunk_no & 1];
            uint16_t *lnext = lists[(chunk_no + 1) & 1];
            for (int k = tid; k < ncur; k += kRadThreads) {
                const int e = use_list ? lcur[k] : k;
                uint8_t fl = EF[e];
                if (!(fl & kEntActive)) continue;
                int p, l1, l2, N;
                decode_entry(sh, e, p, l1, l2, N);
                const double *pwu = cwu + p * kRadRow, *p1 = cf1 + l1 * kRadRow, *p2 = cf2 + l2 * kRadRow,
                             *pn = crn + N * kRadRow;
                double s = Q[e], sp = Sp[e];
                int q = 0, L = lev0;
                while (q < np) {
                    const int lend = level_last_point(L);
                    const int qe = min(np, lend - f0 + 1);
                    for (; q < qe; q++) s = __dadd_rn(s, __dmul_rn(__dmul_rn(__dmul_rn(pwu[q], p1[q]), p2[q]), pn[q]));
                    if (f0 + qe - 1 != lend) break;  // level continues in the next chunk
                    // end of level L for this entry (radial_type2_integral.c:285-315)
                    const bool forced = L == 0 || ((fl & kEntScrOk) && (fabs(s) / fabs(SC[e]) < 0.001));
                    if (!forced && fabs(s - sp) <= 1e-16) {
                        fl &= ~kEntActive;
                        my_lvl = max(my_lvl, L);
                        break;
                    }
                    if (L < kRadMaxLevel) {
                        sp = s;
                        s = 0.5 * s;
                    }
                    L++;
                }
                c_acc += q;
                Q[e] = s;
                Sp[e] = sp;
                EF[e] = fl;
                if (fl & kEntActive) {
                    if (use_list) lnext[atomicAdd(&s_cnt[(chunk_no + 1) & 1], 1)] = (uint16_t)e;
                    my_active = 1;
                    n1 = max(n1, l1);
                    n2 = max(n2, l2);
                    nN = max(nN, N);
                    mask |= 1 << p;
                }
            }
            if (my_active) {
                atomicMax(&s_need[chunk_no & 1][0], n1);
                atomicMax(&s_need[chunk_no & 1][1], n2);
                atomicMax(&s_need[chunk_no & 1][2], nN);
                atomicOr(&s_need[chunk_no & 1][3], mask);
            }
            if (my_lvl) atomicMax(&s_lvl, my_lvl);
            any = my_active;
        }
        any = __syncthreads_or(any);
        // deepest level walked: the cap if entries are still active, else the last convergence
        const int level_reached = any ? kRadMaxLevel : s_lvl;
        if (tid == 0 && a.stop_level) a.stop_level[item] = (int8_t)level_reached;
        if (tid == 0 && a.pred_level && level_reached > a.pred_level[item] + 1) atomicAdd(a.fallback_count, 1);
        if (a.counters) {
            unsigned long long v = c_acc;
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) atomicAdd(a.counters + kRadCntAccum, v);
            if (tid == 0) {
                // algorithmic work of the shared grid up to the stop level (every point once,
                // every order and potential term at every point)
                const unsigned long long pts = (unsigned long long)((1 << (level_reached + 5)) - 1);
                atomicAdd(a.counters + kRadCntPoints, pts);
                atomicAdd(a.counters + kRadCntBessel, pts * (unsigned long long)(np_a * (l1m + 1) + np_b * (l2m + 1)));
                atomicAdd(a.counters + kRadCntPrimPts, pts * (unsigned long long)(np_a + np_b));
                atomicAdd(a.counters + kRadCntTermPts, pts * (unsigned long long)sh.nterm_tot);
                atomicAdd(a.counters + kRadCntPowPts, pts * (unsigned long long)dn);
                atomicAdd(a.counters + kRadCntQuadCycles, (unsigned long long)(clock64() - t0));
                atomicAdd(a.counters + kRadCntItems, 1ull);
                atomicAdd(a.counters + kRadCntLevels, (unsigned long long)(level_reached + 1));
            }
        }
    }
}
#endif  // GRPP_RADIAL_TABLES_ONLY

}  // namespace grpp
