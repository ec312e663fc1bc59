// Host generation of the engine's constant tables (uploaded by engine.cu).
//
// Values that libgrpp ships as precomputed data (Bessel values on a 0.01 grid,
// specfunc_bessel_table.c; Boys values on a 0.1 grid, specfunc_boys.c) are
// generated here from convergent positive power series in long double:
//   exp(-x) i_l(x) = exp(-x) x^l/(2l+1)!! sum_k (x^2/2)^k / (k! prod_{j<=k} (2l+2j+1))
//   F_n(x)         = exp(-x) sum_k (2x)^k / prod_{j<=k} (2n+2j+1)
//   Daw(y)         = exp(-y^2) sum_k y^(2k+1) / (k! (2k+1))
// Derivatives of M_l follow the exact recurrence
//   M_l' = l/(2l+1) M_{l-1} + (l+1)/(2l+1) M_{l+1} - M_l
// (libgrpp/specfunc_scaled_mod_sph_bessel.c:135-156).
// Real spherical harmonic coefficients follow Flores-Moreno et al.,
// J. Comput. Chem. 27, 1009 (2006), eq. 32 (libgrpp/spherical_harmonics.c:115-166),
// L matrices the complex-to-real transform of libgrpp/lmatrix.c:28-141.
// The Fermi-model function S_j(x) = sum_{i>=1} (-1)^i e^{ix} / i^j (x <= 0), which libgrpp
// ships as data (specfunc_fermi_sk.c), is generated from its closed forms for j <= 1 and,
// for j >= 2, from its alternating series summed by the acceleration of Cohen,
// Rodriguez Villegas and Zagier (Exp. Math. 9, 3 (2000), algorithm 1), in long double.
#include <cmath>
#include <mutex>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "grpp_common.cuh"
#include "nucmodel.h"
#include "tables.h"

namespace grpp {

namespace {

long double bessel_series(int l, long double x)
{
    if (x == 0.0L) return l == 0 ? 1.0L : 0.0L;
    long double pref = 1.0L;
    for (int j = 1; j <= l; j++) pref *= x / (2.0L * j + 1.0L);
    long double h = 0.5L * x * x, term = 1.0L, sum = 1.0L;
    for (int k = 1; k < 4000; k++) {
        term *= h / ((long double)k * (2.0L * l + 2.0L * k + 1.0L));
        sum += term;
        if (term < 1e-24L * sum) break;
    }
    return expl(-x) * pref * sum;
}

long double boys_series(int n, long double x)
{
    long double term = 1.0L / (2.0L * n + 1.0L), sum = term;
    for (int k = 1; k < 8000; k++) {
        term *= 2.0L * x / (2.0L * n + 2.0L * k + 1.0L);
        sum += term;
        if (term < 1e-24L * sum) break;
    }
    return expl(-x) * sum;
}

long double dawson_series(long double y)
{
    long double y2 = y * y, p = y, sum = y;
    for (int k = 1; k < 8000; k++) {
        p *= y2 / k;
        long double t = p / (2.0L * k + 1.0L);
        sum += t;
        if (t < 1e-24L * sum) break;
    }
    return expl(-y2) * sum;
}

double factorial(int n)
{
    double r = 1.0;
    for (int k = 2; k <= n; k++) r *= k;
    return r;
}

double binom_d(int n, int k)
{
    if (k < 0 || k > n || n < 0) return 0.0;
    // exact for the small n used here (n <= 47 fits in a double's 53-bit mantissa)
    long double r = 1.0L;
    for (int j = 1; j <= k; j++) r = r * (n - k + j) / j;
    return (double)llroundl(r);
}

// libgrpp/spherical_harmonics.c:115-166
double sph_to_cart(int l, int m, int lx, int ly)
{
    int am = std::abs(m);
    int j = lx + ly - am;
    if (j % 2 != 0) return 0.0;
    j /= 2;
    bool ok = (m > 0 && (am - lx) % 2 == 0) || (m == 0 && lx % 2 == 0) || (m < 0 && (am - lx) % 2 != 0);
    if (!ok) return 0.0;
    double pref = std::sqrt((2 * l + 1) / (2 * kPi) * factorial(l - am) / factorial(l + am));
    pref /= std::pow(2, l) * factorial(l);
    double u = 0.0;
    for (int i = j; i <= (l - am) / 2; i++) {
        double fr = 1.0;  // (2l-2i)! / (l-|m|-2i)!
        for (int q = l - am - 2 * i + 1; q <= 2 * l - 2 * i; q++) fr *= q;
        double f1 = binom_d(l, i) * binom_d(i, j) * ((i % 2) ? -1.0 : 1.0) * fr;
        double s = 0.0;
        for (int k = 0; k <= j; k++) {
            int e = (am - lx + 2 * k) / 2;  // truncating division, as in C
            s += binom_d(j, k) * binom_d(am, lx - 2 * k) * ((e % 2) ? -1.0 : 1.0);
        }
        u += f1 * s;
    }
    u *= pref;
    if (m == 0 && lx % 2 == 0) u *= M_SQRT1_2;
    return u;
}

struct Cplx {
    double re, im;
};
Cplx cmul(Cplx a, Cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

void csh_to_rsh(int m, Cplx &a, Cplx &b)
{
    if (m == 0) {
        a = {0.5, 0.0};
        b = {0.5, 0.0};
    } else if (m < 0) {
        a = {0.0, 1.0 / std::sqrt(2.0)};
        b = {0.0, -1.0 / std::sqrt(2.0) * ((std::abs(m) % 2) ? -1.0 : 1.0)};
    } else {
        a = {1.0 / std::sqrt(2.0), 0.0};
        b = {1.0 / std::sqrt(2.0) * ((m % 2) ? -1.0 : 1.0), 0.0};
    }
}

}  // namespace

// S_j(x), j = -2..7, on x = -10 + 0.005 i, i = 0..2000: row i holds S_{-2} .. S_7
static void build_fermi_table(std::vector<double> &tab)
{
    tab.assign((size_t)kFermiNX * kFermiNK, 0.0);
    const int n = 48;  // CRVZ terms: error below (3 + sqrt 8)^-48 of the first term
    for (int i = 0; i < kFermiNX; i++) {
        const long double x = -10.0L + 0.005L * i, e = expl(x), z = -e;
        double *row = &tab[(size_t)i * kFermiNK];
        row[0] = (double)(z * (1 + z) / ((1 - z) * (1 - z) * (1 - z)));  // Li_{-2}(z), z = -e^x
        row[1] = (double)(z / ((1 - z) * (1 - z)));                    // Li_{-1}
        row[2] = (double)(z / (1 - z));                                // Li_0
        row[3] = (double)(-log1pl(e));                                 // Li_1
        for (int j = 2; j <= 7; j++) {
            // sum_{k>=0} (-1)^k a_k with a_k = e^{(k+1)x} / (k+1)^j, a moment sequence: S_j = -that sum
            long double d = powl(3.0L + sqrtl(8.0L), n);
            d = (d + 1.0L / d) / 2.0L;
            long double b = -1.0L, c = -d, s = 0.0L;
            for (int k = 0; k < n; k++) {
                c = b - c;
                s += c * (expl((k + 1) * x) / powl((long double)(k + 1), j));
                b = (long double)(k + n) * (long double)(k - n) * b / ((k + 0.5L) * (k + 1.0L));
            }
            row[j + 2] = (double)(-s / d);
        }
    }
}

const double *fermi_table()
{
    static std::vector<double> tab;
    static std::once_flag once;
    std::call_once(once, [] { build_fermi_table(tab); });
    return tab.data();
}

// The nested Log3 grid in walk order (grpp_common.cuh), with libgrpp's own expressions and the
// C library's log and pow, evaluated in this host unit without contraction: r and w of
// radial_type2_integral.c:357-365 (w at the point's own level nr), r^N = pow(r, N) of :440-441 and
// r^(n-2) = pow(r, n-2) of potential.c:70-81 for the powers n = 0, 1.
static void build_grid(std::vector<double> &g)
{
    g.assign((size_t)kGridRows * kGridPts, 0.0);
    const double R = 5.0;
    const double R3 = R * R * R;
    for (int f = 0; f < kGridPts; f++) {
        int level = 0;
        while ((1 << (level + 5)) - 2 < f) level++;
        const int nr = (1 << (level + 5)) - 1;
        const int i = level == 0 ? f + 1 : 2 * (f - ((1 << (level + 4)) - 1)) + 1;
        const double xi = i / (nr + 1.0);
        const double xi3 = xi * xi * xi;
        const double ln_xi = log(1 - xi3);
        const double wi = 3 * R3 * xi * xi * ln_xi * ln_xi / ((1 - xi3) * (nr + 1.0));
        const double ri = -R * ln_xi;
        g[(size_t)kGridRowR * kGridPts + f] = ri;
        g[(size_t)kGridRowW * kGridPts + f] = wi;
        // exponents through a volatile so that the compiler calls pow as libgrpp does (its
        // exponents are data) instead of folding pow(r, -1) into 1 / r
        volatile double e1 = -1.0, e2 = -2.0;
        g[(size_t)kGridRowRinv * kGridPts + f] = pow(ri, e1);
        g[(size_t)kGridRowRinv2 * kGridPts + f] = pow(ri, e2);
        for (int n = 0; n <= kGridMaxN; n++) {
            volatile double en = n;
            g[(size_t)(kGridRowPow0 + n) * kGridPts + f] = pow(ri, en);
        }
    }
}

void build_host_tables(HostTables &t)
{
    t.fermi.assign(fermi_table(), fermi_table() + (size_t)kFermiNX * kFermiNK);
    build_grid(t.grid);
    // Bessel values for orders 0..kBesL+4 so that all 4 derivative orders of 0..kBesL-1 are exact
    const int LV = kBesL + 5;
    std::vector<double> v((size_t)kBesNX * LV * 5, 0.0);
    for (int i = 0; i < kBesNX; i++) {
        long double x = 0.01L * i;
        double *row = &v[(size_t)i * LV * 5];
        for (int l = 0; l < LV; l++) row[5 * l] = (double)bessel_series(l, x);
        for (int k = 1; k < 5; k++)
            for (int l = 0; l < LV - k; l++) {
                double d = 0.0;
                if (l > 0) d += l / (2.0 * l + 1.0) * row[5 * (l - 1) + k - 1];
                d += (l + 1.0) / (2.0 * l + 1.0) * row[5 * (l + 1) + k - 1];
                d -= row[5 * l + k - 1];
                row[5 * l + k] = d;
            }
    }
    t.bessel.assign((size_t)kBesNX * kBesL * 5, 0.0);
    for (int i = 0; i < kBesNX; i++)
        memcpy(&t.bessel[(size_t)i * kBesL * 5], &v[(size_t)i * LV * 5], kBesL * 5 * sizeof(double));
    // pair layout: per x, per order pair p, coefficient k of orders 2p and 2p+1 side by side
    static_assert(kBesL % 2 == 0, "the pair layout needs an even number of orders");
    t.bessel_p.assign(t.bessel.size(), 0.0);
    for (int i = 0; i < kBesNX; i++)
        for (int l = 0; l < kBesL; l++)
            for (int k = 0; k < 5; k++)
                t.bessel_p[(size_t)i * kBesL * 5 + (l / 2) * 10 + 2 * k + (l % 2)] = t.bessel[((size_t)i * kBesL + l) * 5 + k];

    t.rfun.assign(kRfunL * kRfunL, 0.0);
    for (int n = 0; n < kRfunL; n++)
        for (int k = 0; k <= n; k++) {
            long double c = 1.0L;
            for (int q = 0; q < 2 * k; q++) c *= (long double)(n - k + 1 + q);  // (n+k)! / (n-k)!
            for (int j = 1; j <= k; j++) c /= 2.0L * j;
            t.rfun[n * kRfunL + k] = (double)c;
        }

    t.boys.assign(kBoysNX * kBoysNN, 0.0);
    for (int i = 0; i < kBoysNX; i++)
        for (int n = 0; n < kBoysNN; n++) t.boys[i * kBoysNN + n] = (double)boys_series(n, 0.1L * i);

    t.dawson.assign(kDawNY, 0.0);
    for (int j = 0; j < kDawNY; j++) t.dawson[j] = (double)dawson_series((long double)kDawY0 + (long double)j / 32.0L);

    t.rsh_off.assign(kRshL + 2, 0);
    t.rsh_comb_off.assign(kRshL + 2, 0);
    t.rsh_coef.clear();
    t.rsh_comb.clear();
    for (int l = 0; l <= kRshL; l++) {
        t.rsh_off[l] = (int)t.rsh_coef.size();
        t.rsh_comb_off[l] = (int)(t.rsh_comb.size() / 3);
        std::vector<int> comb;
        for (int i = 0; i <= l; i++)
            for (int j = 0; j <= l - i; j++) {
                comb.push_back(i);
                comb.push_back(j);
                comb.push_back(l - i - j);
            }
        int nc = (int)comb.size() / 3;
        for (int m = -l; m <= l; m++)
            for (int c = 0; c < nc; c++) t.rsh_coef.push_back(sph_to_cart(l, m, comb[3 * c], comb[3 * c + 1]));
        for (int x : comb) t.rsh_comb.push_back((int8_t)x);
    }
    t.rsh_off[kRshL + 1] = (int)t.rsh_coef.size();
    t.rsh_comb_off[kRshL + 1] = (int)(t.rsh_comb.size() / 3);

    t.lmat_off.assign(kMaxL + 3, 0);
    t.lmat.clear();
    for (int L = 0; L <= kMaxL + 1; L++) {
        t.lmat_off[L] = (int)t.lmat.size();
        int d = 2 * L + 1;
        std::vector<double> cx(d * d), cy(d * d), cz(d * d), out(3 * d * d);
        for (int m1 = -L; m1 <= L; m1++)
            for (int m2 = -L; m2 <= L; m2++) {
                double z = m2 * (m1 == m2);
                double lp = std::sqrt((double)((L - m2) * (L + m2 + 1))) * (m1 == m2 + 1);
                double lm = std::sqrt((double)((L + m2) * (L - m2 + 1))) * (m1 == m2 - 1);
                cx[(m1 + L) * d + m2 + L] = 0.5 * (lp + lm);
                cy[(m1 + L) * d + m2 + L] = 0.5 * (lp - lm);
                cz[(m1 + L) * d + m2 + L] = z;
            }
        for (int m1 = -L; m1 <= L; m1++)
            for (int m2 = -L; m2 <= L; m2++) {
                Cplx a1, b1, a2, b2;
                csh_to_rsh(m1, a1, b1);
                csh_to_rsh(m2, a2, b2);
                Cplx ca1 = {a1.re, -a1.im}, cb1 = {b1.re, -b1.im};
                int i1m = -std::abs(m1) + L, i1p = std::abs(m1) + L, i2m = -std::abs(m2) + L, i2p = std::abs(m2) + L;
                Cplx w[4] = {cmul(ca1, a2), cmul(ca1, b2), cmul(cb1, a2), cmul(cb1, b2)};
                int id[4] = {d * i1m + i2m, d * i1m + i2p, d * i1p + i2m, d * i1p + i2p};
                Cplx sx = {0, 0}, sy = {0, 0}, sz = {0, 0};
                for (int q = 0; q < 4; q++) {
                    sx.re += w[q].re * cx[id[q]];
                    sx.im += w[q].im * cx[id[q]];
                    sy.re += w[q].re * cy[id[q]];
                    sy.im += w[q].im * cy[id[q]];
                    sz.re += w[q].re * cz[id[q]];
                    sz.im += w[q].im * cz[id[q]];
                }
                int o = (m1 + L) * d + m2 + L;
                out[o] = sx.im;
                out[d * d + o] = -sy.re;
                out[2 * d * d + o] = sz.im;
            }
        t.lmat.insert(t.lmat.end(), out.begin(), out.end());
    }
    t.lmat_off[kMaxL + 2] = (int)t.lmat.size();

    t.dfact.assign(kDfMax + 2, 1.0);
    for (int n = 1; n <= kDfMax; n++) t.dfact[n + 1] = n * (n >= 2 ? t.dfact[n - 1] : 1.0);

    t.binom.assign(kBinN * kBinN, 0.0);
    for (int n = 0; n < kBinN; n++)
        for (int k = 0; k <= n; k++) t.binom[n * kBinN + k] = binom_d(n, k);
}

}  // namespace grpp
