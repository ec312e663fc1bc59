/*
 * ORACLE — test infrastructure only (see orc_common.h).
 *
 * Special functions and exact integer helpers, restated from libgrpp:
 *   factorials ........ libgrpp/factorial.c:37-115
 *   binomials ......... libgrpp/binomial.c:24-59 (exact uint64; here via Pascal's triangle)
 *   scaled modified spherical Bessel M_l(x) = exp(-x) i_l(x)
 *                       libgrpp/specfunc_scaled_mod_sph_bessel.c:45-190
 *   Boys function ..... libgrpp/specfunc_boys.c:21-57
 *   G_n function ...... libgrpp/specfunc_gfun.c:40-93
 *   Dawson integral ... used by specfunc_gfun.c:69; libgrpp takes it from a
 *                       third-party long-double Chebyshev code (specfunc_dawson.c);
 *                       here it is evaluated from its own positive power series
 *                       (long double) and its asymptotic series.
 *
 * The tabulated values libgrpp ships as data (Bessel values at 0.01 steps,
 * Boys values at 0.1 steps) are regenerated here at init from convergent
 * positive series in long double, then used with the same Taylor schemes.
 */
#include "orc_common.h"

#include <assert.h>
#include <math.h>
#include <string.h>

/* ---------------------------------------------------------------- factorials */

static const uint64_t fact_tab[21] = {
    1ULL, 1ULL, 2ULL, 6ULL, 24ULL, 120ULL, 720ULL, 5040ULL, 40320ULL, 362880ULL, 3628800ULL,
    39916800ULL, 479001600ULL, 6227020800ULL, 87178291200ULL, 1307674368000ULL,
    20922789888000ULL, 355687428096000ULL, 6402373705728000ULL, 121645100408832000ULL,
    2432902008176640000ULL};

/* factorial.c:37-47: n<0 -> 1; exact table to 20; recursion beyond */
double orc_factorial(int n)
{
    if (n < 0) return 1.0;
    if (n <= 20) return (double)fact_tab[n];
    return n * orc_factorial(n - 1);
}

/* factorial.c:55-70 */
double orc_factorial_ratio(int n, int m)
{
    if (n == m) return 1.0;
    if (n < m) return 1.0 / orc_factorial_ratio(m, n);
    double prod = 1.0;
    for (int i = m + 1; i <= n; i++) prod *= i;
    return prod;
}

/* factorial.c:105-115: n!! for -1 <= n <= 30, exact (computed here as uint64 products) */
double orc_double_factorial(int n)
{
    assert(n >= -1 && n <= 30);
    uint64_t r = 1;
    for (int k = n; k > 1; k -= 2) r *= (uint64_t)k;
    return (double)r;
}

/* binomial.c:24-59 semantics: exact C(n,k); k>n -> 0 (negative k also -> 0) */
static uint64_t pascal[65][65];
static int pascal_ready = 0;

static void pascal_init(void)
{
    memset(pascal, 0, sizeof(pascal));
    for (int n = 0; n <= 64; n++) {
        pascal[n][0] = 1;
        for (int k = 1; k <= n; k++) pascal[n][k] = pascal[n - 1][k - 1] + (k <= n - 1 ? pascal[n - 1][k] : 0);
    }
    pascal_ready = 1;
}

uint64_t orc_binomial(int n, int k)
{
    if (!pascal_ready) pascal_init();
    if (k < 0 || n < 0 || k > n) return 0;
    assert(n <= 64);
    return pascal[n][k];
}

/* ------------------------------------------------------------ Bessel M_l(x) */

#define BES_NL_EXT 64 /* values generated up to l=63 so that derivatives up to l=54 are complete */
static double bes_tab[ORC_BES_NX][BES_NL_EXT][5];
static double rfun[50][50];

/* exp(-x) i_l(x) from the positive series x^l/(2l+1)!! sum_k (x^2/2)^k / (k! prod_{j=1..k}(2l+2j+1)) */
static long double bessel_scaled_series(int l, long double x)
{
    if (x == 0.0L) return l == 0 ? 1.0L : 0.0L;
    long double pref = 1.0L;
    for (int j = 1; j <= l; j++) pref *= x / (2.0L * j + 1.0L);
    long double h = 0.5L * x * x, term = 1.0L, sum = 1.0L;
    for (int k = 1; k < 2000; k++) {
        term *= h / ((long double)k * (2.0L * l + 2.0L * k + 1.0L));
        sum += term;
        if (term < 1e-24L * sum) break;
    }
    return expl(-x) * pref * sum;
}

static void bessel_tables_init(void)
{
    for (int i = 0; i < ORC_BES_NX; i++) {
        long double x = 0.01L * i;
        for (int l = 0; l < BES_NL_EXT; l++) bes_tab[i][l][0] = (double)bessel_scaled_series(l, x);
        /* derivatives by the exact recurrence
         * M'_l = l/(2l+1) M_{l-1} + (l+1)/(2l+1) M_{l+1} - M_l
         * (specfunc_scaled_mod_sph_bessel.c:135-156) */
        for (int k = 1; k < 5; k++) {
            for (int l = 0; l < BES_NL_EXT - k; l++) {
                double d = 0.0;
                if (l > 0) d += l / (2.0 * l + 1.0) * bes_tab[i][l - 1][k - 1];
                d += (l + 1.0) / (2.0 * l + 1.0) * bes_tab[i][l + 1][k - 1];
                d -= bes_tab[i][l][k - 1];
                bes_tab[i][l][k] = d;
            }
        }
    }
    /* asymptotic coefficients (k+n)!/(k!(n-k)! 2^k)  (specfunc_scaled_mod_sph_bessel.c:163-190) */
    memset(rfun, 0, sizeof(rfun));
    for (int n = 0; n < 50; n++) {
        for (int k = 0; k <= n; k++) {
            long double v = 1.0L;
            for (int q = 0; q < 2 * k; q++) v *= (long double)(n - k + 1 + q); /* (n+k)!/(n-k)! */
            for (int j = 1; j <= k; j++) v /= (2.0L * j);    /* / (k! 2^k) */
            rfun[n][k] = (double)v;
        }
    }
}

/* specfunc_scaled_mod_sph_bessel.c:72-122 */
double orc_bessel_scaled(int n, double x)
{
    orc_stats.bessel_calls++;
    if (x <= 1e-7) {
        switch (n) {
        case 0: return 1.0 - x;
        case 1: return (1.0 - x) * x * (1.0 / 3.0);
        case 2: return (1.0 - x) * x * x * (1.0 / 15.0);
        default: return 0.0;
        }
    } else if (x <= 16.0) {
        int i0 = (int)(round(x * 100) + 1e-5);
        double dx = x - i0 * 0.01;
        const double *d = bes_tab[i0][n];
        double dx2 = dx * dx, dx3 = dx2 * dx, dx4 = dx3 * dx;
        return d[0] + d[1] * dx + d[2] * dx2 * 0.5 + d[3] * dx3 * (1.0 / 6.0) + d[4] * dx4 * (1.0 / 24.0);
    } else {
        double z = -x, sum = 0.0, den = 1.0, inv = 1.0 / z;
        for (int k = 0; k <= n; k++) {
            sum += rfun[n][k] * den;
            den *= inv;
        }
        return sum / (2.0 * x);
    }
}

/* --------------------------------------------------------------- Boys F_n(x) */

static double boys_tab[ORC_BOYS_NX][ORC_BOYS_NN];

/* F_n(x) = exp(-x) sum_k (2x)^k / prod_{j=0..k} (2n+2j+1) */
static long double boys_series(int n, long double x)
{
    long double term = 1.0L / (2.0L * n + 1.0L), sum = term;
    for (int k = 1; k < 5000; k++) {
        term *= 2.0L * x / (2.0L * n + 2.0L * k + 1.0L);
        sum += term;
        if (term < 1e-24L * sum) break;
    }
    return expl(-x) * sum;
}

static void boys_tables_init(void)
{
    for (int i = 0; i < ORC_BOYS_NX; i++)
        for (int n = 0; n < ORC_BOYS_NN; n++) boys_tab[i][n] = (double)boys_series(n, 0.1L * i);
}

/* specfunc_boys.c:21-47: 6th-order Taylor on the 0.1 grid for x<=30, asymptotic above */
double orc_boys(int n, double x)
{
    if (x <= 30.0) {
        int idx = (int)(round(x / 0.1) + 1e-6);
        double dx = x - idx * 0.1;
        double dx2 = dx * dx, dx3 = dx * dx2, dx4 = dx * dx3, dx5 = dx * dx4, dx6 = dx * dx5;
        const double *b = boys_tab[idx];
        return +b[n] - b[n + 1] * dx + b[n + 2] * dx2 / 2.0 - b[n + 3] * dx3 / 6.0 +
               b[n + 4] * dx4 / 24.0 - b[n + 5] * dx5 / 120.0 + b[n + 6] * dx6 / 720.0;
    }
    return orc_double_factorial(2 * n - 1) / pow(2.0, n + 1) * sqrt(M_PI / pow(x, 2 * n + 1));
}

void orc_boys_values(double x, int nmax, double *b)
{
    for (int n = 0; n <= nmax; n++) b[n] = orc_boys(n, x);
}

/* ----------------------------------------------------------- Dawson, G_n(x) */

/* Daw(y) = exp(-y^2) int_0^y exp(t^2) dt */
double orc_dawson(double y)
{
    int sgn = y < 0 ? -1 : 1;
    long double a = fabsl((long double)y);
    if (a <= 10.0L) {
        /* exp(-a^2) sum_k a^(2k+1) / (k! (2k+1)): all terms positive */
        long double a2 = a * a, p = a, sum = a;
        for (int k = 1; k < 5000; k++) {
            p *= a2 / k;
            long double t = p / (2.0L * k + 1.0L);
            sum += t;
            if (t < 1e-24L * sum) break;
        }
        return sgn * (double)(expl(-a2) * sum);
    }
    /* asymptotic: 1/(2a) sum_k (2k-1)!! / (2a^2)^k, summed while terms decrease */
    long double x2 = 2.0L * a * a, term = 1.0L, sum = 1.0L;
    for (int k = 1; k < 200; k++) {
        long double nt = term * (2.0L * k - 1.0L) / x2;
        if (nt >= term) break;
        term = nt;
        sum += term;
        if (term < 1e-24L * sum) break;
    }
    return sgn * (double)(sum / (2.0L * a));
}

/* specfunc_gfun.c:77-93: series sum_k exp(-x) x^k / k! / (2n+2k+1), stop when a term < 1e-15 */
static double gfun_taylor(int n, double x)
{
    double sum = 0.0;
    for (int k = 0; k < 100; k++) {
        double c = exp(-x) * pow(x, k) / orc_factorial(k) / (2.0 * n + 2.0 * k + 1.0);
        sum += c;
        if (fabs(c) < 1e-15) break;
    }
    return sum;
}

/* specfunc_gfun.c:40-71: downward recursion from the series (x<=12) or upward from Dawson */
void orc_gfun_values(double x, int nmax, double *g)
{
    memset(g, 0, (nmax + 1) * sizeof(double));
    if (x <= 12.0) {
        g[nmax] = gfun_taylor(nmax, x);
        for (int n = nmax; n > 0; n--) g[n - 1] = (1.0 - 2.0 * x * g[n]) / (2.0 * n - 1.0);
    } else {
        double sx = sqrt(x);
        g[0] = orc_dawson(sx) / sx;
        for (int n = 0; n < nmax; n++) g[n + 1] = (1.0 - (2 * n + 1) * g[n]) / (2.0 * x);
    }
}

void orc_tables_init(void)
{
    if (!pascal_ready) pascal_init();
    bessel_tables_init();
    boys_tables_init();
}

/* screening.c:226-236: int_0^inf r^n exp(-a r^2) dr */
double orc_gaussian_integral(int n, double a)
{
    if (n % 2 == 0) {
        int k = n / 2;
        return orc_double_factorial(2 * k - 1) / (pow(2.0, k + 1) * pow(a, k)) * sqrt(M_PI / a);
    }
    int k = (n - 1) / 2;
    return orc_factorial(k) / (2.0 * pow(a, k + 1));
}
