/*
 * ORACLE — test infrastructure only (see orc_common.h).
 *
 * Real spherical harmonics, angular integrals and L matrices, restated from:
 *   spherical_to_cartesian_coef ......... libgrpp/spherical_harmonics.c:115-166
 *                                         (Flores-Moreno et al., J. Comput. Chem. 27, 1009 (2006), eq. 32)
 *   coefficient tables / combinations .... libgrpp/spherical_harmonics.c:48-89, 283-305
 *   RSH values at k/|k| .................. libgrpp/spherical_harmonics.c:227-280
 *   unit-sphere polynomial integral ...... libgrpp/angular_integrals.c:118-130
 *   type 2 angular integral .............. libgrpp/angular_integrals.c:63-111
 *                                         (McMurchie & Davidson, J. Comput. Phys. 44, 289 (1981), eq. 29)
 *   L matrices in the RSH basis .......... libgrpp/lmatrix.c:28-141
 */
#include "orc_common.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static int rsh_ready = 0;
static int rsh_ncomb[ORC_LMAX_RSH + 1];
static int *rsh_comb[ORC_LMAX_RSH + 1];
static double *rsh_coef[ORC_LMAX_RSH + 1];

double orc_sph_to_cart_coef(int l, int m, int lx, int ly, int lz)
{
    (void)lz;
    int am = abs(m);
    int j = lx + ly - am;
    if (j % 2 != 0) return 0.0;
    j /= 2;
    int ok = (m > 0 && (am - lx) % 2 == 0) || (m == 0 && lx % 2 == 0) || (m < 0 && (am - lx) % 2 != 0);
    if (!ok) return 0.0;

    double pref = sqrt((2 * l + 1) / (2 * M_PI) * orc_factorial(l - am) / orc_factorial(l + am));
    pref /= pow(2, l) * orc_factorial(l);

    double u = 0.0;
    for (int i = j; i <= (l - am) / 2; i++) {
        if (2 * l - 2 * i < 0 || l - am - 2 * i < 0) {
            u = 0.0;
            break;
        }
        double f1 = (double)orc_binomial(l, i) * (double)orc_binomial(i, j) * pow(-1, i) *
                    orc_factorial_ratio(2 * l - 2 * i, l - am - 2 * i);
        double s = 0.0;
        for (int k = 0; k <= j; k++) {
            /* C-style truncating division of a possibly negative odd number, as in the reference */
            int e = (am - lx + 2 * k) / 2;
            s += (double)orc_binomial(j, k) * (double)orc_binomial(am, lx - 2 * k) * pow(-1, e);
        }
        u += f1 * s;
    }
    u *= pref;
    if (m == 0 && lx % 2 == 0) u *= M_SQRT1_2;
    return u;
}

static void rsh_tables_init(void)
{
    for (int L = 0; L <= ORC_LMAX_RSH; L++) {
        int n = (L + 1) * (L + 2) / 2;
        rsh_ncomb[L] = n;
        rsh_comb[L] = (int *)calloc(3 * n, sizeof(int));
        int c = 0;
        /* lexicographic order of (i,j,k), i+j+k=L (spherical_harmonics.c:283-305) */
        for (int i = 0; i <= L; i++)
            for (int jj = 0; jj <= L; jj++)
                for (int k = 0; k <= L; k++)
                    if (i + jj + k == L) {
                        rsh_comb[L][3 * c] = i;
                        rsh_comb[L][3 * c + 1] = jj;
                        rsh_comb[L][3 * c + 2] = k;
                        c++;
                    }
        rsh_coef[L] = (double *)calloc((2 * L + 1) * n, sizeof(double));
        for (int m = -L; m <= L; m++)
            for (int ic = 0; ic < n; ic++)
                rsh_coef[L][(m + L) * n + ic] =
                    orc_sph_to_cart_coef(L, m, rsh_comb[L][3 * ic], rsh_comb[L][3 * ic + 1], rsh_comb[L][3 * ic + 2]);
    }
    rsh_ready = 1;
}

int orc_rsh_ncomb(int L) { if (!rsh_ready) rsh_tables_init(); return rsh_ncomb[L]; }
const int *orc_rsh_comb(int L) { if (!rsh_ready) rsh_tables_init(); return rsh_comb[L]; }
const double *orc_rsh_coef(int L) { if (!rsh_ready) rsh_tables_init(); return rsh_coef[L]; }

void orc_rsh_array(int l, const double *k, double *out)
{
    if (!rsh_ready) rsh_tables_init();
    double ux = 0.0, uy = 0.0, uz = 0.0;
    double len = sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]);
    if (len > LIBGRPP_ZERO_THRESH) {
        double inv = 1.0 / len;
        ux = k[0] * inv;
        uy = k[1] * inv;
        uz = k[2] * inv;
    }
    double px[64], py[64], pz[64];
    px[0] = py[0] = pz[0] = 1.0;
    for (int i = 1; i <= l; i++) {
        px[i] = px[i - 1] * ux;
        py[i] = py[i - 1] * uy;
        pz[i] = pz[i - 1] * uz;
    }
    memset(out, 0, (2 * l + 1) * sizeof(double));
    int n = rsh_ncomb[l];
    for (int ic = 0; ic < n; ic++) {
        const int *c = rsh_comb[l] + 3 * ic;
        double kxyz = px[c[0]] * py[c[1]] * pz[c[2]];
        for (int m = -l; m <= l; m++) out[m + l] += rsh_coef[l][(m + l) * n + ic] * kxyz;
    }
}

/* 4 pi (i-1)!!(j-1)!!(k-1)!! / (i+j+k+1)!! for even i,j,k; zero otherwise */
double orc_usp_integral(int i, int j, int k)
{
    if (i % 2 == 0 && j % 2 == 0 && k % 2 == 0) {
        return 4 * M_PI * orc_double_factorial(i - 1) * orc_double_factorial(j - 1) *
               orc_double_factorial(k - 1) / orc_double_factorial(i + j + k + 1);
    }
    return 0.0;
}

double orc_angular_type2(int lambda, int L, int m, int a, int b, int c, const double *rsh_values)
{
    if (!rsh_ready) rsh_tables_init();
    double sum = 0.0;
    int nrst = rsh_ncomb[lambda], nuvw = rsh_ncomb[L];
    const int *rst = rsh_comb[lambda], *uvw = rsh_comb[L];
    const double *clam = rsh_coef[lambda], *cL = rsh_coef[L];
    for (int mu = -lambda; mu <= lambda; mu++) {
        double rv = rsh_values[mu + lambda];
        if (fabs(rv) < LIBGRPP_ZERO_THRESH) continue;
        double s2 = 0.0;
        for (int iu = 0; iu < nuvw; iu++) {
            double y1 = cL[(m + L) * nuvw + iu];
            if (fabs(y1) < LIBGRPP_ZERO_THRESH) continue;
            for (int ir = 0; ir < nrst; ir++) {
                double y2 = clam[(mu + lambda) * nrst + ir];
                if (fabs(y2) < LIBGRPP_ZERO_THRESH) continue;
                double usp = orc_usp_integral(a + rst[3 * ir] + uvw[3 * iu], b + rst[3 * ir + 1] + uvw[3 * iu + 1],
                                              c + rst[3 * ir + 2] + uvw[3 * iu + 2]);
                s2 += y2 * y1 * usp;
            }
        }
        sum += s2 * rv;
    }
    return sum;
}

/*
 * L matrices in the RSH basis. The reference forms <S_m1|L|S_m2> from the
 * complex-harmonic matrices through S_m = a Y_{-|m|} + b Y_{|m|}
 * (lmatrix.c:28-141); the same products are written out here in real
 * arithmetic on (re, im) pairs.
 */
typedef struct { double re, im; } cplx;
static cplx cmul(cplx x, cplx y) { cplx r = {x.re * y.re - x.im * y.im, x.re * y.im + x.im * y.re}; return r; }
static cplx cconj(cplx x) { cplx r = {x.re, -x.im}; return r; }

static void csh_to_rsh(int m, cplx *a, cplx *b)
{
    if (m == 0) {
        a->re = 0.5; a->im = 0.0;
        b->re = 0.5; b->im = 0.0;
    } else if (m < 0) {
        a->re = 0.0; a->im = 1.0 / sqrt(2);
        b->re = 0.0; b->im = -1.0 / sqrt(2) * pow(-1, abs(m));
    } else {
        a->re = 1.0 / sqrt(2); a->im = 0.0;
        b->re = 1.0 / sqrt(2) * pow(-1, m); b->im = 0.0;
    }
}

void orc_lmatrices_rsh(int L, double *lx, double *ly, double *lz)
{
    int dim = 2 * L + 1;
    double *cx = calloc(dim * dim, sizeof(double)), *cy = calloc(dim * dim, sizeof(double)),
           *cz = calloc(dim * dim, sizeof(double));
    for (int m1 = -L; m1 <= L; m1++)
        for (int m2 = -L; m2 <= L; m2++) {
            double z = m2 * (m1 == m2);
            double lp = sqrt((L - m2) * (L + m2 + 1)) * (m1 == m2 + 1);
            double lm = sqrt((L + m2) * (L - m2 + 1)) * (m1 == m2 - 1);
            cx[(m1 + L) * dim + m2 + L] = 0.5 * (lp + lm);
            cy[(m1 + L) * dim + m2 + L] = 0.5 * (lp - lm);
            cz[(m1 + L) * dim + m2 + L] = z;
        }
    for (int m1 = -L; m1 <= L; m1++)
        for (int m2 = -L; m2 <= L; m2++) {
            cplx a1, b1, a2, b2;
            csh_to_rsh(m1, &a1, &b1);
            csh_to_rsh(m2, &a2, &b2);
            int i1m = -abs(m1) + L, i1p = abs(m1) + L, i2m = -abs(m2) + L, i2p = abs(m2) + L;
            cplx w[4] = {cmul(cconj(a1), a2), cmul(cconj(a1), b2), cmul(cconj(b1), a2), cmul(cconj(b1), b2)};
            int idx[4] = {dim * i1m + i2m, dim * i1m + i2p, dim * i1p + i2m, dim * i1p + i2p};
            cplx sx = {0, 0}, sy = {0, 0}, sz = {0, 0};
            for (int q = 0; q < 4; q++) {
                sx.re += w[q].re * cx[idx[q]]; sx.im += w[q].im * cx[idx[q]];
                sy.re += w[q].re * cy[idx[q]]; sy.im += w[q].im * cy[idx[q]];
                sz.re += w[q].re * cz[idx[q]]; sz.im += w[q].im * cz[idx[q]];
            }
            lx[(m1 + L) * dim + m2 + L] = sx.im;
            ly[(m1 + L) * dim + m2 + L] = -sy.re;
            lz[(m1 + L) * dim + m2 + L] = sz.im;
        }
    free(cx);
    free(cy);
    free(cz);
}
