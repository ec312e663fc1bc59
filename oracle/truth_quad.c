/*
 * ORACLE — test infrastructure only (see orc_common.h).
 *
 * Extended-precision values of the GRPP integrals libgrpp approximates, for
 * judging elements on which libgrpp itself keeps few or no significant digits.
 *
 * The operators are libgrpp's own definitions:
 *   type 1      <A| U_L(|r-C|) |B>, McMurchie-Davidson over primitive triples
 *               (libgrpp/type1_mcmurchie_davidson.c:107-622: E, R (1/r, Boys),
 *               G (1/r^2) recursions);
 *   type 2      <A| U_l(|r-C|) P_l |B>, binomial re-centring of both shells on C,
 *               Bessel expansion of the off-centre Gaussians, angular integrals
 *               over real spherical harmonics (libgrpp/type2_integrals.c:34-243,
 *               libgrpp/angular_integrals.c:63-130,
 *               libgrpp/spherical_harmonics.c:115-166);
 *   spin-orbit  the same with the L matrices in the real-harmonic basis
 *               (libgrpp/spin_orbit_integrals.c:41-288, libgrpp/lmatrix.c:28-141);
 *   outercore   parts 1 and 2 (libgrpp/outercore_integrals.c:83-553);
 *   full GRPP   their sum as libgrpp_full_grpp_integrals forms it
 *               (libgrpp/full_grpp_integrals.c:27-104).
 * What differs from libgrpp is only how accurately they are evaluated:
 *   - every operation is IEEE binary128 (__float128, 113-bit significand);
 *   - special functions are computed directly to full binary128 accuracy
 *     (Boys and G_n from their positive series or, for x >= 80, from erf /
 *     the asymptotic Dawson series whose truncation error is below e^-x,
 *     with stable upward recursion; M_l(x) = e^-x i_l(x) from its positive
 *     series with the stable downward recurrence, or the closed form for x > 60);
 *   - every radial integral is summed on the nested Log3 grid libgrpp uses
 *     (r = -5 ln(1 - x^3)), with Richardson elimination of the rule's h^6, h^12,
 *     h^18, h^24 error terms, until two successive levels agree to 1e-30 of the
 *     sum of the absolute values of its terms (no absolute 1e-16 stop, no
 *     screening estimate returned in place of the integral), up to 2^19 points;
 *   - no term is skipped by a size threshold (only exact zeros).
 * Inputs are libgrpp's double-precision inputs as given (potential terms with
 * |c| < 1e-14 and primitives with |c| < 1e-14 are dropped, as libgrpp's
 * constructors and shell shrinking define the operator and the shells).
 * Outputs are rounded to double at the end.
 */
#include <math.h>
#include <quadmath.h>
#include <stdio.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/libgrpp_b200.h"

typedef __float128 qr;

#define TQ_FACT 200
#define TQ_LMAX 24        /* largest lambda of the expansions */
#define TQ_LEVEL_MIN 8    /* 8191 points, libgrpp's deepest level */
#define TQ_LEVEL_MAX 14   /* 2^19 - 1 points */
#define TQ_RICH_START 3   /* first level of the Richardson table (255 points) */
#define TQ_RICH_K 4       /* orders h^6 .. h^24 eliminated */
#define TQ_ZERO 1e-14     /* libgrpp's LIBGRPP_ZERO_THRESH: dropped terms and primitives */

static qr q_fact[TQ_FACT + 1];
static qr q_dfact[2 * TQ_FACT + 4]; /* (n)!! stored at n + 1, n >= -1 */
static int q_ready = 0;

#define DF(n) q_dfact[(n) + 1]

static void q_init(void)
{
    if (q_ready) return;
    q_fact[0] = 1;
    for (int n = 1; n <= TQ_FACT; n++) q_fact[n] = q_fact[n - 1] * n;
    q_dfact[0] = 1; /* (-1)!! */
    q_dfact[1] = 1; /* 0!! */
    for (int n = 1; n < 2 * TQ_FACT + 2; n++) q_dfact[n + 1] = n * (n >= 2 ? q_dfact[n - 1] : (qr)1);
    q_ready = 1;
}

static qr q_binom(int n, int k)
{
    if (n < 0 || k < 0 || k > n) return 0;
    return q_fact[n] / (q_fact[k] * q_fact[n - k]);
}

static qr q_ipow(qr x, int n)
{
    qr r = 1;
    for (int i = 0; i < n; i++) r *= x;
    return r;
}

/* (2 alpha / pi)^(3/4) (4 alpha)^(L/2): libgrpp's primitive norm (libgrpp/norm_gaussian.c:16-23) */
static qr q_gnorm(int L, qr a) { return powq(2 * a / M_PIq, 0.75Q) * powq(4 * a, 0.5Q * L); }

/* ============================================================ special functions */

/* Boys F_n(x) = int_0^1 t^(2n) exp(-x t^2) dt, n = 0..nmax */
static void q_boys(int nmax, qr x, qr *F)
{
    qr ex = expq(-x);
    if (x < 80) {
        qr t = 1 / (qr)(2 * nmax + 1), s = t;
        for (int k = 1; k < 5000; k++) {
            t *= 2 * x / (2 * nmax + 2 * k + 1);
            s += t;
            if (t < s * 1e-36Q && k > x) break;
        }
        F[nmax] = ex * s;
        for (int n = nmax; n > 0; n--) F[n - 1] = (2 * x * F[n] + ex) / (2 * n - 1); /* positive terms */
    } else {
        F[0] = 0.5Q * sqrtq(M_PIq / x) * erfq(sqrtq(x));
        for (int n = 0; n < nmax; n++) F[n + 1] = ((2 * n + 1) * F[n] - ex) / (2 * x); /* x > n: stable */
    }
}

/* G_n(x) = int_0^1 exp(-x (1 - t^2)) t^(2n) dt, n = 0..nmax (the 1/r^2 kernel) */
static void q_gfun(int nmax, qr x, qr *G)
{
    if (x < 80) {
        /* G_n = e^-x sum_k x^k / (k! (2n + 2k + 1)), every n from its own positive series
         * (the downward recursion loses a factor 2x/(2n-1) per step) */
        qr ex = expq(-x);
        for (int n = 0; n <= nmax; n++) {
            qr p = 1, s = 1 / (qr)(2 * n + 1);
            for (int k = 1; k < 5000; k++) {
                p *= x / k;
                qr t = p / (2 * n + 2 * k + 1);
                s += t;
                if (t < s * 1e-36Q && k > x) break;
            }
            G[n] = ex * s;
        }
    } else {
        /* G_0 = D(sqrt x)/sqrt x = 1/(2x) sum_k (2k-1)!!/(2x)^k, cut at its smallest term
         * (truncation error of order e^-x < 2e-35 relative) */
        qr t = 1, s = 1;
        for (int k = 1; k < 100000; k++) {
            qr tn = t * (2 * k - 1) / (2 * x);
            if (tn >= t) break;
            t = tn;
            s += t;
            if (t < s * 1e-36Q) break;
        }
        G[0] = s / (2 * x);
        for (int n = 0; n < nmax; n++) G[n + 1] = (1 - (2 * n + 1) * G[n]) / (2 * x); /* factor (2n+1)/2x < 1 */
    }
}

/* M_l(x) = exp(-x) i_l(x), l = 0..lmax */
static void q_bessel(int lmax, qr x, qr *M)
{
    if (x == 0) {
        M[0] = 1;
        for (int l = 1; l <= lmax; l++) M[l] = 0;
        return;
    }
    if (x <= 60) {
        /* i_l(x) = x^l sum_k (x^2/2)^k / (k! (2l+2k+1)!!) for l = lmax, lmax+1, then
         * i_{l-1} = i_{l+1} + (2l+1)/x i_l downwards (positive terms) */
        qr I[TQ_LMAX + 3];
        for (int l = lmax; l <= lmax + 1; l++) {
            qr t = q_ipow(x, l) / DF(2 * l + 1), s = t;
            for (int k = 1; k < 5000; k++) {
                t *= x * x / (2 * k * (qr)(2 * l + 2 * k + 1));
                s += t;
                if (t < s * 1e-36Q && k > x) break;
            }
            I[l] = s;
        }
        for (int l = lmax; l > 0; l--) I[l - 1] = I[l + 1] + (2 * l + 1) / x * I[l];
        qr ex = expq(-x);
        for (int l = 0; l <= lmax; l++) M[l] = ex * I[l];
    } else {
        /* e^-x i_l(x) = 1/(2x) [sum_k (-1)^k a_k y^k - (-1)^l e^-2x sum_k a_k y^k],
         * a_k = (l+k)!/(k!(l-k)!), y = 1/(2x) */
        qr y = 1 / (2 * x), e2 = expq(-2 * x);
        for (int l = 0; l <= lmax; l++) {
            qr s1 = 0, s2 = 0, yk = 1;
            for (int k = 0; k <= l; k++) {
                qr a = q_fact[l + k] / (q_fact[k] * q_fact[l - k]) * yk;
                s1 += (k % 2 ? -a : a);
                s2 += a;
                yk *= y;
            }
            M[l] = y * (s1 - ((l % 2) ? -e2 : e2) * s2);
        }
    }
}

/* int_0^inf r^n exp(-p r^2) dr */
static qr q_gauss_int(int n, qr p) { return tgammaq((n + 1) / 2.0Q) / (2 * powq(p, (n + 1) / 2.0Q)); }

/* ============================================================ angular tables */

/* Flores-Moreno coefficient of x^lx y^ly z^lz in the real solid harmonic S_lm
 * (libgrpp/spherical_harmonics.c:115-166; the same integer arithmetic, binary128 values) */
static qr q_sph_coef(int l, int m, int lx, int ly, int lz)
{
    (void)lz;
    int am = abs(m);
    int j = lx + ly - am;
    if (j % 2 != 0) return 0;
    j /= 2;
    int ok = (m > 0 && (am - lx) % 2 == 0) || (m == 0 && lx % 2 == 0) || (m < 0 && (am - lx) % 2 != 0);
    if (!ok) return 0;
    qr pref = sqrtq((2 * l + 1) / (2 * M_PIq) * q_fact[l - am] / q_fact[l + am]);
    pref /= q_ipow(2, l) * q_fact[l];
    qr u = 0;
    for (int i = j; i <= (l - am) / 2; i++) {
        if (2 * l - 2 * i < 0 || l - am - 2 * i < 0) {
            u = 0;
            break;
        }
        qr f1 = q_binom(l, i) * q_binom(i, j) * ((i % 2) ? -1 : 1) * (q_fact[2 * l - 2 * i] / q_fact[l - am - 2 * i]);
        qr s = 0;
        for (int k = 0; k <= j; k++) {
            int e = (am - lx + 2 * k) / 2; /* C truncating division, as libgrpp */
            s += q_binom(j, k) * q_binom(am, lx - 2 * k) * ((abs(e) % 2) ? -1 : 1);
        }
        u += f1 * s;
    }
    u *= pref;
    if (m == 0 && lx % 2 == 0) u *= M_SQRT1_2q;
    return u;
}

typedef struct {
    int n;             /* components of degree L */
    int comb[400][3];  /* lexicographic (i, j, k), i + j + k = L */
    qr *coef;          /* [(m + L) * n + ic] */
} q_rsh_t;

static q_rsh_t q_rsh[TQ_LMAX + 1];

static void q_rsh_init(void)
{
    for (int L = 0; L <= TQ_LMAX; L++) {
        q_rsh_t *t = &q_rsh[L];
        t->n = 0;
        for (int i = 0; i <= L; i++)
            for (int j = 0; j <= L; j++)
                for (int k = 0; k <= L; k++)
                    if (i + j + k == L) {
                        t->comb[t->n][0] = i;
                        t->comb[t->n][1] = j;
                        t->comb[t->n][2] = k;
                        t->n++;
                    }
        t->coef = calloc((size_t)(2 * L + 1) * t->n, sizeof(qr));
        for (int m = -L; m <= L; m++)
            for (int ic = 0; ic < t->n; ic++)
                t->coef[(m + L) * t->n + ic] = q_sph_coef(L, m, t->comb[ic][0], t->comb[ic][1], t->comb[ic][2]);
    }
}

/* S_lm(u), m = -l..l, at the unit vector u (zero vector: only l = 0 survives) */
static void q_rsh_values(int l, const qr *u, qr *out)
{
    const q_rsh_t *t = &q_rsh[l];
    for (int m = 0; m <= 2 * l; m++) out[m] = 0;
    for (int ic = 0; ic < t->n; ic++) {
        qr v = q_ipow(u[0], t->comb[ic][0]) * q_ipow(u[1], t->comb[ic][1]) * q_ipow(u[2], t->comb[ic][2]);
        for (int m = 0; m <= 2 * l; m++) out[m] += t->coef[m * t->n + ic] * v;
    }
}

/* int over the unit sphere of x^i y^j z^k */
static qr q_usp(int i, int j, int k)
{
    if (i % 2 || j % 2 || k % 2) return 0;
    return 4 * M_PIq * DF(i - 1) * DF(j - 1) * DF(k - 1) / DF(i + j + k + 1);
}

/* A[mu][m] = sum over the Cartesian terms of S_Lm and S_lambda,mu of the unit-sphere integral of
 * x^(a+..) y^(b+..) z^(c+..): the k-independent part of libgrpp's type 2 angular integral
 * (libgrpp/angular_integrals.c:63-111). Cached per thread by (lambda, L, a, b, c). */
#define TQ_AMAX 12 /* a, b, c < TQ_AMAX */
static __thread qr *q_atab[TQ_LMAX + 1][8][TQ_AMAX][TQ_AMAX][TQ_AMAX];

static const qr *q_angular_tensor(int lambda, int L, int a, int b, int c)
{
    qr **slot = &q_atab[lambda][L][a][b][c];
    if (*slot) return *slot;
    const q_rsh_t *tl = &q_rsh[lambda], *tL = &q_rsh[L];
    qr *A = calloc((size_t)(2 * lambda + 1) * (2 * L + 1), sizeof(qr));
    for (int mu = -lambda; mu <= lambda; mu++)
        for (int m = -L; m <= L; m++) {
            qr s2 = 0;
            for (int iu = 0; iu < tL->n; iu++) {
                qr y1 = tL->coef[(m + L) * tL->n + iu];
                if (y1 == 0) continue;
                for (int ir = 0; ir < tl->n; ir++) {
                    qr y2 = tl->coef[(mu + lambda) * tl->n + ir];
                    if (y2 == 0) continue;
                    s2 += y2 * y1 * q_usp(a + tl->comb[ir][0] + tL->comb[iu][0], b + tl->comb[ir][1] + tL->comb[iu][1],
                                          c + tl->comb[ir][2] + tL->comb[iu][2]);
                }
            }
            A[(mu + lambda) * (2 * L + 1) + m + L] = s2;
        }
    *slot = A;
    return A;
}

/* omega(lambda, L, m; a, b, c) = sum_mu S_lambda,mu(k) A[mu][m] */
static qr q_omega(int lambda, int L, int m, int a, int b, int c, const qr *rsh_k)
{
    const qr *A = q_angular_tensor(lambda, L, a, b, c);
    qr sum = 0;
    for (int mu = -lambda; mu <= lambda; mu++) sum += rsh_k[mu + lambda] * A[(mu + lambda) * (2 * L + 1) + m + L];
    return sum;
}

/* <S_m1| L_x,y,z |S_m2> in the real-harmonic basis, libgrpp's sign convention (lmatrix.c:28-141):
 * products of the complex-harmonic matrices with S_m = a Y_-|m| + b Y_|m| written out in pairs */
static void q_lmatrices(int L, qr *lx, qr *ly, qr *lz)
{
    int d = 2 * L + 1;
    qr *cx = calloc(d * d, sizeof(qr)), *cy = calloc(d * d, sizeof(qr)), *cz = calloc(d * d, sizeof(qr));
    for (int m1 = -L; m1 <= L; m1++)
        for (int m2 = -L; m2 <= L; m2++) {
            qr lp = (m1 == m2 + 1) ? sqrtq((qr)((L - m2) * (L + m2 + 1))) : 0;
            qr lm = (m1 == m2 - 1) ? sqrtq((qr)((L + m2) * (L - m2 + 1))) : 0;
            cx[(m1 + L) * d + m2 + L] = 0.5Q * (lp + lm);
            cy[(m1 + L) * d + m2 + L] = 0.5Q * (lp - lm);
            cz[(m1 + L) * d + m2 + L] = (m1 == m2) ? (qr)m2 : 0;
        }
    for (int m1 = -L; m1 <= L; m1++)
        for (int m2 = -L; m2 <= L; m2++) {
            qr ar[2][2], ai[2][2]; /* [side][a or b] real and imaginary parts */
            int ms[2] = {m1, m2};
            for (int s = 0; s < 2; s++) {
                int m = ms[s];
                if (m == 0) {
                    ar[s][0] = 0.5Q; ai[s][0] = 0;
                    ar[s][1] = 0.5Q; ai[s][1] = 0;
                } else if (m < 0) {
                    ar[s][0] = 0; ai[s][0] = M_SQRT1_2q;
                    ar[s][1] = 0; ai[s][1] = -M_SQRT1_2q * ((abs(m) % 2) ? -1 : 1);
                } else {
                    ar[s][0] = M_SQRT1_2q; ai[s][0] = 0;
                    ar[s][1] = M_SQRT1_2q * ((m % 2) ? -1 : 1); ai[s][1] = 0;
                }
            }
            int i1m = -abs(m1) + L, i1p = abs(m1) + L, i2m = -abs(m2) + L, i2p = abs(m2) + L;
            int idx[4] = {d * i1m + i2m, d * i1m + i2p, d * i1p + i2m, d * i1p + i2p};
            int sel[4][2] = {{0, 0}, {0, 1}, {1, 0}, {1, 1}};
            qr sxi = 0, syr = 0, szi = 0;
            for (int q = 0; q < 4; q++) {
                /* conj(x1) * x2 */
                qr xr = ar[0][sel[q][0]], xi = -ai[0][sel[q][0]], yr = ar[1][sel[q][1]], yi = ai[1][sel[q][1]];
                qr wr = xr * yr - xi * yi, wi = xr * yi + xi * yr;
                sxi += wi * cx[idx[q]];
                syr += wr * cy[idx[q]];
                szi += wi * cz[idx[q]];
            }
            lx[(m1 + L) * d + m2 + L] = sxi;
            ly[(m1 + L) * d + m2 + L] = -syr;
            lz[(m1 + L) * d + m2 + L] = szi;
        }
    free(cx);
    free(cy);
    free(cz);
}

/* ============================================================ objects from the flat batch */

typedef struct {
    int L, n;          /* angular momentum, primitives kept */
    qr c[64], a[64];   /* raw coefficients and exponents (|c| >= 1e-14) */
    qr o[3];
    const int *cart;   /* 3 ints per component */
} q_shell_t;

typedef struct {
    int L, J, n;
    int pw[64];
    qr c[64], z[64];
} q_pot_t;

static void q_shell(const libgrpp_b200_batch_t *b, int s, q_shell_t *sh)
{
    sh->L = b->shell_L[s];
    sh->n = 0;
    for (int k = 0; k < b->shell_nprim[s]; k++) {
        double c = b->prim_coef[b->shell_prim_off[s] + k];
        if (fabs(c) < TQ_ZERO) continue;
        sh->c[sh->n] = c;
        sh->a[sh->n] = b->prim_alpha[b->shell_prim_off[s] + k];
        sh->n++;
    }
    for (int i = 0; i < 3; i++) sh->o[i] = b->shell_origin[3 * s + i];
    sh->cart = b->cart_list + 3 * b->shell_cart_off[s];
}

static void q_pot(const libgrpp_b200_batch_t *b, int p, q_pot_t *P)
{
    P->L = b->pot_L[p];
    P->J = b->pot_J[p];
    P->n = 0;
    for (int k = 0; k < b->pot_nprim[p]; k++) {
        int o = b->pot_prim_off[p] + k;
        if (fabs(b->pot_coef[o]) < TQ_ZERO) continue;
        P->pw[P->n] = b->pot_powers[o];
        P->c[P->n] = b->pot_coef[o];
        P->z[P->n] = b->pot_alpha[o];
        P->n++;
    }
}

static int ncart(int L) { return (L + 1) * (L + 2) / 2; }

/* ============================================================ type 1 (MMD) */

/* coef <A| r_C^(n-2) exp(-zeta r_C^2) |B> over all primitive pairs, added to out (nA x nB) */
static void q_type1_term(const q_shell_t *A, const q_shell_t *B, const qr *C, qr zeta, int npow, qr coef, qr *out)
{
    int la = A->L, lb = B->L, S = la + lb, nA = ncart(la), nB = ncart(lb);
    int dE = S + 1, dR = S + 1;
    qr *E = calloc(3 * (la + 1) * (lb + 1) * dE, sizeof(qr));
    qr *R = calloc((size_t)dR * dR * dR * (S + 2), sizeof(qr));
#define EI(c, i, j, t) ((((c) * (la + 1) + (i)) * (lb + 1) + (j)) * dE + (t))
#define RI(t, u, v, n) ((((t) * dR + (u)) * dR + (v)) * (S + 2) + (n))
    for (int i = 0; i < A->n; i++)
        for (int j = 0; j < B->n; j++) {
            qr a = A->a[i], bb = B->a[j], q = a + bb + zeta;
            qr Q[3], K[3];
            for (int x = 0; x < 3; x++) {
                Q[x] = (a * A->o[x] + bb * B->o[x] + zeta * C[x]) / q;
                qr xab = A->o[x] - B->o[x], xac = A->o[x] - C[x], xbc = B->o[x] - C[x];
                K[x] = expq(-(a * bb * xab * xab + a * zeta * xac * xac + bb * zeta * xbc * xbc) / q);
            }
            for (int x = 0; x < 3; x++)
                for (int ii = 0; ii <= la; ii++)
                    for (int jj = 0; jj <= lb; jj++)
                        for (int t = 0; t <= ii + jj; t++) {
                            qr v;
                            if (t == 0) {
                                if (ii == 0 && jj == 0) v = K[x];
                                else if (ii == 0) v = (Q[x] - B->o[x]) * E[EI(x, 0, jj - 1, 0)] + E[EI(x, 0, jj - 1, 1)];
                                else v = (Q[x] - A->o[x]) * E[EI(x, ii - 1, jj, 0)] + E[EI(x, ii - 1, jj, 1)];
                            } else {
                                qr f = 1 / (2 * q * t);
                                v = 0;
                                if (ii > 0) v += f * ii * E[EI(x, ii - 1, jj, t - 1)];
                                if (jj > 0) v += f * jj * E[EI(x, ii, jj - 1, t - 1)];
                            }
                            E[EI(x, ii, jj, t)] = v;
                        }
            qr NA = q_gnorm(la, a), NB = q_gnorm(lb, bb), w = coef * A->c[i] * B->c[j] * NA * NB;
            if (npow == 2) {
                qr pf = w * powq(M_PIq / q, 1.5Q);
                for (int m = 0; m < nA; m++)
                    for (int n = 0; n < nB; n++) {
                        const int *ca = A->cart + 3 * m, *cb = B->cart + 3 * n;
                        out[m * nB + n] += pf * E[EI(0, ca[0], cb[0], 0)] * E[EI(1, ca[1], cb[1], 0)] * E[EI(2, ca[2], cb[2], 0)];
                    }
                continue;
            }
            qr QC[3] = {Q[0] - C[0], Q[1] - C[1], Q[2] - C[2]};
            qr x2 = q * (QC[0] * QC[0] + QC[1] * QC[1] + QC[2] * QC[2]);
            qr aux[64];
            int g = npow == 0;
            if (g) q_gfun(S, x2, aux);
            else q_boys(S, x2, aux);
            for (int t = 0; t <= S; t++)
                for (int u = 0; u <= S - t; u++)
                    for (int v = 0; v <= S - t - u; v++)
                        for (int n = 0; n <= S - (t + u + v); n++) {
                            qr val = 0;
                            if (t + u + v == 0) {
                                val = q_ipow(g ? 2 * q : -2 * q, n) * aux[n];
                            } else {
                                int dt = 0, du = 0, dv = 0, k;
                                qr X;
                                if (t + u == 0) { dv = 1; k = v; X = QC[2]; }
                                else if (t == 0) { du = 1; k = u; X = QC[1]; }
                                else { dt = 1; k = t; X = QC[0]; }
                                qr r2n1 = 0, r2n = 0;
                                if (k > 1) {
                                    r2n1 = R[RI(t - 2 * dt, u - 2 * du, v - 2 * dv, n + 1)];
                                    r2n = R[RI(t - 2 * dt, u - 2 * du, v - 2 * dv, n)];
                                }
                                qr r1n1 = R[RI(t - dt, u - du, v - dv, n + 1)], r1n = R[RI(t - dt, u - du, v - dv, n)];
                                if (g) {
                                    if (k > 1) val += (k - 1) * (r2n1 - 2 * q * r2n);
                                    val += X * (r1n1 - 2 * q * r1n);
                                } else {
                                    if (k > 1) val += (k - 1) * r2n1;
                                    val += X * r1n1;
                                }
                            }
                            R[RI(t, u, v, n)] = val;
                        }
            qr pf = g ? w * 2 * powq(M_PIq, 1.5Q) / sqrtq(q) : w * 2 * M_PIq / q;
            for (int m = 0; m < nA; m++)
                for (int n = 0; n < nB; n++) {
                    const int *ca = A->cart + 3 * m, *cb = B->cart + 3 * n;
                    qr s = 0;
                    for (int t = 0; t <= ca[0] + cb[0]; t++)
                        for (int u = 0; u <= ca[1] + cb[1]; u++)
                            for (int v = 0; v <= ca[2] + cb[2]; v++)
                                s += E[EI(0, ca[0], cb[0], t)] * E[EI(1, ca[1], cb[1], u)] * E[EI(2, ca[2], cb[2], v)] *
                                     R[RI(t, u, v, 0)];
                    out[m * nB + n] += pf * s;
                }
        }
#undef EI
#undef RI
    free(E);
    free(R);
}

static void q_type1(const q_shell_t *A, const q_shell_t *B, const qr *C, const q_pot_t *P, qr *out)
{
    for (int k = 0; k < P->n; k++) q_type1_term(A, B, C, P->z[k], P->pw[k], P->c[k], out);
}

/* Obara-Saika overlap <A|B> of two contracted shells, added to out */
static void q_overlap(const q_shell_t *A, const q_shell_t *B, qr *out)
{
    int la = A->L, lb = B->L, nA = ncart(la), nB = ncart(lb);
    for (int i = 0; i < A->n; i++)
        for (int j = 0; j < B->n; j++) {
            qr a = A->a[i], b = B->a[j], p = a + b, mu = a * b / p, S[3][16][16];
            for (int x = 0; x < 3; x++) {
                qr P = (a * A->o[x] + b * B->o[x]) / p, xab = A->o[x] - B->o[x], xpa = P - A->o[x], xpb = P - B->o[x];
                qr pf = 1 / (2 * p);
                for (int ii = 0; ii <= la; ii++)
                    for (int jj = 0; jj <= lb; jj++) {
                        qr s = 0;
                        if (ii + jj == 0) s = sqrtq(M_PIq / p) * expq(-mu * xab * xab);
                        else if (ii == 0) {
                            s = xpb * S[x][0][jj - 1];
                            if (jj > 1) s += (jj - 1) * pf * S[x][0][jj - 2];
                        } else {
                            s = xpa * S[x][ii - 1][jj];
                            if (ii > 1) s += (ii - 1) * pf * S[x][ii - 2][jj];
                            if (jj > 0) s += jj * pf * S[x][ii - 1][jj - 1];
                        }
                        S[x][ii][jj] = s;
                    }
            }
            qr w = A->c[i] * B->c[j] * q_gnorm(la, a) * q_gnorm(lb, b);
            for (int m = 0; m < nA; m++)
                for (int n = 0; n < nB; n++) {
                    const int *ca = A->cart + 3 * m, *cb = B->cart + 3 * n;
                    out[m * nB + n] += w * S[0][ca[0]][cb[0]] * S[1][ca[1]][cb[1]] * S[2][ca[2]][cb[2]];
                }
        }
}

/* ============================================================ radial tables */

typedef struct {
    int l1max, l2max, nmax, npot;
    int ne;                /* entries listed */
    int (*ent)[4];         /* (pot, lambda1, lambda2, N) */
    qr *val;               /* converged integrals */
    int level;             /* deepest level used */
    double resid;          /* last change between levels / sum of |terms| (worst entry) */
} q_radial_t;

/* F_l(r) = sum_i c_i N_i exp(-a_i (r - CA)^2) M_l(2 a_i CA r), l = 0..lmax */
static void q_radial_shell(const q_shell_t *S, qr CA, qr r, int lmax, qr *F)
{
    qr M[TQ_LMAX + 3];
    for (int l = 0; l <= lmax; l++) F[l] = 0;
    for (int i = 0; i < S->n; i++) {
        qr a = S->a[i], e = a * (r - CA) * (r - CA);
        if (e > 160) continue; /* exp < 3e-70: below anything that can reach an output */
        qr g = S->c[i] * q_gnorm(S->L, a) * expq(-e);
        q_bessel(lmax, 2 * a * CA * r, M);
        for (int l = 0; l <= lmax; l++) F[l] += g * M[l];
    }
}

static qr q_pot_value(const q_pot_t *P, qr r)
{
    qr u = 0;
    for (int k = 0; k < P->n; k++) u += P->c[k] * q_ipow(r, P->pw[k]) / (r * r) * expq(-P->z[k] * r * r);
    return u;
}

/* integrals int_0^inf r^2 U_p(r) F^A_l1(r) F^B_l2(r) r^N dr of the listed entries */
static void q_radial(const q_shell_t *A, const q_shell_t *B, qr CA, qr CB, const q_pot_t *const *pots, q_radial_t *T)
{
    int ne = T->ne;
    qr *raw = calloc(ne > 0 ? ne : 1, sizeof(qr)), *prev = calloc(ne > 0 ? ne : 1, sizeof(qr));
    qr *mag = calloc(ne > 0 ? ne : 1, sizeof(qr)); /* sums of |terms|: the scale of each integral's rounding */
    qr (*rich)[TQ_RICH_K + 1] = calloc(ne > 0 ? ne : 1, sizeof(qr[TQ_RICH_K + 1])); /* previous Richardson row */
    T->level = 0;
    T->resid = 0;
    if (CA == 0 && CB == 0) {
        /* one centre: only lambda1 = lambda2 = 0, analytic radial integrals */
        for (int e = 0; e < ne; e++) {
            const int *en = T->ent[e];
            qr s = 0;
            if (en[1] == 0 && en[2] == 0) {
                const q_pot_t *P = pots[en[0]];
                for (int i = 0; i < A->n; i++)
                    for (int j = 0; j < B->n; j++)
                        for (int k = 0; k < P->n; k++)
                            s += A->c[i] * q_gnorm(A->L, A->a[i]) * B->c[j] * q_gnorm(B->L, B->a[j]) * P->c[k] *
                                 q_gauss_int(P->pw[k] + en[3], A->a[i] + B->a[j] + P->z[k]);
            }
            T->val[e] = s;
        }
        free(raw);
        free(prev);
        free(mag);
        free(rich);
        return;
    }
    const qr R = 5, R3 = R * R * R;
    qr F1[TQ_LMAX + 3], F2[TQ_LMAX + 3], U[64], rN[32];
    int conv_streak = 0;
    for (int level = 0; level <= TQ_LEVEL_MAX; level++) {
        int64_t den = (int64_t)1 << (level + 5); /* x = i / den, nr = den - 1 points */
        for (int64_t i = 1; i < den; i++) {
            if (level > 0 && (i % 2) == 0) continue; /* points of coarser levels */
            qr x = (qr)i / den, x3 = x * x * x, ln = logq(1 - x3);
            qr r = -R * ln, om = 3 * R3 * x * x * ln * ln / (1 - x3); /* weight without 1/(nr+1) */
            q_radial_shell(A, CA, r, T->l1max, F1);
            q_radial_shell(B, CB, r, T->l2max, F2);
            for (int p = 0; p < T->npot; p++) U[p] = om * q_pot_value(pots[p], r);
            rN[0] = 1;
            for (int n = 1; n <= T->nmax; n++) rN[n] = rN[n - 1] * r;
            for (int e = 0; e < ne; e++) {
                const int *en = T->ent[e];
                qr v = U[en[0]] * F1[en[1]] * F2[en[2]] * rN[en[3]];
                raw[e] += v;
                mag[e] += fabsq(v);
            }
        }
        /* S_level = raw / den. Near r = 0 the integrand in x is x^2 g(x^3) (r = 5 x^3 (1 + x^3/2 + ...),
         * potential terms r^(n-2), n >= 0), so the nested rule's error has only the
         * Euler-Maclaurin terms of the odd powers x^5, x^11, x^17, ...: h^6, h^12, h^18, ...
         * (the decay at x -> 1 adds none). Richardson elimination of those orders: row k of the
         * table at this level removes h^6 ... h^(6k). */
        int all = 1;
        double worst = 0;
        int kmax = level - TQ_RICH_START;
        if (kmax > TQ_RICH_K) kmax = TQ_RICH_K;
        for (int e = 0; e < ne; e++) {
            qr row[TQ_RICH_K + 1];
            row[0] = raw[e] / den;
            for (int k = 1; k <= kmax; k++) {
                qr f = q_ipow(64, k);
                row[k] = row[k - 1] + (row[k - 1] - rich[e][k - 1]) / (f - 1);
            }
            qr best = kmax >= 0 ? row[kmax] : row[0];
            if (level >= TQ_LEVEL_MIN && kmax >= 1) {
                qr d = fabsq(best - prev[e]);
                if (!(d <= 1e-30Q * mag[e] / den || d <= 1e-60Q)) all = 0;
                if (mag[e] > 0 && d > 1e-60Q && (double)(d / (mag[e] / den)) > worst) worst = (double)(d / (mag[e] / den));
            } else {
                all = 0;
            }
            prev[e] = best;
            for (int k = 0; k <= TQ_RICH_K; k++) rich[e][k] = (k <= (kmax > 0 ? kmax : 0)) ? row[k] : 0;
        }
        T->level = level;
        T->resid = worst;
        conv_streak = all ? conv_streak + 1 : 0;
        if (conv_streak >= 2) break;
    }
    for (int e = 0; e < ne; e++) T->val[e] = prev[e];
    free(raw);
    free(prev);
    free(mag);
    free(rich);
}

/* ============================================================ type 2 and spin-orbit */

/* entries (lambda1, lambda2, N) the angular sums read for projector L and shells la, lb */
static int q_needed(int L, int la, int lb, int l1, int l2, int N)
{
    for (int n1 = 0; n1 <= la; n1++) {
        int n2 = N - n1;
        if (n2 < 0 || n2 > lb) continue;
        if (l1 < L - n1 || l1 > L + n1 || (L + n1 - l1) % 2) continue;
        if (l2 < L - n2 || l2 > L + n2 || (L + n2 - l2) % 2) continue;
        return 1;
    }
    return 0;
}

/* semilocal potentials pots[0..npot): type 2 (so[p] = 0) into arep, or spin-orbit (so[p] = 1)
 * into sx, sy, sz, each scaled by scale[p] */
static void q_semilocal(const q_shell_t *A, const q_shell_t *B, const qr *C, const q_pot_t *const *pots, const int *so,
                        const qr *scale, int npot, qr *arep, qr *sx, qr *sy, qr *sz, int *level_out, double *resid_out)
{
    if (npot == 0) return;
    int la = A->L, lb = B->L, nA = ncart(la), nB = ncart(lb);
    qr CAv[3], CBv[3], uA[3] = {0, 0, 0}, uB[3] = {0, 0, 0};
    for (int x = 0; x < 3; x++) {
        CAv[x] = C[x] - A->o[x];
        CBv[x] = C[x] - B->o[x];
    }
    qr CA = sqrtq(CAv[0] * CAv[0] + CAv[1] * CAv[1] + CAv[2] * CAv[2]);
    qr CB = sqrtq(CBv[0] * CBv[0] + CBv[1] * CBv[1] + CBv[2] * CBv[2]);
    for (int x = 0; x < 3; x++) {
        if (CA > 0) uA[x] = -CAv[x] / CA; /* direction of k_A = -2 a (C - A) */
        if (CB > 0) uB[x] = -CBv[x] / CB;
    }
    int Lmax = 0;
    for (int p = 0; p < npot; p++) Lmax = pots[p]->L > Lmax ? pots[p]->L : Lmax;
    q_radial_t T;
    memset(&T, 0, sizeof(T));
    T.l1max = Lmax + la;
    T.l2max = Lmax + lb;
    T.nmax = la + lb;
    T.npot = npot;
    int d1 = T.l1max + 1, d2 = T.l2max + 1, dn = T.nmax + 1;
    int *map = malloc(sizeof(int) * npot * d1 * d2 * dn);
    T.ent = malloc(sizeof(int[4]) * npot * d1 * d2 * dn);
    for (int p = 0; p < npot; p++)
        for (int l1 = 0; l1 < d1; l1++)
            for (int l2 = 0; l2 < d2; l2++)
                for (int n = 0; n < dn; n++) {
                    int id = ((p * d1 + l1) * d2 + l2) * dn + n;
                    map[id] = -1;
                    if (q_needed(pots[p]->L, la, lb, l1, l2, n)) {
                        map[id] = T.ne;
                        T.ent[T.ne][0] = p;
                        T.ent[T.ne][1] = l1;
                        T.ent[T.ne][2] = l2;
                        T.ent[T.ne][3] = n;
                        T.ne++;
                    }
                }
    T.val = calloc(T.ne > 0 ? T.ne : 1, sizeof(qr));
    q_radial(A, B, CA, CB, pots, &T);
    if (T.level > *level_out) *level_out = T.level;
    if (T.resid > *resid_out) *resid_out = T.resid;

    int lam = Lmax + (la > lb ? la : lb);
    qr *rA = calloc((lam + 1) * (2 * lam + 1), sizeof(qr)), *rB = calloc((lam + 1) * (2 * lam + 1), sizeof(qr));
    for (int l = 0; l <= lam; l++) {
        q_rsh_values(l, uA, rA + l * (2 * lam + 1));
        q_rsh_values(l, uB, rB + l * (2 * lam + 1));
    }
    for (int p = 0; p < npot; p++) {
        int L = pots[p]->L, dim = 2 * L + 1;
        qr *Lm[3] = {0, 0, 0};
        if (so[p]) {
            for (int c = 0; c < 3; c++) Lm[c] = calloc(dim * dim, sizeof(qr));
            q_lmatrices(L, Lm[0], Lm[1], Lm[2]);
        }
        /* omega tables of both sides: [lambda][a][b][c][m], a + b + c <= l_shell */
        int dA = la + 1, dB = lb + 1, l1m = L + la, l2m = L + lb;
        qr *WA = calloc((size_t)(l1m + 1) * dA * dA * dA * dim, sizeof(qr));
        qr *WB = calloc((size_t)(l2m + 1) * dB * dB * dB * dim, sizeof(qr));
#define WAI(l, a, b, c, m) (((((l) * dA + (a)) * dA + (b)) * dA + (c)) * dim + (m))
#define WBI(l, a, b, c, m) (((((l) * dB + (a)) * dB + (b)) * dB + (c)) * dim + (m))
        for (int a = 0; a <= la; a++)
            for (int bq = 0; a + bq <= la; bq++)
                for (int c = 0; a + bq + c <= la; c++)
                    for (int l1 = 0; l1 <= l1m; l1++)
                        for (int m = -L; m <= L; m++)
                            WA[WAI(l1, a, bq, c, m + L)] = q_omega(l1, L, m, a, bq, c, rA + l1 * (2 * lam + 1));
        for (int a = 0; a <= lb; a++)
            for (int bq = 0; a + bq <= lb; bq++)
                for (int c = 0; a + bq + c <= lb; c++)
                    for (int l2 = 0; l2 <= l2m; l2++)
                        for (int m = -L; m <= L; m++)
                            WB[WBI(l2, a, bq, c, m + L)] = q_omega(l2, L, m, a, bq, c, rB + l2 * (2 * lam + 1));
        for (int ic = 0; ic < nA; ic++)
            for (int jc = 0; jc < nB; jc++) {
                const int *ca = A->cart + 3 * ic, *cb = B->cart + 3 * jc;
                qr acc[3] = {0, 0, 0};
                for (int a = 0; a <= ca[0]; a++)
                    for (int bq = 0; bq <= ca[1]; bq++)
                        for (int c = 0; c <= ca[2]; c++)
                            for (int d = 0; d <= cb[0]; d++)
                                for (int e = 0; e <= cb[1]; e++)
                                    for (int f = 0; f <= cb[2]; f++) {
                                        qr factor = q_binom(ca[0], a) * q_binom(ca[1], bq) * q_binom(ca[2], c) *
                                                    q_binom(cb[0], d) * q_binom(cb[1], e) * q_binom(cb[2], f) *
                                                    q_ipow(CAv[0], ca[0] - a) * q_ipow(CAv[1], ca[1] - bq) *
                                                    q_ipow(CAv[2], ca[2] - c) * q_ipow(CBv[0], cb[0] - d) *
                                                    q_ipow(CBv[1], cb[1] - e) * q_ipow(CBv[2], cb[2] - f);
                                        if (factor == 0) continue;
                                        int nabc = a + bq + c, ndef = d + e + f, N = nabc + ndef;
                                        qr s[3] = {0, 0, 0};
                                        for (int l1 = (L - nabc > 0 ? L - nabc : 0); l1 <= L + nabc; l1++) {
                                            if ((L + nabc - l1) % 2) continue;
                                            for (int l2 = (L - ndef > 0 ? L - ndef : 0); l2 <= L + ndef; l2++) {
                                                if ((L + ndef - l2) % 2) continue;
                                                int id = map[((p * d1 + l1) * d2 + l2) * dn + N];
                                                qr QN = T.val[id];
                                                if (QN == 0) continue;
                                                const qr *w1 = WA + WAI(l1, a, bq, c, 0), *w2 = WB + WBI(l2, d, e, f, 0);
                                                if (!so[p]) {
                                                    qr ang = 0;
                                                    for (int m = 0; m < dim; m++) ang += w1[m] * w2[m];
                                                    s[0] += QN * ang;
                                                } else {
                                                    qr ax = 0, ay = 0, az = 0;
                                                    for (int m1 = 0; m1 < dim; m1++)
                                                        for (int m2 = 0; m2 < dim; m2++) {
                                                            qr ww = w1[m1] * w2[m2];
                                                            ax += ww * Lm[0][m1 * dim + m2];
                                                            ay += ww * Lm[1][m1 * dim + m2];
                                                            az += ww * Lm[2][m1 * dim + m2];
                                                        }
                                                    s[0] += QN * ax;
                                                    s[1] += QN * ay;
                                                    s[2] += QN * az;
                                                }
                                            }
                                        }
                                        for (int k = 0; k < 3; k++) acc[k] += factor * s[k];
                                    }
                qr f16 = 16 * M_PIq * M_PIq * scale[p];
#undef WAI
#undef WBI
                if (!so[p]) arep[ic * nB + jc] += acc[0] * f16;
                else {
                    sx[ic * nB + jc] += acc[0] * f16;
                    sy[ic * nB + jc] += acc[1] * f16;
                    sz[ic * nB + jc] += acc[2] * f16;
                }
            }
        for (int c = 0; c < 3; c++) free(Lm[c]);
        free(WA);
        free(WB);
    }
    free(rA);
    free(rB);
    free(map);
    free(T.ent);
    free(T.val);
}

/* ============================================================ outercore */

static qr q_radial_gto_norm(int L, qr a)
{
    qr g = DF(2 * L + 1) * sqrtq(M_PIq) / q_ipow(2, L + 1); /* Gamma(L + 3/2) */
    return sqrtq(powq(2, L + 2.5Q) / g) * powq(a, 0.75Q + L / 2.0Q);
}

static qr q_one_centre_prim(int L, qr a1, qr a2, int n, qr zeta)
{
    qr a = a1 + a2 + zeta;
    if (n % 2 == 0) {
        int k = L + n / 2;
        return DF(2 * k - 1) / (q_ipow(2, k + 1) * q_ipow(a, k)) * sqrtq(M_PIq / a);
    }
    int k = L + (n - 1) / 2;
    return q_fact[k] / (2 * q_ipow(a, k + 1));
}

static qr q_one_centre(const q_shell_t *s1, const q_shell_t *s2, const q_pot_t *P)
{
    qr sum = 0;
    int L = P->L;
    for (int i = 0; i < s1->n; i++)
        for (int j = 0; j < s2->n; j++) {
            qr f = q_radial_gto_norm(L, s1->a[i]) * q_radial_gto_norm(L, s2->a[j]) * s1->c[i] * s2->c[j];
            for (int k = 0; k < P->n; k++) sum += f * P->c[k] * q_one_centre_prim(L, s1->a[i], s2->a[j], P->pw[k], P->z[k]);
        }
    return sum;
}

/* S[(m + L) * ncart + ic]: Cartesian -> real spherical coefficients of an oc shell */
static void q_oc_sph(const q_shell_t *oc, qr *S)
{
    int L = oc->L, n = ncart(L);
    for (int m = -L; m <= L; m++)
        for (int ic = 0; ic < n; ic++) {
            const int *c = oc->cart + 3 * ic;
            qr an = sqrtq(DF(2 * L + 1)) / (2 * sqrtq(M_PIq));
            S[n * (m + L) + ic] = q_sph_coef(L, m, c[0], c[1], c[2]) / an;
        }
}

/* out[i][m] = sum_c S[m][c] in[i][c] (ket side); out[m][j] = sum_c S[m][c] in[c][j] (bra side) */
static void q_sph_ket(int na, int nc, int d, const qr *in, const qr *S, qr *out)
{
    for (int i = 0; i < na; i++)
        for (int m = 0; m < d; m++) {
            qr s = 0;
            for (int c = 0; c < nc; c++) s += S[nc * m + c] * in[i * nc + c];
            out[i * d + m] = s;
        }
}
static void q_sph_bra(int nc, int d, int nb, const qr *in, const qr *S, qr *out)
{
    for (int j = 0; j < nb; j++)
        for (int m = 0; m < d; m++) {
            qr s = 0;
            for (int c = 0; c < nc; c++) s += S[nc * m + c] * in[c * nb + j];
            out[m * nb + j] = s;
        }
}

static void q_outercore(const q_shell_t *A, const q_shell_t *B, const qr *C, int noc, const q_pot_t *const *pots,
                        q_shell_t *const *ocs, qr *arep, qr *sx, qr *sy, qr *sz)
{
    int nA = ncart(A->L), nB = ncart(B->L);
    qr *outs[3] = {sx, sy, sz};
    /* part 1 */
    for (int i = 0; i < noc; i++) {
        const q_pot_t *P = pots[i];
        q_shell_t oc = *ocs[i];
        for (int x = 0; x < 3; x++) oc.o[x] = C[x];
        int L = oc.L, no = ncart(L), d = 2 * L + 1;
        qr J = P->J / 2.0Q;
        qr *Sc = calloc(d * no, sizeof(qr)), *t1 = calloc(no * nB, sizeof(qr)), *t2 = calloc(nA * no, sizeof(qr));
        qr *S_a = calloc(nA * d, sizeof(qr)), *S_b = calloc(d * nB, sizeof(qr)), *U_a = calloc(nA * d, sizeof(qr)),
           *U_b = calloc(d * nB, sizeof(qr));
        q_oc_sph(&oc, Sc);
        q_overlap(&oc, B, t1);
        q_overlap(A, &oc, t2);
        q_sph_ket(nA, no, d, t2, Sc, S_a);
        q_sph_bra(no, d, nB, t1, Sc, S_b);
        memset(t1, 0, no * nB * sizeof(qr));
        memset(t2, 0, nA * no * sizeof(qr));
        q_type1(&oc, B, C, P, t1);
        q_type1(A, &oc, C, P, t2);
        q_sph_ket(nA, no, d, t2, Sc, U_a);
        q_sph_bra(no, d, nB, t1, Sc, U_b);
        qr farep = (J < L) ? (qr)L / (2 * L + 1) : (qr)(L + 1) / (2 * L + 1);
        qr fso = (J < L) ? -2.0Q / (2 * L + 1) : 2.0Q / (2 * L + 1);
        qr *Lm[3];
        for (int c = 0; c < 3; c++) Lm[c] = calloc(d * d, sizeof(qr));
        q_lmatrices(L, Lm[0], Lm[1], Lm[2]);
        for (int a = 0; a < nA; a++)
            for (int b = 0; b < nB; b++) {
                qr s = 0;
                for (int m = 0; m < d; m++) s += S_a[a * d + m] * U_b[m * nB + b] + U_a[a * d + m] * S_b[m * nB + b];
                arep[a * nB + b] += farep * s;
                for (int c = 0; c < 3; c++) {
                    qr v = 0;
                    for (int m1 = 0; m1 < d; m1++)
                        for (int m2 = 0; m2 < d; m2++)
                            v += (U_a[a * d + m1] * S_b[m2 * nB + b] + S_a[a * d + m1] * U_b[m2 * nB + b]) * Lm[c][m1 * d + m2];
                    outs[c][a * nB + b] += fso * v;
                }
            }
        for (int c = 0; c < 3; c++) free(Lm[c]);
        free(Sc); free(t1); free(t2); free(S_a); free(S_b); free(U_a); free(U_b);
    }
    /* part 2 */
    for (int i = 0; i < noc; i++)
        for (int j = 0; j < noc; j++) {
            const q_pot_t *P1 = pots[i], *P2 = pots[j];
            if (P1->L != P2->L || P1->J != P2->J) continue;
            q_shell_t o1 = *ocs[i], o2 = *ocs[j];
            for (int x = 0; x < 3; x++) o1.o[x] = o2.o[x] = C[x];
            int L = P1->L, no = ncart(L), d = 2 * L + 1;
            qr J = P1->J / 2.0Q;
            qr delta = 0.5Q * (q_one_centre(&o1, &o2, P1) + q_one_centre(&o1, &o2, P2));
            qr *Sc = calloc(d * no, sizeof(qr)), *t1 = calloc(no * nB, sizeof(qr)), *t2 = calloc(nA * no, sizeof(qr));
            qr *S_a = calloc(nA * d, sizeof(qr)), *S_b = calloc(d * nB, sizeof(qr));
            q_oc_sph(&o1, Sc);
            q_overlap(&o2, B, t1);
            q_overlap(A, &o1, t2);
            q_sph_ket(nA, no, d, t2, Sc, S_a);
            q_sph_bra(no, d, nB, t1, Sc, S_b);
            qr farep = (J < L) ? (qr)L / (2 * L + 1) : (qr)(L + 1) / (2 * L + 1);
            qr fso = (J < L) ? -2.0Q / (2 * L + 1) : 2.0Q / (2 * L + 1);
            qr *Lm[3];
            for (int c = 0; c < 3; c++) Lm[c] = calloc(d * d, sizeof(qr));
            q_lmatrices(L, Lm[0], Lm[1], Lm[2]);
            for (int a = 0; a < nA; a++)
                for (int b = 0; b < nB; b++) {
                    qr s = 0;
                    for (int m = 0; m < d; m++) s += S_a[a * d + m] * S_b[m * nB + b];
                    arep[a * nB + b] -= delta * farep * s;
                    for (int c = 0; c < 3; c++) {
                        qr v = 0;
                        for (int m1 = 0; m1 < d; m1++)
                            for (int m2 = 0; m2 < d; m2++) v += S_a[a * d + m1] * S_b[m2 * nB + b] * Lm[c][m1 * d + m2];
                        outs[c][a * nB + b] -= delta * fso * v;
                    }
                }
            for (int c = 0; c < 3; c++) free(Lm[c]);
            free(Sc); free(t1); free(t2); free(S_a); free(S_b);
        }
}

/* ============================================================ batch driver */

static void q_task(const libgrpp_b200_batch_t *b, int64_t t, qr *arep, qr *sx, qr *sy, qr *sz, int *level, double *resid)
{
    q_shell_t *A = malloc(sizeof(q_shell_t)), *B = malloc(sizeof(q_shell_t));
    q_shell(b, b->task_a[t], A);
    q_shell(b, b->task_b[t], B);
    int c = b->task_c[t], g = b->centre_grpp[c];
    qr C[3] = {b->centre_origin[3 * c], b->centre_origin[3 * c + 1], b->centre_origin[3 * c + 2]};
    if (b->grpp_UL[g] >= 0) {
        q_pot_t P;
        q_pot(b, b->grpp_UL[g], &P);
        q_type1(A, B, C, &P, arep);
    }
    int na = b->grpp_n_arep[g], ns = b->grpp_n_so[g], np = na + ns;
    q_pot_t *P = malloc(sizeof(q_pot_t) * (np > 0 ? np : 1));
    const q_pot_t **pp = malloc(sizeof(void *) * (np > 0 ? np : 1));
    int *so = malloc(sizeof(int) * (np > 0 ? np : 1));
    qr *scale = malloc(sizeof(qr) * (np > 0 ? np : 1));
    for (int i = 0; i < na; i++) {
        q_pot(b, b->grpp_pot_list[b->grpp_arep_off[g] + i], &P[i]);
        so[i] = 0;
        scale[i] = 1;
    }
    for (int i = 0; i < ns; i++) {
        q_pot(b, b->grpp_pot_list[b->grpp_so_off[g] + i], &P[na + i]);
        so[na + i] = 1;
        scale[na + i] = 2.0Q / (2 * P[na + i].L + 1);
    }
    for (int i = 0; i < np; i++) pp[i] = &P[i];
    q_semilocal(A, B, C, pp, so, scale, np, arep, sx, sy, sz, level, resid);
    int noc = b->grpp_n_oc[g];
    if (noc > 0) {
        q_pot_t *op = malloc(sizeof(q_pot_t) * noc);
        q_shell_t *os = malloc(sizeof(q_shell_t) * noc);
        const q_pot_t **opp = malloc(sizeof(void *) * noc);
        q_shell_t **osp = malloc(sizeof(void *) * noc);
        for (int i = 0; i < noc; i++) {
            int k = b->grpp_oc_off[g] + i;
            q_pot(b, b->grpp_oc_pot[k], &op[i]);
            q_shell(b, b->grpp_oc_shell[k], &os[i]);
            opp[i] = &op[i];
            osp[i] = &os[i];
        }
        q_outercore(A, B, C, noc, opp, osp, arep, sx, sy, sz);
        free(op); free(os); free(opp); free(osp);
    }
    free(P); free(pp); free(so); free(scale);
    free(A);
    free(B);
}

static void q_global_init(void)
{
    static int done = 0;
#ifdef _OPENMP
#pragma omp critical(truth_init)
#endif
    {
        if (!done) {
            q_init();
            q_rsh_init();
            done = 1;
        }
    }
}

/* Full GRPP blocks (arep, so_x, so_y, so_z) of tasks t0..t1-1, laid out as the batched
 * entry point lays them out (task by task, row-major cart(A) x cart(B)), rounded to
 * double. level[t - t0] receives the deepest radial grid level used (0 = 31 points)
 * and resid[t - t0] the largest final change between levels of the task's radial
 * integrals relative to the sum of the absolute values of their terms (below 1e-30
 * when every integral converged; NULL to skip either). Returns 0. */
int truth_full_batch(const libgrpp_b200_batch_t *b, int64_t t0, int64_t t1, int nthreads, double *arep, double *sx,
                     double *sy, double *sz, int *level, double *resid)
{
    q_global_init();
    int64_t n = t1 - t0;
    int64_t *off = malloc(sizeof(int64_t) * (n + 1));
    off[0] = 0;
    for (int64_t t = 0; t < n; t++)
        off[t + 1] = off[t] + (int64_t)ncart(b->shell_L[b->task_a[t0 + t]]) * ncart(b->shell_L[b->task_b[t0 + t]]);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int64_t t = 0; t < n; t++) {
        int m = (int)(off[t + 1] - off[t]), lev = 0;
        double res = 0;
        qr *o = calloc(4 * (size_t)m, sizeof(qr));
        q_task(b, t0 + t, o, o + m, o + 2 * m, o + 3 * m, &lev, &res);
        for (int i = 0; i < m; i++) {
            arep[off[t] + i] = (double)o[i];
            sx[off[t] + i] = (double)o[m + i];
            sy[off[t] + i] = (double)o[2 * m + i];
            sz[off[t] + i] = (double)o[3 * m + i];
        }
        if (level) level[t] = lev;
        if (resid) resid[t] = res;
        free(o);
    }
    free(off);
    return 0;
}

/* special functions in binary128, rounded to double (for the tests of this file) */
double truth_boys(int n, double x)
{
    q_init();
    qr F[64];
    q_boys(n, x, F);
    return (double)F[n];
}
double truth_gfun(int n, double x)
{
    q_init();
    qr G[64];
    q_gfun(n, x, G);
    return (double)G[n];
}
double truth_bessel_scaled(int l, double x)
{
    q_init();
    qr M[TQ_LMAX + 3];
    q_bessel(l, x, M);
    return (double)M[l];
}
