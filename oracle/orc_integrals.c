/*
 * ORACLE — test infrastructure only (see orc_common.h).
 *
 * CPU restatement of libgrpp's GRPP integral path. Every function names the
 * reference file:line it follows. The exported libgrpp_* symbols make this
 * library a CPU drop-in with the reference's C API, so tests drive the
 * oracle, the compiled reference and the CUDA product through one binding.
 */
#include "orc_common.h"

#include <assert.h>
#include <math.h>
#include <stdio.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

orc_stats_t orc_stats;

/* ================================================================ parameters
 * parameters.c:17-134 */
static int gen_dirac(int L, int *cl)
{
    int c = 0;
    for (int r = L; r >= 0; r--)
        for (int s = L; s >= 0; s--)
            for (int t = L; t >= 0; t--)
                if (r + s + t == L) {
                    cl[3 * c] = r;
                    cl[3 * c + 1] = s;
                    cl[3 * c + 2] = t;
                    c++;
                }
    return (L + 1) * (L + 2) / 2;
}

static int gen_turbomole(int L, int *cl)
{
    int c = 0;
    for (int r = L; r >= 0; r--)
        for (int s = L - r; s >= 0; s--) {
            cl[3 * c] = r;
            cl[3 * c + 1] = s;
            cl[3 * c + 2] = L - r - s;
            c++;
        }
    return (L + 1) * (L + 2) / 2;
}

libgrpp_parameters_t libgrpp_params = {1e-16, 1e-16, 1e-16, gen_dirac};

void libgrpp_set_radial_tolerance(double t) { libgrpp_params.radial_tolerance = t; }
void libgrpp_set_angular_screening_tolerance(double t) { libgrpp_params.angular_screening_tolerance = t; }
void libgrpp_set_modified_bessel_tolerance(double t) { libgrpp_params.modified_bessel_tolerance = t; }
void libgrpp_set_cartesian_generator(int (*g)(int, int *)) { libgrpp_params.cartesian_generator = g; }
void libgrpp_set_cartesian_order(int order)
{
    assert(order == LIBGRPP_CART_ORDER_DIRAC || order == LIBGRPP_CART_ORDER_TURBOMOLE);
    libgrpp_params.cartesian_generator = order == LIBGRPP_CART_ORDER_DIRAC ? gen_dirac : gen_turbomole;
}
void libgrpp_set_default_parameters(void)
{
    libgrpp_params.radial_tolerance = 1e-16;
    libgrpp_params.angular_screening_tolerance = 1e-16;
    libgrpp_params.modified_bessel_tolerance = 1e-16;
    libgrpp_params.cartesian_generator = gen_dirac;
}

/* init_finalize.c:19-50 */
static int orc_initialized = 0;
void libgrpp_init(void)
{
    if (!orc_initialized) {
        orc_tables_init();
        orc_rsh_ncomb(0);
        orc_initialized = 1;
    }
}
void libgrpp_finalize(void) { orc_initialized = 0; }
int libgrpp_is_initialized(void) { return orc_initialized; }

/* ================================================================ containers */

/* potential.c:22-46: terms with |c| < 1e-14 are dropped */
libgrpp_potential_t *libgrpp_new_potential(int L, int J, int n, int *powers, double *coeffs, double *alpha)
{
    libgrpp_potential_t *p = calloc(1, sizeof(*p));
    p->L = L;
    p->J = J;
    p->powers = calloc(n > 0 ? n : 1, sizeof(int));
    p->coeffs = calloc(n > 0 ? n : 1, sizeof(double));
    p->alpha = calloc(n > 0 ? n : 1, sizeof(double));
    for (int i = 0; i < n; i++) {
        if (fabs(coeffs[i]) < LIBGRPP_ZERO_THRESH) continue;
        p->coeffs[p->num_primitives] = coeffs[i];
        p->powers[p->num_primitives] = powers[i];
        p->alpha[p->num_primitives] = alpha[i];
        p->num_primitives++;
    }
    return p;
}

void libgrpp_delete_potential(libgrpp_potential_t *p)
{
    if (!p) return;
    free(p->powers);
    free(p->coeffs);
    free(p->alpha);
    free(p);
}

/* Rounding model (test infrastructure, off by default). With a nonzero seed, the results of the
 * transcendental calls of the type 2 radial path -- exp and pow of the potential and of the
 * contracted integrands, log of the grid, pow of r^N, the scaled Bessel values and the screening
 * estimate -- are moved by -1, 0 or +1 unit in the last place, chosen by a hash of the seed, the
 * call site and the argument (so a run does not depend on the thread schedule). Such a run stands
 * for another implementation of libgrpp's algorithm whose math library and tables differ from
 * libgrpp's in the last bit, which is what a GPU implementation is; the spread of a few runs
 * measures how closely libgrpp's double-precision arithmetic determines each element. */
static uint64_t rm_seed = 0;

void orc_set_rounding_model(uint64_t seed) { rm_seed = seed; }

static double rm(double x, uint64_t site)
{
    if (!rm_seed || x == 0.0 || !isfinite(x)) return x;
    uint64_t h, b;
    memcpy(&b, &x, sizeof b);
    h = rm_seed * 0x9E3779B97F4A7C15ull ^ (b + 0x632BE59BD9B4E019ull * (site + 1));
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 29;
    h *= 0x94D049BB133111EBull;
    h ^= h >> 32;
    switch (h % 3) {
    case 0: return nextafter(x, -INFINITY);
    case 1: return nextafter(x, INFINITY);
    default: return x;
    }
}

/* Rounding model, stop decisions: with a nonzero seed, the convergence test |S_L - S_{L-1}| <= tol
 * of a radial integral is taken on a difference moved by k units in the last place of S_L,
 * k in [-64, 64] from a hash of the seed, the level and the sum (radial_type2_integral.c:305-310).
 * An implementation whose sums differ from libgrpp's in the last bits (the GPU engine's differ
 * from this restatement's by 59 ulps at the median and up to 68 on the sums that stop at the same
 * level, KCs g x f shells with the Cs potential) stops some entries at another level where
 * |S_L - S_{L-1}| is within that many ulps of the tolerance. */
static double rm_conv_diff(double sum, double prev, int level)
{
    const double d = fabs(sum - prev);
    if (!rm_seed) return d;
    uint64_t b, h;
    memcpy(&b, &sum, sizeof b);
    h = rm_seed * 0x9E3779B97F4A7C15ull ^ (b + 0xD1B54A32D192ED03ull * (uint64_t)(level + 17));
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 29;
    const int k = (int)(h % 129) - 64;
    const double ulp = nextafter(fabs(sum), INFINITY) - fabs(sum);
    return fabs(d + k * ulp);
}

/* potential.c:70-81 */
double libgrpp_potential_value(libgrpp_potential_t *p, double r)
{
    double v = 0.0, r2 = r * r;
    for (int i = 0; i < p->num_primitives; i++)
        v += p->coeffs[i] * rm(pow(r, p->powers[i] - 2), 1) * rm(exp(-p->alpha[i] * r2), 2);
    return v;
}

/* potential.c:88-115 (terms with |c| > 1e-14 kept) */
libgrpp_potential_t *libgrpp_shrink_potential(libgrpp_potential_t *src)
{
    int n = src->num_primitives, m = 0;
    int *pw = calloc(n + 1, sizeof(int));
    double *c = calloc(n + 1, sizeof(double)), *a = calloc(n + 1, sizeof(double));
    for (int i = 0; i < n; i++)
        if (fabs(src->coeffs[i]) > LIBGRPP_ZERO_THRESH) {
            pw[m] = src->powers[i];
            c[m] = src->coeffs[i];
            a[m] = src->alpha[i];
            m++;
        }
    libgrpp_potential_t *p = libgrpp_new_potential(src->L, src->J, m, pw, c, a);
    free(pw);
    free(c);
    free(a);
    return p;
}

int *libgrpp_generate_shell_cartesians(int L)
{
    int n = (L + 1) * (L + 2) / 2;
    int *cl = calloc(3 * n, sizeof(int));
    libgrpp_params.cartesian_generator(L, cl);
    return cl;
}

/* shell.c:23-44 */
libgrpp_shell_t *libgrpp_new_shell(double *origin, int L, int n, double *coeffs, double *alpha)
{
    libgrpp_shell_t *s = malloc(sizeof(*s));
    s->L = L;
    s->origin[0] = origin[0];
    s->origin[1] = origin[1];
    s->origin[2] = origin[2];
    s->cart_size = (L + 1) * (L + 2) / 2;
    s->cart_list = libgrpp_generate_shell_cartesians(L);
    s->num_primitives = n;
    s->coeffs = calloc(n > 0 ? n : 1, sizeof(double));
    s->alpha = calloc(n > 0 ? n : 1, sizeof(double));
    for (int i = 0; i < n; i++) {
        s->coeffs[i] = coeffs[i];
        s->alpha[i] = alpha[i];
    }
    return s;
}

libgrpp_shell_t *libgrpp_shell_deep_copy(libgrpp_shell_t *s)
{
    return libgrpp_new_shell(s->origin, s->L, s->num_primitives, s->coeffs, s->alpha);
}

/* shell.c:64-77 */
void libgrpp_shell_shrink(libgrpp_shell_t *s)
{
    int n = 0;
    for (int i = 0; i < s->num_primitives; i++)
        if (fabs(s->coeffs[i]) > LIBGRPP_ZERO_THRESH) {
            s->coeffs[n] = s->coeffs[i];
            s->alpha[n] = s->alpha[i];
            n++;
        }
    s->num_primitives = n;
}

/* norm_gaussian.c:16-23: (2a/pi)^(3/4) (4a)^(L/2), no double-factorial term */
double orc_gaussian_norm(int L, double alpha)
{
    return pow(2 * alpha / M_PI, 0.75) * pow(4 * alpha, 0.5 * L);
}

void libgrpp_shell_mult_normcoef(libgrpp_shell_t *s)
{
    for (int i = 0; i < s->num_primitives; i++) s->coeffs[i] *= orc_gaussian_norm(s->L, s->alpha[i]);
}

int libgrpp_get_shell_size(libgrpp_shell_t *s) { return s->cart_size; }

void libgrpp_delete_shell(libgrpp_shell_t *s)
{
    if (!s) return;
    free(s->cart_list);
    free(s->coeffs);
    free(s->alpha);
    free(s);
}

/* grpp.c:15-109 */
#define ORC_MAX_POTS 100
libgrpp_grpp_t *libgrpp_new_grpp(void) { return calloc(1, sizeof(libgrpp_grpp_t)); }
void libgrpp_grpp_set_local_potential(libgrpp_grpp_t *g, libgrpp_potential_t *p)
{
    if (g->U_L) libgrpp_delete_potential(g->U_L);
    g->U_L = p;
}
void libgrpp_grpp_add_averaged_potential(libgrpp_grpp_t *g, libgrpp_potential_t *p)
{
    if (g->n_arep == 0) g->U_arep = calloc(ORC_MAX_POTS, sizeof(void *));
    g->U_arep[g->n_arep++] = p;
}
void libgrpp_grpp_add_spin_orbit_potential(libgrpp_grpp_t *g, libgrpp_potential_t *p)
{
    if (g->n_esop == 0) g->U_esop = calloc(ORC_MAX_POTS, sizeof(void *));
    g->U_esop[g->n_esop++] = p;
}
void libgrpp_grpp_add_outercore_potential(libgrpp_grpp_t *g, libgrpp_potential_t *p, libgrpp_shell_t *s)
{
    if (g->n_oc_shells == 0) {
        g->U_oc = calloc(ORC_MAX_POTS, sizeof(void *));
        g->oc_shells = calloc(ORC_MAX_POTS, sizeof(void *));
    }
    g->U_oc[g->n_oc_shells] = p;
    g->oc_shells[g->n_oc_shells] = s;
    g->n_oc_shells++;
}
void libgrpp_delete_grpp(libgrpp_grpp_t *g)
{
    if (!g) return;
    if (g->U_L) libgrpp_delete_potential(g->U_L);
    for (int i = 0; i < g->n_arep; i++) libgrpp_delete_potential(g->U_arep[i]);
    free(g->U_arep);
    for (int i = 0; i < g->n_esop; i++) libgrpp_delete_potential(g->U_esop[i]);
    free(g->U_esop);
    for (int i = 0; i < g->n_oc_shells; i++) {
        libgrpp_delete_potential(g->U_oc[i]);
        libgrpp_delete_shell(g->oc_shells[i]);
    }
    free(g->U_oc);
    free(g->oc_shells);
    free(g);
}

static void daxpy(int n, double a, const double *x, double *y)
{
    for (int i = 0; i < n; i++) y[i] += a * x[i];
}

/* utils.c:64-75: C += A(MxK) B(KxN) */
static void gemm_acc(int M, int N, int K, const double *A, const double *B, double *C)
{
    for (int i = 0; i < M; i++)
        for (int j = 0; j < N; j++) {
            double s = 0.0;
            for (int k = 0; k < K; k++) s += A[i * K + k] * B[k * N + j];
            C[i * N + j] += s;
        }
}

/* utils.c:95-107 */
static int points_equal(const double *a, const double *b)
{
    return fabs(a[0] - b[0]) < 1e-12 && fabs(a[1] - b[1]) < 1e-12 && fabs(a[2] - b[2]) < 1e-12;
}

/* ======================================================== type 1: MMD
 * type1_mcmurchie_davidson.c:107-622 */

typedef struct {
    int S;           /* L_A + L_B */
    double *E;       /* [3][la+1][lb+1][S+1] */
    double *R;       /* [(S+1)^3][S+2] */
    int la, lb;
} mmd_ws_t;

#define EIDX(ws, c, i, j, t) ((((c) * ((ws)->la + 1) + (i)) * ((ws)->lb + 1) + (j)) * ((ws)->S + 1) + (t))
#define RIDX(ws, t, u, v, n) (((((t) * ((ws)->S + 1) + (u)) * ((ws)->S + 1) + (v)) * ((ws)->S + 2)) + (n))

/* type1_mcmurchie_davidson.c:569-622 */
static void setup_E(mmd_ws_t *ws, double q, const double *Q, const double *A, const double *B, const double *K)
{
    for (int c = 0; c < 3; c++)
        for (int i = 0; i <= ws->la; i++)
            for (int j = 0; j <= ws->lb; j++)
                for (int t = 0; t <= i + j; t++) {
                    double v;
                    if (t == 0) {
                        if (i == 0 && j == 0) v = K[c];
                        else if (i == 1 && j == 0) v = (Q[c] - A[c]) * ws->E[EIDX(ws, c, 0, 0, 0)];
                        else if (i == 0 && j == 1) v = (Q[c] - B[c]) * ws->E[EIDX(ws, c, 0, 0, 0)];
                        else if (i == 0)
                            v = (Q[c] - B[c]) * ws->E[EIDX(ws, c, i, j - 1, 0)] + ws->E[EIDX(ws, c, i, j - 1, 1)];
                        else
                            v = (Q[c] - A[c]) * ws->E[EIDX(ws, c, i - 1, j, 0)] + ws->E[EIDX(ws, c, i - 1, j, 1)];
                    } else {
                        double f = 1.0 / (2.0 * q * t);
                        v = 0.0;
                        if (i > 0) v += f * i * ws->E[EIDX(ws, c, i - 1, j, t - 1)];
                        if (j > 0) v += f * j * ws->E[EIDX(ws, c, i, j - 1, t - 1)];
                    }
                    ws->E[EIDX(ws, c, i, j, t)] = v;
                }
}

/* R (1/r: type1_mcmurchie_davidson.c:457-507) or G (1/r^2: :512-564) auxiliary integrals */
static void setup_RG(mmd_ws_t *ws, double q, const double *QC, const double *aux, int is_g)
{
    int S = ws->S;
    for (int t = 0; t <= S; t++)
        for (int u = 0; u <= S; u++)
            for (int v = 0; v <= S; v++) {
                if (t + u + v > S) continue;
                for (int n = 0; n <= S - (t + u + v); n++) {
                    double val = 0.0;
                    if (t + u + v == 0) {
                        val = pow(is_g ? 2.0 * q : -2.0 * q, n) * aux[n];
                    } else {
                        int dt = 0, du = 0, dv = 0, k;
                        double X;
                        if (t + u == 0) { dv = 1; k = v; X = QC[2]; }
                        else if (t == 0) { du = 1; k = u; X = QC[1]; }
                        else { dt = 1; k = t; X = QC[0]; }
                        double r2n1 = 0.0, r2n = 0.0;
                        if (k > 1) {
                            r2n1 = ws->R[RIDX(ws, t - 2 * dt, u - 2 * du, v - 2 * dv, n + 1)];
                            r2n = ws->R[RIDX(ws, t - 2 * dt, u - 2 * du, v - 2 * dv, n)];
                        }
                        double r1n1 = ws->R[RIDX(ws, t - dt, u - du, v - dv, n + 1)];
                        double r1n = ws->R[RIDX(ws, t - dt, u - du, v - dv, n)];
                        if (is_g) {
                            if (k > 1) val += (k - 1) * (r2n1 - 2.0 * q * r2n);
                            val += X * (r1n1 - 2.0 * q * r1n);
                        } else {
                            if (k > 1) val += (k - 1) * r2n1;
                            val += X * r1n1;
                        }
                    }
                    ws->R[RIDX(ws, t, u, v, n)] = val;
                }
            }
}

/* one primitive pair of one potential term c r^(n-2) exp(-zeta r^2) without c:
 * type1_mcmurchie_davidson.c:172-451 */
static void mmd_prim_pair(mmd_ws_t *ws, libgrpp_shell_t *SA, double a, libgrpp_shell_t *SB, double b,
                          const double *C, double c, int npow, double *out)
{
    const double *A = SA->origin, *B = SB->origin;
    double q = a + b + c, muab = a * b / q, muac = a * c / q, mubc = b * c / q;
    double Q[3], K[3];
    for (int i = 0; i < 3; i++) {
        Q[i] = (a * A[i] + b * B[i] + c * C[i]) / q;
        double xab = A[i] - B[i], xac = A[i] - C[i], xbc = B[i] - C[i];
        K[i] = exp(-muab * xab * xab) * exp(-muac * xac * xac) * exp(-mubc * xbc * xbc);
    }
    double QC[3] = {Q[0] - C[0], Q[1] - C[1], Q[2] - C[2]};
    double RQC2 = QC[0] * QC[0] + QC[1] * QC[1] + QC[2] * QC[2];
    int la = SA->L, lb = SB->L, nA = SA->cart_size, nB = SB->cart_size;
    double NA = orc_gaussian_norm(la, a), NB = orc_gaussian_norm(lb, b);

    setup_E(ws, q, Q, A, B, K);
    orc_stats.mmd_prim_pairs++;

    if (npow == 2) {
        for (int m = 0; m < nA; m++)
            for (int n = 0; n < nB; n++) {
                const int *ca = SA->cart_list + 3 * m, *cb = SB->cart_list + 3 * n;
                out[m * nB + n] = NA * NB * ws->E[EIDX(ws, 0, ca[0], cb[0], 0)] * ws->E[EIDX(ws, 1, ca[1], cb[1], 0)] *
                                  ws->E[EIDX(ws, 2, ca[2], cb[2], 0)] * pow(M_PI / q, 1.5);
            }
        return;
    }
    double aux[64];
    if (npow == 1) orc_boys_values(q * RQC2, ws->S, aux);
    else orc_gfun_values(q * RQC2, ws->S, aux);
    setup_RG(ws, q, QC, aux, npow == 0);
    double pref = npow == 1 ? NA * NB * 2.0 * M_PI / q : NA * NB * 2.0 * pow(M_PI, 1.5) / sqrt(q);
    for (int m = 0; m < nA; m++)
        for (int n = 0; n < nB; n++) {
            const int *ca = SA->cart_list + 3 * m, *cb = SB->cart_list + 3 * n;
            double s = 0.0;
            for (int t = 0; t <= ca[0] + cb[0]; t++) {
                double ex = ws->E[EIDX(ws, 0, ca[0], cb[0], t)];
                for (int u = 0; u <= ca[1] + cb[1]; u++) {
                    double ey = ws->E[EIDX(ws, 1, ca[1], cb[1], u)];
                    for (int v = 0; v <= ca[2] + cb[2]; v++) {
                        double ez = ws->E[EIDX(ws, 2, ca[2], cb[2], v)];
                        s += ex * ey * ez * ws->R[RIDX(ws, t, u, v, 0)];
                    }
                }
            }
            out[m * nB + n] = s * pref;
        }
}

/* type1_mcmurchie_davidson.c:107-166: contraction over primitive pairs */
void orc_type1_mmd(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, double zeta, int n, double *out)
{
    assert(n == 0 || n == 1 || n == 2);
    int nA = A->cart_size, nB = B->cart_size;
    mmd_ws_t ws;
    ws.la = A->L;
    ws.lb = B->L;
    ws.S = A->L + B->L;
    ws.E = calloc(3 * (ws.la + 1) * (ws.lb + 1) * (ws.S + 1), sizeof(double));
    ws.R = calloc((size_t)(ws.S + 1) * (ws.S + 1) * (ws.S + 1) * (ws.S + 2), sizeof(double));
    double *buf = calloc(nA * nB, sizeof(double));
    memset(out, 0, nA * nB * sizeof(double));
    for (int i = 0; i < A->num_primitives; i++) {
        double ci = A->coeffs[i];
        if (fabs(ci) < LIBGRPP_ZERO_THRESH) continue;
        for (int j = 0; j < B->num_primitives; j++) {
            double cj = B->coeffs[j];
            if (fabs(cj) < LIBGRPP_ZERO_THRESH) continue;
            mmd_prim_pair(&ws, A, A->alpha[i], B, B->alpha[j], C, zeta, n, buf);
            daxpy(nA * nB, ci * cj, buf, out);
        }
    }
    free(buf);
    free(ws.E);
    free(ws.R);
}

/* type1_integrals.c:43-78 */
void libgrpp_type1_integrals(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, libgrpp_potential_t *pot,
                             double *matrix)
{
    assert(libgrpp_is_initialized());
    int n = A->cart_size * B->cart_size;
    memset(matrix, 0, n * sizeof(double));
    if (!pot) return;
    double *buf = calloc(n, sizeof(double));
    for (int k = 0; k < pot->num_primitives; k++) {
        orc_type1_mmd(A, B, C, pot->alpha[k], pot->powers[k], buf);
        daxpy(n, pot->coeffs[k], buf, matrix);
    }
    free(buf);
}

/* ======================================================== overlap (Obara-Saika)
 * overlap.c:39-139 */
void orc_overlap(libgrpp_shell_t *SA, libgrpp_shell_t *SB, double *out)
{
    int nA = SA->cart_size, nB = SB->cart_size, la = SA->L, lb = SB->L;
    double *buf = calloc(nA * nB, sizeof(double));
    memset(out, 0, nA * nB * sizeof(double));
    for (int i = 0; i < SA->num_primitives; i++)
        for (int j = 0; j < SB->num_primitives; j++) {
            double a = SA->alpha[i], b = SB->alpha[j];
            double NA = orc_gaussian_norm(la, a), NB = orc_gaussian_norm(lb, b);
            double p = a + b, mu = a * b / p;
            double S[3][12][12];
            for (int c = 0; c < 3; c++) {
                double A = SA->origin[c], B = SB->origin[c];
                double P = (a * A + b * B) / p, xab = A - B, xpa = P - A, xpb = P - B, pf = 1.0 / (2.0 * p);
                for (int ii = 0; ii <= la; ii++)
                    for (int jj = 0; jj <= lb; jj++) {
                        double s = 0.0;
                        if (ii + jj == 0) {
                            S[c][0][0] = sqrt(M_PI / p) * exp(-mu * xab * xab);
                            continue;
                        }
                        if (ii == 0) {
                            s += xpb * S[c][ii][jj - 1];
                            if (jj - 1 > 0) s += (jj - 1) * pf * S[c][ii][jj - 2];
                        } else {
                            s += xpa * S[c][ii - 1][jj];
                            if (ii - 1 > 0) s += (ii - 1) * pf * S[c][ii - 2][jj];
                            if (jj > 0) s += jj * pf * S[c][ii - 1][jj - 1];
                        }
                        S[c][ii][jj] = s;
                    }
            }
            for (int m = 0; m < nA; m++)
                for (int n = 0; n < nB; n++) {
                    const int *ca = SA->cart_list + 3 * m, *cb = SB->cart_list + 3 * n;
                    buf[m * nB + n] = NA * NB * S[0][ca[0]][cb[0]] * S[1][ca[1]][cb[1]] * S[2][ca[2]][cb[2]];
                }
            daxpy(nA * nB, SA->coeffs[i] * SB->coeffs[j], buf, out);
        }
    free(buf);
}

/* ======================================================== radial type 2
 * radial_type2_integral.c:101-489, screening.c:193-378 */

#define R2_MIN_GRID 31
#define R2_MAX_GRID 10000

typedef struct {
    double CA, CB;
    libgrpp_potential_t *pot;
    libgrpp_shell_t *bra, *ket;
    int nr, nmax, l1max, l2max;
    double *r, *w, *u, **F1, **F2, **rN;
} r2grid_t;

/* radial_type2_integral.c:465-481 */
static double integrand_contracted(double r, int lambda, double CA, libgrpp_shell_t *g)
{
    double F = 0.0, d2 = (r - CA) * (r - CA);
    for (int i = 0; i < g->num_primitives; i++) {
        double k = 2.0 * g->alpha[i] * CA;
        F += g->coeffs[i] * rm(exp(-g->alpha[i] * d2), 3) * rm(orc_bessel_scaled(lambda, k * r), 4);
    }
    return F;
}

static void r2grid_point(r2grid_t *g, int idx, int i, int nr)
{
    const double R = 5.0, R3 = R * R * R;
    double xi = i / (nr + 1.0), xi3 = xi * xi * xi, ln = rm(log(1 - xi3), 5);
    double wi = 3 * R3 * xi * xi * ln * ln / ((1 - xi3) * (nr + 1.0)), ri = -R * ln;
    g->r[idx] = ri;
    g->w[idx] = wi;
    g->u[idx] = libgrpp_potential_value(g->pot, ri);
    for (int n = 0; n <= g->nmax; n++) g->rN[n][idx] = rm(pow(ri, n), 6);
    for (int l = 0; l <= g->l1max; l++) g->F1[l][idx] = integrand_contracted(ri, l, g->CA, g->bra);
    for (int l = 0; l <= g->l2max; l++) g->F2[l][idx] = integrand_contracted(ri, l, g->CB, g->ket);
    orc_stats.grid_points++;
}

/* radial_type2_integral.c:324-387 (initial 31 points) and :390-444 (nested expansion) */
static void r2grid_expand(r2grid_t *g, int nr)
{
    if (nr > R2_MAX_GRID || nr <= g->nr) return;
    int idx = g->nr;
    for (int i = 1; i <= nr; i += 2) r2grid_point(g, idx++, i, nr);
    g->nr = nr;
}

static double **alloc2(int n, int m)
{
    double **a = calloc(n, sizeof(double *));
    for (int i = 0; i < n; i++) a[i] = calloc(m, sizeof(double));
    return a;
}
static void free2(double **a, int n)
{
    for (int i = 0; i < n; i++) free(a[i]);
    free(a);
}

/* screening.c:329-362: fixed point of the integrand maximum */
static double scr_eq(double r, int n, int l1, int l2, double p, double k1, double k2)
{
    double x1 = k1 * r, x2 = k2 * r;
    double K1 = l1 == 0 ? orc_bessel_scaled(1, x1) / orc_bessel_scaled(0, x1)
                        : orc_bessel_scaled(l1 - 1, x1) / orc_bessel_scaled(l1, x1);
    double K2 = l2 == 0 ? orc_bessel_scaled(1, x2) / orc_bessel_scaled(0, x2)
                        : orc_bessel_scaled(l2 - 1, x2) / orc_bessel_scaled(l2, x2);
    double a = K1 * x1 + K2 * x2 + n;
    if (l1 > 0) a = a - l1 - 1;
    if (l2 > 0) a = a - l2 - 1;
    return sqrt(a / (2.0 * p));
}

/* screening.c:243-322: returns 0 on success (EXIT_SUCCESS), 1 on failure */
static int scr_prim(int l1, int l2, int n, double CA2, double CB2, double aA, double aB, double k1, double k2,
                    double eta, double *val)
{
    *val = 0.0;
    orc_stats.scr_prim_calls++;
    if (l1 >= 1 && fabs(k1) <= LIBGRPP_ZERO_THRESH) return 0;
    if (l2 >= 1 && fabs(k2) <= LIBGRPP_ZERO_THRESH) return 0;
    double p = aA + aB + eta, CA = sqrt(CA2), CB = sqrt(CB2);
    if (l1 == 0 && l2 == 0 && fabs(k1) <= LIBGRPP_ZERO_THRESH && fabs(k2) <= LIBGRPP_ZERO_THRESH) {
        *val = exp(-aA * CA * CA - aB * CB * CB) * orc_gaussian_integral(n, p);
        return 0;
    }
    double r0 = (aA * CA + aB * CB) / p, r0p;
    int steps = 0;
    do {
        steps++;
        if (steps == 5) {
            *val = 0.0;
            return 1;
        }
        r0p = r0;
        r0 = scr_eq(r0, n, l1, l2, p, k1, k2);
    } while (fabs(r0 - r0p) > 1e-2);
    *val = sqrt(M_PI / p) * pow(r0, n) * orc_bessel_scaled(l1, k1 * r0) * orc_bessel_scaled(l2, k2 * r0) *
           exp(-eta * r0 * r0 - aA * (r0 - CA) * (r0 - CA) - aB * (r0 - CB) * (r0 - CB)) * 0.5 *
           (1 + erf(sqrt(p) * r0));
    *val = rm(*val, 7);
    return 0;
}

/* screening.c:193-220 */
static int scr_contracted(int l1, int l2, int n, double CA2, double CB2, libgrpp_shell_t *bra,
                          libgrpp_shell_t *ket, libgrpp_potential_t *pot, double *val)
{
    *val = 0.0;
    double CA = sqrt(CA2), CB = sqrt(CB2);
    for (int i = 0; i < bra->num_primitives; i++) {
        double k1 = 2 * bra->alpha[i] * CA;
        for (int j = 0; j < ket->num_primitives; j++) {
            double k2 = 2 * ket->alpha[j] * CB;
            for (int k = 0; k < pot->num_primitives; k++) {
                double v = 0.0;
                if (scr_prim(l1, l2, n + pot->powers[k], CA2, CB2, bra->alpha[i], ket->alpha[j], k1, k2,
                             pot->alpha[k], &v))
                    return 1;
                *val += bra->coeffs[i] * ket->coeffs[j] * pot->coeffs[k] * v;
            }
        }
    }
    return 0;
}

/* radial_type2_integral.c:242-318 */
static double r2_integral(r2grid_t *g, int n, int l1, int l2, double tol)
{
    int nr = R2_MIN_GRID, conv = 0, level = 0;
    double sum = 0.0, prev, scr = 0.0;
    int scr_fail = scr_contracted(l1, l2, n, g->CA * g->CA, g->CB * g->CB, g->bra, g->ket, g->pot, &scr);
    orc_stats.radial_entries++;
    if (scr_fail) orc_stats.scr_fail++;
    if (!scr_fail && fabs(scr) < tol) {
        orc_stats.screened_out++;
        return scr;
    }
    double *F1 = g->F1[l1], *F2 = g->F2[l2], *rN = g->rN[n];
    for (int i = 0; i < nr; i++) sum += g->w[i] * g->u[i] * F1[i] * F2[i] * rN[i];
    do {
        int idx = nr;
        nr = 2 * nr + 1;
        if (nr > R2_MAX_GRID) {
            level = 9;
            break;
        }
        level++;
        prev = sum;
        sum = 0.5 * sum;
        r2grid_expand(g, nr);
        F1 = g->F1[l1];
        F2 = g->F2[l2];
        rN = g->rN[n];
        for (int i = idx; i < nr; i++) sum += g->w[i] * g->u[i] * F1[i] * F2[i] * rN[i];
        if (!scr_fail && fabs(sum) / fabs(scr) < 0.001) {
            conv = 0;
            continue;
        }
        conv = rm_conv_diff(sum, prev, level) <= tol;
    } while (!conv);
    orc_stats.level_hist[level]++;
    return sum;
}

/* radial_type2_integral.c:101-207 */
double *orc_radial_type2_table(int l1max, int l2max, int nmax, double CA2, double CB2, libgrpp_potential_t *pot,
                               libgrpp_shell_t *bra, libgrpp_shell_t *ket)
{
    int d1 = l1max + 1, d2 = l2max + 1, dn = nmax + 1;
    double *T = calloc(d1 * d2 * dn, sizeof(double));

    if (CA2 < 1e-14 && CB2 < 1e-14) {
        /* one-centre case, analytic; only lambda1 = lambda2 = 0 entries are non-zero */
        for (int i = 0; i < bra->num_primitives; i++) {
            double ci = bra->coeffs[i] * orc_gaussian_norm(bra->L, bra->alpha[i]);
            for (int j = 0; j < ket->num_primitives; j++) {
                double cj = ket->coeffs[j] * orc_gaussian_norm(ket->L, ket->alpha[j]);
                for (int k = 0; k < pot->num_primitives; k++) {
                    double p = bra->alpha[i] + ket->alpha[j] + pot->alpha[k], f = ci * cj * pot->coeffs[k];
                    for (int n = 0; n <= nmax; n++) T[n] += f * orc_gaussian_integral(pot->powers[k] + n, p);
                }
            }
        }
        return T;
    }

    r2grid_t g;
    memset(&g, 0, sizeof(g));
    g.CA = sqrt(CA2);
    g.CB = sqrt(CB2);
    g.pot = libgrpp_shrink_potential(pot);
    g.bra = libgrpp_shell_deep_copy(bra);
    libgrpp_shell_shrink(g.bra);
    libgrpp_shell_mult_normcoef(g.bra);
    g.ket = libgrpp_shell_deep_copy(ket);
    libgrpp_shell_shrink(g.ket);
    libgrpp_shell_mult_normcoef(g.ket);
    g.nmax = nmax;
    g.l1max = l1max;
    g.l2max = l2max;
    g.r = calloc(R2_MAX_GRID, sizeof(double));
    g.w = calloc(R2_MAX_GRID, sizeof(double));
    g.u = calloc(R2_MAX_GRID, sizeof(double));
    g.F1 = alloc2(d1, R2_MAX_GRID);
    g.F2 = alloc2(d2, R2_MAX_GRID);
    g.rN = alloc2(dn, R2_MAX_GRID);
    g.nr = 0;
    for (int i = 1; i <= R2_MIN_GRID; i++) r2grid_point(&g, i - 1, i, R2_MIN_GRID);
    g.nr = R2_MIN_GRID;

    for (int l1 = 0; l1 <= l1max; l1++)
        for (int l2 = 0; l2 <= l2max; l2++)
            for (int n = 0; n <= nmax; n++) T[(l1 * d2 + l2) * dn + n] = r2_integral(&g, n, l1, l2, 1e-16);

    libgrpp_delete_potential(g.pot);
    libgrpp_delete_shell(g.bra);
    libgrpp_delete_shell(g.ket);
    free(g.r);
    free(g.w);
    free(g.u);
    free2(g.F1, d1);
    free2(g.F2, d2);
    free2(g.rN, dn);
    return T;
}

/* ======================================================== type 2 and spin-orbit
 * type2_integrals.c:34-243, spin_orbit_integrals.c:41-288 */

#define ORC_RSH_STRIDE 64

/* shared driver of the binomial re-centring loops; so != 0 selects the type 3 angular sum */
static void semilocal_integrals(libgrpp_shell_t *SA, libgrpp_shell_t *SB, double *C, libgrpp_potential_t *pot,
                                int so, double *out0, double *outx, double *outy, double *outz)
{
    int nA = SA->cart_size, nB = SB->cart_size, L = pot->L;
    int la = SA->cart_list[0] + SA->cart_list[1] + SA->cart_list[2];
    int lb = SB->cart_list[0] + SB->cart_list[1] + SB->cart_list[2];
    double CAv[3], CBv[3], kA[3], kB[3];
    for (int i = 0; i < 3; i++) {
        CAv[i] = C[i] - SA->origin[i];
        CBv[i] = C[i] - SB->origin[i];
        kA[i] = -2.0 * (SA->alpha[0] * CAv[i]);
        kB[i] = -2.0 * (SB->alpha[0] * CBv[i]);
    }
    double CA2 = CAv[0] * CAv[0] + CAv[1] * CAv[1] + CAv[2] * CAv[2];
    double CB2 = CBv[0] * CBv[0] + CBv[1] * CBv[1] + CBv[2] * CBv[2];
    int l1max = L + la, l2max = L + lb, nmax = la + lb;
    int lmax = l1max > l2max ? l1max : l2max;
    if (L > lmax) lmax = L;
    /* type 2 uses 1e-13 / 1e-16 skip thresholds, spin-orbit uses 1e-14 everywhere */
    double fthr = so ? LIBGRPP_ZERO_THRESH : 1e-13, qthr = so ? LIBGRPP_ZERO_THRESH : 1e-16,
           wthr = so ? LIBGRPP_ZERO_THRESH : 1e-16;

    double *T = orc_radial_type2_table(l1max, l2max, nmax, CA2, CB2, pot, SA, SB);
    double *rA = calloc((lmax + 1) * ORC_RSH_STRIDE, sizeof(double));
    double *rB = calloc((lmax + 1) * ORC_RSH_STRIDE, sizeof(double));
    for (int l = 0; l <= lmax; l++) {
        orc_rsh_array(l, kA, rA + l * ORC_RSH_STRIDE);
        orc_rsh_array(l, kB, rB + l * ORC_RSH_STRIDE);
    }
    int dim = 2 * L + 1;
    double *Lm[3] = {NULL, NULL, NULL};
    if (so) {
        for (int c = 0; c < 3; c++) Lm[c] = calloc(dim * dim, sizeof(double));
        orc_lmatrices_rsh(L, Lm[0], Lm[1], Lm[2]);
    }

    for (int ic = 0; ic < nA; ic++)
        for (int jc = 0; jc < nB; jc++) {
            const int *ca = SA->cart_list + 3 * ic, *cb = SB->cart_list + 3 * jc;
            double acc[3] = {0, 0, 0};
            for (int a = 0; a <= ca[0]; a++)
                for (int b = 0; b <= ca[1]; b++)
                    for (int c = 0; c <= ca[2]; c++)
                        for (int d = 0; d <= cb[0]; d++)
                            for (int e = 0; e <= cb[1]; e++)
                                for (int f = 0; f <= cb[2]; f++) {
                                    double factor = (double)orc_binomial(ca[0], a) * (double)orc_binomial(ca[1], b) *
                                                    (double)orc_binomial(ca[2], c) * (double)orc_binomial(cb[0], d) *
                                                    (double)orc_binomial(cb[1], e) * (double)orc_binomial(cb[2], f) *
                                                    pow(CAv[0], ca[0] - a) * pow(CAv[1], ca[1] - b) *
                                                    pow(CAv[2], ca[2] - c) * pow(CBv[0], cb[0] - d) *
                                                    pow(CBv[1], cb[1] - e) * pow(CBv[2], cb[2] - f);
                                    if (fabs(factor) < fthr) continue;
                                    int N = a + b + c + d + e + f;
                                    int nabc = a + b + c, ndef = d + e + f;
                                    int l1lo = L - nabc > 0 ? L - nabc : 0, l2lo = L - ndef > 0 ? L - ndef : 0;
                                    double s[3] = {0, 0, 0};
                                    for (int l1 = l1lo; l1 <= L + nabc; l1++) {
                                        if ((L + nabc - l1) % 2 != 0) continue;
                                        for (int l2 = l2lo; l2 <= L + ndef; l2++) {
                                            if ((L + ndef - l2) % 2 != 0) continue;
                                            double QN = T[(l1 * (l2max + 1) + l2) * (nmax + 1) + N];
                                            if (fabs(QN) < qthr) continue;
                                            if (!so) {
                                                double ang = 0.0;
                                                for (int m = -L; m <= L; m++) {
                                                    double w1 = orc_angular_type2(l1, L, m, a, b, c, rA + l1 * ORC_RSH_STRIDE);
                                                    if (fabs(w1) < wthr) continue;
                                                    double w2 = orc_angular_type2(l2, L, m, d, e, f, rB + l2 * ORC_RSH_STRIDE);
                                                    ang += w1 * w2;
                                                }
                                                s[0] += QN * ang;
                                            } else {
                                                double ax = 0, ay = 0, az = 0;
                                                for (int m1 = -L; m1 <= L; m1++)
                                                    for (int m2 = -L; m2 <= L; m2++) {
                                                        int id = dim * (m1 + L) + m2 + L;
                                                        double lx = Lm[0][id], ly = Lm[1][id], lz = Lm[2][id];
                                                        if (fabs(lx) < LIBGRPP_ZERO_THRESH && fabs(ly) < LIBGRPP_ZERO_THRESH &&
                                                            fabs(lz) < LIBGRPP_ZERO_THRESH)
                                                            continue;
                                                        double w1 = orc_angular_type2(l1, L, m1, a, b, c, rA + l1 * ORC_RSH_STRIDE);
                                                        if (fabs(w1) < LIBGRPP_ZERO_THRESH) continue;
                                                        double w2 = orc_angular_type2(l2, L, m2, d, e, f, rB + l2 * ORC_RSH_STRIDE);
                                                        ax += w1 * w2 * lx;
                                                        ay += w1 * w2 * ly;
                                                        az += w1 * w2 * lz;
                                                    }
                                                s[0] += QN * ax;
                                                s[1] += QN * ay;
                                                s[2] += QN * az;
                                            }
                                        }
                                    }
                                    acc[0] += factor * s[0];
                                    acc[1] += factor * s[1];
                                    acc[2] += factor * s[2];
                                }
            if (!so) out0[ic * nB + jc] = acc[0] * (16 * M_PI * M_PI);
            else {
                outx[ic * nB + jc] = acc[0] * (16.0 * M_PI * M_PI);
                outy[ic * nB + jc] = acc[1] * (16.0 * M_PI * M_PI);
                outz[ic * nB + jc] = acc[2] * (16.0 * M_PI * M_PI);
            }
        }
    free(T);
    free(rA);
    free(rB);
    for (int c = 0; c < 3; c++) free(Lm[c]);
}

void libgrpp_type2_integrals(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, libgrpp_potential_t *pot,
                             double *matrix)
{
    assert(libgrpp_is_initialized());
    memset(matrix, 0, A->cart_size * B->cart_size * sizeof(double));
    semilocal_integrals(A, B, C, pot, 0, matrix, NULL, NULL, NULL);
}

void libgrpp_spin_orbit_integrals(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, libgrpp_potential_t *pot,
                                  double *sx, double *sy, double *sz)
{
    assert(libgrpp_is_initialized());
    int n = A->cart_size * B->cart_size;
    memset(sx, 0, n * sizeof(double));
    memset(sy, 0, n * sizeof(double));
    memset(sz, 0, n * sizeof(double));
    semilocal_integrals(A, B, C, pot, 1, NULL, sx, sy, sz);
}

/* ======================================================== outercore
 * outercore_integrals.c:83-553 */

/* outercore_integrals.c:545-553 */
static double ang_norm_factor(int lx, int ly, int lz)
{
    int L = lx + ly + lz;
    return 1.0 / (2.0 * sqrt(M_PI)) * sqrt(orc_double_factorial(2 * L + 1));
}

/* outercore_integrals.c:481-510: radial GTO norm sqrt(2^(L+5/2)/Gamma(L+3/2)) alpha^(3/4+L/2) */
static double radial_gto_norm(int L, double alpha)
{
    /* Gamma(L+3/2) = (2L+1)!! sqrt(pi) / 2^(L+1) */
    double g = orc_double_factorial(2 * L + 1) * sqrt(M_PI) / pow(2.0, L + 1);
    return sqrt(pow(2.0, L + 2.5) / g) * pow(alpha, 0.75 + L / 2.0);
}

/* outercore_integrals.c:457-478 */
static double one_centre_prim(int L, double a1, double a2, int n, double zeta)
{
    double a = a1 + a2 + zeta;
    if (n % 2 == 0) {
        int k = L + n / 2;
        return orc_double_factorial(2 * k - 1) / (pow(2.0, k + 1) * pow(a, k)) * sqrt(M_PI / a);
    }
    int k = L + (n - 1) / 2;
    return orc_factorial(k) / (2.0 * pow(a, k + 1));
}

/* outercore_integrals.c:425-450 */
static double one_centre_contracted(libgrpp_shell_t *bra, libgrpp_shell_t *ket, libgrpp_potential_t *pot)
{
    double sum = 0.0;
    int L = pot->L;
    for (int i = 0; i < bra->num_primitives; i++) {
        double Ni = radial_gto_norm(L, bra->alpha[i]);
        for (int j = 0; j < ket->num_primitives; j++) {
            double Nj = radial_gto_norm(L, ket->alpha[j]);
            double f = Ni * Nj * bra->coeffs[i] * ket->coeffs[j];
            for (int k = 0; k < pot->num_primitives; k++)
                sum += f * pot->coeffs[k] * one_centre_prim(L, bra->alpha[i], ket->alpha[j], pot->powers[k], pot->alpha[k]);
        }
    }
    return sum;
}

/* outercore_integrals.c:397-418 */
static double delta_integral(libgrpp_potential_t *p1, libgrpp_shell_t *s1, libgrpp_potential_t *p2,
                             libgrpp_shell_t *s2)
{
    if (p1->L != p2->L || p1->J != p2->J) return 0.0;
    return 0.5 * (one_centre_contracted(s1, s2, p1) + one_centre_contracted(s1, s2, p2));
}

/* Cartesian -> real spherical coefficients of an oc shell (outercore_integrals.c:165-177) */
static double *oc_sph_coef(libgrpp_shell_t *oc)
{
    int L = oc->L, n = oc->cart_size;
    double *S = calloc((2 * L + 1) * n, sizeof(double));
    for (int m = -L; m <= L; m++)
        for (int ic = 0; ic < n; ic++) {
            const int *c = oc->cart_list + 3 * ic;
            S[n * (m + L) + ic] = orc_sph_to_cart_coef(L, m, c[0], c[1], c[2]) / ang_norm_factor(c[0], c[1], c[2]);
        }
    return S;
}

/* outercore_integrals.c:514-542 */
static void to_sph_ket(int dbra, int dcart, int dsph, const double *in, double *out, const double *S)
{
    for (int i = 0; i < dbra; i++)
        for (int j = 0; j < dsph; j++) {
            double s = 0.0;
            for (int ic = 0; ic < dcart; ic++) s += S[dcart * j + ic] * in[i * dcart + ic];
            out[i * dsph + j] = s;
        }
}
static void to_sph_bra(int dcart, int dsph, int dket, const double *in, double *out, const double *S)
{
    for (int j = 0; j < dket; j++)
        for (int i = 0; i < dsph; i++) {
            double s = 0.0;
            for (int ic = 0; ic < dcart; ic++) s += S[dcart * i + ic] * in[ic * dket + j];
            out[i * dket + j] = s;
        }
}

/* outercore_integrals.c:147-270 */
static void oc_part1(libgrpp_shell_t *SA, libgrpp_shell_t *SB, double *C, libgrpp_potential_t *pot,
                     libgrpp_shell_t *oc, double *arep, double *sx, double *sy, double *sz)
{
    int L = oc->L, nA = SA->cart_size, nB = SB->cart_size, no = oc->cart_size, d = 2 * L + 1;
    double J = pot->J / 2.0;
    double *Sc = oc_sph_coef(oc);
    double *t1 = calloc(no * nB, sizeof(double)), *t2 = calloc(nA * no, sizeof(double));
    double *S_b = calloc(d * nB, sizeof(double)), *S_a = calloc(nA * d, sizeof(double));
    double *U_b = calloc(d * nB, sizeof(double)), *U_a = calloc(nA * d, sizeof(double));
    orc_overlap(oc, SB, t1);
    orc_overlap(SA, oc, t2);
    to_sph_ket(nA, no, d, t2, S_a, Sc);
    to_sph_bra(no, d, nB, t1, S_b, Sc);
    libgrpp_type1_integrals(oc, SB, C, pot, t1);
    libgrpp_type1_integrals(SA, oc, C, pot, t2);
    to_sph_ket(nA, no, d, t2, U_a, Sc);
    to_sph_bra(no, d, nB, t1, U_b, Sc);

    double farep = (J < L) ? (L / (2.0 * L + 1)) : ((L + 1) / (2.0 * L + 1));
    double *buf = calloc(nA * nB, sizeof(double));
    gemm_acc(nA, nB, d, S_a, U_b, buf);
    gemm_acc(nA, nB, d, U_a, S_b, buf);
    daxpy(nA * nB, farep, buf, arep);

    double *Lm[3];
    for (int c = 0; c < 3; c++) Lm[c] = calloc(d * d, sizeof(double));
    orc_lmatrices_rsh(L, Lm[0], Lm[1], Lm[2]);
    int mx = nA > nB ? nA : nB;
    double *tmp = calloc(d * mx, sizeof(double));
    double *outs[3] = {sx, sy, sz};
    double fso = (J < L) ? (-2.0 / (2 * L + 1)) : (+2.0 / (2 * L + 1));
    for (int c = 0; c < 3; c++) {
        double *so = calloc(nA * nB, sizeof(double));
        memset(tmp, 0, d * nB * sizeof(double));
        gemm_acc(d, nB, d, Lm[c], S_b, tmp);
        gemm_acc(nA, nB, d, U_a, tmp, so);
        memset(tmp, 0, d * nA * sizeof(double));
        gemm_acc(nA, d, d, S_a, Lm[c], tmp);
        gemm_acc(nA, nB, d, tmp, U_b, so);
        daxpy(nA * nB, fso, so, outs[c]);
        free(so);
        free(Lm[c]);
    }
    free(tmp);
    free(buf);
    free(Sc);
    free(t1);
    free(t2);
    free(S_a);
    free(S_b);
    free(U_a);
    free(U_b);
}

/* outercore_integrals.c:277-390 */
static void oc_part2(libgrpp_shell_t *SA, libgrpp_shell_t *SB, libgrpp_potential_t *p1, libgrpp_shell_t *oc1,
                     libgrpp_potential_t *p2, libgrpp_shell_t *oc2, double *arep, double *sx, double *sy, double *sz)
{
    if (p1->L != p2->L || p1->J != p2->J) return;
    int L = p1->L, nA = SA->cart_size, nB = SB->cart_size, no = oc1->cart_size, d = 2 * L + 1;
    double J = p1->J / 2.0;
    double delta = delta_integral(p1, oc1, p2, oc2);
    double *Sc = oc_sph_coef(oc1);
    double *t1 = calloc(no * nB, sizeof(double)), *t2 = calloc(nA * no, sizeof(double));
    double *S_b = calloc(d * nB, sizeof(double)), *S_a = calloc(nA * d, sizeof(double));
    orc_overlap(oc2, SB, t1);
    orc_overlap(SA, oc1, t2);
    to_sph_ket(nA, no, d, t2, S_a, Sc);
    to_sph_bra(no, d, nB, t1, S_b, Sc);
    double farep = (J < L) ? (L / (2.0 * L + 1)) : ((L + 1) / (2.0 * L + 1));
    double *buf = calloc(nA * nB, sizeof(double));
    gemm_acc(nA, nB, d, S_a, S_b, buf);
    daxpy(nA * nB, -1.0 * delta * farep, buf, arep);

    double *Lm[3];
    for (int c = 0; c < 3; c++) Lm[c] = calloc(d * d, sizeof(double));
    orc_lmatrices_rsh(L, Lm[0], Lm[1], Lm[2]);
    double *tmp = calloc(d * nB, sizeof(double));
    double *outs[3] = {sx, sy, sz};
    double fso = (J < L) ? (-2.0 / (2 * L + 1)) : (+2.0 / (2 * L + 1));
    for (int c = 0; c < 3; c++) {
        double *so = calloc(nA * nB, sizeof(double));
        memset(tmp, 0, d * nB * sizeof(double));
        gemm_acc(d, nB, d, Lm[c], S_b, tmp);
        gemm_acc(nA, nB, d, S_a, tmp, so);
        daxpy(nA * nB, -1.0 * delta * fso, so, outs[c]);
        free(so);
        free(Lm[c]);
    }
    free(tmp);
    free(buf);
    free(Sc);
    free(t1);
    free(t2);
    free(S_a);
    free(S_b);
}

/* outercore_integrals.c:83-140. The oc shells are bound to the RPP centre on
 * private copies: the caller's objects are not written. */
void libgrpp_outercore_potential_integrals(libgrpp_shell_t *SA, libgrpp_shell_t *SB, double *C, int noc,
                                           libgrpp_potential_t **pots, libgrpp_shell_t **ocs, double *arep,
                                           double *sx, double *sy, double *sz)
{
    assert(libgrpp_is_initialized());
    int n = SA->cart_size * SB->cart_size;
    memset(arep, 0, n * sizeof(double));
    memset(sx, 0, n * sizeof(double));
    memset(sy, 0, n * sizeof(double));
    memset(sz, 0, n * sizeof(double));
    libgrpp_shell_t **loc = calloc(noc > 0 ? noc : 1, sizeof(void *));
    for (int i = 0; i < noc; i++) {
        loc[i] = libgrpp_shell_deep_copy(ocs[i]);
        memcpy(loc[i]->cart_list, ocs[i]->cart_list, 3 * ocs[i]->cart_size * sizeof(int));
        loc[i]->origin[0] = C[0];
        loc[i]->origin[1] = C[1];
        loc[i]->origin[2] = C[2];
    }
    for (int i = 0; i < noc; i++) oc_part1(SA, SB, C, pots[i], loc[i], arep, sx, sy, sz);
    for (int i = 0; i < noc; i++)
        for (int j = 0; j < noc; j++) oc_part2(SA, SB, pots[i], loc[i], pots[j], loc[j], arep, sx, sy, sz);
    for (int i = 0; i < noc; i++) libgrpp_delete_shell(loc[i]);
    free(loc);
}

/* ======================================================== full GRPP
 * full_grpp_integrals.c:27-104 */
void libgrpp_full_grpp_integrals(libgrpp_shell_t *A, libgrpp_shell_t *B, libgrpp_grpp_t *g, double *C,
                                 double *arep, double *sx, double *sy, double *sz)
{
    assert(libgrpp_is_initialized());
    int n = A->cart_size * B->cart_size;
    double *b0 = calloc(n, sizeof(double)), *bx = calloc(n, sizeof(double)), *by = calloc(n, sizeof(double)),
           *bz = calloc(n, sizeof(double));
    memset(arep, 0, n * sizeof(double));
    memset(sx, 0, n * sizeof(double));
    memset(sy, 0, n * sizeof(double));
    memset(sz, 0, n * sizeof(double));
    libgrpp_type1_integrals(A, B, C, g->U_L, b0);
    daxpy(n, 1.0, b0, arep);
    for (int L = 0; L < g->n_arep; L++) {
        libgrpp_type2_integrals(A, B, C, g->U_arep[L], b0);
        daxpy(n, 1.0, b0, arep);
    }
    for (int i = 0; i < g->n_esop; i++) {
        libgrpp_spin_orbit_integrals(A, B, C, g->U_esop[i], bx, by, bz);
        int L = g->U_esop[i]->L;
        daxpy(n, 2.0 / (2 * L + 1), bx, sx);
        daxpy(n, 2.0 / (2 * L + 1), by, sy);
        daxpy(n, 2.0 / (2 * L + 1), bz, sz);
    }
    libgrpp_outercore_potential_integrals(A, B, C, g->n_oc_shells, g->U_oc, g->oc_shells, b0, bx, by, bz);
    daxpy(n, 1.0, b0, arep);
    daxpy(n, 1.0, bx, sx);
    daxpy(n, 1.0, by, sy);
    daxpy(n, 1.0, bz, sz);
    free(b0);
    free(bx);
    free(by);
    free(bz);
}

/* ======================================================== gradients
 * grpp_integrals_gradient.c:123-1045, diff_gaussian.c:35-72, overlap_gradient.c:219-241 */

/* diff_gaussian.c:35-63: the "2 alpha" factor is absorbed into the L+1 coefficients */
static void differentiate_shell(libgrpp_shell_t *s, libgrpp_shell_t **down, libgrpp_shell_t **up)
{
    *down = NULL;
    if (s->L > 0) {
        *down = libgrpp_new_shell(s->origin, s->L - 1, s->num_primitives, s->coeffs, s->alpha);
        for (int i = 0; i < s->num_primitives; i++)
            (*down)->coeffs[i] *= orc_gaussian_norm(s->L, s->alpha[i]) / orc_gaussian_norm(s->L - 1, s->alpha[i]);
    }
    *up = libgrpp_new_shell(s->origin, s->L + 1, s->num_primitives, s->coeffs, s->alpha);
    for (int i = 0; i < s->num_primitives; i++)
        (*up)->coeffs[i] *= 2.0 * s->alpha[i] * orc_gaussian_norm(s->L, s->alpha[i]) / orc_gaussian_norm(s->L + 1, s->alpha[i]);
}

/* overlap_gradient.c:219-241 */
static int nlm_to_linear(const int *nlm)
{
    int L = nlm[0] + nlm[1] + nlm[2], n = (L + 1) * (L + 2) / 2;
    int *cl = libgrpp_generate_shell_cartesians(L), idx;
    for (idx = 0; idx < n; idx++)
        if (cl[3 * idx] == nlm[0] && cl[3 * idx + 1] == nlm[1] && cl[3 * idx + 2] == nlm[2]) break;
    free(cl);
    return idx;
}

/* grpp_integrals_gradient.c:786-906 (general form of the bra/ket differentiated contribution;
 * :403-595 and :597-785 are the same assembly for the ACA case) */
static void grad_contribution(libgrpp_shell_t *A, libgrpp_shell_t *B, libgrpp_grpp_t *g, double *C, double **gr[4],
                              int diff_bra, double factor)
{
    libgrpp_shell_t *dsh = diff_bra ? A : B, *down, *up;
    differentiate_shell(dsh, &down, &up);
    int nA = A->cart_size, nB = B->cart_size;
    double *Md[4] = {NULL, NULL, NULL, NULL}, *Mu[4];
    int nd = down ? down->cart_size : 0, nu = up->cart_size;
    if (down) {
        int sz = (diff_bra ? nB : nA) * nd;
        for (int c = 0; c < 4; c++) Md[c] = calloc(sz, sizeof(double));
        libgrpp_full_grpp_integrals(diff_bra ? down : A, diff_bra ? B : down, g, C, Md[0], Md[1], Md[2], Md[3]);
    }
    int szu = (diff_bra ? nB : nA) * nu;
    for (int c = 0; c < 4; c++) Mu[c] = calloc(szu, sizeof(double));
    libgrpp_full_grpp_integrals(diff_bra ? up : A, diff_bra ? B : up, g, C, Mu[0], Mu[1], Mu[2], Mu[3]);

    for (int k = 0; k < 3; k++)
        for (int i = 0; i < nA; i++)
            for (int j = 0; j < nB; j++) {
                int bra[3] = {A->cart_list[3 * i], A->cart_list[3 * i + 1], A->cart_list[3 * i + 2]};
                int ket[3] = {B->cart_list[3 * j], B->cart_list[3 * j + 1], B->cart_list[3 * j + 2]};
                int *dn = diff_bra ? bra : ket, idx = i * nB + j;
                /* libgrpp forms this term also when the exponent is 0; it then reads outside
                 * the L-1 block (nlm_to_linear finds no match) and multiplies by 0. The term
                 * is skipped here, which is the same value without the out-of-bounds read. */
                if (nd > 0 && dn[k] > 0) {
                    dn[k] -= 1;
                    int bi = nlm_to_linear(bra), ki = nlm_to_linear(ket);
                    dn[k] += 1;
                    int n = dn[k], row = diff_bra ? nB : nd, id = row * bi + ki;
                    for (int c = 0; c < 4; c++) gr[c][k][idx] -= factor * n * Md[c][id];
                }
                dn[k] += 1;
                int bi = nlm_to_linear(bra), ki = nlm_to_linear(ket);
                dn[k] -= 1;
                int row = diff_bra ? nB : nu, id = row * bi + ki;
                for (int c = 0; c < 4; c++) gr[c][k][idx] += factor * Mu[c][id];
            }
    for (int c = 0; c < 4; c++) {
        free(Md[c]);
        free(Mu[c]);
    }
    if (down) libgrpp_delete_shell(down);
    libgrpp_delete_shell(up);
}

/* grpp_integrals_gradient.c:280-393 */
void libgrpp_full_grpp_integrals_gradient(libgrpp_shell_t *SA, libgrpp_shell_t *SB, libgrpp_grpp_t *g, double *C,
                                          double *D, double **ga, double **gx, double **gy, double **gz)
{
    int n = SA->cart_size * SB->cart_size;
    double **gr[4] = {ga, gx, gy, gz};
    for (int c = 0; c < 4; c++)
        for (int k = 0; k < 3; k++) memset(gr[c][k], 0, n * sizeof(double));
    double *A = SA->origin, *B = SB->origin;
    if (points_equal(A, C) && points_equal(B, C)) return;
    if (!points_equal(A, D) && !points_equal(B, D) && !points_equal(C, D)) return;
    if (!points_equal(A, C) && !points_equal(C, B) && !points_equal(A, B)) { /* ACB */
        if (points_equal(A, D)) grad_contribution(SA, SB, g, C, gr, 1, +1.0);
        if (points_equal(B, D)) grad_contribution(SA, SB, g, C, gr, 0, +1.0);
        if (points_equal(C, D)) {
            grad_contribution(SA, SB, g, C, gr, 1, -1.0);
            grad_contribution(SA, SB, g, C, gr, 0, -1.0);
        }
    }
    if (points_equal(A, B) && !points_equal(A, C)) { /* ACA */
        double f = points_equal(A, D) ? +1.0 : -1.0;
        grad_contribution(SA, SB, g, C, gr, 1, f);
        grad_contribution(SA, SB, g, C, gr, 0, f);
    }
    if (!points_equal(A, C) && points_equal(C, B)) /* ACC */
        grad_contribution(SA, SB, g, C, gr, 1, points_equal(A, D) ? +1.0 : -1.0);
    if (points_equal(A, C) && !points_equal(C, B)) /* CCB */
        grad_contribution(SA, SB, g, C, gr, 0, points_equal(B, D) ? +1.0 : -1.0);
}

static double **alloc_grad(int n)
{
    double **g = calloc(3, sizeof(double *));
    for (int k = 0; k < 3; k++) g[k] = calloc(n, sizeof(double));
    return g;
}
static void free_grad(double **g)
{
    for (int k = 0; k < 3; k++) free(g[k]);
    free(g);
}

/* grpp_integrals_gradient.c:123-272: single-term wrappers through a temporary GRPP */
void libgrpp_type1_integrals_gradient(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, libgrpp_potential_t *p,
                                      double *D, double **ga)
{
    libgrpp_grpp_t *g = libgrpp_new_grpp();
    g->U_L = p;
    int n = A->cart_size * B->cart_size;
    double **x = alloc_grad(n), **y = alloc_grad(n), **z = alloc_grad(n);
    libgrpp_full_grpp_integrals_gradient(A, B, g, C, D, ga, x, y, z);
    free_grad(x);
    free_grad(y);
    free_grad(z);
    g->U_L = NULL;
    libgrpp_delete_grpp(g);
}

void libgrpp_type2_integrals_gradient(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, libgrpp_potential_t *p,
                                      double *D, double **ga)
{
    libgrpp_grpp_t *g = libgrpp_new_grpp();
    libgrpp_grpp_add_averaged_potential(g, p);
    int n = A->cart_size * B->cart_size;
    double **x = alloc_grad(n), **y = alloc_grad(n), **z = alloc_grad(n);
    libgrpp_full_grpp_integrals_gradient(A, B, g, C, D, ga, x, y, z);
    free_grad(x);
    free_grad(y);
    free_grad(z);
    g->n_arep = 0;
    libgrpp_delete_grpp(g);
}

void libgrpp_spin_orbit_integrals_gradient(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, libgrpp_potential_t *p,
                                           double *D, double **gx, double **gy, double **gz)
{
    libgrpp_grpp_t *g = libgrpp_new_grpp();
    libgrpp_grpp_add_spin_orbit_potential(g, p);
    int n = A->cart_size * B->cart_size;
    double **a = alloc_grad(n);
    libgrpp_full_grpp_integrals_gradient(A, B, g, C, D, a, gx, gy, gz);
    int L = p->L;
    for (int k = 0; k < 3; k++)
        for (int i = 0; i < n; i++) {
            gx[k][i] *= (2.0 * L + 1.0) / 2.0;
            gy[k][i] *= (2.0 * L + 1.0) / 2.0;
            gz[k][i] *= (2.0 * L + 1.0) / 2.0;
        }
    free_grad(a);
    g->n_esop = 0;
    libgrpp_delete_grpp(g);
}

void libgrpp_outercore_potential_integrals_gradient(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, int noc,
                                                    libgrpp_potential_t **pots, libgrpp_shell_t **ocs, double *D,
                                                    double **ga, double **gx, double **gy, double **gz)
{
    libgrpp_grpp_t *g = libgrpp_new_grpp();
    for (int i = 0; i < noc; i++) libgrpp_grpp_add_outercore_potential(g, pots[i], ocs[i]);
    libgrpp_full_grpp_integrals_gradient(A, B, g, C, D, ga, gx, gy, gz);
    g->n_oc_shells = 0;
    libgrpp_delete_grpp(g);
}

/* ======================================================== oracle-only helpers */

void orc_stats_reset(void) { memset(&orc_stats, 0, sizeof(orc_stats)); }
const orc_stats_t *orc_stats_get(void) { return &orc_stats; }

double orc_bessel_scaled_export(int n, double x) { return orc_bessel_scaled(n, x); }
double orc_boys_export(int n, double x) { return orc_boys(n, x); }
void orc_gfun_export(double x, int nmax, double *g) { orc_gfun_values(x, nmax, g); }
double orc_dawson_export(double y) { return orc_dawson(y); }
