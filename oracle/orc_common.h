/*
 * ORACLE — test infrastructure only.
 *
 * CPU restatement of libgrpp's GRPP integral path, used by tests/, by
 * __graft_entry__.smoke() and by bench.py's cpu_baseline leg as the checker.
 * The product (libgrpp_b200) never links, loads or calls anything here.
 *
 * Internal declarations shared by the oracle translation units.
 */
#ifndef ORC_COMMON_H
#define ORC_COMMON_H

#include <stdint.h>
#include "../include/libgrpp.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define ORC_LMAX_RSH 40      /* RSH tables are built up to L=40 (init_finalize.c:24) */
#define ORC_BES_NX 1601      /* Bessel table x = 0.00 .. 16.00 step 0.01 (specfunc_bessel_table.c:14-17) */
#define ORC_BES_NL 60        /* lambda = 0 .. 59 */
#define ORC_BOYS_NX 301      /* Boys table x = 0.0 .. 30.0 step 0.1 (specfunc_boys.c:24) */
#define ORC_BOYS_NN 40

/* math helpers: factorial.c, binomial.c */
double orc_factorial(int n);
double orc_factorial_ratio(int n, int m);
double orc_double_factorial(int n);
uint64_t orc_binomial(int n, int k);

/* special functions */
void orc_tables_init(void);
double orc_bessel_scaled(int n, double x);
double orc_boys(int n, double x);
void orc_boys_values(double x, int nmax, double *b);
void orc_gfun_values(double x, int nmax, double *g);
double orc_dawson(double y);

/* real spherical harmonics */
double orc_sph_to_cart_coef(int l, int m, int lx, int ly, int lz);
void orc_rsh_array(int l, const double *k, double *out);
int orc_rsh_ncomb(int L);
const int *orc_rsh_comb(int L);
const double *orc_rsh_coef(int L);
double orc_usp_integral(int i, int j, int k);
double orc_angular_type2(int lambda, int L, int m, int a, int b, int c, const double *rsh_values);
void orc_lmatrices_rsh(int L, double *lx, double *ly, double *lz);

/* integrals on single primitives / shells */
double orc_gaussian_norm(int L, double alpha);
void orc_type1_mmd(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, double zeta, int n,
                   double *out);
void orc_overlap(libgrpp_shell_t *A, libgrpp_shell_t *B, double *out);
double orc_gaussian_integral(int n, double a);

/* radial type 2 table: Q[(l1*(l2max+1) + l2)*(nmax+1) + n] */
double *orc_radial_type2_table(int l1max, int l2max, int nmax, double CA2, double CB2,
                               libgrpp_potential_t *pot, libgrpp_shell_t *bra,
                               libgrpp_shell_t *ket);

/* operation counters for the flop convention of the measurement */
typedef struct {
    uint64_t grid_points;       /* integrand points evaluated */
    uint64_t radial_entries;    /* (lambda1, lambda2, N) integrals */
    uint64_t screened_out;      /* entries returned by the screening gate */
    uint64_t level_hist[10];    /* stop level histogram (index 9 = capped) */
    uint64_t mmd_prim_pairs;    /* primitive shell pairs through MMD */
    uint64_t scr_prim_calls;    /* primitive screening estimates */
    uint64_t scr_fail;          /* contracted screenings that failed */
    uint64_t bessel_calls;      /* scaled Bessel evaluations */
} orc_stats_t;
extern orc_stats_t orc_stats;

#endif
