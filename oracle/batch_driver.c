/*
 * ORACLE — test infrastructure only.
 *
 * Batch driver over the libgrpp C API. The same source is compiled twice:
 * with the reference's own sources into oracle/_ref/libgrpp_ref.so (the CPU
 * baseline and the pin for the restatement), and with the CPU restatement into
 * oracle/_build/libgrpp_oracle.so. It only calls public libgrpp_* functions,
 * in the way libgrpp's own test driver does
 * (test_libgrpp_c/eval_integrals.c:42-208, eval_integrals_grad.c:37-163):
 * one call per (shell pair, centre), OpenMP over tasks, and one private copy
 * of every GRPP object per thread because libgrpp writes the outercore shells'
 * origins during a call (libgrpp/outercore_integrals.c:107-111).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/libgrpp.h"
#include "../include/libgrpp_b200.h"

typedef struct {
    libgrpp_shell_t **shells;
    libgrpp_grpp_t **grpps;
    int n_shells, n_grpps;
} built_t;

static libgrpp_shell_t *make_shell(const libgrpp_b200_batch_t *b, int s)
{
    double o[3] = {b->shell_origin[3 * s], b->shell_origin[3 * s + 1], b->shell_origin[3 * s + 2]};
    int off = b->shell_prim_off[s];
    libgrpp_shell_t *sh = libgrpp_new_shell(o, b->shell_L[s], b->shell_nprim[s], (double *)b->prim_coef + off,
                                            (double *)b->prim_alpha + off);
    memcpy(sh->cart_list, b->cart_list + 3 * b->shell_cart_off[s], 3 * sh->cart_size * sizeof(int));
    return sh;
}

static libgrpp_potential_t *make_pot(const libgrpp_b200_batch_t *b, int p)
{
    int off = b->pot_prim_off[p];
    return libgrpp_new_potential(b->pot_L[p], b->pot_J[p], b->pot_nprim[p], (int *)b->pot_powers + off,
                                 (double *)b->pot_coef + off, (double *)b->pot_alpha + off);
}

static built_t build(const libgrpp_b200_batch_t *b)
{
    built_t r;
    r.n_shells = b->n_shells;
    r.n_grpps = b->n_grpps;
    r.shells = calloc(b->n_shells, sizeof(void *));
    for (int s = 0; s < b->n_shells; s++) r.shells[s] = make_shell(b, s);
    r.grpps = calloc(b->n_grpps, sizeof(void *));
    for (int g = 0; g < b->n_grpps; g++) {
        libgrpp_grpp_t *G = libgrpp_new_grpp();
        if (b->grpp_UL[g] >= 0) libgrpp_grpp_set_local_potential(G, make_pot(b, b->grpp_UL[g]));
        for (int i = 0; i < b->grpp_n_arep[g]; i++)
            libgrpp_grpp_add_averaged_potential(G, make_pot(b, b->grpp_pot_list[b->grpp_arep_off[g] + i]));
        for (int i = 0; i < b->grpp_n_so[g]; i++)
            libgrpp_grpp_add_spin_orbit_potential(G, make_pot(b, b->grpp_pot_list[b->grpp_so_off[g] + i]));
        for (int i = 0; i < b->grpp_n_oc[g]; i++) {
            int k = b->grpp_oc_off[g] + i;
            libgrpp_grpp_add_outercore_potential(G, make_pot(b, b->grpp_oc_pot[k]), make_shell(b, b->grpp_oc_shell[k]));
        }
        r.grpps[g] = G;
    }
    return r;
}

static void destroy(built_t *r)
{
    for (int s = 0; s < r->n_shells; s++) libgrpp_delete_shell(r->shells[s]);
    for (int g = 0; g < r->n_grpps; g++) libgrpp_delete_grpp(r->grpps[g]);
    free(r->shells);
    free(r->grpps);
}

static int ncart(int L) { return (L + 1) * (L + 2) / 2; }

int grpp_driver_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Full GRPP blocks for tasks [t0, t1) (outputs hold only those tasks' blocks, consecutively).
 * nthreads <= 0 uses every available thread. Returns 0. */
int grpp_driver_full_batch(const libgrpp_b200_batch_t *b, int64_t t0, int64_t t1, int nthreads, double *arep,
                           double *sx, double *sy, double *sz)
{
    int64_t nt = t1 - t0;
    int64_t *off = malloc((nt + 1) * sizeof(int64_t));
    off[0] = 0;
    for (int64_t t = 0; t < nt; t++)
        off[t + 1] = off[t] + (int64_t)ncart(b->shell_L[b->task_a[t0 + t]]) * ncart(b->shell_L[b->task_b[t0 + t]]);
    libgrpp_init();
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
#endif
    {
        built_t r = build(b);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
        for (int64_t t = 0; t < nt; t++) {
            int64_t tt = t0 + t;
            int c = b->task_c[tt];
            double C[3] = {b->centre_origin[3 * c], b->centre_origin[3 * c + 1], b->centre_origin[3 * c + 2]};
            libgrpp_full_grpp_integrals(r.shells[b->task_a[tt]], r.shells[b->task_b[tt]], r.grpps[b->centre_grpp[c]], C,
                                        arep + off[t], sx + off[t], sy + off[t], sz + off[t]);
        }
        destroy(&r);
    }
    (void)nthreads;
    free(off);
    return 0;
}

/* Single-term integrators for parity tests: kind 1 = type 1, 2 = type 2, 3 = spin-orbit
 * (three outputs, unscaled), applied to potential index pot of the batch on task t. */
int grpp_driver_term(const libgrpp_b200_batch_t *b, int64_t t, int kind, int pot, double *o0, double *o1, double *o2)
{
    libgrpp_init();
    libgrpp_shell_t *A = make_shell(b, b->task_a[t]), *B = make_shell(b, b->task_b[t]);
    int c = b->task_c[t];
    double C[3] = {b->centre_origin[3 * c], b->centre_origin[3 * c + 1], b->centre_origin[3 * c + 2]};
    libgrpp_potential_t *P = make_pot(b, pot);
    if (kind == 1) libgrpp_type1_integrals(A, B, C, P, o0);
    else if (kind == 2) libgrpp_type2_integrals(A, B, C, P, o0);
    else libgrpp_spin_orbit_integrals(A, B, C, P, o0, o1, o2);
    libgrpp_delete_potential(P);
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
    return 0;
}

/*
 * Gradient of the four GRPP matrices contracted with a density:
 *   g[m][atom][k] += sum_{tasks} sum_{ij} D[off_A+i, off_B+j] d V^m_ij / d R_atom,k
 * using libgrpp_full_grpp_integrals_gradient for each atom that can contribute
 * (the atoms of A, B and C; every other point gives zero, grpp_integrals_gradient.c:311-321).
 * shell_atom / centre_atom map shells and centres to atoms; bf_off is the basis
 * offset of each shell; D is n_bf x n_bf row-major; g is [4][n_atoms][3] (accumulated).
 */
int grpp_driver_grad_contract(const libgrpp_b200_batch_t *b, int64_t t0, int64_t t1, int nthreads,
                              const int *shell_atom, const int *centre_atom, const double *atom_xyz, int n_atoms,
                              const int *bf_off, int n_bf, const double *D, double *g)
{
    libgrpp_init();
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
#endif
    {
        built_t r = build(b);
        double *gl = calloc(4 * 3 * (size_t)n_atoms, sizeof(double));
        double *buf = malloc(12 * 28 * 28 * sizeof(double) * 4);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
        for (int64_t t = t0; t < t1; t++) {
            int a = b->task_a[t], bb = b->task_b[t], c = b->task_c[t];
            libgrpp_shell_t *A = r.shells[a], *B = r.shells[bb];
            int nA = A->cart_size, nB = B->cart_size, n = nA * nB;
            double C[3] = {b->centre_origin[3 * c], b->centre_origin[3 * c + 1], b->centre_origin[3 * c + 2]};
            int atoms[3] = {shell_atom[a], shell_atom[bb], centre_atom[c]};
            double *gr[4][3];
            double *p = realloc(buf, 12 * (size_t)n * sizeof(double));
            buf = p;
            for (int m = 0; m < 4; m++)
                for (int k = 0; k < 3; k++) gr[m][k] = buf + (m * 3 + k) * n;
            for (int q = 0; q < 3; q++) {
                int at = atoms[q], dup = 0;
                for (int qq = 0; qq < q; qq++) dup |= atoms[qq] == at;
                if (dup) continue;
                double P[3] = {atom_xyz[3 * at], atom_xyz[3 * at + 1], atom_xyz[3 * at + 2]};
                libgrpp_full_grpp_integrals_gradient(A, B, r.grpps[b->centre_grpp[c]], C, P, gr[0], gr[1], gr[2], gr[3]);
                for (int m = 0; m < 4; m++)
                    for (int k = 0; k < 3; k++) {
                        double s = 0.0;
                        for (int i = 0; i < nA; i++)
                            for (int j = 0; j < nB; j++) s += D[(size_t)(bf_off[a] + i) * n_bf + bf_off[bb] + j] * gr[m][k][i * nB + j];
                        gl[(m * n_atoms + at) * 3 + k] += s;
                    }
            }
        }
#ifdef _OPENMP
#pragma omp critical
#endif
        for (int i = 0; i < 12 * n_atoms; i++) g[i] += gl[i];
        free(gl);
        free(buf);
        destroy(&r);
    }
    (void)nthreads;
    return 0;
}
