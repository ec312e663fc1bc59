// Fortran ABI of the engine: the symbols libgrpp's Fortran bindings call
// (libgrpp/fortran.c:29-1083), same names (trailing underscore), same argument lists
// (every argument by address, 32-bit integers). Each one builds libgrpp objects from its
// arguments and calls the C API of this library, so the integrals run on the GPU.
//
// Two entry points have no C-API counterpart here: the outercore terms split into
//   part 1  U|nlj><nlj| + |nlj><nlj|U for one outercore shell, and
//   part 2  |nlj><nlj| U |n'lj><n'lj| for a pair of outercore shells
// (libgrpp/outercore_integrals.c:147-390). Part 2 needs only the overlaps <A|oc> and
// <oc'|B> (GPU, libgrpp_overlap_integrals) and the one-centre integral delta; it is formed
// here with libgrpp's factors. Part 1 is the GPU outercore term of the single shell
// (libgrpp_outercore_potential_integrals, which is part 1 + part 2 of that shell with
// itself) minus that shell's part 2. Both add their result to the caller's arrays, as
// libgrpp's parts do (outercore_integrals.c:228-258, 366-388).
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/libgrpp.h"
#include "../../include/libgrpp_f90.h"
#include "grpp_common.cuh"
#include "tables.h"

namespace {

const grpp::HostTables &host_tables()
{
    static grpp::HostTables t;
    static std::once_flag once;
    std::call_once(once, [] { grpp::build_host_tables(t); });
    return t;
}

std::vector<int> ints(const int32_t *p, int n) { return std::vector<int>(p, p + n); }

libgrpp_shell_t *shell(double *o, const int32_t *L, const int32_t *n, double *c, double *a)
{
    return libgrpp_new_shell(o, *L, *n, c, a);
}

double dfact(int n)
{
    double r = 1.0;
    for (int k = n; k > 1; k -= 2) r *= k;
    return r;
}

// outercore_integrals.c:481-510: sqrt(2^(L+5/2) / Gamma(L+3/2)) alpha^(3/4+L/2)
double radial_gto_norm(int L, double a)
{
    const double g = dfact(2 * L + 1) * std::sqrt(M_PI) / std::pow(2.0, L + 1);
    return std::sqrt(std::pow(2.0, L + 2.5) / g) * std::pow(a, 0.75 + L / 2.0);
}

// outercore_integrals.c:425-478: <oc1| U |oc2> on one centre, analytic
double one_centre(const libgrpp_shell_t *s1, const libgrpp_shell_t *s2, const libgrpp_potential_t *p)
{
    const int L = p->L;
    double sum = 0.0;
    for (int i = 0; i < s1->num_primitives; i++)
        for (int j = 0; j < s2->num_primitives; j++) {
            const double f = radial_gto_norm(L, s1->alpha[i]) * radial_gto_norm(L, s2->alpha[j]) * s1->coeffs[i] * s2->coeffs[j];
            for (int k = 0; k < p->num_primitives; k++) {
                const double a = s1->alpha[i] + s2->alpha[j] + p->alpha[k];
                const int n = p->powers[k];
                double v;
                if (n % 2 == 0) {
                    const int kk = L + n / 2;
                    v = dfact(2 * kk - 1) / (std::pow(2.0, kk + 1) * std::pow(a, kk)) * std::sqrt(M_PI / a);
                } else {
                    const int kk = L + (n - 1) / 2;
                    double fk = 1.0;
                    for (int q = 2; q <= kk; q++) fk *= q;
                    v = fk / (2.0 * std::pow(a, kk + 1));
                }
                sum += f * p->coeffs[k] * v;
            }
        }
    return sum;
}

// real spherical / Cartesian coefficient of one oc-shell component over its angular norm
double oc_sph(int L, int m, const int *c)
{
    const grpp::HostTables &t = host_tables();
    const int nc = (L + 1) * (L + 2) / 2;
    const int8_t *comb = t.rsh_comb.data() + 3 * t.rsh_comb_off[L];
    int ic = 0;
    while (ic < nc && !(comb[3 * ic] == c[0] && comb[3 * ic + 1] == c[1] && comb[3 * ic + 2] == c[2])) ic++;
    const double y = t.rsh_coef[t.rsh_off[L] + (m + L) * nc + ic];
    return y / (1.0 / (2.0 * std::sqrt(M_PI)) * std::sqrt(dfact(2 * L + 1)));
}

double lmat(int L, int comp, int m1, int m2)
{
    const grpp::HostTables &t = host_tables();
    const int d = 2 * L + 1;
    return t.lmat[t.lmat_off[L] + comp * d * d + (m1 + L) * d + (m2 + L)];
}

// part 2 of a pair of outercore shells (outercore_integrals.c:277-390), added to the outputs
void oc_part2(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, libgrpp_potential_t *p1, libgrpp_shell_t *oc1,
              libgrpp_potential_t *p2, libgrpp_shell_t *oc2, double *arep, double *sx, double *sy, double *sz)
{
    if (p1->L != p2->L || p1->J != p2->J) return;
    const int L = p1->L, nA = A->cart_size, nB = B->cart_size, no = oc1->cart_size, d = 2 * L + 1;
    const double J = p1->J / 2.0;
    const double delta = 0.5 * (one_centre(oc1, oc2, p1) + one_centre(oc1, oc2, p2));
    for (int x = 0; x < 3; x++) oc1->origin[x] = oc2->origin[x] = C[x];
    std::vector<double> t1(no * nB), t2(nA * no), Sa(nA * d), Sb(d * nB);
    libgrpp_overlap_integrals(oc2, B, t1.data());
    libgrpp_overlap_integrals(A, oc1, t2.data());
    for (int i = 0; i < nA; i++)
        for (int m = 0; m < d; m++) {
            double s = 0.0;
            for (int c = 0; c < no; c++) s += oc_sph(L, m - L, oc1->cart_list + 3 * c) * t2[i * no + c];
            Sa[i * d + m] = s;
        }
    for (int j = 0; j < nB; j++)
        for (int m = 0; m < d; m++) {
            double s = 0.0;
            for (int c = 0; c < no; c++) s += oc_sph(L, m - L, oc1->cart_list + 3 * c) * t1[c * nB + j];
            Sb[m * nB + j] = s;
        }
    const double farep = (J < L) ? L / (2.0 * L + 1) : (L + 1) / (2.0 * L + 1);
    const double fso = (J < L) ? -2.0 / (2 * L + 1) : +2.0 / (2 * L + 1);
    double *so[3] = {sx, sy, sz};
    for (int i = 0; i < nA; i++)
        for (int j = 0; j < nB; j++) {
            double s = 0.0;
            for (int m = 0; m < d; m++) s += Sa[i * d + m] * Sb[m * nB + j];
            arep[i * nB + j] += -1.0 * delta * farep * s;
            for (int c = 0; c < 3; c++) {
                double v = 0.0;
                for (int m1 = 0; m1 < d; m1++)
                    for (int m2 = 0; m2 < d; m2++) v += Sa[i * d + m1] * lmat(L, c, m1 - L, m2 - L) * Sb[m2 * nB + j];
                so[c][i * nB + j] += -1.0 * delta * fso * v;
            }
        }
}

}  // namespace

#pragma GCC visibility push(default)
extern "C" {

void libgrpp_set_default_parameters_(void) { libgrpp_set_default_parameters(); }
void libgrpp_set_radial_tolerance_(const double *t) { libgrpp_set_radial_tolerance(*t); }
void libgrpp_set_angular_screening_tolerance_(const double *t) { libgrpp_set_angular_screening_tolerance(*t); }
void libgrpp_set_modified_bessel_tolerance_(const double *t) { libgrpp_set_modified_bessel_tolerance(*t); }
void libgrpp_set_cartesian_order_(const int32_t *order) { libgrpp_set_cartesian_order(*order); }
void libgrpp_init_(void) { libgrpp_init(); }
void libgrpp_finalize_(void) { libgrpp_finalize(); }

void libgrpp_type1_integrals_(double *oA, int32_t *LA, int32_t *nA, double *cA, double *aA, double *oB, int32_t *LB,
                              int32_t *nB, double *cB, double *aB, double *C, int32_t *np, int32_t *pw, double *pc,
                              double *pa, double *matrix)
{
    std::vector<int> p = ints(pw, *np);
    libgrpp_potential_t *pot = libgrpp_new_potential(0, 0, *np, p.data(), pc, pa);
    libgrpp_shell_t *A = shell(oA, LA, nA, cA, aA), *B = shell(oB, LB, nB, cB, aB);
    libgrpp_type1_integrals(A, B, C, pot, matrix);
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
    libgrpp_delete_potential(pot);
}

void libgrpp_type2_integrals_(double *oA, int32_t *LA, int32_t *nA, double *cA, double *aA, double *oB, int32_t *LB,
                              int32_t *nB, double *cB, double *aB, double *C, int32_t *L, int32_t *np, int32_t *pw,
                              double *pc, double *pa, double *matrix)
{
    std::vector<int> p = ints(pw, *np);
    libgrpp_potential_t *pot = libgrpp_new_potential(*L, 0, *np, p.data(), pc, pa);
    libgrpp_shell_t *A = shell(oA, LA, nA, cA, aA), *B = shell(oB, LB, nB, cB, aB);
    libgrpp_type2_integrals(A, B, C, pot, matrix);
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
    libgrpp_delete_potential(pot);
}

void libgrpp_spin_orbit_integrals_(double *oA, int32_t *LA, int32_t *nA, double *cA, double *aA, double *oB, int32_t *LB,
                                   int32_t *nB, double *cB, double *aB, double *C, int32_t *L, int32_t *np, int32_t *pw,
                                   double *pc, double *pa, double *sx, double *sy, double *sz)
{
    std::vector<int> p = ints(pw, *np);
    libgrpp_potential_t *pot = libgrpp_new_potential(*L, 0, *np, p.data(), pc, pa);
    libgrpp_shell_t *A = shell(oA, LA, nA, cA, aA), *B = shell(oB, LB, nB, cB, aB);
    libgrpp_spin_orbit_integrals(A, B, C, pot, sx, sy, sz);
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
    libgrpp_delete_potential(pot);
}

void libgrpp_outercore_potential_integrals_part_1_(double *oA, int32_t *LA, int32_t *nA, double *cA, double *aA, double *oB,
                                                   int32_t *LB, int32_t *nB, double *cB, double *aB, double *C,
                                                   int32_t *L, int32_t *J, int32_t *np, int32_t *pw, double *pc,
                                                   double *pa, int32_t *n_oc, double *c_oc, double *a_oc, double *arep,
                                                   double *sx, double *sy, double *sz)
{
    std::vector<int> p = ints(pw, *np);
    libgrpp_potential_t *pot = libgrpp_new_potential(*L, *J, *np, p.data(), pc, pa);
    libgrpp_shell_t *A = shell(oA, LA, nA, cA, aA), *B = shell(oB, LB, nB, cB, aB);
    libgrpp_shell_t *oc = libgrpp_new_shell(C, *L, *n_oc, c_oc, a_oc);
    // the outercore term of this one shell is part 1 + part 2 of the shell with itself;
    // like libgrpp's part 1, the result is added to the caller's arrays
    const int n = A->cart_size * B->cart_size;
    std::vector<double> t[4], q[4];
    for (int k = 0; k < 4; k++) {
        t[k].assign(n, 0.0);
        q[k].assign(n, 0.0);
    }
    libgrpp_outercore_potential_integrals(A, B, C, 1, &pot, &oc, t[0].data(), t[1].data(), t[2].data(), t[3].data());
    oc_part2(A, B, C, pot, oc, pot, oc, q[0].data(), q[1].data(), q[2].data(), q[3].data());
    double *outs[4] = {arep, sx, sy, sz};
    for (int k = 0; k < 4; k++)
        for (int i = 0; i < n; i++) outs[k][i] += t[k][i] - q[k][i];
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
    libgrpp_delete_shell(oc);
    libgrpp_delete_potential(pot);
}

void libgrpp_outercore_potential_integrals_part_2_(
    double *oA, int32_t *LA, int32_t *nA, double *cA, double *aA, double *oB, int32_t *LB, int32_t *nB, double *cB,
    double *aB, double *C, int32_t *L1, int32_t *J1, int32_t *np1, int32_t *pw1, double *pc1, double *pa1, int32_t *no1,
    double *co1, double *ao1, int32_t *L2, int32_t *J2, int32_t *np2, int32_t *pw2, double *pc2, double *pa2, int32_t *no2,
    double *co2, double *ao2, double *arep, double *sx, double *sy, double *sz)
{
    std::vector<int> p1 = ints(pw1, *np1), p2 = ints(pw2, *np2);
    libgrpp_potential_t *u1 = libgrpp_new_potential(*L1, *J1, *np1, p1.data(), pc1, pa1);
    libgrpp_potential_t *u2 = libgrpp_new_potential(*L2, *J2, *np2, p2.data(), pc2, pa2);
    libgrpp_shell_t *A = shell(oA, LA, nA, cA, aA), *B = shell(oB, LB, nB, cB, aB);
    libgrpp_shell_t *oc1 = libgrpp_new_shell(C, *L1, *no1, co1, ao1), *oc2 = libgrpp_new_shell(C, *L2, *no2, co2, ao2);
    oc_part2(A, B, C, u1, oc1, u2, oc2, arep, sx, sy, sz);  // added to the caller's arrays, as libgrpp does
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
    libgrpp_delete_shell(oc1);
    libgrpp_delete_shell(oc2);
    libgrpp_delete_potential(u1);
    libgrpp_delete_potential(u2);
}

void libgrpp_type1_integrals_gradient_(double *oA, int32_t *LA, int32_t *nA, double *cA, double *aA, double *oB,
                                       int32_t *LB, int32_t *nB, double *cB, double *aB, double *C, int32_t *np,
                                       int32_t *pw, double *pc, double *pa, double *D, double *gx, double *gy, double *gz)
{
    std::vector<int> p = ints(pw, *np);
    libgrpp_potential_t *pot = libgrpp_new_potential(0, 0, *np, p.data(), pc, pa);
    libgrpp_shell_t *A = shell(oA, LA, nA, cA, aA), *B = shell(oB, LB, nB, cB, aB);
    double *g[3] = {gx, gy, gz};
    libgrpp_type1_integrals_gradient(A, B, C, pot, D, g);
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
    libgrpp_delete_potential(pot);
}

void libgrpp_type2_integrals_gradient_(double *oA, int32_t *LA, int32_t *nA, double *cA, double *aA, double *oB,
                                       int32_t *LB, int32_t *nB, double *cB, double *aB, double *C, int32_t *L,
                                       int32_t *np, int32_t *pw, double *pc, double *pa, double *D, double *gx, double *gy,
                                       double *gz)
{
    std::vector<int> p = ints(pw, *np);
    libgrpp_potential_t *pot = libgrpp_new_potential(*L, 0, *np, p.data(), pc, pa);
    libgrpp_shell_t *A = shell(oA, LA, nA, cA, aA), *B = shell(oB, LB, nB, cB, aB);
    double *g[3] = {gx, gy, gz};
    libgrpp_type2_integrals_gradient(A, B, C, pot, D, g);
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
    libgrpp_delete_potential(pot);
}

void libgrpp_spin_orbit_integrals_gradient_(double *oA, int32_t *LA, int32_t *nA, double *cA, double *aA, double *oB,
                                            int32_t *LB, int32_t *nB, double *cB, double *aB, double *C, int32_t *L,
                                            int32_t *np, int32_t *pw, double *pc, double *pa, double *D, double *xx,
                                            double *xy, double *xz, double *yx, double *yy, double *yz, double *zx,
                                            double *zy, double *zz)
{
    std::vector<int> p = ints(pw, *np);
    libgrpp_potential_t *pot = libgrpp_new_potential(*L, 0, *np, p.data(), pc, pa);
    libgrpp_shell_t *A = shell(oA, LA, nA, cA, aA), *B = shell(oB, LB, nB, cB, aB);
    double *gx[3] = {xx, xy, xz}, *gy[3] = {yx, yy, yz}, *gz[3] = {zx, zy, zz};
    libgrpp_spin_orbit_integrals_gradient(A, B, C, pot, D, gx, gy, gz);
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
    libgrpp_delete_potential(pot);
}

// fortran.c:641-687: <x^n y^l z^m | x^n' y^l' z^m'> of two contracted Gaussians, one component each
void evaluate_overlap_integral_contracted_(double *oA, int32_t *nxA, int32_t *nyA, int32_t *nzA, int32_t *npA,
                                           double *cA, double *aA, double *oB, int32_t *nxB, int32_t *nyB,
                                           int32_t *nzB, int32_t *npB, double *cB, double *aB, double *value)
{
    libgrpp_shell_t *A = libgrpp_new_shell(oA, *nxA + *nyA + *nzA, *npA, cA, aA);
    libgrpp_shell_t *B = libgrpp_new_shell(oB, *nxB + *nyB + *nzB, *npB, cB, aB);
    A->cart_size = 1;
    A->cart_list[0] = *nxA;
    A->cart_list[1] = *nyA;
    A->cart_list[2] = *nzA;
    B->cart_size = 1;
    B->cart_list[0] = *nxB;
    B->cart_list[1] = *nyB;
    B->cart_list[2] = *nzB;
    libgrpp_overlap_integrals(A, B, value);
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
}

// fortran.c:689-703: sqrt((2L-1)!!) / sqrt(<x^L|x^L>) of a contracted radial Gaussian
void radial_gto_norm_factor_(int32_t *L, int32_t *np, double *c, double *a, double *norm)
{
    double S = 0.0, origin[3] = {0, 0, 0};
    int32_t zero = 0;
    evaluate_overlap_integral_contracted_(origin, L, &zero, &zero, np, c, a, origin, L, &zero, &zero, np, c, a, &S);
    *norm = std::sqrt(dfact(2 * (*L) - 1)) / std::sqrt(S);
}

void libgrpp_overlap_integrals_(double *oA, int32_t *LA, int32_t *nA, double *cA, double *aA, double *oB, int32_t *LB,
                                int32_t *nB, double *cB, double *aB, double *matrix)
{
    libgrpp_shell_t *A = shell(oA, LA, nA, cA, aA), *B = shell(oB, LB, nB, cB, aB);
    libgrpp_overlap_integrals(A, B, matrix);
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
}

void libgrpp_kinetic_energy_integrals_(double *oA, int32_t *LA, int32_t *nA, double *cA, double *aA, double *oB,
                                       int32_t *LB, int32_t *nB, double *cB, double *aB, double *matrix)
{
    libgrpp_shell_t *A = shell(oA, LA, nA, cA, aA), *B = shell(oB, LB, nB, cB, aB);
    libgrpp_kinetic_energy_integrals(A, B, matrix);
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
}

void libgrpp_momentum_integrals_(double *oA, int32_t *LA, int32_t *nA, double *cA, double *aA, double *oB, int32_t *LB,
                                 int32_t *nB, double *cB, double *aB, double *mx, double *my, double *mz)
{
    libgrpp_shell_t *A = shell(oA, LA, nA, cA, aA), *B = shell(oB, LB, nB, cB, aB);
    libgrpp_momentum_integrals(A, B, mx, my, mz);
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
}

void libgrpp_nuclear_attraction_integrals_(double *oA, int32_t *LA, int32_t *nA, double *cA, double *aA, double *oB,
                                           int32_t *LB, int32_t *nB, double *cB, double *aB, double *C, int32_t *charge,
                                           int32_t *model, double *params, double *matrix)
{
    libgrpp_shell_t *A = shell(oA, LA, nA, cA, aA), *B = shell(oB, LB, nB, cB, aB);
    libgrpp_nuclear_attraction_integrals(A, B, C, *charge, *model, params, matrix);
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
}

void libgrpp_nuclear_attraction_integrals_point_charge_(double *oA, int32_t *LA, int32_t *nA, double *cA, double *aA,
                                                        double *oB, int32_t *LB, int32_t *nB, double *cB, double *aB,
                                                        double *C, int32_t *charge, double *matrix)
{
    libgrpp_shell_t *A = shell(oA, LA, nA, cA, aA), *B = shell(oB, LB, nB, cB, aB);
    libgrpp_nuclear_attraction_integrals_point_charge(A, B, C, *charge, matrix);
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
}

void libgrpp_nuclear_attraction_integrals_charged_ball_(double *oA, int32_t *LA, int32_t *nA, double *cA, double *aA,
                                                        double *oB, int32_t *LB, int32_t *nB, double *cB, double *aB,
                                                        double *C, int32_t *charge, double *r_rms, double *matrix)
{
    libgrpp_shell_t *A = shell(oA, LA, nA, cA, aA), *B = shell(oB, LB, nB, cB, aB);
    libgrpp_nuclear_attraction_integrals_charged_ball(A, B, C, *charge, *r_rms, matrix);
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
}

void libgrpp_nuclear_attraction_integrals_gaussian_model_(double *oA, int32_t *LA, int32_t *nA, double *cA, double *aA,
                                                          double *oB, int32_t *LB, int32_t *nB, double *cB, double *aB,
                                                          double *C, int32_t *charge, double *r_rms, double *matrix)
{
    libgrpp_shell_t *A = shell(oA, LA, nA, cA, aA), *B = shell(oB, LB, nB, cB, aB);
    libgrpp_nuclear_attraction_integrals_gaussian_model(A, B, C, *charge, *r_rms, matrix);
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
}

void libgrpp_nuclear_attraction_integrals_fermi_model_(double *oA, int32_t *LA, int32_t *nA, double *cA, double *aA,
                                                       double *oB, int32_t *LB, int32_t *nB, double *cB, double *aB,
                                                       double *C, int32_t *charge, double *fc, double *fa, double *matrix)
{
    libgrpp_shell_t *A = shell(oA, LA, nA, cA, aA), *B = shell(oB, LB, nB, cB, aB);
    libgrpp_nuclear_attraction_integrals_fermi_model(A, B, C, *charge, *fc, *fa, matrix);
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
}

void libgrpp_nuclear_attraction_integrals_fermi_bubble_model_(double *oA, int32_t *LA, int32_t *nA, double *cA,
                                                              double *aA, double *oB, int32_t *LB, int32_t *nB,
                                                              double *cB, double *aB, double *C, int32_t *charge,
                                                              double *fc, double *fa, double *fk, double *matrix)
{
    libgrpp_shell_t *A = shell(oA, LA, nA, cA, aA), *B = shell(oB, LB, nB, cB, aB);
    libgrpp_nuclear_attraction_integrals_fermi_bubble_model(A, B, C, *charge, *fc, *fa, *fk, matrix);
    libgrpp_delete_shell(A);
    libgrpp_delete_shell(B);
}

void libgrpp_estimate_nuclear_rms_radius_johnson_1985_(int32_t *A, double *R) { *R = libgrpp_estimate_nuclear_rms_radius_johnson_1985(*A); }
void libgrpp_estimate_nuclear_rms_radius_golovko_2008_(int32_t *A, double *R) { *R = libgrpp_estimate_nuclear_rms_radius_golovko_2008(*A); }
void libgrpp_estimate_fermi_model_parameters_(double *R, double *c, double *a, int32_t *err)
{
    *err = libgrpp_estimate_fermi_model_parameters(*R, c, a);
}
void libgrpp_charge_density_ball_(double *r, double *Z, double *R, double *rho) { *rho = libgrpp_charge_density_ball(*r, *Z, *R); }
void libgrpp_charge_density_gaussian_(double *r, double *Z, double *R, double *rho) { *rho = libgrpp_charge_density_gaussian(*r, *Z, *R); }
void libgrpp_charge_density_fermi_(double *r, double *Z, double *c, double *a, double *rho)
{
    *rho = libgrpp_charge_density_fermi(*r, *Z, *c, *a);
}
void libgrpp_charge_density_fermi_bubble_(double *r, double *Z, double *c, double *a, double *k, double *rho)
{
    *rho = libgrpp_charge_density_fermi_bubble(*r, *Z, *c, *a, *k);
}
void libgrpp_coulomb_potential_point_(double *r, double *Z, double *v) { *v = libgrpp_coulomb_potential_point(*r, *Z); }
void libgrpp_coulomb_potential_ball_(double *r, double *Z, double *R, double *v) { *v = libgrpp_coulomb_potential_ball(*r, *Z, *R); }
void libgrpp_coulomb_potential_gaussian_(double *r, double *Z, double *R, double *v)
{
    *v = libgrpp_coulomb_potential_gaussian(*r, *Z, *R);
}
void libgrpp_coulomb_potential_fermi_(double *r, double *Z, double *c, double *a, double *v)
{
    *v = libgrpp_coulomb_potential_fermi(*r, *Z, *c, *a);
}
void libgrpp_coulomb_potential_fermi_bubble_(double *r, double *Z, double *c, double *a, double *k, double *v)
{
    *v = libgrpp_coulomb_potential_fermi_bubble(*r, *Z, *c, *a, *k);
}
void libgrpp_rms_radius_fermi_(int32_t *Z, double *c, double *a, double *r) { *r = libgrpp_rms_radius_fermi(*Z, *c, *a); }
void libgrpp_rms_radius_fermi_bubble_(int32_t *Z, double *c, double *a, double *k, double *r)
{
    *r = libgrpp_rms_radius_fermi_bubble(*Z, *c, *a, *k);
}

}  // extern "C"
#pragma GCC visibility pop
