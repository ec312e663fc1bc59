// Nuclear charge models: electrostatic potentials of a point, charged-ball, Gaussian,
// Fermi and Fermi-bubble nucleus (libgrpp/nuclear_models.c), for host and device code.
//
// The Fermi forms use S_k(x) = sum_{i >= 1} (-1)^i exp(i x) / i^k (x <= 0), evaluated as
// libgrpp does (specfunc_fermi_sk.c:42-90): exponential tails below x = -10, else a
// 3rd-order Taylor expansion about the 0.005 grid x0 = -10 + 0.005 i of a table holding
// S_j(x0) for j = -2..7 (S_j' = S_{j-1}). The table is generated from the function's
// definition by build_fermi_table (tables.cpp).
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define GRPP_HD __host__ __device__
#else
#define GRPP_HD
#endif

namespace grpp {

constexpr int kFermiNX = 2001;  // x = -10.000 .. 0.000 step 0.005
constexpr int kFermiNK = 10;    // S_j, j = -2 .. 7
constexpr double kNucPi = 3.14159265358979323846;

// radially local potentials of the numeric type 1 path
enum Type1Pot : int {
    kPotGrpp = 0,         // sum_k c_k r^(n_k - 2) exp(-zeta_k r^2) (libgrpp_potential_value, potential.c:70-81)
    kPotPointNum = 1,     // -Z / r
    kPotBall = 2,         // charged ball of rms radius R
    kPotGauss = 3,        // Gaussian charge of rms radius R
    kPotFermi = 4,        // Fermi distribution (c, a)
    kPotFermiBubble = 5   // Fermi distribution with a quadratic hole (c, a, k)
};

GRPP_HD inline double fermi_sk(int k, double x, const double *tab)
{
    if (x <= -30) return -1.0 * exp(x);
    if (x <= -14) return -1.0 * exp(x) + 1.0 * exp(2 * x) / pow(2.0, (double)k);
    if (x <= -10) return -1.0 * exp(x) + 1.0 * exp(2 * x) / pow(2.0, (double)k) - 1.0 * exp(3 * x) / pow(3.0, (double)k);
    const int i0 = (int)(floor((x + 10.0) * 200) + 1e-10);
    const double x0 = -10.0 + i0 * 0.005, dx = x - x0;
    const double *d = tab + (long)i0 * kFermiNK;
    if (i0 == kFermiNX - 1) return d[k + 2];
    const double dx2 = dx * dx, dx3 = dx2 * dx;
    return d[k + 2] + d[k + 1] * dx + d[k] * dx2 * 0.5 + d[k - 1] * dx3 * (1.0 / 6.0);
}

GRPP_HD inline double fermi_norm(double c, double a, const double *tab)
{
    const double a2 = a * a, a3 = a * a * a, c2 = c * c, c3 = c * c * c;
    return 1.0 + kNucPi * kNucPi * a2 / c2 - 6.0 * a3 / c3 * fermi_sk(3, -c / a, tab);
}

GRPP_HD inline double fermi_bubble_norm(double c, double a, double k, const double *tab)
{
    const double a2 = a * a, a3 = a * a2, a4 = a * a3, a5 = a * a4;
    const double c2 = c * c, c3 = c * c2, c4 = c * c3, c5 = c * c4;
    (void)c3;
    return fermi_norm(c, a, tab) + 3.0 / 5.0 * k + 2.0 * kNucPi * kNucPi * a2 * k / c2 +
           7.0 * kNucPi * kNucPi * kNucPi * kNucPi * a4 * k / (5.0 * c4) - 72.0 * a5 * k / c5 * fermi_sk(5, -c / a, tab);
}

GRPP_HD inline double coulomb_ball(double r, double Z, double R_rms)
{
    const double R0 = sqrt(5.0 / 3.0) * R_rms;
    return r <= R0 ? -Z / (2.0 * R0) * (3.0 - r * r / (R0 * R0)) : -Z / r;
}

GRPP_HD inline double coulomb_gauss(double r, double Z, double R_rms)
{
    const double xi = 3.0 / (2.0 * R_rms * R_rms);
    return -Z / r * erf(sqrt(xi) * r);
}

GRPP_HD inline double coulomb_fermi(double r, double Z, double c, double a, const double *tab)
{
    const double a2 = a * a, a3 = a * a * a, c3 = c * c * c;
    const double N = fermi_norm(c, a, tab);
    if (r > c) {
        const double S2 = fermi_sk(2, (c - r) / a, tab), S3 = fermi_sk(3, (c - r) / a, tab);
        return -Z / (N * r) * (N + 3 * a2 * r / c3 * S2 + 6 * a3 / c3 * S3);
    }
    const double P2 = fermi_sk(2, (r - c) / a, tab), P3 = fermi_sk(3, (r - c) / a, tab);
    const double S3 = fermi_sk(3, -c / a, tab), r3 = r * r * r;
    return -Z / (N * r) *
           (1.5 * r / c - r3 / (2 * c3) + kNucPi * kNucPi * a2 * r / (2 * c3) - 3 * a2 * r / c3 * P2 + 6 * a3 / c3 * (P3 - S3));
}

GRPP_HD inline double coulomb_fermi_bubble(double r, double Z, double c, double a, double k, const double *tab)
{
    const double Nk = fermi_bubble_norm(c, a, k, tab);
    double F0, F2;
    if (r < c) {
        const double x = (r - c) / a;
        const double S2 = fermi_sk(2, x, tab), S3 = fermi_sk(3, x, tab), S4 = fermi_sk(4, x, tab), S5 = fermi_sk(5, x, tab);
        F0 = -pow(r, 3) / 6.0 - r * a * a * S2 + 2.0 * pow(a, 3) * S3 + r * c * c / 2.0 + kNucPi * kNucPi / 6.0 * r * a * a -
             2.0 * pow(a, 3) * fermi_sk(3, -c / a, tab);
        F2 = -pow(r, 5) / 20.0 - pow(r, 3) * pow(a, 2) * S2 + 6.0 * pow(r, 2) * pow(a, 3) * S3 - 18.0 * r * pow(a, 4) * S4 +
             24.0 * pow(a, 5) * S5 + r * pow(c, 4) / 4.0 + r * kNucPi * kNucPi * c * c * a * a / 2.0 +
             r * pow(a, 4) * pow(kNucPi, 4) * 7.0 / 60.0 - 24.0 * pow(a, 5) * fermi_sk(5, -c / a, tab);
    } else {
        const double x = (c - r) / a;
        const double S2 = fermi_sk(2, x, tab), S3 = fermi_sk(3, x, tab), S4 = fermi_sk(4, x, tab), S5 = fermi_sk(5, x, tab);
        F0 = pow(c, 3) / 3.0 + kNucPi * kNucPi / 3.0 * c * a * a - 2.0 * pow(a, 3) * fermi_sk(3, -c / a, tab) +
             r * a * a * S2 + 2.0 * pow(a, 3) * S3;
        F2 = pow(c, 5) / 5.0 + 2.0 * pow(c, 3) * a * a * kNucPi * kNucPi / 3.0 + 7.0 * pow(a, 4) * c * pow(kNucPi, 4) / 15.0 -
             24.0 * pow(a, 5) * fermi_sk(5, -c / a, tab) + pow(a, 2) * pow(r, 3) * S2 + 6.0 * pow(a, 3) * pow(r, 2) * S3 +
             18.0 * r * pow(a, 4) * S4 + 24.0 * pow(a, 5) * S5;
    }
    return -Z / (Nk * r) * 3.0 / pow(c, 3) * (F0 + k / (c * c) * F2);
}

// prm = {Z, model parameters...}: ball and Gaussian {Z, R_rms}, Fermi {Z, c, a}, bubble {Z, c, a, k}
GRPP_HD inline double nuclear_potential(int model, const double *prm, double r, const double *tab)
{
    switch (model) {
    case kPotPointNum: return -prm[0] / r;
    case kPotBall: return coulomb_ball(r, prm[0], prm[1]);
    case kPotGauss: return coulomb_gauss(r, prm[0], prm[1]);
    case kPotFermi: return coulomb_fermi(r, prm[0], prm[1], prm[2], tab);
    default: return coulomb_fermi_bubble(r, prm[0], prm[1], prm[2], prm[3], tab);
    }
}

}  // namespace grpp
