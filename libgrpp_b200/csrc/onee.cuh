// One-electron integrals over contracted Cartesian Gaussian shell pairs (FP64).
//
//   onee_os_kernel     overlap, kinetic energy and momentum blocks by the Obara-Saika
//                      recurrences (libgrpp/overlap.c:39-139, kinetic.c:48-162,
//                      momentum.c:48-181). One warp per shell pair: three lanes build the
//                      per-axis tables S_ij (and D1_ij or D2_ij) of one primitive pair in
//                      shared memory, then every lane owns Cartesian pairs of the block and
//                      adds c_i c_j N_i N_j S S S with libgrpp's rounding (primitive pairs
//                      outer, products left to right, no fused multiply-add).
//   type1_ang_kernel   k-independent angular factors of the numeric type 1 integral,
//                      A1[lambda][mu][IJK] = sum_rst y_{lambda mu, rst} I(I+r, J+s, K+t)
//                      (libgrpp/angular_integrals.c:35-56), once per batch.
//   type1_num_kernel   numeric type 1 integrals <A| V(|r - C|) |B> of a radially local
//                      potential: a GRPP's U_L, or the electrostatic potential of a point,
//                      charged-ball, Gaussian, Fermi or Fermi-bubble nucleus
//                      (libgrpp/nuclear_models.c). libgrpp's per-primitive-pair scheme
//                      (type1_integrals.c:144-270, radial_type1_integral.c:73-325): the
//                      radial integrals Q(lambda, N) of the pair on the nested Log3 grid
//                      (2047 -> 4095 -> 8191 points, stop at |S_L - S_{L-1}| <= tol), then the
//                      binomial re-centring of both shells on C with the angular factors of
//                      k = -2 (a CA + b CB). One CTA per shell pair, primitive pairs in order:
//                      threads evaluate the integrand at 128 grid points per chunk, then one
//                      thread per (lambda, N) entry adds the chunk's terms in point order, so
//                      each sum is formed in libgrpp's order; threads own Cartesian pairs for
//                      the angular assembly.
#pragma once

#include "angular.cuh"
#include "nucmodel.h"

namespace grpp {

__device__ __forceinline__ double rn_add(double x, double y) { return __dadd_rn(x, y); }
__device__ __forceinline__ double rn_mul(double x, double y) { return __dmul_rn(x, y); }

// ------------------------------------------------------------------ Obara-Saika
enum OneeKind : int { kOneeOverlap = 0, kOneeKinetic = 1, kOneeMomentum = 2 };

struct OneeArgs {
    int n_tasks, kind;
    const int *task_a, *task_b;
    const int64_t *out_off;
    const int *shell_L, *shell_nprim, *shell_prim_off, *shell_cart_off;
    const double *prim_coef, *prim_alpha, *shell_origin;
    const int8_t *cart;
    double *out0, *out1, *out2;
};

constexpr int kOneeWarps = 4;
constexpr int kOneeT = kMaxL + 3;  // table rows 0..L+2 (kinetic)

__global__ void __launch_bounds__(32 * kOneeWarps) onee_os_kernel(OneeArgs a)
{
    __shared__ double sS[kOneeWarps][3][kOneeT][kOneeT];
    __shared__ double sD[kOneeWarps][3][kOneeT][kOneeT];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int t = blockIdx.x * kOneeWarps + w; t < a.n_tasks; t += gridDim.x * kOneeWarps) {
        const int A = a.task_a[t], B = a.task_b[t];
        const int la = a.shell_L[A], lb = a.shell_L[B], nA = ncart(la), nB = ncart(lb), np = nA * nB;
        const int ext = a.kind == kOneeKinetic ? 2 : (a.kind == kOneeMomentum ? 1 : 0);
        const double *oA = a.shell_origin + 3 * A, *oB = a.shell_origin + 3 * B;
        const int8_t *ca = a.cart + 3 * a.shell_cart_off[A], *cb = a.cart + 3 * a.shell_cart_off[B];
        double *o0 = a.out0 + a.out_off[t];
        double *o1 = a.kind == kOneeMomentum ? a.out1 + a.out_off[t] : nullptr;
        double *o2 = a.kind == kOneeMomentum ? a.out2 + a.out_off[t] : nullptr;
        for (int p = lane; p < np; p += 32) {
            o0[p] = 0.0;
            if (o1) {
                o1[p] = 0.0;
                o2[p] = 0.0;
            }
        }
        double(*S)[kOneeT][kOneeT] = sS[w];
        double(*D)[kOneeT][kOneeT] = sD[w];
        const int pa = a.shell_prim_off[A], pb = a.shell_prim_off[B];
        for (int i = 0; i < a.shell_nprim[A]; i++)
            for (int j = 0; j < a.shell_nprim[B]; j++) {
                const double ai = a.prim_alpha[pa + i], aj = a.prim_alpha[pb + j];
                const double cc = rn_mul(a.prim_coef[pa + i], a.prim_coef[pb + j]);
                __syncwarp();
                if (lane < 3) {
                    const int c = lane;
                    const double p = ai + aj, mu = ai * aj / p;
                    const double P = rn_add(rn_mul(ai, oA[c]), rn_mul(aj, oB[c])) / p;
                    const double xab = oA[c] - oB[c], xpa = P - oA[c], xpb = P - oB[c], pf = 1.0 / (2.0 * p);
                    for (int ii = 0; ii <= la + ext; ii++)
                        for (int jj = 0; jj <= lb + ext; jj++) {
                            double s = 0.0;
                            if (ii + jj == 0) {
                                s = sqrt(kPi / p) * exp(-mu * xab * xab);
                            } else if (ii == 0) {
                                s = rn_mul(xpb, S[c][0][jj - 1]);
                                if (jj - 1 > 0) s = rn_add(s, rn_mul(rn_mul(jj - 1, pf), S[c][0][jj - 2]));
                            } else {
                                s = rn_mul(xpa, S[c][ii - 1][jj]);
                                if (ii - 1 > 0) s = rn_add(s, rn_mul(rn_mul(ii - 1, pf), S[c][ii - 2][jj]));
                                if (jj > 0) s = rn_add(s, rn_mul(rn_mul(jj, pf), S[c][ii - 1][jj - 1]));
                            }
                            S[c][ii][jj] = s;
                        }
                    if (a.kind == kOneeKinetic) {
                        for (int ii = 0; ii <= la; ii++)
                            for (int jj = 0; jj <= lb; jj++) {
                                double d = rn_mul(rn_mul(4.0 * ai, ai), S[c][ii + 2][jj]);
                                d = rn_add(d, -rn_mul(rn_mul(2.0 * ai, 2 * ii + 1), S[c][ii][jj]));
                                if (ii >= 2) d = rn_add(d, rn_mul(ii * (ii - 1), S[c][ii - 2][jj]));
                                D[c][ii][jj] = d;
                            }
                    } else if (a.kind == kOneeMomentum) {
                        for (int ii = 0; ii <= la; ii++)
                            for (int jj = 0; jj <= lb; jj++) {
                                double d = rn_mul(2.0 * ai, S[c][ii + 1][jj]);
                                if (ii >= 1) d = rn_add(d, -rn_mul(ii, S[c][ii - 1][jj]));
                                D[c][ii][jj] = d;
                            }
                    }
                }
                __syncwarp();
                const double NA = gaussian_norm(la, ai), NB = gaussian_norm(lb, aj), NN = rn_mul(NA, NB);
                for (int p = lane; p < np; p += 32) {
                    const int m = p / nB, n = p - m * nB;
                    const int x1 = ca[3 * m], y1 = ca[3 * m + 1], z1 = ca[3 * m + 2];
                    const int x2 = cb[3 * n], y2 = cb[3 * n + 1], z2 = cb[3 * n + 2];
                    const double Sx = S[0][x1][x2], Sy = S[1][y1][y2], Sz = S[2][z1][z2];
                    if (a.kind == kOneeOverlap) {
                        const double v = rn_mul(rn_mul(rn_mul(NN, Sx), Sy), Sz);
                        o0[p] = rn_add(o0[p], rn_mul(cc, v));
                    } else if (a.kind == kOneeKinetic) {
                        const double Dx = D[0][x1][x2], Dy = D[1][y1][y2], Dz = D[2][z1][z2];
                        double s = rn_mul(rn_mul(Dx, Sy), Sz);
                        s = rn_add(s, rn_mul(rn_mul(Sx, Dy), Sz));
                        s = rn_add(s, rn_mul(rn_mul(Sx, Sy), Dz));
                        const double v = rn_mul(rn_mul(-0.5 * NA, NB), s);
                        o0[p] = rn_add(o0[p], rn_mul(cc, v));
                    } else {
                        const double Dx = D[0][x1][x2], Dy = D[1][y1][y2], Dz = D[2][z1][z2];
                        const double mNN = rn_mul(-NA, NB);
                        o0[p] = rn_add(o0[p], rn_mul(cc, rn_mul(rn_mul(rn_mul(mNN, Dx), Sy), Sz)));
                        o1[p] = rn_add(o1[p], rn_mul(cc, rn_mul(rn_mul(rn_mul(mNN, Sx), Dy), Sz)));
                        o2[p] = rn_add(o2[p], rn_mul(cc, rn_mul(rn_mul(rn_mul(mNN, Sx), Sy), Dz)));
                    }
                }
            }
    }
}

// ------------------------------------------------------------------ numeric type 1
constexpr int kT1Threads = 128;
constexpr int kT1MaxLam = 12;       // L_A + L_B <= 12

struct Type1NumArgs {
    int n_tasks, model;
    const int *task_a, *task_b, *task_c;
    const int64_t *out_off;
    const int *shell_L, *shell_nprim, *shell_prim_off, *shell_cart_off;
    const double *prim_coef, *prim_alpha, *shell_origin;
    const int8_t *cart;
    const double *centre_origin;
    const double *centre_param;        // [n_centres][4]: Z and the model's parameters
    const int *centre_pot_off, *centre_pot_n;  // kPotGrpp: the centre's U_L terms
    const int *pot_pow;
    const double *pot_coef, *pot_alpha;
    const double *fermi;               // [kFermiNX][kFermiNK]
    const double *ang1;                // type1_ang_kernel output for lmax_tab
    int lmax_tab;
    double tol;                        // radial stop tolerance (libgrpp_params.radial_tolerance)
    double pair_skip;                  // primitive pairs with |c_i c_j| below it are skipped
    double *out;
};

// A1 layout for lmax_tab = Lt: [lambda (0..Lt)][mu (0..2 Lt)][IJK index among I+J+K <= Lt]
__host__ __device__ inline int64_t ang1_index(int Lt, int lam, int mu_off, int ijk)
{
    return ((int64_t)lam * (2 * Lt + 1) + mu_off) * n_abc(Lt) + ijk;
}

__global__ void type1_ang_kernel(int Lt, double *A1)
{
    const int64_t n = (int64_t)(Lt + 1) * (2 * Lt + 1) * n_abc(Lt);
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int ijk = (int)(e % n_abc(Lt));
        const int mu_off = (int)((e / n_abc(Lt)) % (2 * Lt + 1));
        const int lam = (int)(e / ((int64_t)n_abc(Lt) * (2 * Lt + 1)));
        const int mu = mu_off - lam;
        double v = 0.0;
        if (mu <= lam) {
            // (I, J, K) of index ijk: lexicographic among I+J+K <= Lt
            int I = 0, J = 0, K = 0, q = 0;
            for (int a = 0; a <= Lt && q <= ijk; a++)
                for (int b = 0; a + b <= Lt && q <= ijk; b++)
                    for (int c = 0; a + b + c <= Lt && q <= ijk; c++, q++)
                        if (q == ijk) {
                            I = a;
                            J = b;
                            K = c;
                        }
            const int nc = ncart(lam);
            const int8_t *cc = c_tab.rsh_comb + 3 * c_tab.rsh_comb_off[lam];
            const double *y = c_tab.rsh_coef + c_tab.rsh_off[lam] + (mu + lam) * nc;
            for (int r = 0; r < nc; r++) v = rn_add(v, rn_mul(y[r], usp_integral(I + cc[3 * r], J + cc[3 * r + 1], K + cc[3 * r + 2])));
        }
        A1[e] = v;
    }
}

// dynamic shared memory of type1_num_kernel (doubles)
__host__ __device__ inline int t1_smem_doubles(int lmax)
{
    const int ne = (lmax + 1) * (lmax + 1);
    return kT1Threads * (1 + 2 * (lmax + 1))   // wpg, M_lambda, r^N per chunk point
           + 3 * ne                             // running sums, previous level sums, active flags
           + (lmax + 1) * (2 * lmax + 1)        // S_lambda,mu(k)
           + (lmax + 1) * n_abc(lmax);          // omega[lambda][IJK]
}

__global__ void __launch_bounds__(kT1Threads) type1_num_kernel(Type1NumArgs a)
{
    extern __shared__ double t1_sm[];
    const int tid = threadIdx.x;
    for (int t = blockIdx.x; t < a.n_tasks; t += gridDim.x) {
        const int A = a.task_a[t], B = a.task_b[t], C = a.task_c[t];
        const int la = a.shell_L[A], lb = a.shell_L[B], nA = ncart(la), nB = ncart(lb), np = nA * nB;
        const int lmax = la + lb, ne = (lmax + 1) * (lmax + 1);
        double *wpg = t1_sm, *bes = wpg + kT1Threads, *rpw = bes + kT1Threads * (lmax + 1);
        double *sum = rpw + kT1Threads * (lmax + 1), *prev = sum + ne, *act = prev + ne;
        double *rsh = act + ne, *om = rsh + (lmax + 1) * (2 * lmax + 1);
        const double *oA = a.shell_origin + 3 * A, *oB = a.shell_origin + 3 * B, *oC = a.centre_origin + 3 * C;
        const int8_t *ca = a.cart + 3 * a.shell_cart_off[A], *cb = a.cart + 3 * a.shell_cart_off[B];
        const double *prm = a.centre_param + 4 * C;
        double *out = a.out + a.out_off[t];
        for (int p = tid; p < np; p += kT1Threads) out[p] = 0.0;
        const double CAx = oC[0] - oA[0], CAy = oC[1] - oA[1], CAz = oC[2] - oA[2];
        const double CBx = oC[0] - oB[0], CBy = oC[1] - oB[1], CBz = oC[2] - oB[2];
        const double CA2 = CAx * CAx + CAy * CAy + CAz * CAz, CB2 = CBx * CBx + CBy * CBy + CBz * CBz;
        const int pa = a.shell_prim_off[A], pb = a.shell_prim_off[B];
        for (int i = 0; i < a.shell_nprim[A]; i++)
            for (int j = 0; j < a.shell_nprim[B]; j++) {
                const double ci = a.prim_coef[pa + i], cj = a.prim_coef[pb + j];
                if (fabs(ci * cj) < a.pair_skip) continue;
                const double ai = a.prim_alpha[pa + i], aj = a.prim_alpha[pb + j];
                const double kv[3] = {-2.0 * (ai * CAx + aj * CBx), -2.0 * (ai * CAy + aj * CBy), -2.0 * (ai * CAz + aj * CBz)};
                const double k = sqrt(kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2]);
                const double Dabc = 4 * kPi * gaussian_norm(la, ai) * gaussian_norm(lb, aj);
                __syncthreads();
                for (int e = tid; e < ne; e += kT1Threads) {
                    sum[e] = 0.0;
                    act[e] = 1.0;
                }
                // ---- radial integrals, level by level
                int any = 1;
                for (int level = 0; level < 3 && any; level++) {
                    const int nr = level == 0 ? 2047 : (level == 1 ? 4095 : 8191);
                    const int npts = level == 0 ? nr : (nr + 1) / 2;
                    __syncthreads();
                    if (level > 0)
                        for (int e = tid; e < ne; e += kT1Threads)
                            if (act[e] != 0.0) {
                                prev[e] = sum[e];
                                sum[e] = 0.5 * sum[e];
                            }
                    for (int c0 = 0; c0 < npts; c0 += kT1Threads) {
                        __syncthreads();
                        const int q = c0 + tid;
                        if (q < npts) {
                            const int ip = level == 0 ? q + 1 : 2 * q + 1;
                            const double xi = ip / (nr + 1.0), xi3 = xi * xi * xi, ln = log(1 - xi3);
                            const double R = 5.0, R3 = R * R * R;
                            const double w = 3 * R3 * xi * xi * ln * ln / ((1 - xi3) * (nr + 1.0)), r = -R * ln;
                            double pot;
                            if (a.model == kPotGrpp) {
                                pot = 0.0;
                                const int o = a.centre_pot_off[C];
                                const double r2 = r * r;
                                for (int u = 0; u < a.centre_pot_n[C]; u++)
                                    pot = rn_add(pot, rn_mul(rn_mul(a.pot_coef[o + u], pow(r, (double)(a.pot_pow[o + u] - 2))),
                                                             exp(-a.pot_alpha[o + u] * r2)));
                            } else {
                                pot = nuclear_potential(a.model, prm, r, a.fermi);
                            }
                            const double power = rn_add(rn_add(rn_add(rn_mul(k, r), -rn_mul(rn_mul(ai + aj, r), r)),
                                                               -rn_mul(ai, CA2)),
                                                        -rn_mul(aj, CB2));
                            const double gto = Dabc * exp(power);
                            wpg[tid] = w * pot * gto;
                            double M[kT1MaxLam + 1];
                            bessel_scaled_row<kT1MaxLam>(lmax, r * k, M);
                            for (int l = 0; l <= lmax; l++) bes[l * kT1Threads + tid] = M[l];
                            for (int n = 0; n <= lmax; n++) rpw[n * kT1Threads + tid] = pow(r, (double)n);
                        }
                        __syncthreads();
                        const int cn = min(kT1Threads, npts - c0);
                        for (int e = tid; e < ne; e += kT1Threads) {
                            if (act[e] == 0.0) continue;
                            const int lam = e / (lmax + 1), n = e - lam * (lmax + 1);
                            double s = sum[e];
                            for (int u = 0; u < cn; u++)
                                s = rn_add(s, rn_mul(rn_mul(wpg[u], rpw[n * kT1Threads + u]), bes[lam * kT1Threads + u]));
                            sum[e] = s;
                        }
                    }
                    __syncthreads();
                    if (level > 0) {
                        for (int e = tid; e < ne; e += kT1Threads)
                            if (act[e] != 0.0 && fabs(sum[e] - prev[e]) <= a.tol) act[e] = 0.0;
                        __syncthreads();
                        any = 0;
                        for (int e = 0; e < ne; e++)
                            if (act[e] != 0.0) any = 1;
                    }
                }
                __syncthreads();
                // ---- angular factors at k/|k| (spherical_harmonics.c:172-220)
                {
                    const double len = k;
                    double ux = 0.0, uy = 0.0, uz = 0.0;
                    if (len > kZeroThresh) {
                        ux = kv[0] / len;
                        uy = kv[1] / len;
                        uz = kv[2] / len;
                    }
                    const int st = 2 * lmax + 1;
                    for (int e = tid; e < (lmax + 1) * st; e += kT1Threads) {
                        const int l = e / st, mu = e % st - l;
                        double v = 0.0;
                        if (mu <= l) {
                            const int nc = ncart(l);
                            const int8_t *cc = c_tab.rsh_comb + 3 * c_tab.rsh_comb_off[l];
                            const double *y = c_tab.rsh_coef + c_tab.rsh_off[l] + (mu + l) * nc;
                            for (int q = 0; q < nc; q++) {
                                double px = 1.0, py = 1.0, pz = 1.0;
                                for (int s = 0; s < cc[3 * q]; s++) px *= ux;
                                for (int s = 0; s < cc[3 * q + 1]; s++) py *= uy;
                                for (int s = 0; s < cc[3 * q + 2]; s++) pz *= uz;
                                v = rn_add(v, rn_mul(rn_mul(rn_mul(y[q], px), py), pz));
                            }
                        }
                        rsh[e] = v;
                    }
                    __syncthreads();
                    const int nijk = n_abc(lmax);
                    for (int e = tid; e < (lmax + 1) * nijk; e += kT1Threads) {
                        const int l = e / nijk, ijk = e - l * nijk;
                        // (I, J, K) of the batch table index: the same triple under lmax_tab
                        int I = 0, J = 0, K = 0, q = 0;
                        for (int x = 0; x <= lmax && q <= ijk; x++)
                            for (int y = 0; x + y <= lmax && q <= ijk; y++)
                                for (int z = 0; x + y + z <= lmax && q <= ijk; z++, q++)
                                    if (q == ijk) {
                                        I = x;
                                        J = y;
                                        K = z;
                                    }
                        const int tij = abc_index(a.lmax_tab, I, J, K);
                        double v = 0.0;
                        for (int mu = -l; mu <= l; mu++)
                            v = rn_add(v, rn_mul(a.ang1[ang1_index(a.lmax_tab, l, mu + l, tij)], rsh[l * st + mu + l]));
                        om[e] = v;
                    }
                }
                __syncthreads();
                // ---- binomial re-centring of both shells on C (type1_integrals.c:206-262)
                const double cc = ci * cj;
                const int nijk = n_abc(lmax);
                for (int p = tid; p < np; p += kT1Threads) {
                    const int m = p / nB, n = p - m * nB;
                    const int nxA = ca[3 * m], nyA = ca[3 * m + 1], nzA = ca[3 * m + 2];
                    const int nxB = cb[3 * n], nyB = cb[3 * n + 1], nzB = cb[3 * n + 2];
                    double chi = 0.0;
                    for (int aa = 0; aa <= nxA; aa++) {
                        const double C1 = c_tab.binom[nxA * kBinN + aa], P1 = pow(CAx, (double)(nxA - aa));
                        for (int bb = 0; bb <= nyA; bb++) {
                            const double C2 = c_tab.binom[nyA * kBinN + bb], P2 = pow(CAy, (double)(nyA - bb));
                            for (int cq = 0; cq <= nzA; cq++) {
                                const double C3 = c_tab.binom[nzA * kBinN + cq], P3 = pow(CAz, (double)(nzA - cq));
                                for (int d = 0; d <= nxB; d++) {
                                    const double C4 = c_tab.binom[nxB * kBinN + d], P4 = pow(CBx, (double)(nxB - d));
                                    for (int e = 0; e <= nyB; e++) {
                                        const double C5 = c_tab.binom[nyB * kBinN + e], P5 = pow(CBy, (double)(nyB - e));
                                        for (int f = 0; f <= nzB; f++) {
                                            const double C6 = c_tab.binom[nzB * kBinN + f], P6 = pow(CBz, (double)(nzB - f));
                                            const double factor = C1 * C2 * C3 * C4 * C5 * C6 * P1 * P2 * P3 * P4 * P5 * P6;
                                            if (fabs(factor) < 1e-13) continue;
                                            const int N = aa + bb + cq + d + e + f;
                                            const int ijk = abc_index(lmax, aa + d, bb + e, cq + f);
                                            double sq = 0.0;
                                            for (int lam = 0; lam <= lmax; lam++) {
                                                const double Q = sum[lam * (lmax + 1) + N];
                                                if (fabs(Q) < 1e-16) continue;
                                                sq = rn_add(sq, rn_mul(om[lam * nijk + ijk], Q));
                                            }
                                            chi = rn_add(chi, rn_mul(factor, sq));
                                        }
                                    }
                                }
                            }
                        }
                    }
                    out[p] = rn_add(out[p], rn_mul(cc, chi));
                }
            }
    }
}

}  // namespace grpp
