// Angular part of the semilocal (type 2) and spin-orbit integrals, outercore
// assembly and the final per-task combination of all GRPP terms.
//
// Reference algorithm: libgrpp/type2_integrals.c:34-243,
// libgrpp/spin_orbit_integrals.c:41-288, libgrpp/angular_integrals.c:63-130,
// libgrpp/outercore_integrals.c:83-390, libgrpp/full_grpp_integrals.c:27-104.
//
// Restructuring (same sums, same order, same skip rules):
//  * the type 2 angular integral
//      omega(l,L,m,a,b,c; k) = sum_mu S_{l mu}(k) sum_uvw y_{Lm,uvw} sum_rst y_{l mu,rst} I(a+r+u, b+s+v, c+t+w)
//    is split into the k-independent tensor Atab[l,mu,L,m,abc] (the inner two
//    sums, built once per (L, l_shell) and cached on the device) and the sum
//    over mu done per shell and centre;
//  * the reference's inner quantity for one binomial term (a..f),
//      V[abc][def] = sum_{l1,l2} Q[l1][l2][|abc|+|def|] sum_m omega_A omega_B,
//    depends only on (abc, def): it is computed once per task and potential
//    and reused by every Cartesian pair (i, j), which then only forms
//      gamma_ij = 16 pi^2 sum_{abc<=i, def<=j} C(..) CA^(..) CB^(..) V[abc][def].
// Threshold skips of the reference (|factor| < 1e-13, |Q| < 1e-16,
// |omega_1| < 1e-16 for type 2; 1e-14 everywhere for spin-orbit;
// |S_{l mu}|, |y| < 1e-14 inside omega) are applied at the same places.
#pragma once

#include "grpp_common.cuh"
#include "specfunc.cuh"

namespace grpp {

// lexicographic index of (a, b, c), a+b+c <= l (a outer, then b, then c)
__host__ __device__ inline int abc_index(int l, int a, int b, int c)
{
    // triples with first component < a: sum_{q<a} (l-q+1)(l-q+2)/2 = tet(l+1) - tet(l+1-a),
    // tet(m) = m(m+1)(m+2)/6; then those with first a and second < b
    const int m = l + 1, r = l + 1 - a;
    return (m * (m + 1) * (m + 2) - r * (r + 1) * (r + 2)) / 6 + b * (l - a + 1) - b * (b - 1) / 2 + c;
}
__host__ __device__ constexpr int n_abc(int l) { return (l + 1) * (l + 2) * (l + 3) / 6; }

// lambda slots for |abc| = n: lambda = lo, lo+2, ..., L+n
__host__ __device__ inline int lam_lo(int L, int n) { return L - n >= 0 ? L - n : ((L + n) & 1); }
__host__ __device__ inline int lam_count(int L, int n) { return (L + n - lam_lo(L, n)) / 2 + 1; }
__host__ __device__ inline int lam_slots(int L, int l)
{
    int m = 0;
    for (int n = 0; n <= l; n++) m = m > lam_count(L, n) ? m : lam_count(L, n);
    return m;
}

// Atab layout per (L, l): [abc][slot][mu (0..2*lmax_lam)][m (0..2L)], lmax_lam = L + l
__host__ __device__ inline int64_t atab_size(int L, int l)
{
    return (int64_t)n_abc(l) * lam_slots(L, l) * (2 * (L + l) + 1) * (2 * L + 1);
}

__device__ __forceinline__ double usp_integral(int i, int j, int k)
{
    if ((i & 1) || (j & 1) || (k & 1)) return 0.0;
    return 4 * kPi * dfact(i - 1) * dfact(j - 1) * dfact(k - 1) / dfact(i + j + k + 1);
}

#ifndef GRPP_NO_ANGULAR_KERNELS
// Atab[abc][slot][mu][m] = sum_uvw sum_rst y_{Lm,uvw} y_{lam mu,rst} I(a+r+u, ...),
// terms skipped when |y| < 1e-14, accumulated in the reference's order
// (angular_integrals.c:78-106: uvw outer, rst inner, y_lam * y_L * usp).
__global__ void atab_kernel(int L, int l, double *out)
{
    const int nslot = lam_slots(L, l), nmu = 2 * (L + l) + 1, nm = 2 * L + 1;
    const int64_t total = (int64_t)n_abc(l) * nslot * nmu * nm;
    for (int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; id < total; id += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = id;
        const int m = (int)(r % nm) - L;
        r /= nm;
        const int mui = (int)(r % nmu);
        r /= nmu;
        const int slot = (int)(r % nslot);
        const int abc = (int)(r / nslot);
        // decode abc
        int a = 0, b = 0, c = 0, idx = abc;
        for (a = 0; a <= l; a++) {
            const int cnt = (l - a + 1) * (l - a + 2) / 2;
            if (idx < cnt) break;
            idx -= cnt;
        }
        for (b = 0; b <= l - a; b++) {
            const int cnt = l - a - b + 1;
            if (idx < cnt) break;
            idx -= cnt;
        }
        c = idx;
        const int n = a + b + c;
        double val = 0.0;
        const int lam = lam_lo(L, n) + 2 * slot;
        if (slot < lam_count(L, n) && mui <= 2 * lam) {
            const int mu = mui - lam;
            const int nuvw = ncart(L), nrst = ncart(lam);
            const double *yL = c_tab.rsh_coef + c_tab.rsh_off[L] + (m + L) * nuvw;
            const double *yl = c_tab.rsh_coef + c_tab.rsh_off[lam] + (mu + lam) * nrst;
            const int8_t *cu = c_tab.rsh_comb + 3 * c_tab.rsh_comb_off[L];
            const int8_t *cr = c_tab.rsh_comb + 3 * c_tab.rsh_comb_off[lam];
            for (int iu = 0; iu < nuvw; iu++) {
                const double y1 = yL[iu];
                if (fabs(y1) < kZeroThresh) continue;
                for (int ir = 0; ir < nrst; ir++) {
                    const double y2 = yl[ir];
                    if (fabs(y2) < kZeroThresh) continue;
                    const double usp = usp_integral(a + cr[3 * ir] + cu[3 * iu], b + cr[3 * ir + 1] + cu[3 * iu + 1],
                                                    c + cr[3 * ir + 2] + cu[3 * iu + 2]);
                    val += y2 * y1 * usp;
                }
            }
        }
        out[id] = val;
    }
}

#endif  // GRPP_NO_ANGULAR_KERNELS

// ---- outercore spherical projections ---------------------------------------------
// S_sph[i][m] = sum_icart coef[m][icart] S_cart[i][icart] (outercore_integrals.c:514-525),
// coef = spherical_to_cartesian_coef(L, m, r, s, t) / ang_norm_factor(r, s, t) (:165-177).
struct OcProjArgs {
    int n;                       // number of (proj, oc) blocks
    const int *blk_shell;        // basis shell
    const int *blk_ocshell;      // outercore shell
    const int64_t *blk_cart_off; // offset of the n_s x ncart(oc) Cartesian block (S and U scratch)
    const int64_t *blk_sph_off;  // offset of the n_s x (2L+1) spherical block
    const int *shell_L, *shell_cart_off;
    const int8_t *cart;
    const double *S_cart, *U_cart;
    double *S_sph, *U_sph;
};

__device__ inline double sph_coef_oc(int L, int m, int r, int s, int t)
{
    // find the combo (r,s,t) in the RSH table of L (lexicographic), divide by the
    // angular norm (2 sqrt(pi))^-1 sqrt((2L+1)!!)
    const int nc = ncart(L);
    const int8_t *cc = c_tab.rsh_comb + 3 * c_tab.rsh_comb_off[L];
    double y = 0.0;
    for (int q = 0; q < nc; q++)
        if (cc[3 * q] == r && cc[3 * q + 1] == s && cc[3 * q + 2] == t) y = c_tab.rsh_coef[c_tab.rsh_off[L] + (m + L) * nc + q];
    const double an = 1.0 / (2.0 * sqrt(kPi)) * sqrt(dfact(2 * L + 1));
    return y / an;
}

#ifndef GRPP_NO_ANGULAR_KERNELS
__global__ void oc_proj_kernel(OcProjArgs a)
{
    for (int blk = blockIdx.x; blk < a.n; blk += gridDim.x) {
        const int s = a.blk_shell[blk], o = a.blk_ocshell[blk];
        const int ns = ncart(a.shell_L[s]), L = a.shell_L[o], no = ncart(L), d = 2 * L + 1;
        const int8_t *co = a.cart + 3 * a.shell_cart_off[o];
        for (int e = threadIdx.x; e < ns * d; e += blockDim.x) {
            const int i = e / d, m = e % d - L;
            double ss = 0.0, su = 0.0;
            for (int ic = 0; ic < no; ic++) {
                const double u = sph_coef_oc(L, m, co[3 * ic], co[3 * ic + 1], co[3 * ic + 2]);
                ss += u * a.S_cart[a.blk_cart_off[blk] + i * no + ic];
                su += u * a.U_cart[a.blk_cart_off[blk] + i * no + ic];
            }
            a.S_sph[a.blk_sph_off[blk] + i * d + m + L] = ss;
            a.U_sph[a.blk_sph_off[blk] + i * d + m + L] = su;
        }
    }
}
#endif  // GRPP_NO_ANGULAR_KERNELS

// ---- final per-task assembly -----------------------------------------------------

constexpr int kFinThreads = 128;       // omega tables; the assembly kernel is instantiated for 128, 256, 512
constexpr int kFinMaxPairs = 1024;     // Cartesian pairs of one task block (i x i = 784)
constexpr int kFinElemPerThread = kFinMaxPairs / kFinThreads;
constexpr int kFinMaxLam = 24;
constexpr int kLmatPairs = 100;  // (m1, m2) pairs of the L matrices with a non-zero component: 10L - 4 <= 96 for L <= 10
constexpr int kFinMaxSl = 24;         // semilocal potentials per centre
constexpr int kFinMaxOc = 32;         // outercore shells per centre

struct FinalArgs {
    int n_tasks;
    const int *task_a, *task_b, *task_c;
    const int64_t *task_out_off;
    const uint8_t *task_has_ul;
    const int64_t *task_q_off;        // -1 if no semilocal part
    const int *task_proj_a, *task_proj_b; // outercore projection index of (A,C), (B,C), -1 if none
    const int *shell_L, *shell_cart_off, *shell_prim_off;
    const double *prim_alpha, *shell_origin;
    const int8_t *cart;
    const double *centre_origin;
    const int *centre_grpp;
    const int *grpp_sl_off, *grpp_sl_n, *grpp_n_arep, *sl_pot;
    const int *grpp_oc_off, *grpp_n_oc, *oc_L, *oc_J;  // per outercore entry (grpp_oc_off indexing)
    const double *oc_delta;                          // per grpp: n_oc x n_oc matrix, offset grpp_delta_off
    const int *grpp_delta_off;
    const int *pot_L;
    const double *Q;
    const int64_t *atab_off;          // [(kMaxL+2) * (kMaxL+2)] offsets of Atab per (L, l), -1 if absent
    const double *atab;
    const int64_t *proj_off;          // per projection: offset of its first oc block in S_sph / U_sph
    const double *S_sph, *U_sph;
    int raw_so;                       // 1: spin-orbit output without the 2/(2L+1) factor
    double *arep, *so_x, *so_y, *so_z;
    int *status;
    // dynamic schedule: blocks pop positions from *queue (zeroed before the launch) and take
    // task order[position], largest estimated work first; queue may be null: static round-robin
    const int *order;
    int *queue;
    // omega tables per (shell, centre) pair (omega_tab_kernel): for each semilocal potential
    // of the centre's GRPP in order, omega[abc][slot][m] of that side, from om_off[pair];
    // task_fpa / task_fpb: the pairs (A, C) and (B, C) of a task. omtab null: computed here
    const double *omtab;
    const int64_t *om_off;
    const int *task_fpa, *task_fpb;
};

// RSH values S_{l mu}(k/|k|) for l = 0..lmax (spherical_harmonics.c:227-280); out[l*(2*kFinMaxLam+1) + mu + l]
__device__ void rsh_values(int lmax, const double *k, double *out, int tid, int nthr)
{
    const double len = sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]);
    double ux = 0.0, uy = 0.0, uz = 0.0;
    if (len > kZeroThresh) {
        const double inv = 1.0 / len;
        ux = k[0] * inv;
        uy = k[1] * inv;
        uz = k[2] * inv;
    }
    for (int e = tid; e < (lmax + 1) * (2 * kFinMaxLam + 1); e += nthr) {
        const int l = e / (2 * kFinMaxLam + 1), mu = e % (2 * kFinMaxLam + 1) - l;
        if (mu > l) continue;
        const int nc = ncart(l);
        const int8_t *cc = c_tab.rsh_comb + 3 * c_tab.rsh_comb_off[l];
        const double *y = c_tab.rsh_coef + c_tab.rsh_off[l] + (mu + l) * nc;
        double v = 0.0;
        for (int q = 0; q < nc; q++) {
            double px = 1.0, py = 1.0, pz = 1.0;
            for (int i = 0; i < cc[3 * q]; i++) px *= ux;
            for (int i = 0; i < cc[3 * q + 1]; i++) py *= uy;
            for (int i = 0; i < cc[3 * q + 2]; i++) pz *= uz;
            v += y[q] * (px * py * pz);
        }
        out[e] = v;
    }
}

}  // namespace grpp

namespace grpp {

struct FinalSmem {
    // offsets (in doubles) of the dynamic shared regions, computed on the host
    int rsh_stride;  // 2*lam_max+1
    int n_rsh;       // (lam_max+1) * rsh_stride
    int n_omega;     // per side
    int n_q;
    int n_v;
    int n_w;         // W[j][abc][comp] of the factored re-centring sum (0: not used)
};

__device__ __forceinline__ double lmat_val(int L, int comp, int m1, int m2)
{
    const int d = 2 * L + 1;
    return c_tab.lmat[c_tab.lmat_off[L] + comp * d * d + (m1 + L) * d + (m2 + L)];
}

#ifndef GRPP_NO_ANGULAR_KERNELS
// Omega tables of one side for every (shell, centre) pair: a CTA per pair computes the
// real spherical harmonics of the unit vector along k = -2 a (C - S) (a the shell's first
// exponent) and, for each semilocal potential of the centre's GRPP in order,
// omega[abc][slot][m] = sum_mu S_{lam mu} Atab[abc][slot][mu][m] with the skips of
// angular_integrals.c:78-108 — the same expressions as final_kernel's own evaluation.
// Dynamic shared memory: (lam_max + 1) x sm.rsh_stride doubles.
__global__ void __launch_bounds__(kFinThreads) omega_tab_kernel(FinalArgs a, FinalSmem sm, const int *op_shell,
                                                                const int *op_centre, int n_pairs, double *omtab)
{
    extern __shared__ double rsh[];
    __shared__ double upow[3][kFinMaxLam + 1];
    __shared__ int8_t nabc[n_abc(kMaxL)];
    const int tid = threadIdx.x, rs = sm.rsh_stride;
    for (int pr = blockIdx.x; pr < n_pairs; pr += gridDim.x) {
        const int sx = op_shell[pr], c = op_centre[pr], l = a.shell_L[sx], g = a.centre_grpp[c];
        const int nsl = a.grpp_sl_n[g];
        int lam_max = 0;
        for (int p = 0; p < nsl; p++) lam_max = max(lam_max, a.pot_L[a.sl_pot[a.grpp_sl_off[g] + p]] + l);
        double k[3];
        const double al = a.prim_alpha[a.shell_prim_off[sx]];
        for (int d = 0; d < 3; d++) k[d] = -2.0 * (al * (a.centre_origin[3 * c + d] - a.shell_origin[3 * sx + d]));
        const double len = sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]);
        double u[3] = {0, 0, 0};
        if (len > kZeroThresh) {
            const double inv = 1.0 / len;
            for (int d = 0; d < 3; d++) u[d] = k[d] * inv;
        }
        __syncthreads();  // the previous pair's readers of upow, nabc and rsh are done
        if (tid < 3) {
            const double ud = tid == 0 ? u[0] : (tid == 1 ? u[1] : u[2]);
            double pw = 1.0;
            upow[tid][0] = pw;
            for (int i = 1; i <= lam_max; i++) {
                pw *= ud;
                upow[tid][i] = pw;
            }
        }
        for (int e = tid; e < n_abc(l); e += kFinThreads) {
            int idx = e, aa, bb;
            for (aa = 0; aa <= l; aa++) {
                const int cnt = (l - aa + 1) * (l - aa + 2) / 2;
                if (idx < cnt) break;
                idx -= cnt;
            }
            for (bb = 0; bb <= l - aa; bb++) {
                const int cnt = l - aa - bb + 1;
                if (idx < cnt) break;
                idx -= cnt;
            }
            nabc[e] = (int8_t)(aa + bb + idx);
        }
        __syncthreads();
        const int nlm = (lam_max + 1) * (lam_max + 1);
        for (int e = tid; e < nlm; e += kFinThreads) {
            int ll = (int)sqrtf((float)e);
            while (ll * ll > e) ll--;
            while ((ll + 1) * (ll + 1) <= e) ll++;
            const int mu = e - ll * ll - ll;
            const int nc = ncart(ll);
            const int8_t *cc = c_tab.rsh_comb + 3 * c_tab.rsh_comb_off[ll];
            const double *y = c_tab.rsh_coef + c_tab.rsh_off[ll] + (mu + ll) * nc;
            double v = 0.0;
            for (int q = 0; q < nc; q++) v += y[q] * (upow[0][cc[3 * q]] * upow[1][cc[3 * q + 1]] * upow[2][cc[3 * q + 2]]);
            rsh[ll * rs + mu + ll] = v;
        }
        __syncthreads();
        int64_t off = a.om_off[pr];
        for (int p = 0; p < nsl; p++) {
            const int L = a.pot_L[a.sl_pot[a.grpp_sl_off[g] + p]];
            const int sl = lam_slots(L, l), nab = n_abc(l), nm = 2 * L + 1, nmu = 2 * (L + l) + 1;
            const double *At = a.atab + a.atab_off[L * (kMaxL + 2) + l];
            for (int e = tid; e < nab * sl * nm; e += kFinThreads) {
                const int m = e % nm, slot = (e / nm) % sl, abc = e / (nm * sl);
                const int n = nabc[abc];
                double w = 0.0;
                if (slot < lam_count(L, n)) {
                    const int lam = lam_lo(L, n) + 2 * slot;
                    const double *S = rsh + lam * rs;
                    const double *Ap = At + ((int64_t)(abc * sl + slot) * nmu) * nm + m;
                    for (int mu = -lam; mu <= lam; mu++) {
                        const double rv = S[mu + lam];
                        if (fabs(rv) < kZeroThresh) continue;
                        w += Ap[(int64_t)(mu + lam) * nm] * rv;
                    }
                }
                omtab[off + e] = w;
            }
            off += (int64_t)nab * sl * nm;
        }
    }
}

template <int NT>
__global__ void __launch_bounds__(NT) final_kernel(FinalArgs a, FinalSmem sm)
{
    constexpr int EPT = kFinMaxPairs / NT;  // Cartesian pairs per thread
    extern __shared__ double dsm[];
    __shared__ double powA[3][kMaxL + 2], powB[3][kMaxL + 2];
    __shared__ double sCA[3], sCB[3];
    // powers u^0..u^lam of the unit vectors along kA, kB: [side][axis][power], each the same
    // chain of products 1 * u * u ... as the reference's per-term loops
    __shared__ double upow[2][3][kFinMaxLam + 1];
    __shared__ int8_t nabcA[n_abc(kMaxL)], nabcB[n_abc(kMaxL)];  // |abc| of each abc index
    // spin-orbit: the (m1, m2) pairs, in m1-major order, at which some L matrix component is
    // non-zero (spin_orbit_integrals.c:206-222 skips the others), with the three values
    __shared__ int8_t lpm1[kLmatPairs], lpm2[kLmatPairs];
    __shared__ double lpv[3][kLmatPairs];
    __shared__ int s_npair;
    const int tid = threadIdx.x;
    double *rshA = dsm, *rshB = rshA + sm.n_rsh, *omA = rshB + sm.n_rsh, *omB = omA + sm.n_omega, *Qs = omB + sm.n_omega,
           *V = Qs + sm.n_q;
    const int rs = sm.rsh_stride;

    __shared__ int s_next;
    int t_static = blockIdx.x;
    for (;;) {
        int t;
        if (a.queue) {
            __syncthreads();  // every thread has read the previous s_next
            if (tid == 0) {
                const int k = atomicAdd(a.queue, 1);
                s_next = k < a.n_tasks ? a.order[k] : -1;
            }
            __syncthreads();
            t = s_next;
            if (t < 0) break;
        } else {
            if (t_static >= a.n_tasks) break;
            t = a.order ? a.order[t_static] : t_static;
            t_static += gridDim.x;
        }
        const int sa = a.task_a[t], sb = a.task_b[t], c = a.task_c[t];
        const int la = a.shell_L[sa], lb = a.shell_L[sb], nA = ncart(la), nB = ncart(lb), nel = nA * nB;
        const int8_t *cA = a.cart + 3 * a.shell_cart_off[sa], *cB = a.cart + 3 * a.shell_cart_off[sb];
        const int g = a.centre_grpp[c];
        const int64_t oo = a.task_out_off[t];
        __syncthreads();
        if (tid < 3) {
            sCA[tid] = a.centre_origin[3 * c + tid] - a.shell_origin[3 * sa + tid];
            sCB[tid] = a.centre_origin[3 * c + tid] - a.shell_origin[3 * sb + tid];
        }
        __syncthreads();
        if (tid < 3) {
            for (int k = 0; k <= la; k++) powA[tid][k] = pow(sCA[tid], k);
            for (int k = 0; k <= lb; k++) powB[tid][k] = pow(sCB[tid], k);
        }
        double acc[4][EPT];
#pragma unroll
        for (int q = 0; q < EPT; q++) {
            const int e = tid + q * NT;
            acc[0][q] = (e < nel && a.task_has_ul[t]) ? a.arep[oo + e] : 0.0;
            acc[1][q] = acc[2][q] = acc[3][q] = 0.0;
        }

        const int nsl = a.grpp_sl_n[g];
        if (nsl > 0 && a.task_q_off[t] >= 0) {
            int lam_max = 0;
            for (int p = 0; p < nsl; p++) {
                const int Lp = a.pot_L[a.sl_pot[a.grpp_sl_off[g] + p]];
                lam_max = max(lam_max, Lp + max(la, lb));
            }
            double kA[3], kB[3];
            const double alA = a.prim_alpha[a.shell_prim_off[sa]], alB = a.prim_alpha[a.shell_prim_off[sb]];
            for (int d = 0; d < 3; d++) {
                kA[d] = -2.0 * (alA * (a.centre_origin[3 * c + d] - a.shell_origin[3 * sa + d]));
                kB[d] = -2.0 * (alB * (a.centre_origin[3 * c + d] - a.shell_origin[3 * sb + d]));
            }
            __syncthreads();
            // RSH values with stride rs (rsh_values uses 2*kFinMaxLam+1; use a local variant)
            const bool omt = a.omtab != nullptr;
            if (omt) {  // only the |abc| tables are needed: omega comes from the pair tables
                for (int e = tid; e < n_abc(la) + n_abc(lb); e += NT) {
                    const bool sideB = e >= n_abc(la);
                    const int l = sideB ? lb : la;
                    int idx = sideB ? e - n_abc(la) : e, aa, bb;
                    for (aa = 0; aa <= l; aa++) {
                        const int cnt = (l - aa + 1) * (l - aa + 2) / 2;
                        if (idx < cnt) break;
                        idx -= cnt;
                    }
                    for (bb = 0; bb <= l - aa; bb++) {
                        const int cnt = l - aa - bb + 1;
                        if (idx < cnt) break;
                        idx -= cnt;
                    }
                    (sideB ? nabcB : nabcA)[sideB ? e - n_abc(la) : e] = (int8_t)(aa + bb + idx);
                }
            } else {
                const double lenA = sqrt(kA[0] * kA[0] + kA[1] * kA[1] + kA[2] * kA[2]);
                const double lenB = sqrt(kB[0] * kB[0] + kB[1] * kB[1] + kB[2] * kB[2]);
                double uA[3] = {0, 0, 0}, uB[3] = {0, 0, 0};
                if (lenA > kZeroThresh) {
                    const double inv = 1.0 / lenA;
                    for (int d = 0; d < 3; d++) uA[d] = kA[d] * inv;
                }
                if (lenB > kZeroThresh) {
                    const double inv = 1.0 / lenB;
                    for (int d = 0; d < 3; d++) uB[d] = kB[d] * inv;
                }
                if (tid < 6) {
                    const int side = tid / 3, d = tid % 3;
                    const double ud = side ? (d == 0 ? uB[0] : (d == 1 ? uB[1] : uB[2]))
                                           : (d == 0 ? uA[0] : (d == 1 ? uA[1] : uA[2]));
                    double pw = 1.0;
                    upow[side][d][0] = pw;
                    for (int i = 1; i <= lam_max; i++) {
                        pw *= ud;
                        upow[side][d][i] = pw;
                    }
                }
                for (int e = tid; e < n_abc(la) + n_abc(lb); e += NT) {
                    const bool sideB = e >= n_abc(la);
                    const int l = sideB ? lb : la;
                    int idx = sideB ? e - n_abc(la) : e, aa, bb;
                    for (aa = 0; aa <= l; aa++) {
                        const int cnt = (l - aa + 1) * (l - aa + 2) / 2;
                        if (idx < cnt) break;
                        idx -= cnt;
                    }
                    for (bb = 0; bb <= l - aa; bb++) {
                        const int cnt = l - aa - bb + 1;
                        if (idx < cnt) break;
                        idx -= cnt;
                    }
                    (sideB ? nabcB : nabcA)[sideB ? e - n_abc(la) : e] = (int8_t)(aa + bb + idx);
                }
                __syncthreads();
                // (l, mu) pairs e = l^2 + l + mu of both sides
                const int nlm = (lam_max + 1) * (lam_max + 1);
                for (int e = tid; e < 2 * nlm; e += NT) {
                    const int side = e >= nlm, r = side ? e - nlm : e;
                    int l = (int)sqrtf((float)r);
                    while (l * l > r) l--;
                    while ((l + 1) * (l + 1) <= r) l++;
                    const int mu = r - l * l - l;
                    const double(*up)[kFinMaxLam + 1] = upow[side];
                    const int nc = ncart(l);
                    const int8_t *cc = c_tab.rsh_comb + 3 * c_tab.rsh_comb_off[l];
                    const double *y = c_tab.rsh_coef + c_tab.rsh_off[l] + (mu + l) * nc;
                    double v = 0.0;
                    for (int q = 0; q < nc; q++) v += y[q] * (up[0][cc[3 * q]] * up[1][cc[3 * q + 1]] * up[2][cc[3 * q + 2]]);
                    (side ? rshB : rshA)[l * rs + mu + l] = v;
                }
            }
            // The binomial factor of a re-centring term is F_A(abc) F_B(def) (binomials times powers
            // of CA, CB components), so the sum over (a..f) factors as sum_abc F_A W[abc] with
            // W[abc] = sum_def F_B V[abc][def]. libgrpp skips terms whose factor is below its
            // threshold (1e-13; 1e-14 for spin-orbit); when a lower bound of every non-zero factor
            // clears twice that, only exact zeros are skipped and the factored sum has the same
            // terms. Otherwise the term-by-term loop runs.
            bool fact = sm.n_w > 0;
            if (fact) {
                double mA = 1.0, mB = 1.0;
                for (int d = 0; d < 3; d++) {
                    const double xa = fabs(powA[d][la]), xb = fabs(powB[d][lb]);
                    if (sCA[d] != 0.0 && xa < 1.0) mA *= xa;
                    if (sCB[d] != 0.0 && xb < 1.0) mB *= xb;
                }
                fact = mA * mB >= 2e-13;
            }
            const int64_t qbase = a.task_q_off[t];
            int64_t qoff = 0;
            int64_t omoA = omt ? a.om_off[a.task_fpa[t]] : 0, omoB = omt ? a.om_off[a.task_fpb[t]] : 0;
            const int n_arep = a.grpp_n_arep[g];
            for (int p = 0; p < nsl; p++) {
                const int L = a.pot_L[a.sl_pot[a.grpp_sl_off[g] + p]];
                const bool so = p >= n_arep;
                const int d1 = L + la + 1, d2 = L + lb + 1, dn = la + lb + 1, nm = 2 * L + 1;
                const int slA = lam_slots(L, la), slB = lam_slots(L, lb);
                const int nabA = n_abc(la), nabB = n_abc(lb);
                const int nmuA = 2 * (L + la) + 1, nmuB = 2 * (L + lb) + 1;
                const double *AtA = a.atab + a.atab_off[L * (kMaxL + 2) + la];
                const double *AtB = a.atab + a.atab_off[L * (kMaxL + 2) + lb];
                __syncthreads();
                // omega tables: omega[abc][slot][m] = sum_mu S_{lam mu} Atab (angular_integrals.c:78-108)
                if (omt) {
                    for (int e = tid; e < nabA * slA * nm; e += NT) omA[e] = a.omtab[omoA + e];
                    for (int e = tid; e < nabB * slB * nm; e += NT) omB[e] = a.omtab[omoB + e];
                    omoA += nabA * slA * nm;
                    omoB += nabB * slB * nm;
                }
                for (int e = tid; !omt && e < nabA * slA * nm + nabB * slB * nm; e += NT) {
                    const bool sideB = e >= nabA * slA * nm;
                    const int r = sideB ? e - nabA * slA * nm : e;
                    const int sl = sideB ? slB : slA, nab = sideB ? nabB : nabA, l = sideB ? lb : la;
                    const int m = r % nm, slot = (r / nm) % sl, abc = r / (nm * sl);
                    (void)nab;
                    (void)l;
                    const int n = sideB ? nabcB[abc] : nabcA[abc];
                    double w = 0.0;
                    if (slot < lam_count(L, n)) {
                        const int lam = lam_lo(L, n) + 2 * slot;
                        const double *S = (sideB ? rshB : rshA) + lam * rs;
                        const double *At = (sideB ? AtB : AtA) + ((int64_t)(abc * sl + slot) * (sideB ? nmuB : nmuA)) * nm + m;
                        for (int mu = -lam; mu <= lam; mu++) {
                            const double rv = S[mu + lam];
                            if (fabs(rv) < kZeroThresh) continue;
                            w += At[(int64_t)(mu + lam) * nm] * rv;
                        }
                    }
                    (sideB ? omB : omA)[r] = w;
                }
                for (int e = tid; e < d1 * d2 * dn; e += NT) Qs[e] = a.Q[qbase + qoff + e];
                qoff += (int64_t)d1 * d2 * dn;
                if (so && tid == 0) {
                    int np = 0;
                    for (int m1 = -L; m1 <= L; m1++)
                        for (int m2 = -L; m2 <= L; m2++) {
                            const double lx = lmat_val(L, 0, m1, m2), ly = lmat_val(L, 1, m1, m2), lz = lmat_val(L, 2, m1, m2);
                            if (fabs(lx) < kZeroThresh && fabs(ly) < kZeroThresh && fabs(lz) < kZeroThresh) continue;
                            if (np < kLmatPairs) {
                                lpm1[np] = (int8_t)(m1 + L);
                                lpm2[np] = (int8_t)(m2 + L);
                                lpv[0][np] = lx;
                                lpv[1][np] = ly;
                                lpv[2][np] = lz;
                            }
                            np++;
                        }
                    s_npair = np;  // never above kLmatPairs for L <= 10 (10L - 4 pairs)
                }
                __syncthreads();

                const int ncomp = so ? 3 : 1;
                const double thrF = so ? kZeroThresh : 1e-13, thrQ = so ? kZeroThresh : 1e-16, thrW = so ? kZeroThresh : 1e-16;
                const int rows = max(1, min(nabA, sm.n_v / (nabB * ncomp)));
                double gam[3][EPT];
#pragma unroll
                for (int q = 0; q < EPT; q++) gam[0][q] = gam[1][q] = gam[2][q] = 0.0;

                for (int r0 = 0; r0 < nabA; r0 += rows) {
                    const int r1 = min(nabA, r0 + rows);
                    __syncthreads();
                    // V[abc][def] (type2_integrals.c:174-196, spin_orbit_integrals.c:197-224)
                    for (int e = tid; e < (r1 - r0) * nabB; e += NT) {
                        const int abc = r0 + e / nabB, def = e % nabB;
                        const int n1 = nabcA[abc], n2 = nabcB[def], N = n1 + n2;
                        double v0 = 0.0, v1 = 0.0, v2 = 0.0;
                        const int c1 = lam_count(L, n1), c2 = lam_count(L, n2);
                        for (int s1 = 0; s1 < c1; s1++) {
                            const int l1 = lam_lo(L, n1) + 2 * s1;
                            const double *w1 = omA + (abc * slA + s1) * nm;
                            for (int s2 = 0; s2 < c2; s2++) {
                                const int l2 = lam_lo(L, n2) + 2 * s2;
                                const double QN = Qs[(l1 * d2 + l2) * dn + N];
                                if (fabs(QN) < thrQ) continue;
                                const double *w2 = omB + (def * slB + s2) * nm;
                                if (!so) {
                                    double sa2 = 0.0;
                                    for (int m = 0; m < nm; m++) {
                                        if (fabs(w1[m]) < thrW) continue;
                                        sa2 += w1[m] * w2[m];
                                    }
                                    v0 += QN * sa2;
                                } else {
                                    // the non-zero (m1, m2) pairs in the reference's loop order: the same terms,
                                    // added in the same order, as the dense double loop with its skip
                                    double sx = 0.0, sy = 0.0, sz = 0.0;
                                    const int npair = min(s_npair, kLmatPairs);
                                    for (int q = 0; q < npair; q++) {
                                        const double o1 = w1[lpm1[q]];
                                        if (fabs(o1) < kZeroThresh) continue;
                                        const double o2 = w2[lpm2[q]];
                                        sx += o1 * o2 * lpv[0][q];
                                        sy += o1 * o2 * lpv[1][q];
                                        sz += o1 * o2 * lpv[2][q];
                                    }
                                    v0 += QN * sx;
                                    v1 += QN * sy;
                                    v2 += QN * sz;
                                }
                            }
                        }
                        V[e * ncomp] = v0;
                        if (so) {
                            V[e * ncomp + 1] = v1;
                            V[e * ncomp + 2] = v2;
                        }
                    }
                    __syncthreads();
                    // elements whose factored sum is not certified fall back to the term-by-term loop
                    unsigned tbt = fact ? 0u : ~0u;
                    if (fact) {
                        // W[j][abc] = sum_def F_B V[abc][def] and Wa[j][abc] = sum_def |F_B| max_c |V[abc][def]|
                        double *W = V + sm.n_v;
                        const int nrow = r1 - r0;
                        double *Wa = W + nB * nrow * ncomp;
                        for (int e = tid; e < nB * nrow; e += NT) {
                            const int j = e / nrow, ar = e % nrow;
                            const int bx = cB[3 * j], by = cB[3 * j + 1], bz = cB[3 * j + 2];
                            double w0 = 0.0, w1 = 0.0, w2 = 0.0, wa = 0.0;
                            for (int dd = 0; dd <= bx; dd++)
                                for (int ee = 0; ee <= by; ee++)
                                    for (int ff = 0; ff <= bz; ff++) {
                                        const double fb = c_tab.binom[bx * kBinN + dd] * c_tab.binom[by * kBinN + ee] *
                                                          c_tab.binom[bz * kBinN + ff] * powB[0][bx - dd] * powB[1][by - ee] *
                                                          powB[2][bz - ff];
                                        if (fb == 0.0) continue;
                                        const double *vv = V + (ar * nabB + abc_index(lb, dd, ee, ff)) * ncomp;
                                        w0 += fb * vv[0];
                                        double vm = fabs(vv[0]);
                                        if (so) {
                                            w1 += fb * vv[1];
                                            w2 += fb * vv[2];
                                            vm = fmax(vm, fmax(fabs(vv[1]), fabs(vv[2])));
                                        }
                                        wa += fabs(fb) * vm;
                                    }
                            double *ww = W + (j * nrow + ar) * ncomp;
                            ww[0] = w0;
                            if (so) {
                                ww[1] = w1;
                                ww[2] = w2;
                            }
                            Wa[j * nrow + ar] = wa;
                        }
                        __syncthreads();
#pragma unroll
                        for (int q = 0; q < EPT; q++) {
                            const int el = tid + q * NT;
                            if (el >= nel) continue;
                            const int i = el / nB, j = el % nB;
                            const int ax = cA[3 * i], ay = cA[3 * i + 1], az = cA[3 * i + 2];
                            const int bx = cB[3 * j], by = cB[3 * j + 1], bz = cB[3 * j + 2];
                            double g0 = 0.0, g1 = 0.0, g2 = 0.0, ga = 0.0;
                            int nta = 0;
                            for (int aa = 0; aa <= ax; aa++)
                                for (int bb = 0; bb <= ay; bb++)
                                    for (int cc = 0; cc <= az; cc++) {
                                        const int abc = abc_index(la, aa, bb, cc);
                                        if (abc < r0 || abc >= r1) continue;
                                        const double fa = c_tab.binom[ax * kBinN + aa] * c_tab.binom[ay * kBinN + bb] *
                                                          c_tab.binom[az * kBinN + cc] * powA[0][ax - aa] * powA[1][ay - bb] *
                                                          powA[2][az - cc];
                                        if (fa == 0.0) continue;
                                        nta++;
                                        const double *ww = W + (j * nrow + abc - r0) * ncomp;
                                        g0 += fa * ww[0];
                                        if (so) {
                                            g1 += fa * ww[1];
                                            g2 += fa * ww[2];
                                        }
                                        ga += fabs(fa) * Wa[j * nrow + abc - r0];
                                    }
                            // Both this sum and libgrpp's term-by-term sum of the same terms are within
                            // (n + 12) u sum|terms| of the exact value, n = the number of terms and 12 u the
                            // rounding of a term's factors; the two differ by at most twice that. The
                            // factored result is kept when that worst-case bound, scaled by 16 pi^2, is below
                            // 1e-11 absolute or 1e-10 of the partial sum itself (a tenth of the 1e-10 / 1e-9
                            // comparator); otherwise, where the re-centring sum cancels, the element is summed
                            // term by term in libgrpp's order.
                            const double nterm = (double)nta * (double)((bx + 1) * (by + 1) * (bz + 1));
                            const double bound = 2.0 * (nterm + 12.0) * 1.1102230246251565e-16 * ga * (16 * kPi * kPi);
                            const double gmax = fmax(fabs(g0), fmax(fabs(g1), fabs(g2)));
                            if (bound <= fmax(1e-11, 1e-10 * gmax * (16 * kPi * kPi))) {
                                gam[0][q] += g0;
                                gam[1][q] += g1;
                                gam[2][q] += g2;
                            } else {
                                tbt |= 1u << q;
                            }
                        }
                    }
                    // Cartesian pairs: binomial re-centring sums over (a..f) in the reference's loop order
#pragma unroll
                    for (int q = 0; q < EPT; q++) {
                        const int el = tid + q * NT;
                        if (el >= nel || !((tbt >> q) & 1u)) continue;
                        const int i = el / nB, j = el % nB;
                        const int ax = cA[3 * i], ay = cA[3 * i + 1], az = cA[3 * i + 2];
                        const int bx = cB[3 * j], by = cB[3 * j + 1], bz = cB[3 * j + 2];
                        double g0 = gam[0][q], g1 = gam[1][q], g2 = gam[2][q];
                        for (int aa = 0; aa <= ax; aa++)
                            for (int bb = 0; bb <= ay; bb++)
                                for (int cc = 0; cc <= az; cc++) {
                                    const int abc = abc_index(la, aa, bb, cc);
                                    if (abc < r0 || abc >= r1) continue;
                                    const double cabc = c_tab.binom[ax * kBinN + aa] * c_tab.binom[ay * kBinN + bb] *
                                                        c_tab.binom[az * kBinN + cc];
                                    for (int dd = 0; dd <= bx; dd++)
                                        for (int ee = 0; ee <= by; ee++)
                                            for (int ff = 0; ff <= bz; ff++) {
                                                const double f = cabc * c_tab.binom[bx * kBinN + dd] * c_tab.binom[by * kBinN + ee] *
                                                                 c_tab.binom[bz * kBinN + ff] * powA[0][ax - aa] * powA[1][ay - bb] *
                                                                 powA[2][az - cc] * powB[0][bx - dd] * powB[1][by - ee] *
                                                                 powB[2][bz - ff];
                                                if (fabs(f) < thrF) continue;
                                                const int def = abc_index(lb, dd, ee, ff);
                                                const double *vv = V + ((abc - r0) * nabB + def) * ncomp;
                                                g0 += f * vv[0];
                                                if (so) {
                                                    g1 += f * vv[1];
                                                    g2 += f * vv[2];
                                                }
                                            }
                                }
                        gam[0][q] = g0;
                        gam[1][q] = g1;
                        gam[2][q] = g2;
                    }
                }
                const double pi16 = 16 * kPi * kPi;
                const double fso = a.raw_so ? 1.0 : 2.0 / (2 * L + 1);
#pragma unroll
                for (int q = 0; q < EPT; q++) {
                    if (!so) {
                        acc[0][q] += 1.0 * (gam[0][q] * pi16);
                    } else {
                        acc[1][q] += fso * (gam[0][q] * pi16);
                        acc[2][q] += fso * (gam[1][q] * pi16);
                        acc[3][q] += fso * (gam[2][q] * pi16);
                    }
                }
            }
        }

        // ---- outercore non-local terms (outercore_integrals.c:147-390)
        const int noc = a.grpp_n_oc[g];
        if (noc > 0 && a.task_proj_a[t] >= 0) {
            const int64_t pa = a.proj_off[a.task_proj_a[t]], pb = a.proj_off[a.task_proj_b[t]];
            const int ocoff = a.grpp_oc_off[g];
            const double *dl = a.oc_delta + a.grpp_delta_off[g];
#pragma unroll
            for (int q = 0; q < EPT; q++) {
                const int el = tid + q * NT;
                if (el >= nel) continue;
                const int i = el / nB, j = el % nB;
                double oa = 0.0, ox = 0.0, oy = 0.0, oz = 0.0;
                // part 1
                int64_t offA = pa, offB = pb;
                for (int k = 0; k < noc; k++) {
                    const int L = a.oc_L[ocoff + k], d = 2 * L + 1;
                    const double J = a.oc_J[ocoff + k] / 2.0;
                    const double *SA = a.S_sph + offA + i * d, *UA = a.U_sph + offA + i * d;
                    const double *SB = a.S_sph + offB + j * d, *UB = a.U_sph + offB + j * d;
                    const double farep = (J < L) ? (L / (2.0 * L + 1)) : ((L + 1) / (2.0 * L + 1));
                    const double fso = (J < L) ? (-2.0 / (2 * L + 1)) : (+2.0 / (2 * L + 1));
                    double s1 = 0.0, s2 = 0.0;
                    for (int m = 0; m < d; m++) s1 += SA[m] * UB[m];
                    for (int m = 0; m < d; m++) s2 += UA[m] * SB[m];
                    double buf = 0.0;
                    buf += s1;
                    buf += s2;
                    oa += farep * buf;
                    double *oso[3] = {&ox, &oy, &oz};
                    for (int comp = 0; comp < 3; comp++) {
                        // so_buf = U_a (L S_b) + (S_a L) U_b
                        double t1 = 0.0;
                        for (int m1 = 0; m1 < d; m1++) {
                            double tm = 0.0;
                            for (int m2 = 0; m2 < d; m2++) tm += lmat_val(L, comp, m1 - L, m2 - L) * SB[m2];
                            double tmp = 0.0;
                            tmp += tm;
                            t1 += UA[m1] * tmp;
                        }
                        double sob = 0.0;
                        sob += t1;
                        double t2 = 0.0;
                        for (int m = 0; m < d; m++) {
                            double tm = 0.0;
                            for (int k2 = 0; k2 < d; k2++) tm += SA[k2] * lmat_val(L, comp, k2 - L, m - L);
                            double tmp = 0.0;
                            tmp += tm;
                            t2 += tmp * UB[m];
                        }
                        sob += t2;
                        *oso[comp] += fso * sob;
                    }
                    offA += (int64_t)nA * d;
                    offB += (int64_t)nB * d;
                }
                // part 2
                int64_t offA1 = pa;
                for (int k1 = 0; k1 < noc; k1++) {
                    const int L1 = a.oc_L[ocoff + k1], d = 2 * L1 + 1;
                    int64_t offB2 = pb;
                    for (int k2 = 0; k2 < noc; k2++) {
                        const int L2 = a.oc_L[ocoff + k2];
                        const int d2 = 2 * L2 + 1;
                        if (L1 == L2 && a.oc_J[ocoff + k1] == a.oc_J[ocoff + k2]) {
                            const double delta = dl[k1 * noc + k2];
                            const double J = a.oc_J[ocoff + k1] / 2.0;
                            const int L = L1;
                            const double farep = (J < L) ? (L / (2.0 * L + 1)) : ((L + 1) / (2.0 * L + 1));
                            const double fso = (J < L) ? (-2.0 / (2 * L + 1)) : (+2.0 / (2 * L + 1));
                            const double *SA = a.S_sph + offA1 + i * d, *SB = a.S_sph + offB2 + j * d;
                            double s = 0.0;
                            for (int m = 0; m < d; m++) s += SA[m] * SB[m];
                            double buf = 0.0;
                            buf += s;
                            oa += (-1.0) * delta * farep * buf;
                            double *oso[3] = {&ox, &oy, &oz};
                            for (int comp = 0; comp < 3; comp++) {
                                double t1 = 0.0;
                                for (int m1 = 0; m1 < d; m1++) {
                                    double tm = 0.0;
                                    for (int m2 = 0; m2 < d; m2++) tm += lmat_val(L, comp, m1 - L, m2 - L) * SB[m2];
                                    double tmp = 0.0;
                                    tmp += tm;
                                    t1 += SA[m1] * tmp;
                                }
                                double sob = 0.0;
                                sob += t1;
                                *oso[comp] += (-1.0) * delta * fso * sob;
                            }
                        }
                        offB2 += (int64_t)nB * d2;
                    }
                    offA1 += (int64_t)nA * d;
                }
                acc[0][q] += 1.0 * oa;
                acc[1][q] += 1.0 * ox;
                acc[2][q] += 1.0 * oy;
                acc[3][q] += 1.0 * oz;
            }
        }
#pragma unroll
        for (int q = 0; q < EPT; q++) {
            const int e = tid + q * NT;
            if (e < nel) {
                a.arep[oo + e] = acc[0][q];
                a.so_x[oo + e] = acc[1][q];
                a.so_y[oo + e] = acc[2][q];
                a.so_z[oo + e] = acc[3][q];
            }
        }
    }
}
#endif  // GRPP_NO_ANGULAR_KERNELS

}  // namespace grpp
