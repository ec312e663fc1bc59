// Type 1 (radially local) GRPP integrals by McMurchie-Davidson, and
// two-centre overlaps by Obara-Saika, one warp per work item.
//
// Reference algorithm: libgrpp/type1_mcmurchie_davidson.c:107-622 and
// libgrpp/type1_integrals.c:43-78 (sum over potential terms k of c_k times
// the primitive-pair contraction), libgrpp/overlap.c:39-139.
//
// A work item is <bra| c r^(n-2) exp(-zeta r^2) (centred at C) |ket> summed
// over the terms of one potential, or the overlap <bra|ket>. Per primitive
// pair and term the warp builds
//   E[axis][i][j][t]  Hermite expansion coefficients, by wavefronts w = i+j
//                     (each E^{ij} depends on E^{i-1,j} or E^{i,j-1} only),
//   R^n_{tuv}         auxiliary integrals (Boys for n=1, G_n for n=0), by
//                     levels s = t+u+v (each level depends on s-1, s-2 only),
// in shared memory, then each lane accumulates its Cartesian pairs
//   sum_{tuv} E^x_t E^y_u E^z_v R^0_{tuv}.
// The contraction order (terms outer, primitive pairs inner, c_i c_j then
// c_k applied as in the reference's daxpy calls) is kept.
#pragma once

#include "grpp_common.cuh"
#include "specfunc.cuh"
#include "radial.cuh"  // RadialCounter slots shared with the type 1 kernel

namespace grpp {

struct MmdItem {
    int bra, ket;        // shell indices
    int ket_at_centre;   // 1: ket origin is the centre C (outercore shells)
    int centre;          // centre index (origin of the potential)
    int pot;             // potential index, or -1 for an overlap
    int out_kind;        // 0: arep output, 1: outercore U scratch, 2: outercore S scratch
    int64_t out_off;     // offset of the nbra x nket row-major block
    int sched;           // offset of the item's Cartesian pair schedule (MmdArgs::sched)
    int sched_rows;      // slot couples (2h, 2h+1) of the schedule in use
};

struct MmdArgs {
    const MmdItem *items;
    int n_items;
    const int *shell_L, *shell_nprim, *shell_prim_off, *shell_cart_off;
    const double *prim_coef, *prim_alpha, *shell_origin;
    const int8_t *cart;
    const int *pot_nprim, *pot_prim_off, *pot_powers;
    const double *pot_coef, *pot_alpha;
    const double *centre_origin;
    double *out[3];
    int smax;            // max la+lb over the items (sizes the shared workspace)
    int lmax;            // max l over the items
    int *status;
    unsigned long long *counters;  // kRadCntMmdTriples / kRadCntMmdFlops slots (may be null)
    // per class of (bra, ket) Cartesian tables, 32 x KPL slots: slot (q, lane) at q * 32 + lane
    // holds the pair index m * nket + n the lane owns in its q-th register, or kMmdNoPair. Slots
    // (2h, 2h+1) of a lane hold pairs with equal (ax+bx, ay+by, az+bz), or one pair and an empty
    // slot; the 32 lanes of a slot row hold pairs of equal or adjacent (ax+bx, ay+by, az+bz)
    const uint16_t *sched;
    // update programs of the Hermite coefficients, per (la, lb) at etab_off[la * (kMaxL + 1) + lb]:
    // one int per coefficient in wavefront order (see mmd_e_code); and of the R^n_tuv table, per
    // S at rtab_off[S]: one int2 per entry of levels s >= 1, at the entry's own index (see mmd_r_code)
    const int *etab, *etab_off;
    const int2 *rtab;
    const int *rtab_off;
    // dynamic schedule: warps pop positions from *queue (zeroed before the launch) and take
    // item order[position]; the host orders items by decreasing estimated work
    const int *order;
    int *queue;
};
constexpr uint16_t kMmdNoPair = 0xffff;

// Hermite coefficient E[ax][i][j][t] (row-major over (ax, i, j, t), extents 3, la+1, lb+1, S+1):
// bits 0-12 its index, 13-14 ax, 15-18 i, 19-22 j, 23-27 t, 28-30 the recurrence form
// (type1_mcmurchie_davidson.c:569-622):
//   0: K[ax] (i = j = 0)           1: (Q-A)[ax] E[ax][0][0][0] (i = 1, j = 0)
//   2: (Q-B)[ax] E[ax][0][0][0] (i = 0, j = 1)
//   3: (Q-B)[ax] E[ax][0][j-1][0] + E[ax][0][j-1][1] (i = 0, j >= 2)
//   4: (Q-A)[ax] E[ax][i-1][j][0] + E[ax][i-1][j][1] (other t = 0)
//   5: (i E[ax][i-1][j][t-1] + j E[ax][i][j-1][t-1]) / (2 q t) (t >= 1), each term as f i E
__host__ __device__ inline int mmd_e_code(int dst, int ax, int i, int j, int t)
{
    int ty;
    if (t > 0) ty = 5;
    else if (i == 0 && j == 0) ty = 0;
    else if (i == 1 && j == 0) ty = 1;
    else if (i == 0 && j == 1) ty = 2;
    else if (i == 0) ty = 3;
    else ty = 4;
    return dst | (ax << 13) | (i << 15) | (j << 19) | (t << 23) | (ty << 28);
}
constexpr int kMmdNoR0 = 4095;  // R^n_tuv entry with n > 0: not an R^0 value


// FP64 operations of one primitive triple, by phase (FMA = 2, exp/div/sqrt/pow = 1):
// setup (q, 3 mu, 3 Q, 9 exponentials, K) 40; a Hermite coefficient 5; an auxiliary
// function value 16 (Boys, 6th-order Taylor) or 100 per G_n series; an R^n_tuv entry 5;
// a term E_x E_y E_z R of the contraction 3, plus 3 per Cartesian pair.
__host__ __device__ inline unsigned long long mmd_e_count(int la, int lb)
{
    return 3ull * ((la + 1) * (lb + 1) + (lb + 1) * la * (la + 1) / 2 + (la + 1) * lb * (lb + 1) / 2);
}

// shared workspace per warp, in doubles
__host__ __device__ inline int mmd_e_size(int lmax) { return 3 * (lmax + 1) * (lmax + 1) * (2 * lmax + 1); }
__host__ __device__ inline int mmd_r_size(int smax)
{
    // sum over levels s of (s+1)(s+2)/2 entries x (smax-s+1) orders
    int tot = 0;
    for (int s = 0; s <= smax; s++) tot += (s + 1) * (s + 2) / 2 * (smax - s + 1);
    return tot;
}
constexpr int kMmdMaxPrims = 64;     // primitives per shell (the engine's limit)
constexpr double kPi15 = 5.568327996831708;  // pi^(3/2), correctly rounded

// R^0_tuv (t+u+v <= S) in rows (t, u) of consecutive v: tet(S) = (S+1)(S+2)(S+3)/6 values
__host__ __device__ inline int mmd_tet(int m) { return (m + 1) * (m + 2) * (m + 3) / 6; }
__host__ __device__ inline int mmd_ws_size(int lmax, int smax)
{
    return mmd_e_size(lmax) + mmd_r_size(smax) + mmd_tet(smax) + 2 * (smax + 2) + 16 + 2 * kMmdMaxPrims + 12 +
           (smax + 1) + 7 * 32;
}

// start of row (t, u) in the R^0 layout: rows ordered t-major, then u
__host__ __device__ __forceinline__ int r0_row(int S, int t, int u)
{
    return mmd_tet(S) - mmd_tet(S - t) + u * (S - t + 1) - u * (u - 1) / 2;
}

// sum_{t<=tx, u<=uy, v<=vz} E^x_t E^y_u E^z_v R^0_tuv for two pairs with equal (tx, uy, vz),
// side by side on shared R^0 loads; each sum in the reference's (t, u, v) order
__device__ __forceinline__ void mmd_contract2(const double *E, const double *R0, int S, int2 d0, int2 d1, double &s0,
                                              double &s1)
{
    const int tx = (d0.y >> 16) & 31, uy = (d0.y >> 21) & 31, vz = (d0.y >> 26) & 31;
    const int ox0 = d0.x & 0xffff, oy0 = (int)((unsigned)d0.x >> 16);
    const int ox1 = d1.x & 0xffff, oy1 = (int)((unsigned)d1.x >> 16);
    const double *ez0 = E + (d0.y & 0xffff), *ez1 = E + (d1.y & 0xffff);
    s0 = 0.0;
    s1 = 0.0;
    for (int t = 0; t <= tx; t++) {
        const double ex0 = E[ox0 + t], ex1 = E[ox1 + t];
        for (int u = 0; u <= uy; u++) {
            const double exy0 = ex0 * E[oy0 + u], exy1 = ex1 * E[oy1 + u];
            const double *r0 = R0 + r0_row(S, t, u);
#pragma unroll 4
            for (int v = 0; v <= vz; v++) {
                const double rv = r0[v];
                s0 += exy0 * ez0[v] * rv;
                s1 += exy1 * ez1[v] * rv;
            }
        }
    }
}

constexpr int kMmdMaxPairsPerLane = 32;  // up to 1024 Cartesian pairs per pass (KPL = 32 variant)

__device__ __forceinline__ int eidx(int lb1, int S1, int ax, int i, int j, int t, int la1)
{
    return ((ax * la1 + i) * lb1 + j) * S1 + t;
}

// level offsets of the R table: lvl_off[s] = sum_{s'<s} ne(s') (S-s'+1)
__device__ __forceinline__ int r_level_off(int S, int s)
{
    int o = 0;
    for (int q = 0; q < s; q++) o += (q + 1) * (q + 2) / 2 * (S - q + 1);
    return o;
}

// index of (u+v = k, v) within level s: tri(k) + v
__host__ __device__ __forceinline__ int r_in_level(int u, int v) { return (u + v) * (u + v + 1) / 2 + v; }

// KPL: Cartesian pairs held per lane per pass (8: up to 256 pairs, 32: up to 1024)
// COUNT: keep the operation counters (a separate instantiation, so the timed kernel carries none)
template <int KPL, bool COUNT>
__global__ void __launch_bounds__(128) mmd_kernel(MmdArgs a)
{
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int ws = mmd_ws_size(a.lmax, a.smax);
    double *E = smem + warp * ws;
    double *R = E + mmd_e_size(a.lmax);
    double *R0 = R + mmd_r_size(a.smax);
    double *aux = R0 + mmd_tet(a.smax);
    int *lvl = (int *)(aux + (a.smax + 2));
    double *normA = aux + 2 * (a.smax + 2) + 16, *normB = normA + kMmdMaxPrims;  // per item
    // per primitive triple: (Q-A)[3], (Q-B)[3], K[3], (Q-C)[3], then 1/(2 q t) for t = 1..S
    double *sQA = normB + kMmdMaxPrims, *sQB = sQA + 3, *sK = sQB + 3, *sQC = sK + 3, *finv = sQC + 3;
    // per chunk of 32 primitive pairs, lane l's pair: q, Q[3], K[3] at spre[v * 32 + l]
    double *spre = finv + (a.smax + 1);
    // lane-private descriptors of the Cartesian pairs of the current pass (after all warps'
    // workspaces): x = E row of axis x | E row of axis y << 16, y = E row of axis z |
    // (ax+bx) << 16 | (ay+by) << 21 | (az+bz) << 26 — each pair is decoded once per pass,
    // not once per primitive triple
    int2 *pdesc = reinterpret_cast<int2 *>(smem + wpb * ws) + warp * 32 * KPL;

    unsigned long long c_trip = 0, c_fl = 0;  // operation counters of this lane
    for (;;) {
        int k = 0;
        if (lane == 0) k = atomicAdd(a.queue, 1);
        k = __shfl_sync(0xffffffffu, k, 0);
        if (k >= a.n_items) break;
        const MmdItem item = a.items[a.order[k]];
        const int la = a.shell_L[item.bra], lb = a.shell_L[item.ket];
        const int nA = ncart(la), nB = ncart(lb), S = la + lb;
        const int la1 = la + 1, lb1 = lb + 1, S1 = S + 1;
        const double *Ao = a.shell_origin + 3 * item.bra;
        const double *Bo = item.ket_at_centre ? a.centre_origin + 3 * item.centre : a.shell_origin + 3 * item.ket;
        const double *Co = a.centre_origin + 3 * item.centre;
        const double A[3] = {Ao[0], Ao[1], Ao[2]}, B[3] = {Bo[0], Bo[1], Bo[2]}, C[3] = {Co[0], Co[1], Co[2]};
        const int8_t *ca = a.cart + 3 * a.shell_cart_off[item.bra];
        const int8_t *cb = a.cart + 3 * a.shell_cart_off[item.ket];
        const int npA = a.shell_nprim[item.bra], npB = a.shell_nprim[item.ket];
        const double *cA = a.prim_coef + a.shell_prim_off[item.bra], *xA = a.prim_alpha + a.shell_prim_off[item.bra];
        const double *cB = a.prim_coef + a.shell_prim_off[item.ket], *xB = a.prim_alpha + a.shell_prim_off[item.ket];
        const bool overlap = item.pot < 0;
        const int nterms = overlap ? 1 : a.pot_nprim[item.pot];
        double *out = a.out[item.out_kind] + item.out_off;

        __syncwarp();  // the previous item's readers of lvl and the norms are done
        if (lane == 0) {
            int o = 0;
            for (int s = 0; s <= S; s++) {
                lvl[s] = o;
                o += (s + 1) * (s + 2) / 2 * (S - s + 1);
            }
        }
        // primitive norms depend on (shell, primitive) only: once per item, one per lane
        for (int q = lane; q < npA; q += 32) normA[q] = gaussian_norm(la, xA[q]);
        for (int q = lane; q < npB; q += 32) normB[q] = gaussian_norm(lb, xB[q]);
        __syncwarp();

        const int npairs = nA * nB;
        {  // one pass over all pairs: npairs <= 32 x KPL (the host checks it)
            const int pass = 0;
            // operations of one primitive triple's contraction over this pass's Cartesian pairs (counters)
            const int pend = min(npairs, pass + 32 * KPL);
            unsigned long long contract_fl = 0;
            if (COUNT) {
                for (int pr = pass + lane; pr < pend; pr += 32) {
                    const int m = pr / nB, n = pr % nB;
                    contract_fl += 3ull * (ca[3 * m] + cb[3 * n] + 1) * (ca[3 * m + 1] + cb[3 * n + 1] + 1) *
                                       (ca[3 * m + 2] + cb[3 * n + 2] + 1) + 3ull;
                }
                for (int o = 16; o > 0; o >>= 1) contract_fl += __shfl_xor_sync(0xffffffffu, contract_fl, o);
            }
            const uint16_t *sch = a.sched + item.sched;
            const int nslots = 2 * item.sched_rows;
#pragma unroll
            for (int qq = 0; qq < KPL; qq++) {
                if (qq >= nslots) break;
                const int pr = sch[qq * 32 + lane];
                if (pr == kMmdNoPair) {
                    pdesc[qq * 32 + lane] = make_int2(0, -1);  // empty slot
                    continue;
                }
                const int m = pr / nB, n = pr % nB;
                const int ax = ca[3 * m], ay = ca[3 * m + 1], az = ca[3 * m + 2];
                const int bx = cb[3 * n], by = cb[3 * n + 1], bz = cb[3 * n + 2];
                pdesc[qq * 32 + lane] =
                    make_int2(eidx(lb1, S1, 0, ax, bx, 0, la1) | (eidx(lb1, S1, 1, ay, by, 0, la1) << 16),
                              eidx(lb1, S1, 2, az, bz, 0, la1) | ((ax + bx) << 16) | ((ay + by) << 21) | ((az + bz) << 26));
            }
            double res[KPL];
#pragma unroll
            for (int q = 0; q < KPL; q++) res[q] = 0.0;

            for (int k = 0; k < nterms; k++) {
                const double zeta = overlap ? 0.0 : a.pot_alpha[a.pot_prim_off[item.pot] + k];
                const int npow = overlap ? 3 : a.pot_powers[a.pot_prim_off[item.pot] + k];
                double accp[KPL];
#pragma unroll
                for (int q = 0; q < KPL; q++) accp[q] = 0.0;

                // primitive pairs (i, j) in the reference's order, 32 at a time: first each lane
                // evaluates the scalars of one pair (q, Q, the Gaussian factors K per axis,
                // K[d] = e(d,ab) e(d,ac) e(d,bc)); pairs with a zero coefficient (|c| < 1e-14)
                // or a K[d] that underflowed to exactly 0 add exact zeros and are dropped
                const int np2 = npA * npB;
                for (int base = 0; base < np2; base += 32) {
                    const int rr = base + lane;
                    bool live = false;
                    __syncwarp();  // the previous chunk's readers of spre are done
                    if (rr < np2) {
                        const int i = rr / npB, j = rr - i * npB;
                        if (overlap) {
                            live = true;
                        } else if (!(fabs(cA[i]) < kZeroThresh) && !(fabs(cB[j]) < kZeroThresh)) {
                            const double al = xA[i], be = xB[j];
                            const double q = al + be + zeta;
                            const double muab = (al * be) / q, muac = (al * zeta) / q, mubc = (be * zeta) / q;
                            spre[lane] = q;
#pragma unroll
                            for (int d = 0; d < 3; d++) {
                                // each product rounded, as the reference's (a A + b B + c C) / q
                                // (type1_mcmurchie_davidson.c:198); no contraction into an FMA
                                spre[(1 + d) * 32 + lane] =
                                    __dadd_rn(__dadd_rn(__dmul_rn(al, A[d]), __dmul_rn(be, B[d])), __dmul_rn(zeta, C[d])) / q;
                                const double dab = A[d] - B[d], dac = A[d] - C[d], dbc = B[d] - C[d];
                                const double Kd = exp(-muab * dab * dab) * exp(-muac * dac * dac) * exp(-mubc * dbc * dbc);
                                spre[(4 + d) * 32 + lane] = Kd;
                                live = d == 0 ? Kd != 0.0 : (live && Kd != 0.0);
                            }
                        }
                    }
                    unsigned live_mask = __ballot_sync(0xffffffffu, live);
                    __syncwarp();
                    while (live_mask) {
                        const int bl = __ffs(live_mask) - 1;
                        live_mask &= live_mask - 1;
                        const int i = (base + bl) / npB, j = (base + bl) - i * npB;
                        const double ci = cA[i], cj = cB[j];
                        const double al = xA[i], be = xB[j];
                        const double NA = normA[i], NB = normB[j];
                        double pref;
                        if (!overlap) {
                            // ---- Hermite E by wavefronts (type1_mcmurchie_davidson.c:569-622)
                            const double q = spre[bl];
                            double Q[3], K[3];
#pragma unroll
                            for (int d = 0; d < 3; d++) {
                                Q[d] = spre[(1 + d) * 32 + bl];
                                K[d] = spre[(4 + d) * 32 + bl];
                            }
                            if (COUNT && lane == 0) {
                                c_trip++;
                                c_fl += 40 + 5 * mmd_e_count(la, lb);
                                if (npow != 2)
                                    c_fl += (npow == 1 ? 16ull * (S + 1) : 100ull) + 2ull * (S + 1) +
                                            5ull * (mmd_r_size(S) - (S + 1)) + contract_fl;
                                else
                                    c_fl += 4ull * (pend - pass);
                            }
                            // per-triple scalars shared by the coefficient updates (the same
                            // expressions the updates would evaluate)
                            if (lane < 3) {
                                const double Qd = lane == 0 ? Q[0] : (lane == 1 ? Q[1] : Q[2]);
                                const double Ad = lane == 0 ? A[0] : (lane == 1 ? A[1] : A[2]);
                                const double Bd = lane == 0 ? B[0] : (lane == 1 ? B[1] : B[2]);
                                const double Cd = lane == 0 ? C[0] : (lane == 1 ? C[1] : C[2]);
                                sQA[lane] = Qd - Ad;
                                sQB[lane] = Qd - Bd;
                                sQC[lane] = Qd - Cd;
                                sK[lane] = lane == 0 ? K[0] : (lane == 1 ? K[1] : K[2]);
                            }
                            if (lane >= 1 && lane <= S) finv[lane] = 1.0 / (2.0 * q * lane);
                            __syncwarp();
                            const int *ecode = a.etab + __ldg(a.etab_off + la * (kMaxL + 1) + lb);
                            const int sj = S1, si = lb1 * S1;  // index steps of j and i
                            for (int w = 0, wo = 0; w <= S; w++) {
                                // entries (axis, i, j=w-i, t<=w)
                                const int ilo = max(0, w - lb), ihi = min(la, w);
                                const int tot = 3 * (ihi - ilo + 1) * (w + 1);
                                for (int e = lane; e < tot; e += 32) {
                                    const int c = __ldg(ecode + wo + e);
                                    const int dst = c & 8191, ax = (c >> 13) & 3, ty = c >> 28;
                                    const int e000 = ax * la1 * lb1 * S1;
                                    double v;
                                    if (ty == 0) v = sK[ax];
                                    else if (ty == 1) v = sQA[ax] * E[e000];
                                    else if (ty == 2) v = sQB[ax] * E[e000];
                                    else if (ty == 3) v = sQB[ax] * E[dst - sj] + E[dst - sj + 1];
                                    else if (ty == 4) v = sQA[ax] * E[dst - si] + E[dst - si + 1];
                                    else {
                                        const int ii = (c >> 15) & 15, jj = (c >> 19) & 15, t = (c >> 23) & 31;
                                        const double f = finv[t];
                                        v = 0.0;
                                        if (ii > 0) v += f * ii * E[dst - si - 1];
                                        if (jj > 0) v += f * jj * E[dst - sj - 1];
                                    }
                                    E[dst] = v;
                                }
                                wo += tot;
                                __syncwarp();
                            }
                            const double p15 = npow == 2 ? pow(kPi / q, 1.5) : 0.0;  // once per primitive triple
                            if (npow == 2) {
                                pref = 0.0;
                            } else {
                                // ---- auxiliary functions and R by levels (type1_mcmurchie_davidson.c:457-564)
                                const double dx = Q[0] - C[0], dy = Q[1] - C[1], dz = Q[2] - C[2];
                                const double x = q * (dx * dx + dy * dy + dz * dz);
                                if (npow == 1) {
                                    if (lane <= S) aux[lane] = boys(lane, x);
                                } else {
                                    gfun_values_warp(x, S, aux, lane);
                                }
                                __syncwarp();
                                const bool isg = npow == 0;
                                const double q2 = isg ? 2.0 * q : -2.0 * q;
                                if (lane <= S) R[lane] = pow(q2, lane) * aux[lane];  // level 0: n = 0..S
                                if (lane == 0) R0[0] = R[0];
                                __syncwarp();
                                const int2 *rcode = a.rtab + __ldg(a.rtab_off + S);
                                for (int s = 1; s <= S; s++) {
                                    const int ne = (s + 1) * (s + 2) / 2, nn = S - s + 1, tot = ne * nn;
                                    const int o = lvl[s], ne1 = s * (s + 1) / 2, ne2 = (s - 1) * s / 2;
                                    for (int e = lane; e < tot; e += 32) {
                                        // entry (t, u, v) of order n from its step down along one axis
                                        // (the first of z, y, x with t+u, t, ... as in the reference)
                                        const int2 c = __ldg(rcode + o + e);
                                        const int src1 = c.x & 0xffff, src2 = (int)((unsigned)c.x >> 16);
                                        const int kq = c.y & 31, ax = (c.y >> 5) & 3, r0d = (c.y >> 7) & 4095;
                                        const double X = sQC[ax];
                                        const double r1n1 = R[src1 + ne1], r1n = R[src1];
                                        double val = 0.0;
                                        if (kq > 1) {
                                            const double r2n1 = R[src2 + ne2], r2n = R[src2];
                                            if (isg) val += (kq - 1) * (r2n1 - 2.0 * q * r2n);
                                            else val += (kq - 1) * r2n1;
                                        }
                                        if (isg) val += X * (r1n1 - 2.0 * q * r1n);
                                        else val += X * r1n1;
                                        R[o + e] = val;
                                        if (r0d != kMmdNoR0) R0[r0d] = val;
                                    }
                                    __syncwarp();
                                }
                                pref = npow == 1 ? NA * NB * 2.0 * kPi / q : NA * NB * 2.0 * kPi15 / sqrt(q);
                            }
                            // ---- Cartesian pairs of this lane, by slot couples (2h, 2h+1) of equal
                            // (tx, uy, vz); a lone pair runs with itself as partner, so every lane of a
                            // row takes the same path
#pragma unroll
                            for (int h = 0; h < KPL; h += 2) {
                                if (h >= nslots) break;
                                const int2 d0 = pdesc[h * 32 + lane], d1 = pdesc[(h + 1) * 32 + lane];
                                if (d0.y < 0) continue;
                                if (npow == 2) {
                                    accp[h] += (ci * cj) * (NA * NB * E[d0.x & 0xffff] * E[(int)((unsigned)d0.x >> 16)] *
                                                            E[d0.y & 0xffff] * p15);
                                    if (d1.y >= 0)
                                        accp[h + 1] += (ci * cj) * (NA * NB * E[d1.x & 0xffff] *
                                                                    E[(int)((unsigned)d1.x >> 16)] * E[d1.y & 0xffff] * p15);
                                    continue;
                                }
                                const bool same = (d1.y >> 16) == (d0.y >> 16);  // false for an empty d1
                                double s0, s1;
                                mmd_contract2(E, R0, S, d0, same ? d1 : d0, s0, s1);
                                accp[h] += (ci * cj) * (s0 * pref);
                                if (same) accp[h + 1] += (ci * cj) * (s1 * pref);
                                else if (d1.y >= 0) {  // unequal couple (not produced by the schedule builder)
                                    mmd_contract2(E, R0, S, d1, d1, s0, s1);
                                    accp[h + 1] += (ci * cj) * (s0 * pref);
                                }
                            }
                        } else {
                            // ---- overlap: 1D Obara-Saika tables per axis (overlap.c:92-120)
                            const double p = al + be, mu = al * be / p, pf = 1.0 / (2.0 * p);
                            if (lane < 3) {
                                const int ax = lane;
                                const double P = (al * A[ax] + be * B[ax]) / p, xab = A[ax] - B[ax];
                                const double xpa = P - A[ax], xpb = P - B[ax];
                                for (int ii = 0; ii <= la; ii++)
                                    for (int jj = 0; jj <= lb; jj++) {
                                        double s = 0.0;
                                        if (ii + jj == 0) {
                                            E[eidx(lb1, S1, ax, 0, 0, 0, la1)] = sqrt(kPi / p) * exp(-mu * xab * xab);
                                            continue;
                                        }
                                        if (ii == 0) {
                                            s += xpb * E[eidx(lb1, S1, ax, ii, jj - 1, 0, la1)];
                                            if (jj - 1 > 0) s += (jj - 1) * pf * E[eidx(lb1, S1, ax, ii, jj - 2, 0, la1)];
                                        } else {
                                            s += xpa * E[eidx(lb1, S1, ax, ii - 1, jj, 0, la1)];
                                            if (ii - 1 > 0) s += (ii - 1) * pf * E[eidx(lb1, S1, ax, ii - 2, jj, 0, la1)];
                                            if (jj > 0) s += jj * pf * E[eidx(lb1, S1, ax, ii - 1, jj - 1, 0, la1)];
                                        }
                                        E[eidx(lb1, S1, ax, ii, jj, 0, la1)] = s;
                                    }
                            }
                            __syncwarp();
                            if (COUNT && lane == 0) {
                                c_trip++;
                                c_fl += 12ull * (la + 1) * (lb + 1) + 10 + 4ull * (pend - pass);  // Obara-Saika + pairs
                            }
#pragma unroll
                            for (int qq = 0; qq < KPL; qq++) {
                                if (qq >= nslots) break;
                                const int2 dsc = pdesc[qq * 32 + lane];
                                if (dsc.y < 0) continue;
                                const double buf = NA * NB * E[dsc.x & 0xffff] * E[(int)((unsigned)dsc.x >> 16)] *
                                                   E[dsc.y & 0xffff];
                                accp[qq] += (ci * cj) * buf;
                            }
                        }
                        __syncwarp();
                    }
                }
                const double ck = overlap ? 1.0 : a.pot_coef[a.pot_prim_off[item.pot] + k];
#pragma unroll
                for (int qq = 0; qq < KPL; qq++) res[qq] += ck * accp[qq];
            }
#pragma unroll
            for (int qq = 0; qq < KPL; qq++) {
                if (qq >= nslots) break;
                const int pr = sch[qq * 32 + lane];
                if (pr != kMmdNoPair) out[pr] = res[qq];
            }
        }
        __syncwarp();
    }
    if (COUNT && a.counters) {
        for (int o = 16; o > 0; o >>= 1) {
            c_trip += __shfl_down_sync(0xffffffffu, c_trip, o);
            c_fl += __shfl_down_sync(0xffffffffu, c_fl, o);
        }
        if (lane == 0) {
            atomicAdd(a.counters + kRadCntMmdTriples, c_trip);
            atomicAdd(a.counters + kRadCntMmdFlops, c_fl);
        }
    }
}

}  // namespace grpp
