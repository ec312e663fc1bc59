// Density-contracted GRPP gradient: per task (shells A, B, centre C), the GRPP
// blocks of the differentiated shells are contracted with the density block
// D[A, B] on the device, so per-coordinate gradient matrices are never formed.
//
// libgrpp differentiates a Cartesian Gaussian as (diff_gaussian.c:35-73,
// grpp_integrals_gradient.c:395-470)
//   d/dA_k |a> = |a + 1_k>' - a_k |a - 1_k>'
// where ' marks the shells of angular momentum L+1 (coefficients times
// 2 alpha N_L / N_{L+1}) and L-1 (times N_L / N_{L-1}). For every task the
// kernel forms, for the four matrices m (arep, so_x, so_y, so_z), the bra and
// ket sides and the three directions k,
//   G[side][k][m] = sum_ij D[A_i, B_j] (V^m(A+1 or B+1)[up] - n_k V^m(A-1 or B-1)[down]),
// skipping the L-1 term when n_k = 0 (its weight). The host then applies
// libgrpp's rule for which atoms receive which side and sign
// (grpp_integrals_gradient.c:280-393).
#pragma once

#include "grpp_common.cuh"

namespace grpp {

constexpr int kGradMaxCart = 66;  // ncart(kMaxL)

struct GradTask {
    int t_ad, t_au, t_bd, t_bu;  // sub-task indices (-1: no L-1 shell)
    int la, lb;
    int64_t d_row, d_col;        // basis offsets of A and B (rows / columns of D)
};

struct GradArgs {
    const GradTask *tasks;
    int n_tasks;
    const int *cart_tab;         // [L][i][k][3]: n_k, index of +1_k in L+1, index of -1_k in L-1 (or -1)
    const int64_t *sub_off;      // block offset of every sub-task
    const double *out[4];        // sub-task blocks of the four matrices
    const double *D;             // n_bf x n_bf, row-major
    int64_t n_bf;
    double *g;                   // [n_tasks][2][3][4]
};

__device__ __forceinline__ const int *cart_entry(const int *tab, int L, int i, int k)
{
    return tab + ((L * kGradMaxCart + i) * 3 + k) * 3;
}

// one warp per task; lanes over the Cartesian pairs (i, j)
__global__ void __launch_bounds__(128) grad_contract_kernel(GradArgs a)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int t = blockIdx.x * 4 + warp; t < a.n_tasks; t += gridDim.x * 4) {
        const GradTask T = a.tasks[t];
        const int nA = ncart(T.la), nB = ncart(T.lb);
        const int nBu = ncart(T.lb + 1), nBd = T.lb > 0 ? ncart(T.lb - 1) : 0;
        double acc[24];
#pragma unroll
        for (int q = 0; q < 24; q++) acc[q] = 0.0;
        for (int pr = lane; pr < nA * nB; pr += 32) {
            const int i = pr / nB, j = pr % nB;
            const double d = a.D[(T.d_row + i) * a.n_bf + T.d_col + j];
            if (d == 0.0) continue;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const int *eb = cart_entry(a.cart_tab, T.la, i, k);
                const int *ek = cart_entry(a.cart_tab, T.lb, j, k);
#pragma unroll
                for (int m = 0; m < 4; m++) {
                    double vb = a.out[m][a.sub_off[T.t_au] + (int64_t)eb[1] * nB + j];
                    if (eb[0] > 0 && T.t_ad >= 0) vb -= eb[0] * a.out[m][a.sub_off[T.t_ad] + (int64_t)eb[2] * nB + j];
                    double vk = a.out[m][a.sub_off[T.t_bu] + (int64_t)i * nBu + ek[1]];
                    if (ek[0] > 0 && T.t_bd >= 0) vk -= ek[0] * a.out[m][a.sub_off[T.t_bd] + (int64_t)i * nBd + ek[2]];
                    acc[k * 4 + m] += d * vb;
                    acc[12 + k * 4 + m] += d * vk;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 24; q++) {
            double v = acc[q];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) a.g[(int64_t)t * 24 + q] = v;
        }
    }
}

}  // namespace grpp
