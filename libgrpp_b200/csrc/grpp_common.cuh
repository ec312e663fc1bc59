// Shared device-side declarations of the B200 GRPP engine.
//
// All arithmetic is FP64. Tables are generated on the host at libgrpp_init()
// (tables.cu) and live in global memory; their addresses and small constant
// tables sit in __constant__ memory.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace grpp {

// ---- limits ------------------------------------------------------------------
constexpr int kMaxL = 10;          // basis and projector angular momentum (libgrpp.h:16-21), +1 for gradients
constexpr int kBesL = 40;          // Bessel table orders 0..kBesL-1 (even: the pair layout)
constexpr int kBesNX = 1601;       // x = 0.00 .. 16.00 step 0.01 (specfunc_bessel_table.c:14-17)
constexpr int kRfunL = 40;         // asymptotic R_l coefficients (specfunc_scaled_mod_sph_bessel.c:163-190)
constexpr int kBoysNX = 301;       // x = 0.0 .. 30.0 step 0.1 (specfunc_boys.c:24)
constexpr int kBoysNN = 40;
constexpr int kRshL = 32;          // real spherical harmonic tables l = 0..kRshL
constexpr int kDfMax = 96;         // double factorial table n = -1..kDfMax
constexpr int kDawNY = 256;        // Dawson table y = 3.0 + k/32
constexpr double kDawY0 = 3.0;
constexpr double kDawH = 1.0 / 32.0;
constexpr int kBinN = 48;          // binomial table n = 0..kBinN-1
constexpr double kPi = 3.14159265358979323846;
constexpr double kZeroThresh = 1e-14;  // LIBGRPP_ZERO_THRESH

// Nested Log3 grid of the type 2 radial integrals: the 8191 points of levels 0..8 in walk
// order (level 0: points 1..31 of 31; level L >= 1: the odd points of 2^(L+5) - 1). The host
// tabulates per point, with libgrpp's expressions and C library (radial_type2_integral.c:357-365,
// 440-441; potential.c:70-81): r, the weight w at the point's own level, r^-1 = pow(r, -1),
// r^-2 = pow(r, -2) and r^N = pow(r, N) for N = 0..kGridMaxN.
constexpr int kGridPts = 8191;
constexpr int kGridMaxN = 24;
constexpr int kGridRowR = 0, kGridRowW = 1, kGridRowRinv = 2, kGridRowRinv2 = 3, kGridRowPow0 = 4;
constexpr int kGridRows = kGridRowPow0 + kGridMaxN + 1;

struct DeviceTables {
    const double *bessel;     // [kBesNX][kBesL][5]: value + 4 derivatives
    const double *bessel_p;   // the same values as [kBesNX][kBesL/2][5][2]: orders 2p, 2p+1 side by side
    const double *rfun;       // [kRfunL][kRfunL]
    const double *boys;       // [kBoysNX][kBoysNN]
    const double *dawson;     // [kDawNY]
    const double *rsh_coef;   // concatenated per l: [(2l+1)][ncomb(l)]
    const int *rsh_off;       // [kRshL+1] offsets into rsh_coef
    const int8_t *rsh_comb;   // concatenated per l: ncomb(l) x 3
    const int *rsh_comb_off;  // [kRshL+1] offsets (in combos)
    const double *lmat;       // concatenated per L: 3 x (2L+1)^2 (x, y, z)
    const int *lmat_off;      // [kMaxL+2]
    const double *dfact;      // dfact[n+1] = n!!, n = -1..kDfMax
    const double *binom;      // [kBinN][kBinN]
    const double *grid;       // [kGridRows][kGridPts] (null: the kernels compute r and w themselves)
};

__host__ __device__ inline int ncart(int L) { return (L + 1) * (L + 2) / 2; }

// ---- error reporting from kernels --------------------------------------------
// Kernels never trap: they record the first problem in a status word the host reads.
enum DeviceStatus : int {
    kDevOk = 0,
    kDevLimit = 1,      // an index exceeded a table limit; the affected value was skipped
    kDevTimeout = 2,    // a bounded loop gave up
};

}  // namespace grpp
