// Host-side constant tables of the GRPP engine (see tables.cpp).
#pragma once

#include <cstdint>
#include <vector>

namespace grpp {

struct HostTables {
    std::vector<double> bessel, bessel_p, rfun, boys, dawson, rsh_coef, lmat, dfact, binom;
    std::vector<double> grid;   // [kGridRows][kGridPts], grpp_common.cuh
    std::vector<double> fermi;  // S_j(x) of the Fermi nuclear models, [kFermiNX][kFermiNK] (nucmodel.h)
    std::vector<int> rsh_off, rsh_comb_off, lmat_off;
    std::vector<int8_t> rsh_comb;
};

void build_host_tables(HostTables &t);

// the Fermi S_j table alone (built once, thread-safe), for host evaluation of the nuclear models
const double *fermi_table();

}  // namespace grpp
