// Host-side constant tables of the GRPP engine (see tables.cpp).
#pragma once

#include <cstdint>
#include <vector>

namespace grpp {

struct HostTables {
    std::vector<double> bessel, bessel_p, rfun, boys, dawson, rsh_coef, lmat, dfact, binom;
    std::vector<int> rsh_off, rsh_comb_off, lmat_off;
    std::vector<int8_t> rsh_comb;
};

void build_host_tables(HostTables &t);

}  // namespace grpp
