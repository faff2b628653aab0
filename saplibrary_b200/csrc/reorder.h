// Host-side pieces shared by the solver: the sparse reordering state and
// the synthetic banded-matrix generator.
#pragma once

#include <cstdint>
#include <vector>

namespace sapb {

// BandedMatrix(n, k, d) generator (sap/banded_matrix.h:59-95), row-major.
void generate_band(int n, int k, double d, int dist, uint64_t seed, double* out);

}  // namespace sapb
